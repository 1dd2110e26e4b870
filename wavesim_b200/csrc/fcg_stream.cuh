// fcg_stream.cuh — the learned path's flexible-CG passes with streaming sweeps.
//
// The passes of lpc.cuh (pre, post, dir; the update pass is pointwise and stays there) compute
// one matrix product each of a vector that is formed, cell by cell, from the inputs it is made of:
//   pre   v = z1 = w r / D          out: z1, and the network's input (r - A z1) / D
//   post  v = z2 = z1 + m y         out: z = z2 + w (r - A z2) / D, partial <z, q>
//   dir   v = p = z + beta p_old    out: p, q = A p, partials <p, q>, <r, p>
// Here a warp forms v on strips of 28 columns and marches down them (ps_strip, pcg_stream.cuh)
// instead of staging tiles in shared memory between block barriers. The arithmetic per cell is
// the tiled passes'; the dot products' partials are summed per block over a fixed partition of the
// strips, so runs are reproducible. For the network on the solver's own grid (stride 1); a coarser
// network grid keeps the per-pixel kernels of lpc.cuh.
#pragma once

#include "lpc.cuh"
#include "pcg_stream.cuh"

namespace wcb {

#ifndef WCB_FS_MINB
#define WCB_FS_MINB 3
#endif
constexpr int FS_NT = 256, FS_WARPS = FS_NT / 32, FS_MINB = WCB_FS_MINB;
// Ring fields per row (the post pass's: z1, y as pairs and r, D, q of the own cell two rows up;
// c, heff, y as two planes).
constexpr int FS_NF2 = 5, FS_NF1 = 4;
constexpr int FS_SMEM = FS_WARPS * ps_ring_bytes<FS_NF2, FS_NF1>();  // dynamic shared memory per block

struct FsRaw {
    float2 a, b;   // the pass's inputs at the cell
    float cc, he, sy;
};
struct FsRow {
    float2 v;
    float cc, he;
};
// What an own cell's output reads besides the product: r, D and q, as the pass needs them.
struct FsOwn {
    float2 r, d, q;
};

__device__ __forceinline__ FsRow fs_row(const FsRaw& r, float2 v, float sx) {
    FsRow o;
    o.v = make_float2(v.x * sx, v.y * r.sy);
    o.cc = r.cc;
    o.he = r.he;
    return o;
}

// The warp's strips of one pass: strips gw, gw + nw, ... with rows per strip `rows`.
template <class Fetch, class Make, class Out, class FetchOwn>
__device__ __forceinline__ void fs_sweep(const DevGrid& g, int rows, Fetch fetch, Make make, Out out,
                                         FetchOwn fetch_own) {
    const int nstrips = ps_strips(g.nx, g.ny, rows);
    const int strips_x = (g.nx + PS_OUT - 1) / PS_OUT;
    const int gw = blockIdx.x * FS_WARPS + (threadIdx.x >> 5), nw = gridDim.x * FS_WARPS;
    for (int st = gw; st < nstrips; st += nw) {
        const int i_lane = (st % strips_x) * PS_OUT - PS_HALO + (threadIdx.x & 31);
        const float sx = ((unsigned)i_lane < (unsigned)g.nx) ? 1.f : -1.f;
        ps_strip<FsRaw, FsRow, FS_NF2, FS_NF1>(
            g, st, rows, fetch, [&](const FsRaw& r) { return make(r, sx); }, out, fetch_own);
    }
}

__device__ __forceinline__ void fs_partials(double s0, double s1, double* part) {
    __shared__ double red[100];
    double s2 = 0.0;
    block_sum3<FS_NT>(s0, s1, s2, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0;
        part[3 * blockIdx.x + 1] = s1;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// pre: z1 = w r / D and the network's input (r - A z1) / D (NHWC BF16 pairs in xh, else 2 planes in x)
__global__ void __launch_bounds__(FS_NT, FS_MINB) fcg_pre_stream_kernel(
    DevGrid g, int rows, const float2* __restrict__ r, const float2* __restrict__ d, const float* __restrict__ cc,
    const float* __restrict__ heff, float2* __restrict__ z1, float omega, float* __restrict__ x,
    unsigned* __restrict__ xh, int Hp, int Wp, const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    const size_t plane = (size_t)Hp * Wp;
    fs_sweep(
        g, rows,
        [&](const auto& ld, int k, float sy, int, bool, int, int) {
            FsRaw o;
            o.a = ld.ld2(0, r + k, true);
            o.b = ld.ld2(1, d + k, true);
            o.cc = ld.ld1(0, cc + k, true);
            o.he = ld.ld1(1, heff + k, true);
            o.sy = sy;
            return o;
        },
        [&](const FsRaw& w, float sx) {
            return fs_row(w, make_float2(omega * w.a.x * w.b.x, omega * w.a.y * w.b.y), sx);
        },
        [&](int k, int i, int j, const FsRow& row, float2 tv, float, float, float, float, const FsOwn& ow) {
            const float2 rr = ow.r, dd = ow.d;
            z1[k] = row.v;  // own cells: no sign flip
            const float vx = (rr.x - tv.x) * dd.x, vy = (rr.y - tv.y) * dd.y;
            const size_t q = (size_t)j * Wp + i;
            if (xh) {
                xh[q] = bf16_pack(vx, vy);
            } else {
                x[q] = vx;
                x[plane + q] = vy;
            }
        },
        [&](const auto& ld, int k, bool en) {
            FsOwn o;
            o.r = ld.ld2(2, r + k, en);
            o.d = ld.ld2(3, d + k, en);
            return o;
        });
}

// post: z = z2 + w (r - A z2) / D with z2 = z1 + m y (y the network's output); partial <z, q>
__global__ void __launch_bounds__(FS_NT, FS_MINB) fcg_post_stream_kernel(
    DevGrid g, int rows, const float2* __restrict__ z1, const float* __restrict__ y, int nhwc,
    const float2* __restrict__ r, const float2* __restrict__ d, const float* __restrict__ cc,
    const float* __restrict__ heff, float2* __restrict__ z, const float2* __restrict__ qv, float omega, int Hp,
    int Wp, double* __restrict__ part, const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    const size_t plane = (size_t)Hp * Wp;
    double s0 = 0.0;
    fs_sweep(
        g, rows,
        [&](const auto& ld, int k, float sy, int, bool, int mi, int mj) {
            FsRaw o;
            const int q = mj * Wp + mi;
            o.a = ld.ld2(0, z1 + k, true);
            const float2 yp = ld.ld2(1, reinterpret_cast<const float2*>(y) + q, nhwc);
            const float y0 = ld.ld1(2, y + q, !nhwc), y1 = ld.ld1(3, y + plane + q, !nhwc);
            o.b = nhwc ? yp : make_float2(y0, y1);
            o.cc = ld.ld1(0, cc + k, true);
            o.he = ld.ld1(1, heff + k, true);
            o.sy = sy;
            return o;
        },
        [&](const FsRaw& w, float sx) {
            const float mk = w.he >= H_DISP_MIN ? 1.f : 0.f;
            return fs_row(w, make_float2(w.a.x + mk * w.b.x, w.a.y + mk * w.b.y), sx);
        },
        [&](int k, int, int, const FsRow& row, float2 tv, float, float, float, float, const FsOwn& ow) {
            const float2 a2 = row.v, rr = ow.r, dd = ow.d;
            const float2 zz = make_float2(a2.x + omega * (rr.x - tv.x) * dd.x, a2.y + omega * (rr.y - tv.y) * dd.y);
            z[k] = zz;
            const float2 qq = ow.q;
            s0 += (double)zz.x * qq.x + (double)zz.y * qq.y;
        },
        [&](const auto& ld, int k, bool en) {
            FsOwn o;
            o.r = ld.ld2(2, r + k, en);
            o.d = ld.ld2(3, d + k, en);
            o.q = ld.ld2(4, qv + k, en);
            return o;
        });
    fs_partials(s0, 0.0, part);
}

// dir: p = z + beta p_old (first: p = z), q = A p; partials <p, q>, <r, p>
__global__ void __launch_bounds__(FS_NT, FS_MINB) fcg_dir_stream_kernel(
    DevGrid g, int rows, const float2* __restrict__ zv, const float2* __restrict__ p_old, float2* __restrict__ p_new,
    const float* __restrict__ cc, const float* __restrict__ heff, float2* __restrict__ qv,
    const float2* __restrict__ r, double* __restrict__ part, const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    const bool first = sc->iterations == 0;
    const float beta = first ? 0.f : (float)sc->beta;
    double s0 = 0.0, s1 = 0.0;
    fs_sweep(
        g, rows,
        [&](const auto& ld, int k, float sy, int, bool, int, int) {
            FsRaw o;
            o.a = ld.ld2(0, zv + k, true);
            o.b = ld.ld2(1, p_old + k, !first);
            o.cc = ld.ld1(0, cc + k, true);
            o.he = ld.ld1(1, heff + k, true);
            o.sy = sy;
            return o;
        },
        [&](const FsRaw& w, float sx) {
            return fs_row(w, make_float2(w.a.x + beta * w.b.x, w.a.y + beta * w.b.y), sx);
        },
        [&](int k, int, int, const FsRow& row, float2 qq, float, float, float, float, const FsOwn& ow) {
            const float2 pp = row.v, rr = ow.r;
            p_new[k] = pp;
            qv[k] = qq;
            s0 += (double)pp.x * qq.x + (double)pp.y * qq.y;
            s1 += (double)rr.x * pp.x + (double)rr.y * pp.y;
        },
        [&](const auto& ld, int k, bool en) {
            FsOwn o;
            o.r = ld.ld2(2, r + k, en);
            return o;
        });
    fs_partials(s0, s1, part);
}

}  // namespace wcb
