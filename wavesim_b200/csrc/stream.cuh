// stream.cuh — the shallow-water RK stage (first and second order) as a streaming kernel.
//
// Each warp owns a strip of SW_OUT = 32 SW_CPL - 4 interior columns and marches down SW_ROWS rows
// of it. Its 32 lanes hold the strip's columns plus two halo columns on each side (SW_CPL adjacent
// columns per lane), so the x-neighbours a reconstruction needs come from the lane itself or from
// the lanes beside it by warp shuffles. Down the march, a three-row window of (eta, h, u, v, b),
// the high-side y reconstruction of the current row and the y-face flux just above it stay in
// registers; the rows below are copied ahead by cp.async into the warp's ring in shared memory,
// each lane its own columns. Per cell and row the kernel reconstructs once per axis
// (solver.rs:140-183), computes one x face and one y face (solver.rs:185-226) and updates the cell
// (solver.rs:481-616): no tile staging, no block barriers, every face once. The
// arithmetic is the tiled stage kernel's (stage.cuh), operation for operation: the same
// reconstruction, the remainder-form HLL, the well-balanced momentum update and the FP64 mass
// telescoping, so both kernels give the same bits.
//
// Ghost cells are synthesised on load by the boundary rule (map_cell): mirrored with the normal
// momentum's sign flipped at walls, wrapped when periodic in y. The CFL rate of a finishing stage
// is folded per block into the device clock, as the tiled kernel does.
#pragma once

#include "common.cuh"
#include "stage.cuh"

namespace wcb {

// Launch shape. Rows are fetched SW_DEPTH rows before they enter the window, by cp.async into a
// per-warp ring in shared memory (no registers held while in flight); SW_DEPTH 0 keeps SW_AHEAD
// rows in registers instead. On 4096 x 4096 (ms per stage): the ring with 3 rows in flight, one
// column per lane, 128 threads, 6 blocks per SM and 32 rows per strip 0.335 (4 or 6 rows the same;
// 7 or 8 blocks per SM 0.337-0.345); registers with 3 rows ahead 0.386, the best of seven register
// shapes (one or two columns per lane, 128 or 256 threads, 2-6 blocks per SM, 16-64 rows per
// strip, 2-5 rows in flight: 0.396-0.448 before the ring). The macros let a tuning build try others.
#ifndef WCB_SW_CPL
#define WCB_SW_CPL 1
#endif
#ifndef WCB_SW_NT
#define WCB_SW_NT 128
#endif
#ifndef WCB_SW_MINB
#define WCB_SW_MINB 6
#endif
#ifndef WCB_SW_ROWS
#define WCB_SW_ROWS 32
#endif
#ifndef WCB_SW_AHEAD
#define WCB_SW_AHEAD 3
#endif
#ifndef WCB_SW_DEPTH
#define WCB_SW_DEPTH 3
#endif
constexpr int SW_HALO = 2;
constexpr int SW_CPL = WCB_SW_CPL;      // columns per lane
constexpr int SW_NT = WCB_SW_NT, SW_WARPS = SW_NT / 32, SW_MINB = WCB_SW_MINB;
constexpr int SW_ROWS = WCB_SW_ROWS;    // rows per strip
constexpr int SW_AHEAD = WCB_SW_AHEAD;  // register mode: rows in flight beyond the window
constexpr int SW_DEPTH = WCB_SW_DEPTH;  // ring mode (> 0): rows in flight, by cp.async into shared memory
constexpr int SW_SLOTS = SW_DEPTH + 1;  // ring slots: a slot is refilled one row after it is read
constexpr int sw_out(int cpl) { return 32 * cpl - 2 * SW_HALO; }
constexpr int SW_OUT = sw_out(SW_CPL);

// A ring slot holds one row of the lane's columns: the state and bed of row R and, for a finishing
// second stage, the own cells' state at the start of the step of row R - 2 (the row that is
// updated when row R enters the window). Laid out [field][column][lane]: conflict-free accesses.
template <int CPL>
__host__ __device__ constexpr int sw_slot_bytes() { return CPL * 32 * (16 + 16 + 4); }
template <int CPL>
__host__ __device__ constexpr int sw_smem() { return SW_DEPTH > 0 ? SW_WARPS * SW_SLOTS * sw_slot_bytes<CPL>() : 0; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

// One loaded cell: the state as stored (h_hi, h_lo, hu, hv with the ghost sign flips applied) and
// the bed.
struct SwRaw {
    float4 q;
    float b;
};

// What the reconstructions read of a cell.
struct SwCell {
    float eta, h, u, v, b;
};

__device__ __forceinline__ SwRaw sw_load(const StageArgs& a, int k, float sx, float sy) {
    SwRaw r;
    r.q = __ldg(a.qin + k);
    r.q.z *= sx;
    r.q.w *= sy;
    r.b = __ldg(a.bed + k);
    return r;
}

__device__ __forceinline__ SwCell sw_cell(const SwRaw& r) {
    SwCell c;
    c.h = r.q.x;
    c.b = r.b;
    c.eta = c.h + c.b;
    c.u = velocity(c.h, r.q.z);
    c.v = velocity(c.h, r.q.w);
    return c;
}

// solver.rs:140-183 for one cell from its two neighbours along the axis (n: the normal velocity,
// t: the tangential one), as reconstruct() in stage.cuh computes it for first and second order.
template <int ORDER>
__device__ __forceinline__ void sw_recon(float em, float ec, float ep, float nm, float nc, float np,
                                         float tm, float tc, float tp, float hm, float hc, float hp,
                                         float bm, float bc, float bp, Side& lo, Side& hi, float& P) {
    Side first;
    first.eta = ec;
    first.un = nc;
    first.ut = tc;
    first.z = bc;
    first.h = hc;
    if (ORDER == 0 || hm < H_SECOND || hc < H_SECOND || hp < H_SECOND) {
        lo = first;
        hi = first;
        P = 0.f;
        return;
    }
    float elo, ehi, ulo, uhi, tlo, thi;
    face_values(em, em, ec, ep, ep, 0.f, elo, ehi);
    face_values(nm, nm, nc, np, np, 0.f, ulo, uhi);
    face_values(tm, tm, tc, tp, tp, 0.f, tlo, thi);
    const float sz = 0.25f * (bp - bm);
    const float zlo = bc - sz, zhi = bc + sz;
    const float hlo = elo - zlo, hhi = ehi - zhi;
    if (hlo < H_FACE_MIN || hhi < H_FACE_MIN) {
        lo = first;
        hi = first;
        P = 0.f;
        return;
    }
    lo.eta = elo; lo.un = ulo; lo.ut = tlo; lo.z = zlo; lo.h = hlo;
    hi.eta = ehi; hi.un = uhi; hi.ut = thi; hi.z = zhi; hi.h = hhi;
    P = 0.5f * G * (hlo + hhi) * (ehi - elo);
}

// The y reconstruction of the middle row of three (y-normal velocity v, tangential u).
template <int ORDER>
__device__ __forceinline__ void sw_recon_y(const SwCell& m, const SwCell& c, const SwCell& p, Side& lo,
                                           Side& hi, float& P) {
    sw_recon<ORDER>(m.eta, c.eta, p.eta, m.v, c.v, p.v, m.u, c.u, p.u, m.h, c.h, p.h, m.b, c.b, p.b, lo, hi, P);
}

struct SwFlux {
    float F0, RL, RR, F2;
};

__device__ __forceinline__ SwFlux sw_face(const Side& l, const Side& r, bool wall) {
    SwFlux f;
    hll_face(l, r, f.F0, f.RL, f.RR, f.F2);
    if (wall) f.F0 = 0.f;  // a wall face carries no mass (see stage.cuh, P4)
    return f;
}

__device__ __forceinline__ float shfl_dn(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float shfl_up(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }

// The stage over one strip per warp. Lane l holds the CPL adjacent columns xs + CPL l + c of the
// strip (c = 0 .. CPL-1); a cell's neighbour in the same lane is read directly, across lanes by a
// shuffle, so only the first and last cell of a lane exchange values.
template <int MODE, int ORDER, int CPL>
__global__ void __launch_bounds__(SW_NT, SW_MINB) swe_stream_kernel(StageArgs a, int strips_x) {
    constexpr int OUT = sw_out(CPL);
    __shared__ float s_maker[2];
    __shared__ float s_red[SW_WARPS];
    __shared__ int s_nan;
    const DevGrid& g = a.g;
    const Ctl* ctl = a.ctl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_nan = 0;
        if (a.maker.on) {
            // forcing.rs:124-138 split as profile(x) * ramp(t) * (sin wt cos k_y y - cos wt sin k_y y)
            const double dt = ctl->dt;
            const double t = ctl->t + (a.stage_time_plus_dt ? dt : 0.0);
            const double ramp = t >= a.maker.ramp_time
                                    ? 1.0
                                    : 0.5 * (1.0 - cos(3.141592653589793 * t / a.maker.ramp_time));
            s_maker[0] = (float)(ramp * sin(a.maker.omega * t));
            s_maker[1] = (float)(ramp * cos(a.maker.omega * t));
        }
    }
    __syncthreads();
    if (!ctl->active) return;  // uniform over the grid: every block returns before its fold

    const double dt = ctl->dt;
    const float dt_f = (float)dt;
    const float dtdx = (float)(dt / g.dxd), dtdy = (float)(dt / g.dyd);
    const float mk0 = s_maker[0], mk1 = s_maker[1];

    const int strip = blockIdx.x * SW_WARPS + warp;  // strips_x strips across, gridDim.y down
    const bool strip_on = strip < strips_x;
    const int xs = (strip_on ? strip : 0) * OUT - SW_HALO;  // column of lane 0's first cell
    const int j0 = blockIdx.y * SW_ROWS;
    int col[CPL], mi[CPL];
    float sx[CPL], prof[CPL];
    bool own[CPL], wall_x[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const int l = CPL * lane + c;
        col[c] = xs + l;
        mi[c] = reflect_idx(col[c], g.nx);
        sx[c] = ((unsigned)col[c] < (unsigned)g.nx) ? 1.f : -1.f;
        own[c] = strip_on && l >= SW_HALO && l < SW_HALO + OUT && col[c] < g.nx;
        wall_x[c] = (col[c] + 1 == 0) || (col[c] + 1 == g.nx);  // the face to the cell's right
        prof[c] = (a.maker.on && own[c]) ? __ldg(a.maker.prof + col[c]) : 0.f;
    }

    // padded row j: its stored row and the sign of the y-normal momentum there
    auto map_row = [&](int j, int& mj, float& sy) {
        if (g.periodic) {
            mj = wrap_idx(j, g.ny);
            sy = 1.f;
        } else {
            mj = reflect_idx(j, g.ny);
            sy = ((unsigned)j < (unsigned)g.ny) ? 1.f : -1.f;
        }
    };
    // row j of this lane's columns, ghost rows mirrored or wrapped
    auto load_row = [&](int j, SwRaw* out) {
        int mj;
        float sy;
        map_row(j, mj, sy);
#pragma unroll
        for (int c = 0; c < CPL; c++) out[c] = sw_load(a, mj * g.pitch + mi[c], sx[c], sy);
    };
    auto wall_y = [&](int jf) -> bool { return !g.periodic && (jf == 0 || jf == g.ny); };  // face below row jf

    // Rows enter the window through take(R), in order from j0-2; the row updated when row R
    // enters is R-2, and its start-of-step state comes with it (q_old, own cells of a finishing
    // second stage).
    const int j_end = (j0 + SW_ROWS < g.ny ? j0 + SW_ROWS : g.ny) - 1;  // the strip's last row
    const int j_last = j_end + 2;                                      // the last row it reads
    unsigned char* ring = nullptr;
    int slot_in = 0, slot_out = 0;
    auto ring_q = [&](int sl, int c) {
        return reinterpret_cast<float4*>(ring + sl * sw_slot_bytes<CPL>()) + c * 32 + lane;
    };
    auto ring_qo = [&](int sl, int c) {
        return reinterpret_cast<float4*>(ring + sl * sw_slot_bytes<CPL>()) + (CPL + c) * 32 + lane;
    };
    auto ring_b = [&](int sl, int c) {
        return reinterpret_cast<float*>(ring + sl * sw_slot_bytes<CPL>() + CPL * 32 * 32) + c * 32 + lane;
    };
    auto issue = [&](int R) {  // start row R's copies (and row R-2's q_old) into the next free slot
        if (R <= j_last) {
            int mj;
            float sy;
            map_row(R, mj, sy);
            const bool qo_on = MODE == MODE_STAGE2 && R - 2 >= j0 && R - 2 <= j_end;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                cp_async16(ring_q(slot_in, c), a.qin + mj * g.pitch + mi[c]);
                cp_async4(ring_b(slot_in, c), a.bed + mj * g.pitch + mi[c]);
                if (qo_on && own[c]) cp_async16(ring_qo(slot_in, c), a.qold + (size_t)(R - 2) * g.pitch + col[c]);
            }
        }
        cp_async_commit();
        slot_in = slot_in + 1 == SW_SLOTS ? 0 : slot_in + 1;
    };
    SwRaw ahead[SW_DEPTH > 0 ? 1 : SW_AHEAD][CPL];
    auto take = [&](int R, SwRaw* out, float4* q_old) {
        if constexpr (SW_DEPTH > 0) {
            cp_async_wait<SW_DEPTH - 1>();
            int mj;
            float sy;
            map_row(R, mj, sy);
            const bool qo_on = MODE == MODE_STAGE2 && R - 2 >= j0 && R - 2 <= j_end;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                out[c].q = *ring_q(slot_out, c);
                out[c].q.z *= sx[c];
                out[c].q.w *= sy;
                out[c].b = *ring_b(slot_out, c);
                q_old[c] = (qo_on && own[c]) ? *ring_qo(slot_out, c) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            slot_out = slot_out + 1 == SW_SLOTS ? 0 : slot_out + 1;
            issue(R + SW_DEPTH);
        } else {
#pragma unroll
            for (int c = 0; c < CPL; c++) out[c] = ahead[0][c];
#pragma unroll
            for (int d = 0; d < SW_AHEAD - 1; d++)
#pragma unroll
                for (int c = 0; c < CPL; c++) ahead[d][c] = ahead[d + 1][c];
            load_row(R + SW_AHEAD, ahead[SW_AHEAD - 1]);
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                q_old[c] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (MODE == MODE_STAGE2 && own[c] && R - 2 >= j0 && R - 2 <= j_end)
                    q_old[c] = __ldg(a.qold + (size_t)(R - 2) * g.pitch + col[c]);
            }
        }
    };
    if constexpr (SW_DEPTH > 0) {
        extern __shared__ __align__(16) unsigned char sw_dyn[];
        ring = sw_dyn + warp * SW_SLOTS * sw_slot_bytes<CPL>();
#pragma unroll
        for (int d = 0; d < SW_DEPTH; d++) issue(j0 - 2 + d);
    } else {
#pragma unroll
        for (int d = 0; d < SW_AHEAD; d++) load_row(j0 - 2 + d, ahead[d]);
    }

    // ---- prologue: rows j0-2 .. j0+1, the y faces below j0 ----------------------------------
    SwRaw rw[4][CPL];
    float4 q_old[CPL];
#pragma unroll
    for (int d = 0; d < 4; d++) take(j0 - 2 + d, rw[d], q_old);
    SwCell c0[CPL], c1[CPL];
    float4 q_own[CPL], q_nxt[CPL];
    float b_own[CPL], b_nxt[CPL];
    Side hi_y[CPL];
    float Py0[CPL];
    SwFlux fy_lo[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const SwCell cm2 = sw_cell(rw[0][c]), cm1 = sw_cell(rw[1][c]);
        c0[c] = sw_cell(rw[2][c]);
        c1[c] = sw_cell(rw[3][c]);
        Side lo_y, hi_prev;
        float Ptmp;
        sw_recon_y<ORDER>(cm2, cm1, c0[c], lo_y, hi_prev, Ptmp);     // row j0-1
        sw_recon_y<ORDER>(cm1, c0[c], c1[c], lo_y, hi_y[c], Py0[c]);  // row j0
        fy_lo[c] = sw_face(hi_prev, lo_y, wall_y(j0));
        q_own[c] = rw[2][c].q;  // as stored: interior cells carry no sign flip
        b_own[c] = rw[2][c].b;
        q_nxt[c] = rw[3][c].q;
        b_nxt[c] = rw[3][c].b;
    }

    float rmax = 0.f;
    int nan_here = 0;
    for (int r = 0; r < SW_ROWS; r++) {
        const int j = j0 + r;
        if (j >= g.ny) break;  // uniform over the warp
        // the next row enters the window (with row j's start-of-step state)
        SwRaw r2[CPL];
        take(j + 2, r2, q_old);

        // y: reconstruct row j+1, the face above row j
        SwCell c2[CPL];
        Side hi_n[CPL];
        float Py1[CPL];
        SwFlux fy_hi[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            c2[c] = sw_cell(r2[c]);
            Side lo_n;
            sw_recon_y<ORDER>(c0[c], c1[c], c2[c], lo_n, hi_n[c], Py1[c]);
            fy_hi[c] = sw_face(hi_y[c], lo_n, wall_y(j + 1));
        }

        // x: reconstruct row j; the lane's first cell takes its left neighbour from the lane
        // before, its last cell its right neighbour from the lane after
        SwCell left, right;
        left.eta = shfl_up(c0[CPL - 1].eta);
        left.u = shfl_up(c0[CPL - 1].u);
        left.v = shfl_up(c0[CPL - 1].v);
        left.h = shfl_up(c0[CPL - 1].h);
        left.b = shfl_up(c0[CPL - 1].b);
        right.eta = shfl_dn(c0[0].eta);
        right.u = shfl_dn(c0[0].u);
        right.v = shfl_dn(c0[0].v);
        right.h = shfl_dn(c0[0].h);
        right.b = shfl_dn(c0[0].b);
        Side lo_x[CPL], hi_x[CPL];
        float Px[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const SwCell& m = c > 0 ? c0[c - 1] : left;
            const SwCell& p = c < CPL - 1 ? c0[c + 1] : right;
            const SwCell& o = c0[c];
            sw_recon<ORDER>(m.eta, o.eta, p.eta, m.u, o.u, p.u, m.v, o.v, p.v, m.h, o.h, p.h, m.b, o.b, p.b,
                            lo_x[c], hi_x[c], Px[c]);
        }
        // the face to each cell's right; the one right of the lane's last cell needs the next
        // lane's first low side; the face left of the lane's first cell is the lane before's last
        Side lo_next;
        lo_next.eta = shfl_dn(lo_x[0].eta);
        lo_next.un = shfl_dn(lo_x[0].un);
        lo_next.ut = shfl_dn(lo_x[0].ut);
        lo_next.z = shfl_dn(lo_x[0].z);
        lo_next.h = 0.f;
        SwFlux fx_r[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) fx_r[c] = sw_face(hi_x[c], c < CPL - 1 ? lo_x[c + 1] : lo_next, wall_x[c]);
        SwFlux fx_l0;
        fx_l0.F0 = shfl_up(fx_r[CPL - 1].F0);
        fx_l0.RL = shfl_up(fx_r[CPL - 1].RL);
        fx_l0.RR = shfl_up(fx_r[CPL - 1].RR);
        fx_l0.F2 = shfl_up(fx_r[CPL - 1].F2);

        float2 cs = make_float2(0.f, 0.f);
        if (a.maker.on) cs = __ldg(a.maker.ycs + j);
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            if (!own[c]) continue;
            const SwFlux& fx_hi = fx_r[c];
            const SwFlux& fx_lo = c > 0 ? fx_r[c - 1] : fx_l0;
            const float maker = a.maker.on ? prof[c] * (mk0 * cs.x - mk1 * cs.y) : 0.f;
            const float lh = -(fx_hi.F0 - fx_lo.F0) * g.inv_dx - (fy_hi[c].F0 - fy_lo[c].F0) * g.inv_dy + maker;
            const float lhu = -(fx_hi.RL - fx_lo.RR) * g.inv_dx - Px[c] * g.inv_dx -
                              (fy_hi[c].F2 - fy_lo[c].F2) * g.inv_dy;
            const float lhv = -(fy_hi[c].RL - fy_lo[c].RR) * g.inv_dy - Py0[c] * g.inv_dy -
                              (fx_hi.F2 - fx_lo.F2) * g.inv_dx;
            // Mass: each face's dt/dx-scaled flux is rounded once; both neighbours add the same value.
            const double dh = ((double)__fmul_rn(dtdx, fx_lo.F0) - (double)__fmul_rn(dtdx, fx_hi.F0)) +
                              ((double)__fmul_rn(dtdy, fy_lo[c].F0) - (double)__fmul_rn(dtdy, fy_hi[c].F0)) +
                              dt * (double)maker;
            double hn = depth64(q_own[c]) + dh;
            float hu = q_own[c].z + dt_f * lhu, hv = q_own[c].w + dt_f * lhv;
            clean_dry(hn, hu, hv);
            const size_t k = (size_t)j * g.pitch + col[c];
            if (MODE == MODE_STAGE1) {
                a.qout[k] = pack_state(hn, hu, hv);
            } else {
                if (MODE == MODE_STAGE2) {
                    // RK2 average over the step (solver.rs:492-501), then clean_dry
                    hn = 0.5 * (depth64(q_old[c]) + hn);
                    hu = 0.5f * (q_old[c].z + hu);
                    hv = 0.5f * (q_old[c].w + hv);
                    clean_dry(hn, hu, hv);
                }
                damp_cell(a.damp, g, col[c], j, b_own[c], dt, hn, hu, hv);
                a.qout[k] = pack_state(hn, hu, hv);
                const float rt = cfl_rate(g, (float)hn, hu, hv);
                if (rt != rt) nan_here = 1;
                else rmax = fmaxf(rmax, rt);
            }
        }
        // advance the window
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            c0[c] = c1[c];
            c1[c] = c2[c];
            q_own[c] = q_nxt[c];
            b_own[c] = b_nxt[c];
            q_nxt[c] = r2[c].q;
            b_nxt[c] = r2[c].b;
            hi_y[c] = hi_n[c];
            Py0[c] = Py1[c];
            fy_lo[c] = fy_hi[c];
        }
    }

    if constexpr (SW_DEPTH > 0) cp_async_wait<0>();  // rows past the strip's end copy nothing

    if (MODE != MODE_STAGE1) {
        rmax = warp_max(rmax);
        if (nan_here) s_nan = 1;  // every writer stores 1
        if (lane == 0) s_red[warp] = rmax;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = 0.f;
            for (int w = 0; w < SW_WARPS; w++) m = fmaxf(m, s_red[w]);
            s_red[0] = m;
        }
        __syncthreads();
        fold_rate_and_finish(a.ctl, s_red[0], s_nan, gridDim.x * gridDim.y);
    }
}

}  // namespace wcb
