// pcg.cuh — the SGN dispersive solve as one persistent cooperative kernel.
//
// The reference solves  h w - grad(c div w) = r  by Jacobi-preconditioned conjugate gradients
// from the previous solution, stopping when ||r|| <= tol ||b|| + 1e-10 or after max_iterations
// (crates/wavecore/src/dispersion.rs:493-545). Here every CTA owns a fixed set of 32x8 tiles for
// the whole solve; the sweeps are separated by grid barriers whose waits are bounded in time
// (on expiry the kernel sets an error bit and returns, never traps), and the dot products are
// FP64, reduced per CTA with a fixed tree and then over CTAs in a fixed order by every CTA, so
// all CTAs take the same convergence decision and results are reproducible run to run.
//
// After the loop the same kernel finishes the stage: hu = pred + dt * h * w (the reference's
// lhu = h w + u lh, dispersion.rs:547-562), clean_dry, and on the last stage the RK2 average,
// sponge, friction and the CFL rate of the new state.
#pragma once

#include "common.cuh"
#include "stage.cuh"

namespace wcb {

constexpr int PG_TX = 32, PG_TY = 8, PG_NT = 256;
constexpr int PB_W = PG_TX + 4, PB_H = PG_TY + 4, PB_N = PB_W * PB_H;  // vector box, halo 2
constexpr int PC_W = PG_TX + 2, PC_H = PG_TY + 2, PC_N = PC_W * PC_H;  // c and c div p, halo 1

struct PcgArgs {
    DevGrid g;
    const float* cc;
    const float* heff;
    const float2* bv;
    float2* w;
    float2* r;
    float2* p;
    float2* ap;
    float2* diag;
    double* part;     // [2][gridDim.x][4]: double-buffered so that a CTA publishing the next
                      // sums never overwrites values a slower CTA is still reading
    unsigned* bar;    // [2]: arrivals, released epoch; zeroed before each launch
    const float2* hn;
    const float2* pred;
    const float4* qold;
    float4* qout;
    const float* bed;
    Ctl* ctl;
    double tol;
    long long max_iter;
    int mode;         // StageMode
    int tiles_x, tiles_y;
    DampParams damp;
    unsigned long long timeout_ns;
};

// Bounded grid barrier: a monotonic arrival counter and a released-epoch word. Every CTA is
// co-resident (cooperative launch), so the wait ends unless a CTA has failed; it gives up after
// timeout_ns, sets ERR_TIMEOUT and makes every CTA leave.
__device__ __forceinline__ bool grid_barrier(const PcgArgs& a, unsigned& epoch) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch += 1;
        int ok = 1;
        __threadfence();
        const unsigned arrived = atomicAdd(&a.bar[0], 1u) + 1u;
        if (arrived == epoch * gridDim.x) {
            st_release_u32(&a.bar[1], epoch);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (ld_acquire_u32(&a.bar[1]) < epoch) {
                if (ld_volatile_int(&a.ctl->error) & ERR_TIMEOUT) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > a.timeout_ns) {
                    atomicOr(&a.ctl->error, ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// The CTAs' partial sums of one slot, summed in CTA order by every CTA.
__device__ __forceinline__ void grid_totals(const PcgArgs& a, int buf, int nslots, double* out,
                                            double* red) {
    double v[3] = {0.0, 0.0, 0.0};
    const double* part = a.part + (size_t)buf * gridDim.x * 4;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += PG_NT)
        for (int s = 0; s < nslots; s++) v[s] += __ldcg(part + 4 * b + s);
    block_sum3<PG_NT>(v[0], v[1], v[2], red);
    for (int s = 0; s < nslots; s++) out[s] = v[s];
}

__device__ __forceinline__ void publish(const PcgArgs& a, int buf, double x, double y, double z,
                                        double* red) {
    block_sum3<PG_NT>(x, y, z, red);
    if (threadIdx.x == 0) {
        double* part = a.part + ((size_t)buf * gridDim.x + blockIdx.x) * 4;
        part[0] = x;
        part[1] = y;
        part[2] = z;
    }
}

// A v on one tile (dispersion.rs:269-317): v is staged with a 2-cell halo of ghost-synthesised
// values (vector ghosts: the wall-normal component flips), c with a 1-cell halo, c div v on
// the tile plus one ring, then mask (heff v - grad(c div v)). With INIT the source is the warm
// start, masked on the fly (dispersion.rs:480-490), and the tile also writes the Jacobi diagonal.
template <bool INIT>
__device__ __forceinline__ float2 tile_matvec(const PcgArgs& a, int i0, int j0, const float2* src,
                                              float2* sv, float* scc, float* sf, bool& own_valid,
                                              int& k_own, float& heff_own) {
    const DevGrid& g = a.g;
    const int tid = threadIdx.x;
    for (int q = tid; q < PB_N; q += PG_NT) {
        const int bx = q % PB_W, by = q / PB_W;
        const Mapped m = map_cell(g, i0 - 2 + bx, j0 - 2 + by);
        float2 v = INIT ? src[m.k] : __ldcg(src + m.k);
        if (INIT && !(__ldg(a.heff + m.k) >= H_DISP_MIN)) v = make_float2(0.f, 0.f);
        sv[q] = make_float2(v.x * m.sx, v.y * m.sy);
    }
    for (int q = tid; q < PC_N; q += PG_NT) {
        const int bx = q % PC_W, by = q / PC_W;
        const Mapped m = map_cell(g, i0 - 1 + bx, j0 - 1 + by);
        scc[q] = __ldg(a.cc + m.k);
    }
    __syncthreads();
    for (int q = tid; q < PC_N; q += PG_NT) {
        const int bx = q % PC_W, by = q / PC_W;
        const int pv = (by + 1) * PB_W + (bx + 1);
        sf[q] = scc[q] * ((sv[pv + 1].x - sv[pv - 1].x) * g.ix + (sv[pv + PB_W].y - sv[pv - PB_W].y) * g.iy);
    }
    __syncthreads();
    const int cx = tid % PG_TX, cy = tid / PG_TX;
    const int i = i0 + cx, j = j0 + cy;
    own_valid = i < g.nx && j < g.ny;
    float2 av = make_float2(0.f, 0.f);
    if (own_valid) {
        k_own = j * g.pitch + i;
        heff_own = __ldg(a.heff + k_own);
        const float mask = heff_own >= H_DISP_MIN ? 1.f : 0.f;
        const int pc = (cy + 1) * PC_W + (cx + 1);
        const float2 v = sv[(cy + 2) * PB_W + (cx + 2)];
        av.x = mask * (heff_own * v.x - (sf[pc + 1] - sf[pc - 1]) * g.ix);
        av.y = mask * (heff_own * v.y - (sf[pc + PC_W] - sf[pc - PC_W]) * g.iy);
        if (INIT) {
            float2 d = make_float2(1.f, 1.f);
            if (mask != 0.f) {
                d.x = heff_own + (scc[pc + 1] + scc[pc - 1]) * 0.25f / (g.dx * g.dx);
                d.y = heff_own + (scc[pc + PC_W] + scc[pc - PC_W]) * 0.25f / (g.dy * g.dy);
            }
            a.diag[k_own] = d;
            a.w[k_own] = v;  // the warm start, masked
        }
    }
    __syncthreads();  // the boxes are reused by the next tile
    return av;
}

__global__ void __launch_bounds__(PG_NT) pcg_kernel(PcgArgs a) {
    __shared__ float2 sv[PB_N];
    __shared__ float scc[PC_N];
    __shared__ float sf[PC_N];
    __shared__ double red[100];
    __shared__ float s_rate[PG_NT / 32];
    __shared__ int s_nan;

    Ctl* ctl = a.ctl;
    if (!ctl->active) return;
    const DevGrid& g = a.g;
    const int tid = threadIdx.x;
    const int ntiles = a.tiles_x * a.tiles_y;
    const double dt = ctl->dt;
    const float dt_f = (float)dt;
    unsigned epoch = 0;
    int buf = 0;  // partial-sum buffer of the next reduction
    if (tid == 0) s_nan = 0;

    // ---- initial residual: r = b - A w, z = r / diag, p = z (dispersion.rs:493-515) ----------
    double bb = 0.0, rz_p = 0.0, rr_p = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = (t % a.tiles_x) * PG_TX, j0 = (t / a.tiles_x) * PG_TY;
        bool ok;
        int k;
        float he;
        const float2 aw = tile_matvec<true>(a, i0, j0, a.w, sv, scc, sf, ok, k, he);
        if (ok) {
            const float2 b = __ldg(a.bv + k);
            const float2 d = a.diag[k];
            const float2 r = make_float2(b.x - aw.x, b.y - aw.y);
            const float2 z = make_float2(r.x / d.x, r.y / d.y);
            a.r[k] = r;
            a.p[k] = z;
            bb += (double)b.x * b.x + (double)b.y * b.y;
            rz_p += (double)r.x * z.x + (double)r.y * z.y;
            rr_p += (double)r.x * r.x + (double)r.y * r.y;
        }
    }
    publish(a, buf, bb, rz_p, rr_p, red);
    if (!grid_barrier(a, epoch)) return;
    double tot[3];
    grid_totals(a, buf, 3, tot, red);
    buf ^= 1;
    const double target = a.tol * sqrt(tot[0]) + 1e-10;
    double rz = tot[1];
    bool converged = sqrt(tot[2]) <= target;
    long long it = 0;

    while (!converged && it < a.max_iter) {
        // sweep A: Ap and <p, Ap>
        double pap = 0.0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int i0 = (t % a.tiles_x) * PG_TX, j0 = (t / a.tiles_x) * PG_TY;
            bool ok;
            int k;
            float he;
            const float2 av = tile_matvec<false>(a, i0, j0, a.p, sv, scc, sf, ok, k, he);
            if (ok) {
                a.ap[k] = av;
                const float2 p = __ldcg(a.p + k);
                pap += (double)p.x * av.x + (double)p.y * av.y;
            }
        }
        publish(a, buf, pap, 0.0, 0.0, red);
        if (!grid_barrier(a, epoch)) return;
        grid_totals(a, buf, 1, tot, red);
        buf ^= 1;
        const double alpha = rz / tot[0];
        const float alpha_f = (float)alpha;
        // sweep B: w += alpha p, r -= alpha Ap, z = r / diag; <r, r> and <r, z>
        double rr = 0.0, rzn = 0.0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int i = (t % a.tiles_x) * PG_TX + tid % PG_TX;
            const int j = (t / a.tiles_x) * PG_TY + tid / PG_TX;
            if (i < g.nx && j < g.ny) {
                const int k = j * g.pitch + i;
                const float2 p = __ldcg(a.p + k), ap = __ldcg(a.ap + k);
                float2 w = __ldcg(a.w + k), r = __ldcg(a.r + k);
                const float2 d = __ldcg(a.diag + k);
                w.x += alpha_f * p.x;
                w.y += alpha_f * p.y;
                r.x -= alpha_f * ap.x;
                r.y -= alpha_f * ap.y;
                a.w[k] = w;
                a.r[k] = r;
                rr += (double)r.x * r.x + (double)r.y * r.y;
                rzn += (double)r.x * (r.x / d.x) + (double)r.y * (r.y / d.y);
            }
        }
        publish(a, buf, rr, rzn, 0.0, red);
        if (!grid_barrier(a, epoch)) return;
        grid_totals(a, buf, 2, tot, red);
        buf ^= 1;
        it += 1;
        converged = sqrt(tot[0]) <= target;
        const double beta = tot[1] / rz;
        rz = tot[1];
        if (converged || it >= a.max_iter) break;
        // sweep C: p = z + beta p
        const float beta_f = (float)beta;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int i = (t % a.tiles_x) * PG_TX + tid % PG_TX;
            const int j = (t / a.tiles_x) * PG_TY + tid / PG_TX;
            if (i < g.nx && j < g.ny) {
                const int k = j * g.pitch + i;
                const float2 r = __ldcg(a.r + k), d = __ldcg(a.diag + k);
                float2 p = __ldcg(a.p + k);
                p.x = r.x / d.x + beta_f * p.x;
                p.y = r.y / d.y + beta_f * p.y;
                a.p[k] = p;
            }
        }
        if (!grid_barrier(a, epoch)) return;
    }
    if (blockIdx.x == 0 && tid == 0) {
        ctl->solves += 1;
        ctl->iterations += (unsigned long long)it;
        if (!converged) ctl->unconverged += 1;
        ctl->last_iterations = (int)it;
    }
    // The solution of every cell must be final before any CTA finishes the stage.
    if (!grid_barrier(a, epoch)) return;

    // ---- finish the stage: the state from the solve --------------------------------------------
    float rmax = 0.f;
    int nan_here = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = (t % a.tiles_x) * PG_TX + tid % PG_TX;
        const int j = (t / a.tiles_x) * PG_TY + tid / PG_TX;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const float2 hn = __ldg(a.hn + k);
        const float2 pr = __ldg(a.pred + k);
        const float2 w = __ldcg(a.w + k);
        const float he = __ldg(a.heff + k);
        double h = (double)hn.x + (double)hn.y;
        float hu = pr.x + dt_f * (he * w.x);
        float hv = pr.y + dt_f * (he * w.y);
        clean_dry(h, hu, hv);
        if (a.mode == MODE_STAGE1) {
            a.qout[k] = pack_state(h, hu, hv);
            continue;
        }
        if (a.mode == MODE_STAGE2) {
            const float4 q0 = __ldg(a.qold + k);
            h = 0.5 * (depth64(q0) + h);
            hu = 0.5f * (q0.z + hu);
            hv = 0.5f * (q0.w + hv);
            clean_dry(h, hu, hv);
        }
        damp_cell(a.damp, g, i, j, __ldg(a.bed + k), dt, h, hu, hv);
        a.qout[k] = pack_state(h, hu, hv);
        const float rt = cfl_rate(g, (float)h, hu, hv);
        if (rt != rt) nan_here = 1;
        else rmax = fmaxf(rmax, rt);
    }
    if (a.mode != MODE_STAGE1) {
        rmax = warp_max(rmax);
        if (nan_here) s_nan = 1;
        if ((tid & 31) == 0) s_rate[tid >> 5] = rmax;
        __syncthreads();
        if (tid == 0) {
            float m = 0.f;
            for (int w = 0; w < PG_NT / 32; w++) m = fmaxf(m, s_rate[w]);
            s_rate[0] = m;
        }
        __syncthreads();
        fold_rate_and_finish(ctl, s_rate[0], s_nan, gridDim.x);
    }
}

}  // namespace wcb
