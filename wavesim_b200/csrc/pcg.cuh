// pcg.cuh — the SGN dispersive solve as one persistent cooperative kernel.
//
// The reference solves  h w - grad(c div w) = r  by Jacobi-preconditioned conjugate gradients
// from the previous solution, stopping when ||r|| <= tol ||b|| + 1e-10 or after max_iterations
// (crates/wavecore/src/dispersion.rs:493-545). This kernel runs the same method in its
// single-reduction (Chronopoulos-Gear) form, which has the same iterates in exact arithmetic:
//   init   r = b - A w, the inverse diagonal, <b,b>, <r,r>             (one reduction)
//          q = A (r / diag), <r, u>, <u, q>                              (one reduction)
//   iter   p = u + beta p, s = q + beta s, w += alpha p, r -= alpha s,
//          u = r / diag, q = A u, <r,u>, <u,q>, <r,r>                    (one reduction)
// one sweep and one grid-wide reduction per iteration instead of the textbook's two.
//
// Every CTA owns a fixed set of 32x16 tiles for the whole solve, and every sweep is software-
// pipelined: the next tile's halo box is loaded into registers while the current tile computes.
// A reduction is also the grid barrier: CTAs publish FP64 partials and arrive; after the release
// every CTA adds all partials in CTA order with the same tree, so every CTA holds the same bits
// and takes the same convergence decision (reproducible runs). Waits are bounded in time; on
// expiry the kernel sets ERR_TIMEOUT and every CTA returns.
//
// After the loop the same kernel finishes the stage: hu = pred + dt * h * w (the reference's
// lhu = h w + u lh, dispersion.rs:547-562), clean_dry, and on the last stage the RK2 average,
// sponge, friction and the CFL rate of the new state.
#pragma once

#include "common.cuh"
#include "stage.cuh"

namespace wcb {

constexpr int PG_TX = 32, PG_TY = 16, PG_NT = PG_TX * PG_TY;
constexpr int PB_W = PG_TX + 4, PB_H = PG_TY + 4, PB_N = PB_W * PB_H;  // vector box, halo 2
constexpr int PC_W = PG_TX + 2, PC_H = PG_TY + 2, PC_N = PC_W * PC_H;  // c and c div p, halo 1
struct PcgArgs {
    DevGrid g;
    const float* cc;
    const float* heff;
    const float2* bv;
    float2* w;
    float2* r;
    float2* p0;       // p (the CG sweep's search direction; own cells only)
    float2* p1;
    float2* rb[2];    // the CG sweep's banks of r (bank 0 is r), s = A p and q = A (r / diag)
    float2* sb[2];
    float2* qb[2];
    float2* ap;
    float2* diag;     // the inverse Jacobi diagonal (written by the initial sweep)
    double* part;     // [ncta][4] CTA partials
    unsigned* cnt;    // [0] arrivals, [1] released epoch; zeroed before each launch
    const float2* hn;
    const float2* pred;
    const float4* qold;
    float4* qout;
    const float* bed;
    Ctl* ctl;
    const FcgScalars* fcg;  // non-null: the solve ran in the learned path's kernels; finish only
    double tol;
    long long max_iter;
    int mode;         // StageMode
    int defer_finish; // the step's last kernel comes later (followed fronts): do not close the step
    int tiles_x, tiles_y;
    int strip_rows;   // rows per strip of the streaming sweeps (pcg_stream.cuh)
    DampParams damp;
    unsigned long long timeout_ns;
};

// Grid-wide sum of up to three values that is also a barrier. Each CTA publishes its partials
// and arrives; the last to arrive releases; every CTA then adds all partials in CTA order with
// the same reduction tree, so all CTAs hold identical totals. Partials alternate between two
// banks by epoch parity: a CTA that has left barrier e can reach barrier e+1 while a slower CTA
// still reads the partials of e, but it cannot reach e+2 before every CTA has arrived at e+1,
// i.e. finished reading e. Returns false if the wait timed out.
template <int NT = PG_NT>
__device__ bool reduce_barrier(const PcgArgs& a, unsigned& epoch, double v0, double v1, double v2,
                               double* out, double* red, int cta, int ncta) {
    __shared__ int s_ok;
    block_sum3<NT>(v0, v1, v2, red);
    epoch += 1;  // every thread keeps the count: it selects the bank below
    if (threadIdx.x == 0) {
        double* pp = a.part + 4 * ((size_t)cta + (epoch & 1u) * (size_t)ncta);
        pp[0] = v0;
        pp[1] = v1;
        pp[2] = v2;
        __threadfence();
        int ok = 1;
        const unsigned arrived = atomicAdd(a.cnt, 1u) + 1u;
        if (arrived == epoch * (unsigned)ncta) {
            st_release_u32(a.cnt + 1, epoch);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (ld_acquire_u32(a.cnt + 1) < epoch) {
                if (ld_volatile_int(&a.ctl->error) & ERR_TIMEOUT) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > a.timeout_ns) {
                    atomicOr(&a.ctl->error, ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return false;
    double x = 0.0, y = 0.0, z = 0.0;
    const double* bank = a.part + 4 * (size_t)(epoch & 1u) * (size_t)ncta;
    for (int b = threadIdx.x; b < ncta; b += NT) {
        const double* pp = bank + 4 * (size_t)b;
        x += __ldcg(pp);
        y += __ldcg(pp + 1);
        z += __ldcg(pp + 2);
    }
    block_sum3<NT>(x, y, z, red);
    out[0] = x;
    out[1] = y;
    out[2] = z;
    return true;
}

struct TileSmem {
    float2 sv[PB_N];
    float scc[PC_N];
    float sf[PC_N];
    float2 sr[PB_N], ss[PB_N], su[PB_N];  // the CG sweep's r', s and u = r / diag on the box
};

constexpr int PB_PER = (PB_N + PG_NT - 1) / PG_NT;  // box positions per thread
constexpr int PC_PER = (PC_N + PG_NT - 1) / PG_NT;

// A tile's box of vector data, c box and own-cell heff, held in registers between the loads
// and the moment the tile's shared memory is free: the next tile's loads overlap this tile's
// arithmetic.
struct BoxPrefetch {
    float2 v0[PB_PER];
    float he_box[PB_PER];
    float sx[PB_PER], sy[PB_PER];
    float c[PC_PER];
    float he;
};

__device__ __forceinline__ void tile_origin(const PcgArgs& a, int tl, int& i0, int& j0) {
    i0 = (tl % a.tiles_x) * PG_TX;
    j0 = (tl / a.tiles_x) * PG_TY;
}

// The initial sweep's loads for a tile: the warm start w and heff on the box, c on the tile
// plus 1, heff of the own cell.
__device__ __forceinline__ void box_prefetch_init(const PcgArgs& a, int tl, BoxPrefetch& f) {
    int i0, j0;
    tile_origin(a, tl, i0, j0);
    const DevGrid& g = a.g;
#pragma unroll
    for (int n = 0; n < PB_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PB_N) {
            const Mapped m = map_cell(g, i0 - 2 + q % PB_W, j0 - 2 + q / PB_W);
            f.sx[n] = m.sx;
            f.sy[n] = m.sy;
            f.v0[n] = a.w[m.k];
            f.he_box[n] = __ldg(a.heff + m.k);
        }
    }
#pragma unroll
    for (int n = 0; n < PC_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PC_N) {
            const Mapped m = map_cell(g, i0 - 1 + q % PC_W, j0 - 1 + q / PC_W);
            f.c[n] = __ldg(a.cc + m.k);
        }
    }
    const int i = i0 + threadIdx.x % PG_TX, j = j0 + threadIdx.x / PG_TX;
    f.he = (i < g.nx && j < g.ny) ? __ldg(a.heff + j * g.pitch + i) : 0.f;
}

// The warm start masked (dispersion.rs:480-490) and signed for ghost positions; c.
__device__ __forceinline__ void box_commit_init(const BoxPrefetch& f, TileSmem& t) {
#pragma unroll
    for (int n = 0; n < PB_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PB_N) {
            const float2 v = f.he_box[n] >= H_DISP_MIN ? f.v0[n] : make_float2(0.f, 0.f);
            t.sv[q] = make_float2(v.x * f.sx[n], v.y * f.sy[n]);
        }
    }
#pragma unroll
    for (int n = 0; n < PC_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PC_N) t.scc[q] = f.c[n];
    }
}

// f = c div v on the tile plus one ring, then A v = mask (heff v - grad f) for the own cell
// (dispersion.rs:269-317). sv holds v on the tile plus a 2-cell halo.
__device__ __forceinline__ float2 apply_a(const DevGrid& g, TileSmem& t, int cx, int cy, float heff_own) {
    for (int q = threadIdx.x; q < PC_N; q += PG_NT) {
        const int bx = q % PC_W, by = q / PC_W;
        const int pv = (by + 1) * PB_W + (bx + 1);
        t.sf[q] = t.scc[q] * ((t.sv[pv + 1].x - t.sv[pv - 1].x) * g.ix + (t.sv[pv + PB_W].y - t.sv[pv - PB_W].y) * g.iy);
    }
    __syncthreads();
    const float mask = heff_own >= H_DISP_MIN ? 1.f : 0.f;
    const int pc = (cy + 1) * PC_W + (cx + 1);
    const float2 v = t.sv[(cy + 2) * PB_W + (cx + 2)];
    float2 av;
    av.x = mask * (heff_own * v.x - (t.sf[pc + 1] - t.sf[pc - 1]) * g.ix);
    av.y = mask * (heff_own * v.y - (t.sf[pc + PC_W] - t.sf[pc - PC_W]) * g.iy);
    return av;
}

// One CG sweep's loads for a tile, taken one tile ahead: r, q = A u and the previous s on the
// box (tile plus 2 cells), the inverse diagonal there, c on the tile plus 1, and the own cell's p, w.
struct CgPrefetch {
    float2 r[PB_PER], q[PB_PER], s[PB_PER], d[PB_PER];
    float sx[PB_PER], sy[PB_PER];
    float c[PC_PER];
    float he;
    float2 p, x;
};

__device__ __forceinline__ void cg_prefetch(const PcgArgs& a, int tl, int rb, bool init, bool first, CgPrefetch& f) {
    int i0, j0;
    tile_origin(a, tl, i0, j0);
    const DevGrid& g = a.g;
#pragma unroll
    for (int n = 0; n < PB_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PB_N) {
            const Mapped m = map_cell(g, i0 - 2 + q % PB_W, j0 - 2 + q / PB_W);
            f.sx[n] = m.sx;
            f.sy[n] = m.sy;
            f.r[n] = __ldcg(a.rb[rb] + m.k);
            f.d[n] = __ldcg(a.diag + m.k);
            if (!init) {
                f.q[n] = __ldcg(a.qb[rb] + m.k);
                if (!first) f.s[n] = __ldcg(a.sb[rb] + m.k);
            }
        }
    }
#pragma unroll
    for (int n = 0; n < PC_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PC_N) {
            const Mapped m = map_cell(g, i0 - 1 + q % PC_W, j0 - 1 + q / PC_W);
            f.c[n] = __ldg(a.cc + m.k);
        }
    }
    const int i = i0 + threadIdx.x % PG_TX, j = j0 + threadIdx.x / PG_TX;
    const bool own = i < g.nx && j < g.ny;
    const int k = j * g.pitch + i;
    f.he = own ? __ldg(a.heff + k) : 0.f;
    if (!init && own) {
        f.x = __ldcg(a.w + k);
        if (!first) f.p = __ldcg(a.p0 + k);
    }
}

// s = q + beta s, r' = r - alpha s and u' = r' / diag at every box position (the diagonal is
// stored inverted) (the halo's copies
// are this CTA's own recomputation from the old banks); u' (signed for ghost positions) feeds
// A u'; s, r' and u = r / diag are kept for the own cells.
__device__ __forceinline__ void cg_commit(const CgPrefetch& f, TileSmem& t, float alpha, float beta, bool init, bool first) {
#pragma unroll
    for (int n = 0; n < PB_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PB_N) {
            const float2 r = f.r[n], d = f.d[n];
            float2 rn = r;
            if (!init) {
                float2 sk = f.q[n];
                if (!first) {
                    sk.x += beta * f.s[n].x;
                    sk.y += beta * f.s[n].y;
                }
                rn = make_float2(r.x - alpha * sk.x, r.y - alpha * sk.y);
                t.ss[q] = sk;
                t.su[q] = make_float2(r.x * d.x, r.y * d.y);
            }
            t.sr[q] = rn;
            t.sv[q] = make_float2(rn.x * d.x * f.sx[n], rn.y * d.y * f.sy[n]);
        }
    }
#pragma unroll
    for (int n = 0; n < PC_PER; n++) {
        const int q = threadIdx.x + n * PG_NT;
        if (q < PC_N) t.scc[q] = f.c[n];
    }
}


// The solve and the stage epilogue, by the `ncta` CTAs (this one is number `cta`) that own this
// run. `epoch` counts the run's grid barriers within the launch. Returns false if a bounded
// wait expired (every CTA of the run then returns).
__device__ __forceinline__ bool pcg_solve(const PcgArgs& a, int cta, int ncta, unsigned& epoch) {
    __shared__ TileSmem t;
    __shared__ double red[100];
    __shared__ float s_rate[PG_NT / 32];
    __shared__ int s_nan;

    Ctl* ctl = a.ctl;
    const DevGrid& g = a.g;
    const int tid = threadIdx.x;
    const int cx = tid % PG_TX, cy = tid / PG_TX;
    const int ntiles = a.tiles_x * a.tiles_y;
    const double dt = ctl->dt;
    const float dt_f = (float)dt;
    double tot[3];
    if (tid == 0) s_nan = 0;
    BoxPrefetch f;

    long long it = 0;
    bool converged = false;
    if (a.fcg && a.fcg->converged) {  // solved by the learned flexible CG: finish only
        converged = true;
    } else {  // the Jacobi solve; after a learned solve that failed, from where that one stopped
        // ---- initial residual: r = b - A w (dispersion.rs:493-515) ---------------------------
        double bb = 0.0, rr_p = 0.0;
        if (cta < ntiles) box_prefetch_init(a, cta, f);
        for (int tl = cta; tl < ntiles; tl += ncta) {
            int i0, j0;
            tile_origin(a, tl, i0, j0);
            box_commit_init(f, t);
            const float he = f.he;
            __syncthreads();
            if (tl + ncta < ntiles) box_prefetch_init(a, tl + ncta, f);
            const float2 aw = apply_a(g, t, cx, cy, he);
            const int i = i0 + cx, j = j0 + cy;
            if (i < g.nx && j < g.ny) {
                const int k = j * g.pitch + i;
                const int pc = (cy + 1) * PC_W + (cx + 1);
                float2 d = make_float2(1.f, 1.f);
                if (he >= H_DISP_MIN) {
                    d.x = he + (t.scc[pc + 1] + t.scc[pc - 1]) * 0.25f / (g.dx * g.dx);
                    d.y = he + (t.scc[pc + PC_W] + t.scc[pc - PC_W]) * 0.25f / (g.dy * g.dy);
                }
                const float2 b = __ldg(a.bv + k);
                const float2 r = make_float2(b.x - aw.x, b.y - aw.y);
                a.w[k] = t.sv[(cy + 2) * PB_W + (cx + 2)];  // the warm start, masked
                a.diag[k] = make_float2(1.f / d.x, 1.f / d.y);  // the CG sweeps multiply by the inverse
                a.r[k] = r;
                bb += (double)b.x * b.x + (double)b.y * b.y;
                rr_p += (double)r.x * r.x + (double)r.y * r.y;
            }
            __syncthreads();
        }
        if (!reduce_barrier(a, epoch, bb, 0.0, rr_p, tot, red, cta, ncta)) return false;
        const double target = a.tol * sqrt(tot[0]) + 1e-10;
        converged = sqrt(tot[2]) <= target;
        // ---- single-reduction CG (Chronopoulos-Gear form of the same Jacobi PCG) --------------
        // With u = r / diag and q = A u, the direction's image s = A p obeys s = q + beta s, and
        // <p, s> = delta - beta gamma / alpha_prev (gamma = <r, u>, delta = <u, q>), so one sweep
        // per iteration does p = u + beta p, s = q + beta s, w += alpha p, r -= alpha s,
        // u = r / diag, q = A u and the three dots, with one grid reduction. r, s and q are read
        // on a 2-cell halo and alternate between two banks by iteration; the halo's new u is
        // recomputed from the old banks, so no CTA waits for its neighbours within a sweep.
        // Sweep "first" (k = -1) only forms q0 = A u0 and gamma0, delta0 from r0.
        double gamma = 0.0, delta = 0.0, alpha_prev = 1.0, beta = 0.0;
        CgPrefetch cf;
        auto cg_sweep = [&](int k, float alpha_f, float beta_f, double* dots) -> bool {
            const bool init = k < 0;
            const bool first = k == 0;
            const int rb = init ? 0 : (k & 1), wb = init ? 0 : ((k + 1) & 1);
            double g1 = 0.0, g2 = 0.0, g3 = 0.0;
            if (cta < ntiles) cg_prefetch(a, cta, rb, init, first, cf);
            for (int tl = cta; tl < ntiles; tl += ncta) {
                int i0, j0;
                tile_origin(a, tl, i0, j0);
                cg_commit(cf, t, alpha_f, beta_f, init, first);
                const float he = cf.he;
                const float2 p_own = cf.p, w_own = cf.x;
                __syncthreads();
                if (tl + ncta < ntiles) cg_prefetch(a, tl + ncta, rb, init, first, cf);
                const float2 q = apply_a(g, t, cx, cy, he);
                const int i = i0 + cx, j = j0 + cy;
                if (i < g.nx && j < g.ny) {
                    const int kk = j * g.pitch + i;
                    const int c0 = (cy + 2) * PB_W + (cx + 2);
                    const float2 u = t.sv[c0];
                    const float2 r = t.sr[c0];
                    if (!init) {
                        const float2 sk = t.ss[c0], uk = t.su[c0];
                        float2 pk = uk;
                        if (!first) {
                            pk.x += beta_f * p_own.x;
                            pk.y += beta_f * p_own.y;
                        }
                        a.p0[kk] = pk;
                        a.w[kk] = make_float2(w_own.x + alpha_f * pk.x, w_own.y + alpha_f * pk.y);
                        a.sb[wb][kk] = sk;
                        a.rb[wb][kk] = r;
                    }
                    a.qb[wb][kk] = q;
                    g1 += (double)r.x * u.x + (double)r.y * u.y;
                    g2 += (double)u.x * q.x + (double)u.y * q.y;
                    g3 += (double)r.x * r.x + (double)r.y * r.y;
                }
                __syncthreads();
            }
            return reduce_barrier(a, epoch, g1, g2, g3, dots, red, cta, ncta);
        };
        if (!converged) {
            if (!cg_sweep(-1, 0.f, 0.f, tot)) return false;
            gamma = tot[0];
            delta = tot[1];
        }
        while (!converged && it < a.max_iter) {
            const double alpha = it == 0 ? gamma / delta : gamma / (delta - beta * gamma / alpha_prev);
            if (!cg_sweep((int)it, (float)alpha, (float)beta, tot)) return false;
            it += 1;
            converged = sqrt(tot[2]) <= target;
            beta = tot[0] / gamma;
            gamma = tot[0];
            delta = tot[1];
            alpha_prev = alpha;
        }
    }
    if (a.fcg) it += a.fcg->iterations;
    if (cta == 0 && tid == 0) {
        if (a.fcg) ctl->fcg_iterations += (unsigned long long)a.fcg->iterations;
        ctl->solves += 1;
        ctl->iterations += (unsigned long long)it;
        if (!converged) ctl->unconverged += 1;
        ctl->last_iterations = (int)it;
    }

    // ---- finish the stage from the solution (every w is final: the last reduction was a barrier)
    float rmax = 0.f;
    int nan_here = 0;
    for (int tl = cta; tl < ntiles; tl += ncta) {
        int i0, j0;
        tile_origin(a, tl, i0, j0);
        const int i = i0 + cx, j = j0 + cy;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const float2 hn = __ldg(a.hn + k);
        const float2 pr = __ldg(a.pred + k);
        const float2 w = __ldcg(a.w + k);
        const float he = __ldg(a.heff + k);
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a.mode == MODE_STAGE2) q0 = __ldg(a.qold + k);
        double h = (double)hn.x + (double)hn.y;
        float hu = pr.x + dt_f * (he * w.x);
        float hv = pr.y + dt_f * (he * w.y);
        clean_dry(h, hu, hv);
        if (a.mode == MODE_STAGE1) {
            a.qout[k] = pack_state(h, hu, hv);
            continue;
        }
        if (a.mode == MODE_STAGE2) {
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
    if (a.mode != MODE_STAGE1 && !a.defer_finish) {
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
        fold_rate_and_finish(ctl, s_rate[0], s_nan, (unsigned)ncta);
    }
    return true;
}

__global__ void __launch_bounds__(PG_NT, 2) pcg_kernel(PcgArgs a) {
    if (!a.ctl->active) return;
    unsigned epoch = 0;
    pcg_solve(a, blockIdx.x, gridDim.x, epoch);
}

}  // namespace wcb
