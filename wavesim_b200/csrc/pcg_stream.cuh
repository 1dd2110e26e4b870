// pcg_stream.cuh — the dispersive solve with streaming sweeps.
//
// The same method as pcg.cuh's pcg_solve: the reference's Jacobi-preconditioned CG
// (crates/wavecore/src/dispersion.rs:493-545) in its single-reduction form, one persistent
// cooperative launch per solve, one grid-wide reduction per iteration (reduce_barrier), the same
// stopping rule and the same epilogue. What differs is how a sweep walks the cells. Instead of
// staging a tile plus its 2-cell halo in shared memory between block barriers, each warp owns
// strips of PS_OUT = 28 columns by a grid's rows per strip and marches down them: its 32 lanes hold the strip's
// columns plus two halo columns on each side, a five-row window of the vector being multiplied (the
// new u = r / diag, recomputed at halo cells from the banks, as pcg_solve does) stays in
// registers, and the x-neighbours of the matrix product
//   A v = mask (heff v - grad f),  f = c div v   (dispersion.rs:269-317)
// come from the lanes beside by warp shuffles: no block barrier inside a sweep. Each lane copies
// its column's rows a few rows ahead with cp.async into the warp's ring in shared memory and reads
// them back as they enter the window, so the loads in flight hold no registers.
#pragma once

#include "common.cuh"
#include "pcg.cuh"

namespace wcb {

// Launch shape. Rows are fetched PS_DEPTH rows before they are used, by cp.async into a ring in
// shared memory (the rows in flight hold no registers), or, with PS_DEPTH 0, PS_AHEAD rows ahead
// into registers. Measured on 2048 x 1024 and 4096 x 4096 (Jacobi, ms per step): the ring with 3
// rows in flight and 2 blocks of 256 threads per SM (127 registers, no spills) 4.95 and 75.4; 4 or
// 5 rows 5.00-5.09 and 74.7-77.9; 3 blocks per SM (80 registers, spills) 5.50 and 80.5; registers
// with 1 or 2 rows ahead 5.83-5.89 and 90.7-92.3 at 2 blocks, 5.49 and 79.5 at 3. Rows per strip
// are fitted so that every warp gets one strip. The macros let a tuning build try others.
#ifndef WCB_PS_MINB
#define WCB_PS_MINB 2
#endif
#ifndef WCB_PS_AHEAD
#define WCB_PS_AHEAD 1
#endif
#ifndef WCB_PS_DEPTH
#define WCB_PS_DEPTH 3
#endif
constexpr int PS_NT = 256, PS_WARPS = PS_NT / 32, PS_MINB = WCB_PS_MINB;
constexpr int PS_HALO = 2, PS_OUT = 32 - 2 * PS_HALO;  // 28 own columns per strip
// Strips of at least 8 rows: at 1024 x 512 (2368 co-resident warps, 37 strips across) 8-row
// strips give every warp one (1.62 ms per step against 1.80 with 16-row strips on half the warps).
#ifndef WCB_PS_ROWS_MIN
#define WCB_PS_ROWS_MIN 8
#endif
constexpr int PS_ROWS_MIN = WCB_PS_ROWS_MIN, PS_ROWS_MAX = 512;  // rows per strip, chosen per grid
constexpr int PS_AHEAD = WCB_PS_AHEAD;                 // register mode: rows in flight beyond the window
constexpr int PS_DEPTH = WCB_PS_DEPTH;                 // ring mode: rows in flight
constexpr int PS_SLOTS = PS_DEPTH + 1;                 // ring slots: a slot is refilled one row after it is read

__device__ __forceinline__ float ps_up(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float ps_dn(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }

__host__ __device__ constexpr int ps_strips(int nx, int ny, int rows) {
    return ((nx + PS_OUT - 1) / PS_OUT) * ((ny + rows - 1) / rows);
}

// Rows per strip for `warps` co-resident warps: as few strips as warps where that leaves strips of
// at least PS_ROWS_MIN rows (the two halo rows above and below a strip are fetched twice).
inline int ps_rows_for(int nx, int ny, int warps) {
    const int sx = (nx + PS_OUT - 1) / PS_OUT;
    const int per_col = warps / sx > 0 ? warps / sx : 1;
    int rows = (ny + per_col - 1) / per_col;
    rows = rows < PS_ROWS_MIN ? PS_ROWS_MIN : rows;
    return rows > PS_ROWS_MAX ? PS_ROWS_MAX : rows;
}

// A warp's ring of rows in flight: PS_SLOTS slots of NF2 float2 and NF1 float fields, laid out
// [slot][field][lane] so that a field of a row is one conflict-free shared access of 32 lanes.
// Bytes per warp, and per block of `warps` warps (dynamic shared memory).
template <int NF2, int NF1>
__host__ __device__ constexpr int ps_ring_bytes() {
    return PS_DEPTH > 0 ? PS_SLOTS * 32 * (8 * NF2 + 4 * NF1) : 0;
}

// The loads of one row go through a loader: ld2(n, p, en) / ld1(n, p, en) give field n of the row,
// the float2 or float at p, or zero where en is false. A fetch names every load of its row in the
// same order with the same en on every call.
//   PsDirect  loads into registers now;
//   PsIssue   starts the copies into the row's ring slot (returns zeros);
//   PsRead    reads the slot back once its copies have landed.
struct PsDirect {
    __device__ __forceinline__ float2 ld2(int, const float2* p, bool en) const {
        return en ? __ldcg(p) : make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ float ld1(int, const float* p, bool en) const { return en ? __ldg(p) : 0.f; }
};
struct PsIssue {
    float2* f2;  // the lane's field 0 in the slot; field n at +32 n
    float* f1;
    bool on;     // false: the row is past the strip's end, nothing is copied
    __device__ __forceinline__ float2 ld2(int n, const float2* p, bool en) const {
        if (on && en) cp_async8(f2 + 32 * n, p);
        return make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ float ld1(int n, const float* p, bool en) const {
        if (on && en) cp_async4(f1 + 32 * n, p);
        return 0.f;
    }
};
struct PsRead {
    const float2* f2;
    const float* f1;
    __device__ __forceinline__ float2 ld2(int n, const float2*, bool en) const {
        return en ? f2[32 * n] : make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ float ld1(int n, const float*, bool en) const { return en ? f1[32 * n] : 0.f; }
};

// The calling warp's ring in the block's dynamic shared memory.
template <int NF2, int NF1>
__device__ __forceinline__ unsigned char* ps_ring() {
    extern __shared__ __align__(16) unsigned char ps_dyn[];
    return ps_dyn + (threadIdx.x >> 5) * ps_ring_bytes<NF2, NF1>();
}

// Loads of an own cell that only its output needs (none by default).
struct PsNoOwn {};
struct PsNoFetchOwn {
    template <class Ld>
    __device__ __forceinline__ PsNoOwn operator()(const Ld&, int, bool) const { return PsNoOwn{}; }
};

// One strip: rows j0-2 .. j0+rows+1 of the lane's column are fetched
// (`fetch(loader, k, sy, j, own, mi, mj)`: the loads at stored index k = mj pitch + mi of padded
// row j, sy the sign of the y-normal component there, own whether the cell is one the strip
// updates) and turned into window rows (`make(raw)`: a Row with the signed vector v, c and heff);
// for every own cell `out(k, i, j, row, Av, c_left, c_right, c_below, c_above, own)` gets the
// row, the product, the four neighbouring c and what `fetch_own(loader, k, en)` loaded for the
// cell: in ring mode those loads travel with the row two below (they are read as that row enters
// the window, just before the cell's output), so they do not wait at the output. NF2 / NF1: the
// ring's fields per row (at least those of fetch and fetch_own together).
template <class Raw, class Row, int NF2, int NF1, class Fetch, class Make, class Out,
          class FetchOwn = PsNoFetchOwn>
__device__ __forceinline__ void ps_strip(const DevGrid& g, int strip, int rows, Fetch fetch, Make make, Out out,
                                         FetchOwn fetch_own = FetchOwn{}) {
    using Own = decltype(fetch_own(PsDirect{}, 0, false));
    const int strips_x = (g.nx + PS_OUT - 1) / PS_OUT;
    const int lane = threadIdx.x & 31;
    const int i = (strip % strips_x) * PS_OUT - PS_HALO + lane;
    const int j0 = (strip / strips_x) * rows;
    const int mi = reflect_idx(i, g.nx);
    const bool own_col = lane >= PS_HALO && lane < PS_HALO + PS_OUT && i < g.nx;
    auto map_row = [&](int j, int& mj, float& sy) {
        if (g.periodic) {
            mj = wrap_idx(j, g.ny);
            sy = 1.f;
        } else {
            mj = reflect_idx(j, g.ny);
            sy = ((unsigned)j < (unsigned)g.ny) ? 1.f : -1.f;
        }
    };
    auto is_own = [&](int j) { return own_col && j >= j0 && j < j0 + rows && j < g.ny; };
    auto get = [&](const auto& ld, int j) -> Raw {
        int mj;
        float sy;
        map_row(j, mj, sy);
        return fetch(ld, mj * g.pitch + mi, sy, j, is_own(j), mi, mj);
    };
    // the own-cell loads of row j (an interior row where they are enabled)
    auto get_own = [&](const auto& ld, int j) -> Own { return fetch_own(ld, j * g.pitch + i, is_own(j)); };
    // f = c div v of the window's middle row
    auto fval = [&](const Row& m, const Row& c, const Row& p) -> float {
        const float vl = ps_up(c.v.x), vr = ps_dn(c.v.x);
        return c.cc * ((vr - vl) * g.ix + (p.v.y - m.v.y) * g.iy);
    };
    // The last row the strip reads: the window reaches two rows below its last own row.
    const int j_last = (j0 + rows < g.ny ? j0 + rows : g.ny) + 1;
    unsigned char* ring = nullptr;
    int slot_in = 0, slot_out = 0;
    auto slot_f2 = [&](int sl) { return reinterpret_cast<float2*>(ring) + sl * NF2 * 32 + lane; };
    auto slot_f1 = [&](int sl) {
        return reinterpret_cast<float*>(ring + PS_SLOTS * NF2 * 32 * 8) + sl * NF1 * 32 + lane;
    };
    auto issue = [&](int j) {  // start row j's copies (and row j-2's own-cell loads) into the next free slot
        PsIssue ld{slot_f2(slot_in), slot_f1(slot_in), j <= j_last};
        (void)get(ld, j);
        (void)get_own(ld, j - 2);
        cp_async_commit();
        slot_in = slot_in + 1 == PS_SLOTS ? 0 : slot_in + 1;
    };
    Raw ahead[PS_DEPTH > 0 ? 1 : PS_AHEAD];
    Own own_cur{};  // the own-cell loads of the row two above the one taken last
    // row j, the oldest row in flight: wait for it, read it (and row j-2's own-cell loads), and
    // start row j + (rows in flight)
    auto take = [&](int j) -> Raw {
        if constexpr (PS_DEPTH > 0) {
            cp_async_wait<PS_DEPTH - 1>();
            const PsRead ld{slot_f2(slot_out), slot_f1(slot_out)};
            const Raw raw = get(ld, j);
            own_cur = get_own(ld, j - 2);
            slot_out = slot_out + 1 == PS_SLOTS ? 0 : slot_out + 1;
            issue(j + PS_DEPTH);
            return raw;
        } else {
            const Raw raw = ahead[0];
#pragma unroll
            for (int d = 0; d < PS_AHEAD - 1; d++) ahead[d] = ahead[d + 1];
            ahead[PS_AHEAD - 1] = get(PsDirect{}, j + PS_AHEAD);
            own_cur = get_own(PsDirect{}, j - 2);
            return raw;
        }
    };
    if constexpr (PS_DEPTH > 0) {
        ring = ps_ring<NF2, NF1>();
#pragma unroll
        for (int d = 0; d < PS_DEPTH; d++) issue(j0 - 2 + d);
    } else {
#pragma unroll
        for (int d = 0; d < PS_AHEAD; d++) ahead[d] = get(PsDirect{}, j0 - 2 + d);
    }
    Row rm2 = make(take(j0 - 2)), rm1 = make(take(j0 - 1)), r0 = make(take(j0)), r1 = make(take(j0 + 1));
    float f_m = fval(rm2, rm1, r0);  // row j0-1
    float f_0 = fval(rm1, r0, r1);   // row j0
    float c_m = rm1.cc;
    for (int r = 0; r < rows; r++) {
        const int j = j0 + r;
        if (j >= g.ny) break;  // uniform over the warp
        const Row r2 = make(take(j + 2));  // row j+2, with row j's own-cell loads
        const float f_1 = fval(r0, r1, r2);
        const float fl = ps_up(f_0), fr = ps_dn(f_0);
        const float cl = ps_up(r0.cc), cr = ps_dn(r0.cc);
        if (own_col) {
            const float mask = r0.he >= H_DISP_MIN ? 1.f : 0.f;
            float2 av;
            av.x = mask * (r0.he * r0.v.x - (fr - fl) * g.ix);
            av.y = mask * (r0.he * r0.v.y - (f_1 - f_m) * g.iy);
            out(j * g.pitch + i, i, j, r0, av, cl, cr, c_m, r1.cc, own_cur);
        }
        c_m = r0.cc;
        r0 = r1;
        r1 = r2;
        f_m = f_0;
        f_0 = f_1;
    }
    if constexpr (PS_DEPTH > 0) cp_async_wait<0>();  // the rows started past the strip's end copy nothing
}

// The initial sweep's loads: the warm start, c, heff; the right-hand side on own cells.
struct PsInitRaw {
    float2 w, b;
    float cc, he, sy;
};
struct PsInitRow {
    float2 v, b;
    float cc, he;
};
// A CG sweep's loads: r, q = A u and the previous s of the read bank, the inverse diagonal, c,
// heff; p and w on own cells (k: their index, -1 elsewhere). An own cell's new p, w, s and r do
// not depend on the product, so they are written, and <r, u>, <r, r> added, as its row enters
// the window; the window keeps only u (signed), c and heff.
struct PsCgRaw {
    float2 r, q, s, d, p, x;
    float cc, he, sy;
    int k;
};
struct PsCgRow {
    float2 v;
    float cc, he;
};
// Ring fields per row of the solve's sweeps (the CG sweep's; the initial sweep's fit).
constexpr int PS_NF2 = 6, PS_NF1 = 2;
constexpr int PS_SMEM = PS_WARPS * ps_ring_bytes<PS_NF2, PS_NF1>();  // dynamic shared memory per block

// The solve and the stage epilogue by the `ncta` CTAs (this one is number `cta`) of the launch;
// returns false if a bounded wait expired (every CTA then returns).
__device__ __forceinline__ bool pcg_solve_stream(const PcgArgs& a, int cta, int ncta, unsigned& epoch) {
    __shared__ double red[100];
    __shared__ float s_rate[PS_NT / 32];
    __shared__ int s_nan;

    Ctl* ctl = a.ctl;
    const DevGrid& g = a.g;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int rows = a.strip_rows;
    const int nstrips = ps_strips(g.nx, g.ny, rows);
    const int gw = cta * PS_WARPS + warp, nw = ncta * PS_WARPS;
    const double dt = ctl->dt;
    const float dt_f = (float)dt;
    const int lane_i = tid & 31;
    double tot[3];
    if (tid == 0) s_nan = 0;
    __syncthreads();

    long long it = 0;
    bool converged = false;
    // w takes the iterations' steps alpha p in pairs (odd sweeps add their own and the even sweep's
    // before them): after an odd number of iterations the last step is still to be added.
    bool w_pending = false;
    float alpha_last = 0.f;
    if (a.fcg && a.fcg->converged) {  // solved by the learned flexible CG: finish only
        converged = true;
    } else {  // the Jacobi solve; after a learned solve that failed, from where that one stopped
        // ---- initial residual: r = b - A w with the masked warm start (dispersion.rs:480-515)
        double bb = 0.0, rr_p = 0.0;
        for (int st = gw; st < nstrips; st += nw) {
            const int strips_x = (g.nx + PS_OUT - 1) / PS_OUT;
            const int i_lane = (st % strips_x) * PS_OUT - PS_HALO + lane_i;
            const float sx = ((unsigned)i_lane < (unsigned)g.nx) ? 1.f : -1.f;
            ps_strip<PsInitRaw, PsInitRow, PS_NF2, PS_NF1>(
                g, st, rows,
                [&](const auto& ld, int k, float sy, int, bool own, int, int) {
                    PsInitRaw r;
                    r.w = ld.ld2(0, a.w + k, true);
                    r.b = ld.ld2(1, a.bv + k, own);
                    r.cc = ld.ld1(0, a.cc + k, true);
                    r.he = ld.ld1(1, a.heff + k, true);
                    r.sy = sy;
                    return r;
                },
                [&](const PsInitRaw& r) {
                    PsInitRow o;
                    const float2 v = r.he >= H_DISP_MIN ? r.w : make_float2(0.f, 0.f);
                    o.v = make_float2(v.x * sx, v.y * r.sy);
                    o.b = r.b;
                    o.cc = r.cc;
                    o.he = r.he;
                    return o;
                },
                [&](int k, int, int, const PsInitRow& row, float2 aw, float cl, float cr, float cb, float ca,
                    PsNoOwn) {
                    float2 d = make_float2(1.f, 1.f);
                    if (row.he >= H_DISP_MIN) {
                        d.x = row.he + (cr + cl) * 0.25f / (g.dx * g.dx);
                        d.y = row.he + (ca + cb) * 0.25f / (g.dy * g.dy);
                    }
                    const float2 b = row.b;
                    const float2 r = make_float2(b.x - aw.x, b.y - aw.y);
                    a.w[k] = row.v;  // the warm start, masked (own cells carry no sign flip)
                    a.diag[k] = make_float2(1.f / d.x, 1.f / d.y);
                    a.r[k] = r;
                    bb += (double)b.x * b.x + (double)b.y * b.y;
                    rr_p += (double)r.x * r.x + (double)r.y * r.y;
                });
        }
        if (!reduce_barrier<PS_NT>(a, epoch, bb, 0.0, rr_p, tot, red, cta, ncta)) return false;
        const double target = a.tol * sqrt(tot[0]) + 1e-10;
        converged = sqrt(tot[2]) <= target;
        // ---- single-reduction CG (see pcg.cuh): with u = r / diag and q = A u, one sweep per
        // iteration does p = u + beta p, s = q + beta s, r -= alpha s, u = r / diag, q = A u and the
        // three dots <r, u>, <u, q>, <r, r>, and every second sweep w += alpha' p' + alpha p (the
        // steps of the sweep before and its own: w is read and written half as often); sweep
        // k = -1 only forms q0 = A u0.
        double gamma = 0.0, delta = 0.0, alpha_prev = 1.0, beta = 0.0;
        auto cg_sweep = [&](int kk, float alpha_f, float beta_f, float alpha_prev_f, double* dots) -> bool {
            const bool init = kk < 0;
            const bool first = kk == 0;
            const bool w_step = !init && (kk & 1);  // w takes this and the previous iteration's steps
            const int rb = init ? 0 : (kk & 1), wb = init ? 0 : ((kk + 1) & 1);
            double g1 = 0.0, g2 = 0.0, g3 = 0.0;
            for (int st = gw; st < nstrips; st += nw) {
                const int strips_x = (g.nx + PS_OUT - 1) / PS_OUT;
                const int i_lane = (st % strips_x) * PS_OUT - PS_HALO + lane_i;
                const float sx = ((unsigned)i_lane < (unsigned)g.nx) ? 1.f : -1.f;
                ps_strip<PsCgRaw, PsCgRow, PS_NF2, PS_NF1>(
                    g, st, rows,
                    [&](const auto& ld, int k, float sy, int, bool own, int, int) {
                        PsCgRaw r;
                        r.r = ld.ld2(0, a.rb[rb] + k, true);
                        r.d = ld.ld2(1, a.diag + k, true);
                        r.q = ld.ld2(2, a.qb[rb] + k, !init);
                        r.s = ld.ld2(3, a.sb[rb] + k, !init && !first);
                        r.x = ld.ld2(4, a.w + k, w_step && own);
                        r.p = ld.ld2(5, a.p0 + k, !init && !first && own);
                        r.cc = ld.ld1(0, a.cc + k, true);
                        r.he = ld.ld1(1, a.heff + k, true);
                        r.sy = sy;
                        r.k = own ? k : -1;
                        return r;
                    },
                    [&](const PsCgRaw& r) {
                        float2 rn = r.r;
                        if (!init) {
                            float2 sk = r.q;
                            if (!first) {
                                sk.x += beta_f * r.s.x;
                                sk.y += beta_f * r.s.y;
                            }
                            rn = make_float2(r.r.x - alpha_f * sk.x, r.r.y - alpha_f * sk.y);
                            if (r.k >= 0) {
                                float2 pk = make_float2(r.r.x * r.d.x, r.r.y * r.d.y);  // the old u
                                if (!first) {
                                    pk.x += beta_f * r.p.x;
                                    pk.y += beta_f * r.p.y;
                                }
                                a.p0[r.k] = pk;
                                if (w_step)
                                    a.w[r.k] = make_float2(r.x.x + (alpha_prev_f * r.p.x + alpha_f * pk.x),
                                                           r.x.y + (alpha_prev_f * r.p.y + alpha_f * pk.y));
                                a.sb[wb][r.k] = sk;
                                a.rb[wb][r.k] = rn;
                            }
                        }
                        const float2 u = make_float2(rn.x * r.d.x, rn.y * r.d.y);
                        if (r.k >= 0) {
                            g1 += (double)rn.x * u.x + (double)rn.y * u.y;
                            g3 += (double)rn.x * rn.x + (double)rn.y * rn.y;
                        }
                        PsCgRow o;
                        o.v = make_float2(u.x * sx, u.y * r.sy);
                        o.cc = r.cc;
                        o.he = r.he;
                        return o;
                    },
                    [&](int k, int, int, const PsCgRow& row, float2 q, float, float, float, float, PsNoOwn) {
                        const float2 u = row.v;  // own cells: no sign flip
                        a.qb[wb][k] = q;
                        g2 += (double)u.x * q.x + (double)u.y * q.y;
                    });
            }
            return reduce_barrier<PS_NT>(a, epoch, g1, g2, g3, dots, red, cta, ncta);
        };
        if (!converged) {
            if (!cg_sweep(-1, 0.f, 0.f, 0.f, tot)) return false;
            gamma = tot[0];
            delta = tot[1];
        }
        while (!converged && it < a.max_iter) {
            const double alpha = it == 0 ? gamma / delta : gamma / (delta - beta * gamma / alpha_prev);
            if (!cg_sweep((int)it, (float)alpha, (float)beta, (float)alpha_prev, tot)) return false;
            it += 1;
            converged = sqrt(tot[2]) <= target;
            beta = tot[0] / gamma;
            gamma = tot[0];
            delta = tot[1];
            alpha_prev = alpha;
        }
        w_pending = (it & 1) != 0;
        alpha_last = (float)alpha_prev;
    }
    if (a.fcg) it += a.fcg->iterations;
    if (cta == 0 && tid == 0) {
        if (a.fcg) ctl->fcg_iterations += (unsigned long long)a.fcg->iterations;
        ctl->solves += 1;
        ctl->iterations += (unsigned long long)it;
        if (!converged) ctl->unconverged += 1;
        ctl->last_iterations = (int)it;
    }

    // ---- finish the stage from the solution (every w and p is final: the last reduction was a
    // barrier); a pending step of w is added here and w kept as the next solve's warm start
    float rmax = 0.f;
    int nan_here = 0;
    const long long ncell = (long long)g.nx * g.ny;
    for (long long c = (long long)cta * PS_NT + tid; c < ncell; c += (long long)ncta * PS_NT) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const int k = j * g.pitch + i;
        const float2 hn = __ldg(a.hn + k);
        const float2 pr = __ldg(a.pred + k);
        float2 w = __ldcg(a.w + k);
        if (w_pending) {
            const float2 pk = __ldcg(a.p0 + k);
            w = make_float2(w.x + alpha_last * pk.x, w.y + alpha_last * pk.y);
            a.w[k] = w;
        }
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
            for (int w = 0; w < PS_NT / 32; w++) m = fmaxf(m, s_rate[w]);
            s_rate[0] = m;
        }
        __syncthreads();
        fold_rate_and_finish(ctl, s_rate[0], s_nan, (unsigned)ncta);
    }
    return true;
}

__global__ void __launch_bounds__(PS_NT, PS_MINB) pcg_stream_kernel(PcgArgs a) {
    if (!a.ctl->active) return;
    unsigned epoch = 0;
    pcg_solve_stream(a, blockIdx.x, gridDim.x, epoch);
}

}  // namespace wcb
