// stage.cuh — the fused RK-stage stencil kernel.
//
// One CTA advances a TX x TY tile of interior cells through one stage of SSP-RK2:
//   P1  the tile plus a 4-cell halo of (h, hu, hv, b) is staged in shared memory, ghost cells
//       synthesised by the boundary rule as they are loaded; in stage_tma_kernel a tile whose
//       box holds no ghost cell is brought in by two TMA box loads (state and bed) instead;
//   P2  the breaking switch phi (dispersion.rs:113-160) on the tile plus 3 cells;
//   P2b (dispersive runs) masked velocities, their divergence, c = phi h^3/3 and c N
//       (dispersion.rs:380-438) on the tile plus 1-2 cells;
//   P3  every cell's reconstruction, once per axis (solver.rs:140-183; the reference redoes
//       each cell's reconstruction three times per axis, solver.rs:229-233);
//   P4  every face's hydrostatic reconstruction and HLL flux, once (solver.rs:185-226);
//   P5  per cell: rates, wave-maker source, the update, clean_dry, and for the last stage the
//       RK2 average, sponge, friction and the CFL rate (solver.rs:481-616).
//
// Precision. The state is FP32 except the depth, which is compensated (hi + lo, ~48 bits) so
// that mass is conserved to ~1e-15 relative: each face's mass flux is scaled by dt/dx once, in
// FP32, and both cells beside the face add the same value in FP64, so the sum over cells
// telescopes. The surface eta = h_hi + b is reconstructed; still water has eta bitwise
// constant, and the momentum update is written in the well-balanced form
//   -(R_L(high face) - R_R(low face))/dx - g/2 (h_hi + h_lo)(eta_hi - eta_lo)/dx
// where R = (HLL flux) - g/2 h*^2 is the flux less its hydrostatic part and the second term is the
// reference's face pressures plus its centred bed source (solver.rs:229-239, :700-711)
// combined; algebraically identical, it is exactly zero for a lake at rest.
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace wcb {

constexpr int ST_TX = 32, ST_HALO = 4, ST_BX = ST_TX + 2 * ST_HALO;
constexpr int ST_TY = 8;   // tile height of the standalone stage kernel (measured best of 4, 8, 16)
constexpr int ST_NT = 256; // its block size

// Tile geometry for a TX x TY tile (TX = 32) with an H-cell halo (4 for the fifth order and the
// dispersive coefficients, 2 suffices for second order) and the shared-memory layout of one tile,
// in floats.
template <int TY, int H = ST_HALO>
struct StageGeom {
    static constexpr int HALO = H, BX = ST_TX + 2 * H;
    static constexpr int BY = TY + 2 * H, NB = BX * BY;
    static constexpr int SX_W = ST_TX + 2, SX_N = SX_W * TY;   // x reconstructions: cx in [-1, TX]
    static constexpr int SY_H = TY + 2, SY_N = ST_TX * SY_H;   // y reconstructions: cy in [-1, TY]
    static constexpr int FX_W = ST_TX + 1, FX_N = FX_W * TY;   // x faces
    static constexpr int FY_H = TY + 1, FY_N = ST_TX * FY_H;   // y faces
    static constexpr int DV_W = ST_TX + 4, DV_H = TY + 4, DV_N = DV_W * DV_H;  // div on [-2, T+2)
    static constexpr int CF_W = ST_TX + 2, CF_H = TY + 2, CF_N = CF_W * CF_H;  // c, cN on [-1, T+1)
    static constexpr int OWN = ST_TX * TY;
    static constexpr int OFF_ETA = 0, OFF_H = NB, OFF_U = 2 * NB, OFF_V = 3 * NB, OFF_B = 4 * NB;
    static constexpr int OFF_PHI = 5 * NB;
    static constexpr int OFF_SX = 6 * NB;             // 8 arrays of SX_N
    static constexpr int OFF_SY = OFF_SX + 8 * SX_N;  // 8 arrays of SY_N
    static constexpr int OFF_P = OFF_SY + 8 * SY_N;   // Px, Py: 2 * OWN
    static constexpr int OFF_DIV = OFF_P + 2 * OWN;   // dispersive runs only
    static constexpr int OFF_C = OFF_DIV + DV_N;
    static constexpr int OFF_F = OFF_C + CF_N;
    static constexpr int SMEM_SWE = OFF_DIV * 4;
    static constexpr int SMEM_SGN = (OFF_F + CF_N) * 4;
    // Face fluxes reuse the box (dead after P3; the phi slot too, read only in P3): 4 arrays of
    // FX_N, then 4 of FY_N.
    static constexpr int OFF_FX = 0, OFF_FY = 4 * FX_N;
    static_assert(4 * FX_N + 4 * FY_N <= 6 * NB, "face arrays must fit in the box");
};

// The halo a stage variant needs.
template <int ORDER, bool SGN>
constexpr int stage_halo() { return (ORDER == 2 || SGN) ? ST_HALO : 2; }

constexpr int SMEM_SWE = StageGeom<ST_TY>::SMEM_SWE;                // fifth order
constexpr int SMEM_SWE2 = StageGeom<ST_TY, 2>::SMEM_SWE;            // first and second order
constexpr int SMEM_SGN = StageGeom<ST_TY>::SMEM_SGN;

enum StageMode { MODE_STAGE1 = 0, MODE_STAGE2 = 1, MODE_FIRST = 2 };

struct MakerDev {
    int on;
    double omega, ramp_time;
    const float* prof;   // strength * Gaussian profile per column (0 where below 1e-12)
    const float2* ycs;   // (cos k_y y, sin k_y y) per row
};

struct StageArgs {
    DevGrid g;
    const float4* qin;    // state read with halo
    const float4* qold;   // s^n, for the RK2 average (stage 2)
    float4* qout;         // state written (SWE)
    const float* bed;
    const uint8_t* shallow;  // held cells (interior, pitch) or null
    const double* mem;       // breaking memory of followed fronts (interior, pitch) or null
    BreakingDev br;
    MakerDev maker;
    DampParams damp;
    Ctl* ctl;
    int stage_time_plus_dt;  // the maker is evaluated at t + dt in stage 2 (solver.rs:489-491)
    int nonlinear;
    // dispersive outputs
    float2* hn;    // depth after the mass update (hi, lo)
    float2* pred;  // momentum predictor: hu + dt*(u lh) on dispersive cells, hu + dt*lhu elsewhere
    float* cc;     // c = phi h^3 / 3
    float* heff;   // max(h, H_DRY)
    float2* bv;    // right-hand side of the SGN system
};

struct Side {
    float eta, un, ut, z, h;
};

// solver.rs:102-116, without branches: the smallest of three positive slopes, the largest of
// three negative ones, else zero (a zero or mixed-sign triple has min <= 0 <= max).
__device__ __forceinline__ float minmod3(float a, float b, float c) {
    const float mn = fminf(fminf(a, b), c), mx = fmaxf(fmaxf(a, b), c);
    return mn > 0.f ? mn : (mx < 0.f ? mx : 0.f);
}

// solver.rs:118-138, as offsets from the centre value: the reference's
// (2 v0 - 13 v1 + 47 c + 27 v3 - 3 v4)/60 is c + (2(v0-c) - 13(v1-c) + 27(v3-c) - 3(v4-c))/60
// because the weights sum to 60; a flat field gives exactly c at both faces.
// The MC slope s = minmod(2 dl, (dl + dh)/2, 2 dh) enters only as s/2, which is
// minmod(dl, (dl + dh)/4, dh): scaling by powers of two is exact, so this is the same value
// unless (dl + dh)/4 falls below the normal range (differences of 1e-42 in momenta near zero).
__device__ __forceinline__ void face_values(float v0, float v1, float c, float v3, float v4,
                                            float blend, float& lo, float& hi) {
    const float dl = c - v1, dh = v3 - c;
    float mhi = minmod3(dl, 0.25f * (dl + dh), dh);
    float mlo = -mhi;
    if (blend > 0.f) {
        const float a0 = v0 - c, a1 = -dl, a3 = dh, a4 = v4 - c;
        const float fh = (2.f * a0 - 13.f * a1 + 27.f * a3 - 3.f * a4) * (1.f / 60.f);
        const float fl = (2.f * a4 - 13.f * a3 + 27.f * a1 - 3.f * a0) * (1.f / 60.f);
        mlo = mlo + blend * (fl - mlo);
        mhi = mhi + blend * (fh - mhi);
    }
    lo = c + mlo;
    hi = c + mhi;
}

// solver.rs:140-183 for the cell at shared index p, stencil stride s. Writes both face sides and
// the cell's combined pressure + bed-source term P = g/2 (h_hi + h_lo)(eta_hi - eta_lo).
template <int ORDER, typename Gm>
__device__ __forceinline__ void reconstruct(const float* __restrict__ sm, int p, int s,
                                            bool x_axis, Side& lo, Side& hi, float& P) {
    const float* eta = sm + Gm::OFF_ETA;
    const float* hh = sm + Gm::OFF_H;
    const float* un = sm + (x_axis ? Gm::OFF_U : Gm::OFF_V);
    const float* ut = sm + (x_axis ? Gm::OFF_V : Gm::OFF_U);
    const float* bb = sm + Gm::OFF_B;
    const float* phi = sm + Gm::OFF_PHI;
    const float hc = hh[p];
    Side first;
    first.eta = eta[p];
    first.un = un[p];
    first.ut = ut[p];
    first.z = bb[p];
    first.h = hc;
    if (ORDER == 0 || hh[p - s] < H_SECOND || hc < H_SECOND || hh[p + s] < H_SECOND) {
        lo = first;
        hi = first;
        P = 0.f;
        return;
    }
    float blend = 0.f;
    if (ORDER == 2 && hh[p - 2 * s] >= H_SECOND && hh[p + 2 * s] >= H_SECOND) {
        blend = fminf(1.f, phi[p - 2 * s]);
        blend = fminf(blend, phi[p - s]);
        blend = fminf(blend, phi[p]);
        blend = fminf(blend, phi[p + s]);
        blend = fminf(blend, phi[p + 2 * s]);
    }
    float elo, ehi, ulo, uhi, tlo, thi;
    // The outer stencil points are read only by the fifth order (blend > 0), and only its tiles
    // carry the halo that holds them.
    const int s2 = ORDER == 2 ? 2 * s : s;
    face_values(eta[p - s2], eta[p - s], eta[p], eta[p + s], eta[p + s2], blend, elo, ehi);
    face_values(un[p - s2], un[p - s], un[p], un[p + s], un[p + s2], blend, ulo, uhi);
    face_values(ut[p - s2], ut[p - s], ut[p], ut[p + s], ut[p + s2], blend, tlo, thi);
    const float sz = 0.25f * (bb[p + s] - bb[p - s]);
    const float zlo = bb[p] - sz, zhi = bb[p] + sz;
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

// solver.rs:185-226 in remainder form. Outputs the mass flux F0, the tangential flux F2, and the
// normal-momentum flux less the hydrostatic part of each side, R_L = F1 - g/2 hl*^2 and
// R_R = F1 - g/2 hr*^2; each equals the reference's F1 (+ its corr_left/corr_right) minus the
// side's g/2 h^2, which the cell update adds back through P. Equal states give exactly zero
// dissipation, so still water gives exactly zero flux.
__device__ __forceinline__ void hll_face(const Side& l, const Side& r, float& F0, float& RL,
                                         float& RR, float& F2) {
    const float zs = fmaxf(l.z, r.z);
    const float hl = fmaxf(l.eta - zs, 0.f);
    const float hr = fmaxf(r.eta - zs, 0.f);
    if (hl <= H_DRY && hr <= H_DRY) {
        F0 = 0.f;
        F2 = 0.f;
        RL = -0.5f * G * hl * hl;
        RR = -0.5f * G * hr * hr;
        return;
    }
    const float cl = sqrt_approx(G * hl), cr = sqrt_approx(G * hr);
    const float sl = fminf(l.un - cl, r.un - cr);
    const float sr = fmaxf(l.un + cl, r.un + cr);
    const float ql = hl * l.un, qr = hr * r.un;   // mass flux = normal momentum
    const float ml = ql * l.un, mr = qr * r.un;   // advective normal-momentum flux
    const float tl = ql * l.ut, tr = qr * r.ut;   // tangential-momentum flux
    const float dp = 0.5f * G * (hr - hl) * (hr + hl);  // jump of the hydrostatic flux
    if (sl >= 0.f) {
        F0 = ql; F2 = tl; RL = ml; RR = ml - dp;
    } else if (sr <= 0.f) {
        F0 = qr; F2 = tr; RR = mr; RL = mr + dp;
    } else {
        const float inv = __fdividef(1.f, sr - sl);
        const float du0 = hr - hl, du1 = qr - ql, du2 = hr * r.ut - hl * l.ut;
        const float df0 = qr - ql, df1 = (mr - ml) + dp, df2 = tr - tl;
        F0 = ql + sl * (sr * du0 - df0) * inv;
        F2 = tl + sl * (sr * du2 - df2) * inv;
        RL = ml + sl * (sr * du1 - df1) * inv;
        RR = mr + sr * (sl * du1 - df1) * inv;
    }
}

// Shared scalars of one tile's work.
struct StageShared {
    float maker[2];
    unsigned long long bar;  // the TMA box loads' mbarrier
};

// The TMA boxes of a tile with a 4-cell halo: the state (4 floats per cell) and the bed, both
// BX x BY cells, landed in the reconstruction arrays' space (unused until P3).
template <typename Gm>
struct StageTma {
    static constexpr int OFF_RQ = Gm::OFF_SX;              // float4 per box cell
    static constexpr int OFF_RB = Gm::OFF_SX + 4 * Gm::NB; // float per box cell
    static constexpr unsigned BYTES = 5u * 4u * Gm::NB;
    static_assert(5 * Gm::NB <= 8 * Gm::SX_N + 8 * Gm::SY_N, "the boxes must fit before OFF_P");
    static_assert((OFF_RQ * 4) % 128 == 0 && (OFF_RB * 4) % 128 == 0, "TMA destinations are 128-byte aligned");
    static_assert(Gm::HALO % 4 == 0, "a box starts at a column that is a multiple of 4 (16 bytes of bed)");
};
constexpr unsigned long long ST_TMA_WAIT_NS = 100000000ull;  // 0.1 s: a 13 KB box takes microseconds

// One RK stage on the TX x TY tile at (i0, j0), by a block of NT threads, in the dynamic shared
// memory `sm`. Finishing shallow-water stages fold the tile's CFL rate into rmax / nan_here.
// With TMA (one tile per CTA, 4-cell halo, `sm` 128-byte aligned), a tile whose box lies inside
// the grid is staged by the copy engine from the tensor maps tq (the state as 4 floats per cell)
// and tb (the bed); other tiles gather as without.
template <int MODE, int ORDER, bool SGN, int TY, int NT, bool TMA = false>
__device__ __forceinline__ void stage_tile(const StageArgs& a, int i0, int j0, float* sm,
                                           StageShared& ss, float& rmax, int& nan_here,
                                           const CUtensorMap* tq = nullptr,
                                           const CUtensorMap* tb = nullptr) {
    using Gm = StageGeom<TY, stage_halo<ORDER, SGN>()>;
    constexpr int ST_BX = Gm::BX, ST_BY = Gm::BY, ST_NB = Gm::NB, ST_HALO = Gm::HALO;
    constexpr int SX_W = Gm::SX_W, SX_N = Gm::SX_N, SY_N = Gm::SY_N, FX_W = Gm::FX_W;
    constexpr int FX_N = Gm::FX_N, FY_N = Gm::FY_N, DV_W = Gm::DV_W, DV_N = Gm::DV_N;
    constexpr int CF_W = Gm::CF_W, CF_N = Gm::CF_N, OWN = Gm::OWN;
    constexpr int OFF_ETA = Gm::OFF_ETA, OFF_H = Gm::OFF_H, OFF_U = Gm::OFF_U, OFF_V = Gm::OFF_V;
    constexpr int OFF_B = Gm::OFF_B, OFF_PHI = Gm::OFF_PHI, OFF_SX = Gm::OFF_SX, OFF_SY = Gm::OFF_SY;
    constexpr int OFF_P = Gm::OFF_P, OFF_DIV = Gm::OFF_DIV, OFF_C = Gm::OFF_C, OFF_F = Gm::OFF_F;
    constexpr int OFF_FX = Gm::OFF_FX, OFF_FY = Gm::OFF_FY;
    constexpr int ST_TY_ = TY;
    const Ctl* ctl = a.ctl;
    const DevGrid& g = a.g;
    const int tid = threadIdx.x;
    float* s_maker = ss.maker;
    const double dt = ctl->dt;
    const float dt_f = (float)dt;
    const float dtdx = (float)(dt / g.dxd), dtdy = (float)(dt / g.dyd);

    bool boxed = false;  // this tile's box comes by TMA
    if constexpr (TMA) {
        boxed = i0 >= ST_HALO && i0 + ST_TX + ST_HALO <= g.nx && j0 >= ST_HALO &&
                j0 + ST_TY_ + ST_HALO <= g.ny && (smem_addr(sm) & 127u) == 0;
        if (boxed && tid == 0) mbar_init(&ss.bar, 1);
    }
    __syncthreads();  // the previous tile's shared memory is free
    if (tid == 0) {
        if constexpr (TMA) {
            if (boxed) {
                using Tm = StageTma<Gm>;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_expect_tx(&ss.bar, Tm::BYTES);
                tma_load_2d(sm + Tm::OFF_RQ, tq, 4 * (i0 - ST_HALO), j0 - ST_HALO, &ss.bar);
                tma_load_2d(sm + Tm::OFF_RB, tb, i0 - ST_HALO, j0 - ST_HALO, &ss.bar);
            }
        }
        if (a.maker.on) {
            // forcing.rs:124-138 split as profile(x) * ramp(t) * (sin wt cos k_y y - cos wt sin k_y y)
            const double t = ctl->t + (a.stage_time_plus_dt ? dt : 0.0);
            const double ramp = t >= a.maker.ramp_time
                                    ? 1.0
                                    : 0.5 * (1.0 - cos(3.141592653589793 * t / a.maker.ramp_time));
            s_maker[0] = (float)(ramp * sin(a.maker.omega * t));
            s_maker[1] = (float)(ramp * cos(a.maker.omega * t));
        }
    }

    // ---- P1: the box with ghost cells synthesised ------------------------------------------
    if constexpr (TMA) {
        if (boxed) {
            using Tm = StageTma<Gm>;
            if (!mbar_wait_bounded(&ss.bar, 0, ST_TMA_WAIT_NS)) {
                atomicOr(&a.ctl->error, ERR_TMA);
                mbar_wait_bounded(&ss.bar, 0, ST_TMA_WAIT_NS);  // let a late copy land first
            }
            const float4* rq = reinterpret_cast<const float4*>(sm + Tm::OFF_RQ);
            const float* rb = sm + Tm::OFF_RB;
            for (int p = tid; p < ST_NB; p += NT) {
                const float4 q = rq[p];
                const float b = rb[p];
                const float h = q.x;
                sm[OFF_H + p] = h;
                sm[OFF_B + p] = b;
                sm[OFF_ETA + p] = h + b;
                sm[OFF_U + p] = velocity(h, q.z);
                sm[OFF_V + p] = velocity(h, q.w);
            }
        }
    }
    for (int p = tid; p < ST_NB && !boxed; p += NT) {
        const int bx = p % ST_BX, by = p / ST_BX;
        const Mapped m = map_cell(g, i0 - ST_HALO + bx, j0 - ST_HALO + by);
        const float4 q = __ldg(a.qin + m.k);
        const float b = __ldg(a.bed + m.k);
        const float h = q.x;
        sm[OFF_H + p] = h;
        sm[OFF_B + p] = b;
        sm[OFF_ETA + p] = h + b;
        sm[OFF_U + p] = velocity(h, q.z * m.sx);
        sm[OFF_V + p] = velocity(h, q.w * m.sy);
    }
    __syncthreads();

    // ---- P2: breaking switch on [-3, T+3) ----------------------------------------------------
    if (ORDER == 2 || SGN) {
        constexpr int W = ST_BX - 2, H = ST_BY - 2;
        for (int w = tid; w < W * H; w += NT) {
            const int bx = 1 + w % W, by = 1 + w / W;
            const int p = by * ST_BX + bx;
            const float h = sm[OFF_H + p];
            float phi = 0.f;
            if (h >= H_DISP_MIN) {
                const float ex = (sm[OFF_ETA + p + 1] - sm[OFF_ETA + p - 1]) * g.ix;
                const float ey = (sm[OFF_ETA + p + ST_BX] - sm[OFF_ETA + p - ST_BX]) * g.iy;
                const float ratio = fmaxf(sm[OFF_ETA + p] / h, 0.f);
                const float off = fmaxf(smoothstep(a.br.er_lo, a.br.er_inv, ratio),
                                        smoothstep(a.br.sl_lo, a.br.sl_inv, hypotf(ex, ey)));
                phi = 1.f - off;
                // a front still breaking, or the water just behind it (dispersion.rs:149-152)
                if (a.mem && a.mem[map_cell(g, i0 - ST_HALO + bx, j0 - ST_HALO + by).k] != 0.0) phi = 0.f;
            }
            if (a.shallow) {
                const Mapped m = map_cell(g, i0 - ST_HALO + bx, j0 - ST_HALO + by);
                if (__ldg(a.shallow + m.k)) phi = 0.f;
            }
            sm[OFF_PHI + p] = phi;
        }
    }
    // ---- P2b: the dispersive system's coefficients (dispersion.rs:380-438) ---------------------
    if (SGN) {
        __syncthreads();
        // div of the masked velocities on [-2, T+2)
        for (int w = tid; w < DV_N; w += NT) {
            const int bx = 2 + w % DV_W, by = 2 + w / DV_W;
            const int p = by * ST_BX + bx;
            auto um = [&](int q) { return sm[OFF_H + q] >= H_DISP_MIN ? sm[OFF_U + q] : 0.f; };
            auto vm = [&](int q) { return sm[OFF_H + q] >= H_DISP_MIN ? sm[OFF_V + q] : 0.f; };
            sm[OFF_DIV + w] = (um(p + 1) - um(p - 1)) * g.ix + (vm(p + ST_BX) - vm(p - ST_BX)) * g.iy;
        }
        __syncthreads();
        // c and c N on [-1, T+1)
        for (int w = tid; w < CF_N; w += NT) {
            const int cx = w % CF_W, cy = w / CF_W;
            const int p = (cy + 3) * ST_BX + (cx + 3);
            const int d = (cy + 1) * DV_W + (cx + 1);
            const float h = sm[OFF_H + p];
            const float coeff = h < H_DISP_MIN ? 0.f : sm[OFF_PHI + p] * h * h * h / 3.f;
            float f = 0.f;
            if (a.nonlinear && coeff > 0.f) {
                const float um = sm[OFF_U + p], vm = sm[OFF_V + p];  // masked: h >= H_DISP_MIN here
                const float dv = sm[OFF_DIV + d];
                const float n = um * (sm[OFF_DIV + d + 1] - sm[OFF_DIV + d - 1]) * g.ix +
                                vm * (sm[OFF_DIV + d + DV_W] - sm[OFF_DIV + d - DV_W]) * g.iy -
                                dv * dv;
                f = coeff * n;
            }
            sm[OFF_C + w] = coeff;
            sm[OFF_F + w] = f;
        }
    }
    __syncthreads();

    // ---- P3: reconstructions, one per cell and axis -------------------------------------------
    for (int w = tid; w < SX_N + SY_N; w += NT) {
        Side lo, hi;
        float P;
        float* side;
        int idx, n;
        if (w < SX_N) {
            const int cx = w % SX_W - 1, cy = w / SX_W;
            const int p = (cy + ST_HALO) * ST_BX + (cx + ST_HALO);
            reconstruct<ORDER, Gm>(sm, p, 1, true, lo, hi, P);
            if (cx >= 0 && cx < ST_TX) sm[OFF_P + cy * ST_TX + cx] = P;
            side = sm + OFF_SX;
            idx = w;
            n = SX_N;
        } else {
            const int v = w - SX_N;
            const int cx = v % ST_TX, cy = v / ST_TX - 1;
            const int p = (cy + ST_HALO) * ST_BX + (cx + ST_HALO);
            reconstruct<ORDER, Gm>(sm, p, ST_BX, false, lo, hi, P);
            if (cy >= 0 && cy < ST_TY_) sm[OFF_P + OWN + cy * ST_TX + cx] = P;
            side = sm + OFF_SY;
            idx = v;
            n = SY_N;
        }
        side[0 * n + idx] = lo.eta;
        side[1 * n + idx] = lo.un;
        side[2 * n + idx] = lo.ut;
        side[3 * n + idx] = lo.z;
        side[4 * n + idx] = hi.eta;
        side[5 * n + idx] = hi.un;
        side[6 * n + idx] = hi.ut;
        side[7 * n + idx] = hi.z;
    }
    __syncthreads();

    // ---- P4: face fluxes, once per face (writes over the dead box) ----------------------------
    for (int w = tid; w < FX_N + FY_N; w += NT) {
        Side l, r;
        float* out;
        int idx, n;
        if (w < FX_N) {
            const int fx = w % FX_W, cy = w / FX_W;
            const float* sx = sm + OFF_SX;
            const int il = cy * SX_W + fx, ir = il + 1;  // hi side of cell fx-1, lo side of cell fx
            l.eta = sx[4 * SX_N + il]; l.un = sx[5 * SX_N + il]; l.ut = sx[6 * SX_N + il]; l.z = sx[7 * SX_N + il];
            r.eta = sx[0 * SX_N + ir]; r.un = sx[1 * SX_N + ir]; r.ut = sx[2 * SX_N + ir]; r.z = sx[3 * SX_N + ir];
            out = sm + OFF_FX;
            idx = w;
            n = FX_N;
        } else {
            const int v = w - FX_N;
            const int cx = v % ST_TX, fy = v / ST_TX;
            const float* sy = sm + OFF_SY;
            const int il = fy * ST_TX + cx, ir = il + ST_TX;
            l.eta = sy[4 * SY_N + il]; l.un = sy[5 * SY_N + il]; l.ut = sy[6 * SY_N + il]; l.z = sy[7 * SY_N + il];
            r.eta = sy[0 * SY_N + ir]; r.un = sy[1 * SY_N + ir]; r.ut = sy[2 * SY_N + ir]; r.z = sy[3 * SY_N + ir];
            out = sm + OFF_FY;
            idx = v;
            n = FY_N;
        }
        float F0, RL, RR, F2;
        hll_face(l, r, F0, RL, RR, F2);
        // A wall face (the domain's x ends; its y ends unless periodic) carries no mass: the
        // mirrored state's HLL mass flux is zero up to rounding, which in FP32 would leak
        // ~1e-12 of the volume per few hundred steps; the reference's FP64 rounding is 1e-16.
        if (w < FX_N) {
            const int gf = i0 + w % FX_W;
            if (gf == 0 || gf == g.nx) F0 = 0.f;
        } else if (!g.periodic) {
            const int gf = j0 + (w - FX_N) / ST_TX;
            if (gf == 0 || gf == g.ny) F0 = 0.f;
        }
        out[0 * n + idx] = F0;
        out[1 * n + idx] = RL;
        out[2 * n + idx] = RR;
        out[3 * n + idx] = F2;
    }
    __syncthreads();

    // ---- P5: per-cell update ------------------------------------------------------------------
    const float* fx = sm + OFF_FX;
    const float* fy = sm + OFF_FY;
    for (int c = tid; c < OWN; c += NT) {
        const int cx = c % ST_TX, cy = c / ST_TX;
        const int i = i0 + cx, j = j0 + cy;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const int xl = cy * FX_W + cx, xh = xl + 1;
        const int yl = cy * ST_TX + cx, yh = yl + ST_TX;
        float maker = 0.f;
        if (a.maker.on) {
            const float2 cs = __ldg(a.maker.ycs + j);
            maker = __ldg(a.maker.prof + i) * (s_maker[0] * cs.x - s_maker[1] * cs.y);
        }
        const float lh = -(fx[xh] - fx[xl]) * g.inv_dx - (fy[yh] - fy[yl]) * g.inv_dy + maker;
        const float lhu = -(fx[FX_N + xh] - fx[2 * FX_N + xl]) * g.inv_dx -
                          sm[OFF_P + c] * g.inv_dx - (fy[3 * FY_N + yh] - fy[3 * FY_N + yl]) * g.inv_dy;
        const float lhv = -(fy[FY_N + yh] - fy[2 * FY_N + yl]) * g.inv_dy -
                          sm[OFF_P + OWN + c] * g.inv_dy - (fx[3 * FX_N + xh] - fx[3 * FX_N + xl]) * g.inv_dx;
        // Mass: each face's dt/dx-scaled flux is rounded once; both neighbours add the same value.
        const double dh = ((double)__fmul_rn(dtdx, fx[xl]) - (double)__fmul_rn(dtdx, fx[xh])) +
                          ((double)__fmul_rn(dtdy, fy[yl]) - (double)__fmul_rn(dtdy, fy[yh])) +
                          dt * (double)maker;
        const float4 q = __ldg(a.qin + k);
        const double h1 = depth64(q) + dh;
        if (SGN) {
            // Outputs for the SGN solve (dispersion.rs:441-490); the state is finished after it.
            const float h = q.x;
            const float u = velocity(h, q.z), v = velocity(h, q.w);
            const int pc = (cy + 1) * CF_W + (cx + 1);
            float2 b, pr;
            if (h >= H_DISP_MIN) {
                b.x = lhu - u * lh + (sm[OFF_F + pc + 1] - sm[OFF_F + pc - 1]) * g.ix;
                b.y = lhv - v * lh + (sm[OFF_F + pc + CF_W] - sm[OFF_F + pc - CF_W]) * g.iy;
                pr.x = q.z + dt_f * (u * lh);
                pr.y = q.w + dt_f * (v * lh);
            } else {
                b.x = 0.f;
                b.y = 0.f;
                pr.x = q.z + dt_f * lhu;
                pr.y = q.w + dt_f * lhv;
            }
            a.hn[k] = pack_depth(h1);
            a.pred[k] = pr;
            a.cc[k] = sm[OFF_C + pc];
            a.heff[k] = fmaxf(h, H_DRY);
            a.bv[k] = b;
        } else {
            double hn = h1;
            float hu = q.z + dt_f * lhu, hv = q.w + dt_f * lhv;
            clean_dry(hn, hu, hv);
            if (MODE == MODE_STAGE1) {
                a.qout[k] = pack_state(hn, hu, hv);
            } else {
                if (MODE == MODE_STAGE2) {
                    // RK2 average over the step (solver.rs:492-501), then clean_dry
                    const float4 q0 = __ldg(a.qold + k);
                    hn = 0.5 * (depth64(q0) + hn);
                    hu = 0.5f * (q0.z + hu);
                    hv = 0.5f * (q0.w + hv);
                    clean_dry(hn, hu, hv);
                }
                damp_cell(a.damp, g, i, j, __ldg(a.bed + k), dt, hn, hu, hv);
                a.qout[k] = pack_state(hn, hu, hv);
                const float r = cfl_rate(g, (float)hn, hu, hv);
                if (r != r) nan_here = 1;
                else rmax = fmaxf(rmax, r);
            }
        }
    }
}

// A finishing shallow-water stage: the block's CFL rate, folded into the device clock.
template <int NT>
__device__ __forceinline__ void stage_fold(Ctl* ctl, float rmax, int nan_here, unsigned nblocks) {
    __shared__ float s_red[NT / 32];
    __shared__ int s_nan;
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    rmax = warp_max(rmax);
    if (nan_here) s_nan = 1;  // every writer stores 1
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = rmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int w = 0; w < NT / 32; w++) m = fmaxf(m, s_red[w]);
        s_red[0] = m;
    }
    __syncthreads();
    fold_rate_and_finish(ctl, s_red[0], s_nan, nblocks);
}

template <int MODE, int ORDER, bool SGN>
__global__ void __launch_bounds__(ST_NT) stage_kernel(StageArgs a) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    __shared__ StageShared ss;
    if (!a.ctl->active) return;
    float rmax = 0.f;
    int nan_here = 0;
    stage_tile<MODE, ORDER, SGN, ST_TY, ST_NT>(a, blockIdx.x * ST_TX, blockIdx.y * ST_TY, sm, ss, rmax, nan_here);
    if (!SGN && MODE != MODE_STAGE1) stage_fold<ST_NT>(a.ctl, rmax, nan_here, gridDim.x * gridDim.y);
}

// The same stage with every interior tile's box staged by TMA (4-cell-halo variants: fifth order
// or dispersive). tq maps the state as {4 * nx, ny} floats with a row stride of 16 * pitch bytes
// and a {4 * BX, BY} box; tb maps the bed as {nx, ny} floats, stride 4 * pitch, box {BX, BY}.
template <int MODE, int ORDER, bool SGN>
__global__ void __launch_bounds__(ST_NT) stage_tma_kernel(StageArgs a, const __grid_constant__ CUtensorMap tq,
                                                         const __grid_constant__ CUtensorMap tb) {
    static_assert(stage_halo<ORDER, SGN>() == ST_HALO, "TMA staging serves the 4-cell halo");
    extern __shared__ __align__(128) float4 smem_tma[];
    float* sm = reinterpret_cast<float*>(smem_tma);
    __shared__ StageShared ss;
    if (!a.ctl->active) return;
    float rmax = 0.f;
    int nan_here = 0;
    stage_tile<MODE, ORDER, SGN, ST_TY, ST_NT, true>(a, blockIdx.x * ST_TX, blockIdx.y * ST_TY, sm, ss, rmax,
                                                     nan_here, &tq, &tb);
    if (!SGN && MODE != MODE_STAGE1) stage_fold<ST_NT>(a.ctl, rmax, nan_here, gridDim.x * gridDim.y);
}

}  // namespace wcb
