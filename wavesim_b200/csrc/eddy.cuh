// eddy.cuh — breaking fronts followed from step to step, and their eddy viscosity.
//
// crates/wavecore/src/eddy.rs, opt-in through `Breaking::viscosity` and only with dispersion
// (solver.rs:509-532). After each step a cell breaks where the switch, read afresh from the
// surface, says the wave breaks while the surface rises (rise = -div(hu), from the mass
// equation), or where the surface rises faster than Kennedy et al.'s threshold for the oldest
// front among it and its four neighbours; it then carries that front's age plus dt. A cell a
// front has left counts down `linger` seconds (negative memory). The memory holds the switch off
// (dispersion.rs:149-152), and breaking cells get the eddy viscosity nu = B (mixing h)^2 rise,
// applied to the momentum in explicit sub-steps (eddy.rs:221-302).
//
// On the device the whole of it is one cooperative launch appended to the step, after the
// kernel that finishes the state:
//   follow   per cell: the new memory (FP64, as the reference's State::breaking), nu (FP64
//            arithmetic, stored FP32) and the momentum copied into a bank; the CTA's largest nu
//            -> one grid barrier that also takes the grid-wide maximum
//   diffuse  n = ceil(dt / limit) sub-steps (eddy.rs:236-243), each reading one momentum bank
//            and writing the other, the last writing the state; a grid barrier between two
//   finish   the new memory replaces the old (every read of the old one was before the first
//            barrier), the CFL rate of the final state and the step's clock.
// Ghost cells are never stored: h, the momentum (sign-flipped at walls) and the memory read at a
// ghost position come from the cell the reference's ghost fill copies (map_cell), while nu is 0
// outside the interior, as the reference's scratch leaves it. The reference's clean_dry after the
// viscosity changes nothing (h is untouched and cells thinner than H_BREAKING_MIN keep their
// momentum), so it is not repeated.
//
// Every wait is bounded in time: on expiry the kernel sets ERR_TIMEOUT and every CTA returns.
#pragma once

#include "common.cuh"

namespace wcb {

constexpr int ED_NT = 256;
constexpr double H_BREAKING_MIN_D = 0.01;  // eddy.rs:54-56
constexpr double BREAKING_ONSET_D = 0.8;   // eddy.rs:58-59
constexpr double H_DISP_MIN_D = 0.05;      // dispersion.rs:41
constexpr int ED_MAX_SUB = 1 << 16;        // more viscous sub-steps than this set ERR_EDDY
constexpr int ERR_EDDY = 4;

// EddyViscosity (eddy.rs:62-90) and the switch's thresholds (dispersion.rs:44-54), FP64.
struct EddyParams {
    double initial, settled, duration, mixing, linger;
    double er_lo, er_hi, sl_lo, sl_hi;
};

struct EddyArgs {
    DevGrid g;
    float4* q;            // the step's finished state; its momentum is updated in place
    const float* bed;
    double* mem;          // breaking memory: seconds a front has broken; < 0 lingering; 0 none
    double* mem_new;
    float* nu;            // eddy viscosity of the step (interior cells)
    float2* mb[2];        // momentum banks of the sub-steps
    double* part;         // [2][ncta] CTA maxima of nu, banked by barrier epoch
    unsigned* cnt;        // [0] arrivals, [1] released epoch; zeroed before each launch
    Ctl* ctl;
    int* sub_out;         // sub-steps taken, or null
    EddyParams e;
    int finish;           // fold the CFL rate and close the step (0: a standalone application)
    unsigned long long timeout_ns;
};

// eddy.rs:114-124
__device__ __forceinline__ double eddy_threshold(const EddyParams& e, double age, double h) {
    const double span = e.duration * sqrt(h / G_D);
    if (age >= span) return e.settled;
    return e.initial + (e.settled - e.initial) * age / span;
}

// dispersion.rs:108-111 in FP64 (Rust's clamp keeps NaN, and so do these comparisons). The
// follow step's arithmetic is written with round-to-nearest intrinsics where a multiply feeds an
// add, so that no FMA contraction separates it from the reference's separately rounded FP64.
__device__ __forceinline__ double smoothstep64(double lo, double hi, double x) {
    double t = (x - lo) / (hi - lo);
    t = t < 0.0 ? 0.0 : t;
    t = t > 1.0 ? 1.0 : t;
    return __dmul_rn(__dmul_rn(t, t), __dsub_rn(3.0, __dmul_rn(2.0, t)));
}

// The depth of a stored cell, read as its own 8 bytes (hi, lo), which share no word with the
// momentum that the last sub-step writes.
__device__ __forceinline__ double depth_at(const float4* q, int k) {
    const float2 d = reinterpret_cast<const float2*>(q + k)[0];
    return (double)d.x + (double)d.y;
}

__device__ __forceinline__ double block_max64(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < ED_NT / 32; w++) m = fmax(m, red[w]);
        red[ED_NT / 32] = m;
    }
    __syncthreads();
    return red[ED_NT / 32];
}

// A grid-wide barrier that also returns the largest of one value per CTA (fmax drops NaN, as
// the reference's row maxima do, par.rs:99-107). Partials alternate between two banks by epoch
// parity: a CTA cannot reach barrier e+2 before every CTA has left barrier e.
__device__ bool eddy_barrier(const EddyArgs& a, unsigned& epoch, double v, double* out, int cta, int ncta,
                             double* red) {
    __shared__ int s_ok;
    v = block_max64(v, red);
    epoch += 1;
    if (threadIdx.x == 0) {
        a.part[(size_t)(epoch & 1u) * ncta + cta] = v;
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
    if (out) {
        double m = 0.0;
        const double* bank = a.part + (size_t)(epoch & 1u) * ncta;
        for (int b = threadIdx.x; b < ncta; b += ED_NT) m = fmax(m, __ldcg(bank + b));
        *out = block_max64(m, red);
    }
    return true;
}

// eddy.rs:155-219 (`follow`) for interior cell (i, j): the new memory and nu. The momentum and
// the old memory of the neighbours come through the ghost rule.
__device__ __forceinline__ void follow_cell(const EddyArgs& a, double dt, int i, int j, int k, double depth,
                                            double& m_new, double& nu) {
    const DevGrid& g = a.g;
    const EddyParams& e = a.e;
    m_new = 0.0;
    nu = 0.0;
    if (depth < H_BREAKING_MIN_D) return;
    const double ix = 0.5 / g.dxd, iy = 0.5 / g.dyd;
    auto hu_at = [&](int di, int dj) {
        const Mapped m = map_cell(g, i + di, j + dj);
        return (double)(a.q[m.k].z * m.sx);
    };
    auto hv_at = [&](int di, int dj) {
        const Mapped m = map_cell(g, i + di, j + dj);
        return (double)(a.q[m.k].w * m.sy);
    };
    const double rise = -__dadd_rn(__dmul_rn(hu_at(1, 0) - hu_at(-1, 0), ix), __dmul_rn(hv_at(0, 1) - hv_at(0, -1), iy));
    // the switch as the surface alone reads it, without the fronts (dispersion.rs:134-148)
    double phi = 0.0;
    if (depth >= H_DISP_MIN_D) {
        auto eta = [&](int di, int dj) {
            const Mapped m = map_cell(g, i + di, j + dj);
            return depth_at(a.q, m.k) + (double)__ldg(a.bed + m.k);
        };
        const double ex = (eta(1, 0) - eta(-1, 0)) * ix;
        const double ey = (eta(0, 1) - eta(0, -1)) * iy;
        const double ratio = fmax(eta(0, 0) / depth, 0.0);
        const double off = fmax(smoothstep64(e.er_lo, e.er_hi, ratio), smoothstep64(e.sl_lo, e.sl_hi, hypot(ex, ey)));
        phi = 1.0 - off;
    }
    auto old_at = [&](int di, int dj) { return __ldcg(a.mem + map_cell(g, i + di, j + dj).k); };
    const double old = __ldcg(a.mem + k);
    double front = fmax(0.0, old);
    front = fmax(front, old_at(-1, 0));
    front = fmax(front, old_at(1, 0));
    front = fmax(front, old_at(0, -1));
    front = fmax(front, old_at(0, 1));
    const double c = sqrt(G_D * depth);
    const bool starts = depth >= H_DISP_MIN_D && 1.0 - phi >= BREAKING_ONSET_D && rise > 0.0;
    const bool goes_on = front > 0.0 && rise > eddy_threshold(e, front, depth) * c;
    const double age = (front > 0.0 && (starts || goes_on)) ? front + dt : (starts ? dt : 0.0);
    if (age > 0.0) {
        double b = rise / (eddy_threshold(e, age, depth) * c) - 1.0;
        b = b < 0.0 ? 0.0 : b;
        b = b > 1.0 ? 1.0 : b;
        m_new = age;
        nu = b * e.mixing * e.mixing * depth * rise;
    } else if (old > 0.0) {
        m_new = -e.linger * sqrt(depth / G_D);
    } else if (old < 0.0) {
        m_new = fmin(old + dt, 0.0);
    }
}

// One explicit viscous sub-step of eddy.rs:252-296 for interior cell (i, j) from momentum bank
// `src`; FP32 arithmetic on the FP32 momentum.
__device__ __forceinline__ float2 diffuse_cell(const EddyArgs& a, const float2* src, int i, int j, int k, float sub,
                                               float idx2, float idy2, float cross) {
    const DevGrid& g = a.g;
    const float2 mk = __ldcg(src + k);
    if (depth_at(a.q, k) < H_BREAKING_MIN_D) return mk;
    struct Nb {
        bool wet;   // at least H_BREAKING_MIN deep
        float nu;   // 0 outside the interior
        float hu, hv;
    };
    auto nb = [&](int di, int dj) {
        const Mapped m = map_cell(g, i + di, j + dj);
        Nb n;
        n.wet = !(depth_at(a.q, m.k) < H_BREAKING_MIN_D);
        const bool inside = (unsigned)(i + di) < (unsigned)g.nx && (unsigned)(j + dj) < (unsigned)g.ny;
        n.nu = inside ? __ldcg(a.nu + m.k) : 0.f;
        const float2 v = __ldcg(src + m.k);
        n.hu = v.x * m.sx;
        n.hv = v.y * m.sy;
        return n;
    };
    const float nk = __ldcg(a.nu + k);
    const Nb e = nb(1, 0), w = nb(-1, 0), n = nb(0, 1), s = nb(0, -1);
    const Nb ne = nb(1, 1), nw = nb(-1, 1), se = nb(1, -1), sw = nb(-1, -1);
    // the viscosity between two cells, none if either is too thin; a cell's own where wet
    auto link = [&](const Nb& o) { return o.wet ? 0.5f * (nk + o.nu) : 0.f; };
    auto wetnu = [&](const Nb& o) { return o.wet ? o.nu : 0.f; };
    const float le = link(e), lw = link(w), ln = link(n), ls = link(s);
    const float xx_u = (le * (e.hu - mk.x) - lw * (mk.x - w.hu)) * idx2;
    const float yy_u = (ln * (n.hu - mk.x) - ls * (mk.x - s.hu)) * idy2;
    const float xx_v = (le * (e.hv - mk.y) - lw * (mk.y - w.hv)) * idx2;
    const float yy_v = (ln * (n.hv - mk.y) - ls * (mk.y - s.hv)) * idy2;
    const float yx_v = (wetnu(n) * (ne.hv - nw.hv) - wetnu(s) * (se.hv - sw.hv)) * cross;
    const float xy_u = (wetnu(e) * (ne.hu - se.hu) - wetnu(w) * (nw.hu - sw.hu)) * cross;
    return make_float2(mk.x + sub * (xx_u + 0.5f * (yy_u + yx_v)), mk.y + sub * (yy_v + 0.5f * (xx_v + xy_u)));
}

__global__ void __launch_bounds__(ED_NT) eddy_kernel(EddyArgs a) {
    __shared__ double red[ED_NT / 32 + 1];
    __shared__ float s_rate[ED_NT / 32];
    __shared__ int s_nan;
    if (!a.ctl->active) return;
    const DevGrid& g = a.g;
    const int cta = blockIdx.x, ncta = gridDim.x, tid = threadIdx.x;
    const long long cells = (long long)g.nx * g.ny;
    const long long stride = (long long)ncta * ED_NT;
    const double dt = a.ctl->dt;
    if (tid == 0) s_nan = 0;
    unsigned epoch = 0;

    // ---- follow
    double local = 0.0;
    for (long long c = (long long)cta * ED_NT + tid; c < cells; c += stride) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx), k = j * g.pitch + i;
        const float4 qc = a.q[k];
        a.mb[0][k] = make_float2(qc.z, qc.w);
        double m_new, nu;
        follow_cell(a, dt, i, j, k, (double)qc.x + (double)qc.y, m_new, nu);
        a.mem_new[k] = m_new;
        a.nu[k] = (float)nu;
        local = fmax(local, nu);
    }
    double top = 0.0;
    if (!eddy_barrier(a, epoch, local, &top, cta, ncta, red)) return;

    // ---- how many sub-steps (eddy.rs:233-246): identical in every CTA
    int n = 0;
    double sub = 0.0;
    const double idx2 = 1.0 / (g.dxd * g.dxd), idy2 = 1.0 / (g.dyd * g.dyd);
    if (top > 0.0 && a.e.mixing > 0.0) {
        const double limit = 0.5 / (top * fmax(2.0 * idx2 + idy2, idx2 + 2.0 * idy2));
        const double fs = fmax(ceil(dt / limit), 1.0);
        if (fs <= (double)ED_MAX_SUB) {
            n = (int)fs;
            sub = dt / (double)n;
        } else if (cta == 0 && tid == 0) {
            atomicOr(&a.ctl->error, ERR_EDDY);
        }
    }
    const float subf = (float)sub, idx2f = (float)idx2, idy2f = (float)idy2;
    const float crossf = (float)(0.25 / (g.dxd * g.dyd));

    // ---- sub-steps; the last (or, with none, a plain pass) writes the state and takes its rate
    float rmax = 0.f;
    int nan_here = 0;
    const int passes = n > 0 ? n : 1;
    for (int st = 0; st < passes; st++) {
        const bool last = st == passes - 1;
        const float2* src = a.mb[st & 1];
        float2* dst = a.mb[(st + 1) & 1];
        for (long long c = (long long)cta * ED_NT + tid; c < cells; c += stride) {
            const int i = (int)(c % g.nx), j = (int)(c / g.nx), k = j * g.pitch + i;
            const float2 out = n > 0 ? diffuse_cell(a, src, i, j, k, subf, idx2f, idy2f, crossf) : __ldcg(src + k);
            if (!last) {
                dst[k] = out;
                continue;
            }
            if (n > 0) reinterpret_cast<float2*>(a.q + k)[1] = out;
            a.mem[k] = __ldcg(a.mem_new + k);
            const float rt = cfl_rate(g, (float)depth_at(a.q, k), out.x, out.y);
            if (rt != rt) nan_here = 1;
            else rmax = fmaxf(rmax, rt);
        }
        if (!last && !eddy_barrier(a, epoch, 0.0, nullptr, cta, ncta, red)) return;
    }
    if (cta == 0 && tid == 0 && a.sub_out) *a.sub_out = n;
    if (!a.finish) return;
    rmax = warp_max(rmax);
    if (nan_here) s_nan = 1;
    if ((tid & 31) == 0) s_rate[tid >> 5] = rmax;
    __syncthreads();
    if (tid == 0) {
        float m = 0.f;
        for (int w = 0; w < ED_NT / 32; w++) m = fmaxf(m, s_rate[w]);
        s_rate[0] = m;
    }
    __syncthreads();
    fold_rate_and_finish(a.ctl, s_rate[0], s_nan, (unsigned)ncta);
}

// A padded FP64 array (the host's breaking memory) -> interior FP64, and back with the ghost
// cells copied by the boundary rule (grid.rs:60-87, no sign change).
__global__ void pack_f64_kernel(DevGrid g, const double* __restrict__ src, double* __restrict__ dst) {
    const int W = g.nx + 6;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)g.nx * g.ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        dst[(long long)j * g.pitch + i] = src[(long long)(j + 3) * W + (i + 3)];
    }
}

__global__ void unpack_f64_kernel(DevGrid g, const double* __restrict__ src, double* __restrict__ dst) {
    const int W = g.nx + 6, R = g.ny + 6;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)W * R;
         c += (long long)gridDim.x * blockDim.x) {
        const int pi = (int)(c % W), pj = (int)(c / W);
        dst[c] = src[map_cell(g, pi - 3, pj - 3).k];
    }
}

}  // namespace wcb
