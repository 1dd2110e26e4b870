// common.cuh — shared device definitions of the B200 wavecore step.
//
// Layout in HBM: every field is stored over the interior cells only, row-major with y outer and
// a row pitch of `pitch` elements (a multiple of 32). Ghost cells are never stored: a load at an
// index outside the interior is redirected to the cell the reference's ghost fill would copy
// (mirrored at walls, wrapped when periodic in y; crates/wavecore/src/grid.rs:60-114,
// state.rs:42-76), with the sign of the wall-normal vector component flipped.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wcb {

// crates/wavecore/src/solver.rs:26-32; dispersion.rs:41; forcing.rs:286
constexpr float G = 9.81f;
constexpr float H_DRY = 1e-8f;
constexpr float H_SECOND = 1e-3f;
constexpr float H_FACE_MIN = 1e-4f;
constexpr float H_DISP_MIN = 0.05f;
constexpr float H_FRICTION_MIN = 1e-3f;
constexpr double G_D = 9.81;
constexpr double H_DRY_D = 1e-8;
constexpr int MAX_SPONGES = 8;

// Error bits in Ctl::error.
constexpr int ERR_TIMEOUT = 1;
constexpr int ERR_NAN = 2;
constexpr int ERR_TMA = 8;  // a stage kernel's TMA box did not arrive within its wait limit

struct DevGrid {
    int nx, ny, pitch, periodic;
    float dx, dy;
    float ix, iy;          // 0.5 / dx, 0.5 / dy (centred differences)
    float inv_dx, inv_dy;  // 1 / dx, 1 / dy
    double dxd, dyd;
};

// Step control, resident on the device so that steps chain without the host.
struct Ctl {
    double t;              // time of the state
    double dt;             // size of the step being taken
    double t_end;          // adaptive stepping stops once t >= t_end
    double cfl;
    double stable_dt;      // cfl / max rate of the last finished state (inf if dry, NaN if NaN)
    unsigned int rate_bits;   // running max of the CFL rate (FP32 bits; non-negative floats order as uints)
    unsigned int nan_seen;
    unsigned int blocks_done;
    int adaptive;
    int active;
    int error;
    unsigned long long steps;
    unsigned long long solves, iterations, unconverged;
    int last_iterations;
    int pad_;
    unsigned long long fcg_iterations;  // of them, learned flexible-CG iterations
};

struct SpongeDev {
    int width;
    float strength, inv_w;
    double level;
    int west, east, south, north;
};

struct DampParams {
    int nsp;
    float manning;
    SpongeDev sp[MAX_SPONGES];
};

__device__ __forceinline__ int reflect_idx(int i, int n) {
    if ((unsigned)i < (unsigned)n) return i;
    const int p = 2 * n;
    int t = i % p;
    if (t < 0) t += p;
    return t < n ? t : p - 1 - t;
}

__device__ __forceinline__ int wrap_idx(int j, int n) {
    if ((unsigned)j < (unsigned)n) return j;
    int t = j % n;
    return t < 0 ? t + n : t;
}

// Scalars of the learned path's flexible CG, kept on the device so that iterations chain
// without the host; `done` stops every later kernel of the solve.
struct FcgScalars {
    double bb, rr, pq, rp, zq, target, alpha, beta;
    int converged, iterations, done, pad_;
};

struct Mapped {
    int k;        // linear index of the source cell
    int i, j;     // its interior coordinates
    float sx, sy; // sign of the x- and y-normal vector components
};

// The stored cell a padded position (i, j) (interior coordinates, may be outside) reads.
__device__ __forceinline__ Mapped map_cell(const DevGrid& g, int i, int j) {
    Mapped m;
    const int mi = reflect_idx(i, g.nx);
    const int mj = g.periodic ? wrap_idx(j, g.ny) : reflect_idx(j, g.ny);
    m.k = mj * g.pitch + mi;
    m.i = mi;
    m.j = mj;
    m.sx = ((unsigned)i < (unsigned)g.nx) ? 1.f : -1.f;
    m.sy = (g.periodic || (unsigned)j < (unsigned)g.ny) ? 1.f : -1.f;
    return m;
}

// The hardware square root (PTX sqrt.approx.f32: a couple of ulps, exact at 0). The wave speeds
// and the CFL rate take it: their FP32 values are already further from the FP64 reference than
// that, and the correctly rounded sqrtf costs several instructions more per call.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// solver.rs:90-92, with the fast single-precision division (two ulps; the FP32 state is already
// further from the FP64 reference than that).
__device__ __forceinline__ float velocity(float h, float hm) { return h > H_DRY ? __fdividef(hm, h) : 0.f; }

// A compensated depth (hi + lo as FP32) widened to FP64, and packed back.
__device__ __forceinline__ double depth64(float4 q) { return (double)q.x + (double)q.y; }
__device__ __forceinline__ float4 pack_state(double h, float hu, float hv) {
    const float hi = (float)h;
    const float lo = (float)(h - (double)hi);
    return make_float4(hi, lo, hu, hv);
}
__device__ __forceinline__ float2 pack_depth(double h) {
    const float hi = (float)h;
    return make_float2(hi, (float)(h - (double)hi));
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile_int(const int* p) { return *(const volatile int*)p; }

// Asynchronous global -> shared copies of 8 and 4 bytes (PTX cp.async): the data in flight holds
// no registers; a thread's own copies are visible to it after cp_async_wait. Both addresses are
// aligned to the copy's size.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's committed groups are still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Sum over the block with a fixed reduction tree; every thread gets the same value.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double x = lane < NT / 32 ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[32] = x;
    }
    __syncthreads();
    return red[32];
}

// Three sums at once.
template <int NT>
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c, double* red) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
        red[warp] = a;
        red[32 + warp] = b;
        red[64 + warp] = c;
    }
    __syncthreads();
    if (warp == 0) {
        double x = lane < NT / 32 ? red[lane] : 0.0;
        double y = lane < NT / 32 ? red[32 + lane] : 0.0;
        double z = lane < NT / 32 ? red[64 + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(0xffffffffu, x, o);
            y += __shfl_down_sync(0xffffffffu, y, o);
            z += __shfl_down_sync(0xffffffffu, z, o);
        }
        if (lane == 0) {
            red[96] = x;
            red[97] = y;
            red[98] = z;
        }
    }
    __syncthreads();
    a = red[96];
    b = red[97];
    c = red[98];
}

// Max of non-negative floats over the block (NaN handled by the caller's flag).
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// dispersion.rs:108-111, with the reciprocal width precomputed.
__device__ __forceinline__ float smoothstep(float lo, float inv_w, float x) {
    float t = (x - lo) * inv_w;
    t = t < 0.f ? 0.f : t;
    t = t > 1.f ? 1.f : t;
    return t * t * (3.f - 2.f * t);
}

struct BreakingDev {
    float er_lo, er_inv, sl_lo, sl_inv;
};

// Sponge rate at interior cell (i, j): forcing.rs:180-206.
__device__ __forceinline__ float sponge_rate(const SpongeDev& sp, const DevGrid& g, int i, int j) {
    float r = 0.f;
    auto ramp = [&](int d) -> float {
        if (d < sp.width) {
            const float f = ((float)sp.width - (float)d) * sp.inv_w;
            return f * f;
        }
        return 0.f;
    };
    if (sp.west) r = fmaxf(r, ramp(i));
    if (sp.east) r = fmaxf(r, ramp(g.nx - 1 - i));
    if (sp.south) r = fmaxf(r, ramp(j));
    if (sp.north) r = fmaxf(r, ramp(g.ny - 1 - j));
    return sp.strength * r;
}

// solver.rs:576-591 on one cell.
__device__ __forceinline__ void clean_dry(double& h, float& hu, float& hv) {
    if (h < H_DRY_D) {
        h = h > 0.0 ? h : 0.0;
        hu = 0.f;
        hv = 0.f;
    }
}

// Sponge relaxation and Manning friction on one interior cell, then clean_dry:
// solver.rs:534-574 with forcing.rs:209-225 and :288-297. The relaxation of the depth is
// written h + (1-f)(ht - h), which equals the reference's f h + (1-f) ht and leaves a cell that
// is already at its target exactly unchanged.
__device__ __forceinline__ void damp_cell(const DampParams& dp, const DevGrid& g, int i, int j,
                                          float bed, double dt, double& h, float& hu, float& hv) {
    for (int m = 0; m < dp.nsp; m++) {
        const float rate = sponge_rate(dp.sp[m], g, i, j);
        if (rate > 0.f) {
            const double f = exp(-(double)rate * dt);
            double ht = dp.sp[m].level - (double)bed;
            ht = ht > 0.0 ? ht : 0.0;
            h = h + (1.0 - f) * (ht - h);
            hu = (float)f * hu;
            hv = (float)f * hv;
        }
    }
    if (dp.manning > 0.f) {
        const float h32 = (float)h;
        if (h32 > H_FRICTION_MIN) {
            // speed = |hu| / h and k = g n^2 h^(-4/3), from the hardware reciprocal, square root,
            // log2 and exp2 (a few ulps; the reference's hypot only guards overflow, which physical
            // momenta cannot reach in FP32)
            const float inv_h = __fdividef(1.f, h32);
            const float speed = sqrt_approx(hu * hu + hv * hv) * inv_h;
            const float k = G * dp.manning * dp.manning * exp2f(-1.3333333f * __log2f(h32));
            const float f = __fdividef(1.f, 1.f + (float)dt * k * speed);
            hu *= f;
            hv *= f;
        }
    }
    clean_dry(h, hu, hv);
}

// CFL rate of one cell: solver.rs:94-100.
__device__ __forceinline__ float cfl_rate(const DevGrid& g, float h, float hu, float hv) {
    const float c = sqrt_approx(G * h);
    const float u = fabsf(velocity(h, hu));
    const float v = fabsf(velocity(h, hv));
    return (u + c) * g.inv_dx + (v + c) * g.inv_dy;
}

// Close a step: called by exactly one thread after every block of the step's last kernel has
// folded its CFL rate into ctl. Advances the clock and, when adaptive, sets the next dt from
// the new state (solver.rs:431-450; the test loop of crates/wavecore/tests/common/mod.rs:53-60).
__device__ __forceinline__ void finish_step(Ctl* ctl) {
    const double t_new = ctl->t + ctl->dt;
    ctl->t = t_new;
    ctl->steps += 1;
    const unsigned bits = atomicExch(&ctl->rate_bits, 0u);
    const unsigned nan = atomicExch(&ctl->nan_seen, 0u);
    ctl->blocks_done = 0;
    const float rate = __uint_as_float(bits);
    double sdt;
    if (nan) sdt = __longlong_as_double(0x7ff8000000000000ll);
    else if (rate > 0.f) sdt = ctl->cfl / (double)rate;
    else sdt = __longlong_as_double(0x7ff0000000000000ll);
    ctl->stable_dt = sdt;
    if (nan) ctl->error |= ERR_NAN;
    if (ctl->adaptive) {
        const double left = ctl->t_end - t_new;
        ctl->dt = sdt < left ? sdt : left;
        if (nan || !(t_new < ctl->t_end)) ctl->active = 0;
    }
}

// Fold this block's rate into ctl and let the last block close the step. No waiting: the
// last block to arrive finishes (the classic threadfence reduction).
__device__ __forceinline__ void fold_rate_and_finish(Ctl* ctl, float block_rate, int block_nan,
                                                     unsigned nblocks) {
    if (threadIdx.x == 0) {
        atomicMax(&ctl->rate_bits, __float_as_uint(block_rate));
        if (block_nan) atomicOr(&ctl->nan_seen, 1u);
        __threadfence();
        const unsigned done = atomicAdd(&ctl->blocks_done, 1u);
        if (done == nblocks - 1) {
            __threadfence();
            finish_step(ctl);
        }
    }
}

}  // namespace wcb
