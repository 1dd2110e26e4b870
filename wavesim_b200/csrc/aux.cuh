// aux.cuh — kernels around the step: state transfer, the time-step limit, the limiting cell,
// the breaking indicator and the FP64 diagnostics.
#pragma once

#include "common.cuh"

namespace wcb {

constexpr int AUX_NT = 256;

// Padded FP64 host layout (width W = nx + 6) -> device state (interior, pitch). Sets the clock.
__global__ void upload_kernel(DevGrid g, const double* __restrict__ h, const double* __restrict__ hu,
                              const double* __restrict__ hv, float4* __restrict__ q) {
    const int W = g.nx + 6;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)g.nx * g.ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const long long s = (long long)(j + 3) * W + (i + 3);
        q[(long long)j * g.pitch + i] = pack_state(h[s], (float)hu[s], (float)hv[s]);
    }
}

// Device state -> padded FP64 host layout, ghost cells filled by the boundary rule.
__global__ void download_kernel(DevGrid g, const float4* __restrict__ q, double* __restrict__ h,
                                double* __restrict__ hu, double* __restrict__ hv) {
    const int W = g.nx + 6, R = g.ny + 6;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)W * R;
         c += (long long)gridDim.x * blockDim.x) {
        const int pi = (int)(c % W), pj = (int)(c / W);
        const Mapped m = map_cell(g, pi - 3, pj - 3);
        const float4 v = q[m.k];
        h[c] = depth64(v);
        hu[c] = (double)(v.z * m.sx);
        hv[c] = (double)(v.w * m.sy);
    }
}

// A padded FP64 array -> interior FP32 (the bed).
__global__ void pack_f32_kernel(DevGrid g, const double* __restrict__ src, float* __restrict__ dst) {
    const int W = g.nx + 6;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)g.nx * g.ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        dst[(long long)j * g.pitch + i] = (float)src[(long long)(j + 3) * W + (i + 3)];
    }
}

__global__ void set_dt_kernel(Ctl* ctl, double dt) {
    ctl->dt = dt;
    ctl->active = 1;
}

__global__ void set_adaptive_kernel(Ctl* ctl, double t_end) {
    ctl->t_end = t_end;
    ctl->adaptive = 1;
    ctl->active = ctl->t < t_end ? 1 : 0;
    const double sdt = ctl->stable_dt;
    const double left = t_end - ctl->t;
    ctl->dt = sdt < left ? sdt : left;
    if (sdt != sdt) ctl->active = 0;
}

__global__ void clear_adaptive_kernel(Ctl* ctl) {
    ctl->adaptive = 0;
    ctl->active = 1;
}

// CFL rate of the device state, folded into ctl; the last block stores ctl->stable_dt without
// advancing the clock (solver.rs:431-450).
__global__ void state_rate_kernel(DevGrid g, const float4* __restrict__ q, Ctl* ctl) {
    __shared__ float s_red[AUX_NT / 32];
    __shared__ int s_nan;
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    float rmax = 0.f;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)g.nx * g.ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const float4 v = q[(long long)j * g.pitch + i];
        const float r = cfl_rate(g, v.x, v.z, v.w);
        if (r != r) s_nan = 1;
        else rmax = fmaxf(rmax, r);
    }
    rmax = warp_max(rmax);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = rmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = 0.f;
        for (int w = 0; w < AUX_NT / 32; w++) m = fmaxf(m, s_red[w]);
        atomicMax(&ctl->rate_bits, __float_as_uint(m));
        if (s_nan) atomicOr(&ctl->nan_seen, 1u);
        __threadfence();
        const unsigned done = atomicAdd(&ctl->blocks_done, 1u);
        if (done == gridDim.x - 1) {
            __threadfence();
            const unsigned bits = atomicExch(&ctl->rate_bits, 0u);
            const unsigned nan = atomicExch(&ctl->nan_seen, 0u);
            ctl->blocks_done = 0;
            const float rate = __uint_as_float(bits);
            if (nan) ctl->stable_dt = __longlong_as_double(0x7ff8000000000000ll);
            else if (rate > 0.f) ctl->stable_dt = ctl->cfl / (double)rate;
            else ctl->stable_dt = __longlong_as_double(0x7ff0000000000000ll);
        }
    }
}

// solver.rs:94-100 in FP64 on padded host-layout arrays, exactly as the reference computes it
// (IEEE sqrt and division; no contraction across the divisions).
__device__ __forceinline__ double rate64(const double* h, const double* hu, const double* hv,
                                         long long k, double dx, double dy) {
    const double hh = h[k];
    const double c = sqrt(G_D * hh);
    const double u = fabs(hh > H_DRY_D ? hu[k] / hh : 0.0);
    const double v = fabs(hh > H_DRY_D ? hv[k] / hh : 0.0);
    return __dadd_rn(__ddiv_rn(__dadd_rn(u, c), dx), __ddiv_rn(__dadd_rn(v, c), dy));
}

struct Rate64Out {
    unsigned long long max_bits;   // max rate (FP64 bits of a non-negative double)
    unsigned long long first_nan;  // smallest row-major interior index whose rate is NaN
    unsigned long long first_max;  // smallest row-major interior index whose rate equals the max
};

// Pass 1: max rate and first NaN over the interior. Both are order-independent (a max of
// non-negative doubles compared as integers, a min of indices), so each thread keeps its own,
// the warp and the block reduce them, and one thread per block folds them into `out`.
__global__ void rate64_kernel(int nx, int ny, double dx, double dy, const double* __restrict__ h,
                              const double* __restrict__ hu, const double* __restrict__ hv,
                              Rate64Out* out) {
    __shared__ unsigned long long s_max[32], s_nan[32];
    const int W = nx + 6;
    unsigned long long mx = 0ull, first_nan = ~0ull;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)nx * ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)(c / nx);
        const double r = rate64(h, hu, hv, (long long)(j + 3) * W + (i + 3), dx, dy);
        if (r != r) {
            if ((unsigned long long)c < first_nan) first_nan = (unsigned long long)c;
        } else {
            const unsigned long long b = (unsigned long long)__double_as_longlong(r);
            if (b > mx) mx = b;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long om = __shfl_down_sync(0xffffffffu, mx, o);
        const unsigned long long on = __shfl_down_sync(0xffffffffu, first_nan, o);
        mx = om > mx ? om : mx;
        first_nan = on < first_nan ? on : first_nan;
    }
    if ((threadIdx.x & 31) == 0) {
        s_max[threadIdx.x >> 5] = mx;
        s_nan[threadIdx.x >> 5] = first_nan;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (unsigned w = 1; w < blockDim.x / 32; w++) {
            mx = s_max[w] > mx ? s_max[w] : mx;
            first_nan = s_nan[w] < first_nan ? s_nan[w] : first_nan;
        }
        if (mx) atomicMax(&out->max_bits, mx);
        if (first_nan != ~0ull) atomicMin(&out->first_nan, first_nan);
    }
}

// Pass 2: first cell whose rate equals the maximum (solver.rs:464-466 keeps the first).
__global__ void argmax64_kernel(int nx, int ny, double dx, double dy, const double* __restrict__ h,
                                const double* __restrict__ hu, const double* __restrict__ hv,
                                Rate64Out* out) {
    const int W = nx + 6;
    const double best = __longlong_as_double((long long)out->max_bits);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)nx * ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)(c / nx);
        const double r = rate64(h, hu, hv, (long long)(j + 3) * W + (i + 3), dx, dy);
        if (r == best) atomicMin(&out->first_max, (unsigned long long)c);
    }
}

// dispersion.rs:162-201: 1 - phi where the water is at least H_DISP_MIN deep, on the interior.
// h is a device state; bed the FP32 bed; mem the breaking memory of followed fronts, or null
// (a cell whose memory is not 0 reads breaking, dispersion.rs:149-152).
__global__ void breaking_kernel(DevGrid g, const float4* __restrict__ q, const float* __restrict__ bed,
                                BreakingDev br, const double* __restrict__ mem, double* __restrict__ out) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < (long long)g.nx * g.ny;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const long long k = (long long)j * g.pitch + i;
        const float h = q[k].x;
        if (h < H_DISP_MIN) {
            out[c] = 0.0;
            continue;
        }
        if (mem && mem[k] != 0.0) {
            out[c] = 1.0;
            continue;
        }
        auto eta = [&](int di, int dj) {
            const Mapped m = map_cell(g, i + di, j + dj);
            return q[m.k].x + bed[m.k];
        };
        const float ex = (eta(1, 0) - eta(-1, 0)) * g.ix;
        const float ey = (eta(0, 1) - eta(0, -1)) * g.iy;
        const float ratio = fmaxf(eta(0, 0) / h, 0.f);
        const float off = fmaxf(smoothstep(br.er_lo, br.er_inv, ratio),
                                smoothstep(br.sl_lo, br.sl_inv, hypotf(ex, ey)));
        out[c] = (double)off;  // 1 - phi = off
    }
}

// state.rs:78-102: volume (sum of depth), largest momentum, smallest depth, in FP64. One block
// per row band; the last block adds the bands in order, so the sum is reproducible.
__global__ void diagnostics_kernel(DevGrid g, const float4* __restrict__ q, double* band_sum,
                                   double* band_mom, double* band_min, unsigned* done, double* out) {
    __shared__ double red[100];
    const int rows_per = (g.ny + gridDim.x - 1) / gridDim.x;
    const int j0 = blockIdx.x * rows_per, j1 = min(g.ny, j0 + rows_per);
    double s = 0.0, mom = 0.0, mn = __longlong_as_double(0x7ff0000000000000ll);
    for (int j = j0; j < j1; j++)
        for (int i = threadIdx.x; i < g.nx; i += blockDim.x) {
            const float4 v = q[(long long)j * g.pitch + i];
            const double h = depth64(v);
            s += h;
            mom = fmax(mom, fmax(fabs((double)v.z), fabs((double)v.w)));
            mn = fmin(mn, h);
        }
    double a = s, b = -0.0, c = 0.0;
    block_sum3<AUX_NT>(a, b, c, red);
    // max / min with shuffles
    for (int o = 16; o > 0; o >>= 1) {
        mom = fmax(mom, __shfl_down_sync(0xffffffffu, mom, o));
        mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    }
    __shared__ double smom[AUX_NT / 32], smin[AUX_NT / 32];
    if ((threadIdx.x & 31) == 0) {
        smom[threadIdx.x >> 5] = mom;
        smin[threadIdx.x >> 5] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < AUX_NT / 32; w++) {
            mom = fmax(mom, smom[w]);
            mn = fmin(mn, smin[w]);
        }
        band_sum[blockIdx.x] = a;
        band_mom[blockIdx.x] = mom;
        band_min[blockIdx.x] = mn;
        __threadfence();
        const unsigned d = atomicAdd(done, 1u);
        if (d == gridDim.x - 1) {
            __threadfence();
            double vs = 0.0, vm = 0.0, vn = __longlong_as_double(0x7ff0000000000000ll);
            for (unsigned b2 = 0; b2 < gridDim.x; b2++) {
                vs += ((volatile double*)band_sum)[b2];
                vm = fmax(vm, ((volatile double*)band_mom)[b2]);
                vn = fmin(vn, ((volatile double*)band_min)[b2]);
            }
            out[0] = vs * g.dxd * g.dyd;
            out[1] = vm;
            out[2] = vn;
            *done = 0;
        }
    }
}

}  // namespace wcb
