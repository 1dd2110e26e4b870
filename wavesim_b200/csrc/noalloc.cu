// noalloc.cu — the CFL time-step limit on caller-owned device arrays, allocating nothing.
//
// Some callers cannot have a library allocate device memory when they need the time step: host
// applications that hand all of the GPU's memory to their own pool allocator at start-up and run
// under a fixed device-memory budget (a cudaMalloc from the library would fail or break that
// budget), and simulation loops that must not allocate or free per step because cudaFree
// synchronises the whole device. wc_stable_dt allocates its scratch inside its solver; this entry
// point instead takes the state as device pointers from the caller and keeps its own scratch —
// one partial result per CTA plus the final result — in a file-scope __device__ array of fixed
// size, which every GPU that loads the library holds until the process exits.
//
// The computation is the same FP64 rate, cell for cell, as wc_stable_dt's
// (crates/wavecore/src/solver.rs:94-100 and :431-450), so both return the same bits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/wavecore_c.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_BLOCKS = 4096;
constexpr unsigned long long NA_MAX_CELLS = 16777216ull;  // interior cells, e.g. 4096 x 4096
constexpr int NA_SLOTS = 2 * (NA_MAX_BLOCKS + 1);          // (max rate bits, first NaN) per CTA + result

// The scratch: 2 words per CTA and 2 for the result, 64 KiB in all. Shared by every call.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[NA_SLOTS];

std::mutex g_na_mutex;
void* g_na_ptr[64] = {nullptr};             // the scratch's device address, per device
unsigned long long g_na_ctx[64] = {0};      // the context that address belongs to, per device

// The id of the calling thread's current context (0 if none is current), through the driver
// entry points the runtime hands out, so the library needs no link-time libcuda. A context id is
// unique for the life of the process: a device reset gives the device a new one.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess)
            get_id = reinterpret_cast<GetId>(f);
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// The device address of the scratch on the current device. Host code must not pass the symbol
// itself to a kernel: on the host it names a stand-in, not device memory. The address is looked
// up (cudaGetSymbolAddress, which also makes the device's primary context current) on the first
// call on a device, and again whenever the current context is not the one it was looked up in,
// as after cudaDeviceReset, which unloads the module the old address belonged to.
cudaError_t scratch_on_current_device(unsigned long long** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_na_ptr[dev] || ctx == 0 || ctx != g_na_ctx[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_na_ptr[dev] = p;
        g_na_ctx[dev] = current_context_id();
    }
    *out = static_cast<unsigned long long*>(g_na_ptr[dev]);
    return cudaSuccess;
}

__device__ __forceinline__ double na_rate(const double* h, const double* hu, const double* hv,
                                          long long k, double dx, double dy) {
    const double hh = h[k];
    const double c = sqrt(9.81 * hh);
    const double u = fabs(hh > 1e-8 ? hu[k] / hh : 0.0);
    const double v = fabs(hh > 1e-8 ? hv[k] / hh : 0.0);
    return __dadd_rn(__ddiv_rn(__dadd_rn(u, c), dx), __ddiv_rn(__dadd_rn(v, c), dy));
}

// Pass 1: every CTA writes its largest rate (FP64 bits; non-negative doubles order as integers)
// and the first interior index whose rate is NaN, over a grid-stride share of the interior.
// Every slot a pass reads is written by this pass, so nothing needs clearing between calls.
__global__ void __launch_bounds__(NA_THREADS) na_partial_kernel(int nx, int ny, double dx, double dy,
                                                                const double* __restrict__ h,
                                                                const double* __restrict__ hu,
                                                                const double* __restrict__ hv,
                                                                unsigned long long* scratch) {
    __shared__ unsigned long long s_max[NA_THREADS / 32], s_nan[NA_THREADS / 32];
    const int W = nx + 6;
    unsigned long long mx = 0ull, first_nan = ~0ull;
    const long long n = (long long)nx * ny;
    for (long long c = blockIdx.x * (long long)NA_THREADS + threadIdx.x; c < n;
         c += (long long)gridDim.x * NA_THREADS) {
        const int i = (int)(c % nx), j = (int)(c / nx);
        const double r = na_rate(h, hu, hv, (long long)(j + 3) * W + (i + 3), dx, dy);
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
        for (int w = 1; w < NA_THREADS / 32; w++) {
            mx = s_max[w] > mx ? s_max[w] : mx;
            first_nan = s_nan[w] < first_nan ? s_nan[w] : first_nan;
        }
        scratch[2 * blockIdx.x] = mx;
        scratch[2 * blockIdx.x + 1] = first_nan;
    }
}

// Pass 2: one CTA folds the partials of pass 1 into the result slot.
__global__ void __launch_bounds__(NA_THREADS) na_final_kernel(int nblocks, unsigned long long* scratch) {
    __shared__ unsigned long long s_max[NA_THREADS / 32], s_nan[NA_THREADS / 32];
    unsigned long long mx = 0ull, first_nan = ~0ull;
    for (int b = threadIdx.x; b < nblocks; b += NA_THREADS) {
        const unsigned long long m = scratch[2 * b], f = scratch[2 * b + 1];
        mx = m > mx ? m : mx;
        first_nan = f < first_nan ? f : first_nan;
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
        for (int w = 1; w < NA_THREADS / 32; w++) {
            mx = s_max[w] > mx ? s_max[w] : mx;
            first_nan = s_nan[w] < first_nan ? s_nan[w] : first_nan;
        }
        scratch[2 * NA_MAX_BLOCKS] = mx;
        scratch[2 * NA_MAX_BLOCKS + 1] = first_nan;
    }
}

}  // namespace

// The thread's last-error text, kept by wavecore.cu and read by wc_last_error.
namespace wcb_host {
void set_last_error(const std::string& msg);
}

namespace {
wc_status na_fail(wc_status st, const std::string& msg) {
    wcb_host::set_last_error(msg);
    return st;
}
}  // namespace

extern "C" {

wc_status wc_stable_dt_noalloc(const wc_grid* grid, double cfl, const double* d_h, const double* d_hu,
                               const double* d_hv, void* stream, double* dt_out) {
    if (!grid || !d_h || !d_hu || !d_hv || !dt_out) return na_fail(WC_EINVAL, "null argument");
    if (!(grid->nx > 0 && grid->ny > 0)) return na_fail(WC_EINVAL, "grid must have at least one interior cell");
    if (!(grid->dx > 0.0 && grid->dy > 0.0)) return na_fail(WC_EINVAL, "cell size must be positive");
    if (grid->nx > (1ull << 30) || grid->ny > (1ull << 30) ||
        (unsigned long long)grid->nx * grid->ny > NA_MAX_CELLS)
        return na_fail(WC_EINVAL, "grid has more than 16777216 interior cells, the largest the "
                                  "fixed scratch of wc_stable_dt_noalloc serves");
    unsigned long long* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess)
        return na_fail(WC_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    const int nx = (int)grid->nx, ny = (int)grid->ny;
    const unsigned long long n = (unsigned long long)nx * ny;
    const int blocks = (int)std::min<unsigned long long>((n + NA_THREADS - 1) / NA_THREADS, NA_MAX_BLOCKS);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    na_partial_kernel<<<blocks, NA_THREADS, 0, st>>>(nx, ny, grid->dx, grid->dy, d_h, d_hu, d_hv, scratch);
    na_final_kernel<<<1, NA_THREADS, 0, st>>>(blocks, scratch);
    unsigned long long res[2];
    e = cudaMemcpyAsync(res, scratch + 2 * NA_MAX_BLOCKS, sizeof res, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return na_fail(WC_ECUDA, std::string("stable_dt: ") + cudaGetErrorString(e));
    if (res[1] != ~0ull) {
        *dt_out = std::nan("");
        return na_fail(WC_ENAN, "a cell's water is not a number");
    }
    double rate;
    std::memcpy(&rate, &res[0], sizeof rate);
    *dt_out = rate > 0.0 ? cfl / rate : INFINITY;
    return WC_OK;
}

}  // extern "C"
