// wavecore.cu — the C ABI of include/wavecore_c.h on sm_100a.
//
// Host side of the B200 build: owns the device buffers of one solver, its stream and its launch
// sequence. The reference's `Solver` (crates/wavecore/src/solver.rs) is a host object whose
// `step` runs the whole update on the CPU; here `wc_step` moves the caller's FP64 arrays to the
// device, runs the step there and moves them back, and the device-resident entry points keep
// the state in HBM across steps with the clock and the adaptive time step on the device.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wavecore_c.h"
#include "aux.cuh"
#include "common.cuh"
#include "eddy.cuh"
#include "ensemble.cuh"
#include "lpc_host.cuh"
#include "nest.cuh"
#include "pcg.cuh"
#include "pcg_stream.cuh"
#include "fcg_stream.cuh"
#include "record.cuh"
#include "stage.cuh"
#include "stream.cuh"

using namespace wcb;

namespace {

thread_local std::string g_err;

wc_status set_err(wc_status st, const std::string& msg) {
    g_err = msg;
    return st;
}

#define CK(call)                                                                                \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return set_err(WC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

constexpr double TAU = 6.283185307179586;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 2000000000ull;  // 2 s per grid barrier

struct Drive {
    double omega = 0, ky = 0, strength = 0;
};

// forcing.rs:46-75
wc_status linear_wave(double omega, double h, bool dispersive, double* k, double* cg) {
    if (!dispersive) {
        const double c = std::sqrt(9.81 * h);
        *k = omega / c;
        *cg = c;
        return WC_OK;
    }
    const double nu = omega * omega * h / 9.81;
    if (!(nu < 3.0))
        return set_err(WC_EINVAL, "a wave of this angular frequency is too short for the dispersive "
                                  "model at the wave-maker's depth");
    const double kh = std::sqrt(nu / (1.0 - nu / 3.0));
    *k = kh / h;
    const double ps = omega / *k;
    *cg = ps / (1.0 + kh * kh / 3.0);
    return WC_OK;
}

}  // namespace

namespace wcb_host {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace wcb_host

struct wc_solver {
    wc_grid grid{};
    DevGrid g{};
    int W = 0, R = 0;      // padded width and rows (host layout)
    size_t npad = 0;       // padded cells
    size_t ncell = 0;      // device cells: ny * pitch
    int order = WC_ORDER_SECOND;
    double cfl = 0.4;
    int sgn = 0;
    wc_dispersion disp{};
    BreakingDev br{};
    DampParams damp{};
    int has_maker = 0;
    wc_wavemaker maker{};
    Drive drive{};

    cudaStream_t stream = nullptr;      // the stream work is queued on
    cudaStream_t own_stream = nullptr;  // the solver's own stream
    float4 *q0 = nullptr, *q1 = nullptr;
    float* bed = nullptr;
    float* prof = nullptr;
    float2* ycs = nullptr;
    uint8_t* shallow = nullptr;
    float2 *hn = nullptr, *pred = nullptr, *bv = nullptr, *w = nullptr, *r = nullptr, *p0 = nullptr,
           *p1 = nullptr, *ap = nullptr, *diag = nullptr;
    float2 *r2 = nullptr, *s_a = nullptr, *s_b = nullptr, *q_a = nullptr, *q_b = nullptr;  // CG banks
    float *cc = nullptr, *heff = nullptr;
    double* part = nullptr;   // CTA partials of the solve's reductions
    unsigned* bar = nullptr;  // grid-barrier counters: arrivals, released epoch
    Ctl* ctl = nullptr;
    Ctl* ctl_host = nullptr;  // pinned mirror
    double *st_h = nullptr, *st_hu = nullptr, *st_hv = nullptr;  // padded FP64 staging
    Rate64Out* r64 = nullptr;
    double* diag_bands = nullptr;
    unsigned* diag_done = nullptr;
    double* diag_out = nullptr;
    int pcg_blocks = 0, pcg_tiles_x = 0, pcg_tiles_y = 0;
    // The Jacobi solve: register-streaming sweeps (pcg_stream.cuh) in pcg_stream_blocks CTAs, or,
    // with WAVECORE_B200_SOLVE=tiled in the environment at creation, the shared-memory tiled
    // sweeps of pcg.cuh (which the ensemble's persistent launch uses).
    bool solve_streaming = true;
    int pcg_stream_blocks = 0, pcg_strip_rows = 16;
    // The learned path's passes with a network on the solver's own grid: streaming (fcg_stream.cuh)
    // or, with WAVECORE_B200_FCG=tiled at creation, the tiled passes of lpc.cuh.
    bool fcg_streaming = true;
    int fcg_stream_blocks = 0, fcg_strip_rows = 16;
    unsigned long long launches = 0;
    unsigned long long seen_unconverged = 0;
    // Opt-in per-kernel timing: event pairs per launch, read back by wc_profile_read.
    bool prof_on = false;
    struct ProfEv {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<ProfEv> prof_live;
    std::vector<cudaEvent_t> prof_pool;
    // One captured step, replayed by the device-resident stepping (not used while profiling).
    cudaGraphExec_t step_graph = nullptr;
    unsigned long long graph_launches = 0;  // kernels of one replay (a while-node's body: per iteration)
    bool graph_failed = false;
    // The device clock's stable_dt describes the resident state (set by every step's last kernel,
    // cleared by an upload), so adaptive stepping need not recompute it.
    bool rate_current = false;
    // The learned preconditioner (WC_PC_LEARNED): the attached network (not owned), its
    // activations at this grid's size and the flexible CG's extra buffers.
    int pc = WC_PC_JACOBI;
    LpcModel* lpc = nullptr;
    LpcNet lnet;
    int lpc_hp = 0, lpc_wp = 0;
    float2* tv = nullptr;
    FcgScalars* fsc = nullptr;
    double* fpart = nullptr;
    int* done_host = nullptr;
    cudaStream_t body_stream = nullptr;
    unsigned long long fcg_body_launches = 0;  // kernels per flexible-CG iteration
    unsigned long long fcg_iter_base = 0;      // flexible-CG iterations before the network was attached
    // Per-step statistics (wc_recorder): recorded after every step when attached.
    struct wc_recorder* rec = nullptr;
    float* frame = nullptr;  // staging of wc_frame: eta and the breaking indicator, FP32
    // Followed breaking fronts (Breaking::viscosity, eddy.rs): the memory, the step's viscosity,
    // the sub-steps' momentum banks and the cooperative kernel's barrier state.
    int eddy_on = 0;
    EddyParams eddy{};
    // The limit of every bounded device wait (grid barriers of the persistent kernels).
    unsigned long long wait_ns = BARRIER_TIMEOUT_NS;
    // Shallow-water stages of first and second order: the register-streaming kernel (stream.cuh),
    // or, with WAVECORE_B200_STAGE=tiled in the environment at creation, the shared-memory tiled
    // kernel (stage.cuh) that dispersive and fifth-order stages use; both give the same bits.
    bool swe_streaming = true;
    bool stage_tma = true;  // 4-cell-halo stages stage interior tiles by TMA
    double *mem = nullptr, *mem_new = nullptr;
    float* nu = nullptr;
    float2 *mb0 = nullptr, *mb1 = nullptr;
    double* ed_part = nullptr;
    unsigned* ed_bar = nullptr;
    int* ed_sub = nullptr;
    int ed_blocks = 0;

    ~wc_solver();
    void free_all() {
        void* bufs[] = {q0, q1, bed, prof, ycs, shallow, hn, pred, bv, w, r, p0, p1, ap, diag, cc, heff,
                        part, bar, ctl, st_h, st_hu, st_hv, r64, diag_bands, diag_done, diag_out, tv, fsc, fpart,
                        r2, s_a, s_b, q_a, q_b, frame, mem, mem_new, nu, mb0, mb1, ed_part, ed_bar, ed_sub};
        for (void* b : bufs)
            if (b) cudaFree(b);
        if (done_host) cudaFreeHost(done_host);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (ctl_host) cudaFreeHost(ctl_host);
        for (auto& e : prof_live) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        for (auto e : prof_pool) cudaEventDestroy(e);
        if (step_graph) cudaGraphExecDestroy(step_graph);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace {

template <typename T>
wc_status dalloc(T** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return set_err(WC_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemset(*p, 0, n * sizeof(T));
    // cudaMemset and pageable cudaMemcpy run on the legacy stream and may return before they
    // finish; the solvers' streams are non-blocking, so wait here rather than race them.
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) return set_err(WC_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    return WC_OK;
}

#define TRY(x)                          \
    do {                                \
        wc_status st_ = (x);            \
        if (st_ != WC_OK) return st_;   \
    } while (0)

cudaEvent_t prof_event(wc_solver* s) {
    if (!s->prof_pool.empty()) {
        cudaEvent_t e = s->prof_pool.back();
        s->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when profiling is on.
struct ProfScope {
    wc_solver* s;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(wc_solver* s_, int kind_) : s(s_), kind(kind_) {
        if (s->prof_on) {
            a = prof_event(s);
            cudaEventRecord(a, s->stream);
        }
    }
    ~ProfScope() {
        if (a) {
            cudaEvent_t b = prof_event(s);
            cudaEventRecord(b, s->stream);
            s->prof_live.push_back({kind, a, b});
        }
    }
};

dim3 aux_grid(size_t n) {
    size_t b = (n + AUX_NT - 1) / AUX_NT;
    return dim3((unsigned)std::min<size_t>(std::max<size_t>(b, 1), 148 * 16));
}

// Configure every stage-kernel instantiation for its dynamic shared memory.
wc_status configure_kernels_once() {
#define ATTR(K, B) CK(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, B))
    ATTR((stage_kernel<MODE_STAGE1, 1, false>), SMEM_SWE2);
    ATTR((stage_kernel<MODE_STAGE1, 2, false>), SMEM_SWE);
    ATTR((stage_kernel<MODE_STAGE2, 1, false>), SMEM_SWE2);
    ATTR((stage_kernel<MODE_STAGE2, 2, false>), SMEM_SWE);
    ATTR((stage_kernel<MODE_FIRST, 0, false>), SMEM_SWE2);
    ATTR((stage_kernel<MODE_STAGE1, 0, true>), SMEM_SGN);
    ATTR((stage_kernel<MODE_STAGE1, 1, true>), SMEM_SGN);
    ATTR((stage_kernel<MODE_STAGE1, 2, true>), SMEM_SGN);
    ATTR((stage_tma_kernel<MODE_STAGE1, 2, false>), SMEM_SWE);
    ATTR((stage_tma_kernel<MODE_STAGE2, 2, false>), SMEM_SWE);
    ATTR((stage_tma_kernel<MODE_STAGE1, 0, true>), SMEM_SGN);
    ATTR((stage_tma_kernel<MODE_STAGE1, 1, true>), SMEM_SGN);
    ATTR((stage_tma_kernel<MODE_STAGE1, 2, true>), SMEM_SGN);
    ATTR((ensemble_step_kernel<8, 1>), StageGeom<8>::SMEM_SGN);
    ATTR((ensemble_step_kernel<8, 2>), StageGeom<8>::SMEM_SGN);
    ATTR((ensemble_step_kernel<16, 1>), StageGeom<16>::SMEM_SGN);
    ATTR((ensemble_step_kernel<16, 2>), StageGeom<16>::SMEM_SGN);
#undef ATTR
    return WC_OK;
}

// Once per process: a function-local static is initialised once, also when several host threads
// (each with its own solver) reach it together, and every later call returns the first status.
wc_status configure_kernels() {
    static const wc_status st = configure_kernels_once();
    if (st != WC_OK) return set_err(st, "setting the stage kernels' shared-memory limits failed");
    return st;
}

StageArgs stage_args(const wc_solver* s, const float4* qin, const float4* qold, float4* qout, bool plus_dt) {
    StageArgs a{};
    a.g = s->g;
    a.qin = qin;
    a.qold = qold;
    a.qout = qout;
    a.bed = s->bed;
    a.shallow = s->shallow;
    a.mem = s->eddy_on ? s->mem : nullptr;
    a.br = s->br;
    a.maker.on = s->has_maker;
    a.maker.omega = s->drive.omega;
    a.maker.ramp_time = s->maker.ramp_periods * s->maker.period;
    a.maker.prof = s->prof;
    a.maker.ycs = s->ycs;
    a.damp = s->damp;
    a.ctl = s->ctl;
    a.stage_time_plus_dt = plus_dt ? 1 : 0;
    a.nonlinear = s->disp.nonlinear;
    a.hn = s->hn;
    a.pred = s->pred;
    a.cc = s->cc;
    a.heff = s->heff;
    a.bv = s->bv;
    return a;
}

// The tensor maps of a 4-cell-halo stage's TMA boxes over the state `qin` (4 floats per cell,
// {4 nx, ny}, rows 16 pitch bytes apart) and the bed ({nx, ny}, rows 4 pitch bytes apart), with
// the boxes of StageGeom<ST_TY>. False if the driver's encoder is unavailable or refuses.
bool stage_tensor_maps(const wc_solver* s, const float4* qin, CUtensorMap& tq, CUtensorMap& tb) {
    // looked up once per process (a function-local static is initialised once, even when several
    // host threads, each with its own solver, reach it together)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return false;
    using Gm = StageGeom<ST_TY>;
    const DevGrid& g = s->g;
    const cuuint32_t one[2] = {1, 1};
    const cuuint64_t dq[2] = {4ull * (cuuint64_t)g.nx, (cuuint64_t)g.ny};
    const cuuint64_t sq[1] = {16ull * (cuuint64_t)g.pitch};
    const cuuint32_t bq[2] = {4u * Gm::BX, (cuuint32_t)Gm::BY};
    if (encode(&tq, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float4*>(qin), dq, sq, bq, one,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    const cuuint64_t db[2] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny};
    const cuuint64_t sb[1] = {4ull * (cuuint64_t)g.pitch};
    const cuuint32_t bb[2] = {(cuuint32_t)Gm::BX, (cuuint32_t)Gm::BY};
    return encode(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(s->bed), db, sb, bb, one,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

wc_status launch_stage(wc_solver* s, int mode, const float4* qin, const float4* qold, float4* qout,
                       bool plus_dt) {
    const StageArgs a = stage_args(s, qin, qold, qout, plus_dt);
    dim3 grid((s->g.nx + ST_TX - 1) / ST_TX, (s->g.ny + ST_TY - 1) / ST_TY);
    dim3 block(ST_NT);
    cudaStream_t st = s->stream;
    ProfScope ps(s, 0);
    const int o = s->order;
    if (!s->sgn && o <= 1 && s->swe_streaming) {
        const int strips_x = (s->g.nx + SW_OUT - 1) / SW_OUT;
        const dim3 sgrid((strips_x + SW_WARPS - 1) / SW_WARPS, (s->g.ny + SW_ROWS - 1) / SW_ROWS);
        if (mode == MODE_FIRST) swe_stream_kernel<MODE_FIRST, 0, SW_CPL><<<sgrid, SW_NT, sw_smem<SW_CPL>(), st>>>(a, strips_x);
        else if (mode == MODE_STAGE1) swe_stream_kernel<MODE_STAGE1, 1, SW_CPL><<<sgrid, SW_NT, sw_smem<SW_CPL>(), st>>>(a, strips_x);
        else swe_stream_kernel<MODE_STAGE2, 1, SW_CPL><<<sgrid, SW_NT, sw_smem<SW_CPL>(), st>>>(a, strips_x);
        s->launches++;
        CK(cudaGetLastError());
        return WC_OK;
    }
    // Fifth-order and dispersive stages (4-cell halo) on grids with interior tiles: TMA boxes.
    const bool halo4 = s->sgn || (o == 2 && mode != MODE_FIRST);
    CUtensorMap tq, tb;
    if (halo4 && s->stage_tma && s->g.nx >= ST_TX + 2 * ST_HALO && s->g.ny >= ST_TY + 2 * ST_HALO &&
        stage_tensor_maps(s, qin, tq, tb)) {
        if (s->sgn) {
            if (o == 0) stage_tma_kernel<MODE_STAGE1, 0, true><<<grid, block, SMEM_SGN, st>>>(a, tq, tb);
            else if (o == 1) stage_tma_kernel<MODE_STAGE1, 1, true><<<grid, block, SMEM_SGN, st>>>(a, tq, tb);
            else stage_tma_kernel<MODE_STAGE1, 2, true><<<grid, block, SMEM_SGN, st>>>(a, tq, tb);
        } else if (mode == MODE_STAGE1) {
            stage_tma_kernel<MODE_STAGE1, 2, false><<<grid, block, SMEM_SWE, st>>>(a, tq, tb);
        } else {
            stage_tma_kernel<MODE_STAGE2, 2, false><<<grid, block, SMEM_SWE, st>>>(a, tq, tb);
        }
        s->launches++;
        CK(cudaGetLastError());
        return WC_OK;
    }
    if (s->sgn) {
        if (o == 0) stage_kernel<MODE_STAGE1, 0, true><<<grid, block, SMEM_SGN, st>>>(a);
        else if (o == 1) stage_kernel<MODE_STAGE1, 1, true><<<grid, block, SMEM_SGN, st>>>(a);
        else stage_kernel<MODE_STAGE1, 2, true><<<grid, block, SMEM_SGN, st>>>(a);
    } else if (mode == MODE_FIRST) {
        stage_kernel<MODE_FIRST, 0, false><<<grid, block, SMEM_SWE2, st>>>(a);
    } else if (mode == MODE_STAGE1) {
        if (o == 1) stage_kernel<MODE_STAGE1, 1, false><<<grid, block, SMEM_SWE2, st>>>(a);
        else stage_kernel<MODE_STAGE1, 2, false><<<grid, block, SMEM_SWE, st>>>(a);
    } else {
        if (o == 1) stage_kernel<MODE_STAGE2, 1, false><<<grid, block, SMEM_SWE2, st>>>(a);
        else stage_kernel<MODE_STAGE2, 2, false><<<grid, block, SMEM_SWE, st>>>(a);
    }
    s->launches++;
    CK(cudaGetLastError());
    return WC_OK;
}

PcgArgs pcg_args(const wc_solver* s, int mode, const float4* qold, float4* qout, const FcgScalars* fcg = nullptr) {
    PcgArgs a{};
    a.fcg = fcg;
    a.g = s->g;
    a.cc = s->cc;
    a.heff = s->heff;
    a.bv = s->bv;
    a.w = s->w;
    a.r = s->r;
    a.p0 = s->p0;
    a.p1 = s->p1;
    a.ap = s->ap;
    a.diag = s->diag;
    a.rb[0] = s->r;
    a.rb[1] = s->r2;
    a.sb[0] = s->s_a;
    a.sb[1] = s->s_b;
    a.qb[0] = s->q_a;
    a.qb[1] = s->q_b;
    a.part = s->part;
    a.cnt = s->bar;
    a.hn = s->hn;
    a.pred = s->pred;
    a.qold = qold;
    a.qout = qout;
    a.bed = s->bed;
    a.ctl = s->ctl;
    a.tol = s->disp.tolerance;
    a.max_iter = (long long)s->disp.max_iterations;
    a.mode = mode;
    a.defer_finish = s->eddy_on;
    a.tiles_x = s->pcg_tiles_x;
    a.strip_rows = s->pcg_strip_rows;
    a.tiles_y = s->pcg_tiles_y;
    a.damp = s->damp;
    a.timeout_ns = s->wait_ns;
    return a;
}

wc_status launch_pcg(wc_solver* s, int mode, const float4* qold, float4* qout, const FcgScalars* fcg = nullptr) {
    const PcgArgs a = pcg_args(s, mode, qold, qout, fcg);
    CK(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned), s->stream));
    ProfScope ps(s, 1);
    // A cooperative launch: every CTA is resident at once, so the grid barriers cannot deadlock.
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(s->pcg_blocks);
    lc.blockDim = dim3(PG_NT);
    lc.dynamicSmemBytes = 0;
    lc.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    if (s->solve_streaming) {
        lc.gridDim = dim3(s->pcg_stream_blocks);
        lc.blockDim = dim3(PS_NT);
        lc.dynamicSmemBytes = PS_SMEM;
        CK(cudaLaunchKernelEx(&lc, pcg_stream_kernel, a));
    } else {
        CK(cudaLaunchKernelEx(&lc, pcg_kernel, a));
    }
    s->launches++;
    return WC_OK;
}

// ---- the learned path: flexible CG with the network preconditioner --------------------------
//
// Same system, warm start and stopping rule as the Jacobi solve (dispersion.rs:493-545); the
// preconditioner is the two-level cycle of the network (lpc.cuh), so directions are
// A-orthogonalised against the previous one (flexible CG). An iteration is a chain of ordinary
// kernels; in a captured step the chain is the body of a graph while-node whose condition the
// residual kernel sets, so the loop runs on the device without the host.

constexpr int FCG_BLOCKS = 148 * 4;
constexpr int FCG_TILE_BLOCKS = 148 * 8;  // the tiled passes: 32 registers, 5.6 KB shared: 8 blocks per SM

int fcg_blocks(const wc_solver* s) {
    const size_t n = (size_t)s->grid.nx * s->grid.ny;
    return (int)std::max<size_t>(1, std::min<size_t>(FCG_BLOCKS, (n + 255) / 256));
}

#define FCG_LAUNCH(...)                 \
    do {                                \
        __VA_ARGS__;                    \
        s->launches++;                  \
        CK(cudaGetLastError());         \
    } while (0)

// dots of up to three pairs, totalled by the scalars kernel at `step`
wc_status fcg_dots(wc_solver* s, cudaStream_t st, int step, const float2* a0, const float2* b0, const float2* a1,
                   const float2* b1, cudaGraphConditionalHandle h, int cond) {
    const int nb = fcg_blocks(s);
    const FcgScalars* guard = step == FCG_INIT ? nullptr : s->fsc;
    FCG_LAUNCH(fcg_dot_partial_kernel<<<nb, 256, 0, st>>>(s->g, a0, b0, a1, b1, nullptr, nullptr, s->fpart, guard));
    FCG_LAUNCH(fcg_scalars_kernel<<<1, 256, 0, st>>>(s->fpart, nb, s->fsc, step, s->disp.tolerance,
                                                     (long long)s->disp.max_iterations, h, cond));
    return WC_OK;
}

// Before the loop: diagonal, warm start, r = b - A w, the norms, the network's gates.
wc_status fcg_pre(wc_solver* s, cudaStream_t st, cudaGraphConditionalHandle h, int cond) {
    const int nb = fcg_blocks(s);
    FCG_LAUNCH(fcg_setup_kernel<<<nb, 256, 0, st>>>(s->g, s->cc, s->heff, s->diag, s->w));
    FCG_LAUNCH(fcg_matvec_kernel<<<nb, 256, 0, st>>>(s->g, s->w, s->cc, s->heff, s->tv, nullptr));
    FCG_LAUNCH(fcg_residual_kernel<<<nb, 256, 0, st>>>(s->g, s->bv, s->tv, s->r));
    TRY(fcg_dots(s, st, FCG_INIT, s->bv, s->bv, s->r, s->r, h, cond));
    const size_t plane = (size_t)s->lpc_hp * s->lpc_wp;
    FCG_LAUNCH(lpc_features_kernel<<<ew_grid(plane), 256, 0, st>>>(s->g, s->heff, s->bed, s->lnet.F[0].p, s->lpc_hp,
                                                                   s->lpc_wp, s->lpc->stride));
    if (s->lnet.nhwc) {
        CK(s->lnet.gates_h(st));
        s->launches += 3 * LPC_LEVELS;
    } else {
        CK(s->lnet.gates(st));
        s->launches += 2 * LPC_LEVELS + (LPC_LEVELS - 1);
    }
    return WC_OK;
}

// the scalars kernel at `step`, over the partials of the `nblocks` blocks of the last pass
wc_status fcg_scalars(wc_solver* s, cudaStream_t st, int step, int nblocks, cudaGraphConditionalHandle h, int cond) {
    FCG_LAUNCH(fcg_scalars_kernel<<<1, 256, 0, st>>>(s->fpart, nblocks, s->fsc, step, s->disp.tolerance,
                                                     (long long)s->disp.max_iterations, h, cond));
    return WC_OK;
}

// blocks of the tiled passes: every tile of 32 x 8 cells once, at most FCG_TILE_BLOCKS blocks
int fcg_tile_blocks(const wc_solver* s) {
    const long long tiles = (long long)((s->grid.nx + FT_X - 1) / FT_X) * (long long)((s->grid.ny + FT_Y - 1) / FT_Y);
    return (int)std::max<long long>(1, std::min<long long>(FCG_TILE_BLOCKS, tiles));
}

// One iteration in four passes over the cells (lpc.cuh): z = M r (pre, the network, post),
// p = z + beta p and q = A p (dir), w and r (upd), with the scalars kernel after each dot.
// Directions alternate between two banks by `parity`: dir reads the previous one at stencil
// neighbours while it writes the new one.
wc_status fcg_body(wc_solver* s, cudaStream_t st, cudaGraphConditionalHandle h, int cond, int parity) {
    const DevGrid& g = s->g;
    const int nb = fcg_blocks(s), nt = fcg_tile_blocks(s);
    FcgScalars* sc = s->fsc;
    float2 *z1 = s->tv, *z = s->p1, *q = s->ap;
    float2* p_old = parity ? s->r2 : s->p0;
    float2* p_new = parity ? s->p0 : s->r2;
    const int hp = s->lpc_hp, wp = s->lpc_wp, S = s->lpc->stride;
    const size_t plane = (size_t)hp * wp;
    const bool nhwc = s->lnet.nhwc;
    {
        ProfScope ps(s, 1);
        unsigned* xh = nhwc ? reinterpret_cast<unsigned*>(s->lnet.Xh.p) : nullptr;
        if (S == 1 && s->fcg_streaming)
            FCG_LAUNCH(fcg_pre_stream_kernel<<<s->fcg_stream_blocks, FS_NT, FS_SMEM, st>>>(
                g, s->fcg_strip_rows, s->r, s->diag, s->cc, s->heff, z1, LPC_OMEGA, s->lnet.X[0].p, xh, hp, wp, sc));
        else if (S == 1)
            FCG_LAUNCH(fcg_pre_tile_kernel<<<nt, FT_NT, 0, st>>>(g, s->r, s->diag, s->cc, s->heff, z1, LPC_OMEGA,
                                                                 s->lnet.X[0].p, xh, hp, wp, sc));
        else
            FCG_LAUNCH(fcg_pre_kernel<<<ew_grid(plane), 256, 0, st>>>(g, s->r, s->diag, s->cc, s->heff, z1, LPC_OMEGA,
                                                                      s->lnet.X[0].p, xh, hp, wp, S, sc));
    }
    {
        ProfScope ps(s, 3);
        CK(nhwc ? s->lnet.forward_h(st) : s->lnet.forward(st, false));
        s->launches += nhwc ? s->lnet.forward_h_launches() : 2 * LPC_LEVELS + 2 * (LPC_LEVELS - 1) + 1;
    }
    ProfScope ps(s, 1);
    const float* y = nhwc ? s->lnet.Yh.p : s->lnet.Y.p;
    const int lgS = S == 1 ? 0 : S == 2 ? 1 : S == 4 ? 2 : 3;
    if (S == 1 && s->fcg_streaming) {
        const int nf = s->fcg_stream_blocks, rows = s->fcg_strip_rows;
        FCG_LAUNCH(fcg_post_stream_kernel<<<nf, FS_NT, FS_SMEM, st>>>(g, rows, z1, y, nhwc ? 1 : 0, s->r, s->diag, s->cc,
                                                                s->heff, z, q, LPC_OMEGA, hp, wp, s->fpart, sc));
        TRY(fcg_scalars(s, st, FCG_BETA, nf, h, 0));
        FCG_LAUNCH(fcg_dir_stream_kernel<<<nf, FS_NT, FS_SMEM, st>>>(g, rows, z, p_old, p_new, s->cc, s->heff, q, s->r,
                                                               s->fpart, sc));
        TRY(fcg_scalars(s, st, FCG_ALPHA, nf, h, 0));
    } else {
        FCG_LAUNCH(fcg_post_tile_kernel<<<nt, FT_NT, 0, st>>>(g, z1, y, nhwc ? 1 : 0, s->r, s->diag, s->cc, s->heff, z,
                                                              q, LPC_OMEGA, hp, wp, lgS, s->fpart, sc));
        TRY(fcg_scalars(s, st, FCG_BETA, nt, h, 0));
        FCG_LAUNCH(fcg_dir_tile_kernel<<<nt, FT_NT, 0, st>>>(g, z, p_old, p_new, s->cc, s->heff, q, s->r, s->fpart, sc));
        TRY(fcg_scalars(s, st, FCG_ALPHA, nt, h, 0));
    }
    FCG_LAUNCH(fcg_upd_kernel<<<nb, 256, 0, st>>>(g, s->w, s->r, p_new, q, s->fpart, sc));
    TRY(fcg_scalars(s, st, FCG_RESID, nb, h, cond));
    return WC_OK;
}

wc_status launch_fcg(wc_solver* s, int mode, const float4* qold, float4* qout) {
    cudaStream_t st = s->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    const bool graph = cs == cudaStreamCaptureStatusActive;
    cudaGraphConditionalHandle h = 0;
    if (graph) {
        cudaGraph_t cg = nullptr;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, nullptr, nullptr));
        CK(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
    }
    {
        {
            ProfScope ps(s, 1);
            TRY(fcg_pre(s, st, h, graph ? 1 : 0));
        }
        if (graph) {
            cudaGraph_t cg = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t node = nullptr;
            CK(cudaGraphAddNode(&node, cg, deps, nd, &np));
            CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
            cudaGraph_t body = np.conditional.phGraph_out[0];
            CK(cudaStreamBeginCaptureToGraph(s->body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            const unsigned long long before = s->launches;
            // two iterations per body, so that the direction banks alternate (the second returns
            // at once when the first converged)
            wc_status bs = fcg_body(s, s->body_stream, h, 1, 0);
            if (bs == WC_OK) bs = fcg_body(s, s->body_stream, h, 1, 1);
            cudaGraph_t captured = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s->body_stream, &captured);
            s->fcg_body_launches = (s->launches - before) / 2;
            s->launches = before;  // body launches are counted per executed iteration
            if (bs != WC_OK) return bs;
            CK(e);
        } else {
            // Without a graph: iterations in chunks, the host looks at `done` between them; the
            // kernels of iterations past the end return at once.
            const long long max_it = (long long)s->disp.max_iterations;
            for (long long k = 0; k < max_it;) {
                const long long chunk = std::min<long long>(4, max_it - k);
                const unsigned long long before = s->launches;
                for (long long c = 0; c < chunk; c++) TRY(fcg_body(s, st, 0, 0, (int)((k + c) & 1)));
                s->fcg_body_launches = (s->launches - before) / (unsigned long long)chunk;
                s->launches = before;
                k += chunk;
                CK(cudaMemcpyAsync(s->done_host, &s->fsc->done, sizeof(int), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (*s->done_host) break;
            }
        }
    }
    return launch_pcg(s, mode, qold, qout, s->fsc);
}

// The dispersive solve of one stage by the configured method.
wc_status launch_solve(wc_solver* s, int mode, const float4* qold, float4* qout) {
    if (s->pc == WC_PC_LEARNED) {
        if (!s->lpc) return set_err(WC_EINVAL, "the learned preconditioner is selected but no network is attached");
        return launch_fcg(s, mode, qold, qout);
    }
    return launch_pcg(s, mode, qold, qout);
}

// One SSP-RK2 step (solver.rs:479-507) of size ctl->dt on the device-resident state q0.
wc_status enqueue_record(wc_solver* s);

// Followed fronts and their eddy viscosity on the resident state (solver.rs:509-532): one
// cooperative launch, so that its grid barriers cannot deadlock. With `finish` it is the step's
// last kernel and closes the step; `sub_out` (device) receives the sub-steps taken.
wc_status launch_eddy(wc_solver* s, int finish, int* sub_out) {
    EddyArgs a{};
    a.g = s->g;
    a.q = s->q0;
    a.bed = s->bed;
    a.mem = s->mem;
    a.mem_new = s->mem_new;
    a.nu = s->nu;
    a.mb[0] = s->mb0;
    a.mb[1] = s->mb1;
    a.part = s->ed_part;
    a.cnt = s->ed_bar;
    a.ctl = s->ctl;
    a.sub_out = sub_out;
    a.e = s->eddy;
    a.finish = finish;
    a.timeout_ns = s->wait_ns;
    CK(cudaMemsetAsync(s->ed_bar, 0, 2 * sizeof(unsigned), s->stream));
    ProfScope ps(s, 4);
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(s->ed_blocks);
    lc.blockDim = dim3(ED_NT);
    lc.dynamicSmemBytes = 0;
    lc.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    CK(cudaLaunchKernelEx(&lc, eddy_kernel, a));
    s->launches++;
    return WC_OK;
}

wc_status enqueue_step_kernels(wc_solver* s) {
    if (s->order == WC_ORDER_FIRST) {
        TRY(launch_stage(s, MODE_FIRST, s->q0, s->q0, s->q1, false));
        if (s->sgn) TRY(launch_solve(s, MODE_FIRST, s->q0, s->q1));
        CK(cudaMemcpyAsync(s->q0, s->q1, s->ncell * sizeof(float4), cudaMemcpyDeviceToDevice, s->stream));
    } else if (!s->sgn) {
        TRY(launch_stage(s, MODE_STAGE1, s->q0, s->q0, s->q1, false));
        TRY(launch_stage(s, MODE_STAGE2, s->q1, s->q0, s->q0, true));
    } else {
        TRY(launch_stage(s, MODE_STAGE1, s->q0, s->q0, s->q1, false));
        TRY(launch_solve(s, MODE_STAGE1, s->q0, s->q1));
        TRY(launch_stage(s, MODE_STAGE1, s->q1, s->q0, s->q1, true));
        TRY(launch_solve(s, MODE_STAGE2, s->q0, s->q0));
    }
    // solver.rs:505: the fronts follow the damped state, and close the step
    if (s->eddy_on) TRY(launch_eddy(s, 1, nullptr));
    return WC_OK;
}

wc_status enqueue_step_direct(wc_solver* s) {
    TRY(enqueue_step_kernels(s));
    if (s->rec) TRY(enqueue_record(s));
    return WC_OK;
}

wc_status enqueue_step(wc_solver* s) {
    s->rate_current = true;
    if (s->prof_on || s->graph_failed) return enqueue_step_direct(s);
    if (!s->step_graph) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            s->graph_failed = true;
            return enqueue_step_direct(s);
        }
        const unsigned long long before = s->launches;
        wc_status st = enqueue_step_direct(s);
        cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
        s->graph_launches = s->launches - before;
        s->launches = before;
        if (st != WC_OK || e != cudaSuccess ||
            cudaGraphInstantiate(&s->step_graph, graph, 0) != cudaSuccess) {
            cudaGetLastError();
            if (graph) cudaGraphDestroy(graph);
            s->step_graph = nullptr;
            s->graph_failed = true;
            return enqueue_step_direct(s);
        }
        cudaGraphDestroy(graph);
    }
    CK(cudaGraphLaunch(s->step_graph, s->stream));
    s->launches += s->graph_launches;
    return WC_OK;
}

wc_status read_ctl(wc_solver* s) {
    CK(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return WC_OK;
}

wc_status status_of(wc_solver* s) {
    TRY(read_ctl(s));
    if (s->ctl_host->error & ERR_TIMEOUT)
        return set_err(WC_ETIMEOUT, "a grid barrier of the dispersive solve timed out");
    if (s->ctl_host->error & ERR_TMA)
        return set_err(WC_ECUDA, "a stage kernel's TMA box load did not complete within its wait limit");
    if (s->ctl_host->error & ERR_NAN) return set_err(WC_ENAN, "the state holds a NaN");
    if (s->ctl_host->error & ERR_EDDY)
        return set_err(WC_EUNSUPPORTED, "the eddy viscosity needed more than 65536 sub-steps; it was not applied");
    return WC_OK;
}

wc_status stage_host(wc_solver* s, const double* h, const double* hu, const double* hv) {
    const size_t bytes = s->npad * sizeof(double);
    CK(cudaMemcpyAsync(s->st_h, h, bytes, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->st_hu, hu, bytes, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->st_hv, hv, bytes, cudaMemcpyHostToDevice, s->stream));
    return WC_OK;
}

// Ghost cells of a padded host array by the boundary rule, without sign changes
// (grid.rs:60-87): the carried `breaking` memory.
void fill_scalar_ghosts(const wc_grid& gr, bool periodic, double* a) {
    const size_t nx = gr.nx, ny = gr.ny, w = nx + 6;
    auto at = [&](size_t i, size_t j) -> double& { return a[j * w + i]; };
    for (size_t j = 3; j < 3 + ny; j++)
        for (size_t k = 0; k < 3; k++) {
            at(2 - k, j) = at(3 + k, j);
            at(3 + nx + k, j) = at(2 + nx - k, j);
        }
    for (size_t i = 0; i < w; i++)
        for (size_t k = 0; k < 3; k++) {
            at(i, 2 - k) = at(i, 3 + k);
            at(i, 3 + ny + k) = at(i, 2 + ny - k);
        }
    if (periodic)
        for (size_t i = 0; i < w; i++)
            for (size_t k = 0; k < 3; k++) {
                at(i, 2 - k) = at(i, 2 + ny - k);
                at(i, 3 + ny + k) = at(i, 3 + k);
            }
}

}  // namespace

extern "C" {

void wc_config_default(wc_config* cfg) {
    std::memset(cfg, 0, sizeof *cfg);
    cfg->cfl = 0.4;
    cfg->order = WC_ORDER_SECOND;
}

void wc_dispersion_default(wc_dispersion* d) {
    std::memset(d, 0, sizeof *d);
    d->breaking.eta_ratio_lo = 0.30;
    d->breaking.eta_ratio_hi = 0.55;
    d->breaking.slope_lo = 0.40;
    d->breaking.slope_hi = 0.65;
    d->nonlinear = 1;
    d->tolerance = 1e-4;
    d->max_iterations = 200;
    d->preconditioner = WC_PC_JACOBI;
    d->breaking.viscosity = 0;
    wc_eddy_default(&d->breaking.eddy);
}

void wc_eddy_default(wc_eddy* e) {
    e->initial = 0.65;
    e->settled = 0.15;
    e->duration = 5.0;
    e->mixing = 1.2;
    e->linger = 5.0;
}

const char* wc_last_error(void) { return g_err.c_str(); }

uint64_t wc_launch_count(const wc_solver* s) {
    if (!s) return 0;
    uint64_t n = s->launches;
    if (s->fcg_body_launches) {  // flexible-CG iterations run as while-node bodies: count them
        Ctl c{};
        if (cudaMemcpyAsync(&c, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream) == cudaSuccess &&
            cudaStreamSynchronize(s->stream) == cudaSuccess)
            n += s->fcg_body_launches * (c.fcg_iterations - s->fcg_iter_base);
    }
    return n;
}

wc_status wc_solver_create(const wc_grid* grid, const double* bed_padded, const wc_config* cfg,
                           wc_solver** out) {
    if (!out) return set_err(WC_EINVAL, "out is null");
    *out = nullptr;
    if (!grid || !bed_padded || !cfg) return set_err(WC_EINVAL, "null argument");
    if (!(grid->nx > 0 && grid->ny > 0)) return set_err(WC_EINVAL, "grid must have at least one interior cell");
    if (!(grid->dx > 0.0 && grid->dy > 0.0)) return set_err(WC_EINVAL, "cell size must be positive");
    if ((double)grid->nx * (double)grid->ny > 1.5e9 || grid->nx > (1u << 30) || grid->ny > (1u << 30))
        return set_err(WC_EINVAL, "grid too large for 32-bit cell indexing");
    if (cfg->order < WC_ORDER_FIRST || cfg->order > WC_ORDER_FIFTH) return set_err(WC_EINVAL, "unknown order");
    if (cfg->n_sponges > (uint64_t)MAX_SPONGES)
        return set_err(WC_EUNSUPPORTED, "at most 8 sponges are supported");
    if (cfg->n_sponges && !cfg->sponges) return set_err(WC_EINVAL, "sponges is null");
    if (cfg->dispersion) {
        if (cfg->dispersion->preconditioner != WC_PC_JACOBI && cfg->dispersion->preconditioner != WC_PC_LEARNED)
            return set_err(WC_EINVAL, "unknown preconditioner");
        if (!(cfg->dispersion->tolerance >= 0.0)) return set_err(WC_EINVAL, "tolerance must be >= 0");
    }
    TRY(configure_kernels());

    wc_solver* s = new wc_solver();
    auto fail = [&](wc_status st) {
        delete s;
        return st;
    };
    s->grid = *grid;
    {
        const char* v = std::getenv("WAVECORE_B200_STAGE");
        s->swe_streaming = !(v && std::strcmp(v, "tiled") == 0);
        const char* t = std::getenv("WAVECORE_B200_STAGE_TMA");
        s->stage_tma = !(t && std::strcmp(t, "0") == 0);
    }
    const int nx = (int)grid->nx, ny = (int)grid->ny;
    s->W = nx + 6;
    s->R = ny + 6;
    s->npad = (size_t)s->W * s->R;
    const int pitch = (nx + 31) / 32 * 32;
    s->ncell = (size_t)ny * pitch;
    DevGrid& g = s->g;
    g.nx = nx;
    g.ny = ny;
    g.pitch = pitch;
    g.periodic = cfg->periodic_y ? 1 : 0;
    g.dx = (float)grid->dx;
    g.dy = (float)grid->dy;
    g.ix = (float)(0.5 / grid->dx);
    g.iy = (float)(0.5 / grid->dy);
    g.inv_dx = (float)(1.0 / grid->dx);
    g.inv_dy = (float)(1.0 / grid->dy);
    g.dxd = grid->dx;
    g.dyd = grid->dy;
    s->order = cfg->order;
    s->cfl = cfg->cfl;
    s->sgn = cfg->dispersion ? 1 : 0;
    if (cfg->dispersion) {
        s->disp = *cfg->dispersion;
        s->pc = cfg->dispersion->preconditioner;
    }
    else wc_dispersion_default(&s->disp);
    const wc_breaking& b = s->disp.breaking;  // Breaking::default() for shallow water (solver.rs:618-623)
    s->br.er_lo = (float)b.eta_ratio_lo;
    s->br.er_inv = (float)(1.0 / (b.eta_ratio_hi - b.eta_ratio_lo));
    s->br.sl_lo = (float)b.slope_lo;
    s->br.sl_inv = (float)(1.0 / (b.slope_hi - b.slope_lo));
    // follow_breaking reads the viscosity of the dispersion only (solver.rs:512-518)
    s->eddy_on = (s->sgn && b.viscosity) ? 1 : 0;
    s->eddy = EddyParams{b.eddy.initial, b.eddy.settled, b.eddy.duration, b.eddy.mixing, b.eddy.linger,
                         b.eta_ratio_lo, b.eta_ratio_hi, b.slope_lo, b.slope_hi};
    s->damp.nsp = (int)cfg->n_sponges;
    s->damp.manning = (float)cfg->manning;
    for (int m = 0; m < s->damp.nsp; m++) {
        const wc_sponge& sp = cfg->sponges[m];
        SpongeDev& d = s->damp.sp[m];
        d.width = (int)std::min<uint64_t>(sp.width, (uint64_t)1 << 30);
        d.strength = (float)sp.strength;
        d.inv_w = (float)(1.0 / (double)sp.width);
        d.level = sp.level;
        d.west = sp.west;
        d.east = sp.east;
        d.south = sp.south;
        d.north = sp.north;
    }

    // The bed as the reference's solver holds it: with_periodic_y wraps its ghost rows; the
    // wave-maker's depth is read at the source column, mid-row (solver.rs:400-409).
    if (cfg->wavemaker) {
        const wc_wavemaker& spec = *cfg->wavemaker;
        double rr = std::round(spec.x / grid->dx - 0.5);
        if (rr < 0.0) rr = 0.0;
        size_t i = (size_t)rr;
        if (i > (size_t)nx - 1) i = nx - 1;
        i += 3;
        const double depth = -bed_padded[(size_t)(3 + ny / 2) * s->W + i];
        // Drive::new (forcing.rs:87-117)
        if (!(depth > 0.0)) return fail(set_err(WC_EINVAL, "wave-maker must sit in water"));
        if (!(spec.period > 0.0 && spec.sigma > 0.0 && spec.amplitude >= 0.0))
            return fail(set_err(WC_EINVAL, "wave-maker period and sigma must be positive, amplitude >= 0"));
        const double omega = TAU / spec.period;
        double k, cg;
        wc_status st = linear_wave(omega, depth, s->sgn != 0, &k, &cg);
        if (st != WC_OK) return fail(st);
        const double ky = k * std::sin(spec.angle), kx = k * std::cos(spec.angle);
        const double rolloff = std::exp(0.5 * kx * kx * spec.sigma * spec.sigma);
        const double flux = 2.0 * cg * spec.amplitude * std::cos(spec.angle) * rolloff;
        double norm = 0.0;
        for (int ii = 0; ii < nx; ii++) {
            const double x = ((double)ii + 0.5) * grid->dx, d = x - spec.x;
            norm += std::exp(-(d * d) / (2.0 * spec.sigma * spec.sigma)) * grid->dx;
        }
        s->drive.omega = omega;
        s->drive.ky = ky;
        s->drive.strength = flux / norm;
        s->maker = spec;
        s->has_maker = 1;
        // check_periodic (solver.rs:421-429)
        if (cfg->periodic_y) {
            const double turns = ky * (double)ny * grid->dy / TAU;
            if (!(std::fabs(turns - std::round(turns)) < 1e-6))
                return fail(set_err(WC_EPERIODIC, "wave-maker does not fit the periodic domain: "
                                                  "k_y * Ly / 2pi must be a whole number"));
        }
    }

    if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "cudaStreamCreate failed"));
    s->stream = s->own_stream;
    wc_status st;
#define ALLOC(p, n)                       \
    if ((st = dalloc(&(p), (n))) != WC_OK) \
        return fail(st);
    ALLOC(s->q0, s->ncell);
    ALLOC(s->q1, s->ncell);
    ALLOC(s->bed, s->ncell);
    ALLOC(s->ctl, 1);
    ALLOC(s->st_h, s->npad);
    ALLOC(s->st_hu, s->npad);
    ALLOC(s->st_hv, s->npad);
    ALLOC(s->r64, 1);
    const int bands = std::max(1, std::min(ny, 1024));
    ALLOC(s->diag_bands, 3 * (size_t)bands);
    ALLOC(s->diag_done, 1);
    ALLOC(s->diag_out, 3);
    if (s->has_maker) {
        ALLOC(s->prof, (size_t)pitch);
        ALLOC(s->ycs, (size_t)ny);
        std::vector<float> prof(pitch, 0.f);
        for (int ii = 0; ii < nx; ii++) {
            const double x = ((double)ii + 0.5) * grid->dx, d = x - s->maker.x;
            const double pr = std::exp(-(d * d) / (2.0 * s->maker.sigma * s->maker.sigma));
            prof[ii] = pr < 1e-12 ? 0.f : (float)(s->drive.strength * pr);
        }
        std::vector<float2> ycs(ny);
        for (int jj = 0; jj < ny; jj++) {
            const double y = ((double)jj + 0.5) * grid->dy;
            ycs[jj] = make_float2((float)std::cos(s->drive.ky * y), (float)std::sin(s->drive.ky * y));
        }
        if (cudaMemcpy(s->prof, prof.data(), pitch * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->ycs, ycs.data(), ny * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaStreamSynchronize(0) != cudaSuccess)
            return fail(set_err(WC_ECUDA, "maker tables upload failed"));
    }
    if (cfg->shallow_cells) {
        ALLOC(s->shallow, s->ncell);
        std::vector<uint8_t> m(s->ncell, 0);
        for (int jj = 0; jj < ny; jj++)
            for (int ii = 0; ii < nx; ii++) m[(size_t)jj * pitch + ii] = cfg->shallow_cells[(size_t)jj * nx + ii] ? 1 : 0;
        if (cudaMemcpy(s->shallow, m.data(), s->ncell, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaStreamSynchronize(0) != cudaSuccess)
            return fail(set_err(WC_ECUDA, "shallow-cell mask upload failed"));
    }
    if (s->sgn) {
        ALLOC(s->hn, s->ncell);
        ALLOC(s->pred, s->ncell);
        ALLOC(s->bv, s->ncell);
        ALLOC(s->w, s->ncell);
        ALLOC(s->r, s->ncell);
        ALLOC(s->p0, s->ncell);
        ALLOC(s->p1, s->ncell);
        ALLOC(s->ap, s->ncell);
        ALLOC(s->diag, s->ncell);
        ALLOC(s->r2, s->ncell);
        ALLOC(s->s_a, s->ncell);
        ALLOC(s->s_b, s->ncell);
        ALLOC(s->q_a, s->ncell);
        ALLOC(s->q_b, s->ncell);
        ALLOC(s->cc, s->ncell);
        ALLOC(s->heff, s->ncell);
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pcg_kernel, PG_NT, 0) != cudaSuccess || occ < 1)
            return fail(set_err(WC_ECUDA, "occupancy query for the solve kernel failed"));
        s->pcg_tiles_x = (nx + PG_TX - 1) / PG_TX;
        s->pcg_tiles_y = (ny + PG_TY - 1) / PG_TY;
        const int tiles = s->pcg_tiles_x * s->pcg_tiles_y;
        s->pcg_blocks = std::max(1, std::min(tiles, sms * std::min(occ, 4)));
        int occ_s = 0;
        // the streaming sweeps' rings of rows in flight are dynamic shared memory
        if (cudaFuncSetAttribute(pcg_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PS_SMEM) != cudaSuccess ||
            cudaFuncSetAttribute(fcg_pre_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FS_SMEM) != cudaSuccess ||
            cudaFuncSetAttribute(fcg_post_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FS_SMEM) != cudaSuccess ||
            cudaFuncSetAttribute(fcg_dir_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FS_SMEM) != cudaSuccess)
            return fail(set_err(WC_ECUDA, "setting the streaming sweeps' shared memory failed"));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, pcg_stream_kernel, PS_NT, PS_SMEM) != cudaSuccess || occ_s < 1)
            return fail(set_err(WC_ECUDA, "occupancy query for the streaming solve kernel failed"));
        s->pcg_strip_rows = ps_rows_for(nx, ny, sms * occ_s * PS_WARPS);
        const int strip_ctas = (ps_strips(nx, ny, s->pcg_strip_rows) + PS_WARPS - 1) / PS_WARPS;
        s->pcg_stream_blocks = std::max(1, std::min(strip_ctas, sms * occ_s));
        {
            const char* v = std::getenv("WAVECORE_B200_SOLVE");
            s->solve_streaming = !(v && std::strcmp(v, "tiled") == 0);
        }
        {
            const char* v = std::getenv("WAVECORE_B200_FCG");
            s->fcg_streaming = !(v && std::strcmp(v, "tiled") == 0);
            int occ_f = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, fcg_dir_stream_kernel, FS_NT, FS_SMEM) != cudaSuccess || occ_f < 1)
                return fail(set_err(WC_ECUDA, "occupancy query for the flexible-CG passes failed"));
            occ_f = std::min(occ_f, FS_MINB);
            s->fcg_strip_rows = ps_rows_for(nx, ny, sms * occ_f * FS_WARPS);
            const int strip_ctas = (ps_strips(nx, ny, s->fcg_strip_rows) + FS_WARPS - 1) / FS_WARPS;
            s->fcg_stream_blocks = std::max(1, std::min(strip_ctas, sms * occ_f));
        }
        ALLOC(s->part, 8 * (size_t)std::max(s->pcg_blocks, s->pcg_stream_blocks));
        ALLOC(s->bar, 2);
    }
    if (s->eddy_on) {
        ALLOC(s->mem, s->ncell);
        ALLOC(s->mem_new, s->ncell);
        ALLOC(s->nu, s->ncell);
        ALLOC(s->mb0, s->ncell);
        ALLOC(s->mb1, s->ncell);
        ALLOC(s->ed_bar, 2);
        ALLOC(s->ed_sub, 1);
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, eddy_kernel, ED_NT, 0) != cudaSuccess || occ < 1)
            return fail(set_err(WC_ECUDA, "occupancy query for the eddy kernel failed"));
        const size_t need = ((size_t)nx * ny + ED_NT - 1) / ED_NT;
        s->ed_blocks = (int)std::max<size_t>(1, std::min<size_t>(need, (size_t)sms * std::min(occ, 4)));
        ALLOC(s->ed_part, 2 * (size_t)s->ed_blocks);
    }
#undef ALLOC
    if (cudaMallocHost(&s->ctl_host, sizeof(Ctl)) != cudaSuccess)
        return fail(set_err(WC_ENOMEM, "cudaMallocHost failed"));

    // The bed, interior only, FP32.
    if (cudaMemcpy(s->st_h, bed_padded, s->npad * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "bed upload failed"));
    pack_f32_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->st_h, s->bed);
    s->launches++;
    Ctl c{};
    c.cfl = s->cfl;
    c.active = 1;
    c.stable_dt = std::nan("");
    std::memcpy(s->ctl_host, &c, sizeof c);
    if (cudaMemcpyAsync(s->ctl, s->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return fail(set_err(WC_ECUDA, std::string("solver setup failed: ") + cudaGetErrorString(cudaGetLastError())));
    *out = s;
    return WC_OK;
}

void wc_solver_destroy(wc_solver* s) {
    if (s) cudaStreamSynchronize(s->stream);
    delete s;
}

wc_status wc_profile_enable(wc_solver* s, int32_t on) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    CK(cudaStreamSynchronize(s->stream));
    for (auto& e : s->prof_live) {
        s->prof_pool.push_back(e.a);
        s->prof_pool.push_back(e.b);
    }
    s->prof_live.clear();
    s->prof_on = on != 0;
    return WC_OK;
}

wc_status wc_profile_read(wc_solver* s, wc_kernel_time out[WC_KERNEL_KINDS]) {
    if (!s || !out) return set_err(WC_EINVAL, "null argument");
    CK(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < WC_KERNEL_KINDS; k++) out[k] = wc_kernel_time{0, 0.0};
    for (auto& e : s->prof_live) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e.a, e.b));
        out[e.kind].launches += 1;
        out[e.kind].total_ms += ms;
    }
    return WC_OK;
}

wc_status wc_set_wait_limit(wc_solver* s, uint64_t ns) {
    if (!s) return set_err(WC_EINVAL, "null argument");
    s->wait_ns = ns ? (unsigned long long)ns : BARRIER_TIMEOUT_NS;
    // A captured step holds the old limit in its kernels' arguments: capture again.
    if (s->step_graph) {
        CK(cudaStreamSynchronize(s->stream));
        CK(cudaGraphExecDestroy(s->step_graph));
        s->step_graph = nullptr;
    }
    return WC_OK;
}

wc_status wc_set_stream(wc_solver* s, void* stream) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    CK(cudaStreamSynchronize(s->stream));
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    return WC_OK;
}

wc_status wc_state_upload(wc_solver* s, const double* h, const double* hu, const double* hv, double time) {
    if (!s || !h || !hu || !hv) return set_err(WC_EINVAL, "null argument");
    TRY(stage_host(s, h, hu, hv));
    upload_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->st_h, s->st_hu, s->st_hv, s->q0);
    s->launches++;
    s->rate_current = false;
    if (s->eddy_on) CK(cudaMemsetAsync(s->mem, 0, s->ncell * sizeof(double), s->stream));
    CK(cudaGetLastError());
    // The clock; a new state clears the error bits.
    TRY(read_ctl(s));
    s->ctl_host->t = time;
    s->ctl_host->error = 0;
    s->ctl_host->active = 1;
    s->ctl_host->adaptive = 0;
    CK(cudaMemcpyAsync(s->ctl, s->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return WC_OK;
}

wc_status wc_state_download(wc_solver* s, double* h, double* hu, double* hv, double* time) {
    if (!s || !h || !hu || !hv) return set_err(WC_EINVAL, "null argument");
    download_kernel<<<aux_grid(s->npad), AUX_NT, 0, s->stream>>>(s->g, s->q0, s->st_h, s->st_hu, s->st_hv);
    s->launches++;
    CK(cudaGetLastError());
    const size_t bytes = s->npad * sizeof(double);
    CK(cudaMemcpyAsync(h, s->st_h, bytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hu, s->st_hu, bytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hv, s->st_hv, bytes, cudaMemcpyDeviceToHost, s->stream));
    TRY(read_ctl(s));
    if (time) *time = s->ctl_host->t;
    return WC_OK;
}

wc_status wc_breaking_upload(wc_solver* s, const double* breaking) {
    if (!s || !breaking) return set_err(WC_EINVAL, "null argument");
    if (!s->eddy_on) return WC_OK;
    CK(cudaMemcpyAsync(s->st_h, breaking, s->npad * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    pack_f64_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->st_h, s->mem);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s->stream));
    return WC_OK;
}

wc_status wc_breaking_download(wc_solver* s, double* breaking) {
    if (!s || !breaking) return set_err(WC_EINVAL, "null argument");
    if (!s->eddy_on) {
        std::memset(breaking, 0, s->npad * sizeof(double));
        return WC_OK;
    }
    unpack_f64_kernel<<<aux_grid(s->npad), AUX_NT, 0, s->stream>>>(s->g, s->mem, s->st_h);
    s->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(breaking, s->st_h, s->npad * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return WC_OK;
}

wc_status wc_follow_breaking(wc_solver* s, double* h, double* hu, double* hv, double* breaking, double dt,
                             int32_t* sub_steps) {
    if (!s || !h || !hu || !hv || !breaking) return set_err(WC_EINVAL, "null argument");
    if (sub_steps) *sub_steps = 0;
    if (!s->eddy_on) return WC_OK;
    TRY(wc_state_upload(s, h, hu, hv, 0.0));
    TRY(wc_breaking_upload(s, breaking));
    set_dt_kernel<<<1, 1, 0, s->stream>>>(s->ctl, dt);
    s->launches++;
    CK(cudaMemsetAsync(s->ed_sub, 0, sizeof(int), s->stream));
    TRY(launch_eddy(s, 0, s->ed_sub));
    TRY(status_of(s));
    TRY(wc_state_download(s, h, hu, hv, nullptr));
    TRY(wc_breaking_download(s, breaking));
    int n = 0;
    CK(cudaMemcpyAsync(&n, s->ed_sub, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (sub_steps) *sub_steps = n;
    return WC_OK;
}

wc_status wc_step_device(wc_solver* s, double dt) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    clear_adaptive_kernel<<<1, 1, 0, s->stream>>>(s->ctl);
    set_dt_kernel<<<1, 1, 0, s->stream>>>(s->ctl, dt);
    s->launches += 2;
    TRY(enqueue_step(s));
    return WC_OK;
}

wc_status wc_step_n(wc_solver* s, uint64_t n_steps, double t_end) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    if (!s->rate_current) {
        state_rate_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->q0, s->ctl);
        s->launches++;
        s->rate_current = true;
    }
    set_adaptive_kernel<<<1, 1, 0, s->stream>>>(s->ctl, t_end);
    s->launches++;
    for (uint64_t n = 0; n < n_steps; n++) TRY(enqueue_step(s));
    clear_adaptive_kernel<<<1, 1, 0, s->stream>>>(s->ctl);
    s->launches++;
    CK(cudaGetLastError());
    return WC_OK;
}

wc_status wc_synchronize(wc_solver* s) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    CK(cudaStreamSynchronize(s->stream));
    return status_of(s);
}

wc_status wc_step(wc_solver* s, double* h, double* hu, double* hv, double* breaking, double* time,
                  double dt) {
    if (!s || !h || !hu || !hv || !time) return set_err(WC_EINVAL, "null argument");
    if (s->eddy_on && !breaking) return set_err(WC_EINVAL, "followed fronts need the state's breaking memory");
    TRY(wc_state_upload(s, h, hu, hv, *time));
    if (s->eddy_on) TRY(wc_breaking_upload(s, breaking));
    TRY(wc_step_device(s, dt));
    TRY(status_of(s));
    TRY(wc_state_download(s, h, hu, hv, nullptr));
    if (s->eddy_on) TRY(wc_breaking_download(s, breaking));
    else if (breaking) fill_scalar_ghosts(s->grid, s->g.periodic != 0, breaking);
    // `s.time = t + dt` (solver.rs:506)
    *time = *time + dt;
    if (s->ctl_host->unconverged != s->seen_unconverged) {
        s->seen_unconverged = s->ctl_host->unconverged;
        return set_err(WC_EUNCONVERGED, "a dispersive solve stopped at max_iterations (counted, "
                                        "as the reference does; the step is complete)");
    }
    return WC_OK;
}

wc_status wc_stable_dt(wc_solver* s, const double* h, const double* hu, const double* hv, double* dt_out) {
    if (!s || !h || !hu || !hv || !dt_out) return set_err(WC_EINVAL, "null argument");
    TRY(stage_host(s, h, hu, hv));
    Rate64Out init{0ull, ~0ull, ~0ull};
    CK(cudaMemcpyAsync(s->r64, &init, sizeof init, cudaMemcpyHostToDevice, s->stream));
    rate64_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g.nx, s->g.ny, s->g.dxd, s->g.dyd,
                                                                s->st_h, s->st_hu, s->st_hv, s->r64);
    s->launches++;
    Rate64Out res;
    CK(cudaMemcpyAsync(&res, s->r64, sizeof res, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (res.first_nan != ~0ull) {
        *dt_out = std::nan("");
        return set_err(WC_ENAN, "a cell's water is not a number");
    }
    double rate;
    std::memcpy(&rate, &res.max_bits, sizeof rate);
    *dt_out = rate > 0.0 ? s->cfl / rate : INFINITY;
    return WC_OK;
}

wc_status wc_limiting_cell(wc_solver* s, const double* h, const double* hu, const double* hv,
                           wc_limiting* out, int32_t* found) {
    if (!s || !h || !hu || !hv || !out || !found) return set_err(WC_EINVAL, "null argument");
    TRY(stage_host(s, h, hu, hv));
    Rate64Out init{0ull, ~0ull, ~0ull};
    CK(cudaMemcpyAsync(s->r64, &init, sizeof init, cudaMemcpyHostToDevice, s->stream));
    rate64_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g.nx, s->g.ny, s->g.dxd, s->g.dyd,
                                                                s->st_h, s->st_hu, s->st_hv, s->r64);
    argmax64_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g.nx, s->g.ny, s->g.dxd, s->g.dyd,
                                                                  s->st_h, s->st_hu, s->st_hv, s->r64);
    s->launches += 2;
    Rate64Out res;
    CK(cudaMemcpyAsync(&res, s->r64, sizeof res, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    unsigned long long c;
    double rate;
    std::memcpy(&rate, &res.max_bits, sizeof rate);
    if (res.first_nan != ~0ull) c = res.first_nan;
    else if (rate > 0.0) c = res.first_max;
    else {
        *found = 0;
        return WC_OK;
    }
    const size_t nx = s->grid.nx;
    const size_t i = c % nx, j = c / nx;
    const size_t k = (j + 3) * (size_t)s->W + (i + 3);
    const double hh = h[k];
    const double u = hh > 1e-8 ? hu[k] / hh : 0.0, v = hh > 1e-8 ? hv[k] / hh : 0.0;
    out->i = i;
    out->j = j;
    out->depth = hh;
    out->speed = std::hypot(u, v);
    *found = 1;
    return WC_OK;
}

wc_status wc_breaking_indicator(wc_solver* s, const double* h, const double* hu, const double* hv,
                                const double* breaking, double* out_interior) {
    if (!s || !h || !hu || !hv || !out_interior) return set_err(WC_EINVAL, "null argument");
    TRY(stage_host(s, h, hu, hv));
    upload_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->st_h, s->st_hu, s->st_hv, s->q1);
    s->launches++;
    const double* mem = nullptr;
    if (s->eddy_on && breaking) {  // the memory into scratch: the resident state's stays as it is
        CK(cudaMemcpyAsync(s->st_hu, breaking, s->npad * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        pack_f64_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->st_hu, s->mem_new);
        s->launches++;
        mem = s->mem_new;
    }
    breaking_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->q1, s->bed, s->br, mem, s->st_h);
    s->launches++;
    CK(cudaMemcpyAsync(out_interior, s->st_h, s->grid.nx * s->grid.ny * sizeof(double),
                       cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return WC_OK;
}

wc_status wc_dispersion_stats(wc_solver* s, wc_stats* out, int32_t* has) {
    if (!s || !out || !has) return set_err(WC_EINVAL, "null argument");
    if (!s->sgn) {
        *has = 0;
        return WC_OK;
    }
    TRY(read_ctl(s));
    out->solves = s->ctl_host->solves;
    out->iterations = s->ctl_host->iterations;
    out->unconverged = s->ctl_host->unconverged;
    *has = 1;
    return WC_OK;
}

wc_status wc_stable_dt_device(wc_solver* s, double* dt_out) {
    if (!s || !dt_out) return set_err(WC_EINVAL, "null argument");
    state_rate_kernel<<<aux_grid(s->ncell), AUX_NT, 0, s->stream>>>(s->g, s->q0, s->ctl);
    s->launches++;
    TRY(read_ctl(s));
    *dt_out = s->ctl_host->stable_dt;
    if (std::isnan(*dt_out)) return set_err(WC_ENAN, "a cell's water is not a number");
    return WC_OK;
}

wc_status wc_diagnostics_device(wc_solver* s, wc_diagnostics* out) {
    if (!s || !out) return set_err(WC_EINVAL, "null argument");
    const int bands = std::max(1, std::min(s->g.ny, 1024));
    diagnostics_kernel<<<bands, AUX_NT, 0, s->stream>>>(s->g, s->q0, s->diag_bands, s->diag_bands + bands,
                                                        s->diag_bands + 2 * bands, s->diag_done, s->diag_out);
    s->launches++;
    double v[3];
    CK(cudaMemcpyAsync(v, s->diag_out, sizeof v, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    out->volume = v[0];
    out->max_abs_momentum = v[1];
    out->min_depth = v[2];
    return WC_OK;
}

wc_status wc_dispersion_system(wc_solver* s, double* c, double* heff, double* bx, double* by, double* wx,
                               double* wy) {
    if (!s) return set_err(WC_EINVAL, "null argument");
    if (!s->sgn) return set_err(WC_EINVAL, "the solver has no dispersion");
    const size_t n = s->ncell;
    std::vector<float> hc(n), hh(n);
    std::vector<float2> hb(n), hw(n);
    CK(cudaMemcpyAsync(hc.data(), s->cc, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hh.data(), s->heff, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hb.data(), s->bv, n * sizeof(float2), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(hw.data(), s->w, n * sizeof(float2), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    const int nx = s->g.nx, ny = s->g.ny, pitch = s->g.pitch;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const size_t k = (size_t)j * pitch + i, o = (size_t)j * nx + i;
            if (c) c[o] = hc[k];
            if (heff) heff[o] = hh[k];
            if (bx) bx[o] = hb[k].x;
            if (by) by[o] = hb[k].y;
            if (wx) wx[o] = hw[k].x;
            if (wy) wy[o] = hw[k].y;
        }
    return WC_OK;
}

wc_status wc_time_device(wc_solver* s, double* time_out) {
    if (!s || !time_out) return set_err(WC_EINVAL, "null argument");
    TRY(read_ctl(s));
    *time_out = s->ctl_host->t;
    return WC_OK;
}

}  // extern "C"

// ---- ensembles ------------------------------------------------------------------------------

namespace {

constexpr int EN_VARIANTS = 4;  // stage tile height {8, 16} x CTAs per SM {1, 2}
// The autotuner's fifth choice: no persistent launch, every member's own captured step on its own
// stream (the only choice of a learned ensemble).
constexpr int EN_STREAMS = EN_VARIANTS;

struct EnVariant {
    int ty, minb;
    int ctas = 0;    // CTAs of the launch
    int budget = 0;  // CTAs the split may hand out (co-resident ones, at least one per member)
    std::vector<EnsembleMember> table;
    EnsembleMember* d_table = nullptr;
    int* d_cta_member = nullptr;
    cudaGraphExec_t graph = nullptr;
};

template <int TY, int MINB>
cudaError_t launch_ensemble_variant(int ctas, const EnsembleMember* table, const int* cta_member,
                                    cudaStream_t st) {
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(ctas);
    lc.blockDim = dim3(EN_NT);
    lc.dynamicSmemBytes = StageGeom<TY>::SMEM_SGN;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, ensemble_step_kernel<TY, MINB>, table, cta_member);
}

cudaError_t launch_variant(const EnVariant& v, cudaStream_t st) {
    if (v.ty == 8 && v.minb == 1) return launch_ensemble_variant<8, 1>(v.ctas, v.d_table, v.d_cta_member, st);
    if (v.ty == 8) return launch_ensemble_variant<8, 2>(v.ctas, v.d_table, v.d_cta_member, st);
    if (v.minb == 1) return launch_ensemble_variant<16, 1>(v.ctas, v.d_table, v.d_cta_member, st);
    return launch_ensemble_variant<16, 2>(v.ctas, v.d_table, v.d_cta_member, st);
}

int variant_occupancy(int ty, int minb) {
    int occ = 0;
    cudaError_t e;
    if (ty == 8 && minb == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ensemble_step_kernel<8, 1>, EN_NT, StageGeom<8>::SMEM_SGN);
    else if (ty == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ensemble_step_kernel<8, 2>, EN_NT, StageGeom<8>::SMEM_SGN);
    else if (minb == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ensemble_step_kernel<16, 1>, EN_NT, StageGeom<16>::SMEM_SGN);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ensemble_step_kernel<16, 2>, EN_NT, StageGeom<16>::SMEM_SGN);
    return e == cudaSuccess ? occ : 0;
}

}  // namespace

struct wc_ensemble {
    std::vector<wc_solver*> members;
    cudaStream_t stream = nullptr;
    unsigned* counters = nullptr;   // [members][2]: group barrier arrivals and released epoch
    double* partials = nullptr;     // [members][max ctas][4]
    int max_ctas = 0;
    EnVariant var[EN_VARIANTS];
    int chosen = -1;
    double tune_ms[EN_VARIANTS + 1] = {0, 0, 0, 0, 0};
    // snapshot of the resident states for tuning trials
    std::vector<float4*> snap_q;
    std::vector<float2*> snap_w;
    unsigned long long launches = 0;
    // Work per member and step, the persistent launch's CTA split: algorithmic bytes per cell of
    // a step times cells (shallow water 88; dispersive 368 + 192 I with I the member's measured
    // PCG iterations per solve, 55 until the autotuner has measured it).
    std::vector<double> work;
    bool work_measured = false;
    // Every member has its own stream: with the EN_STREAMS choice (and always with a learned
    // preconditioner, wc_ensemble_set_lpc) every member steps through its own captured step on it;
    // a step forks from the ensemble's stream to the members' and joins back.
    bool learned = false;
    std::vector<cudaStream_t> member_streams;
    std::vector<cudaEvent_t> member_done;
    cudaEvent_t fork = nullptr;

    ~wc_ensemble() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& v : var) {
            if (v.graph) cudaGraphExecDestroy(v.graph);
            if (v.d_table) cudaFree(v.d_table);
            if (v.d_cta_member) cudaFree(v.d_cta_member);
        }
        for (auto p : snap_q) cudaFree(p);
        for (auto p : snap_w) cudaFree(p);
        if (counters) cudaFree(counters);
        if (partials) cudaFree(partials);
        for (auto m : members) wc_solver_destroy(m);
        for (auto ev : member_done) cudaEventDestroy(ev);
        if (fork) cudaEventDestroy(fork);
        for (auto st : member_streams) cudaStreamDestroy(st);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Split `ctas` CTAs over the members in proportion to their work per step (at least one each, at
// most one per PCG or stage tile), and fill the member table of one variant.
wc_status build_variant(wc_ensemble* e, EnVariant& v, int ctas) {
    const size_t n = e->members.size();
    std::vector<double> cells(n);  // the member's work, in the units of e->work
    double total = 0;
    std::vector<int> cap(n);
    for (size_t m = 0; m < n; m++) {
        cells[m] = e->work[m];
        total += cells[m];
        const int tiles_pcg = e->members[m]->pcg_tiles_x * e->members[m]->pcg_tiles_y;
        const int tiles_st = ((e->members[m]->g.nx + ST_TX - 1) / ST_TX) * ((e->members[m]->g.ny + v.ty - 1) / v.ty);
        cap[m] = std::max(1, std::min(e->max_ctas, std::max(tiles_pcg, tiles_st)));
    }
    std::vector<int> share(n);
    int used = 0;
    for (size_t m = 0; m < n; m++) {
        share[m] = std::max(1, std::min(cap[m], (int)std::floor(ctas * cells[m] / total)));
        used += share[m];
    }
    // hand out what is left to the members with the most cells per CTA
    while (used < ctas) {
        int best = -1;
        double worst = -1;
        for (size_t m = 0; m < n; m++)
            if (share[m] < cap[m] && cells[m] / share[m] > worst) {
                worst = cells[m] / share[m];
                best = (int)m;
            }
        if (best < 0) break;
        share[best]++;
        used++;
    }
    v.ctas = used;
    v.table.assign(n, EnsembleMember{});
    std::vector<int> cta_member(used);
    int first = 0;
    for (size_t m = 0; m < n; m++) {
        wc_solver* s = e->members[m];
        EnsembleMember& M = v.table[m];
        M.sgn = s->sgn;
        M.order = s->order;
        M.first_cta = first;
        M.ncta = share[m];
        for (int c = 0; c < share[m]; c++) cta_member[first + c] = (int)m;
        first += share[m];
        if (s->sgn) {
            M.st[0] = stage_args(s, s->q0, s->q0, s->q1, false);
            M.st[1] = stage_args(s, s->q1, s->q0, s->q1, true);
        } else {
            M.st[0] = stage_args(s, s->q0, s->q0, s->q1, false);
            M.st[1] = stage_args(s, s->q1, s->q0, s->q0, true);
        }
        M.pcg[0] = pcg_args(s, MODE_STAGE1, s->q0, s->q1);
        M.pcg[1] = pcg_args(s, MODE_STAGE2, s->q0, s->q0);
        for (int k = 0; k < 2; k++) {
            M.pcg[k].cnt = e->counters + 2 * m;
            M.pcg[k].part = e->partials + 8 * (size_t)m * e->max_ctas;
        }
    }
    if (v.graph) {  // the captured launch holds the previous grid size
        CK(cudaGraphExecDestroy(v.graph));
        v.graph = nullptr;
    }
    if (!v.d_table) CK(cudaMalloc(&v.d_table, n * sizeof(EnsembleMember)));
    if (!v.d_cta_member) CK(cudaMalloc(&v.d_cta_member, (size_t)e->max_ctas * EN_VARIANTS * sizeof(int)));
    CK(cudaMemcpy(v.d_table, v.table.data(), n * sizeof(EnsembleMember), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(v.d_cta_member, cta_member.data(), used * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(0));
    return WC_OK;
}

// One ensemble step through the variant's captured graph (counters cleared, then the launch).
wc_status ensemble_step(wc_ensemble* e, EnVariant& v) {
    if (!v.graph) {
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = cudaMemsetAsync(e->counters, 0, 2 * e->members.size() * sizeof(unsigned), e->stream);
        cudaError_t e2 = launch_variant(v, e->stream);
        cudaError_t e3 = cudaStreamEndCapture(e->stream, &graph);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
            return set_err(WC_ECUDA, std::string("capturing the ensemble step failed: ") +
                                         cudaGetErrorString(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3)));
        cudaError_t e4 = cudaGraphInstantiate(&v.graph, graph, 0);
        cudaGraphDestroy(graph);
        CK(e4);
    }
    CK(cudaGraphLaunch(v.graph, e->stream));
    e->launches++;
    return WC_OK;
}

wc_status ensemble_prepare(wc_ensemble* e, double t_end) {
    for (wc_solver* s : e->members) {
        if (!s->rate_current) {
            state_rate_kernel<<<aux_grid(s->ncell), AUX_NT, 0, e->stream>>>(s->g, s->q0, s->ctl);
            s->rate_current = true;
            e->launches++;
        }
        set_adaptive_kernel<<<1, 1, 0, e->stream>>>(s->ctl, t_end);
        e->launches++;
    }
    CK(cudaGetLastError());
    return WC_OK;
}

wc_status ensemble_finish(wc_ensemble* e) {
    for (wc_solver* s : e->members) {
        clear_adaptive_kernel<<<1, 1, 0, e->stream>>>(s->ctl);
        e->launches++;
    }
    CK(cudaGetLastError());
    return WC_OK;
}

// Work per member and step from the cells and the PCG iterations per solve (see wc_ensemble).
double member_work(const wc_solver* s, double iterations) {
    const double cells = (double)s->g.nx * s->g.ny;
    return s->sgn ? cells * (368.0 + 192.0 * iterations) : cells * 88.0;
}

// One step of a learned ensemble: every member's own step graph on its own stream, forked from
// and joined back to the ensemble's stream.
wc_status ensemble_step_members(wc_ensemble* e) {
    CK(cudaEventRecord(e->fork, e->stream));
    for (size_t m = 0; m < e->members.size(); m++) {
        wc_solver* s = e->members[m];
        CK(cudaStreamWaitEvent(s->stream, e->fork, 0));
        TRY(enqueue_step(s));
        CK(cudaEventRecord(e->member_done[m], s->stream));
        CK(cudaStreamWaitEvent(e->stream, e->member_done[m], 0));
    }
    e->launches++;
    return WC_OK;
}

// The autotuner: every compiled variant runs `trial` steps on a snapshot of the live state
// (timed with events on the ensemble's stream), the state and clocks are restored after each,
// and the fastest variant is kept. Before that, on its first call, one trial of the cell-split
// launch measures each member's PCG iterations per solve, and the CTAs of every variant are
// split again by the work that gives. A learned ensemble has no variants: its trial times the
// members' own steps.
wc_status ensemble_tune(wc_ensemble* e, int trial) {
    const size_t n = e->members.size();
    if (e->snap_q.empty()) {
        for (wc_solver* s : e->members) {
            float4* q = nullptr;
            float2* w = nullptr;
            TRY(dalloc(&q, s->ncell));
            if (s->sgn) TRY(dalloc(&w, s->ncell));
            e->snap_q.push_back(q);
            e->snap_w.push_back(w);
        }
    }
    std::vector<Ctl> ctl(n);
    for (size_t m = 0; m < n; m++) {
        wc_solver* s = e->members[m];
        CK(cudaMemcpyAsync(e->snap_q[m], s->q0, s->ncell * sizeof(float4), cudaMemcpyDeviceToDevice, e->stream));
        if (s->sgn) CK(cudaMemcpyAsync(e->snap_w[m], s->w, s->ncell * sizeof(float2), cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(&ctl[m], s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->stream));
    }
    CK(cudaStreamSynchronize(e->stream));
    auto restore = [&]() -> wc_status {
        for (size_t m = 0; m < n; m++) {  // the state, the warm start and the clock
            wc_solver* s = e->members[m];
            CK(cudaMemcpyAsync(s->q0, e->snap_q[m], s->ncell * sizeof(float4), cudaMemcpyDeviceToDevice, e->stream));
            if (s->sgn) CK(cudaMemcpyAsync(s->w, e->snap_w[m], s->ncell * sizeof(float2), cudaMemcpyDeviceToDevice, e->stream));
            CK(cudaMemcpyAsync(s->ctl, &ctl[m], sizeof(Ctl), cudaMemcpyHostToDevice, e->stream));
            s->rate_current = false;
        }
        CK(cudaStreamSynchronize(e->stream));
        return WC_OK;
    };
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    if (e->learned) {
        TRY(ensemble_prepare(e, INFINITY));
        TRY(ensemble_step_members(e));  // capture and warm
        CK(cudaEventRecord(a, e->stream));
        for (int t = 0; t < trial; t++) TRY(ensemble_step_members(e));
        CK(cudaEventRecord(b, e->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        for (int k = 0; k < EN_VARIANTS; k++) e->tune_ms[k] = -1.0;
        e->tune_ms[EN_STREAMS] = ms / trial;
        e->chosen = EN_STREAMS;
        TRY(restore());
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        TRY(ensemble_finish(e));
        return WC_OK;
    }
    if (!e->work_measured) {
        int k0 = 0;
        while (k0 < EN_VARIANTS && e->var[k0].ctas <= 0) k0++;
        if (k0 < EN_VARIANTS) {
            TRY(ensemble_prepare(e, INFINITY));
            for (int t = 0; t < std::max(1, trial); t++) TRY(ensemble_step(e, e->var[k0]));
            CK(cudaStreamSynchronize(e->stream));
            for (size_t m = 0; m < n; m++) {
                wc_solver* s = e->members[m];
                Ctl c{};
                CK(cudaMemcpy(&c, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
                const unsigned long long solves = c.solves - ctl[m].solves;
                const double it = solves ? (double)(c.iterations - ctl[m].iterations) / (double)solves : 55.0;
                e->work[m] = member_work(s, it);
            }
            TRY(restore());
            for (int k = 0; k < EN_VARIANTS; k++)
                if (e->var[k].ctas > 0) TRY(build_variant(e, e->var[k], e->var[k].budget));
        }
        e->work_measured = true;
    }
    double best = 1e300;
    for (int k = 0; k < EN_VARIANTS; k++) {
        if (e->var[k].ctas <= 0) {
            e->tune_ms[k] = -1.0;
            continue;
        }
        TRY(ensemble_prepare(e, INFINITY));
        TRY(ensemble_step(e, e->var[k]));  // capture and warm
        CK(cudaEventRecord(a, e->stream));
        for (int t = 0; t < trial; t++) TRY(ensemble_step(e, e->var[k]));
        CK(cudaEventRecord(b, e->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        e->tune_ms[k] = ms / trial;
        if (ms < best) {
            best = ms;
            e->chosen = k;
        }
        TRY(restore());
    }
    {  // the members' own steps on their own streams
        TRY(ensemble_prepare(e, INFINITY));
        TRY(ensemble_step_members(e));  // capture and warm
        CK(cudaEventRecord(a, e->stream));
        for (int t = 0; t < trial; t++) TRY(ensemble_step_members(e));
        CK(cudaEventRecord(b, e->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        e->tune_ms[EN_STREAMS] = ms / trial;
        if (ms < best) {
            best = ms;
            e->chosen = EN_STREAMS;
        }
        TRY(restore());
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e->chosen < 0) return set_err(WC_ECUDA, "no ensemble kernel variant can run on this device");
    TRY(ensemble_finish(e));
    return WC_OK;
}

}  // namespace

extern "C" {

wc_status wc_ensemble_create(uint64_t n, const wc_grid* grids, const double* const* beds,
                             const wc_config* cfgs, wc_ensemble** out) {
    if (!out) return set_err(WC_EINVAL, "out is null");
    *out = nullptr;
    if (n == 0 || !grids || !beds || !cfgs) return set_err(WC_EINVAL, "an ensemble needs members");
    for (uint64_t m = 0; m < n; m++) {
        if (cfgs[m].order == WC_ORDER_FIRST)
            return set_err(WC_EUNSUPPORTED, "ensemble members run second or fifth order (SSP-RK2)");
        if (cfgs[m].dispersion && cfgs[m].dispersion->breaking.viscosity)
            return set_err(WC_EUNSUPPORTED, "ensemble members do not follow breaking fronts (Breaking::viscosity)");
    }
    wc_ensemble* e = new wc_ensemble();
    auto fail = [&](wc_status st) {
        delete e;
        return st;
    };
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "cudaStreamCreate failed"));
    if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "cudaEventCreate failed"));
    for (uint64_t m = 0; m < n; m++) {
        wc_solver* s = nullptr;
        wc_status st = wc_solver_create(&grids[m], beds[m], &cfgs[m], &s);
        if (st != WC_OK) return fail(st);
        e->members.push_back(s);
        cudaStream_t ms = nullptr;
        cudaEvent_t ev = nullptr;
        if (cudaStreamCreateWithFlags(&ms, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            return fail(set_err(WC_ECUDA, "cudaStreamCreate failed"));
        e->member_streams.push_back(ms);
        e->member_done.push_back(ev);
        s->stream = ms;  // the member's own steps; the persistent launches run on the ensemble's stream
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tys[2] = {8, 16};
    int max_ctas = 0;
    for (int k = 0; k < EN_VARIANTS; k++) {
        e->var[k].ty = tys[k / 2];
        e->var[k].minb = 1 + (k % 2);
        const int occ = std::min(variant_occupancy(e->var[k].ty, e->var[k].minb), e->var[k].minb);
        e->var[k].ctas = occ * sms;
        max_ctas = std::max(max_ctas, e->var[k].ctas);
    }
    if (max_ctas <= 0) return fail(set_err(WC_ECUDA, "no ensemble kernel variant fits on this device"));
    if ((int)n > max_ctas) return fail(set_err(WC_EUNSUPPORTED, "more members than co-resident CTAs"));
    e->max_ctas = max_ctas;
    wc_status st;
    if ((st = dalloc(&e->counters, 2 * n)) != WC_OK) return fail(st);
    if ((st = dalloc(&e->partials, 8 * n * (size_t)max_ctas)) != WC_OK) return fail(st);
    e->work.resize(n);
    for (uint64_t m = 0; m < n; m++) e->work[m] = member_work(e->members[m], 55.0);
    for (int k = 0; k < EN_VARIANTS; k++) {
        if (e->var[k].ctas <= 0) continue;
        e->var[k].budget = std::max((int)n, e->var[k].ctas);
        if ((st = build_variant(e, e->var[k], e->var[k].budget)) != WC_OK) return fail(st);
    }
    *out = e;
    return WC_OK;
}

wc_status wc_ensemble_set_lpc(wc_ensemble* e, wc_lpc* l) {
    if (!e || !l) return set_err(WC_EINVAL, "null argument");
    if (e->learned) return set_err(WC_EINVAL, "the ensemble already has a learned preconditioner");
    CK(cudaStreamSynchronize(e->stream));
    for (wc_solver* s : e->members)
        if (s->sgn) TRY(wc_solver_set_lpc(s, l));
    e->learned = true;
    e->chosen = EN_STREAMS;
    return WC_OK;
}

void wc_ensemble_destroy(wc_ensemble* e) { delete e; }

wc_status wc_ensemble_upload(wc_ensemble* e, uint64_t m, const double* h, const double* hu, const double* hv,
                             double time) {
    if (!e || m >= e->members.size()) return set_err(WC_EINVAL, "no such member");
    return wc_state_upload(e->members[m], h, hu, hv, time);
}

wc_status wc_ensemble_download(wc_ensemble* e, uint64_t m, double* h, double* hu, double* hv, double* time) {
    if (!e || m >= e->members.size()) return set_err(WC_EINVAL, "no such member");
    return wc_state_download(e->members[m], h, hu, hv, time);
}

wc_status wc_ensemble_autotune(wc_ensemble* e, uint32_t trial_steps, int32_t* choice, double* ms_per_step) {
    if (!e) return set_err(WC_EINVAL, "null ensemble");
    TRY(ensemble_tune(e, (int)std::max<uint32_t>(1, trial_steps)));
    if (choice) *choice = e->chosen;
    if (ms_per_step)
        for (int k = 0; k <= EN_STREAMS; k++) ms_per_step[k] = e->tune_ms[k];
    return WC_OK;
}

wc_status wc_ensemble_step_n(wc_ensemble* e, uint64_t n_steps, double t_end) {
    if (!e) return set_err(WC_EINVAL, "null ensemble");
    if (e->chosen < 0) TRY(ensemble_tune(e, 2));
    TRY(ensemble_prepare(e, t_end));
    for (uint64_t k = 0; k < n_steps; k++) {
        if (e->chosen == EN_STREAMS) TRY(ensemble_step_members(e));
        else TRY(ensemble_step(e, e->var[e->chosen]));
    }
    TRY(ensemble_finish(e));
    return WC_OK;
}

wc_status wc_ensemble_synchronize(wc_ensemble* e) {
    if (!e) return set_err(WC_EINVAL, "null ensemble");
    CK(cudaStreamSynchronize(e->stream));
    for (wc_solver* s : e->members) TRY(status_of(s));
    return WC_OK;
}

wc_status wc_ensemble_member_stats(wc_ensemble* e, uint64_t m, wc_stats* stats, double* time) {
    if (!e || m >= e->members.size()) return set_err(WC_EINVAL, "no such member");
    wc_solver* s = e->members[m];
    TRY(read_ctl(s));
    if (stats) {
        stats->solves = s->ctl_host->solves;
        stats->iterations = s->ctl_host->iterations;
        stats->unconverged = s->ctl_host->unconverged;
    }
    if (time) *time = s->ctl_host->t;
    return WC_OK;
}

uint64_t wc_ensemble_launch_count(const wc_ensemble* e) {
    if (!e) return 0;
    uint64_t n = e->launches;
    for (const wc_solver* s : e->members) n += wc_launch_count(s);  // the members' own steps' kernels
    return n;
}

}  // extern "C"

// ---- the learned preconditioner ---------------------------------------------------------------

struct wc_lpc {
    LpcModel m;
};

namespace {

wc_status lpc_ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return set_err(WC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return WC_OK;
}

// Scaled normal weights (standard deviation sqrt(1 / fan-in)), zero biases, a zero output layer:
// the untrained network adds nothing to the two Jacobi sweeps.
void lpc_init_host(const LpcNet& net, uint64_t seed, std::vector<float>& p) {
    p.assign(net.nparams, 0.f);
    unsigned long long st = seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
    auto uni = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](const LpcLayer& L) {
        const double sd = std::sqrt(1.0 / (L.ci * L.k * L.k));
        for (int q = 0; q < L.co * L.ci * L.k * L.k; q++) {
            const double u1 = uni(), u2 = uni();  // Box-Muller
            p[L.w + q] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(TAU * u2));
        }
    };
    for (auto* L : {&net.enc_a, &net.enc_b, &net.dec_a, &net.dec_b, &net.gate_a, &net.gate_b})
        for (auto& l : *L)
            if (l.co > 0) fill(l);
}

}  // namespace

extern "C" {

wc_status wc_lpc_create(const int32_t* channels, int32_t gate_hidden, int32_t stride, uint64_t seed, wc_lpc** out) {
    if (!out) return set_err(WC_EINVAL, "out is null");
    *out = nullptr;
    int ch[LPC_LEVELS] = {8, 16, 32, 32};
    if (channels)
        for (int l = 0; l < LPC_LEVELS; l++) ch[l] = channels[l];
    for (int l = 0; l < LPC_LEVELS; l++)
        if (ch[l] < 1 || ch[l] > 256) return set_err(WC_EINVAL, "channels must be in 1..256");
    if (gate_hidden < 1 || gate_hidden > 256) return set_err(WC_EINVAL, "gate_hidden must be in 1..256");
    if (stride != 1 && stride != 2 && stride != 4) return set_err(WC_EINVAL, "stride must be 1, 2 or 4");
    wc_lpc* l = new wc_lpc();
    wc_status st = lpc_ck(l->m.init(ch, gate_hidden, stride), "network allocation");
    if (st == WC_OK) {
        std::vector<float> p;
        lpc_init_host(l->m.net, seed, p);
        st = lpc_ck(cudaMemcpy(l->m.w.p, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
        if (st == WC_OK) st = lpc_ck(cudaStreamSynchronize(0), "upload");
        if (st == WC_OK) st = lpc_ck(l->m.refresh(), "refresh");
        if (st == WC_OK) st = lpc_ck(cudaStreamSynchronize(l->m.st), "init");
    }
    if (st != WC_OK) {
        delete l;
        return st;
    }
    *out = l;
    return WC_OK;
}

void wc_lpc_destroy(wc_lpc* l) {
    if (l) cudaStreamSynchronize(l->m.st);
    delete l;
}

uint64_t wc_lpc_num_params(const wc_lpc* l) { return l ? (uint64_t)l->m.net.nparams : 0; }

wc_status wc_lpc_set_params(wc_lpc* l, const float* params, uint64_t n) {
    if (!l || !params) return set_err(WC_EINVAL, "null argument");
    if (n != (uint64_t)l->m.net.nparams) return set_err(WC_EINVAL, "parameter count mismatch");
    LpcModel& m = l->m;
    TRY(lpc_ck(cudaMemcpyAsync(m.w.p, params, n * sizeof(float), cudaMemcpyHostToDevice, m.st), "upload"));
    TRY(lpc_ck(cudaMemsetAsync(m.m.p, 0, n * sizeof(float), m.st), "memset"));
    TRY(lpc_ck(cudaMemsetAsync(m.v.p, 0, n * sizeof(float), m.st), "memset"));
    m.adam_t = 0;
    TRY(lpc_ck(m.refresh(), "refresh"));
    return lpc_ck(cudaStreamSynchronize(m.st), "set_params");
}

wc_status wc_lpc_get_params(wc_lpc* l, float* params, uint64_t n) {
    if (!l || !params) return set_err(WC_EINVAL, "null argument");
    if (n != (uint64_t)l->m.net.nparams) return set_err(WC_EINVAL, "parameter count mismatch");
    TRY(lpc_ck(cudaMemcpyAsync(params, l->m.w.p, n * sizeof(float), cudaMemcpyDeviceToHost, l->m.st), "download"));
    return lpc_ck(cudaStreamSynchronize(l->m.st), "get_params");
}

wc_status wc_lpc_set_rounding(wc_lpc* l, int32_t bf16) {
    if (!l) return set_err(WC_EINVAL, "null network");
    l->m.round_bf16 = bf16 ? 1 : 0;
    TRY(lpc_ck(l->m.refresh(), "refresh"));
    return lpc_ck(cudaStreamSynchronize(l->m.st), "set_rounding");
}

wc_status wc_lpc_forward_backward(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* x, const float* feat,
                                  const float* dy, float* y, float* grad, float* dx) {
    if (!l || !x || !feat || !dy || !y || !grad || !dx) return set_err(WC_EINVAL, "null argument");
    const int div = 1 << (LPC_LEVELS - 1);
    if (n < 1 || h < div || w < div || h % div || w % div)
        return set_err(WC_EINVAL, "batch must be >= 1 and patch sides positive multiples of 8");
    LpcModel& m = l->m;
    LpcNet& net = m.net;
    cudaStream_t st = m.st;
    const size_t per = (size_t)n * 2 * h * w;
    TRY(lpc_ck(net.shape(n, h, w, true), "activations"));
    DBuf ddy, ddx;
    TRY(lpc_ck(ddy.alloc(per), "alloc"));
    TRY(lpc_ck(ddx.alloc(per), "alloc"));
    TRY(lpc_ck(cudaMemcpyAsync(net.X[0].p, x, per * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(net.F[0].p, feat, per * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(ddy.p, dy, per * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(net.gates(st), "gates"));
    TRY(lpc_ck(net.forward(st, true), "forward"));
    TRY(lpc_ck(cudaMemsetAsync(m.g.p, 0, m.g.n * sizeof(float), st), "memset"));
    TRY(lpc_ck(net.backward(ddy.p, ddx.p, st), "backward"));
    TRY(lpc_ck(cudaMemcpyAsync(y, net.Y.p, per * sizeof(float), cudaMemcpyDeviceToHost, st), "download"));
    TRY(lpc_ck(cudaMemcpyAsync(grad, m.g.p, (size_t)net.nparams * sizeof(float), cudaMemcpyDeviceToHost, st), "download"));
    TRY(lpc_ck(cudaMemcpyAsync(dx, ddx.p, per * sizeof(float), cudaMemcpyDeviceToHost, st), "download"));
    return lpc_ck(cudaStreamSynchronize(st), "forward_backward");
}

wc_status wc_lpc_forward(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* x, const float* feat,
                         int32_t tensor, float* y) {
    if (!l || !x || !feat || !y) return set_err(WC_EINVAL, "null argument");
    const int div = 1 << (LPC_LEVELS - 1);
    if (n < 1 || h < div || w < div || h % div || w % div)
        return set_err(WC_EINVAL, "batch must be >= 1 and map sides positive multiples of 8");
    LpcModel& m = l->m;
    LpcNet net;  // an inference instance: the model's layout and weights, its own activations
    net.layout(m.net.ch, m.net.hidden);
    net.wq = m.wq.p;
    net.tensor = tensor != 0;
    net.fuse_level0 = tensor != 2;
    net.small_tiles = tensor != 3;
    net.configure_nhwc();
    cudaStream_t st = m.st;
    if (net.tensor) {
        TRY(lpc_ck(conv_mma_configure(), "configure"));
        TRY(lpc_ck(net.prepare_tensor(st), "weights"));
    }
    const size_t per = (size_t)n * 2 * h * w;
    TRY(lpc_ck(net.shape(n, h, w, false), "activations"));
    TRY(lpc_ck(cudaMemcpyAsync(net.X[0].p, x, per * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(net.F[0].p, feat, per * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    if (net.nhwc) {  // the solver's path: NHWC BF16 activations
        to_h_kernel<<<ew_grid(per / 2), 256, 0, st>>>(net.X[0].p, n, 2, h, w, LpcNet::hp(net.Xh));
        TRY(lpc_ck(net.gates_h(st), "gates"));
        TRY(lpc_ck(net.forward_h(st), "forward"));
        from_h_kernel<<<ew_grid(per / 2), 256, 0, st>>>(net.Yh.p, n, h, w, net.Y.p);
        TRY(lpc_ck(cudaGetLastError(), "forward"));
    } else {
        TRY(lpc_ck(net.gates(st), "gates"));
        TRY(lpc_ck(net.forward(st, false), "forward"));
    }
    TRY(lpc_ck(cudaMemcpyAsync(y, net.Y.p, per * sizeof(float), cudaMemcpyDeviceToHost, st), "download"));
    return lpc_ck(cudaStreamSynchronize(st), "forward");
}

wc_status wc_lpc_harvest(wc_lpc* l, wc_solver* s) {
    if (!l || !s) return set_err(WC_EINVAL, "null argument");
    if (!s->sgn) return set_err(WC_EINVAL, "the solver has no dispersive solve to harvest");
    TRY(lpc_ck(cudaStreamSynchronize(s->stream), "harvest"));
    auto* q = new LpcSystem();
    q->nx = (int)s->grid.nx;
    q->ny = (int)s->grid.ny;
    q->pitch = s->g.pitch;
    q->dx = (float)s->grid.dx;
    q->dy = (float)s->grid.dy;
    wc_status st = WC_OK;
    for (auto pr : {std::make_pair(&q->c, (const float*)s->cc), std::make_pair(&q->heff, (const float*)s->heff),
                    std::make_pair(&q->bed, (const float*)s->bed)}) {
        if (st == WC_OK) st = lpc_ck(pr.first->alloc(s->ncell), "alloc");
        if (st == WC_OK)
            st = lpc_ck(cudaMemcpy(pr.first->p, pr.second, s->ncell * sizeof(float), cudaMemcpyDeviceToDevice), "copy");
    }
    if (st == WC_OK) st = lpc_ck(cudaStreamSynchronize(0), "copy");  // device copies return early
    if (st != WC_OK) {
        delete q;
        return st;
    }
    l->m.systems.push_back(q);
    return WC_OK;
}

uint64_t wc_lpc_num_systems(const wc_lpc* l) { return l ? l->m.systems.size() : 0; }

wc_status wc_lpc_train(wc_lpc* l, uint32_t steps, uint32_t batch, uint32_t patch, float lr, float rough, uint64_t seed,
                       double* losses) {
    if (!l) return set_err(WC_EINVAL, "null network");
    LpcModel& m = l->m;
    if (m.systems.empty()) return set_err(WC_EINVAL, "no harvested systems");
    const uint32_t div = (1u << (LPC_LEVELS - 1)) * (uint32_t)m.stride;
    if (batch < 1 || batch > 4096 || patch < div || patch % div || patch > 4096)
        return set_err(WC_EINVAL, "batch must be in 1..4096 and the patch side a multiple of 8 x stride up to 4096");
    bool fits = false;
    for (auto* q : m.systems) fits = fits || ((uint32_t)q->nx >= patch && (uint32_t)q->ny >= patch);
    if (!fits) return set_err(WC_EINVAL, "no harvested system is as large as the patch");
    if (steps == 0) return WC_OK;
    if (m.dloss_n < steps) {
        if (m.dloss) cudaFree(m.dloss);
        m.dloss = nullptr;
        m.dloss_n = 0;
        TRY(lpc_ck(cudaMalloc(&m.dloss, steps * sizeof(double)), "alloc"));
        m.dloss_n = steps;
    }
    m.rng = seed * 0x9e3779b97f4a7c15ull + 0x2545f4914f6cdd1dull;
    if (m.rng == 0) m.rng = 1;
    for (uint32_t k = 0; k < steps; k++) {
        const cudaError_t e = m.train_step((int)batch, (int)patch, (int)patch, lr, m.dloss + k, rough);
        if (e == cudaErrorInvalidValue) return set_err(WC_EINVAL, "no harvested system of one spacing fits the patch");
        TRY(lpc_ck(e, "training step"));
    }
    if (losses)
        TRY(lpc_ck(cudaMemcpyAsync(losses, m.dloss, steps * sizeof(double), cudaMemcpyDeviceToHost, m.st), "download"));
    return lpc_ck(cudaStreamSynchronize(m.st), "train");
}

wc_status wc_lpc_loss_grad(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* c, const float* heff,
                           const float* bed, const float* e, double dx, double dy, double* loss, float* grad) {
    if (!l || !c || !heff || !bed || !e || !loss || !grad) return set_err(WC_EINVAL, "null argument");
    LpcModel& m = l->m;
    const int div = (1 << (LPC_LEVELS - 1)) * m.stride;
    if (n < 1 || h < div || w < div || h % div || w % div)
        return set_err(WC_EINVAL, "batch must be >= 1 and patch sides positive multiples of 8 x stride");
    if (!(dx > 0.0 && dy > 0.0)) return set_err(WC_EINVAL, "cell size must be positive");
    cudaStream_t st = m.st;
    TRY(lpc_ck(m.shape_batch(n, h, w), "activations"));
    const size_t plane = (size_t)n * h * w;
    DBuf dbed;
    TRY(lpc_ck(dbed.alloc(plane), "alloc"));
    TRY(lpc_ck(cudaMemcpyAsync(m.tr.c.p, c, plane * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(m.tr.heff.p, heff, plane * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(dbed.p, bed, plane * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    TRY(lpc_ck(cudaMemcpyAsync(m.tr.e.p, e, 2 * plane * sizeof(float), cudaMemcpyHostToDevice, st), "upload"));
    for (int k = 0; k < n; k++) {  // mask and features of each patch, as the crops make them
        const size_t hw = (size_t)h * w;
        crop_kernel<<<ew_grid(hw), 256, 0, st>>>(m.tr.c.p + k * hw, m.tr.heff.p + k * hw, dbed.p + k * hw, w, 0, 0, h, w,
                                                 m.tr.c.p + k * hw, m.tr.heff.p + k * hw, m.tr.mask.p + k * hw,
                                                 m.fine_features() + 2 * k * hw);
    }
    TRY(lpc_ck(m.pool_features(), "features"));
    m.tr.dx = (float)dx;
    m.tr.dy = (float)dy;
    double* dl = nullptr;
    TRY(lpc_ck(cudaMalloc(&dl, sizeof(double)), "alloc"));
    wc_status stt = lpc_ck(m.loss_grad(dl, true), "loss_grad");
    if (stt == WC_OK) stt = lpc_ck(cudaMemcpyAsync(loss, dl, sizeof(double), cudaMemcpyDeviceToHost, st), "download");
    if (stt == WC_OK)
        stt = lpc_ck(cudaMemcpyAsync(grad, m.g.p, (size_t)m.net.nparams * sizeof(float), cudaMemcpyDeviceToHost, st),
                     "download");
    if (stt == WC_OK) stt = lpc_ck(cudaStreamSynchronize(st), "loss_grad");
    cudaFree(dl);
    return stt;
}

wc_status wc_solver_set_lpc(wc_solver* s, wc_lpc* l) {
    if (!s) return set_err(WC_EINVAL, "null solver");
    if (!s->sgn) return set_err(WC_EINVAL, "the solver has no dispersive solve");
    CK(cudaStreamSynchronize(s->stream));
    Ctl c{};
    CK(cudaMemcpy(&c, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
    if (s->fcg_body_launches) s->launches += s->fcg_body_launches * (c.fcg_iterations - s->fcg_iter_base);
    s->fcg_body_launches = 0;
    if (s->step_graph) {  // the captured step names the previous method's buffers
        cudaGraphExecDestroy(s->step_graph);
        s->step_graph = nullptr;
    }
    if (!l) {
        s->lpc = nullptr;
        s->pc = WC_PC_JACOBI;
        return WC_OK;
    }
    if (l->m.net.nparams == 0) return set_err(WC_EINVAL, "network not initialised");
    const int div = 1 << (LPC_LEVELS - 1);
    const int S = l->m.stride;  // the network's grid: ceil(n / S) cells, padded to a multiple of 8
    s->lpc_hp = ((int)s->grid.ny + div * S - 1) / (div * S) * div;
    s->lpc_wp = ((int)s->grid.nx + div * S - 1) / (div * S) * div;
    s->lnet.layout(l->m.net.ch, l->m.net.hidden);
    s->lnet.wq = l->m.wq.p;
    s->lnet.gw = nullptr;
    s->lnet.tensor = true;  // the solve applies the network on the tensor cores
    {
        const char* v = std::getenv("WAVECORE_B200_LPC_SMALL_TILES");  // 0: usual tiles everywhere
        s->lnet.small_tiles = !(v && std::strcmp(v, "0") == 0);
    }
    s->lnet.configure_nhwc();
    CK(conv_mma_configure());
    CK(s->lnet.prepare_tensor(s->stream));
    CK(cudaStreamSynchronize(s->stream));
    CK(s->lnet.shape(1, s->lpc_hp, s->lpc_wp, false));
    if (!s->tv) {
        CK(cudaMalloc(&s->tv, s->ncell * sizeof(float2)));
        CK(cudaMemset(s->tv, 0, s->ncell * sizeof(float2)));
        CK(cudaMalloc(&s->fsc, sizeof(FcgScalars)));
        CK(cudaMemset(s->fsc, 0, sizeof(FcgScalars)));
        CK(cudaStreamSynchronize(0));
        CK(cudaMalloc(&s->fpart, 3 * std::max(FCG_BLOCKS, FCG_TILE_BLOCKS) * sizeof(double)));
        CK(cudaMallocHost(&s->done_host, sizeof(int)));
        CK(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    }
    s->lnet.done = &s->fsc->done;
    // training and inference may run on different streams: the weights are final from here
    CK(cudaStreamSynchronize(l->m.st));
    s->lpc = &l->m;
    s->pc = WC_PC_LEARNED;
    s->fcg_iter_base = c.fcg_iterations;  // the kernels per iteration are counted at the first solve
    return WC_OK;
}

}  // extern "C"

// ---- per-step statistics and frames -----------------------------------------------------------

struct wc_recorder {
    wc_solver* s = nullptr;  // cleared when the solver goes first
    RecDev* rd = nullptr;
    RecArrays ra{};
    double* block = nullptr;  // one allocation behind every array of ra
    size_t cells = 0;
    ~wc_recorder() {
        if (rd) cudaFree(rd);
        if (block) cudaFree(block);
    }
};

wc_solver::~wc_solver() {
    if (rec) rec->s = nullptr;
    free_all();
}

namespace {

wc_status enqueue_record(wc_solver* s) {
    wc_recorder* r = s->rec;
    const size_t cells = r->cells;
    const unsigned blocks = (unsigned)std::min<size_t>(148 * 8, (cells + 255) / 256);
    record_cells_kernel<<<blocks, 256, 0, s->stream>>>(s->g, s->q0, s->bed, s->br, s->eddy_on ? s->mem : nullptr,
                                                       s->ctl, r->rd, r->ra);
    record_finish_kernel<<<1, 32, 0, s->stream>>>(s->ctl, r->rd);
    s->launches += 2;
    CK(cudaGetLastError());
    return WC_OK;
}

__global__ void fill_kernel(double* a, size_t n, double v) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) a[q] = v;
}

// eta = h + b and the breaking indicator of the resident state, FP32, interior row-major.
__global__ void frame_kernel(DevGrid g, const float4* __restrict__ q, const float* __restrict__ bed, BreakingDev br,
                             const double* __restrict__ mem, float* __restrict__ eta, float* __restrict__ brk,
                             float* __restrict__ depth) {
    const size_t cells = (size_t)g.nx * g.ny;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const int k = j * g.pitch + i;
        const double h = depth64(q[k]);
        eta[c] = (float)(h + (double)bed[k]);
        brk[c] = breaking_off(g, q, bed, br, mem, i, j);
        depth[c] = (float)h;
    }
}

}  // namespace

extern "C" {

wc_status wc_recorder_create(wc_solver* s, double from, double period, wc_recorder** out) {
    if (!out) return set_err(WC_EINVAL, "out is null");
    *out = nullptr;
    if (!s) return set_err(WC_EINVAL, "null solver");
    if (!(period > 0.0) || !std::isfinite(period)) return set_err(WC_EINVAL, "period must be positive");
    if (s->rec) return set_err(WC_EINVAL, "the solver already has a recorder");
    CK(cudaStreamSynchronize(s->stream));
    Ctl c{};
    CK(cudaMemcpy(&c, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
    auto* r = new wc_recorder();
    auto fail = [&](wc_status st) {
        delete r;
        return st;
    };
    r->s = s;
    r->cells = (size_t)s->grid.nx * s->grid.ny;
    const size_t n = r->cells;
    if (cudaMalloc(&r->block, 11 * n * sizeof(double)) != cudaSuccess || cudaMalloc(&r->rd, sizeof(RecDev)) != cudaSuccess)
        return fail(set_err(WC_ENOMEM, "recorder allocation failed"));
    double* b = r->block;
    r->ra.eta_max = b;
    r->ra.eta_min = b + n;
    r->ra.wave_max = b + 2 * n;
    r->ra.wave_min = b + 3 * n;
    r->ra.wave_sum = b + 4 * n;
    r->ra.wave_first = b + 5 * n;
    r->ra.wave_last = b + 6 * n;
    r->ra.breaking_seconds = b + 7 * n;
    r->ra.harm = b + 8 * n;
    const unsigned blocks = (unsigned)std::min<size_t>(148 * 8, (n + 255) / 256);
    fill_kernel<<<blocks, 256, 0, s->stream>>>(r->ra.eta_max, n, -INFINITY);
    fill_kernel<<<blocks, 256, 0, s->stream>>>(r->ra.eta_min, n, INFINITY);
    fill_kernel<<<blocks, 256, 0, s->stream>>>(r->ra.wave_max, n, -INFINITY);
    fill_kernel<<<blocks, 256, 0, s->stream>>>(r->ra.wave_min, n, INFINITY);
    if (cudaMemsetAsync(r->ra.wave_sum, 0, 7 * n * sizeof(double), s->stream) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "recorder set-up failed"));
    // lib.rs:1255-1268: the first wave ends a period after the later of the start and `from`
    RecDev d{};
    d.from = from;
    d.period = period;
    d.omega = TAU / period;
    d.next_wave = std::max(from, c.t) + period;
    d.t_last = c.t;
    if (cudaMemcpyAsync(r->rd, &d, sizeof d, cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "recorder set-up failed"));
    if (s->step_graph) {  // the captured step gains the recording kernels
        cudaGraphExecDestroy(s->step_graph);
        s->step_graph = nullptr;
    }
    s->rec = r;
    *out = r;
    return WC_OK;
}

void wc_recorder_destroy(wc_recorder* r) {
    if (!r) return;
    if (r->s) {
        cudaStreamSynchronize(r->s->stream);
        if (r->s->rec == r) {
            r->s->rec = nullptr;
            if (r->s->step_graph) {
                cudaGraphExecDestroy(r->s->step_graph);
                r->s->step_graph = nullptr;
            }
        }
    }
    delete r;
}

wc_status wc_recorder_read(wc_recorder* r, wc_record_summary* sum, double* eta_max, double* eta_min,
                           double* wave_height, double* breaking_fraction, double* harmonic) {
    if (!r || !r->s) return set_err(WC_EINVAL, "null recorder");
    wc_solver* s = r->s;
    const size_t n = r->cells;
    CK(cudaStreamSynchronize(s->stream));
    RecDev d{};
    CK(cudaMemcpy(&d, r->rd, sizeof d, cudaMemcpyDeviceToHost));
    auto get = [&](const double* src, std::vector<double>& v) -> wc_status {
        v.resize(n);
        CK(cudaMemcpy(v.data(), src, n * sizeof(double), cudaMemcpyDeviceToHost));
        return WC_OK;
    };
    if (eta_max) CK(cudaMemcpy(eta_max, r->ra.eta_max, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (eta_min) CK(cudaMemcpy(eta_min, r->ra.eta_min, n * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> first, last, tmp;
    // lib.rs:1303-1314: the mean per-wave height, NaN before a whole wave has passed
    if (wave_height) {
        TRY(get(r->ra.wave_sum, tmp));
        for (size_t c = 0; c < n; c++) wave_height[c] = d.waves > 0 ? tmp[c] / (double)d.waves : NAN;
    }
    // lib.rs:1340-1344
    if (breaking_fraction) {
        TRY(get(r->ra.breaking_seconds, tmp));
        const double t = std::max(d.seconds, 2.2250738585072014e-308);
        for (size_t c = 0; c < n; c++) breaking_fraction[c] = tmp[c] / t;
    }
    // FirstHarmonic::amplitudes (lib.rs:1132-1168): (a, -b) per cell from the 3x3 normal equations
    int has_harmonic = 0;
    if (harmonic || sum) {
        const double S = d.moments[0], C = d.moments[1], N = d.moments[2], CC = d.moments[3], CS = d.moments[4],
                     SS = d.moments[5];
        const double m[3][3] = {{S, C, N}, {C, CC, CS}, {N, CS, SS}};
        auto cof = [&](int rr, int k) {
            const int r1 = (rr + 1) % 3, r2 = (rr + 2) % 3, k1 = (k + 1) % 3, k2 = (k + 2) % 3;
            return m[r1][k1] * m[r2][k2] - m[r1][k2] * m[r2][k1];
        };
        double det = 0.0;
        for (int k = 0; k < 3; k++) det += m[0][k] * cof(0, k);
        has_harmonic = !(std::isnan(det) || det <= 1e-3 * S * S * S / 4.0);
        if (harmonic) {
            std::vector<double> h3(3 * n);
            CK(cudaMemcpy(h3.data(), r->ra.harm, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
            for (size_t c = 0; c < n; c++) {
                if (!has_harmonic) {
                    harmonic[2 * c] = harmonic[2 * c + 1] = NAN;
                    continue;
                }
                const double e[3] = {h3[c], h3[n + c], h3[2 * n + c]};
                auto row = [&](int rr) {
                    double v = 0.0;
                    for (int k = 0; k < 3; k++) v += cof(k, rr) / det * e[k];
                    return v;
                };
                harmonic[2 * c] = row(1);
                harmonic[2 * c + 1] = -row(2);
            }
        }
    }
    if (sum) {
        sum->seconds = d.seconds;
        sum->waves = (uint64_t)d.waves;
        sum->has_harmonic = has_harmonic;
        // lib.rs:1316-1338: median over the middle half of the rows, cells with a first wave
        // above 0.3 m, of |last / first - 1| / (waves - 1)
        sum->has_unsettled = 0;
        sum->unsettled = NAN;
        if (d.waves >= 2) {
            TRY(get(r->ra.wave_first, first));
            TRY(get(r->ra.wave_last, last));
            const size_t nx = s->grid.nx, ny = s->grid.ny;
            std::vector<double> change;
            for (size_t j = ny / 4; j < ny - ny / 4; j++)
                for (size_t i = 0; i < nx; i++) {
                    const size_t c = j * nx + i;
                    if (first[c] > 0.3) change.push_back(std::fabs(last[c] / first[c] - 1.0) / (double)(d.waves - 1));
                }
            if (!change.empty()) {
                std::sort(change.begin(), change.end());
                sum->unsettled = change[change.size() / 2];
                sum->has_unsettled = 1;
            }
        }
    }
    return WC_OK;
}

wc_status wc_frame(wc_solver* s, double tide, float* eta, float* breaking, double* rise) {
    if (!s || !eta || !breaking || !rise) return set_err(WC_EINVAL, "null argument");
    const size_t n = (size_t)s->grid.nx * s->grid.ny;
    if (!s->frame) {
        CK(cudaMalloc(&s->frame, 3 * n * sizeof(float)));
    }
    const unsigned blocks = (unsigned)std::min<size_t>(148 * 8, (n + 255) / 256);
    frame_kernel<<<blocks, 256, 0, s->stream>>>(s->g, s->q0, s->bed, s->br, s->eddy_on ? s->mem : nullptr, s->frame,
                                                s->frame + n, s->frame + 2 * n);
    s->launches++;
    CK(cudaGetLastError());
    std::vector<float> depth(n);
    CK(cudaMemcpyAsync(eta, s->frame, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(breaking, s->frame + n, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(depth.data(), s->frame + 2 * n, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    // lib.rs:1350-1366: the highest surface over still water among wet cells; a surface that is
    // not finite or more than 100 m up means the run is unstable
    double up = 0.0;
    bool finite = true;
    for (size_t c = 0; c < n; c++) {
        if (!std::isfinite(eta[c])) finite = false;
        if (depth[c] > 1e-3f) up = std::max(up, (double)eta[c] - tide);
    }
    *rise = up;
    if (!finite || !std::isfinite(up) || up > 100.0)
        return set_err(WC_ENAN, "the surface is not finite or more than 100 m above still water");
    return WC_OK;
}

}  // extern "C"

// ---- one-way nesting: relaxation zones driven by a coarser run -------------------------------

struct wc_nest {
    wc_solver* fine = nullptr;
    wc_solver* coarse = nullptr;
    NestCell* cells = nullptr;
    int n = 0;
    double* target = nullptr;  // [2 slots][3][n]
    double* times = nullptr;   // [2]
    cudaEvent_t sampled = nullptr;  // the targets are written (coarse stream)
    cudaEvent_t relaxed = nullptr;  // the targets are read (fine stream)
    ~wc_nest() {
        if (cells) cudaFree(cells);
        if (target) cudaFree(target);
        if (times) cudaFree(times);
        if (sampled) cudaEventDestroy(sampled);
        if (relaxed) cudaEventDestroy(relaxed);
    }
};

namespace {

// Sponge::rate (forcing.rs:180-206) at interior cell (a, b).
double sponge_rate_host(const wc_sponge& sp, const wc_grid& g, size_t a, size_t b) {
    const double w = (double)sp.width;
    auto ramp = [&](size_t d) {
        if (d < sp.width) {
            const double f = (w - (double)d) / w;
            return f * f;
        }
        return 0.0;
    };
    double r = 0.0;
    if (sp.west) r = std::max(r, ramp(a));
    if (sp.east) r = std::max(r, ramp(g.nx - 1 - a));
    if (sp.south) r = std::max(r, ramp(b));
    if (sp.north) r = std::max(r, ramp(g.ny - 1 - b));
    return sp.strength * r;
}

int reflect_host(long long i, long long n) {
    if (i >= 0 && i < n) return (int)i;
    const long long p = 2 * n;
    long long t = i % p;
    if (t < 0) t += p;
    return (int)(t < n ? t : p - 1 - t);
}

}  // namespace

extern "C" {

wc_status wc_nest_create(wc_solver* fine, wc_solver* coarse, const wc_sponge* zones, uint64_t n_zones,
                         double x_offset_m, double y_offset_m, wc_nest** out) {
    if (!out) return set_err(WC_EINVAL, "out is null");
    *out = nullptr;
    if (!fine || !coarse || (n_zones && !zones)) return set_err(WC_EINVAL, "null argument");
    if (fine == coarse) return set_err(WC_EINVAL, "the fine and the coarse run must be different solvers");
    const wc_grid& fg = fine->grid;
    const wc_grid& cg = coarse->grid;
    std::vector<NestCell> cells;
    for (size_t b = 0; b < fg.ny; b++)
        for (size_t a = 0; a < fg.nx; a++) {
            double rate = 0.0;  // Relaxation::new: the largest of the zones' rates
            for (uint64_t z = 0; z < n_zones; z++) rate = std::max(rate, sponge_rate_host(zones[z], fg, a, b));
            if (!(rate > 0.0)) continue;
            NestCell c{};
            c.k = (int)(b * fine->g.pitch + a);
            c.rate = rate;
            // Sampler::new (lib.rs:1560-1588): the fine cell's centre in coarse cells
            const double x = x_offset_m + ((double)a + 0.5) * fg.dx, y = y_offset_m + ((double)b + 0.5) * fg.dy;
            const double cx = x / cg.dx - 0.5, cy = y / cg.dy - 0.5;
            const double ix = std::floor(cx), iy = std::floor(cy);
            const double wx = cx - ix, wy = cy - iy;
            const double ws[4] = {(1.0 - wx) * (1.0 - wy), wx * (1.0 - wy), (1.0 - wx) * wy, wx * wy};
            const int dis[4] = {0, 1, 0, 1}, djs[4] = {0, 0, 1, 1};
            for (int e = 0; e < 4; e++) {
                // padded index clamped to one ghost layer, read through the wall fill
                const long long pi = std::min<long long>(std::max<long long>((long long)ix + dis[e], -1), (long long)cg.nx);
                const long long pj = std::min<long long>(std::max<long long>((long long)iy + djs[e], -1), (long long)cg.ny);
                const int mi = reflect_host(pi, (long long)cg.nx), mj = reflect_host(pj, (long long)cg.ny);
                c.kc[e] = mj * coarse->g.pitch + mi;
                c.sx[e] = (pi >= 0 && pi < (long long)cg.nx) ? 1.f : -1.f;
                c.sy[e] = (pj >= 0 && pj < (long long)cg.ny) ? 1.f : -1.f;
                c.w[e] = ws[e];
            }
            cells.push_back(c);
        }
    auto* nz = new wc_nest();
    auto fail = [&](wc_status st) {
        delete nz;
        return st;
    };
    nz->fine = fine;
    nz->coarse = coarse;
    nz->n = (int)cells.size();
    const size_t n = std::max<size_t>(1, cells.size());
    if (cudaMalloc(&nz->cells, n * sizeof(NestCell)) != cudaSuccess ||
        cudaMalloc(&nz->target, 6 * n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&nz->times, 2 * sizeof(double)) != cudaSuccess ||
        cudaEventCreateWithFlags(&nz->sampled, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&nz->relaxed, cudaEventDisableTiming) != cudaSuccess)
        return fail(set_err(WC_ENOMEM, "nest allocation failed"));
    if (!cells.empty() &&
        (cudaMemcpy(nz->cells, cells.data(), cells.size() * sizeof(NestCell), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaStreamSynchronize(0) != cudaSuccess))
        return fail(set_err(WC_ECUDA, "nest set-up failed"));
    if (cudaMemset(nz->target, 0, 6 * n * sizeof(double)) != cudaSuccess ||
        cudaMemset(nz->times, 0, 2 * sizeof(double)) != cudaSuccess || cudaStreamSynchronize(0) != cudaSuccess)
        return fail(set_err(WC_ECUDA, "nest set-up failed"));
    *out = nz;
    return WC_OK;
}

void wc_nest_destroy(wc_nest* nz) {
    if (!nz) return;
    cudaDeviceSynchronize();
    delete nz;
}

uint64_t wc_nest_cells(const wc_nest* nz) { return nz ? (uint64_t)nz->n : 0; }

wc_status wc_nest_sample(wc_nest* nz, int32_t slot) {
    if (!nz) return set_err(WC_EINVAL, "null nest");
    if (slot != 0 && slot != 1) return set_err(WC_EINVAL, "slot must be 0 (the earlier state) or 1 (the later)");
    wc_solver* c = nz->coarse;
    CK(cudaStreamWaitEvent(c->stream, nz->relaxed, 0));  // the last relaxation has read the slots
    const unsigned blocks = (unsigned)std::max(1, std::min(148 * 4, (nz->n + 255) / 256));
    nest_sample_kernel<<<blocks, 256, 0, c->stream>>>(c->q0, c->bed, nz->cells, nz->n, nz->target + (size_t)slot * 3 * nz->n,
                                                      nz->times + slot, c->ctl);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(nz->sampled, c->stream));
    return WC_OK;
}

wc_status wc_nest_step(wc_nest* nz, double dt) {
    if (!nz) return set_err(WC_EINVAL, "null nest");
    wc_solver* f = nz->fine;
    CK(cudaStreamWaitEvent(f->stream, nz->sampled, 0));  // the targets come from the coarse stream
    TRY(wc_step_device(f, dt));
    const unsigned blocks = (unsigned)std::max(1, std::min(148 * 4, (nz->n + 255) / 256));
    nest_relax_kernel<<<blocks, 256, 0, f->stream>>>(f->q0, f->bed, nz->cells, nz->n, nz->target,
                                                     nz->target + 3 * (size_t)nz->n, nz->times, f->ctl);
    f->launches++;
    f->rate_current = false;  // the relaxed state's time-step limit is recomputed when asked
    CK(cudaGetLastError());
    CK(cudaEventRecord(nz->relaxed, f->stream));
    return WC_OK;
}

}  // extern "C"
