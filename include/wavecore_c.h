/*
 * wavecore_c.h — C ABI of the B200 implementation of wavecore's time step.
 *
 * The reference (mlaegn/wavesim, crate `wavecore`) is a Rust library with no FFI. Each entry
 * point below replaces one method or builder of its `Solver` / `State` API, cited as
 * `crates/wavecore/src/<file>.rs:<line>`; a Rust `extern "C"` block binds this header as is
 * (crates/wavecore-b200-sys/src/lib.rs).
 *
 * Conventions shared with the reference:
 *   - every array is "padded": (nx + 2*WC_GHOST) * (ny + 2*WC_GHOST) values, row-major with y
 *     outer, interior cells at [WC_GHOST, WC_GHOST+nx) x [WC_GHOST, WC_GHOST+ny)
 *     (crates/wavecore/src/grid.rs:4-57);
 *   - host arrays are FP64, owned by the caller (crates/wavecore/src/state.rs:7-17);
 *   - the bed `b` is metres relative to still water, negative under water
 *     (crates/wavecore/src/bathymetry.rs:3-9).
 *
 * Differences a caller can observe, all deliberate:
 *   - the device computes in FP32 with a compensated (hi+lo) depth, FP64 reductions and FP64
 *     mass accumulation; results agree with the FP64 reference to the tolerances its parity tests
 *     state, and still water stays exactly still;
 *   - ghost cells of the bed are taken from the boundary rule (mirrored at walls, wrapped when
 *     periodic in y), which is what every `Bathymetry` constructor and `with_periodic_y` produce;
 *     the ghost values the caller passes are not read;
 *   - on return from wc_step the ghost cells of h/hu/hv hold the boundary fill of the new state
 *     (the reference leaves a blend that its next step overwrites);
 *   - setup errors that the reference raises with `assert!`/`panic!` return a status instead.
 */
#ifndef WAVECORE_C_H
#define WAVECORE_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Ghost layers on every side: crates/wavecore/src/grid.rs:4. */
#define WC_GHOST 3

typedef enum wc_status {
    WC_OK = 0,
    WC_EINVAL = 1,        /* invalid argument; the reference panics on these (grid.rs:87-91,
                             forcing.rs:63-66,89-90, solver.rs:377-383) */
    WC_EPERIODIC = 2,     /* oblique wave-maker does not fit the periodic domain (solver.rs:421-429) */
    WC_ENAN = 3,          /* the state holds a NaN (stable_dt is NaN, solver.rs:431-450) */
    WC_EUNCONVERGED = 4,  /* a dispersive solve stopped at max_iterations: reported, not fatal,
                             as the reference only counts it (dispersion.rs:541-545) */
    WC_ETIMEOUT = 5,      /* a bounded device wait ran out; the context stays usable */
    WC_ECUDA = 6,         /* a CUDA runtime call failed */
    WC_ENOMEM = 7,        /* device allocation failed */
    WC_EUNSUPPORTED = 8   /* a configuration this build does not implement */
} wc_status;

/* crates/wavecore/src/grid.rs:12-18 (`Grid { nx, ny, dx, dy }`). */
typedef struct wc_grid {
    uint64_t nx, ny;
    double dx, dy;
} wc_grid;

/* crates/wavecore/src/solver.rs:34-50 (`Order`). */
typedef enum wc_order { WC_ORDER_FIRST = 0, WC_ORDER_SECOND = 1, WC_ORDER_FIFTH = 2 } wc_order;

/* crates/wavecore/src/forcing.rs:146-178 (`Sponge`, built by `Sponge::new(width, strength)
 * .edges(west, east, south, north)`; `level` defaults to 0). */
typedef struct wc_sponge {
    uint64_t width;
    double strength;
    double level;
    int32_t west, east, south, north;
} wc_sponge;

/* crates/wavecore/src/forcing.rs:18-33 (`WaveMaker`). */
typedef struct wc_wavemaker {
    double x, amplitude, period, angle, sigma, ramp_periods;
} wc_wavemaker;

/* crates/wavecore/src/eddy.rs:62-90 (`EddyViscosity`): how breaking fronts are followed from
 * step to step, Kennedy et al.'s (2000) coefficients by default (wc_eddy_default). `initial`
 * and `settled` are rates of rise in sqrt(g h); `duration` and `linger` are times in
 * sqrt(h / g); `mixing` is the mixing length in depths (0 follows fronts without viscosity). */
typedef struct wc_eddy {
    double initial, settled, duration, mixing, linger;
} wc_eddy;

/* crates/wavecore/src/dispersion.rs:44-74 (`Breaking`). `viscosity` = 0 is the reference's
 * `None` (the default): the switch is read afresh at every step. `viscosity` = 1 is
 * `Some(eddy)`: breaking fronts are followed in the state's `breaking` memory, keep the switch
 * off where they are and just behind them, and get Kennedy's eddy viscosity (eddy.rs). Only
 * read with dispersion, as in the reference (solver.rs:509-520). */
typedef struct wc_breaking {
    double eta_ratio_lo, eta_ratio_hi;
    double slope_lo, slope_hi;
    int32_t viscosity;
    wc_eddy eddy;
} wc_breaking;

/* Preconditioner of the dispersive solve. JACOBI is the reference's
 * (dispersion.rs:493-545); LEARNED is this build's network preconditioner (no counterpart in
 * the reference), run inside flexible CG with the same stopping rule. */
typedef enum wc_preconditioner { WC_PC_JACOBI = 0, WC_PC_LEARNED = 1 } wc_preconditioner;

/* crates/wavecore/src/dispersion.rs:76-97 (`Dispersion`). */
typedef struct wc_dispersion {
    wc_breaking breaking;
    int32_t nonlinear;
    double tolerance;
    uint64_t max_iterations;
    int32_t preconditioner; /* wc_preconditioner */
} wc_dispersion;

/* Every builder of `Solver` (crates/wavecore/src/solver.rs:283-419) as one struct. */
typedef struct wc_config {
    double cfl;                       /* `Solver::cfl`, default 0.4 (solver.rs:287) */
    int32_t order;                    /* wc_order, default Second (solver.rs:288, :302-305) */
    double manning;                   /* `with_manning` (solver.rs:307-311) */
    int32_t periodic_y;               /* `with_periodic_y` (solver.rs:411-419) */
    const wc_sponge* sponges;         /* `with_sponge`, repeatable (solver.rs:313-317) */
    uint64_t n_sponges;
    const wc_wavemaker* wavemaker;    /* `with_wavemaker` or NULL (solver.rs:319-325) */
    const wc_dispersion* dispersion;  /* `with_dispersion` or NULL = shallow water (:327-334) */
    const uint8_t* shallow_cells;     /* `with_shallow_cells` or NULL; nx*ny, y outer (:367-384) */
} wc_config;

/* crates/wavecore/src/dispersion.rs:99-106 (`DispersionStats`). */
typedef struct wc_stats {
    uint64_t solves, iterations, unconverged;
} wc_stats;

/* crates/wavecore/src/solver.rs:248-258 (`Limiting`): i, j count interior cells from 0. */
typedef struct wc_limiting {
    uint64_t i, j;
    double depth, speed;
} wc_limiting;

/* crates/wavecore/src/state.rs:78-102 (`volume`, `max_abs_momentum`, `min_depth`). */
typedef struct wc_diagnostics {
    double volume, max_abs_momentum, min_depth;
} wc_diagnostics;

typedef struct wc_solver wc_solver;

/* Defaults of `Solver::new` (solver.rs:283-299): cfl 0.4, Second order, no friction, walls. */
void wc_config_default(wc_config* cfg);
/* `Dispersion::default()` (dispersion.rs:88-97) with `Breaking::default()` (:56-74): no
 * followed fronts (`viscosity` = 0), `eddy` set to `EddyViscosity::default()`. */
void wc_dispersion_default(wc_dispersion* d);
/* `EddyViscosity::default()` (eddy.rs:81-90): 0.65, 0.15, 5, 1.2, 5. */
void wc_eddy_default(wc_eddy* e);

/* `Solver::new(grid, bed)` followed by the builders in `cfg` (solver.rs:283-429).
 * `bed_padded` holds (nx+6)*(ny+6) values; only its interior is read. Returns WC_EINVAL where
 * the reference panics on setup, WC_EPERIODIC for an oblique wave-maker that does not fit a
 * periodic domain, WC_EUNSUPPORTED for configurations this build does not run. */
wc_status wc_solver_create(const wc_grid* grid, const double* bed_padded, const wc_config* cfg,
                           wc_solver** out);
void wc_solver_destroy(wc_solver* s);

/* `Solver::step(&mut State, dt)` (solver.rs:479-507) on host FP64 arrays, in place: uploads the
 * state, runs one SSP-RK2 step on the device, downloads it and advances `*time` by dt.
 * `breaking` is the state's breaking memory (state.rs:11-15): with followed fronts it is read
 * and updated (its interior; ghosts are refilled by the boundary rule), otherwise carried
 * unchanged. It may be NULL only without followed fronts. */
wc_status wc_step(wc_solver* s, double* h, double* hu, double* hv, double* breaking,
                  double* time, double dt);

/* `Solver::stable_dt(&State)` (solver.rs:431-450): *dt_out is NaN when a cell is not a number
 * (status WC_ENAN), 0 when a speed is infinite, +inf when nothing can move (status WC_OK). */
wc_status wc_stable_dt(wc_solver* s, const double* h, const double* hu, const double* hv,
                       double* dt_out);

/* `Solver::limiting_cell(&State)` (solver.rs:452-477): *found = 0 where the reference returns
 * None. */
wc_status wc_limiting_cell(wc_solver* s, const double* h, const double* hu, const double* hv,
                           wc_limiting* out, int32_t* found);

/* `Solver::breaking_indicator(&State)` (solver.rs:336-349): nx*ny values, y outer. With
 * followed fronts the state's `breaking` memory holds the switch off where it is not 0
 * (dispersion.rs:149-152); NULL reads as no memory. */
wc_status wc_breaking_indicator(wc_solver* s, const double* h, const double* hu,
                                const double* hv, const double* breaking, double* out_interior);

/* `Solver::follow_breaking` (solver.rs:509-532, private in the reference; exported for parity
 * checks of eddy.rs): the fronts in `breaking` followed on to the state (h, hu, hv) and their
 * eddy viscosity applied to its momentum over dt, in place, on host FP64 arrays. A no-op
 * without followed fronts. *sub_steps (may be NULL) gets the viscous sub-steps taken. */
wc_status wc_follow_breaking(wc_solver* s, double* h, double* hu, double* hv, double* breaking,
                             double dt, int32_t* sub_steps);

/* `Solver::dispersion_stats()` (solver.rs:391-396): *has = 0 for shallow water. */
wc_status wc_dispersion_stats(wc_solver* s, wc_stats* out, int32_t* has);

/* ---- Device-resident throughput path (no counterpart in the reference) ----------------- */

/* Copy a padded FP64 host state onto the device (interior only) and set the device clock. The
 * breaking memory is cleared (a new state has no wave breaking, state.rs:11-15). */
wc_status wc_state_upload(wc_solver* s, const double* h, const double* hu, const double* hv,
                          double time);
/* The device state's breaking memory (state.rs:11-15) from / to a padded FP64 host array
 * (interior read; ghosts written by the boundary rule). Without followed fronts the memory is
 * not kept: upload ignores it and download writes zeros. */
wc_status wc_breaking_upload(wc_solver* s, const double* breaking);
wc_status wc_breaking_download(wc_solver* s, double* breaking);
/* Copy the device state back into padded FP64 host arrays (ghosts filled by the boundary
 * rule); `time` may be NULL. */
wc_status wc_state_download(wc_solver* s, double* h, double* hu, double* hv, double* time);
/* One step of size dt on the device-resident state. Asynchronous: errors of the step itself
 * surface at the next synchronising call. */
wc_status wc_step_device(wc_solver* s, double dt);
/* n_steps steps on the device-resident state, each of size min(stable_dt, t_end - time) read
 * on the device, as the reference's test loop does (crates/wavecore/tests/common/mod.rs:53-60).
 * Stops early (on the device) once time >= t_end. Asynchronous. */
wc_status wc_step_n(wc_solver* s, uint64_t n_steps, double t_end);
/* stable_dt of the device-resident state, synchronising. */
wc_status wc_stable_dt_device(wc_solver* s, double* dt_out);
/* FP64 reductions over the device-resident state (state.rs:78-102), synchronising. */
wc_status wc_diagnostics_device(wc_solver* s, wc_diagnostics* out);
/* The dispersive system of the solver's last solve and its solution, as the device holds them
 * (FP32 values widened to FP64). The reference keeps the same arrays in Dispersion's private
 * scratch (crates/wavecore/src/dispersion.rs:203-266, :380-490) and exposes none; this is for
 * checking a solve, e.g. its true residual ||b - A w|| / ||b|| in FP64. Each output holds the
 * nx*ny interior values, row-major with y outer: c = phi h^3 / 3, heff = max(h, 1e-8) (a cell
 * takes part in the system where heff >= 0.05), the right-hand side (bx, by) and the solution
 * (wx, wy). Any output may be null. WC_EINVAL if the solver has no dispersion. Synchronising. */
wc_status wc_dispersion_system(wc_solver* s, double* c, double* heff, double* bx, double* by,
                               double* wx, double* wy);
/* Device time of the device-resident state, synchronising. */
wc_status wc_time_device(wc_solver* s, double* time_out);
/* No counterpart in the reference (which has no device waits): the limit, in nanoseconds, of each
 * bounded wait of this solver's persistent kernels (a grid barrier of the dispersive solve or of
 * the followed fronts); 0 restores the default of 2 s. A wait that runs out sets an error bit,
 * every CTA of the kernel returns, and the call that reports the step's status returns
 * WC_ETIMEOUT with the context still usable (the next state upload clears the error). A tiny
 * limit forces that path without any fault, which is how the failure handling is tested. */
wc_status wc_set_wait_limit(wc_solver* s, uint64_t ns);
/* Wait for all queued device work of this solver and report its status: WC_ETIMEOUT if a
 * bounded device wait ran out, WC_ENAN if a step met a NaN. */
wc_status wc_synchronize(wc_solver* s);

/* Run this solver's work on the caller's CUDA stream (a cudaStream_t; NULL restores the solver's
 * own stream), so that a caller can order and time it with its own events, as cublasSetStream
 * does. The caller keeps the stream alive while the solver uses it. */
wc_status wc_set_stream(wc_solver* s, void* stream);

/* Per-kernel device timing (no counterpart in the reference). While enabled, every launch of
 * the step is bracketed by CUDA events on the solver's stream; wc_profile_read synchronises and
 * returns, per kernel kind, the launch count and the summed device milliseconds since the last
 * enable. Kinds: 0 = RK-stage stencil kernel, 1 = dispersive solve (for the learned
 * preconditioner: its vector kernels and the stage epilogue), 2 = other, 3 = the learned
 * preconditioner's network (one count per application), 4 = followed breaking fronts and their
 * eddy viscosity (one launch per step). */
typedef struct wc_kernel_time {
    uint64_t launches;
    double total_ms;
} wc_kernel_time;
#define WC_KERNEL_KINDS 5
wc_status wc_profile_enable(wc_solver* s, int32_t on);
wc_status wc_profile_read(wc_solver* s, wc_kernel_time out[WC_KERNEL_KINDS]);

/* No counterpart in the reference: wc_stable_dt for callers that cannot have the library allocate
 * device memory, such as an application that hands all of the GPU's memory to its own pool
 * allocator at start-up and runs under a fixed budget, or a simulation loop that must not allocate
 * or free per step (cudaFree synchronises the whole device). The state belongs to the caller:
 * padded FP64 device arrays h, hu, hv of (nx+6)*(ny+6) values each, read on `stream` (a
 * cudaStream_t; NULL is the legacy default stream). The call is synchronous: it waits on `stream`
 * for its result and returns it on the host. It allocates nothing: its scratch is a fixed 64 KiB
 * array inside the library, which every GPU that loads the library holds until the process exits,
 * and grids of more than 16,777,216 interior cells (4096 x 4096) are refused with WC_EINVAL. The
 * first call on a device (and the first after a device reset) looks up that array's device
 * address, so make that first call before any stream capture begins. All calls share the one
 * array, which keeps the last call's contents (each call rewrites every slot it reads): calls
 * that overlap on the GPU race, so do not run two at once. Returns in *dt_out, with the same
 * status, what wc_stable_dt returns for the same state. */
wc_status wc_stable_dt_noalloc(const wc_grid* grid, double cfl, const double* d_h,
                               const double* d_hu, const double* d_hv, void* stream,
                               double* dt_out);

/* ---- Ensembles (no counterpart in the reference, which runs one Solver per grid in turn,
 * crates/wavesim/src/lib.rs:1813-1902) ------------------------------------------------------
 * n independent runs, each with its own grid, bed (padded FP64) and configuration (second or
 * fifth order), advanced together: every step of every member is one persistent cooperative
 * launch, replayed from a CUDA graph, in which each member's own group of CTAs runs its whole
 * SSP-RK2 step with its own adaptive time step, clock and PCG state (or, if the autotuner finds it
 * faster, every member's own captured step on its own stream). The CTAs are split over the
 * members by their work per step (cells, and the PCG iterations per solve the autotuner measures
 * on its first call). The stage tile shape and the CTAs per SM are chosen by an autotuner that
 * times each compiled variant on the live state (then restores it); wc_ensemble_step_n runs it on
 * first use. */
typedef struct wc_ensemble wc_ensemble;
typedef struct wc_lpc wc_lpc;  /* the learned preconditioner, below */
wc_status wc_ensemble_create(uint64_t n, const wc_grid* grids, const double* const* beds,
                             const wc_config* cfgs, wc_ensemble** out);
void wc_ensemble_destroy(wc_ensemble* e);
wc_status wc_ensemble_upload(wc_ensemble* e, uint64_t member, const double* h, const double* hu,
                             const double* hv, double time);
wc_status wc_ensemble_download(wc_ensemble* e, uint64_t member, double* h, double* hu, double* hv,
                               double* time);
/* Up to n_steps steps of every member, each of size min(stable_dt, t_end - time); a member stops
 * once its time reaches t_end. Asynchronous. */
wc_status wc_ensemble_step_n(wc_ensemble* e, uint64_t n_steps, double t_end);
/* Time every choice over trial_steps steps and keep the fastest; *choice is its index (0-3: the
 * persistent launch with stage tile height 8 or 16 by CTAs per SM 1 or 2: 0 = 8/1, 1 = 8/2,
 * 2 = 16/1, 3 = 16/2; 4: no persistent launch, every member's own captured step on its own
 * stream, forked from the ensemble's stream and joined back) and ms_per_step[5] the measured times
 * (-1 for a choice that cannot run). A learned ensemble (wc_ensemble_set_lpc) has only choice 4. */
wc_status wc_ensemble_autotune(wc_ensemble* e, uint32_t trial_steps, int32_t* choice,
                               double* ms_per_step);
/* The learned preconditioner for every dispersive member (config 4's method). The network's
 * solve is a chain of kernels with a data-dependent loop, which a persistent launch cannot hold,
 * so a learned ensemble steps each member through its own captured step (the flexible CG's
 * while-node included) on its own stream, forked from the ensemble's stream and joined back every
 * step, so the members' kernels overlap on the GPU. Call once, before stepping; the network must
 * outlive the ensemble. */
wc_status wc_ensemble_set_lpc(wc_ensemble* e, wc_lpc* l);
wc_status wc_ensemble_synchronize(wc_ensemble* e);
wc_status wc_ensemble_member_stats(wc_ensemble* e, uint64_t member, wc_stats* stats,
                                   double* time);
uint64_t wc_ensemble_launch_count(const wc_ensemble* e);

/* ---- The learned preconditioner (no counterpart in the reference) ------------------------------
 *
 * The reference preconditions its dispersive CG with the Jacobi diagonal only
 * (crates/wavecore/src/dispersion.rs:441-457, 493-545). These entry points add a trained
 * alternative: a depth-gated linear 4-level U-net used inside a two-level cycle
 *     z1 = w r / D,  z2 = z1 + mask N(D^-1 (r - A z1)),  z = z2 + w (r - A z2) / D   (w = 0.5)
 * as the preconditioner of flexible CG, with the Jacobi solve's stopping rule; a solve that does
 * not converge (or breaks down) is finished by Jacobi PCG from where it stopped, so the plain
 * method stays the fallback and the arbiter of convergence. Training runs on
 * the GPU by the library's own forward and backward kernels, on patches of SGN systems harvested
 * from solver runs, minimising the energy norm of the cycle's error on random error fields. */

/* channels[4]: feature maps per level, finest first (null: 8, 16, 32, 32); gate_hidden: width of
 * the gate networks' hidden layer (8); stride 1, 2 or 4: the network runs on a grid that many
 * times coarser than the solver's (its input is the block mean of D^-1 (r - A z1), its output is
 * added at every cell of the block). Weights start scaled-normal from `seed`, biases at zero and
 * the output layer at zero (an untrained network adds nothing to the Jacobi sweeps). */
wc_status wc_lpc_create(const int32_t* channels, int32_t gate_hidden, int32_t stride,
                        uint64_t seed, wc_lpc** out);
/* A network must outlive every solver it is attached to. */
void wc_lpc_destroy(wc_lpc* l);
uint64_t wc_lpc_num_params(const wc_lpc* l);
/* The FP32 master weights, in the layout of wavesim_b200/lpc.py (UNetSpec.layers). Setting them
 * resets the optimiser's moments. */
wc_status wc_lpc_set_params(wc_lpc* l, const float* params, uint64_t n);
wc_status wc_lpc_get_params(wc_lpc* l, float* params, uint64_t n);
/* bf16 != 0 (default): the forward pass uses BF16-rounded weights; 0: the FP32 weights. */
wc_status wc_lpc_set_rounding(wc_lpc* l, int32_t bf16);
/* One forward and backward pass on host arrays, for checking gradients: x and feat are
 * [n][2][h][w] (h, w multiples of 8), dy the output gradient of the same shape; returns the
 * output y, the parameter gradient of sum(dy * y) (num_params values) and its input gradient. */
wc_status wc_lpc_forward_backward(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* x,
                                  const float* feat, const float* dy, float* y, float* grad,
                                  float* dx);
/* The network's output (inference: no training state kept) on host arrays x and feat,
 * [n][2][h][w] (h, w multiples of 8). tensor = 1: BF16 activations on the tensor cores, as the
 * solver applies it; 2: the same with the first level's layers run one launch per layer instead
 * of its fused launches; 3: the same with every layer on tiles of its usual height (no 16 x 8
 * tiles for the coarse levels' 32-channel layers); 2 and 3 check that each variant gives the same
 * bits; 0: FP32 FMA, as training does. */
wc_status wc_lpc_forward(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* x,
                         const float* feat, int32_t tensor, float* y);
/* The training objective on given patches, for checking its gradient: c, heff and bed are
 * [n][h][w] (the mask h >= 5 cm and the features h / 20 m, b / 20 m are derived as for harvested
 * crops), e the error fields [n][2][h][w]; returns the loss (as wc_lpc_train defines it) and its
 * gradient with respect to the parameters (num_params values). */
wc_status wc_lpc_loss_grad(wc_lpc* l, int32_t n, int32_t h, int32_t w, const float* c,
                           const float* heff, const float* bed, const float* e, double dx, double dy,
                           double* loss, float* grad);
/* Copies the solver's current SGN system (c, h, bed; the one of its last solve) for training. */
wc_status wc_lpc_harvest(wc_lpc* l, wc_solver* s);
uint64_t wc_lpc_num_systems(const wc_lpc* l);
/* `steps` Adam steps (learning rate lr) on batches of `batch` random patch x patch crops of the
 * harvested systems with random error fields (`rough`: weight of the cell-scale noise in them);
 * losses[steps] (may be null) receives every step's loss, the mean over the batch of
 * <d, A d> / <e, A e> with d the cycle's error. Synchronous. */
wc_status wc_lpc_train(wc_lpc* l, uint32_t steps, uint32_t batch, uint32_t patch, float lr,
                       float rough, uint64_t seed, double* losses);
/* Attach a network: the solver's dispersive solves become learned-preconditioned flexible CG.
 * Null detaches it (Jacobi PCG). A solver created with WC_PC_LEARNED steps only once a network
 * is attached. */
wc_status wc_solver_set_lpc(wc_solver* s, wc_lpc* l);

/* ---- Per-step statistics and frames ------------------------------------------------------------
 *
 * The reference's driver records statistics after every step of a run in a host loop over the
 * grid (crates/wavesim/src/lib.rs:1276-1301, Stage::record; 899-931, Stats; 1095-1169,
 * FirstHarmonic) and writes frames of the surface and the breaking indicator
 * (lib.rs:1348-1380, frame_if_due). A recorder keeps the same per-cell sums on the device and is
 * updated by kernels appended to every step of its solver (host-array or device-resident). */
typedef struct wc_recorder wc_recorder;

typedef struct wc_record_summary {
    double seconds;        /* recorded time */
    uint64_t waves;        /* whole wave periods closed */
    int32_t has_harmonic;  /* 0: too little time to separate a mean, a cosine and a sine */
    int32_t has_unsettled;
    double unsettled;      /* lib.rs:1316-1338: median relative change of the per-wave height per period */
} wc_record_summary;

/* Start recording the solver's steps: statistics count from time `from`; `period` is the swell's
 * period (per-wave heights and the first harmonic). One recorder per solver; it must be destroyed
 * before the solver, or it is detached and inert once the solver is gone. */
wc_status wc_recorder_create(wc_solver* s, double from, double period, wc_recorder** out);
void wc_recorder_destroy(wc_recorder* r);
/* The statistics so far, interior row-major arrays of nx*ny values (any may be null): the surface's
 * maximum and minimum, the mean crest-to-trough height per wave (NaN before a whole wave), the
 * fraction of the recorded time spent breaking (indicator >= 0.8, lib.rs:1222) and, in
 * `harmonic` (2 values per cell), the first harmonic's (a, -b) of eta = m + a cos wt + b sin wt
 * (NaN while has_harmonic is 0). */
wc_status wc_recorder_read(wc_recorder* r, wc_record_summary* summary, double* eta_max,
                           double* eta_min, double* wave_height, double* breaking_fraction,
                           double* harmonic);
/* A frame of the resident state (lib.rs:1348-1380): eta = h + b and the breaking indicator as
 * FP32, interior row-major, and the highest surface above `tide` among cells deeper than 1 mm.
 * Returns WC_ENAN (frame still written) when the surface is not finite or more than 100 m up. */
wc_status wc_frame(wc_solver* s, double tide, float* eta, float* breaking, double* rise);

/* ---- One-way nesting: relaxation zones driven by a coarser run ---------------------------------
 *
 * crates/wavecore/src/forcing.rs:209-283 (Relaxation, relax_cell) and
 * crates/wavesim/src/lib.rs:1554-1605 (Sampler), :1846-1896 (the nested step): the fine run's
 * zone cells (where one of `zones` has a rate, at the largest rate) relax after each fine step
 * towards the surface and velocity of the coarse run, bilinear over the wet coarse cells around
 * the fine cell's centre and interpolated in time between two sampled coarse states. Both runs
 * keep their states on the device. */
typedef struct wc_nest wc_nest;

/* `fine` and `coarse` are solvers of the same sea; the fine grid's origin lies at
 * (x_offset_m, y_offset_m) in the coarse grid's frame. Both solvers must outlive the nest. */
wc_status wc_nest_create(wc_solver* fine, wc_solver* coarse, const wc_sponge* zones, uint64_t n_zones,
                         double x_offset_m, double y_offset_m, wc_nest** out);
void wc_nest_destroy(wc_nest* n);
uint64_t wc_nest_cells(const wc_nest* n);
/* Sample the coarse run's resident state (at its device clock) into slot 0 (the state before
 * the coarse step that brackets the fine step's end) or slot 1 (the state after it). */
wc_status wc_nest_sample(wc_nest* n, int32_t slot);
/* One fine step of dt on the device, then the zone's relaxation towards the targets at the
 * step's end time (clamped to the sampled interval). Asynchronous. */
wc_status wc_nest_step(wc_nest* n, double dt);

/* Kernel launches this solver has queued since it was created (for accounting). */
uint64_t wc_launch_count(const wc_solver* s);
/* Human-readable text of the last error on this thread ("" if none). */
const char* wc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WAVECORE_C_H */
