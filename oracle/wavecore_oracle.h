/*
 * wavecore_oracle.h — FP64 CPU restatement of wavecore's time step.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker and the timed CPU baseline of
 * the B200 build; nothing in the product links, loads or calls it. It restates, line for line
 * and in the reference's loop and summation order, crates/wavecore/src/{grid,state,solver,
 * dispersion,forcing,par}.rs of mlaegn/wavesim. Parity is pinned by the reference's own
 * known-answer tests (ported under tests/), because the reference stores no numeric vectors and
 * its Rust toolchain is absent here. The followed breaking fronts (eddy.rs) are pinned by that
 * file's own unit tests, ported in tests/test_eddy_oracle.py.
 *
 * It shares the configuration structs of include/wavecore_c.h so that one configuration feeds
 * both the oracle and the device build.
 */
#ifndef WAVECORE_ORACLE_H
#define WAVECORE_ORACLE_H

#include "../include/wavecore_c.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_solver or_solver;

/* Threads for the row loops (OpenMP); 1 = serial. Results are bit-identical either way, as
 * in crates/wavecore/src/par.rs:1-6. Returns the count in force. */
int or_set_threads(int n);

wc_status or_solver_create(const wc_grid* grid, const double* bed_padded, const wc_config* cfg,
                           or_solver** out);
void or_solver_destroy(or_solver* s);
const char* or_last_error(void);

/* The bed as the solver holds it (padded; ghost rows wrapped when periodic). */
const double* or_solver_bed(const or_solver* s);

void or_step(or_solver* s, double* h, double* hu, double* hv, double* breaking, double* time,
             double dt);
double or_stable_dt(const or_solver* s, const double* h, const double* hu, const double* hv);
int or_limiting_cell(const or_solver* s, const double* h, const double* hu, const double* hv,
                     wc_limiting* out);
void or_breaking_indicator(or_solver* s, const double* h, const double* hu, const double* hv,
                           const double* breaking, double* out_interior);
int or_dispersion_stats(const or_solver* s, wc_stats* out);
/* The wave-maker's resolved drive (forcing.rs:77-117); returns 0 if there is none. */
int or_drive(const or_solver* s, double* omega, double* ky, double* strength);

/* Pieces exposed for the reference's unit tests. */
void or_face_values(const double v[5], double blend, double* lo, double* hi);
double or_smoothstep(double lo, double hi, double x);
wc_status or_linear_wave(double omega, double h, int dispersive, double* k, double* phase_speed,
                         double* group_speed);
double or_manning_factor(double h, double speed, double dt, double n);
void or_mirror_ghosts(const wc_grid* g, double* a);
void or_wrap_ghosts_y(const wc_grid* g, double* a);
void or_fill_boundaries(const wc_grid* g, int periodic_y, double* h, double* hu, double* hv,
                        double* breaking);
/* matvec of dispersion.rs:269-317; px/py get their ghost cells filled. */
void or_matvec(const wc_grid* g, int periodic_y, const double* heff, const double* mask,
               const double* c, double* px, double* py, double* ax, double* ay);
double or_dot(const wc_grid* g, const double* ax, const double* ay, const double* bx,
              const double* by);
/* Dispersion::apply (dispersion.rs:331-563) with fresh scratch: replaces lhu/lhv. */
void or_dispersion_apply(const wc_grid* g, int periodic_y, const wc_dispersion* d,
                         const double* h, const double* hu, const double* hv, const double* lh,
                         double* lhu, double* lhv, const double* phi);
/* eddy.rs: Kennedy's threshold (:114-124); `follow` (:155-219) on ghost-filled arrays,
 * replacing `breaking` by the new memory and writing nu; `diffuse` (:221-302), returning the
 * sub-steps; and the solver's `follow_breaking` (solver.rs:509-532). */
double or_eddy_threshold(const wc_eddy* e, double age, double h);
void or_eddy_follow(const wc_grid* g, const wc_eddy* e, const double* h, const double* hu,
                    const double* hv, double* breaking, const double* phi, double dt, double* nu);
int or_eddy_diffuse(const wc_grid* g, int periodic_y, double* h, double* hu, double* hv,
                    double* breaking, const double* nu, double dt);
int or_follow_breaking(or_solver* s, double* h, double* hu, double* hv, double* breaking,
                       double dt);
double or_volume(const wc_grid* g, const double* h);
double or_max_abs_momentum(const wc_grid* g, const double* hu, const double* hv);
double or_min_depth(const wc_grid* g, const double* h);

#ifdef __cplusplus
}
#endif

#endif
