/*
 * wavecore_oracle.c — FP64 CPU restatement of wavecore's time step (TEST INFRASTRUCTURE).
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark load this library;
 * the product never does. Each function names the reference lines it restates
 * (mlaegn/wavesim, paths relative to the project root). The reference is Rust; the restatement
 * keeps its expression order (compiled with -ffp-contract=off, no fast-math) and its row order
 * for every reduction (crates/wavecore/src/par.rs:90-115), so the serial and the OpenMP builds
 * give identical numbers, as the reference's serial and rayon builds do.
 */
#include "wavecore_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* crates/wavecore/src/solver.rs:26-32; dispersion.rs:41; forcing.rs:286; par.rs:13 */
#define G 9.81
#define H_DRY 1e-8
#define H_SECOND 1e-3
#define H_FACE_MIN 1e-4
#define H_DISPERSION_MIN 0.05
#define H_FRICTION_MIN 1e-3
#define GH 3
#define MIN_CELLS 40000
#define TAU 6.283185307179586
#define PI_ 3.141592653589793

static _Thread_local char g_err[256];
static int g_threads = 1;

const char* or_last_error(void) { return g_err; }
static wc_status fail(wc_status st, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return st;
}

int or_set_threads(int n) {
#ifdef _OPENMP
    if (n < 1) n = omp_get_num_procs();
    g_threads = n;
#else
    (void)n;
    g_threads = 1;
#endif
    return g_threads;
}

/* ---- grid.rs ---------------------------------------------------------------------------- */

typedef struct {
    size_t nx, ny, w, rows, n;
    double dx, dy;
} Grid;

static Grid mk_grid(const wc_grid* g) {
    Grid r;
    r.nx = (size_t)g->nx;
    r.ny = (size_t)g->ny;
    r.w = r.nx + 2 * GH;
    r.rows = r.ny + 2 * GH;
    r.n = r.w * r.rows;
    r.dx = g->dx;
    r.dy = g->dy;
    return r;
}

#define IDX(g, i, j) ((j) * (g)->w + (i))
/* par.rs:15-18: rows run on threads only for grids of at least MIN_CELLS values */
#define THREADED(g) ((g)->n >= MIN_CELLS && g_threads > 1)

/* grid.rs:60-75 */
static void mirror_ghosts(const Grid* g, double* a) {
    for (size_t j = GH; j < GH + g->ny; j++)
        for (size_t k = 0; k < GH; k++) {
            a[IDX(g, GH - 1 - k, j)] = a[IDX(g, GH + k, j)];
            a[IDX(g, GH + g->nx + k, j)] = a[IDX(g, GH + g->nx - 1 - k, j)];
        }
    for (size_t i = 0; i < g->w; i++)
        for (size_t k = 0; k < GH; k++) {
            a[IDX(g, i, GH - 1 - k)] = a[IDX(g, i, GH + k)];
            a[IDX(g, i, GH + g->ny + k)] = a[IDX(g, i, GH + g->ny - 1 - k)];
        }
}

/* grid.rs:77-87 */
static void wrap_ghosts_y(const Grid* g, double* a) {
    for (size_t i = 0; i < g->w; i++)
        for (size_t k = 0; k < GH; k++) {
            a[IDX(g, i, GH - 1 - k)] = a[IDX(g, i, GH + g->ny - 1 - k)];
            a[IDX(g, i, GH + g->ny + k)] = a[IDX(g, i, GH + k)];
        }
}

/* grid.rs:89-114 */
static void fill_vector_ghosts(const Grid* g, double* vx, double* vy, int periodic_y) {
    mirror_ghosts(g, vx);
    mirror_ghosts(g, vy);
    for (size_t j = 0; j < g->rows; j++)
        for (size_t k = 0; k < GH; k++) {
            size_t l = IDX(g, GH - 1 - k, j), r = IDX(g, GH + g->nx + k, j);
            vx[l] = -vx[l];
            vx[r] = -vx[r];
        }
    for (size_t i = 0; i < g->w; i++)
        for (size_t k = 0; k < GH; k++) {
            size_t lo = IDX(g, i, GH - 1 - k), hi = IDX(g, i, GH + g->ny + k);
            vy[lo] = -vy[lo];
            vy[hi] = -vy[hi];
        }
    if (periodic_y) {
        wrap_ghosts_y(g, vx);
        wrap_ghosts_y(g, vy);
    }
}

/* ---- state.rs --------------------------------------------------------------------------- */

/* state.rs:42-62 */
static void fill_walls(const Grid* g, double* h, double* hu, double* hv, double* br) {
    mirror_ghosts(g, h);
    mirror_ghosts(g, hu);
    mirror_ghosts(g, hv);
    mirror_ghosts(g, br);
    for (size_t j = 0; j < g->rows; j++)
        for (size_t k = 0; k < GH; k++) {
            size_t l = IDX(g, GH - 1 - k, j), r = IDX(g, GH + g->nx + k, j);
            hu[l] = -hu[l];
            hu[r] = -hu[r];
        }
    for (size_t i = 0; i < g->w; i++)
        for (size_t k = 0; k < GH; k++) {
            size_t lo = IDX(g, i, GH - 1 - k), hi = IDX(g, i, GH + g->ny + k);
            hv[lo] = -hv[lo];
            hv[hi] = -hv[hi];
        }
}

/* state.rs:64-76 */
static void fill_boundaries(const Grid* g, int periodic_y, double* h, double* hu, double* hv,
                            double* br) {
    fill_walls(g, h, hu, hv, br);
    if (periodic_y) {
        wrap_ghosts_y(g, h);
        wrap_ghosts_y(g, hu);
        wrap_ghosts_y(g, hv);
        wrap_ghosts_y(g, br);
    }
}

/* state.rs:78-85: the interior summed in iterator order (one running sum) */
double or_volume(const wc_grid* wg, const double* h) {
    Grid g = mk_grid(wg);
    double s = 0.0;
    for (size_t j = GH; j < GH + g.ny; j++)
        for (size_t i = GH; i < GH + g.nx; i++) s += h[IDX(&g, i, j)];
    return s * g.dx * g.dy;
}

/* state.rs:87-95 (f64::max drops NaN, as fmax does) */
double or_max_abs_momentum(const wc_grid* wg, const double* hu, const double* hv) {
    Grid g = mk_grid(wg);
    double m = 0.0;
    for (size_t j = GH; j < GH + g.ny; j++)
        for (size_t i = GH; i < GH + g.nx; i++) {
            size_t k = IDX(&g, i, j);
            m = fmax(m, fmax(fabs(hu[k]), fabs(hv[k])));
        }
    return m;
}

/* state.rs:97-102 */
double or_min_depth(const wc_grid* wg, const double* h) {
    Grid g = mk_grid(wg);
    double m = INFINITY;
    for (size_t j = GH; j < GH + g.ny; j++)
        for (size_t i = GH; i < GH + g.nx; i++) m = fmin(m, h[IDX(&g, i, j)]);
    return m;
}

/* ---- par.rs ----------------------------------------------------------------------------- */

/* par.rs:109-115 */
static inline double max_or_nan(double a, double b) {
    if (isnan(a) || isnan(b)) return NAN;
    return fmax(a, b);
}

/* ---- forcing.rs ------------------------------------------------------------------------- */

typedef struct {
    wc_wavemaker spec;
    double omega, ky, strength;
} Drive;

/* forcing.rs:46-75 */
wc_status or_linear_wave(double omega, double h, int dispersive, double* k, double* phase_speed,
                         double* group_speed) {
    if (!dispersive) {
        double c = sqrt(G * h);
        *k = omega / c;
        *phase_speed = c;
        *group_speed = c;
        return WC_OK;
    }
    double nu = omega * omega * h / G;
    if (!(nu < 3.0))
        return fail(WC_EINVAL, "a wave of this angular frequency is too short for the "
                               "dispersive model at this depth");
    double kh = sqrt(nu / (1.0 - nu / 3.0));
    double kk = kh / h;
    double ps = omega / kk;
    *k = kk;
    *phase_speed = ps;
    *group_speed = ps / (1.0 + kh * kh / 3.0);
    return WC_OK;
}

/* forcing.rs:87-117 */
static wc_status drive_new(Drive* d, const wc_wavemaker* spec, const Grid* g, double still_depth,
                           int dispersive) {
    if (!(still_depth > 0.0)) return fail(WC_EINVAL, "wave-maker must sit in water");
    if (!(spec->period > 0.0 && spec->sigma > 0.0 && spec->amplitude >= 0.0))
        return fail(WC_EINVAL, "wave-maker period and sigma must be positive, amplitude >= 0");
    double omega = TAU / spec->period;
    double k, ps, c;
    wc_status st = or_linear_wave(omega, still_depth, dispersive, &k, &ps, &c);
    if (st != WC_OK) return st;
    double ky = k * sin(spec->angle);
    double kx = k * cos(spec->angle);
    double rolloff = exp(0.5 * kx * kx * spec->sigma * spec->sigma);
    double flux = 2.0 * c * spec->amplitude * cos(spec->angle) * rolloff;
    double norm = 0.0;
    for (size_t i = 0; i < g->nx; i++) {
        double x = ((double)i + 0.5) * g->dx;
        double dd = x - spec->x;
        norm += exp(-(dd * dd) / (2.0 * spec->sigma * spec->sigma)) * g->dx;
    }
    d->spec = *spec;
    d->omega = omega;
    d->ky = ky;
    d->strength = flux / norm;
    return WC_OK;
}

/* forcing.rs:124-138 */
static inline double drive_source(const Drive* d, double x, double y, double t) {
    const wc_wavemaker* s = &d->spec;
    double dd = x - s->x;
    double profile = exp(-(dd * dd) / (2.0 * s->sigma * s->sigma));
    if (profile < 1e-12) return 0.0;
    double ramp_time = s->ramp_periods * s->period;
    double ramp = t >= ramp_time ? 1.0 : 0.5 * (1.0 - cos(PI_ * t / ramp_time));
    return d->strength * profile * ramp * sin(d->omega * t - d->ky * y);
}

/* forcing.rs:180-206 */
static inline double sponge_rate(const wc_sponge* sp, const Grid* g, size_t i, size_t j) {
    size_t a = i - GH, b = j - GH;
    double w = (double)sp->width;
#define RAMP(d) ((d) < sp->width ? ((w - (double)(d)) / w) * ((w - (double)(d)) / w) : 0.0)
    double r = 0.0;
    if (sp->west) r = fmax(r, RAMP(a));
    if (sp->east) r = fmax(r, RAMP(g->nx - 1 - a));
    if (sp->south) r = fmax(r, RAMP(b));
    if (sp->north) r = fmax(r, RAMP(g->ny - 1 - b));
#undef RAMP
    return sp->strength * r;
}

/* forcing.rs:209-225 */
static inline void relax_cell(double* h, double* hu, double* hv, double bed, double eta, double u,
                              double v, double f) {
    double ht = fmax(eta - bed, 0.0);
    *h = f * *h + (1.0 - f) * ht;
    *hu = f * *hu + (1.0 - f) * ht * u;
    *hv = f * *hv + (1.0 - f) * ht * v;
}

/* forcing.rs:288-297 */
double or_manning_factor(double h, double speed, double dt, double n) {
    double k = G * n * n / pow(h, 4.0 / 3.0);
    return 1.0 / (1.0 + dt * k * speed);
}

/* ---- dispersion.rs: switch ---------------------------------------------------------------- */

/* dispersion.rs:108-111 (Rust f64::clamp keeps NaN) */
double or_smoothstep(double lo, double hi, double x) {
    double t = (x - lo) / (hi - lo);
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    return t * t * (3.0 - 2.0 * t);
}

/* dispersion.rs:113-160. `mem` is the state's breaking memory: with followed fronts
 * (br->viscosity) a cell whose memory is not 0 reads breaking (:149-152). */
static void switch_phi(const Grid* g, const double* bed, const double* h, const double* mem,
                       const wc_breaking* br, int periodic_y, double* phi) {
    const size_t w = g->w;
    const double ix = 0.5 / g->dx, iy = 0.5 / g->dy;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++) {
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            if (h[k] < H_DISPERSION_MIN) {
                phi[k] = 0.0;
                continue;
            }
            double ex = ((h[k + 1] + bed[k + 1]) - (h[k - 1] + bed[k - 1])) * ix;
            double ey = ((h[k + w] + bed[k + w]) - (h[k - w] + bed[k - w])) * iy;
            double ratio = fmax((h[k] + bed[k]) / h[k], 0.0);
            double off = fmax(or_smoothstep(br->eta_ratio_lo, br->eta_ratio_hi, ratio),
                              or_smoothstep(br->slope_lo, br->slope_hi, hypot(ex, ey)));
            if (br->viscosity && mem && mem[k] != 0.0) off = 1.0; /* EddyViscosity::keeps_off */
            phi[k] = 1.0 - off;
        }
    }
    mirror_ghosts(g, phi);
    if (periodic_y) wrap_ghosts_y(g, phi);
}

/* ---- eddy.rs: breaking fronts followed from step to step ---------------------------------- */

#define H_BREAKING_MIN 0.01 /* eddy.rs:54-56 */
#define BREAKING_ONSET 0.8  /* eddy.rs:58-59 */

/* eddy.rs:103-106 */
static double eddy_span(const wc_eddy* e, double h) { return e->duration * sqrt(h / G); }

/* eddy.rs:114-124 */
double or_eddy_threshold(const wc_eddy* e, double age, double h) {
    double span = eddy_span(e, h);
    if (age >= span) return e->settled;
    return e->initial + (e->settled - e->initial) * age / span;
}

/* f64::clamp(0, 1), which keeps NaN */
static inline double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

/* eddy.rs:155-219 (`follow`). h, hu, hv and the memory `br` have their ghost cells filled; `br`
 * is replaced by the new memory (ghosts 0, as the reference's swap leaves them) and `nu` gets
 * the eddy viscosity (0 outside the interior). `rise` and `mem` are padded scratch. */
static void eddy_follow(const Grid* g, const wc_eddy* e, const double* h, const double* hu,
                        const double* hv, double* br, const double* phi, double dt, double* rise,
                        double* mem, double* nu) {
    const size_t w = g->w;
    const double ix = 0.5 / g->dx, iy = 0.5 / g->dy;
    memset(rise, 0, g->n * sizeof(double));
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            rise[k] = -((hu[k + 1] - hu[k - 1]) * ix + (hv[k + w] - hv[k - w]) * iy);
        }
    memset(mem, 0, g->n * sizeof(double));
    memset(nu, 0, g->n * sizeof(double));
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            double depth = h[k];
            if (depth < H_BREAKING_MIN) continue;
            double c = sqrt(G * depth);
            const size_t nb[5] = {k, k - 1, k + 1, k - w, k + w};
            double front = 0.0;
            for (int m = 0; m < 5; m++) front = fmax(front, br[nb[m]]);
            int starts = depth >= H_DISPERSION_MIN && 1.0 - phi[k] >= BREAKING_ONSET && rise[k] > 0.0;
            int goes_on = front > 0.0 && rise[k] > or_eddy_threshold(e, front, depth) * c;
            double age = (front > 0.0 && (starts || goes_on)) ? front + dt : (starts ? dt : 0.0);
            if (age > 0.0) {
                double b = clamp01(rise[k] / (or_eddy_threshold(e, age, depth) * c) - 1.0);
                mem[k] = age;
                nu[k] = b * e->mixing * e->mixing * depth * rise[k];
            } else if (br[k] > 0.0) {
                mem[k] = -e->linger * sqrt(depth / G);
            } else if (br[k] < 0.0) {
                mem[k] = fmin(br[k] + dt, 0.0);
            }
        }
    memcpy(br, mem, g->n * sizeof(double));
}

/* eddy.rs:221-302 (`diffuse`): the viscosity `nu` (0 outside the interior) applied to hu, hv over
 * dt in explicit sub-steps, the ghost cells refilled between them. Returns the sub-steps taken.
 * whu, whv are padded scratch. */
static int eddy_diffuse(const Grid* g, int periodic_y, double* h, double* hu, double* hv,
                        double* br, const double* nu, double dt, double* whu, double* whv) {
    const size_t w = g->w;
    /* par.rs:99-107: row maxima (f64::max, which drops NaN) folded in row order */
    double top = 0.0;
    for (size_t j = GH; j < GH + g->ny; j++) {
        double m = 0.0;
        for (size_t k = j * w + GH; k < j * w + GH + g->nx; k++) m = fmax(m, nu[k]);
        top = max_or_nan(top, m);
    }
    if (top <= 0.0) return 0;
    const double idx2 = 1.0 / (g->dx * g->dx), idy2 = 1.0 / (g->dy * g->dy);
    const double limit = 0.5 / (top * fmax(2.0 * idx2 + idy2, idx2 + 2.0 * idy2));
    double fsteps = fmax(ceil(dt / limit), 1.0);
    if (fsteps > 1e9) fsteps = 1e9; /* the reference's `as usize` saturates far beyond this */
    const int steps = (int)fsteps;
    const double sub = dt / (double)steps;
    const double cross = 0.25 / (g->dx * g->dy);
    for (int step = 0; step < steps; step++) {
        if (step > 0) fill_boundaries(g, periodic_y, h, hu, hv, br);
#pragma omp parallel for schedule(static) if (THREADED(g))
        for (size_t j = GH; j < g->ny + GH; j++)
            for (size_t i = GH; i < g->nx + GH; i++) {
                size_t k = j * w + i;
                if (h[k] < H_BREAKING_MIN) {
                    whu[k] = hu[k];
                    whv[k] = hv[k];
                    continue;
                }
                const size_t e = k + 1, west = k - 1, north = k + w, south = k - w;
#define LINK(a, b) ((h[a] < H_BREAKING_MIN || h[b] < H_BREAKING_MIN) ? 0.0 : 0.5 * (nu[a] + nu[b]))
#define WET(a) (h[a] < H_BREAKING_MIN ? 0.0 : nu[a])
#define XX(q) ((LINK(k, e) * (q[e] - q[k]) - LINK(k, west) * (q[k] - q[west])) * idx2)
#define YY(q) ((LINK(k, north) * (q[north] - q[k]) - LINK(k, south) * (q[k] - q[south])) * idy2)
#define YX(q) ((WET(north) * (q[north + 1] - q[north - 1]) - WET(south) * (q[south + 1] - q[south - 1])) * cross)
#define XY(q) ((WET(e) * (q[e + w] - q[e - w]) - WET(west) * (q[west + w] - q[west - w])) * cross)
                whu[k] = hu[k] + sub * (XX(hu) + 0.5 * (YY(hu) + YX(hv)));
                whv[k] = hv[k] + sub * (YY(hv) + 0.5 * (XX(hv) + XY(hu)));
#undef LINK
#undef WET
#undef XX
#undef YY
#undef YX
#undef XY
            }
        /* only the interior was written; the ghost cells are refilled before they are read */
#pragma omp parallel for schedule(static) if (THREADED(g))
        for (size_t j = GH; j < g->ny + GH; j++)
            for (size_t i = GH; i < g->nx + GH; i++) {
                size_t k = j * w + i;
                hu[k] = whu[k];
                hv[k] = whv[k];
            }
    }
    return steps;
}

void or_eddy_follow(const wc_grid* wg, const wc_eddy* e, const double* h, const double* hu,
                    const double* hv, double* breaking, const double* phi, double dt, double* nu) {
    Grid g = mk_grid(wg);
    double* rise = (double*)malloc(g.n * sizeof(double));
    double* mem = (double*)malloc(g.n * sizeof(double));
    eddy_follow(&g, e, h, hu, hv, breaking, phi, dt, rise, mem, nu);
    free(rise);
    free(mem);
}

int or_eddy_diffuse(const wc_grid* wg, int periodic_y, double* h, double* hu, double* hv,
                    double* breaking, const double* nu, double dt) {
    Grid g = mk_grid(wg);
    double* whu = (double*)calloc(g.n, sizeof(double));
    double* whv = (double*)calloc(g.n, sizeof(double));
    int steps = eddy_diffuse(&g, periodic_y, h, hu, hv, breaking, nu, dt, whu, whv);
    free(whu);
    free(whv);
    return steps;
}

/* ---- solver.rs: reconstruction and fluxes ------------------------------------------------- */

typedef struct {
    double h, un, ut, b, phi;
} Cell;
typedef struct {
    double h, un, ut, z;
} Side;
typedef struct {
    double flux[3], corr_left, corr_right;
} Face;
typedef struct {
    Face low, high;
    double source;
} Axis;

/* solver.rs:90-92 */
static inline double velocity(double h, double hm) { return h > H_DRY ? hm / h : 0.0; }

/* solver.rs:94-100 */
static inline double rate_at(const double* h, const double* hu, const double* hv, size_t k,
                             double dx, double dy) {
    double c = sqrt(G * h[k]);
    double u = fabs(velocity(h[k], hu[k]));
    double v = fabs(velocity(h[k], hv[k]));
    return (u + c) / dx + (v + c) / dy;
}

/* solver.rs:102-110 (f64::min/max are fmin/fmax) */
static inline double minmod3(double a, double b, double c) {
    if (a > 0.0 && b > 0.0 && c > 0.0) return fmin(fmin(a, b), c);
    if (a < 0.0 && b < 0.0 && c < 0.0) return fmax(fmax(a, b), c);
    return 0.0;
}

/* solver.rs:112-116 */
static inline double limited_slope(double d_low, double d_high) {
    return minmod3(2.0 * d_low, 0.5 * (d_low + d_high), 2.0 * d_high);
}

/* solver.rs:118-138 */
void or_face_values(const double v[5], double blend, double* lo, double* hi) {
    double low2 = v[0], low = v[1], c = v[2], high = v[3], high2 = v[4];
    double s = limited_slope(c - low, high - c);
    double mc_lo = c - 0.5 * s, mc_hi = c + 0.5 * s;
    if (blend <= 0.0) {
        *lo = mc_lo;
        *hi = mc_hi;
        return;
    }
    double fifth_hi = (2.0 * low2 - 13.0 * low + 47.0 * c + 27.0 * high - 3.0 * high2) / 60.0;
    double fifth_lo = (2.0 * high2 - 13.0 * high + 47.0 * c + 27.0 * low - 3.0 * low2) / 60.0;
    *lo = mc_lo + blend * (fifth_lo - mc_lo);
    *hi = mc_hi + blend * (fifth_hi - mc_hi);
}

/* solver.rs:140-183 */
static inline void reconstruct(const Cell cells[5], int order, Side* out_lo, Side* out_hi) {
    const Cell c = cells[2];
    Side first = {c.h, c.un, c.ut, c.b};
    if (order == WC_ORDER_FIRST || cells[1].h < H_SECOND || c.h < H_SECOND ||
        cells[3].h < H_SECOND) {
        *out_lo = first;
        *out_hi = first;
        return;
    }
    double blend = 0.0;
    if (order == WC_ORDER_FIFTH && cells[0].h >= H_SECOND && cells[4].h >= H_SECOND) {
        blend = 1.0;
        for (int m = 0; m < 5; m++) blend = fmin(blend, cells[m].phi);
    }
    double v[5], eta_lo, eta_hi, un_lo, un_hi, ut_lo, ut_hi;
    for (int m = 0; m < 5; m++) v[m] = cells[m].h + cells[m].b;
    or_face_values(v, blend, &eta_lo, &eta_hi);
    for (int m = 0; m < 5; m++) v[m] = cells[m].un;
    or_face_values(v, blend, &un_lo, &un_hi);
    for (int m = 0; m < 5; m++) v[m] = cells[m].ut;
    or_face_values(v, blend, &ut_lo, &ut_hi);
    double s_z = 0.25 * (cells[3].b - cells[1].b);
    Side lo = {eta_lo - (c.b + -1.0 * s_z), un_lo, ut_lo, c.b + -1.0 * s_z};
    Side hi = {eta_hi - (c.b + 1.0 * s_z), un_hi, ut_hi, c.b + 1.0 * s_z};
    if (lo.h < H_FACE_MIN || hi.h < H_FACE_MIN) {
        *out_lo = first;
        *out_hi = first;
        return;
    }
    *out_lo = lo;
    *out_hi = hi;
}

/* solver.rs:185-226 */
static inline Face face(Side l, Side r) {
    double z_star = fmax(l.z, r.z);
    double hl = fmax(l.h + l.z - z_star, 0.0);
    double hr = fmax(r.h + r.z - z_star, 0.0);
    double cl = sqrt(G * hl), cr = sqrt(G * hr);
    double s_l = fmin(l.un - cl, r.un - cr);
    double s_r = fmax(l.un + cl, r.un + cr);
    double f_l[3] = {hl * l.un, hl * l.un * l.un + 0.5 * G * hl * hl, hl * l.un * l.ut};
    double f_r[3] = {hr * r.un, hr * r.un * r.un + 0.5 * G * hr * hr, hr * r.un * r.ut};
    double u_l[3] = {hl, hl * l.un, hl * l.ut};
    double u_r[3] = {hr, hr * r.un, hr * r.ut};
    Face f;
    if (hl <= H_DRY && hr <= H_DRY) {
        f.flux[0] = f.flux[1] = f.flux[2] = 0.0;
    } else if (s_l >= 0.0) {
        for (int k = 0; k < 3; k++) f.flux[k] = f_l[k];
    } else if (s_r <= 0.0) {
        for (int k = 0; k < 3; k++) f.flux[k] = f_r[k];
    } else {
        double inv = 1.0 / (s_r - s_l);
        for (int k = 0; k < 3; k++)
            f.flux[k] = (s_r * f_l[k] - s_l * f_r[k] + s_l * s_r * (u_r[k] - u_l[k])) * inv;
    }
    f.corr_left = 0.5 * G * (l.h * l.h - hl * hl);
    f.corr_right = 0.5 * G * (r.h * r.h - hr * hr);
    return f;
}

/* solver.rs:228-239 */
static inline Axis axis_terms(const Cell st[7], double spacing, int order) {
    Side hi_m1, lo0, hi0, lo_p1, unused;
    reconstruct(st + 0, order, &unused, &hi_m1);
    reconstruct(st + 1, order, &lo0, &hi0);
    reconstruct(st + 2, order, &lo_p1, &unused);
    Axis a;
    a.low = face(hi_m1, lo0);
    a.high = face(hi0, lo_p1);
    a.source = -G * 0.5 * (lo0.h + hi0.h) * (hi0.z - lo0.z) / spacing;
    return a;
}

/* ---- dispersion.rs: the SGN solve ---------------------------------------------------------- */

typedef struct {
    double *u, *v, *mask, *um, *vm, *div, *c, *f, *heff, *diag_x, *diag_y, *wx, *wy, *bx, *by,
        *rx, *ry, *zx, *zy, *px, *py, *ax, *ay;
    wc_stats stats;
} Work;

static int work_new(Work* w, const Grid* g) {
    double** arrs[] = {&w->u,  &w->v,  &w->mask, &w->um, &w->vm, &w->div,    &w->c,      &w->f,
                       &w->heff, &w->diag_x, &w->diag_y, &w->wx, &w->wy, &w->bx, &w->by, &w->rx,
                       &w->ry, &w->zx, &w->zy, &w->px, &w->py, &w->ax, &w->ay};
    for (size_t m = 0; m < sizeof arrs / sizeof arrs[0]; m++) {
        *arrs[m] = (double*)calloc(g->n, sizeof(double));
        if (!*arrs[m]) return 0;
    }
    memset(&w->stats, 0, sizeof w->stats);
    return 1;
}

static void work_free(Work* w) {
    double* arrs[] = {w->u,  w->v,  w->mask, w->um, w->vm, w->div, w->c,  w->f,
                      w->heff, w->diag_x, w->diag_y, w->wx, w->wy, w->bx, w->by, w->rx,
                      w->ry, w->zx, w->zy, w->px, w->py, w->ax, w->ay};
    for (size_t m = 0; m < sizeof arrs / sizeof arrs[0]; m++) free(arrs[m]);
}

/* dispersion.rs:269-317 */
static void matvec(const Grid* g, int periodic_y, const double* heff, const double* mask,
                   const double* c, double* f, double* px, double* py, double* ax, double* ay) {
    fill_vector_ghosts(g, px, py, periodic_y);
    const size_t w = g->w, nx = g->nx, ny = g->ny;
    const double ix = 0.5 / g->dx, iy = 0.5 / g->dy;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH - 1; j <= ny + GH; j++)
        for (size_t i = GH - 1; i < nx + GH + 1; i++) {
            size_t k = j * w + i;
            f[k] = c[k] * ((px[k + 1] - px[k - 1]) * ix + (py[k + w] - py[k - w]) * iy);
        }
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            ax[k] = mask[k] * (heff[k] * px[k] - (f[k + 1] - f[k - 1]) * ix);
            ay[k] = mask[k] * (heff[k] * py[k] - (f[k + w] - f[k - w]) * iy);
        }
}

/* dispersion.rs:319-329 with par.rs:86-97: per-row sums added in row order */
static double dot_(const Grid* g, const double* ax, const double* ay, const double* bx,
                   const double* by, double* rows_buf) {
    const size_t w = g->w, nx = g->nx, ny = g->ny;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < GH + ny; j++) {
        size_t row = j * w + GH;
        double s = 0.0;
        for (size_t k = row; k < row + nx; k++) s += ax[k] * bx[k] + ay[k] * by[k];
        rows_buf[j - GH] = s;
    }
    double total = 0.0;
    for (size_t j = 0; j < ny; j++) total += rows_buf[j];
    return total;
}

double or_dot(const wc_grid* wg, const double* ax, const double* ay, const double* bx,
              const double* by) {
    Grid g = mk_grid(wg);
    double* buf = (double*)malloc(g.ny * sizeof(double));
    double r = dot_(&g, ax, ay, bx, by, buf);
    free(buf);
    return r;
}

/* dispersion.rs:566-589 */
static void precondition(const Grid* g, const double* rx, const double* ry, const double* dxg,
                         const double* dyg, double* zx, double* zy) {
    const size_t w = g->w;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            zx[k] = rx[k] / dxg[k];
            zy[k] = ry[k] / dyg[k];
        }
}

/* dispersion.rs:613-635 */
static void axpy(const Grid* g, double a, const double* xx, const double* xy, double* yx,
                 double* yy) {
    const size_t w = g->w;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            yx[k] += a * xx[k];
            yy[k] += a * xy[k];
        }
}

/* dispersion.rs:331-563 */
static void dispersion_apply(const wc_dispersion* d, const Grid* g, int periodic_y,
                             const double* h, const double* hu, const double* hv,
                             const double* lh, double* lhu, double* lhv, const double* phi,
                             Work* W, double* rows_buf) {
    const size_t w = g->w, nx = g->nx, ny = g->ny, rows = g->rows;
    const double dx = g->dx, dy = g->dy, ix = 0.5 / dx, iy = 0.5 / dy;
    const int nonlinear = d->nonlinear;
    double *u = W->u, *v = W->v, *mask = W->mask, *um = W->um, *vm = W->vm, *div = W->div;
    double *c = W->c, *f = W->f, *heff = W->heff, *diag_x = W->diag_x, *diag_y = W->diag_y;
    double *wx = W->wx, *wy = W->wy, *bx = W->bx, *by = W->by, *rx = W->rx, *ry = W->ry;
    double *zx = W->zx, *zy = W->zy, *px = W->px, *py = W->py, *ax = W->ax, *ay = W->ay;

    /* :385-391 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = 0; j < rows; j++)
        for (size_t i = 0; i < w; i++) {
            size_t k = j * w + i;
            u[k] = velocity(h[k], hu[k]);
            v[k] = velocity(h[k], hv[k]);
        }
    /* :393-401 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = 0; j < rows; j++)
        for (size_t i = 0; i < w; i++) {
            size_t k = j * w + i;
            double m = h[k] >= H_DISPERSION_MIN ? 1.0 : 0.0;
            mask[k] = m;
            um[k] = m * u[k];
            vm[k] = m * v[k];
        }
    /* :403-411 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = 1; j < rows - 1; j++)
        for (size_t i = 1; i < w - 1; i++) {
            size_t k = j * w + i;
            div[k] = (um[k + 1] - um[k - 1]) * ix + (vm[k + w] - vm[k - w]) * iy;
        }
    /* :414-438 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH - 1; j <= ny + GH; j++)
        for (size_t i = GH - 1; i < nx + GH + 1; i++) {
            size_t k = j * w + i;
            double depth = h[k];
            double coeff = depth < H_DISPERSION_MIN ? 0.0 : phi[k] * depth * depth * depth / 3.0;
            c[k] = coeff;
            if (nonlinear && coeff > 0.0) {
                double n = um[k] * (div[k + 1] - div[k - 1]) * ix +
                           vm[k] * (div[k + w] - div[k - w]) * iy - div[k] * div[k];
                f[k] = coeff * n;
            } else {
                f[k] = 0.0;
            }
        }
    /* :441-457 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            heff[k] = fmax(h[k], H_DRY);
            if (mask[k] == 0.0) {
                diag_x[k] = 1.0;
                diag_y[k] = 1.0;
            } else {
                diag_x[k] = heff[k] + (c[k + 1] + c[k - 1]) * 0.25 / (dx * dx);
                diag_y[k] = heff[k] + (c[k + w] + c[k - w]) * 0.25 / (dy * dy);
            }
        }
    /* :460-479 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            if (mask[k] == 0.0) {
                bx[k] = 0.0;
                by[k] = 0.0;
            } else {
                bx[k] = lhu[k] - u[k] * lh[k] + (f[k + 1] - f[k - 1]) * ix;
                by[k] = lhv[k] - v[k] * lh[k] + (f[k + w] - f[k - w]) * iy;
            }
        }
    /* :480-490 */
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++)
            if (mask[j * w + i] == 0.0) {
                wx[j * w + i] = 0.0;
                wy[j * w + i] = 0.0;
            }

    /* :493-545 */
    matvec(g, periodic_y, heff, mask, c, f, wx, wy, ax, ay);
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            rx[k] = bx[k] - ax[k];
            ry[k] = by[k] - ay[k];
        }
    precondition(g, rx, ry, diag_x, diag_y, zx, zy);
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            px[k] = zx[k];
            py[k] = zy[k];
        }
    double bnorm = sqrt(dot_(g, bx, by, bx, by, rows_buf));
    double target = d->tolerance * bnorm + 1e-10;
    double rz = dot_(g, rx, ry, zx, zy, rows_buf);
    uint64_t iterations = 0;
    int converged = sqrt(dot_(g, rx, ry, rx, ry, rows_buf)) <= target;
    while (!converged && iterations < d->max_iterations) {
        matvec(g, periodic_y, heff, mask, c, f, px, py, ax, ay);
        double pap = dot_(g, px, py, ax, ay, rows_buf);
        double alpha = rz / pap;
        axpy(g, alpha, px, py, wx, wy);
        axpy(g, -alpha, ax, ay, rx, ry);
        precondition(g, rx, ry, diag_x, diag_y, zx, zy);
        iterations += 1;
        converged = sqrt(dot_(g, rx, ry, rx, ry, rows_buf)) <= target;
        double rz_next = dot_(g, rx, ry, zx, zy, rows_buf);
        double beta = rz_next / rz;
        rz = rz_next;
#pragma omp parallel for schedule(static) if (THREADED(g))
        for (size_t j = GH; j < ny + GH; j++)
            for (size_t i = GH; i < nx + GH; i++) {
                size_t k = j * w + i;
                px[k] = zx[k] + beta * px[k];
                py[k] = zy[k] + beta * py[k];
            }
    }
    W->stats.solves += 1;
    W->stats.iterations += iterations;
    if (!converged) W->stats.unconverged += 1;

    /* :547-562 */
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < ny + GH; j++)
        for (size_t i = GH; i < nx + GH; i++) {
            size_t k = j * w + i;
            if (mask[k] > 0.0) {
                lhu[k] = h[k] * wx[k] + u[k] * lh[k];
                lhv[k] = h[k] * wy[k] + v[k] * lh[k];
            }
        }
}

/* ---- solver.rs: the solver ----------------------------------------------------------------- */

struct or_solver {
    Grid g;
    wc_grid wg;
    double* b;
    double cfl, manning;
    int order, periodic_y;
    wc_sponge* sponges;
    size_t nsp;
    int has_drive;
    Drive drive;
    int has_disp;
    wc_dispersion disp;
    Work work;
    double* phi;
    uint8_t* shallow;
    /* scratch: rhs, the two RK stages, row partials */
    double *rh, *rhu, *rhv;
    double *s1h, *s1hu, *s1hv, *s1br, *s2h, *s2hu, *s2hv, *s2br;
    double* rows_buf;
    /* followed fronts (eddy.rs:92-101): rise, memory, viscosity, momentum scratch */
    double *ed_rise, *ed_mem, *ed_nu, *ed_hu, *ed_hv;
};

static const wc_breaking k_default_breaking = {0.30, 0.55, 0.40, 0.65, 0, {0.65, 0.15, 5.0, 1.2, 5.0}};

static const wc_breaking* breaking_config(const or_solver* s) {
    return s->has_disp ? &s->disp.breaking : &k_default_breaking;
}

void or_solver_destroy(or_solver* s) {
    if (!s) return;
    free(s->b);
    free(s->sponges);
    if (s->has_disp) work_free(&s->work);
    free(s->phi);
    free(s->shallow);
    double* arrs[] = {s->rh,     s->rhu,     s->rhv,    s->s1h,    s->s1hu,   s->s1hv,
                      s->s1br,   s->s2h,     s->s2hu,   s->s2hv,   s->s2br,   s->rows_buf,
                      s->ed_rise, s->ed_mem, s->ed_nu, s->ed_hu, s->ed_hv};
    for (size_t m = 0; m < sizeof arrs / sizeof arrs[0]; m++) free(arrs[m]);
    free(s);
}

/* Solver::new plus every builder of solver.rs:283-429, in the reference's semantics:
 * the drive is rebuilt against the final dispersion setting, the periodic check runs once
 * both are known, and the bed's ghost rows wrap when periodic. */
wc_status or_solver_create(const wc_grid* wg, const double* bed, const wc_config* cfg,
                           or_solver** out) {
    *out = NULL;
    if (!wg || !bed || !cfg) return fail(WC_EINVAL, "null argument");
    if (!(wg->nx > 0 && wg->ny > 0)) return fail(WC_EINVAL, "grid must have at least one interior cell");
    if (!(wg->dx > 0.0 && wg->dy > 0.0)) return fail(WC_EINVAL, "cell size must be positive");
    or_solver* s = (or_solver*)calloc(1, sizeof(or_solver));
    if (!s) return fail(WC_ENOMEM, "out of memory");
    s->wg = *wg;
    s->g = mk_grid(wg);
    const Grid* g = &s->g;
    s->cfl = cfg->cfl;
    s->order = cfg->order;
    s->manning = cfg->manning;
    s->periodic_y = cfg->periodic_y != 0;
    s->b = (double*)malloc(g->n * sizeof(double));
    s->phi = (double*)calloc(g->n, sizeof(double));
    double** scratch[] = {&s->rh,  &s->rhu,  &s->rhv,  &s->s1h,  &s->s1hu, &s->s1hv,
                          &s->s1br, &s->s2h, &s->s2hu, &s->s2hv, &s->s2br};
    for (size_t m = 0; m < sizeof scratch / sizeof scratch[0]; m++)
        *scratch[m] = (double*)calloc(g->n, sizeof(double));
    s->rows_buf = (double*)calloc(g->rows, sizeof(double));
    memcpy(s->b, bed, g->n * sizeof(double));
    if (cfg->n_sponges) {
        s->sponges = (wc_sponge*)malloc(cfg->n_sponges * sizeof(wc_sponge));
        memcpy(s->sponges, cfg->sponges, cfg->n_sponges * sizeof(wc_sponge));
        s->nsp = cfg->n_sponges;
    }
    if (cfg->dispersion) {
        s->has_disp = 1;
        s->disp = *cfg->dispersion;
        if (!work_new(&s->work, g)) {
            or_solver_destroy(s);
            return fail(WC_ENOMEM, "out of memory");
        }
        if (s->disp.breaking.viscosity) {
            double** ed[] = {&s->ed_rise, &s->ed_mem, &s->ed_nu, &s->ed_hu, &s->ed_hv};
            for (size_t m = 0; m < sizeof ed / sizeof ed[0]; m++)
                *ed[m] = (double*)calloc(g->n, sizeof(double));
        }
    }
    if (cfg->shallow_cells) {
        s->shallow = (uint8_t*)malloc(g->nx * g->ny);
        memcpy(s->shallow, cfg->shallow_cells, g->nx * g->ny);
    }
    /* with_periodic_y wraps the bed's ghost rows (solver.rs:414-419) */
    if (s->periodic_y) wrap_ghosts_y(g, s->b);
    /* rebuild_drive (solver.rs:400-409) */
    if (cfg->wavemaker) {
        const wc_wavemaker* spec = cfg->wavemaker;
        double r = round(spec->x / g->dx - 0.5);
        if (r < 0.0) r = 0.0;
        size_t i = (size_t)r;
        if (i > g->nx - 1) i = g->nx - 1;
        i += GH;
        double depth = -s->b[IDX(g, i, GH + g->ny / 2)];
        wc_status st = drive_new(&s->drive, spec, g, depth, s->has_disp);
        if (st != WC_OK) {
            or_solver_destroy(s);
            return st;
        }
        s->has_drive = 1;
        /* check_periodic (solver.rs:421-429) */
        if (s->periodic_y) {
            double turns = s->drive.ky * (double)g->ny * g->dy / TAU;
            if (!(fabs(turns - round(turns)) < 1e-6)) {
                or_solver_destroy(s);
                return fail(WC_EPERIODIC, "wave-maker does not fit the periodic domain: "
                                          "k_y * Ly / 2pi must be a whole number");
            }
        }
    }
    *out = s;
    return WC_OK;
}

const double* or_solver_bed(const or_solver* s) { return s->b; }

int or_drive(const or_solver* s, double* omega, double* ky, double* strength) {
    if (!s->has_drive) return 0;
    *omega = s->drive.omega;
    *ky = s->drive.ky;
    *strength = s->drive.strength;
    return 1;
}

int or_dispersion_stats(const or_solver* s, wc_stats* out) {
    if (!s->has_disp) return 0;
    *out = s->work.stats;
    return 1;
}

/* solver.rs:576-591 */
static void clean_dry(const Grid* g, double* h, double* hu, double* hv) {
    const size_t w = g->w;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            if (h[k] < H_DRY) {
                h[k] = fmax(h[k], 0.0);
                hu[k] = 0.0;
                hv[k] = 0.0;
            }
        }
}

/* solver.rs:593-616: next = s + dt * rhs over the interior, ghosts copied from s */
static void advance(const or_solver* S, const double* h, const double* hu, const double* hv,
                    const double* br, double dt, double* nh, double* nhu, double* nhv,
                    double* nbr) {
    const Grid* g = &S->g;
    memcpy(nh, h, g->n * sizeof(double));
    memcpy(nhu, hu, g->n * sizeof(double));
    memcpy(nhv, hv, g->n * sizeof(double));
    memcpy(nbr, br, g->n * sizeof(double));
    const size_t w = g->w;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            nh[k] += dt * S->rh[k];
            nhu[k] += dt * S->rhu[k];
            nhv[k] += dt * S->rhv[k];
        }
    clean_dry(g, nh, nhu, nhv);
}

/* solver.rs:625-733 */
static void rhs(or_solver* S, const double* h, const double* hu, const double* hv,
                const double* br, double t) {
    const Grid* g = &S->g;
    const size_t w = g->w;
    if (S->order == WC_ORDER_FIFTH || S->has_disp) {
        switch_phi(g, S->b, h, br, breaking_config(S), S->periodic_y, S->phi);
        if (S->shallow) {
            size_t n = 0;
            for (size_t j = GH; j < GH + g->ny; j++)
                for (size_t i = GH; i < GH + g->nx; i++, n++)
                    if (S->shallow[n]) S->phi[IDX(g, i, j)] = 0.0;
            mirror_ghosts(g, S->phi);
            if (S->periodic_y) wrap_ghosts_y(g, S->phi);
        }
    }
    const double* phi = S->phi;
    const double* bed = S->b;
    const int order = S->order;
    memset(S->rh, 0, g->n * sizeof(double));
    memset(S->rhu, 0, g->n * sizeof(double));
    memset(S->rhv, 0, g->n * sizeof(double));
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++) {
        for (size_t i = GH; i < g->nx + GH; i++) {
            Cell sx[7], sy[7];
            for (int m = 0; m < 7; m++) {
                size_t k = IDX(g, i + m - 3, j);
                sx[m].h = h[k];
                sx[m].un = velocity(h[k], hu[k]);
                sx[m].ut = velocity(h[k], hv[k]);
                sx[m].b = bed[k];
                sx[m].phi = phi[k];
                k = IDX(g, i, j + m - 3);
                sy[m].h = h[k];
                sy[m].un = velocity(h[k], hv[k]);
                sy[m].ut = velocity(h[k], hu[k]);
                sy[m].b = bed[k];
                sy[m].phi = phi[k];
            }
            Axis x = axis_terms(sx, g->dx, order);
            Axis y = axis_terms(sy, g->dy, order);
            size_t k = j * w + i;
            double r_h = -(x.high.flux[0] - x.low.flux[0]) / g->dx -
                         (y.high.flux[0] - y.low.flux[0]) / g->dy;
            S->rhu[k] = -((x.high.flux[1] + x.high.corr_left) - (x.low.flux[1] + x.low.corr_right)) /
                            g->dx +
                        x.source - (y.high.flux[2] - y.low.flux[2]) / g->dy;
            S->rhv[k] = -((y.high.flux[1] + y.high.corr_left) - (y.low.flux[1] + y.low.corr_right)) /
                            g->dy +
                        y.source - (x.high.flux[2] - x.low.flux[2]) / g->dx;
            if (S->has_drive) {
                double px = ((double)(i - GH) + 0.5) * g->dx;
                double py = ((double)(j - GH) + 0.5) * g->dy;
                r_h += drive_source(&S->drive, px, py, t);
            }
            S->rh[k] = r_h;
        }
    }
    if (S->has_disp)
        dispersion_apply(&S->disp, g, S->periodic_y, h, hu, hv, S->rh, S->rhu, S->rhv, phi,
                         &S->work, S->rows_buf);
}

/* solver.rs:534-574 */
static void damp(const or_solver* S, double* h, double* hu, double* hv, double dt) {
    if (S->nsp == 0 && S->manning == 0.0) return;
    const Grid* g = &S->g;
    const size_t w = g->w;
    const double manning = S->manning;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < g->ny + GH; j++)
        for (size_t i = GH; i < g->nx + GH; i++) {
            size_t k = j * w + i;
            for (size_t m = 0; m < S->nsp; m++) {
                double rate = sponge_rate(&S->sponges[m], g, i, j);
                if (rate > 0.0) {
                    double f = exp(-rate * dt);
                    relax_cell(&h[k], &hu[k], &hv[k], S->b[k], S->sponges[m].level, 0.0, 0.0, f);
                }
            }
            if (manning > 0.0 && h[k] > H_FRICTION_MIN) {
                double speed = hypot(hu[k], hv[k]) / h[k];
                double f = or_manning_factor(h[k], speed, dt, manning);
                hu[k] *= f;
                hv[k] *= f;
            }
        }
    clean_dry(g, h, hu, hv);
}

/* solver.rs:509-532 (`follow_breaking`): returns the viscous sub-steps taken */
int or_follow_breaking(or_solver* S, double* h, double* hu, double* hv, double* br, double dt) {
    if (!S->has_disp || !S->disp.breaking.viscosity) return 0;
    const Grid* g = &S->g;
    fill_boundaries(g, S->periodic_y, h, hu, hv, br);
    /* the switch as the surface alone reads it, without the fronts: where they start */
    wc_breaking fresh = S->disp.breaking;
    fresh.viscosity = 0;
    switch_phi(g, S->b, h, br, &fresh, S->periodic_y, S->phi);
    const wc_eddy* e = &S->disp.breaking.eddy;
    eddy_follow(g, e, h, hu, hv, br, S->phi, dt, S->ed_rise, S->ed_mem, S->ed_nu);
    int steps = 0;
    if (e->mixing > 0.0)
        steps = eddy_diffuse(g, S->periodic_y, h, hu, hv, br, S->ed_nu, dt, S->ed_hu, S->ed_hv);
    clean_dry(g, h, hu, hv);
    return steps;
}

/* solver.rs:479-507 */
void or_step(or_solver* S, double* h, double* hu, double* hv, double* br, double* time,
             double dt) {
    const Grid* g = &S->g;
    double t = *time;
    fill_boundaries(g, S->periodic_y, h, hu, hv, br);
    if (S->order == WC_ORDER_FIRST) {
        rhs(S, h, hu, hv, br, t);
        advance(S, h, hu, hv, br, dt, S->s1h, S->s1hu, S->s1hv, S->s1br);
        memcpy(h, S->s1h, g->n * sizeof(double));
        memcpy(hu, S->s1hu, g->n * sizeof(double));
        memcpy(hv, S->s1hv, g->n * sizeof(double));
        memcpy(br, S->s1br, g->n * sizeof(double));
    } else {
        rhs(S, h, hu, hv, br, t);
        advance(S, h, hu, hv, br, dt, S->s1h, S->s1hu, S->s1hv, S->s1br);
        fill_boundaries(g, S->periodic_y, S->s1h, S->s1hu, S->s1hv, S->s1br);
        rhs(S, S->s1h, S->s1hu, S->s1hv, S->s1br, t + dt);
        advance(S, S->s1h, S->s1hu, S->s1hv, S->s1br, dt, S->s2h, S->s2hu, S->s2hv, S->s2br);
        const size_t n = g->n;
#pragma omp parallel for schedule(static) if (THREADED(g))
        for (size_t k = 0; k < n; k++) {
            h[k] = 0.5 * (h[k] + S->s2h[k]);
            hu[k] = 0.5 * (hu[k] + S->s2hu[k]);
            hv[k] = 0.5 * (hv[k] + S->s2hv[k]);
        }
        clean_dry(g, h, hu, hv);
    }
    damp(S, h, hu, hv, dt);
    or_follow_breaking(S, h, hu, hv, br, dt);
    *time = t + dt;
}

/* solver.rs:431-450 with par.rs:99-107: per-row maxima folded in row order */
double or_stable_dt(const or_solver* S, const double* h, const double* hu, const double* hv) {
    const Grid* g = &S->g;
    const size_t w = g->w;
    double* rows = S->rows_buf;
#pragma omp parallel for schedule(static) if (THREADED(g))
    for (size_t j = GH; j < GH + g->ny; j++) {
        double m = 0.0;
        for (size_t k = j * w + GH; k < j * w + GH + g->nx; k++)
            m = max_or_nan(m, rate_at(h, hu, hv, k, g->dx, g->dy));
        rows[j - GH] = m;
    }
    double rate = 0.0;
    for (size_t j = 0; j < g->ny; j++) rate = max_or_nan(rate, rows[j]);
    if (isnan(rate)) return NAN;
    if (rate > 0.0) return S->cfl / rate;
    return INFINITY;
}

/* solver.rs:452-477 */
int or_limiting_cell(const or_solver* S, const double* h, const double* hu, const double* hv,
                     wc_limiting* out) {
    const Grid* g = &S->g;
    int found = 0;
    double worst = 0.0;
    size_t wi = 0, wj = 0;
    for (size_t j = GH; j < GH + g->ny; j++) {
        for (size_t i = GH; i < GH + g->nx; i++) {
            double r = rate_at(h, hu, hv, IDX(g, i, j), g->dx, g->dy);
            if (isnan(r)) {
                found = 1;
                worst = r;
                wi = i;
                wj = j;
                goto done;
            }
            if (r > (found ? worst : 0.0)) {
                found = 1;
                worst = r;
                wi = i;
                wj = j;
            }
        }
    }
done:
    if (!found) return 0;
    size_t k = IDX(g, wi, wj);
    double u = velocity(h[k], hu[k]), v = velocity(h[k], hv[k]);
    out->i = wi - GH;
    out->j = wj - GH;
    out->depth = h[k];
    out->speed = hypot(u, v);
    return 1;
}

/* dispersion.rs:162-201 via solver.rs:336-349 */
void or_breaking_indicator(or_solver* S, const double* h, const double* hu, const double* hv,
                           const double* br, double* out) {
    const Grid* g = &S->g;
    const size_t n = g->n;
    double* fh = (double*)malloc(n * sizeof(double));
    double* fhu = (double*)malloc(n * sizeof(double));
    double* fhv = (double*)malloc(n * sizeof(double));
    double* fbr = (double*)malloc(n * sizeof(double));
    double* phi = (double*)calloc(n, sizeof(double));
    memcpy(fh, h, n * sizeof(double));
    memcpy(fhu, hu, n * sizeof(double));
    memcpy(fhv, hv, n * sizeof(double));
    memcpy(fbr, br, n * sizeof(double));
    fill_boundaries(g, S->periodic_y, fh, fhu, fhv, fbr);
    switch_phi(g, S->b, fh, fbr, breaking_config(S), S->periodic_y, phi);
    size_t m = 0;
    for (size_t j = GH; j < GH + g->ny; j++)
        for (size_t i = GH; i < GH + g->nx; i++, m++) {
            size_t k = IDX(g, i, j);
            out[m] = fh[k] < H_DISPERSION_MIN ? 0.0 : 1.0 - phi[k];
        }
    free(fh);
    free(fhu);
    free(fhv);
    free(fbr);
    free(phi);
}

/* ---- entry points for the unit tests --------------------------------------------------------- */

void or_mirror_ghosts(const wc_grid* wg, double* a) {
    Grid g = mk_grid(wg);
    mirror_ghosts(&g, a);
}

void or_wrap_ghosts_y(const wc_grid* wg, double* a) {
    Grid g = mk_grid(wg);
    wrap_ghosts_y(&g, a);
}

void or_fill_boundaries(const wc_grid* wg, int periodic_y, double* h, double* hu, double* hv,
                        double* br) {
    Grid g = mk_grid(wg);
    fill_boundaries(&g, periodic_y, h, hu, hv, br);
}

void or_matvec(const wc_grid* wg, int periodic_y, const double* heff, const double* mask,
               const double* c, double* px, double* py, double* ax, double* ay) {
    Grid g = mk_grid(wg);
    double* f = (double*)calloc(g.n, sizeof(double));
    matvec(&g, periodic_y, heff, mask, c, f, px, py, ax, ay);
    free(f);
}

void or_dispersion_apply(const wc_grid* wg, int periodic_y, const wc_dispersion* d,
                         const double* h, const double* hu, const double* hv, const double* lh,
                         double* lhu, double* lhv, const double* phi) {
    Grid g = mk_grid(wg);
    Work W;
    if (!work_new(&W, &g)) return;
    double* rows = (double*)calloc(g.rows, sizeof(double));
    dispersion_apply(d, &g, periodic_y, h, hu, hv, lh, lhu, lhv, phi, &W, rows);
    free(rows);
    work_free(&W);
}
