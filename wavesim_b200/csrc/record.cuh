// record.cuh — per-step statistics of a run, recorded on the device after every step.
//
// The reference's driver records, after each step of a run (crates/wavesim/src/lib.rs:1276-1301,
// Stage::record), per interior cell: the surface's running maximum and minimum, the crest-to-
// trough height of every wave period (Stats::close_wave, :920-931), the seconds spent breaking
// (indicator >= 0.8, :1222) and the least-squares first harmonic of the surface at the swell's
// frequency (FirstHarmonic, :1095-1169); it does so in a host loop over the grid every step.
// Here the same sums are kept in HBM and updated by two kernels appended to the step (in the
// captured graph), so a run records without the host. Reads (wave height, breaking fraction,
// harmonic amplitudes) reduce them on demand.
#pragma once

#include "aux.cuh"
#include "common.cuh"

namespace wcb {

// The recorder's scalars (crates/wavesim/src/lib.rs:899-916 and FirstHarmonic's moments).
struct RecDev {
    double from;        // statistics start at this time
    double period;      // wave period of the swell (for per-wave heights and the harmonic)
    double omega;
    double next_wave;   // the wave in progress ends at this time
    double t_last;      // time of the last recorded state
    double seconds;     // recorded time
    double moments[6];  // sums of w, w cos, w sin, w cos^2, w cos sin, w sin^2
    long long waves;    // closed waves
    // set by the cell kernel for the finishing kernel
    double inside;      // the step's recorded length (0: not recorded)
    int close;          // the step closed a wave
    int pad_;
};

struct RecArrays {
    double* eta_max;
    double* eta_min;
    double* wave_max;
    double* wave_min;
    double* wave_sum;    // sum over closed waves of crest to trough
    double* wave_first;  // the first closed wave's heights
    double* wave_last;   // the last closed wave's heights
    double* breaking_seconds;
    double* harm;        // [3][cells]: sums of w eta, w eta cos, w eta sin
};

// 1 - phi where the water is at least H_DISP_MIN deep (dispersion.rs:162-201); with followed
// fronts, 1 where the breaking memory `mem` (or null) is not 0 (dispersion.rs:149-152).
__device__ __forceinline__ float breaking_off(const DevGrid& g, const float4* __restrict__ q,
                                              const float* __restrict__ bed, const BreakingDev& br,
                                              const double* __restrict__ mem, int i, int j) {
    const float h = q[j * g.pitch + i].x;
    if (h < H_DISP_MIN) return 0.f;
    if (mem && mem[j * g.pitch + i] != 0.0) return 1.f;
    auto eta = [&](int di, int dj) {
        const Mapped m = map_cell(g, i + di, j + dj);
        return q[m.k].x + bed[m.k];
    };
    const float ex = (eta(1, 0) - eta(-1, 0)) * g.ix;
    const float ey = (eta(0, 1) - eta(0, -1)) * g.iy;
    const float ratio = fmaxf(eta(0, 0) / h, 0.f);
    return fmaxf(smoothstep(br.er_lo, br.er_inv, ratio), smoothstep(br.sl_lo, br.sl_inv, hypotf(ex, ey)));
}

// Stage::record for every cell (lib.rs:1276-1301): a closing wave first, then this step's sample.
__global__ void record_cells_kernel(DevGrid g, const float4* __restrict__ q, const float* __restrict__ bed,
                                    BreakingDev br, const double* __restrict__ mem, const Ctl* __restrict__ ctl,
                                    RecDev* rd, RecArrays ra) {
    const double t = ctl->t;
    const double inside = fmin(t - rd->t_last, t - rd->from);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        rd->inside = inside > 0.0 ? inside : 0.0;
        rd->close = inside > 0.0 && t > rd->next_wave + 1e-9;
    }
    if (!(inside > 0.0)) return;
    const bool close = t > rd->next_wave + 1e-9;
    const bool first_wave = rd->waves == 0;
    double sn, cs;
    sincos(rd->omega * t, &sn, &cs);
    const double w0 = inside, w1 = inside * cs, w2 = inside * sn;
    const size_t cells = (size_t)g.nx * g.ny;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.nx), j = (int)(c / g.nx);
        const int k = j * g.pitch + i;
        if (close) {  // Stats::close_wave (lib.rs:920-931)
            const double hi = ra.wave_max[c], lo = ra.wave_min[c];
            const double height = isfinite(hi) ? hi - lo : 0.0;
            ra.wave_sum[c] += height;
            ra.wave_last[c] = height;
            if (first_wave) ra.wave_first[c] = height;
            ra.wave_max[c] = -INFINITY;
            ra.wave_min[c] = INFINITY;
        }
        const double eta = depth64(q[k]) + (double)bed[k];
        ra.harm[c] += w0 * eta;
        ra.harm[cells + c] += w1 * eta;
        ra.harm[2 * cells + c] += w2 * eta;
        ra.eta_max[c] = fmax(ra.eta_max[c], eta);
        ra.eta_min[c] = fmin(ra.eta_min[c], eta);
        ra.wave_max[c] = fmax(ra.wave_max[c], eta);
        ra.wave_min[c] = fmin(ra.wave_min[c], eta);
        if (breaking_off(g, q, bed, br, mem, i, j) >= 0.8f) ra.breaking_seconds[c] += inside;
    }
}

// The scalars after every cell has used the old ones (FirstHarmonic::weights, lib.rs:1116-1128).
__global__ void record_finish_kernel(const Ctl* __restrict__ ctl, RecDev* rd) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double t = ctl->t;
    rd->t_last = t;
    const double w = rd->inside;
    if (!(w > 0.0)) return;
    if (rd->close) {
        rd->waves += 1;
        rd->next_wave += rd->period;
    }
    double sn, cs;
    sincos(rd->omega * t, &sn, &cs);
    const double v[6] = {1.0, cs, sn, cs * cs, cs * sn, sn * sn};
    for (int m = 0; m < 6; m++) rd->moments[m] += w * v[m];
    rd->seconds += w;
}

}  // namespace wcb
