// nest.cuh — relaxation zones driven by a coarser run (one-way nesting) on the device.
//
// The reference drives a fine grid from a coarse run of the same sea: zone cells (where a set of
// sponges has a rate) relax over each fine step towards a target sampled bilinearly from the
// coarse state, interpolated in time between the coarse states that bracket the step's end
// (crates/wavecore/src/forcing.rs:209-283, Relaxation and relax_cell;
// crates/wavesim/src/lib.rs:1554-1605, Sampler; :1846-1896, the nested step). Here the zone's
// cells, their coarse corners and weights are fixed at set-up; one kernel samples the coarse
// resident state into a target slot, one relaxes the fine resident state after its step.
#pragma once

#include "common.cuh"

namespace wcb {

struct NestCell {
    int k;          // fine storage index
    int kc[4];      // coarse storage indices of the four corners (ghosts mapped as walls)
    float sx[4], sy[4];  // sign of the momentum components there (wall ghosts flip the normal one)
    double w[4];    // bilinear weights
    double rate;    // relaxation rate, 1/s
};

// Sampler::sample (lib.rs:1590-1605): (eta, u, v) from the wet corners (h > 1e-3), weights
// renormalised; no wet corner gives eta = -inf (the zone then dries).
__global__ void nest_sample_kernel(const float4* __restrict__ q, const float* __restrict__ bed,
                                   const NestCell* __restrict__ cells, int n, double* __restrict__ target,
                                   double* __restrict__ time_slot, const Ctl* __restrict__ ctl) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *time_slot = ctl->t;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const NestCell c = cells[m];
        double eta = 0.0, u = 0.0, v = 0.0, wt = 0.0;
        for (int e = 0; e < 4; e++) {
            const float4 s = q[c.kc[e]];
            const double h = depth64(s);
            if (h > 1e-3 && c.w[e] > 0.0) {
                eta += c.w[e] * (h + (double)bed[c.kc[e]]);
                u += c.w[e] * ((double)(s.z * c.sx[e]) / h);
                v += c.w[e] * ((double)(s.w * c.sy[e]) / h);
                wt += c.w[e];
            }
        }
        if (wt > 0.0) {
            target[m] = eta / wt;
            target[n + m] = u / wt;
            target[2 * n + m] = v / wt;
        } else {
            target[m] = -INFINITY;
            target[n + m] = 0.0;
            target[2 * n + m] = 0.0;
        }
    }
}

// Relaxation::apply with the time interpolation of the nested step (lib.rs:1875-1893): the target
// at the step's end between the two sampled coarse states; relax_cell (forcing.rs:213-225), then
// the dry-cell cleanup.
__global__ void nest_relax_kernel(float4* __restrict__ q, const float* __restrict__ bed,
                                  const NestCell* __restrict__ cells, int n, const double* __restrict__ then_,
                                  const double* __restrict__ now_, const double* __restrict__ times,
                                  const Ctl* __restrict__ ctl) {
    const double end = ctl->t, dt = ctl->dt;
    const double t0 = times[0], t1 = times[1];
    double w = (end - t0) / (t1 - t0);
    w = w < 0.0 ? 0.0 : (w > 1.0 ? 1.0 : w);
    if (!(w == w)) w = 1.0;  // t1 == t0: the newer sample
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const NestCell c = cells[m];
        double eta, u, v;
        const double a0 = then_[m], c0 = now_[m];
        if (isfinite(a0) && isfinite(c0)) {
            eta = a0 + w * (c0 - a0);
            u = then_[n + m] + w * (now_[n + m] - then_[n + m]);
            v = then_[2 * n + m] + w * (now_[2 * n + m] - then_[2 * n + m]);
        } else if (w < 0.5) {
            eta = a0, u = then_[n + m], v = then_[2 * n + m];
        } else {
            eta = c0, u = now_[n + m], v = now_[2 * n + m];
        }
        const double f = exp(-c.rate * dt);
        const float4 s = q[c.k];
        double ht = eta - (double)bed[c.k];
        ht = ht > 0.0 ? ht : 0.0;
        double h = f * depth64(s) + (1.0 - f) * ht;
        double hu = f * (double)s.z + (1.0 - f) * ht * u;
        double hv = f * (double)s.w + (1.0 - f) * ht * v;
        if (h < H_DRY_D) {
            h = h > 0.0 ? h : 0.0;
            hu = 0.0;
            hv = 0.0;
        }
        q[c.k] = pack_state(h, (float)hu, (float)hv);
    }
}

}  // namespace wcb
