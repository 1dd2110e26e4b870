// ensemble.cuh — many independent runs advanced by one persistent launch per step.
//
// No counterpart in the reference, which runs one `Solver` per grid, one after another
// (crates/wavesim/src/lib.rs:1813-1902). Here the members of an ensemble (grids of any size,
// each with its own bed, wave-maker, time step and PCG state) share one cooperative launch: the
// CTAs are split into one group per member, in proportion to the member's cells, and every group
// runs its member's whole SSP-RK2 step — stage tiles, the dispersive solve, the second stage, the
// second solve — with barriers scoped to the group. Members never wait for one another inside a
// step, and a member that has reached its end time skips its work.
#pragma once

#include "common.cuh"
#include "pcg.cuh"
#include "stage.cuh"

namespace wcb {

constexpr int EN_NT = PG_NT;  // 512 threads: one PCG tile per pass, stage tiles at stride 512

struct EnsembleMember {
    StageArgs st[2];   // stage 1 (s^n -> s1) and stage 2 (s1 -> s^{n+1})
    PcgArgs pcg[2];    // the two solves (dispersive members)
    int sgn, order;
    int first_cta, ncta;
};

// A group-scoped barrier on the member's counters (reusing the solve's reduce-barrier).
__device__ __forceinline__ bool member_barrier(const EnsembleMember& M, unsigned& epoch, int cta) {
    __shared__ double red[100];
    double tot[3];
    return reduce_barrier(M.pcg[0], epoch, 0.0, 0.0, 0.0, tot, red, cta, M.ncta);
}

template <int MODE, int ORDER, bool SGN, int TY>
__device__ __forceinline__ void member_stage(const StageArgs& a, int cta, int ncta, float* sm,
                                             StageShared& ss, float& rmax, int& nan_here) {
    const int tx = (a.g.nx + ST_TX - 1) / ST_TX, ty = (a.g.ny + TY - 1) / TY;
    for (int t = cta; t < tx * ty; t += ncta)
        stage_tile<MODE, ORDER, SGN, TY, EN_NT>(a, (t % tx) * ST_TX, (t / tx) * TY, sm, ss, rmax, nan_here);
}

template <int ORDER, bool SGN, int TY>
__device__ __forceinline__ void member_step(const EnsembleMember& M, int cta, float* sm, StageShared& ss) {
    unsigned epoch = 0;
    float rmax = 0.f;
    int nan_here = 0;
    member_stage<MODE_STAGE1, ORDER, SGN, TY>(M.st[0], cta, M.ncta, sm, ss, rmax, nan_here);
    if (!member_barrier(M, epoch, cta)) return;
    if (SGN) {
        if (!pcg_solve(M.pcg[0], cta, M.ncta, epoch)) return;
        if (!member_barrier(M, epoch, cta)) return;
        member_stage<MODE_STAGE1, ORDER, true, TY>(M.st[1], cta, M.ncta, sm, ss, rmax, nan_here);
        if (!member_barrier(M, epoch, cta)) return;
        pcg_solve(M.pcg[1], cta, M.ncta, epoch);
    } else {
        member_stage<MODE_STAGE2, ORDER, false, TY>(M.st[1], cta, M.ncta, sm, ss, rmax, nan_here);
        stage_fold<EN_NT>(M.st[1].ctl, rmax, nan_here, (unsigned)M.ncta);
    }
}

// One step of every member. cta_member maps each CTA to its member. TY is the stage tile height
// and MINB the CTAs per SM the kernel is compiled for; the autotuner picks among them.
template <int TY, int MINB>
__global__ void __launch_bounds__(EN_NT, MINB) ensemble_step_kernel(const EnsembleMember* __restrict__ members,
                                                                  const int* __restrict__ cta_member) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    __shared__ StageShared ss;
    const EnsembleMember& M = members[cta_member[blockIdx.x]];
    if (!M.st[0].ctl->active) return;
    const int cta = blockIdx.x - M.first_cta;
    if (M.sgn) {
        if (M.order == WC_ORDER_FIFTH) member_step<2, true, TY>(M, cta, sm, ss);
        else member_step<1, true, TY>(M, cta, sm, ss);
    } else {
        if (M.order == WC_ORDER_FIFTH) member_step<2, false, TY>(M, cta, sm, ss);
        else member_step<1, false, TY>(M, cta, sm, ss);
    }
}

}  // namespace wcb
