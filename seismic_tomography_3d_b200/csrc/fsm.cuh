// Noble-Gesret-Belayouni fast sweeping on the device: declarations shared with the host.
#pragma once

#include <cuda_runtime.h>

#include "fim.cuh"

namespace tomo {

// Per-shot data of a batched NGB sweep solve.
struct FsmShot {
    int wx0, wy0, wnx, wny;   // window (model nodes)
    int sidx, sidy, sidz;     // source node in halo-grid coordinates ((int)(s/d) + 1)
    long long t_off;          // offset of the shot's halo grid in the sweep pool (floats)
    float seed_dist[27];      // distances of the 27 seeded nodes (index oz+1 + 3(ox+1) + 9(oy+1))
};

struct FsmLaunch {
    const float *slow;        // model slowness, natural layout nz*nx*ny
    int nx, ny, nz;
    float dx, dy, dz;
    float dz2i, dx2i, dy2i, dz2dx2, dz2dy2, dx2dy2, dsum;  // host-computed as the reference
    float *T;                 // sweep pool: per shot (nz+2)(wnx+2)(wny+2), z fastest
    const FsmShot *shots;
    int nshots;
    int ngroups;              // independent block groups (shots g, g+ngroups, ...)
    unsigned *bar;            // 2 words (count, generation) per group
    unsigned *err;            // DevErr
    unsigned long long spin_limit;
    // result in the brick-major traveltime pool of the FIM (for receivers / rays / volume)
    float *Tb;
    const ShotDesc *desc;
};

cudaError_t fsm_solve(const FsmLaunch &p, int *grid_out, cudaStream_t st);

}  // namespace tomo
