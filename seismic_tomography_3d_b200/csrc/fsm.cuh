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
    long long flag_off;       // tiled schedule: offset of the shot's tile flags
};

// Tiled schedule: a sweep's tiles are kFsmTZ x kFsmTX x kFsmTY nodes of the sweep's own
// (z, x, y) order; tile flags per shot are laid out over the full sweep's tile box.
constexpr int kFsmTZ = 16, kFsmTX = 8, kFsmTY = 8;

// Nodes one sweep visits along one axis: i = i0 + di * l for l in [0, L).
struct FsmRange {
    int i0, di, L;
};

// Sweep q (0..7 source-anchored, 8..15 full) of an axis with sign s (+1 ascending), halo
// extent n and source index sid (accurate_FSM.cpp:267-511).
__host__ __device__ inline FsmRange fsm_sweep_range(int q, int s, int n, int sid)
{
    FsmRange r;
    if (q < 8) {
        if (s > 0) {
            r.i0 = sid > 1 ? sid : 1;
            r.di = 1;
            r.L = n - r.i0;
        } else {
            r.i0 = sid + 1;
            r.di = -1;
            r.L = sid + 2;
        }
    } else {
        if (s > 0) {
            r.i0 = 1;
            r.di = 1;
            r.L = n - 1;
        } else {
            r.i0 = n - 2;
            r.di = -1;
            r.L = n - 1;
        }
    }
    return r;
}

// Octant signs of sweep q (the reference's order): (+,+,+), (-,+,+), (+,+,-), (-,+,-),
// (+,-,+), (-,-,+), (+,-,-), (-,-,-) for (z, x, y).
__host__ __device__ inline int fsm_sign_z(int q) { return (q & 1) ? -1 : 1; }
__host__ __device__ inline int fsm_sign_y(int q) { return (q & 2) ? -1 : 1; }
__host__ __device__ inline int fsm_sign_x(int q) { return (q & 4) ? -1 : 1; }

// Tiles (x, y, z) with x + y + z = d in an A x B x C box: inclusion-exclusion over the
// (n + 1)(n + 2) / 2 non-negative solutions of x + y + z = n.
__host__ __device__ inline long long fsm_tri(long long n) { return n < 0 ? 0 : (n + 1) * (n + 2) / 2; }
__host__ __device__ inline long long fsm_diag_count(int d, int A, int B, int C)
{
    return fsm_tri(d) - fsm_tri(d - A) - fsm_tri(d - B) - fsm_tri(d - C) + fsm_tri(d - A - B) +
           fsm_tri(d - A - C) + fsm_tri(d - B - C) - fsm_tri(d - A - B - C);
}

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
    // Tiled schedule (fsm_solve_tiled).  Sweep q's tiles are handed out in the order
    // (tile diagonal d, shot s, tile on the diagonal); tab[tab_base[q] + d * nshots + s]
    // is the index of the first tile of (d, s) and tab[tab_base[q] + tab_nd[q] * nshots]
    // the sweep's tile count.
    const int *tab;
    int tab_base[16], tab_nd[16];
    unsigned *flags;          // per tile: last sweep (q + 1) that finished it
    unsigned *cursors;        // 16 tile cursors, zeroed before the launch
    unsigned *shot_done;      // per shot and sweep: tiles finished (16 x nshots, zeroed)
    const unsigned *shot_tiles;  // per shot and sweep: tiles of the sweep (16 x nshots)
    int sweep_barrier;        // 1: a grid barrier between sweeps instead of the per-shot counts
};

cudaError_t fsm_solve(const FsmLaunch &p, int *grid_out, cudaStream_t st);
// The same sweeps, tile by tile: every shot's source must lie off the far faces of its
// window (halo index sid <= n - 3 on each axis), so that no read leaves the grid.
cudaError_t fsm_solve_tiled(const FsmLaunch &p, int *grid_out, cudaStream_t st);

}  // namespace tomo
