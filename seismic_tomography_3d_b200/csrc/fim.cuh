// Batched persistent fast-iterative eikonal solver: data structures shared by the
// kernels (fim.cu) and the host context (api.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tomo {

constexpr int kBrick = 4;                    // brick edge (nodes): 4x4x4 bricks, one warp each
constexpr int kBrickNodes = kBrick * kBrick * kBrick;

// Per-shot descriptor of a batched solve (device array, one per shot).
struct ShotDesc {
    int wx0, wy0;        // window origin (nodes, multiples of kBrick)
    int nbx, nby, nbz;   // window brick grid
    int wnx, wny;        // window extent (nodes, unpadded)
    int src_brick;       // local brick id holding the source node
    int src_node;        // node index inside that brick
    float src_dist;      // distance source -> seed node (m); seed = S(seed) * src_dist
    long long t_off;     // offset of the shot's field in the traveltime pool (floats)
    unsigned long long qbase;  // offset of the shot's bricks in the queue-flag array
};

struct FimLaunch {
    const float *S;       // slowness, brick-major over the padded model
    float *T;             // traveltime pool (brick-major per shot)
    const ShotDesc *shots;
    int nshots;
    unsigned *qflag;      // per (shot, brick): round+1 it was last queued for
    unsigned *lists;      // 3 work lists of list_cap entries
    unsigned list_cap;
    unsigned *ctrl;       // kCtrlWords control words
    unsigned long long *stats;  // [0] activations, [1] inner iterations
    int gbx, gbz;         // global brick grid (x, z) for S addressing
    float h;              // grid spacing of the update (dx, as the reference)
    int max_inner, max_rounds;
    float change_tol;     // face drops <= this do not re-queue the neighbour
    float inner_tol;      // in-brick iterations stop when no node drops by more than this
    unsigned local_bits;  // item = shot << local_bits | local brick
    unsigned long long spin_limit;
    // receivers
    int nrec;
    const float *rx, *ry, *rz;
    float *t_recv;        // nshots*nrec
    float dx, dy, dz;
    int nz;
};

// Host-callable launchers (fim.cu).
cudaError_t fim_brick_model(const float *slow, float *S, int nx, int ny, int nz, int nxx, int nyy,
                            int nzz, cudaStream_t st);
cudaError_t fim_init(float *T, size_t t_count, unsigned *qflag, size_t q_count, unsigned *ctrl,
                     unsigned long long *stats, cudaStream_t st);
cudaError_t fim_seed(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz, float *T,
                     unsigned *qflag, unsigned *lists, unsigned local_bits, unsigned *ctrl, cudaStream_t st);
cudaError_t fim_solve(const FimLaunch &p, int block_warps, int occupancy, bool ieee_sqrt, int *grid_out,
                      cudaStream_t st);
cudaError_t fim_unbrick(const float *T, const ShotDesc *shots, int shot, int nz, float *out,
                        cudaStream_t st);
cudaError_t velocity_to_slowness(const float *v, float *s, size_t n, cudaStream_t st);

}  // namespace tomo
