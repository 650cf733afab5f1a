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
    int wx0, wy0;        // window origin (nodes)
    int nbx, nby, nbz;   // window brick grid
    int wnx, wny;        // window extent (nodes, unpadded)
    int src_brick;       // local brick id holding the source node
    int src_node;        // node index inside that brick
    float src_dist;      // distance source -> seed node (m); seed = S(seed) * src_dist
    long long t_off;     // offset of the shot's field in the traveltime pool (floats)
    unsigned long long qbase;  // offset of the shot's bricks in the queue-flag array
    long long v_off;     // offset of the shot's window volume (nz*wnx*wny, z fastest) in
                         // arrays that hold all shots' volumes back to back
    int s_gather;        // 0: the window is brick-aligned, its bricks are model bricks; 1:
                         // slowness is gathered node by node from the model (node_S)
    // Brick index -> coordinates without integer division: b / nbz and (b / nbz) / nbx as
    // (n * m) >> sh, exact for every n below 2^local_bits (set by set_brick_division).
    unsigned long long divz_m, divx_m;
    unsigned divz_sh, divx_sh;
    // 8^3 bricks (TOMO_BRICK_8): 2 x 2 x 2 groups of the 4^3 storage bricks, the last ones
    // partial where nbz, nbx or nby is odd.  Their grid, the group holding the source, the
    // offset of the shot's groups in the group queue flags, and the division constants.
    int gbz8, gbx8, gby8;
    int src_brick8;
    unsigned long long qbase8;
    unsigned long long div8z_m, div8x_m;
    unsigned div8z_sh, div8x_sh;
};

// Multiply-shift constants for an exact n / d over 0 <= n < 2^nbits (nbits <= 31): with
// l = ceil(log2 d) and m = ceil(2^(nbits + l) / d), floor(n / d) = (n m) >> (nbits + l)
// (Granlund & Montgomery, "Division by invariant integers using multiplication", 1994,
// Theorem 4.2: 2^(N+l) <= m d <= 2^(N+l) + 2^l).  n m < 2^63, so it is one 64-bit product.
inline void fastdiv_consts(unsigned d, unsigned nbits, unsigned long long &m, unsigned &sh)
{
    unsigned l = 0;
    while ((1ull << l) < d) l++;
    sh = nbits + l;
    m = ((1ull << sh) + d - 1) / d;
}

// Fills a descriptor's division constants once nbz, nbx (and the 8^3 grid) and the batch's
// local_bits are set.
inline void set_brick_division(ShotDesc &d, unsigned local_bits)
{
    fastdiv_consts((unsigned)d.nbz, local_bits, d.divz_m, d.divz_sh);
    fastdiv_consts((unsigned)d.nbx, local_bits, d.divx_m, d.divx_sh);
    fastdiv_consts((unsigned)(d.gbz8 > 0 ? d.gbz8 : 1), local_bits, d.div8z_m, d.div8z_sh);
    fastdiv_consts((unsigned)(d.gbx8 > 0 ? d.gbx8 : 1), local_bits, d.div8x_m, d.div8x_sh);
}

// The 8^3 group grid of a shot and the group holding its source brick.
inline void set_brick8(ShotDesc &d)
{
    d.gbz8 = (d.nbz + 1) / 2;
    d.gbx8 = (d.nbx + 1) / 2;
    d.gby8 = (d.nby + 1) / 2;
    const int bz = d.src_brick % d.nbz, t = d.src_brick / d.nbz;
    const int bx = t % d.nbx, by = t / d.nbx;
    d.src_brick8 = (bz >> 1) + d.gbz8 * ((bx >> 1) + d.gbx8 * (by >> 1));
}

struct FimLaunch {
    const float *S;       // slowness, brick-major over the padded model
    const void *spare;    // unused.  Without this slot (and with `gather` beside gbx, gbz)
                          // the config-2 batch ran 3 % slower, same inputs, in alternating
                          // runs: the generated code of the parameter loads changes
    float *T;             // traveltime pool (brick-major per shot)
    const ShotDesc *shots;
    int nshots;
    unsigned *qflag;      // per (shot, brick): round+1 it was last queued for
    unsigned *lists;      // 3 work lists of list_cap entries
    unsigned list_cap;
    unsigned *ctrl;       // kCtrlWords control words
    unsigned long long *stats;  // [0] activations, [1] inner iterations, [2] async activation
                                // count, [3] activations that lowered no node
    int gbx, gbz;         // global brick grid (x, z) for S addressing
    float h;              // grid spacing of the update (dx, as the reference)
    int max_inner, max_rounds;
    float change_tol;     // face drops <= this do not re-queue the neighbour
    float inner_tol;      // in-brick iterations stop when no node drops by more than this
    unsigned local_bits;  // item = shot << local_bits | local brick
    unsigned long long spin_limit;
    // Time-band ordering (band > 0, rounds schedule only).  keys[qbase + b]: the smallest
    // new face time pushed to the brick since it was last relaxed (float bits, kNoKey =
    // none); band_min: three rotating arrays of nshots per-shot minima of the keys met in a
    // round.  A brick whose key exceeds its shot's minimum of the previous round by more
    // than band waits for a later round.
    unsigned *keys;
    unsigned *band_min;
    unsigned *park;       // park_rounds + 2 parking lists of list_cap entries (bricks put off)
    unsigned *park_cnt;   // their counts (zeroed before the solve)
    int park_rounds;      // rounds a put-off brick waits before it is tested again (1..14)
    float band;
    // receivers
    int nrec;
    const float *rx, *ry, *rz;
    float *t_recv;        // nshots*nrec
    float dx, dy, dz;
    int nz;
    int gather;           // some shot has ShotDesc::s_gather set (selects the gathering kernel)
    int pair;             // rounds schedule, two bricks per warp (k_fim_pair, k_fim_pair_band)
};

// Host-callable launchers (fim.cu).
cudaError_t fim_brick_model(const float *slow, float *S, int nx, int ny, int nz, int nxx, int nyy,
                            int nzz, cudaStream_t st);
cudaError_t fim_init(float *T, size_t t_count, unsigned *qflag, size_t q_count, unsigned *ctrl,
                     unsigned long long *stats, cudaStream_t st);
// ring_cap > 0: the asynchronous schedule; lists holds a ring of ring_cap = 3 x list_cap
// items (the whole list buffer).
cudaError_t fim_seed(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz, float *T,
                     unsigned *qflag, unsigned *lists, unsigned local_bits, unsigned *ctrl, cudaStream_t st,
                     size_t ring_cap = 0);
// async: the asynchronous schedule (seeded with ring_cap = list_cap), else rounds.
cudaError_t fim_solve(const FimLaunch &p, int block_warps, int occupancy, bool ieee_sqrt, int *grid_out,
                      cudaStream_t st, bool async = false);
// 8^3 bricks, rounds schedule: work items are (shot, 8^3 group); p.qflag / p.list_cap are
// the group queue flags and count; seeded by fim_seed8.  One CTA of 8 warps per group.
cudaError_t fim_solve8(const FimLaunch &p, int occupancy, bool ieee_sqrt, int *grid_out, cudaStream_t st);
cudaError_t fim_seed8(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz, float *T,
                      unsigned *qflag8, unsigned *lists, unsigned local_bits, unsigned *ctrl, cudaStream_t st);
cudaError_t fim_unbrick(const float *T, const ShotDesc *shots, int shot, int nz, float *out,
                        cudaStream_t st);
cudaError_t velocity_to_slowness(const float *v, float *s, size_t n, cudaStream_t st);
// *out_bits = float bits of the largest finite positive entry of v (0 if none).
cudaError_t max_positive(const float *v, size_t n, unsigned *out_bits, cudaStream_t st);

// Warm start (fim.cu): every window node of every shot starts at ceiling * scale
// (volumes at ShotDesc::v_off) instead of INF; non-finite or non-positive entries and
// padding nodes stay INF.
cudaError_t fim_ceiling(float *T, const ShotDesc *shots, int nshots, int nz, const float *ceiling, float scale,
                        cudaStream_t st);
// Per shot (source node excepted): viol[s] counts the nodes whose traveltime is below the
// local update of its final neighbours by more than rel_tol (relative), viol[nshots + s]
// holds the largest such relative deficit (float bits, atomicMax), and viol[2 nshots + s]
// counts the nodes that still hold their ceiling value (ceiling x scale, as fim_ceiling
// stored it): nodes the solve never lowered.  Either count flags a ceiling below the
// true time; the second catches smooth deficits of any size.
cudaError_t fim_verify(const float *T, const float *S, const ShotDesc *shots, int nshots, int gbx,
                       int gbz, float h, float rel_tol, const float *ceiling, float scale, int nz, bool ieee_sqrt,
                       unsigned long long *viol, cudaStream_t st);
// Resets the pool regions (T = INF, queue flags 0) of the listed shots only.
cudaError_t fim_reset_shots(float *T, unsigned *qflag, const ShotDesc *shots, int nshots, cudaStream_t st);
// All shots' window volumes, back to back at ShotDesc::v_off (z fastest, then x, then y).
cudaError_t fim_unbrick_all(const float *T, const ShotDesc *shots, int nshots, int nz, float *out,
                            cudaStream_t st);
cudaError_t receivers_sample(const float *T, const ShotDesc *shots, int nshots, const float *rx, const float *ry,
                             const float *rz, int nrec, float dx, float dy, float dz, int nz, float *t_recv,
                             cudaStream_t st);

}  // namespace tomo
