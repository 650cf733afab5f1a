// Noble-Gesret-Belayouni fast sweeping on the device, bit-exact with the reference's
// Accurate_FSM (src/eikonal/accurate_FSM/accurate_FSM.cpp:159-650).
//
// The reference runs 8 source-anchored sweeps and 8 full sweeps, each a Gauss-Seidel pass
// in one octant order (k outer, j, i inner).  The local operator reads only the node itself
// and its upwind neighbours in that octant, which all lie on earlier diagonal planes
// (constant (i-i0)di + (j-j0)dj + (k-k0)dk), so updating one diagonal plane at a time, all
// nodes of a plane in parallel, performs exactly the same operations on exactly the same
// values as the sequential loop.  With FP32 arithmetic in the reference's order (this file
// is compiled with -fmad=false; division and square root are IEEE) the result is the
// reference's, bit for bit.  All shots of a batch sweep together in one cooperative launch;
// blocks form `ngroups` independent groups (shots g, g+ngroups, ...), each with its own
// bounded barrier between planes.  The default schedule (k_fsm_tiled, below) orders the
// same updates tile by tile instead of plane by plane.
#include "common.cuh"
#include "fsm.cuh"

namespace tomo {

namespace {

// octant signs (z, x, y) of the 8 sweeps, in the reference's order
__device__ __constant__ int kSgn[8][3] = {{1, 1, 1},  {-1, 1, 1},  {1, 1, -1},  {-1, 1, -1},
                                          {1, -1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, -1, -1}};

__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }  // std::max

// Group barrier over the blocks of one group (bounded spin; false on any error).  Every
// thread of a block gets thread 0's reading of the error word, so a block never splits over
// an error raised by another block while it passes the barrier.
__device__ __forceinline__ bool group_barrier(unsigned *bar, unsigned nblocks, unsigned *err,
                                              unsigned long long spin_limit)
{
    __shared__ unsigned err_seen;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = ld_volatile(bar + 1);
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long spins = 0;
            while (ld_volatile(bar + 1) == gen) {
                if (++spins > spin_limit || ld_volatile(err) != 0u) {
                    atomicCAS(err, 0u, (unsigned)kDevBarrierTimeout);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        err_seen = ld_volatile(err);
    }
    __syncthreads();
    return err_seen == 0u;
}

struct ShotGrid {
    const FsmShot *s;
    float *T;
    long long n;
    int nxx, nyy, nzz;
};

// Flattened read like the reference: past a column edge lands in the next column; past the
// end of the shot's grid (undefined in the reference) reads 1e6.
__device__ __forceinline__ float tget(const ShotGrid &g, long long idx)
{
    return (idx >= 0 && idx < g.n) ? __ldcg(g.T + idx) : 1e6f;
}

// Slowness of halo-grid node (i, j, k): the window cropped and replicated by one node.
__device__ __forceinline__ const float *sptr(const FsmLaunch &p, const ShotGrid &g, int i, int j, int k)
{
    const int z = min(max(i - 1, 0), p.nz - 1);
    const int x = g.s->wx0 + min(max(j - 1, 0), g.s->wnx - 1);
    const int y = g.s->wy0 + min(max(k - 1, 0), g.s->wny - 1);
    return p.slow + z + (long long)x * p.nz + (long long)y * p.nx * p.nz;
}

__device__ __forceinline__ float sget(const FsmLaunch &p, const ShotGrid &g, int i, int j, int k)
{
    return __ldg(sptr(p, g, i, j, k));
}

// Traveltimes and slowness of one shot's halo grid as the sweep reads them, from global
// memory with the reference's flattened indexing (the plane schedule).
struct GlobalAcc {
    const FsmLaunch &p;
    const ShotGrid &g;
    __device__ __forceinline__ float t(int i, int j, int k) const
    {
        return tget(g, i + j * (long long)g.nzz + k * ((long long)g.nxx * g.nzz));
    }
    __device__ __forceinline__ float self(int i, int j, int k) const
    {
        return __ldcg(g.T + i + j * (long long)g.nzz + k * ((long long)g.nxx * g.nzz));
    }
    __device__ __forceinline__ float s(int i, int j, int k) const { return sget(p, g, i, j, k); }
};

// Inputs of one node update: the node's own value, its upwind traveltimes, and the
// slowness minima the operator uses -- m1..m3 (the 1D candidates), r1..r3 (the 2D
// candidates) and r0 (the 3D candidate).
struct NgbIn {
    float self, tv, te, tn, tev, ten, tnv, tnve;
    float m1, m2, m3, r1, r2, r3, r0;
};

// Accurate_FSM::inner_sweep (accurate_FSM.cpp:159-265) from the minima on: the same
// operations in the same order (this file is compiled with -fmad=false).
// kBranchFree: every candidate is computed and kept only where the reference's test holds
// (a NaN from a negative discriminant is dropped with it) -- the same values, without the
// branches.  It pays where the warps wait on the wavefront (one shot) and costs where they
// issue (batches, whose branches skip candidates no lane needs).
template <bool kBranchFree = false>
__device__ __forceinline__ float ngb_core(const FsmLaunch &p, const NgbIn &v)
{
    const float tv = v.tv, te = v.te, tn = v.tn, tev = v.tev, ten = v.ten, tnv = v.tnv, tnve = v.tnve;
    const float dz2i = p.dz2i, dx2i = p.dx2i, dy2i = p.dy2i;
    const float t1D1 = tv + p.dz * v.m1;
    const float t1D2 = te + p.dx * v.m2;
    const float t1D3 = tn + p.dy * v.m3;
    const float t1D = smin(t1D1, smin(t1D2, t1D3));

    if (kBranchFree) {
        float Sref = v.r1;
        float ta = tev + te - tv;
        float tb = tev - te + tv;
        float cand = ((tb * dz2i + ta * dx2i) +
                      sqrtf(4.0f * Sref * Sref * (dz2i + dx2i) - dz2i * dx2i * (ta - tb) * (ta - tb))) /
                     (dz2i + dx2i);
        const float c2D1 = ((tv < te + p.dx * Sref) && (te < tv + p.dz * Sref)) ? cand : 1e6f;
        Sref = v.r2;
        ta = tv - tn + tnv;
        tb = tn - tv + tnv;
        cand = ((ta * dz2i + tb * dy2i) +
                sqrtf(4.0f * Sref * Sref * (dz2i + dy2i) - dz2i * dy2i * (ta - tb) * (ta - tb))) /
               (dz2i + dy2i);
        const float c2D2 = ((tv < tn + p.dy * Sref) && (tn < tv + p.dz * Sref)) ? cand : 1e6f;
        Sref = v.r3;
        ta = te - tn + ten;
        tb = tn - te + ten;
        cand = ((ta * dx2i + tb * dy2i) +
                sqrtf(4.0f * Sref * Sref * (dx2i + dy2i) - dx2i * dy2i * (ta - tb) * (ta - tb))) /
               (dx2i + dy2i);
        const float c2D3 = ((te < tn + p.dy * Sref) && (tn < te + p.dx * Sref)) ? cand : 1e6f;
        const float c2D = smin(c2D1, smin(c2D2, c2D3));
        Sref = v.r0;
        ta = te - 0.5f * tn + 0.5f * ten - 0.5f * tv + 0.5f * tev - tnv + tnve;
        tb = tv - 0.5f * tn + 0.5f * tnv - 0.5f * te + 0.5f * tev - ten + tnve;
        const float tc = tn - 0.5f * te + 0.5f * ten - 0.5f * tv + 0.5f * tnv - tev + tnve;
        const float t2 = 9.0f * Sref * Sref * p.dsum;
        const float t3 =
            p.dz2dx2 * (ta - tb) * (ta - tb) + p.dz2dy2 * (tb - tc) * (tb - tc) + p.dx2dy2 * (ta - tc) * (ta - tc);
        const float t1 = tb * dz2i + ta * dx2i + tc * dy2i;
        cand = (t1 + sqrtf(t2 - t3)) / p.dsum;
        const float c3D = (smin(t1D, c2D) > smax(tv, smax(te, tn)) && t2 >= t3) ? cand : 1e6f;
        return smin(v.self, smin(t1D, smin(c2D, c3D)));
    }
    float t2D1 = 1e6f, t2D2 = 1e6f, t2D3 = 1e6f, ta, tb, tc, Sref;
    Sref = v.r1;
    if ((tv < te + p.dx * Sref) && (te < tv + p.dz * Sref)) {
        ta = tev + te - tv;
        tb = tev - te + tv;
        t2D1 = ((tb * dz2i + ta * dx2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dx2i) - dz2i * dx2i * (ta - tb) * (ta - tb))) /
               (dz2i + dx2i);
    }
    Sref = v.r2;
    if ((tv < tn + p.dy * Sref) && (tn < tv + p.dz * Sref)) {
        ta = tv - tn + tnv;
        tb = tn - tv + tnv;
        t2D2 = ((ta * dz2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dy2i) - dz2i * dy2i * (ta - tb) * (ta - tb))) /
               (dz2i + dy2i);
    }
    Sref = v.r3;
    if ((te < tn + p.dy * Sref) && (tn < te + p.dx * Sref)) {
        ta = te - tn + ten;
        tb = tn - te + ten;
        t2D3 = ((ta * dx2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dx2i + dy2i) - dx2i * dy2i * (ta - tb) * (ta - tb))) /
               (dx2i + dy2i);
    }
    const float t2D = smin(t2D1, smin(t2D2, t2D3));

    float t3D = 1e6f;
    Sref = v.r0;
    ta = te - 0.5f * tn + 0.5f * ten - 0.5f * tv + 0.5f * tev - tnv + tnve;
    tb = tv - 0.5f * tn + 0.5f * tnv - 0.5f * te + 0.5f * tev - ten + tnve;
    tc = tn - 0.5f * te + 0.5f * ten - 0.5f * tv + 0.5f * tnv - tev + tnve;
    if (smin(t1D, t2D) > smax(tv, smax(te, tn))) {
        const float t2 = 9.0f * Sref * Sref * p.dsum;
        const float t3 = p.dz2dx2 * (ta - tb) * (ta - tb) + p.dz2dy2 * (tb - tc) * (tb - tc) + p.dx2dy2 * (ta - tc) * (ta - tc);
        if (t2 >= t3) {
            const float t1 = tb * dz2i + ta * dx2i + tc * dy2i;
            t3D = (t1 + sqrtf(t2 - t3)) / p.dsum;
        }
    }
    return smin(v.self, smin(t1D, smin(t2D, t3D)));
}

// The update with the reference's own neighbour indices and minima, read through the
// accessor with the reference's flattened indexing (the plane schedule).
template <class Acc>
__device__ __forceinline__ float ngb_update(const FsmLaunch &p, const Acc &A, int nxx, int nyy, int nzz, int i, int j,
                                            int k, int sgntz, int sgntx, int sgnty)
{
    const int sgnvz = sgntz == 1, sgnvx = sgntx == 1, sgnvy = sgnty == 1;
    const int i1 = i - sgnvz, j1 = j - sgnvx, k1 = k - sgnvy;
    const int jm = max(j - 1, 1), jp = min(j, nxx - 1), km = max(k - 1, 1), kp = min(k, nyy - 1);
    const int im = max(i - 1, 1), ip = min(i, nzz - 1);
    NgbIn v;
    v.self = A.self(i, j, k);
    v.tv = A.t(i - sgntz, j, k);
    v.te = A.t(i, j - sgntx, k);
    v.tn = A.t(i, j, k - sgnty);
    v.tev = A.t(i - sgntz, j - sgntx, k);
    v.ten = A.t(i, j - sgntx, k - sgnty);
    v.tnv = A.t(i - sgntz, j, k - sgnty);
    v.tnve = A.t(i - sgntz, j - sgntx, k - sgnty);
    v.m1 = smin(A.s(i1, jm, km), smin(A.s(i1, jm, kp), smin(A.s(i1, jp, km), A.s(i1, jp, kp))));
    v.m2 = smin(A.s(im, j1, km), smin(A.s(ip, j1, km), smin(A.s(im, j1, kp), A.s(ip, j1, kp))));
    v.m3 = smin(A.s(im, jm, k1), smin(A.s(im, jp, k1), smin(A.s(ip, jm, k1), A.s(ip, jp, k1))));
    v.r1 = smin(A.s(i1, j1, km), A.s(i1, j1, kp));
    v.r2 = smin(A.s(i1, jm, k1), A.s(i1, jp, k1));
    v.r3 = smin(A.s(im, j1, k1), A.s(ip, j1, k1));
    v.r0 = A.s(i1, j1, k1);
    return ngb_core(p, v);
}

}  // namespace

__global__ void __launch_bounds__(256, 3) k_fsm_sweeps(FsmLaunch p)
{
    const int G = p.ngroups;
    const int grp = blockIdx.x % G;
    const unsigned gblocks = (gridDim.x - grp + G - 1) / G;
    const int gb = blockIdx.x / G;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const long long gwarp = (long long)gb * wpb + (threadIdx.x >> 5);
    const long long nwarps = (long long)gblocks * wpb;
    const long long gthread = (long long)gb * blockDim.x + threadIdx.x;
    const long long nthreads = (long long)gblocks * blockDim.x;
    unsigned *bar = p.bar + 2 * grp;
    const int nzz = p.nz + 2;
    const int ns = (p.nshots - grp + G - 1) / G;  // shots of this group: grp + m*G

    // T = 1e6 on the shots' halo grids, then the 27 analytic seeds (accurate_FSM.cpp:591-630)
    for (int m = 0; m < ns; m++) {
        const FsmShot &s = p.shots[grp + m * G];
        const long long n = (long long)nzz * (s.wnx + 2) * (s.wny + 2);
        for (long long q = gthread; q < n; q += nthreads) __stcg(p.T + s.t_off + q, 1e6f);
    }
    if (!group_barrier(bar, gblocks, p.err, p.spin_limit)) return;
    for (long long q = gthread; q < (long long)ns * 27; q += nthreads) {
        const FsmShot &s = p.shots[grp + (int)(q / 27) * G];
        const int e = (int)(q % 27), oz = e % 3 - 1, ox = (e / 3) % 3 - 1, oy = e / 9 - 1;
        const int nxx = s.wnx + 2;
        const long long sid = s.sidz + (long long)s.sidx * nzz + (long long)s.sidy * nxx * nzz;
        ShotGrid g{&s, p.T + s.t_off, 0, nxx, s.wny + 2, nzz};
        const float S0 = sget(p, g, s.sidz, s.sidx, s.sidy);
        __stcg(p.T + s.t_off + sid + oz + (long long)ox * nzz + (long long)oy * nxx * nzz, S0 * s.seed_dist[e]);
    }
    if (!group_barrier(bar, gblocks, p.err, p.spin_limit)) return;

    for (int q = 0; q < 16; q++) {
        const int sgz = kSgn[q & 7][0], sgx = kSgn[q & 7][1], sgy = kSgn[q & 7][2];
        int W = 0;
        for (int m = 0; m < ns; m++) {
            const FsmShot &s = p.shots[grp + m * G];
            const FsmRange rz = fsm_sweep_range(q, sgz, nzz, s.sidz), rx = fsm_sweep_range(q, sgx, s.wnx + 2, s.sidx),
                           ry = fsm_sweep_range(q, sgy, s.wny + 2, s.sidy);
            W = max(W, rz.L + rx.L + ry.L - 2);
        }
        for (int w = 0; w < W; w++) {
            // one warp per (shot, c) row of the plane; lanes stride over a
            for (long long row = gwarp; row < (long long)ns * nzz; row += nwarps) {
                const int m = (int)(row / nzz), c = (int)(row % nzz);
                const FsmShot &s = p.shots[grp + m * G];
                const FsmRange rz = fsm_sweep_range(q, sgz, nzz, s.sidz), rx = fsm_sweep_range(q, sgx, s.wnx + 2, s.sidx),
                               ry = fsm_sweep_range(q, sgy, s.wny + 2, s.sidy);
                if (c >= rz.L) continue;
                const int t = w - c;
                const int a_lo = max(0, t - (ry.L - 1)), a_hi = min(rx.L - 1, t);
                if (a_lo > a_hi) continue;
                ShotGrid g{&s, p.T + s.t_off, (long long)nzz * (s.wnx + 2) * (s.wny + 2), s.wnx + 2, s.wny + 2, nzz};
                const int i = rz.i0 + rz.di * c;
                for (int a = a_lo + lane; a <= a_hi; a += 32) {
                    const int j = rx.i0 + rx.di * a, k = ry.i0 + ry.di * (t - a);
                    const float v = ngb_update(p, GlobalAcc{p, g}, g.nxx, g.nyy, g.nzz, i, j, k, sgz, sgx, sgy);
                    __stcg(g.T + i + (long long)j * nzz + (long long)k * g.nxx * nzz, v);
                }
            }
            if (!group_barrier(bar, gblocks, p.err, p.spin_limit)) return;
        }
    }

    // reduce_model (accurate_FSM.cpp:62-72) into the brick-major pool of the shot
    for (int m = 0; m < ns; m++) {
        const int sidx = grp + m * G;
        const FsmShot &s = p.shots[sidx];
        const ShotDesc &d = p.desc[sidx];
        const long long n = (long long)d.nbx * d.nby * d.nbz * kBrickNodes;
        const int nxx = s.wnx + 2;
        for (long long e = gthread; e < n; e += nthreads) {
            const long long b = e / kBrickNodes;
            const int node = (int)(e % kBrickNodes);
            const int bz = (int)(b % d.nbz);
            const long long tq = b / d.nbz;
            const int bx = (int)(tq % d.nbx), by = (int)(tq / d.nbx);
            const int z = bz * 4 + (node & 3), x = bx * 4 + ((node >> 2) & 3), y = by * 4 + (node >> 4);
            float v = kInf;
            if (z < p.nz && x < s.wnx && y < s.wny)
                v = __ldcg(p.T + s.t_off + (z + 1) + (long long)(x + 1) * nzz + (long long)(y + 1) * nxx * nzz);
            p.Tb[d.t_off + e] = v;
        }
    }
}

cudaError_t fsm_solve(const FsmLaunch &p, int *grid_out, cudaStream_t st)
{
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fsm_sweeps, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = nsm * per_sm;
    if (p.ngroups < 1 || p.ngroups > grid) return cudaErrorInvalidValue;
    if (grid_out) *grid_out = grid;
    FsmLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel((const void *)k_fsm_sweeps, dim3(grid), dim3(256), args, 0, st);
}

// -------------------------------------------------------------------------------------
// Tiled schedule.  One sweep is a Gauss-Seidel pass whose node updates depend only on the
// upwind neighbours of the sweep's octant.  The sweep's node box (sweep order z, x, y) is
// cut into kFsmTZ x kFsmTX x kFsmTY tiles; a tile depends only on the (up to 7) tiles
// below it on some axes, so tiles are handed out in the order of their tile diagonal
// tc + ta + tb.  One warp relaxes one tile in shared memory, diagonal plane by diagonal
// plane (the nodes of a plane are independent), after waiting for its upwind tiles' flags;
// every tile it waits on was handed out before its own and every CTA is resident, so the
// waits end.  Each node sees exactly the values it sees in the sequential loop, and the
// update is the same function, so the result is the plane schedule's bit for bit -- with no
// grid barrier between sweeps of a batch: a shot's tile of sweep q + 1 also waits until all
// of that shot's sweep-q tiles are finished (a per-shot count), since those read its nodes
// in sweep q's order; shots are independent, so one shot's next sweep overlaps another's
// drain.  The sweep-q tiles were all handed out before any sweep-(q + 1) tile, so this
// wait ends too.  A single shot keeps a grid barrier between sweeps (sweep_barrier).
// Every source must lie off
// the far faces of its window (halo index sid <= n - 3), so that no read leaves the grid
// (the reference's flattened reads would otherwise cross a column edge).
// -------------------------------------------------------------------------------------
namespace {

// Unroll depth of the tile staging loop.  Config-2 batch (64 shots), ms per NGB solve with the
// slowness by cp.async and the octant-specialised plane loop: 4 -> 52.1, 5 -> 49.3, 6 -> 48.6,
// 7 -> 49.1, 8 -> 55.6 (128 registers); 6 with node indices by division instead of the
// incremental ones: 49.7.
constexpr int kStageUnroll = 6;
constexpr int kHZ = kFsmTZ + 1, kHX = kFsmTX + 1, kHY = kFsmTY + 1;  // a tile + one layer per axis
// Strides of the staged arrays (z, then x; words): padded from 17 x 9 so that the lanes of a
// diagonal-plane pass, which differ by (+-19 -+ 1) a + (+-190 -+ 1) b words, fall in
// distinct banks (a search over the plane order and the 8 sweep signs: 548 shared-memory
// wavefronts per tile instead of 1,280).
constexpr int kPZ = 19, kPX = 10;
constexpr int kHN = kPZ * kPX * kHY;
constexpr int kTileN = kFsmTZ * kFsmTX * kFsmTY;
constexpr int kNPlanes = kFsmTZ + kFsmTX + kFsmTY - 2;
static_assert(kFsmTZ <= 32 && kFsmTX <= 8 && kFsmTY <= 8, "plane table packs (c, a, b) in 5 + 3 + 3 bits");
static_assert(kPZ >= kHZ && kPX >= kHX, "padded strides");

// The update on a tile staged in shared memory.  sget clamps every index into the window,
// so the slowness at halo indices -1, 0 and 1 of an axis is one value, and the operator's
// max(i - 1, 1) and min(i, n - 1) read the values at i - 1 and i: every minimum comes from
// the node's 2 x 2 x 2 cell cube (halo indices i-1..i, j-1..j, k-1..k).  A minimum of
// floats is exact and independent of its order, so each has the reference's value, and
// ngb_core does the rest of the reference's arithmetic.
//   Tt + tb: the node in the traveltime tile; oz, ox, oy: word offsets of one step against
//   the sweep along z, x, y;  St + sb: cell (i-1, j-1, k-1) in the slowness tile;
//   cz, cx, cy: 1 - sgnv of each axis (the cube index of i1, j1, k1).
template <bool kBranchFree>
__device__ __forceinline__ float ngb_update_tile(const FsmLaunch &p, const float *Tt, int tb, int oz, int ox, int oy,
                                                 const float *St, int sb, int cz, int cx, int cy)
{
    const float *c = St + sb;
    auto C = [&](int dz, int dx, int dy) { return c[dz + kPZ * dx + kPZ * kPX * dy]; };
    NgbIn v;
    v.self = Tt[tb];
    v.tv = Tt[tb - oz];
    v.te = Tt[tb - ox];
    v.tn = Tt[tb - oy];
    v.tev = Tt[tb - oz - ox];
    v.ten = Tt[tb - ox - oy];
    v.tnv = Tt[tb - oz - oy];
    v.tnve = Tt[tb - oz - ox - oy];
    v.m1 = smin(C(cz, 0, 0), smin(C(cz, 0, 1), smin(C(cz, 1, 0), C(cz, 1, 1))));
    v.m2 = smin(C(0, cx, 0), smin(C(1, cx, 0), smin(C(0, cx, 1), C(1, cx, 1))));
    v.m3 = smin(C(0, 0, cy), smin(C(0, 1, cy), smin(C(1, 0, cy), C(1, 1, cy))));
    v.r1 = smin(C(cz, cx, 0), C(cz, cx, 1));
    v.r2 = smin(C(cz, 0, cy), C(cz, 1, cy));
    v.r3 = smin(C(0, cx, cy), C(1, cx, cy));
    v.r0 = C(cz, cx, cy);
    return ngb_core<kBranchFree>(p, v);
}

// Asynchronous 4-byte copy global -> shared (cp.async, through L1).  Only for the slowness,
// which nothing writes while a solve runs, so an L1 line can never be stale; the
// traveltimes, written by other SMs between tiles, are read through L2 (__ldcg).
__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Waits for this thread's cp.async copies; a warp barrier after it shows them to the warp.
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One tile of a sweep of octant Q (sweep q with q & 7 == Q), diagonal plane by diagonal
// plane.  With the octant's steps compile-time constants every staged read is a shared-
// memory load at a constant offset from the node, and the reads of the 2 x 2 x 2 cell cube
// that several minima share are loaded once.
//   t0: the tile's node (0, 0, 0) in Ts; dts: Ts word of a node minus the Ss word of its
//   cell (i-1, j-1, k-1); nc, na, nb: the sweep's nodes left on each axis from the tile's
//   first node.
template <int Q, bool kBranchFree>
__device__ __forceinline__ void relax_tile(const FsmLaunch &p, float *Ts, const float *Ss,
                                           const unsigned short *plane, const int *pstart, int lane, int t0, int dts,
                                           int nc, int na, int nb)
{
    constexpr int sz = (Q & 1) ? -1 : 1, sy = (Q & 2) ? -1 : 1, sx = (Q & 4) ? -1 : 1;
    constexpr int oz = sz, ox = sx * kPZ, oy = sy * kPZ * kPX;  // one step along the sweep
    constexpr int cz = sz == 1 ? 0 : 1, cx = sx == 1 ? 0 : 1, cy = sy == 1 ? 0 : 1;
    for (int w = 0; w < kNPlanes; w++) {
        for (int m = pstart[w] + lane; m < pstart[w + 1]; m += 32) {
            const unsigned e = plane[m];
            const int c = (int)(e & 31u), a = (int)((e >> 5) & 7u), b = (int)(e >> 8);
            if (c < nc && a < na && b < nb) {
                const int tn = t0 + oz * c + ox * a + oy * b;
                Ts[tn] = ngb_update_tile<kBranchFree>(p, Ts, tn, oz, ox, oy, Ss, tn - dts, cz, cx, cy);
            }
        }
        __syncwarp();
    }
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }

// Lowest halo index of the tile's own nodes on one axis (l0: the tile's first local index).
__device__ __forceinline__ int tile_lo(const FsmRange &r, int l0, int T)
{
    return r.di > 0 ? r.i0 + l0 : r.i0 - (l0 + T - 1);
}

}  // namespace

template <bool kBranchFree>
__global__ void __launch_bounds__(256, 2) k_fsm_tiled(FsmLaunch p)
{
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    float *Ts = smem + warp * 2 * kHN, *Ss = Ts + kHN;
    unsigned short *plane = reinterpret_cast<unsigned short *>(smem + wpb * 2 * kHN);
    int *pstart = reinterpret_cast<int *>(plane + kTileN);
    // the tile's nodes (c, a, b) ordered by diagonal plane c + a + b
    if (threadIdx.x < kNPlanes) {
        const int w = threadIdx.x;
        int m = 0;
        for (int v = 0; v < w; v++)
            m += (int)fsm_diag_count(v, kFsmTZ, kFsmTX, kFsmTY);
        pstart[w] = m;
        for (int b = 0; b < kFsmTY; b++)
            for (int a = 0; a < kFsmTX; a++) {
                const int c = w - a - b;
                if (c >= 0 && c < kFsmTZ) plane[m++] = (unsigned short)(c | (a << 5) | (b << 8));
            }
        if (w == kNPlanes - 1) pstart[kNPlanes] = m;
    }
    const long long gthread = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    const int nzz = p.nz + 2;

    // T = 1e6 on the shots' halo grids, then the 27 analytic seeds (accurate_FSM.cpp:591-630)
    for (int m = 0; m < p.nshots; m++) {
        const FsmShot &s = p.shots[m];
        const long long n = (long long)nzz * (s.wnx + 2) * (s.wny + 2);
        for (long long q = gthread; q < n; q += nthreads) __stcg(p.T + s.t_off + q, 1e6f);
    }
    if (!group_barrier(p.bar, gridDim.x, p.err, p.spin_limit)) return;
    for (long long q = gthread; q < (long long)p.nshots * 27; q += nthreads) {
        const FsmShot &s = p.shots[(int)(q / 27)];
        const int e = (int)(q % 27), oz = e % 3 - 1, ox = (e / 3) % 3 - 1, oy = e / 9 - 1;
        const int nxx = s.wnx + 2;
        const long long sid = s.sidz + (long long)s.sidx * nzz + (long long)s.sidy * nxx * nzz;
        ShotGrid g{&s, p.T + s.t_off, 0, nxx, s.wny + 2, nzz};
        const float S0 = sget(p, g, s.sidz, s.sidx, s.sidy);
        __stcg(p.T + s.t_off + sid + oz + (long long)ox * nzz + (long long)oy * nxx * nzz, S0 * s.seed_dist[e]);
    }
    if (!group_barrier(p.bar, gridDim.x, p.err, p.spin_limit)) return;

    const int S = p.nshots;
    for (int q = 0; q < 16; q++) {
        const int sgz = fsm_sign_z(q), sgx = fsm_sign_x(q), sgy = fsm_sign_y(q);
        const int *tab = p.tab + p.tab_base[q];
        const int nd = p.tab_nd[q];
        const int total = tab[nd * S];
        for (;;) {
            int item = 0;
            if (lane == 0) item = ld_volatile(p.err) != 0u ? total : (int)atomicAdd(p.cursors + q, 1u);
            item = __shfl_sync(kFull, item, 0);
            if (item >= total) break;
            // (diagonal, shot): the last table entry <= item (tab[lo] <= item < tab[hi]).  A
            // warp-wide search (32 probes per step, 2-3 dependent loads instead of 12) measured
            // 3 % slower on the config-2 batch: these loads are broadcasts that hit L1.
            int lo = 0, hi = nd * S;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(tab + mid) <= item)
                    lo = mid;
                else
                    hi = mid;
            }
            const int d = lo / S, si = lo % S;
            int r = item - __ldg(tab + lo);
            const FsmShot &sh = p.shots[si];
            const int nxx = sh.wnx + 2, nyy = sh.wny + 2;
            const FsmRange rz = fsm_sweep_range(q, sgz, nzz, sh.sidz), rx = fsm_sweep_range(q, sgx, nxx, sh.sidx),
                           ry = fsm_sweep_range(q, sgy, nyy, sh.sidy);
            const int A = cdiv(rz.L, kFsmTZ), B = cdiv(rx.L, kFsmTX), C = cdiv(ry.L, kFsmTY);
            // the r-th tile (tc, ta, tb) of diagonal d, tb ascending, then ta
            int tc = 0, ta = 0, tb = max(0, d - (A - 1) - (B - 1));
            for (; tb <= min(C - 1, d); tb++) {
                const int e = d - tb, alo = max(0, e - (A - 1)), ahi = min(B - 1, e);
                if (r <= ahi - alo) {
                    ta = alo + r;
                    tc = e - ta;
                    break;
                }
                r -= ahi - alo + 1;
            }
            // wait for the upwind tiles of this sweep (lanes 0-6: one each) and, lane 7, for
            // the end of the shot's previous sweep, whose tiles read this tile's nodes in their
            // own order (a per-shot count of finished tiles instead of a grid barrier, so that
            // shots that finish a sweep early start the next one while others drain theirs)
            const int fa = cdiv(nzz - 1, kFsmTZ), fb = cdiv(nxx - 1, kFsmTX);
            unsigned *flags = p.flags + sh.flag_off;
            bool gave_up = false;
            if (lane == 7 && q > 0 && !p.sweep_barrier) {
                const unsigned need = __ldg(p.shot_tiles + (size_t)si * 16 + (q - 1));
                const unsigned *cnt = p.shot_done + (size_t)si * 16 + (q - 1);
                unsigned long long spins = 0;
                while (ld_acquire(cnt) < need) {
                    if (++spins > p.spin_limit || ld_volatile(p.err) != 0u) {
                        atomicCAS(p.err, 0u, (unsigned)kDevBarrierTimeout);
                        gave_up = true;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            if (lane < 7) {
                const int dc = (lane + 1) & 1, da = ((lane + 1) >> 1) & 1, db = (lane + 1) >> 2;
                if (tc >= dc && ta >= da && tb >= db) {
                    const unsigned *f = flags + (tc - dc) + fa * ((ta - da) + fb * (tb - db));
                    unsigned long long spins = 0;
                    while (ld_acquire(f) != (unsigned)(q + 1)) {
                        if (++spins > p.spin_limit || ld_volatile(p.err) != 0u) {
                            atomicCAS(p.err, 0u, (unsigned)kDevBarrierTimeout);
                            gave_up = true;
                            break;
                        }
                        __nanosleep(32);
                    }
                }
            }
            if (__any_sync(kFull, gave_up)) break;  // the whole warp leaves the sweep
            __syncwarp();  // the upwind tiles' stores, acquired by lanes 0-6, for every lane
            // stage the tile: traveltimes of the tile and its upwind layer (halo index
            // origin tz..), slowness of the halo indices one below the tile's lowest to its
            // highest (origin gz - 1..)
            const int gz = tile_lo(rz, tc * kFsmTZ, kFsmTZ), gx = tile_lo(rx, ta * kFsmTX, kFsmTX),
                      gy = tile_lo(ry, tb * kFsmTY, kFsmTY);
            const int tz = rz.di > 0 ? gz - 1 : gz, tx = rx.di > 0 ? gx - 1 : gx, ty = ry.di > 0 ? gy - 1 : gy;
            const float *T = p.T + sh.t_off;
            ShotGrid g{&sh, p.T + sh.t_off, 0, nxx, nyy, nzz};
            // The slowness goes by cp.async, so all its copies are in flight at once and hold
            // no registers; the traveltime loop is unrolled so that several loads are in
            // flight before their shared-memory stores wait on them.  Staged node m = lane +
            // 32 it is (ci, cj, ck), advanced by 32 nodes per iteration without divisions.
            static_assert(32 / kHZ + 1 <= kHX, "one carry into cj and one into ck per step");
            int ci = lane % kHZ, cj = (lane / kHZ) % kHX, ck = lane / (kHZ * kHX);
#pragma unroll kStageUnroll
            for (int m = lane; m < kHZ * kHX * kHY; m += 32) {
                const int i = tz + ci, j = tx + cj, k = ty + ck;
                cp_async4(Ss + ci + kPZ * (cj + kPX * ck), sptr(p, g, gz - 1 + ci, gx - 1 + cj, gy - 1 + ck));
                Ts[ci + kPZ * (cj + kPX * ck)] = (i >= 0 && i < nzz && j >= 0 && j < nxx && k >= 0 && k < nyy)
                                                     ? __ldcg(T + i + (long long)j * nzz + (long long)k * nxx * nzz)
                                                     : 1e6f;
                ci += 32 % kHZ;
                cj += 32 / kHZ;
                if (ci >= kHZ) { ci -= kHZ; ++cj; }
                if (cj >= kHX) { cj -= kHX; ++ck; }
            }
            cp_async_wait_all();
            __syncwarp();
            // the tile's first node (c, a, b) = (0, 0, 0) in the traveltime tile, the offset of
            // a node's cell (i-1, j-1, k-1) in the slowness tile from it, and the nodes left on
            // each axis; the plane loop is specialised on the sweep's octant
            const int i0 = rz.i0 + rz.di * tc * kFsmTZ, j0 = rx.i0 + rx.di * ta * kFsmTX,
                      k0 = ry.i0 + ry.di * tb * kFsmTY;
            const int t0 = (i0 - tz) + kPZ * ((j0 - tx) + kPX * (k0 - ty));
            const int dts = (gz - tz) + kPZ * ((gx - tx) + kPX * (gy - ty));
            const int nc = rz.L - tc * kFsmTZ, na = rx.L - ta * kFsmTX, nb = ry.L - tb * kFsmTY;
            switch (q & 7) {
            case 0: relax_tile<0, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 1: relax_tile<1, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 2: relax_tile<2, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 3: relax_tile<3, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 4: relax_tile<4, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 5: relax_tile<5, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            case 6: relax_tile<6, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            default: relax_tile<7, kBranchFree>(p, Ts, Ss, plane, pstart, lane, t0, dts, nc, na, nb); break;
            }
            // the tile's nodes back to global memory, then its flag
            float *Tw = p.T + sh.t_off;
            for (int m = lane; m < kTileN; m += 32) {
                const int c = m % kFsmTZ, a = (m / kFsmTZ) % kFsmTX, b = m / (kFsmTZ * kFsmTX);
                const int lc = tc * kFsmTZ + c, la = ta * kFsmTX + a, lb = tb * kFsmTY + b;
                if (lc < rz.L && la < rx.L && lb < ry.L) {
                    const int i = rz.i0 + rz.di * lc, j = rx.i0 + rx.di * la, k = ry.i0 + ry.di * lb;
                    __stcg(Tw + i + (long long)j * nzz + (long long)k * nxx * nzz,
                           Ts[(i - tz) + kPZ * ((j - tx) + kPX * (k - ty))]);
                }
            }
            __threadfence();
            __syncwarp();
            if (lane == 0) {
                st_release(flags + tc + fa * (ta + fb * tb), (unsigned)(q + 1));
                if (!p.sweep_barrier) atomicAdd(p.shot_done + (size_t)si * 16 + q, 1u);
            }
        }
        // one shot: nothing to overlap a sweep's drain with, and a barrier is cheaper than
        // the per-tile counts
        if (p.sweep_barrier && q < 15 && !group_barrier(p.bar, gridDim.x, p.err, p.spin_limit)) return;
    }
    if (!group_barrier(p.bar, gridDim.x, p.err, p.spin_limit)) return;

    // reduce_model (accurate_FSM.cpp:62-72) into the brick-major pool of the shot
    for (int m = 0; m < p.nshots; m++) {
        const FsmShot &s = p.shots[m];
        const ShotDesc &d = p.desc[m];
        const long long n = (long long)d.nbx * d.nby * d.nbz * kBrickNodes;
        const int nxx = s.wnx + 2;
        for (long long e = gthread; e < n; e += nthreads) {
            const long long b = e / kBrickNodes;
            const int node = (int)(e % kBrickNodes);
            const int bz = (int)(b % d.nbz);
            const long long tq = b / d.nbz;
            const int bx = (int)(tq % d.nbx), by = (int)(tq / d.nbx);
            const int z = bz * 4 + (node & 3), x = bx * 4 + ((node >> 2) & 3), y = by * 4 + (node >> 4);
            float v = kInf;
            if (z < p.nz && x < s.wnx && y < s.wny)
                v = __ldcg(p.T + s.t_off + (z + 1) + (long long)(x + 1) * nzz + (long long)(y + 1) * nxx * nzz);
            p.Tb[d.t_off + e] = v;
        }
    }
}

cudaError_t fsm_solve_tiled(const FsmLaunch &p, int *grid_out, cudaStream_t st)
{
    constexpr int threads = 256;
    const size_t smem = (size_t)(threads / 32) * 2 * kHN * sizeof(float) + kTileN * sizeof(unsigned short) +
                        (kNPlanes + 1) * sizeof(int);
    // one shot: the branch-free operator (bound by the wavefront's waits); batches: the
    // branching one (config 1 11.4 vs 11.9 ms; config-2 batch 52.3 vs 48.6 ms)
    const void *fn = p.nshots == 1 ? (const void *)k_fsm_tiled<true> : (const void *)k_fsm_tiled<false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 0, per_sm = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = nsm * per_sm;
    if (grid_out) *grid_out = grid;
    FsmLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st);
}

}  // namespace tomo
