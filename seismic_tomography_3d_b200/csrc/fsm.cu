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
// bounded barrier between planes.
#include "common.cuh"
#include "fsm.cuh"

namespace tomo {

namespace {

struct Range {
    int i0, di, L;
};

// Sweep q (0..7 source-anchored, 8..15 full) of axis with sign s (+1 ascending), halo extent
// n and source index sid (accurate_FSM.cpp:267-511).
__device__ __forceinline__ Range sweep_range(int q, int s, int n, int sid)
{
    Range r;
    if (q < 8) {
        if (s > 0) {
            r.i0 = max(1, sid);
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
__device__ __forceinline__ float sget(const FsmLaunch &p, const ShotGrid &g, int i, int j, int k)
{
    const int z = min(max(i - 1, 0), p.nz - 1);
    const int x = g.s->wx0 + min(max(j - 1, 0), g.s->wnx - 1);
    const int y = g.s->wy0 + min(max(k - 1, 0), g.s->wny - 1);
    return __ldg(p.slow + z + (long long)x * p.nz + (long long)y * p.nx * p.nz);
}

// Accurate_FSM::inner_sweep (accurate_FSM.cpp:159-265), same operations in the same order.
__device__ float ngb_update(const FsmLaunch &p, const ShotGrid &g, int i, int j, int k, int sgntz, int sgntx, int sgnty)
{
    const int nxx = g.nxx, nyy = g.nyy, nzz = g.nzz;
    const long long sx = nzz, sy = (long long)nxx * nzz;
    const int sgnvz = sgntz == 1, sgnvx = sgntx == 1, sgnvy = sgnty == 1;
    const int i1 = i - sgnvz, j1 = j - sgnvx, k1 = k - sgnvy;
    const float tv = tget(g, (i - sgntz) + j * sx + k * sy);
    const float te = tget(g, i + (j - sgntx) * sx + k * sy);
    const float tn = tget(g, i + j * sx + (k - sgnty) * sy);
    const float tev = tget(g, (i - sgntz) + (j - sgntx) * sx + k * sy);
    const float ten = tget(g, i + (j - sgntx) * sx + (k - sgnty) * sy);
    const float tnv = tget(g, (i - sgntz) + j * sx + (k - sgnty) * sy);
    const float tnve = tget(g, (i - sgntz) + (j - sgntx) * sx + (k - sgnty) * sy);
    const long long ijk = i + j * sx + k * sy;
    const int jm = max(j - 1, 1), jp = min(j, nxx - 1), km = max(k - 1, 1), kp = min(k, nyy - 1);
    const int im = max(i - 1, 1), ip = min(i, nzz - 1);
    const float dz2i = p.dz2i, dx2i = p.dx2i, dy2i = p.dy2i;

    const float t1D1 = tv + p.dz * smin(sget(p, g, i1, jm, km),
                                        smin(sget(p, g, i1, jm, kp), smin(sget(p, g, i1, jp, km), sget(p, g, i1, jp, kp))));
    const float t1D2 = te + p.dx * smin(sget(p, g, im, j1, km),
                                        smin(sget(p, g, ip, j1, km), smin(sget(p, g, im, j1, kp), sget(p, g, ip, j1, kp))));
    const float t1D3 = tn + p.dy * smin(sget(p, g, im, jm, k1),
                                        smin(sget(p, g, im, jp, k1), smin(sget(p, g, ip, jm, k1), sget(p, g, ip, jp, k1))));
    const float t1D = smin(t1D1, smin(t1D2, t1D3));

    float t2D1 = 1e6f, t2D2 = 1e6f, t2D3 = 1e6f, ta, tb, tc, Sref;
    Sref = smin(sget(p, g, i1, j1, km), sget(p, g, i1, j1, kp));
    if ((tv < te + p.dx * Sref) && (te < tv + p.dz * Sref)) {
        ta = tev + te - tv;
        tb = tev - te + tv;
        t2D1 = ((tb * dz2i + ta * dx2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dx2i) - dz2i * dx2i * (ta - tb) * (ta - tb))) /
               (dz2i + dx2i);
    }
    Sref = smin(sget(p, g, i1, jm, k1), sget(p, g, i1, jp, k1));
    if ((tv < tn + p.dy * Sref) && (tn < tv + p.dz * Sref)) {
        ta = tv - tn + tnv;
        tb = tn - tv + tnv;
        t2D2 = ((ta * dz2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dy2i) - dz2i * dy2i * (ta - tb) * (ta - tb))) /
               (dz2i + dy2i);
    }
    Sref = smin(sget(p, g, im, j1, k1), sget(p, g, ip, j1, k1));
    if ((te < tn + p.dy * Sref) && (tn < te + p.dx * Sref)) {
        ta = te - tn + ten;
        tb = tn - te + ten;
        t2D3 = ((ta * dx2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dx2i + dy2i) - dx2i * dy2i * (ta - tb) * (ta - tb))) /
               (dx2i + dy2i);
    }
    const float t2D = smin(t2D1, smin(t2D2, t2D3));

    float t3D = 1e6f;
    Sref = sget(p, g, i1, j1, k1);
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
    return smin(__ldcg(g.T + ijk), smin(t1D, smin(t2D, t3D)));
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
            const Range rz = sweep_range(q, sgz, nzz, s.sidz), rx = sweep_range(q, sgx, s.wnx + 2, s.sidx),
                        ry = sweep_range(q, sgy, s.wny + 2, s.sidy);
            W = max(W, rz.L + rx.L + ry.L - 2);
        }
        for (int w = 0; w < W; w++) {
            // one warp per (shot, c) row of the plane; lanes stride over a
            for (long long row = gwarp; row < (long long)ns * nzz; row += nwarps) {
                const int m = (int)(row / nzz), c = (int)(row % nzz);
                const FsmShot &s = p.shots[grp + m * G];
                const Range rz = sweep_range(q, sgz, nzz, s.sidz), rx = sweep_range(q, sgx, s.wnx + 2, s.sidx),
                            ry = sweep_range(q, sgy, s.wny + 2, s.sidy);
                if (c >= rz.L) continue;
                const int t = w - c;
                const int a_lo = max(0, t - (ry.L - 1)), a_hi = min(rx.L - 1, t);
                if (a_lo > a_hi) continue;
                ShotGrid g{&s, p.T + s.t_off, (long long)nzz * (s.wnx + 2) * (s.wny + 2), s.wnx + 2, s.wny + 2, nzz};
                const int i = rz.i0 + rz.di * c;
                for (int a = a_lo + lane; a <= a_hi; a += 32) {
                    const int j = rx.i0 + rx.di * a, k = ry.i0 + ry.di * (t - a);
                    const float v = ngb_update(p, g, i, j, k, sgz, sgx, sgy);
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

}  // namespace tomo
