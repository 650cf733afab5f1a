// Batched persistent fast-iterative eikonal solver for sm_100a.
//
// Replaces Block_FIM (src/eikonal/block_FIM/block_FIM.cpp, cuda_kernel.cu) with a design
// of its own:
//  * All shots of a batch are solved by ONE cooperative launch.  Work items are
//    (shot, 4x4x4 brick) pairs; one warp owns one brick, so the in-brick relaxation is
//    synchronised with __syncwarp/__any_sync only (warp-vote convergence).
//  * The active list lives on the device (3 rotating lists + a per-brick "queued for
//    round" word updated with atomicMax), so there are no host round trips, no per-shot
//    allocations and no re-bricking on the host.
//  * A brick re-queues a neighbour only when a value on the shared face dropped, and
//    itself when its in-brick iteration cap was hit.  Updates are monotone (min), so this
//    chaotic relaxation converges to the same fixed point as Block_FIM's schedule.
//  * Slowness is read from one brick-major copy of the model shared by all shots: whole
//    bricks for a brick-aligned window, node by node (edge replicated into the padding)
//    for any other window.
//  * Optionally (time band), pushes carry the pushing brick's new time, and a brick far
//    ahead of its shot's front waits on a parking list: rounds then follow traveltime
//    rather than brick-graph distance, which removes the re-activation cascades of smooth
//    v(z) models.
#include "common.cuh"
#include "fim.cuh"

namespace tomo {

// -------------------------------------------------------------------------------------
// Local update.  First-order Godunov upwind solution of |grad T| = s on a cubic grid of
// spacing h given the smaller neighbour of each axis (a, b, c): the largest root that is
// causal (exceeds every neighbour it uses), trying 1, 2 then 3 neighbours in ascending
// order -- the Jeong & Whitaker (2008) update of get_time_eikonal
// (src/eikonal/block_FIM/cuda_kernel.cu:217-248), written in symmetric form.
// -------------------------------------------------------------------------------------
// Square root to ~1 ulp (sqrt.approx): the candidates it feeds are compared and min-ed,
// never accumulated, so the rounding stays at the 1e-7 level of the FP32 fixed point.
__device__ __forceinline__ float sqrt_fast(float v)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}

template <bool kFastSqrt>
__device__ __forceinline__ float sqrt_sel(float v)
{
    return kFastSqrt ? sqrt_fast(v) : sqrtf(v);
}

// Loop-invariant part of the local update of a node: h*s and the two discriminant terms.
struct NodeConst {
    float hs, q2c, q3c;  // h s, 2 (h s)^2, 3 (h s)^2
};

__device__ __forceinline__ NodeConst node_const(float h, float s)
{
    NodeConst k;
    k.hs = h * s;
    k.q2c = 2.0f * k.hs * k.hs;
    k.q3c = 3.0f * k.hs * k.hs;
    return k;
}

// Branch-free: all three candidates are computed and the causal one selected, so the lanes
// of a warp (which need different candidates) never diverge.  A candidate whose root is
// imaginary is NaN and fails every comparison, exactly as the sequential tests skip it.
// kGate: return kInf when every neighbour is unreached.  Callers that take the minimum with
// the node's own value (at most kInf) can skip it: with all neighbours at kInf every
// candidate is at least kInf.
template <bool kFastSqrt, bool kGate = true>
__device__ __forceinline__ float godunov_jw(float a, float b, float c, const NodeConst &k)
{
    const float lo = fminf(a, b), hi = fmaxf(a, b);
    const float u0 = fminf(lo, c);
    const float mid = fmaxf(lo, c);
    const float u1 = fminf(mid, hi), u2 = fmaxf(mid, hi);
    const float t1 = u0 + k.hs;
    const float d01 = u1 - u0;
    const float t2 = 0.5f * ((u0 + u1) + sqrt_sel<kFastSqrt>(k.q2c - d01 * d01));
    const float sum = u0 + u1 + u2;
    const float d12 = u2 - u1, d02 = u2 - u0;
    const float t3 = (sum + sqrt_sel<kFastSqrt>(k.q3c - (d01 * d01 + d12 * d12 + d02 * d02))) * (1.0f / 3.0f);
    // Sequential rule: t1 unless it exceeds u1; then t2 unless it exceeds u2; then t3 if
    // causal.  t2's causality needs no test: t1 > u1 means u1 - u0 < hs, so the
    // discriminant exceeds (hs)^2 and t2 > u1.  t3's test stays: when t2 only just exceeds
    // u2 the discriminant of t3 is near zero and may round negative (NaN), and t2 is then
    // the right value to within rounding.
    const float t = (t1 > u1) ? ((t2 > u2 && t3 > u2) ? t3 : t2) : t1;
    return (!kGate || u0 < kInf) ? t : kInf;
}

// Tile of one warp: (4+2)^3 nodes, the brick plus a one-node face halo, z fastest.  The x
// and y strides are padded (12 and 72 words instead of 6 and 36) so that every shared-memory
// access of the relaxation -- a phase's six neighbour reads and its store, over the 32 lanes
// -- falls in 32 distinct banks, and so do the face tests; of the tile fill, two of the
// three halo stores are 2-way conflicted.
constexpr int kTileX = 12;
constexpr int kTileY = 72;
constexpr int kTileNodes = kTileY * (kBrick + 2);

__device__ __forceinline__ int tile_idx(int z, int x, int y)
{
    return (z + 1) + kTileX * (x + 1) + kTileY * (y + 1);
}

__device__ __forceinline__ float brick_T(const float *T, const ShotDesc &d, int x, int y, int z)
{
    const long long b = (z >> 2) + (long long)d.nbz * ((x >> 2) + (long long)d.nbx * (y >> 2));
    return __ldcg(T + d.t_off + b * kBrickNodes + (z & 3) + 4 * (x & 3) + 16 * (y & 3));
}

// Slowness of node `node` (z + 4x + 16y) of the shot's local brick (bz, bx, by), from the
// shared brick-major model.  A brick-aligned window's brick is a model brick.  Any other
// window maps the node into the model, its padding nodes (x >= wnx, y >= wny) taking the
// window's last node: the cropped model padded by edge replication, as the model's own
// padding is (k_brick_model).
__device__ __forceinline__ const float *model_brick_S(const float *S, int gbx, int gbz, const ShotDesc &d, int bz,
                                                      int bx, int by)
{
    return S + (bz + (long long)gbz * ((bx + (d.wx0 >> 2)) + (long long)gbx * (by + (d.wy0 >> 2)))) * kBrickNodes;
}

__device__ __forceinline__ float gather_S(const float *S, int gbx, int gbz, const ShotDesc &d, int bz, int bx, int by,
                                          int node)
{
    const int z = 4 * bz + (node & 3);
    const int x = min(4 * bx + ((node >> 2) & 3), d.wnx - 1) + d.wx0;
    const int y = min(4 * by + (node >> 4), d.wny - 1) + d.wy0;
    return __ldg(S + ((z >> 2) + (long long)gbz * ((x >> 2) + (long long)gbx * (y >> 2))) * kBrickNodes + (z & 3) +
                 4 * (x & 3) + 16 * (y & 3));
}

__device__ __forceinline__ float node_S(const float *S, int gbx, int gbz, const ShotDesc &d, int bz, int bx, int by,
                                        int node)
{
    if (!d.s_gather) return __ldg(model_brick_S(S, gbx, gbz, d, bz, bx, by) + node);
    return gather_S(S, gbx, gbz, d, bz, bx, by, node);
}

// Slowness of a relaxation lane's two nodes (node, node + 16) in a gathered window.
__device__ __forceinline__ void gather_S2(const float *S, int gbx, int gbz, const ShotDesc &d, int bz, int bx, int by,
                                          int node, float &s0, float &s1)
{
    s0 = gather_S(S, gbx, gbz, d, bz, bx, by, node);
    s1 = gather_S(S, gbx, gbz, d, bz, bx, by, node + 16);
}

// Receiver sampling (Block_FIM::write_first_arrival, block_FIM.cpp:228-262): trilinear
// from the floor node of the window-cropped field, with the reference's flattened index
// arithmetic (an offset past a column wraps into the next; past the end: 0).  Grid-stride
// over (shot, receiver); receivers outside a shot's window get kInf.
__device__ void sample_receivers(const float *T, const ShotDesc *shots, int nshots, const float *rx,
                                 const float *ry, const float *rz, int nrec, float dx, float dy, float dz,
                                 int nz_, float *t_recv)
{
    const long long total = (long long)nshots * nrec;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e / nrec), r = (int)(e % nrec);
        const ShotDesc &d = shots[s];
        const float x = fsub(rx[r], fmul((float)d.wx0, dx));
        const float y = fsub(ry[r], fmul((float)d.wy0, dy));
        const float z = rz[r];
        if (x < 0.0f || y < 0.0f || x > fmul((float)(d.wnx - 1), dx) || y > fmul((float)(d.wny - 1), dy)) {
            t_recv[e] = kInf;
            continue;
        }
        const float fx = floorf(fdiv(x, dx)), fy = floorf(fdiv(y, dy)), fz = floorf(fdiv(z, dz));
        const float x0 = fmul(fx, dx), y0 = fmul(fy, dy), z0 = fmul(fz, dz);
        const float x1 = fadd(fmul(fx, dx), dx), y1 = fadd(fmul(fy, dy), dy), z1 = fadd(fmul(fz, dz), dz);
        const long long nz = nz_, wnx = d.wnx, n = nz * wnx * d.wny;
        const long long id = (long long)(int)fdiv(z, dz) + (long long)(int)fdiv(x, dx) * nz +
                             (long long)(int)fdiv(y, dy) * wnx * nz;
        const long long offs[8] = {0, 1, nz, 1 + nz, wnx * nz, 1 + wnx * nz, nz + wnx * nz, 1 + nz + wnx * nz};
        float c[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const long long f = id + offs[q];
            if (f >= 0 && f < n) {
                const int zz = (int)(f % nz);
                const long long rest = f / nz;
                const int xx = (int)(rest % wnx), yy = (int)(rest / wnx);
                c[q] = brick_T(T, d, xx, yy, zz);
            } else {
                c[q] = 0.0f;
            }
        }
        t_recv[e] = trilinear_ref(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], x0, x1, y0, y1, z0, z1, x, y, z);
    }
}

struct WarpStats {
    unsigned long long act, inner, idle;  // idle: activations that lowered no node
    unsigned long long deferred;          // items put off to a later round (time band)
};

constexpr unsigned kNoKey = 0xffffffffu;

// Data of one work item as loaded from global memory (the face halo goes straight to the
// warp's tile).
struct BrickLoad {
    unsigned s, b;
    int bz, bx, by;    // brick coordinates in the shot's window
    float s0, s1;      // slowness of the lane's two nodes
    float i0, i1;      // traveltimes of the lane's two nodes at load time
};

// First of the lane's two nodes (node = z + 4x + 16y); the second is 16 above it (y + 1).
__device__ __forceinline__ int lane_node(int lane) { return (lane & 15) + 32 * (lane >> 4); }

__device__ __forceinline__ void brick_coords(const ShotDesc &d, unsigned b, int &bz, int &bx, int &by)
{
    const unsigned tq = (unsigned)(((unsigned long long)b * d.divz_m) >> d.divz_sh);  // b / nbz
    bz = (int)(b - tq * (unsigned)d.nbz);
    const unsigned q2 = (unsigned)(((unsigned long long)tq * d.divx_m) >> d.divx_sh);  // tq / nbx
    bx = (int)(tq - q2 * (unsigned)d.nbx);
    by = (int)q2;
}

// Face halo slot q (0..2) of a lane: slot q covers the two faces of axis q (z, x, y); lanes
// 0-15 the lower face, 16-31 the upper, one face node each.  Returns the neighbour brick
// (-1 at the grid edge); node = its node index, ti = the tile index of the halo cell.
__device__ __forceinline__ long long halo_slot(const ShotDesc &d, unsigned b, int bz, int bx, int by, int lane, int q,
                                               int &node, int &ti)
{
    const bool lower = lane < 16;
    const int j = lane & 15, u = j & 3, v = j >> 2;
    const int e = lower ? -1 : kBrick;      // halo plane in tile coordinates
    long long step;
    bool ok;
    if (q == 0) {
        node = (lower ? 3 : 0) + 4 * u + 16 * v;
        ti = tile_idx(e, u, v);
        ok = lower ? bz > 0 : bz < d.nbz - 1;
        step = 1;
    } else if (q == 1) {
        node = u + (lower ? 12 : 0) + 16 * v;
        ti = tile_idx(u, e, v);
        ok = lower ? bx > 0 : bx < d.nbx - 1;
        step = d.nbz;
    } else {
        node = u + 4 * v + (lower ? 48 : 0);
        ti = tile_idx(u, v, e);
        ok = lower ? by > 0 : by < d.nby - 1;
        step = (long long)d.nbz * d.nbx;
    }
    return ok ? (long long)b + (lower ? -step : step) : -1;
}

// Loads work item `item` into L and into the warp's tile: the lane's two nodes and its three
// face-halo cells.  The caller synchronises the warp before the tile is read.  kGather: some
// shot of the batch gathers its slowness by node (a separate instance, so that batches of
// brick-aligned windows keep the plain load path).
template <bool kGather>
__device__ __forceinline__ void load_brick(const FimLaunch &p, unsigned item, BrickLoad &L, float *tile)
{
    const int lane = threadIdx.x & 31;
    L.s = item >> p.local_bits;
    L.b = item & ((1u << p.local_bits) - 1u);
    const ShotDesc &d = p.shots[L.s];
    brick_coords(d, L.b, L.bz, L.bx, L.by);
    const float *Tb = p.T + d.t_off + (long long)L.b * kBrickNodes;
    // own nodes: (z, x, y) and (z, x, y + 1) with z = lane & 3, x = (lane >> 2) & 3,
    // y = 2 (lane >> 4)
    const int n0 = lane_node(lane);
    if (!kGather || !d.s_gather) {
        const float *Sb = model_brick_S(p.S, p.gbx, p.gbz, d, L.bz, L.bx, L.by);
        L.s0 = __ldg(Sb + n0);
        L.s1 = __ldg(Sb + n0 + 16);
    } else {
        gather_S2(p.S, p.gbx, p.gbz, d, L.bz, L.bx, L.by, n0, L.s0, L.s1);
    }
    L.i0 = __ldcg(Tb + n0);
    L.i1 = __ldcg(Tb + n0 + 16);
    // Missing neighbours (grid edge) are INF; the reference's "halo = self" at the edge
    // cannot lower a node either.  All loads go out before the first shared-memory store.
    float hv[3];
    int ht[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        int node;
        const long long nb = halo_slot(d, L.b, L.bz, L.bx, L.by, lane, q, node, ht[q]);
        hv[q] = nb >= 0 ? __ldcg(p.T + d.t_off + nb * kBrickNodes + node) : kInf;
    }
    const int ti0 = tile_idx(lane & 3, (lane >> 2) & 3, 2 * (lane >> 4));
    tile[ti0] = L.i0;
    tile[ti0 + kTileY] = L.i1;
#pragma unroll
    for (int q = 0; q < 3; q++) tile[ht[q]] = hv[q];
}

// ---------------------------------------------------------------------------------------
// Asynchronous schedule (no rounds).  One ring of work items (capacity = bricks of the
// batch) and one state word per (shot, brick): 0 idle, 1 queued (exactly one ring entry),
// 2 being relaxed by one warp, 3 being relaxed and re-queued meanwhile ("dirty").  A brick
// therefore never has two owners, and a re-queue that arrives while it is being relaxed
// is kept as the dirty state and honoured by the owner.  `pending` counts queued + owned
// bricks; it is raised before a push and lowered after an owner's pushes, so it reaches
// zero only when the work is done.  Every wait is bounded (error flag, then return).
// ---------------------------------------------------------------------------------------
constexpr unsigned kEmpty = 0xffffffffu;
constexpr unsigned kIdle = 0u, kQueued = 1u, kOwned = 2u, kDirty = 3u;

__device__ __forceinline__ unsigned *ring_of(const FimLaunch &p) { return p.lists; }
// The ring spans the whole list buffer (3 x the batch's bricks).
__device__ __forceinline__ unsigned ring_cap(const FimLaunch &p) { return 3u * p.list_cap; }

// Pushes the items of the lanes with `push` (warp-aggregated): pending first, then the
// ring slots.  The caller fenced its traveltime stores before.
__device__ __forceinline__ void ring_push(const FimLaunch &p, bool push, unsigned item)
{
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kFull, push);
    if (!m) return;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) {
        atomicAdd(p.ctrl + kCnt1, (unsigned)__popc(m));
        base = atomicAdd(p.ctrl + kCnt0, (unsigned)__popc(m));
    }
    base = __shfl_sync(kFull, base, leader);
    if (push) {
        // Slots are handed out in tail order but written later: a slot may still hold the
        // item of the previous lap (its reader not yet there), so claim it only when empty.
        const unsigned slot = (base + __popc(m & ((1u << lane) - 1u))) % ring_cap(p);
        unsigned long long spins = 0;
        while (atomicCAS(ring_of(p) + slot, kEmpty, item) != kEmpty) {
            if (++spins > p.spin_limit) {
                atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevBarrierTimeout);
                break;
            }
            __nanosleep(32);
        }
    }
}

// Lanes 0-5: neighbour tgt to queue (want); lane 6: this brick, `more` = its in-brick
// iteration cap was hit.  Ends this warp's ownership of brick b.
__device__ __forceinline__ void queue_async(const FimLaunch &p, const ShotDesc &d, unsigned s, unsigned b, bool want,
                                            long long tgt, bool self_lane)
{
    const int lane = threadIdx.x & 31;
    __threadfence();  // the brick's traveltimes are visible before anyone is queued
    bool push = false;
    unsigned item = 0;
    if (want && lane < 6) {
        unsigned *st = p.qflag + d.qbase + (unsigned long long)tgt;
        bool settled = false;
        for (int tries = 0; tries < 256 && !settled; tries++) {
            const unsigned old = atomicCAS(st, kIdle, kQueued);
            if (old == kIdle) {
                push = settled = true;
            } else if (old == kQueued || old == kDirty) {
                settled = true;
            } else {  // owned: mark dirty unless the owner let go meanwhile (then retry)
                const unsigned o2 = atomicCAS(st, kOwned, kDirty);
                settled = (o2 == kOwned || o2 == kDirty || o2 == kQueued);
            }
        }
        if (!settled) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevCapacity);
        item = (s << p.local_bits) | (unsigned)tgt;
    }
    // this brick: re-queue when its cap was hit or it turned dirty, else release it
    if (self_lane && lane == 6) {
        unsigned *st = p.qflag + d.qbase + b;
        if (want) {  // `want` on lane 6 = in-brick cap hit
            atomicExch(st, kQueued);
            push = true;
        } else {
            const unsigned old = atomicCAS(st, kOwned, kIdle);
            if (old == kDirty) {
                atomicExch(st, kQueued);
                push = true;
            }
        }
        item = (s << p.local_bits) | b;
    }
    ring_push(p, push, item);
    __syncwarp();
    if (lane == 0) atomicSub(p.ctrl + kCnt1, 1u);  // this ownership ends
}

// Per-warp buffer of queue candidates (items for the next round), in shared memory.  An
// activation adds at most 7, and the buffer is flushed once it holds more than
// kPushCap - 7, so it never overflows.
constexpr unsigned kPushCap = 32;

// Queues the buffered candidates for round+1: one lane per candidate marks its brick
// "queued for round+1" (atomicMax on the brick's flag; only the first marker of the round
// appends it), and the survivors are appended to the next list with one atomic.
template <bool kBand>
__device__ __forceinline__ void flush_pushes(const FimLaunch &p, unsigned *pbuf, const unsigned *pkey,
                                             unsigned &pcnt, unsigned round)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();  // the buffer as the lanes wrote it
    const unsigned tag = round + 2u;  // "queued for round+1", offset by one so 0 = never
    bool want = false;
    unsigned item = 0;
    if ((unsigned)lane < pcnt) {
        item = pbuf[lane];
        const unsigned s = item >> p.local_bits, b = item & ((1u << p.local_bits) - 1u);
        const unsigned long long qi = p.shots[s].qbase + b;
        if (kBand) {
            const unsigned k = pkey[lane];
            if (k != kNoKey) atomicMin(p.keys + qi, k);
        }
        const unsigned old = atomicMax(p.qflag + qi, tag);
        want = old < tag;
    }
    const unsigned wm = __ballot_sync(kFull, want);
    if (wm) {
        const int leader = __ffs(wm) - 1;
        const unsigned nxt = (round + 1u) % 3u;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(p.ctrl + kCnt0 + nxt, (unsigned)__popc(wm));
        base = __shfl_sync(kFull, base, leader);
        if (want) p.lists[(size_t)nxt * p.list_cap + base + __popc(wm & ((1u << lane) - 1u))] = item;
    }
    pcnt = 0;
}

// Time band: a brick put off in round r waits on that round's parking list and is merged
// back at the start of round r + park_rounds (or earlier, when the round's list is empty),
// instead of every round.  park_rounds + 2 lists rotate: the list merged at the start of
// round r is next filled in round r + 2, and block 0 zeroes its count at the start of
// round r + 1, between the two barriers -- the same rotation as the work lists.  Each
// warp buffers kParkCap items in shared memory and appends them with one atomic.
constexpr unsigned kParkCap = 8;

__device__ __forceinline__ unsigned park_slot(const FimLaunch &p, unsigned round)
{
    return round % (unsigned)(p.park_rounds + 2);
}

__device__ __forceinline__ void flush_parks(const FimLaunch &p, const unsigned *kbuf, unsigned &kcnt, unsigned round)
{
    const int lane = threadIdx.x & 31;
    const unsigned j = park_slot(p, round);
    __syncwarp();  // the buffer as lane 0 wrote it
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(p.park_cnt + j, kcnt);
    base = __shfl_sync(kFull, base, 0);
    if ((unsigned)lane < kcnt) p.park[(size_t)j * p.list_cap + base + lane] = kbuf[lane];
    kcnt = 0;
}

// Appends parking list j's items that still hold a key (new information not yet relaxed)
// to the next round's list, unless a push already queued them for it; grid-strided, one
// item per lane.
__device__ __noinline__ void merge_parks(const FimLaunch &p, unsigned j, unsigned np, unsigned round)
{
    const int lane = threadIdx.x & 31;
    const unsigned nxt = (round + 1u) % 3u;
    const unsigned tag = round + 2u;  // "queued for round+1"
    const unsigned *park = p.park + (size_t)j * p.list_cap;
    const unsigned gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (unsigned base = gw * 32u; base < np; base += nw * 32u) {
        const unsigned idx = base + (unsigned)lane;
        bool want = false;
        unsigned item = 0;
        if (idx < np) {
            item = __ldcg(park + idx);
            const unsigned s = item >> p.local_bits;
            const unsigned long long qi = p.shots[s].qbase + (item & ((1u << p.local_bits) - 1u));
            if (__ldcg(p.keys + qi) != kNoKey) want = atomicMax(p.qflag + qi, tag) < tag;
        }
        const unsigned wm = __ballot_sync(kFull, want);
        if (wm) {
            const int leader = __ffs(wm) - 1;
            unsigned b0 = 0;
            if (lane == leader) b0 = atomicAdd(p.ctrl + kCnt0 + nxt, (unsigned)__popc(wm));
            b0 = __shfl_sync(kFull, b0, leader);
            if (want) p.lists[(size_t)nxt * p.list_cap + b0 + __popc(wm & ((1u << lane) - 1u))] = item;
        }
    }
}

// One activation of one (already loaded) brick by one warp.
template <bool kFastSqrt, bool kAsync, bool kBand = false>
__device__ __forceinline__ void relax_brick(const FimLaunch &p, const BrickLoad &L, unsigned round, float *tile,
                                            WarpStats &ws, unsigned *pbuf, unsigned *pkey, unsigned &pcnt,
                                            unsigned *cursor, unsigned &next)
{
    const int lane = threadIdx.x & 31;
    const unsigned s = L.s, b = L.b;
    const ShotDesc &d = p.shots[s];
    const int bz = L.bz, bx = L.bx, by = L.by;
    const int nbz = d.nbz, nbx = d.nbx, nby = d.nby;
    float *Tb = p.T + d.t_off + (long long)b * kBrickNodes;

    const int z0 = lane & 3, x0 = (lane >> 2) & 3, y0 = 2 * (lane >> 4);
    const int ti0 = tile_idx(z0, x0, y0);
    const int ti1 = ti0 + kTileY;  // y + 1
    const float i0 = L.i0, i1 = L.i1;
    __syncwarp();  // the tile as load_brick wrote it

    // Red-black Gauss-Seidel.  A lane's two nodes are y-adjacent, so one is red (z + x + y
    // even) and the other black: phase A relaxes the lane's red node from black neighbours,
    // phase B its black node from the new red ones.  Every neighbour of a node has the other
    // colour, so each phase reads only what the other phase writes, and a dependency chain
    // -- alternating in colour -- advances two nodes per iteration where Jacobi advances one.
    // Of a phase's two y-neighbours one is the lane's other node (a register), the other is
    // in the tile at offset yA (phase A) or -yA (phase B).
    const bool red0 = ((z0 + x0) & 1) == 0;
    const int tA = red0 ? ti0 : ti1, tB = red0 ? ti1 : ti0;
    const int yA = red0 ? -kTileY : kTileY;
    float cA = red0 ? i0 : i1, cB = red0 ? i1 : i0;
    const NodeConst kA = node_const(p.h, red0 ? L.s0 : L.s1), kB = node_const(p.h, red0 ? L.s1 : L.s0);
    // The relaxation has converged as soon as one phase changes nothing, once every black
    // node has been relaxed at least once: the other colour then reads the same inputs as in
    // its previous phase and would reproduce its values.
    bool more = true;
    int it = 0;
    for (; it < p.max_inner; ++it) {
        const float aA = fminf(tile[tA - kTileX], tile[tA + kTileX]);
        const float gA = fminf(tile[tA - 1], tile[tA + 1]);
        const float bA = fminf(tile[tA + yA], cB);
        const float nA = fminf(cA, godunov_jw<kFastSqrt, false>(aA, bA, gA, kA));
        tile[tA] = nA;
        const bool chA = nA < cA - p.inner_tol;
        cA = nA;
        __syncwarp();
        if (it > 0 && !__any_sync(kFull, chA)) {
            more = false;
            ++it;
            break;
        }
        const float aB = fminf(tile[tB - kTileX], tile[tB + kTileX]);
        const float gB = fminf(tile[tB - 1], tile[tB + 1]);
        const float bB = fminf(tile[tB - yA], nA);
        const float nB = fminf(cB, godunov_jw<kFastSqrt, false>(aB, bB, gB, kB));
        tile[tB] = nB;
        const bool chB = nB < cB - p.inner_tol;
        cB = nB;
        __syncwarp();
        if (!__any_sync(kFull, chB)) {
            more = false;
            ++it;
            break;
        }
    }
    // The next item's cursor atomic goes out now, so that it overlaps the stores, face tests
    // and queueing below (1-2 % faster; also reading the next list entry here is not).
    unsigned nx = 0;
    if (!kAsync && lane == 0) nx = atomicAdd(cursor, 1u);
    const float c0 = red0 ? cA : cB, c1 = red0 ? cB : cA;
    ws.act += 1;
    ws.inner += (unsigned long long)it;

    const bool any_drop = __any_sync(kFull, (c0 < i0) | (c1 < i1));
    if (!any_drop) ws.idle += 1;
    if (any_drop) {
        const int n0 = lane_node(lane);
        __stcg(Tb + n0, c0);
        __stcg(Tb + n0 + 16, c1);
    }

    // Queue a neighbour when a node on the shared face dropped by more than change_tol AND
    // its new time is below the neighbour's adjacent node y: a local update of y exceeds
    // every neighbour value it uses (causality), so a face node at or above T(y) cannot lower
    // y.  T(y) is the halo cell loaded at the start of this activation; a concurrent drop of
    // y only makes the test more permissive.
    const bool d0 = c0 < i0 - p.change_tol, d1 = c1 < i1 - p.change_tol;
    // Key of this activation's pushes: the smallest new time among its dropped nodes.
    unsigned key = kNoKey;
    if (kBand) {
        key = __reduce_min_sync(kFull, __float_as_uint(fminf(d0 ? c0 : kInf, d1 ? c1 : kInf)));
        if (key == __float_as_uint(kInf)) key = kNoKey;
    }
    unsigned fl = 0;  // faces: 1 z-, 2 z+, 4 x-, 8 x+, 16 y-, 32 y+
    if (z0 == 0 && ((d0 && c0 < tile[ti0 - 1]) || (d1 && c1 < tile[ti1 - 1]))) fl |= 1u;
    if (z0 == 3 && ((d0 && c0 < tile[ti0 + 1]) || (d1 && c1 < tile[ti1 + 1]))) fl |= 2u;
    if (x0 == 0 && ((d0 && c0 < tile[ti0 - kTileX]) || (d1 && c1 < tile[ti1 - kTileX]))) fl |= 4u;
    if (x0 == 3 && ((d0 && c0 < tile[ti0 + kTileX]) || (d1 && c1 < tile[ti1 + kTileX]))) fl |= 8u;
    if (y0 == 0 && d0 && c0 < tile[ti0 - kTileY]) fl |= 16u;
    if (y0 == 2 && d1 && c1 < tile[ti1 + kTileY]) fl |= 32u;
    const unsigned face = __reduce_or_sync(kFull, fl);

    // Queue the neighbours across those faces (lane 2 axis + up), and this brick (lane 6)
    // if it hit the cap.
    bool want = false;
    int tgt = (int)b;
    if (lane < 6) {
        const int axis = lane >> 1;
        const bool up = lane & 1;
        const int c = axis == 0 ? bz : (axis == 1 ? bx : by);
        const int nmax = axis == 0 ? nbz : (axis == 1 ? nbx : nby);
        const int stride = axis == 0 ? 1 : (axis == 1 ? nbz : nbz * nbx);
        want = ((face >> lane) & 1u) && (up ? c < nmax - 1 : c > 0);
        tgt += up ? stride : -stride;
    } else if (lane == 6) {
        want = more;
    }
    if (kAsync) {
        queue_async(p, d, s, b, want, tgt, lane == 6 ? true : false);
        return;
    }
    // Candidates go to the warp's push buffer; the global dedup and append happen 32 at a
    // time (flush_pushes), so most activations end without a global atomic.
    const unsigned wm = __ballot_sync(kFull, want);
    if (want) {
        const unsigned slot = pcnt + __popc(wm & ((1u << lane) - 1u));
        pbuf[slot] = (s << p.local_bits) | (unsigned)tgt;
        if (kBand) pkey[slot] = key;
    }
    pcnt += __popc(wm);
    // (the banded kernel flushes once per item in its own loop)
    if (!kBand && pcnt > kPushCap - 7u) flush_pushes<kBand>(p, pbuf, pkey, pcnt, round);
    next = __shfl_sync(kFull, nx, 0);
}

// Next item index of the round: one atomic per warp on the round's cursor.
__device__ __forceinline__ unsigned fetch_item(unsigned *cursor)
{
    unsigned i = 0;
    if ((threadIdx.x & 31) == 0) i = atomicAdd(cursor, 1u);
    return __shfl_sync(kFull, i, 0);
}

// Registers a thread may use so that MINB CTAs of 8 warps (or MINB / 2 of 16) fit an SM.
constexpr int fim_regs(int minb) { return minb <= 1 ? 255 : (65536 / (minb * 256)) / 8 * 8; }

// Up to 16 warps per CTA: 2 CTAs x 16 warps measured 1 % faster than 4 x 8 on the config-2
// batch (half as many CTAs arrive at each round barrier).  kBand: time-band ordering
// (FimLaunch::band > 0), a separate instance so that the plain kernel keeps its registers.
template <int MINB, bool kFastSqrt, bool kBand, bool kGather>
__global__ void __launch_bounds__(512) __maxnreg__(fim_regs(MINB)) k_fim_solve(FimLaunch p)
{
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5;
    float *tile = smem + warp * kTileNodes;
    unsigned *pbuf = reinterpret_cast<unsigned *>(smem + (blockDim.x >> 5) * kTileNodes) + warp * kPushCap;
    // the keys of the pushes (time band) sit one push-buffer array above
    unsigned *pkey = kBand ? pbuf + (blockDim.x >> 5) * kPushCap : nullptr;
    // parked items (time band): kParkCap per warp after the keys
    unsigned *kbuf = kBand ? reinterpret_cast<unsigned *>(smem + (blockDim.x >> 5) * kTileNodes) +
                                 2 * (blockDim.x >> 5) * kPushCap + warp * kParkCap
                           : nullptr;
    unsigned pcnt = 0, kcnt = 0;
    unsigned parked_through = 0;  // parking lists of rounds < this one are merged (time band)
    WarpStats ws{0ull, 0ull, 0ull, 0ull};
    const int lane = threadIdx.x & 31;
    const unsigned nwarps = gridDim.x * (blockDim.x >> 5);
    const unsigned gwarp = blockIdx.x * (blockDim.x >> 5) + warp;

    unsigned round = 0, epoch = 0;
    bool ok = true;
    for (;;) {
        const unsigned cur = round % 3u;
        const unsigned n = ld_volatile(p.ctrl + kCnt0 + cur);
        if (kBand) {
            // parked items due now (put off park_rounds rounds ago), or all of them when
            // this round has nothing else; the counts read here were final at the last
            // barrier and nobody appends to these lists this round
            const unsigned K = (unsigned)p.park_rounds;
            const unsigned from = parked_through, to = n == 0u ? round : (round >= K ? round - K + 1u : 0u);
            unsigned pending = 0;
            for (unsigned d = from; d < to; d++) {
                const unsigned j = park_slot(p, d);
                const unsigned np = ld_volatile(p.park_cnt + j);
                if (np) merge_parks(p, j, np, round);
                pending += np;
            }
            if (to > parked_through) parked_through = to;
            // the list of round - K - 1: merged by now, filled again next round
            if (blockIdx.x == 0 && threadIdx.x == 0) p.park_cnt[park_slot(p, round + 1u)] = 0u;
            if (n == 0u && pending == 0u) break;
        } else if (n == 0u) {
            break;
        }
        if ((int)round >= p.max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevRoundCap);
            ok = false;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            p.ctrl[kCnt0 + (round + 2u) % 3u] = 0u;
            p.ctrl[kCur0 + (round + 2u) % 3u] = 0u;
        }
        // Items are fetched one at a time from the round's cursor (warps that draw cheap
        // bricks take more of them).  A halo read may predate a neighbour's update in this
        // round; that neighbour then re-queues the brick, as for any concurrent update.
        const unsigned *list = p.lists + (size_t)cur * p.list_cap;
        unsigned *cursor = p.ctrl + kCur0 + cur;
        // One item at a time, fetched only when the warp is free: loading the next brick
        // ahead doubles the live registers (4 % slower), and reserving the next item index
        // early (its atomic overlapping the relaxation) is 2-5 % slower even when limited
        // to rounds with many items left; so is handing out all but the last ~2 items per
        // warp by stride, with the next item read early (5 % slower), and so are chunks of
        // 1/(G W) of the remaining items per fetch (guided self-scheduling, G = 2, 4, 8:
        // 3-9 % slower): an item held by a busy warp lengthens the round's tail.  Sixteen
        // cursors on separate lines, each over a stripe of the list, are 6 % slower: the
        // one cursor is not contended enough to matter, and the stripe scan lengthens the tail.
        // A warp's first item of the round is its own index; the cursor hands out the rest.
        // time band: per-shot minima of round - 1 (thresholds), of this round, and the array
        // reset for round + 1 (read in round - 1)
        if (kBand && blockIdx.x == 0) {
            unsigned *reset = p.band_min + (size_t)((round + 1u) % 3u) * p.nshots;  // read last round
            for (int j = threadIdx.x; j < p.nshots; j += blockDim.x) reset[j] = kNoKey;
        }
        for (unsigned i = gwarp; i < n;) {
            const unsigned item = __ldcg(list + i);
            unsigned kb = kNoKey, tb = kNoKey;
            if (kBand) {  // key and threshold loads go out with the brick's
                const unsigned s = item >> p.local_bits;
                kb = __ldcg(p.keys + p.shots[s].qbase + (item & ((1u << p.local_bits) - 1u)));
                tb = __ldcg(p.band_min + (size_t)((round + 2u) % 3u) * p.nshots + s);
            }
            BrickLoad A;
            load_brick<kGather>(p, item, A, tile);
            unsigned next = 0;
            bool defer = false;
            if (kBand && kb != kNoKey) {
                if (lane == 0) atomicMin(p.band_min + (size_t)(round % 3u) * p.nshots + A.s, kb);
                // too far ahead of its shot's front: queued again for the next round
                defer = tb != kNoKey && __uint_as_float(kb) > __uint_as_float(tb) + p.band;
                if (!defer && lane == 0) p.keys[p.shots[A.s].qbase + A.b] = kNoKey;  // consumed here
            }
            if (kBand && defer) {
                if (lane == 0) kbuf[kcnt] = item;
                kcnt += 1;
                if (kcnt == kParkCap) flush_parks(p, kbuf, kcnt, round);
                ws.deferred += 1;
                next = fetch_item(cursor);
            } else {
                relax_brick<kFastSqrt, false, kBand>(p, A, round, tile, ws, pbuf, pkey, pcnt, cursor, next);
            }
            if (kBand && pcnt > kPushCap - 7u) flush_pushes<kBand>(p, pbuf, pkey, pcnt, round);
            i = nwarps + next;
        }
        if (pcnt) flush_pushes<kBand>(p, pbuf, pkey, pcnt, round);
        if (kBand && kcnt) flush_parks(p, kbuf, kcnt, round);
        if (!grid_sync(p.ctrl, epoch, p.spin_limit)) { ok = false; break; }
        ++round;
    }
    if ((threadIdx.x & 31) == 0 && ws.act) {
        atomicAdd(p.stats + 0, ws.act);
        atomicAdd(p.stats + 1, ws.inner);
        atomicAdd(p.stats + 3, ws.idle);
    }
    if ((threadIdx.x & 31) == 0 && ws.deferred) atomicAdd(p.stats + 2, ws.deferred);
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = round;
    if (!ok || p.nrec == 0) return;

    sample_receivers(p.T, p.shots, p.nshots, p.rx, p.ry, p.rz, p.nrec, p.dx, p.dy, p.dz, p.nz, p.t_recv);
}

// ---------------------------------------------------------------------------------------
// Pair schedule (FimLaunch::pair): the rounds of k_fim_solve with two bricks per warp.
// Half h (lanes 16 h .. 16 h + 15) relaxes the warp's item 2 k + h; lane hl of a half owns
// the y-column (z, x) = (hl & 3, hl >> 2) of its brick, nodes z + 4x + 16y, y = 0..3, so
// the item fetch, the list read and the epilogue's queueing are shared by two bricks.  A
// column holds two red and two black nodes (colour z + x + y): R0, R1 at y = p, p + 2 and
// K0, K1 at y = 1 - p, 3 - p with p = (z + x) & 1; its y-neighbours are the column's other
// colour (registers) or the y halo, its x and z neighbours are other lanes' nodes (tile).
// kBand: the time band of k_fim_solve, per half (put-offs parked, pushes carry keys).
// kGather: some window of the batch reads its slowness node by node.
// ---------------------------------------------------------------------------------------
struct PairNodes {
    float r0, r1, k0, k1;  // current values
};

// One node update from its neighbour minima, with the node constants formed from h s.
template <bool kFastSqrt>
__device__ __forceinline__ float pair_update(float cur, float a, float b, float g, float hs)
{
    NodeConst k;
    k.hs = hs;
    k.q2c = 2.0f * hs * hs;
    k.q3c = 3.0f * hs * hs;
    return fminf(cur, godunov_jw<kFastSqrt, false>(a, b, g, k));
}

template <int MINB, bool kFastSqrt, bool kGather>
__global__ void __launch_bounds__(512) __maxnreg__(fim_regs(MINB)) k_fim_pair(FimLaunch p)
{
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int half = lane >> 4, hl = lane & 15;
    float *tile = smem + (2 * warp + half) * kTileNodes;
    unsigned *pbuf = reinterpret_cast<unsigned *>(smem + 2 * nw * kTileNodes) + warp * kPushCap;
    unsigned pcnt = 0;
    WarpStats ws{0ull, 0ull, 0ull, 0ull};
    const unsigned nwarps = gridDim.x * nw;
    const unsigned gwarp = blockIdx.x * nw + warp;
    const int z = hl & 3, x = hl >> 2, par = (z + x) & 1;
    // tile indices of the column's nodes and of its y halo
    const int tr0 = tile_idx(z, x, par), tr1 = tile_idx(z, x, par + 2), tk0 = tile_idx(z, x, 1 - par),
              tk1 = tile_idx(z, x, 3 - par);
    const int tylo = tile_idx(z, x, -1), tyhi = tile_idx(z, x, kBrick);

    unsigned round = 0, epoch = 0;
    bool ok = true;
    for (;;) {
        const unsigned cur = round % 3u;
        const unsigned n = ld_volatile(p.ctrl + kCnt0 + cur);
        if (n == 0u) break;
        if ((int)round >= p.max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevRoundCap);
            ok = false;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            p.ctrl[kCnt0 + (round + 2u) % 3u] = 0u;
            p.ctrl[kCur0 + (round + 2u) % 3u] = 0u;
        }
        const unsigned *list = p.lists + (size_t)cur * p.list_cap;
        unsigned *cursor = p.ctrl + kCur0 + cur;
        for (unsigned i = 2u * gwarp; i < n;) {
            // ---- load: this half's item (none when i + half >= n) ----
            const bool valid = i + (unsigned)half < n;
            const unsigned item = valid ? __ldcg(list + i + half) : 0u;
            const unsigned s = item >> p.local_bits, b = item & ((1u << p.local_bits) - 1u);
            const ShotDesc &d = p.shots[s];
            int bz = 0, bx = 0, by = 0;
            float hs0 = 0.f, hs1 = 0.f, hs2 = 0.f, hs3 = 0.f;  // h s at y = 0..3
            float t0 = kInf, t1 = kInf, t2 = kInf, t3 = kInf;
            float *Tb = p.T;
            if (valid) {
                brick_coords(d, b, bz, bx, by);
                Tb = p.T + d.t_off + (long long)b * kBrickNodes;
                const int n0 = z + 4 * x;
                if (!kGather || !d.s_gather) {
                    const float *Sb = model_brick_S(p.S, p.gbx, p.gbz, d, bz, bx, by);
                    hs0 = p.h * __ldg(Sb + n0);
                    hs1 = p.h * __ldg(Sb + n0 + 16);
                    hs2 = p.h * __ldg(Sb + n0 + 32);
                    hs3 = p.h * __ldg(Sb + n0 + 48);
                } else {
                    hs0 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0);
                    hs1 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 16);
                    hs2 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 32);
                    hs3 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 48);
                }
                t0 = __ldcg(Tb + n0);
                t1 = __ldcg(Tb + n0 + 16);
                t2 = __ldcg(Tb + n0 + 32);
                t3 = __ldcg(Tb + n0 + 48);
                // face halo: slot q = 2 axis + upper, one face node per lane (u, v) = (hl & 3, hl >> 2)
                const int u = hl & 3, v = hl >> 2;
                float hv[6];
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const int axis = q >> 1;
                    const bool up = q & 1;
                    long long nb = -1;
                    int node;
                    if (axis == 0) {
                        node = (up ? 0 : 3) + 4 * u + 16 * v;
                        if (up ? bz < d.nbz - 1 : bz > 0) nb = (long long)b + (up ? 1 : -1);
                    } else if (axis == 1) {
                        node = u + (up ? 0 : 12) + 16 * v;
                        if (up ? bx < d.nbx - 1 : bx > 0) nb = (long long)b + (up ? d.nbz : -d.nbz);
                    } else {
                        node = u + 4 * v + (up ? 0 : 48);
                        const long long sy = (long long)d.nbz * d.nbx;
                        if (up ? by < d.nby - 1 : by > 0) nb = (long long)b + (up ? sy : -sy);
                    }
                    hv[q] = nb >= 0 ? __ldcg(p.T + d.t_off + nb * kBrickNodes + node) : kInf;
                }
                tile[tile_idx(z, x, 0)] = t0;
                tile[tile_idx(z, x, 1)] = t1;
                tile[tile_idx(z, x, 2)] = t2;
                tile[tile_idx(z, x, 3)] = t3;
#pragma unroll
                for (int q = 0; q < 6; q++) {  // the halo cells' tile places
                    const int axis = q >> 1, e = (q & 1) ? kBrick : -1;
                    tile[axis == 0 ? tile_idx(e, u, v) : axis == 1 ? tile_idx(u, e, v) : tile_idx(u, v, e)] = hv[q];
                }
            }
            __syncwarp();
            // the column's colours (par = 0: R at y = 0, 2; K at 1, 3)
            PairNodes c;
            c.r0 = par ? t1 : t0;
            c.r1 = par ? t3 : t2;
            c.k0 = par ? t0 : t1;
            c.k1 = par ? t2 : t3;
            const float hr0 = par ? hs1 : hs0, hr1 = par ? hs3 : hs2, hk0 = par ? hs0 : hs1, hk1 = par ? hs2 : hs3;
            const float ylo = valid ? tile[tylo] : kInf, yhi = valid ? tile[tyhi] : kInf;
            // ---- red-black relaxation, each half until its own brick converges ----
            bool active = valid, more = valid;
            int it = 0, my_it = 0;
            for (; it < p.max_inner; ++it) {
                bool ch = false;
                if (active) {
                    const float a0 = fminf(tile[tr0 - kTileX], tile[tr0 + kTileX]);
                    const float g0 = fminf(tile[tr0 - 1], tile[tr0 + 1]);
                    const float b0 = fminf(par ? c.k0 : ylo, par ? c.k1 : c.k0);
                    const float a1 = fminf(tile[tr1 - kTileX], tile[tr1 + kTileX]);
                    const float g1 = fminf(tile[tr1 - 1], tile[tr1 + 1]);
                    const float b1 = fminf(par ? c.k1 : c.k0, par ? yhi : c.k1);
                    const float n0 = pair_update<kFastSqrt>(c.r0, a0, b0, g0, hr0);
                    const float n1 = pair_update<kFastSqrt>(c.r1, a1, b1, g1, hr1);
                    tile[tr0] = n0;
                    tile[tr1] = n1;
                    ch = (n0 < c.r0 - p.inner_tol) | (n1 < c.r1 - p.inner_tol);
                    c.r0 = n0;
                    c.r1 = n1;
                }
                __syncwarp();
                unsigned m = __ballot_sync(kFull, ch) >> (16 * half);
                if (active && it > 0 && (m & 0xffffu) == 0u) {
                    active = false;
                    more = false;
                    my_it = it + 1;
                }
                if (!__any_sync(kFull, active)) {
                    ++it;
                    break;
                }
                ch = false;
                if (active) {
                    const float a0 = fminf(tile[tk0 - kTileX], tile[tk0 + kTileX]);
                    const float g0 = fminf(tile[tk0 - 1], tile[tk0 + 1]);
                    const float b0 = fminf(par ? ylo : c.r0, par ? c.r0 : c.r1);
                    const float a1 = fminf(tile[tk1 - kTileX], tile[tk1 + kTileX]);
                    const float g1 = fminf(tile[tk1 - 1], tile[tk1 + 1]);
                    const float b1 = fminf(par ? c.r0 : c.r1, par ? c.r1 : yhi);
                    const float n0 = pair_update<kFastSqrt>(c.k0, a0, b0, g0, hk0);
                    const float n1 = pair_update<kFastSqrt>(c.k1, a1, b1, g1, hk1);
                    tile[tk0] = n0;
                    tile[tk1] = n1;
                    ch = (n0 < c.k0 - p.inner_tol) | (n1 < c.k1 - p.inner_tol);
                    c.k0 = n0;
                    c.k1 = n1;
                }
                __syncwarp();
                m = __ballot_sync(kFull, ch) >> (16 * half);
                if (active && (m & 0xffffu) == 0u) {
                    active = false;
                    more = false;
                    my_it = it + 1;
                }
                if (!__any_sync(kFull, active)) {
                    ++it;
                    break;
                }
            }
            if (active) my_it = it;  // the cap was hit: `more` stays set
            // next pair of items: the cursor atomic overlaps the epilogue
            unsigned nx = 0;
            if (lane == 0) nx = atomicAdd(cursor, 2u);
            // ---- epilogue per half: values at y = 0..3 against those at load time ----
            const float v0 = par ? c.k0 : c.r0, v1 = par ? c.r0 : c.k0, v2 = par ? c.k1 : c.r1, v3 = par ? c.r1 : c.k1;
            const bool drop = valid && ((v0 < t0) | (v1 < t1) | (v2 < t2) | (v3 < t3));
            const unsigned dm = (__ballot_sync(kFull, drop) >> (16 * half)) & 0xffffu;
            if (dm && valid) {
                const int n0 = z + 4 * x;
                __stcg(Tb + n0, v0);
                __stcg(Tb + n0 + 16, v1);
                __stcg(Tb + n0 + 32, v2);
                __stcg(Tb + n0 + 48, v3);
            }
            const bool d0 = valid && v0 < t0 - p.change_tol, d1 = valid && v1 < t1 - p.change_tol,
                       d2 = valid && v2 < t2 - p.change_tol, d3 = valid && v3 < t3 - p.change_tol;
            unsigned fl = 0;  // faces: 1 z-, 2 z+, 4 x-, 8 x+, 16 y-, 32 y+
            const int t00 = tile_idx(z, x, 0);
            if (z == 0 && ((d0 && v0 < tile[t00 - 1]) || (d1 && v1 < tile[t00 + kTileY - 1]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY - 1]) || (d3 && v3 < tile[t00 + 3 * kTileY - 1])))
                fl |= 1u;
            if (z == 3 && ((d0 && v0 < tile[t00 + 1]) || (d1 && v1 < tile[t00 + kTileY + 1]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY + 1]) || (d3 && v3 < tile[t00 + 3 * kTileY + 1])))
                fl |= 2u;
            if (x == 0 && ((d0 && v0 < tile[t00 - kTileX]) || (d1 && v1 < tile[t00 + kTileY - kTileX]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY - kTileX]) ||
                           (d3 && v3 < tile[t00 + 3 * kTileY - kTileX])))
                fl |= 4u;
            if (x == 3 && ((d0 && v0 < tile[t00 + kTileX]) || (d1 && v1 < tile[t00 + kTileY + kTileX]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY + kTileX]) ||
                           (d3 && v3 < tile[t00 + 3 * kTileY + kTileX])))
                fl |= 8u;
            if (d0 && v0 < ylo) fl |= 16u;
            if (d3 && v3 < yhi) fl |= 32u;
            const unsigned f0 = __reduce_or_sync(kFull, half == 0 ? fl : 0u);
            const unsigned f1 = __reduce_or_sync(kFull, half == 1 ? fl : 0u);
            const unsigned face = half ? f1 : f0;
            bool want = false;
            int tgt = (int)b;
            if (valid && hl < 6) {
                const int axis = hl >> 1;
                const bool up = hl & 1;
                const int cc = axis == 0 ? bz : (axis == 1 ? bx : by);
                const int nmax = axis == 0 ? d.nbz : (axis == 1 ? d.nbx : d.nby);
                const int stride = axis == 0 ? 1 : (axis == 1 ? d.nbz : d.nbz * d.nbx);
                want = ((face >> hl) & 1u) && (up ? cc < nmax - 1 : cc > 0);
                tgt += up ? stride : -stride;
            } else if (valid && hl == 6) {
                want = more;
            }
            const unsigned wm = __ballot_sync(kFull, want);
            if (want) pbuf[pcnt + __popc(wm & ((1u << lane) - 1u))] = (s << p.local_bits) | (unsigned)tgt;
            pcnt += __popc(wm);
            if (pcnt > kPushCap - 14u) flush_pushes<false>(p, pbuf, nullptr, pcnt, round);
            // stats (lane 0 keeps the warp's): both halves' activations and iterations
            const int it_h1 = __shfl_sync(kFull, my_it, 16);
            const bool two = i + 1u < n;
            ws.act += two ? 2ull : 1ull;
            ws.inner += (unsigned long long)(__shfl_sync(kFull, my_it, 0) + (two ? it_h1 : 0));
            if (!__shfl_sync(kFull, dm != 0u, 0)) ws.idle += 1;
            if (two && !__shfl_sync(kFull, dm != 0u, 16)) ws.idle += 1;
            __syncwarp();  // the tile is rewritten by the next item
            i = 2u * nwarps + __shfl_sync(kFull, nx, 0);
        }
        if (pcnt) flush_pushes<false>(p, pbuf, nullptr, pcnt, round);
        if (!grid_sync(p.ctrl, epoch, p.spin_limit)) { ok = false; break; }
        ++round;
    }
    if (lane == 0 && ws.act) {
        atomicAdd(p.stats + 0, ws.act);
        atomicAdd(p.stats + 1, ws.inner);
        atomicAdd(p.stats + 3, ws.idle);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = round;
    if (!ok || p.nrec == 0) return;

    sample_receivers(p.T, p.shots, p.nshots, p.rx, p.ry, p.rz, p.nrec, p.dx, p.dy, p.dz, p.nz, p.t_recv);
}

// The time-band instance of k_fim_pair (configs 3 and 5), a separate function so that the
// unbanded one keeps its registers (folding the band code into it cost it a 12-byte spill
// and 1.6 % on the config-2 batch).
template <int MINB, bool kFastSqrt, bool kGather>
__global__ void __launch_bounds__(512) __maxnreg__(fim_regs(MINB)) k_fim_pair_band(FimLaunch p)
{
    constexpr bool kBand = true;
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int half = lane >> 4, hl = lane & 15;
    float *tile = smem + (2 * warp + half) * kTileNodes;
    unsigned *pbuf = reinterpret_cast<unsigned *>(smem + 2 * nw * kTileNodes) + warp * kPushCap;
    // time band: the pushes' keys one push-buffer array above, then the parked items
    unsigned *pkey = kBand ? reinterpret_cast<unsigned *>(smem + 2 * nw * kTileNodes) + (nw + warp) * kPushCap
                           : nullptr;
    unsigned *kbuf = kBand ? reinterpret_cast<unsigned *>(smem + 2 * nw * kTileNodes) + 2 * nw * kPushCap +
                                 warp * kParkCap
                           : nullptr;
    unsigned pcnt = 0, kcnt = 0;
    unsigned parked_through = 0;
    WarpStats ws{0ull, 0ull, 0ull, 0ull};
    const unsigned nwarps = gridDim.x * nw;
    const unsigned gwarp = blockIdx.x * nw + warp;
    const int z = hl & 3, x = hl >> 2, par = (z + x) & 1;
    // tile indices of the column's nodes and of its y halo
    const int tr0 = tile_idx(z, x, par), tr1 = tile_idx(z, x, par + 2), tk0 = tile_idx(z, x, 1 - par),
              tk1 = tile_idx(z, x, 3 - par);
    const int tylo = tile_idx(z, x, -1), tyhi = tile_idx(z, x, kBrick);

    unsigned round = 0, epoch = 0;
    bool ok = true;
    for (;;) {
        const unsigned cur = round % 3u;
        const unsigned n = ld_volatile(p.ctrl + kCnt0 + cur);
        if (kBand) {  // parked items due now, as in k_fim_solve
            const unsigned K = (unsigned)p.park_rounds;
            const unsigned from = parked_through, to = n == 0u ? round : (round >= K ? round - K + 1u : 0u);
            unsigned pending = 0;
            for (unsigned dd = from; dd < to; dd++) {
                const unsigned j = park_slot(p, dd);
                const unsigned np = ld_volatile(p.park_cnt + j);
                if (np) merge_parks(p, j, np, round);
                pending += np;
            }
            if (to > parked_through) parked_through = to;
            if (blockIdx.x == 0 && threadIdx.x == 0) p.park_cnt[park_slot(p, round + 1u)] = 0u;
            if (n == 0u && pending == 0u) break;
        } else if (n == 0u) {
            break;
        }
        if ((int)round >= p.max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevRoundCap);
            ok = false;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            p.ctrl[kCnt0 + (round + 2u) % 3u] = 0u;
            p.ctrl[kCur0 + (round + 2u) % 3u] = 0u;
        }
        const unsigned *list = p.lists + (size_t)cur * p.list_cap;
        unsigned *cursor = p.ctrl + kCur0 + cur;
        if (kBand && blockIdx.x == 0) {  // per-shot minima for round + 1 (read in round - 1)
            unsigned *reset = p.band_min + (size_t)((round + 1u) % 3u) * p.nshots;
            for (int j = threadIdx.x; j < p.nshots; j += blockDim.x) reset[j] = kNoKey;
        }
        for (unsigned i = 2u * gwarp; i < n;) {
            // ---- load: this half's item (none when i + half >= n) ----
            const bool valid = i + (unsigned)half < n;
            const unsigned item = valid ? __ldcg(list + i + half) : 0u;
            const unsigned s = item >> p.local_bits, b = item & ((1u << p.local_bits) - 1u);
            const ShotDesc &d = p.shots[s];
            unsigned kb = kNoKey, tb = kNoKey;
            if (kBand && valid) {  // key and threshold loads go out with the brick's
                kb = __ldcg(p.keys + d.qbase + b);
                tb = __ldcg(p.band_min + (size_t)((round + 2u) % 3u) * p.nshots + s);
            }
            int bz = 0, bx = 0, by = 0;
            float hs0 = 0.f, hs1 = 0.f, hs2 = 0.f, hs3 = 0.f;  // h s at y = 0..3
            float t0 = kInf, t1 = kInf, t2 = kInf, t3 = kInf;
            float *Tb = p.T;
            if (valid) {
                brick_coords(d, b, bz, bx, by);
                Tb = p.T + d.t_off + (long long)b * kBrickNodes;
                const int n0 = z + 4 * x;
                if (!kGather || !d.s_gather) {
                    const float *Sb = model_brick_S(p.S, p.gbx, p.gbz, d, bz, bx, by);
                    hs0 = p.h * __ldg(Sb + n0);
                    hs1 = p.h * __ldg(Sb + n0 + 16);
                    hs2 = p.h * __ldg(Sb + n0 + 32);
                    hs3 = p.h * __ldg(Sb + n0 + 48);
                } else {
                    hs0 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0);
                    hs1 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 16);
                    hs2 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 32);
                    hs3 = p.h * gather_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 48);
                }
                t0 = __ldcg(Tb + n0);
                t1 = __ldcg(Tb + n0 + 16);
                t2 = __ldcg(Tb + n0 + 32);
                t3 = __ldcg(Tb + n0 + 48);
                // face halo: slot q = 2 axis + upper, one face node per lane (u, v) = (hl & 3, hl >> 2)
                const int u = hl & 3, v = hl >> 2;
                float hv[6];
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const int axis = q >> 1;
                    const bool up = q & 1;
                    long long nb = -1;
                    int node;
                    if (axis == 0) {
                        node = (up ? 0 : 3) + 4 * u + 16 * v;
                        if (up ? bz < d.nbz - 1 : bz > 0) nb = (long long)b + (up ? 1 : -1);
                    } else if (axis == 1) {
                        node = u + (up ? 0 : 12) + 16 * v;
                        if (up ? bx < d.nbx - 1 : bx > 0) nb = (long long)b + (up ? d.nbz : -d.nbz);
                    } else {
                        node = u + 4 * v + (up ? 0 : 48);
                        const long long sy = (long long)d.nbz * d.nbx;
                        if (up ? by < d.nby - 1 : by > 0) nb = (long long)b + (up ? sy : -sy);
                    }
                    hv[q] = nb >= 0 ? __ldcg(p.T + d.t_off + nb * kBrickNodes + node) : kInf;
                }
                tile[tile_idx(z, x, 0)] = t0;
                tile[tile_idx(z, x, 1)] = t1;
                tile[tile_idx(z, x, 2)] = t2;
                tile[tile_idx(z, x, 3)] = t3;
#pragma unroll
                for (int q = 0; q < 6; q++) {  // the halo cells' tile places
                    const int axis = q >> 1, e = (q & 1) ? kBrick : -1;
                    tile[axis == 0 ? tile_idx(e, u, v) : axis == 1 ? tile_idx(u, e, v) : tile_idx(u, v, e)] = hv[q];
                }
            }
            __syncwarp();
            // time band: a brick too far ahead of its shot's front is put off (parked)
            bool defer = false;
            if (kBand && valid && kb != kNoKey) {
                if (hl == 0) atomicMin(p.band_min + (size_t)(round % 3u) * p.nshots + s, kb);
                defer = tb != kNoKey && __uint_as_float(kb) > __uint_as_float(tb) + p.band;
                if (!defer && hl == 0) p.keys[d.qbase + b] = kNoKey;  // consumed here
            }
            const bool relax = valid && !defer;
            if (kBand) {
                const unsigned pm = __ballot_sync(kFull, defer && hl == 0);
                if (defer && hl == 0) kbuf[kcnt + __popc(pm & ((1u << lane) - 1u))] = item;
                kcnt += __popc(pm);
                ws.deferred += __popc(pm);
                if (kcnt > kParkCap - 2u) flush_parks(p, kbuf, kcnt, round);
            }
            // the column's colours (par = 0: R at y = 0, 2; K at 1, 3)
            PairNodes c;
            c.r0 = par ? t1 : t0;
            c.r1 = par ? t3 : t2;
            c.k0 = par ? t0 : t1;
            c.k1 = par ? t2 : t3;
            const float hr0 = par ? hs1 : hs0, hr1 = par ? hs3 : hs2, hk0 = par ? hs0 : hs1, hk1 = par ? hs2 : hs3;
            const float ylo = relax ? tile[tylo] : kInf, yhi = relax ? tile[tyhi] : kInf;
            // ---- red-black relaxation, each half until its own brick converges ----
            bool active = relax, more = relax;
            int it = 0, my_it = 0;
            for (; it < p.max_inner; ++it) {
                bool ch = false;
                if (active) {
                    const float a0 = fminf(tile[tr0 - kTileX], tile[tr0 + kTileX]);
                    const float g0 = fminf(tile[tr0 - 1], tile[tr0 + 1]);
                    const float b0 = fminf(par ? c.k0 : ylo, par ? c.k1 : c.k0);
                    const float a1 = fminf(tile[tr1 - kTileX], tile[tr1 + kTileX]);
                    const float g1 = fminf(tile[tr1 - 1], tile[tr1 + 1]);
                    const float b1 = fminf(par ? c.k1 : c.k0, par ? yhi : c.k1);
                    const float n0 = pair_update<kFastSqrt>(c.r0, a0, b0, g0, hr0);
                    const float n1 = pair_update<kFastSqrt>(c.r1, a1, b1, g1, hr1);
                    tile[tr0] = n0;
                    tile[tr1] = n1;
                    ch = (n0 < c.r0 - p.inner_tol) | (n1 < c.r1 - p.inner_tol);
                    c.r0 = n0;
                    c.r1 = n1;
                }
                __syncwarp();
                unsigned m = __ballot_sync(kFull, ch) >> (16 * half);
                if (active && it > 0 && (m & 0xffffu) == 0u) {
                    active = false;
                    more = false;
                    my_it = it + 1;
                }
                if (!__any_sync(kFull, active)) {
                    ++it;
                    break;
                }
                ch = false;
                if (active) {
                    const float a0 = fminf(tile[tk0 - kTileX], tile[tk0 + kTileX]);
                    const float g0 = fminf(tile[tk0 - 1], tile[tk0 + 1]);
                    const float b0 = fminf(par ? ylo : c.r0, par ? c.r0 : c.r1);
                    const float a1 = fminf(tile[tk1 - kTileX], tile[tk1 + kTileX]);
                    const float g1 = fminf(tile[tk1 - 1], tile[tk1 + 1]);
                    const float b1 = fminf(par ? c.r0 : c.r1, par ? c.r1 : yhi);
                    const float n0 = pair_update<kFastSqrt>(c.k0, a0, b0, g0, hk0);
                    const float n1 = pair_update<kFastSqrt>(c.k1, a1, b1, g1, hk1);
                    tile[tk0] = n0;
                    tile[tk1] = n1;
                    ch = (n0 < c.k0 - p.inner_tol) | (n1 < c.k1 - p.inner_tol);
                    c.k0 = n0;
                    c.k1 = n1;
                }
                __syncwarp();
                m = __ballot_sync(kFull, ch) >> (16 * half);
                if (active && (m & 0xffffu) == 0u) {
                    active = false;
                    more = false;
                    my_it = it + 1;
                }
                if (!__any_sync(kFull, active)) {
                    ++it;
                    break;
                }
            }
            if (active) my_it = it;  // the cap was hit: `more` stays set
            // next pair of items: the cursor atomic overlaps the epilogue
            unsigned nx = 0;
            if (lane == 0) nx = atomicAdd(cursor, 2u);
            // ---- epilogue per half: values at y = 0..3 against those at load time ----
            const float v0 = par ? c.k0 : c.r0, v1 = par ? c.r0 : c.k0, v2 = par ? c.k1 : c.r1, v3 = par ? c.r1 : c.k1;
            const bool drop = relax && ((v0 < t0) | (v1 < t1) | (v2 < t2) | (v3 < t3));
            const unsigned dm = (__ballot_sync(kFull, drop) >> (16 * half)) & 0xffffu;
            if (dm && relax) {
                const int n0 = z + 4 * x;
                __stcg(Tb + n0, v0);
                __stcg(Tb + n0 + 16, v1);
                __stcg(Tb + n0 + 32, v2);
                __stcg(Tb + n0 + 48, v3);
            }
            const bool d0 = relax && v0 < t0 - p.change_tol, d1 = relax && v1 < t1 - p.change_tol,
                       d2 = relax && v2 < t2 - p.change_tol, d3 = relax && v3 < t3 - p.change_tol;
            // time band: key of the half's pushes, the smallest new time among its dropped nodes
            unsigned key = kNoKey;
            if (kBand) {
                const unsigned kl = __float_as_uint(
                    fminf(fminf(d0 ? v0 : kInf, d1 ? v1 : kInf), fminf(d2 ? v2 : kInf, d3 ? v3 : kInf)));
                const unsigned k0 = __reduce_min_sync(kFull, half == 0 ? kl : 0xffffffffu);
                const unsigned k1 = __reduce_min_sync(kFull, half == 1 ? kl : 0xffffffffu);
                key = half ? k1 : k0;
                if (key == __float_as_uint(kInf)) key = kNoKey;
            }
            unsigned fl = 0;  // faces: 1 z-, 2 z+, 4 x-, 8 x+, 16 y-, 32 y+
            const int t00 = tile_idx(z, x, 0);
            if (z == 0 && ((d0 && v0 < tile[t00 - 1]) || (d1 && v1 < tile[t00 + kTileY - 1]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY - 1]) || (d3 && v3 < tile[t00 + 3 * kTileY - 1])))
                fl |= 1u;
            if (z == 3 && ((d0 && v0 < tile[t00 + 1]) || (d1 && v1 < tile[t00 + kTileY + 1]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY + 1]) || (d3 && v3 < tile[t00 + 3 * kTileY + 1])))
                fl |= 2u;
            if (x == 0 && ((d0 && v0 < tile[t00 - kTileX]) || (d1 && v1 < tile[t00 + kTileY - kTileX]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY - kTileX]) ||
                           (d3 && v3 < tile[t00 + 3 * kTileY - kTileX])))
                fl |= 4u;
            if (x == 3 && ((d0 && v0 < tile[t00 + kTileX]) || (d1 && v1 < tile[t00 + kTileY + kTileX]) ||
                           (d2 && v2 < tile[t00 + 2 * kTileY + kTileX]) ||
                           (d3 && v3 < tile[t00 + 3 * kTileY + kTileX])))
                fl |= 8u;
            if (d0 && v0 < ylo) fl |= 16u;
            if (d3 && v3 < yhi) fl |= 32u;
            const unsigned f0 = __reduce_or_sync(kFull, half == 0 ? fl : 0u);
            const unsigned f1 = __reduce_or_sync(kFull, half == 1 ? fl : 0u);
            const unsigned face = half ? f1 : f0;
            bool want = false;
            int tgt = (int)b;
            if (relax && hl < 6) {
                const int axis = hl >> 1;
                const bool up = hl & 1;
                const int cc = axis == 0 ? bz : (axis == 1 ? bx : by);
                const int nmax = axis == 0 ? d.nbz : (axis == 1 ? d.nbx : d.nby);
                const int stride = axis == 0 ? 1 : (axis == 1 ? d.nbz : d.nbz * d.nbx);
                want = ((face >> hl) & 1u) && (up ? cc < nmax - 1 : cc > 0);
                tgt += up ? stride : -stride;
            } else if (relax && hl == 6) {
                want = more;
            }
            const unsigned wm = __ballot_sync(kFull, want);
            if (want) {
                const unsigned slot = pcnt + __popc(wm & ((1u << lane) - 1u));
                pbuf[slot] = (s << p.local_bits) | (unsigned)tgt;
                if (kBand) pkey[slot] = key;
            }
            pcnt += __popc(wm);
            if (pcnt > kPushCap - 14u) flush_pushes<kBand>(p, pbuf, pkey, pcnt, round);
            // stats (lane 0 keeps the warp's): both halves' activations and iterations
            // (without a band every valid half relaxes: half 0 always, half 1 when i + 1 < n)
            const bool r0 = kBand ? __shfl_sync(kFull, relax, 0) : true;
            const bool r1 = kBand ? __shfl_sync(kFull, relax, 16) : i + 1u < n;
            const int it_h0 = __shfl_sync(kFull, my_it, 0), it_h1 = __shfl_sync(kFull, my_it, 16);
            ws.act += (r0 ? 1ull : 0ull) + (r1 ? 1ull : 0ull);
            ws.inner += (unsigned long long)((r0 ? it_h0 : 0) + (r1 ? it_h1 : 0));
            if (r0 && !__shfl_sync(kFull, dm != 0u, 0)) ws.idle += 1;
            if (r1 && !__shfl_sync(kFull, dm != 0u, 16)) ws.idle += 1;
            __syncwarp();  // the tile is rewritten by the next item
            i = 2u * nwarps + __shfl_sync(kFull, nx, 0);
        }
        if (pcnt) flush_pushes<kBand>(p, pbuf, pkey, pcnt, round);
        if (kBand && kcnt) flush_parks(p, kbuf, kcnt, round);
        if (!grid_sync(p.ctrl, epoch, p.spin_limit)) { ok = false; break; }
        ++round;
    }
    if (lane == 0 && ws.act) {
        atomicAdd(p.stats + 0, ws.act);
        atomicAdd(p.stats + 1, ws.inner);
        atomicAdd(p.stats + 3, ws.idle);
    }
    if (lane == 0 && ws.deferred) atomicAdd(p.stats + 2, ws.deferred);
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = round;
    if (!ok || p.nrec == 0) return;

    sample_receivers(p.T, p.shots, p.nshots, p.rx, p.ry, p.rz, p.nrec, p.dx, p.dy, p.dz, p.nz, p.t_recv);
}

template <int MINB, bool kFastSqrt>
__global__ void __launch_bounds__(256, MINB) k_fim_async(FimLaunch p)
{
    extern __shared__ float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *tile = smem + warp * kTileNodes;
    WarpStats ws{0ull, 0ull, 0ull};
    unsigned *ring = ring_of(p);
    const unsigned long long act_cap =
        p.max_rounds > 0 ? (unsigned long long)p.max_rounds * p.list_cap : ~0ull;  // activations
    for (;;) {
        unsigned h = 0, item = kEmpty;
        int done = 0;
        if (lane == 0) {
            h = atomicAdd(p.ctrl + kCur0, 1u) % ring_cap(p);
            unsigned long long spins = 0;
            for (;;) {
                // Claim the slot's item with an exchange: with fewer slots than warps two
                // consumers can wait on one slot (one lap apart); only one gets the item.
                if (ld_volatile(ring + h) != kEmpty) {
                    item = atomicExch(ring + h, kEmpty);
                    if (item != kEmpty) break;
                }
                if (ld_volatile(p.ctrl + kCnt1) == 0u || ld_volatile(p.ctrl + kErr) != 0u) {
                    done = 1;
                    break;
                }
                if (++spins > p.spin_limit) {
                    atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevBarrierTimeout);
                    done = 1;
                    break;
                }
                __nanosleep(32);
            }
            if (!done) {
                // Owned before any of the brick is read (and fenced below): a neighbour that
                // stored before finding the brick queued is seen; one that stores later
                // finds it owned and marks it dirty.
                const unsigned s = item >> p.local_bits, b = item & ((1u << p.local_bits) - 1u);
                atomicExch(p.qflag + p.shots[s].qbase + b, kOwned);
                if (atomicAdd(p.stats + 2, 1ull) >= act_cap) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevRoundCap);
            }
        }
        done = __shfl_sync(kFull, done, 0);
        if (done) break;
        item = __shfl_sync(kFull, item, 0);
        __threadfence();  // the previous owner's stores of neighbouring bricks are visible
        BrickLoad A;
        load_brick<true>(p, item, A, tile);
        unsigned unused = 0, unused_next = 0;
        relax_brick<kFastSqrt, true>(p, A, 0u, tile, ws, nullptr, nullptr, unused, nullptr, unused_next);
    }
    if (lane == 0 && ws.act) {
        atomicAdd(p.stats + 0, ws.act);
        atomicAdd(p.stats + 1, ws.inner);
        atomicAdd(p.stats + 3, ws.idle);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = 0u;
    // receivers once every brick is done: wait until no work is pending (bounded)
    if (p.nrec == 0) return;
    if (threadIdx.x == 0) {
        unsigned long long spins = 0;
        while (ld_volatile(p.ctrl + kCnt1) != 0u && ld_volatile(p.ctrl + kErr) == 0u) {
            if (++spins > p.spin_limit) {
                atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevBarrierTimeout);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    if (ld_volatile(p.ctrl + kErr) != 0u) return;
    sample_receivers(p.T, p.shots, p.nshots, p.rx, p.ry, p.rz, p.nrec, p.dx, p.dy, p.dz, p.nz, p.t_recv);
}

// -------------------------------------------------------------------------------------
// 8^3 bricks.  A work item is a 2 x 2 x 2 group of the 4^3 storage bricks (so every other
// reader of the traveltime pool is unchanged), relaxed by one CTA of 8 warps: warp w owns
// the group's brick (w & 1, (w >> 1) & 1, w >> 2) in (z, x, y), two y-adjacent nodes per
// lane as in the 4^3 kernel, and the group's 10^3 tile (the 8^3 nodes and the one-node
// halo of its six faces) sits in shared memory.  The red-black phases are separated by
// __syncthreads_or, which is both the barrier and the convergence vote.  Halo, face tests
// and re-queueing are per group: a dropped node on an outer face below the neighbouring
// halo cell queues the neighbouring group.  Groups at the far edges of a window where a
// brick count is odd are partial; their missing bricks stay INF and are never relaxed.
// Rounds, lists, cursors and the grid barrier are those of the 4^3 kernel.
// -------------------------------------------------------------------------------------
constexpr int kT8X = 12;         // tile strides, z fastest: 10 z padded to 12, then 10 x
constexpr int kT8Y = kT8X * 10;  // the lane pattern of a phase falls in 32 distinct banks
constexpr int kT8N = kT8Y * 10;
constexpr unsigned kPushCap8 = 64;

__device__ __forceinline__ int t8(int z, int x, int y) { return (z + 1) + kT8X * (x + 1) + kT8Y * (y + 1); }

__device__ __forceinline__ void group_coords(const ShotDesc &d, unsigned g, int &gz, int &gx, int &gy)
{
    const unsigned tq = (unsigned)(((unsigned long long)g * d.div8z_m) >> d.div8z_sh);  // g / gbz8
    gz = (int)(g - tq * (unsigned)d.gbz8);
    const unsigned q2 = (unsigned)(((unsigned long long)tq * d.div8x_m) >> d.div8x_sh);  // / gbx8
    gx = (int)(tq - q2 * (unsigned)d.gbx8);
    gy = (int)q2;
}

// Warp 0: queues the buffered groups for round + 1 (de-duplicated by the groups' queue flags).
__device__ __forceinline__ void flush_pushes8(const FimLaunch &p, const unsigned *pbuf, unsigned cnt, unsigned round)
{
    const int lane = threadIdx.x & 31;
    const unsigned tag = round + 2u;  // "queued for round+1", offset by one so 0 = never
    const unsigned nxt = (round + 1u) % 3u;
    for (unsigned base = 0; base < cnt; base += 32u) {
        bool want = false;
        unsigned item = 0;
        if (base + (unsigned)lane < cnt) {
            item = pbuf[base + lane];
            const unsigned s = item >> p.local_bits, g = item & ((1u << p.local_bits) - 1u);
            want = atomicMax(p.qflag + p.shots[s].qbase8 + g, tag) < tag;
        }
        const unsigned wm = __ballot_sync(kFull, want);
        if (wm) {
            const int leader = __ffs(wm) - 1;
            unsigned b0 = 0;
            if (lane == leader) b0 = atomicAdd(p.ctrl + kCnt0 + nxt, (unsigned)__popc(wm));
            b0 = __shfl_sync(kFull, b0, leader);
            if (want) p.lists[(size_t)nxt * p.list_cap + b0 + __popc(wm & ((1u << lane) - 1u))] = item;
        }
    }
}

template <int MINB, bool kFastSqrt>
__global__ void __launch_bounds__(256) __maxnreg__(fim_regs(MINB)) k_fim_solve8(FimLaunch p)
{
    __shared__ float tile[kT8N];
    __shared__ unsigned pbuf[kPushCap8];
    __shared__ unsigned s_face, s_next, s_pcnt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wz = warp & 1, wx = (warp >> 1) & 1, wy = warp >> 2;
    const int z0 = 4 * wz + (lane & 3), x0 = 4 * wx + ((lane >> 2) & 3), y0 = 4 * wy + 2 * (lane >> 4);
    const int ti0 = t8(z0, x0, y0), ti1 = ti0 + kT8Y;  // the lane's nodes (y, y + 1)
    const int n0 = lane_node(lane);
    // red: z + x + y even (y0 is even); the lane's two nodes have opposite colours
    const bool red0 = ((z0 + x0) & 1) == 0;
    const int tA = red0 ? ti0 : ti1, tB = red0 ? ti1 : ti0;
    const int yA = red0 ? -kT8Y : kT8Y;
    unsigned long long act = 0, inner = 0, idle = 0;
    if (threadIdx.x == 0) s_pcnt = 0;
    unsigned round = 0, epoch = 0;
    bool ok = true;
    for (;;) {
        const unsigned cur = round % 3u;
        const unsigned n = ld_volatile(p.ctrl + kCnt0 + cur);
        if (n == 0u) break;
        if ((int)round >= p.max_rounds) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(p.ctrl + kErr, 0u, (unsigned)kDevRoundCap);
            ok = false;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            p.ctrl[kCnt0 + (round + 2u) % 3u] = 0u;
            p.ctrl[kCur0 + (round + 2u) % 3u] = 0u;
        }
        const unsigned *list = p.lists + (size_t)cur * p.list_cap;
        unsigned *cursor = p.ctrl + kCur0 + cur;
        for (unsigned i = blockIdx.x; i < n;) {
            const unsigned item = __ldcg(list + i);
            const unsigned s = item >> p.local_bits, g = item & ((1u << p.local_bits) - 1u);
            const ShotDesc &d = p.shots[s];
            int gz, gx, gy;
            group_coords(d, g, gz, gx, gy);
            const int bz = 2 * gz + wz, bx = 2 * gx + wx, by = 2 * gy + wy;
            const bool present = bz < d.nbz && bx < d.nbx && by < d.nby;
            const long long b = bz + (long long)d.nbz * (bx + (long long)d.nbx * by);
            float *Tb = p.T + d.t_off + b * kBrickNodes;
            float s0 = 0.f, s1 = 0.f, i0 = kInf, i1 = kInf;
            if (present) {
                s0 = node_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0);
                s1 = node_S(p.S, p.gbx, p.gbz, d, bz, bx, by, n0 + 16);
                i0 = __ldcg(Tb + n0);
                i1 = __ldcg(Tb + n0 + 16);
            }
            tile[ti0] = i0;
            tile[ti1] = i1;
            // outer-face halo next to this warp's brick: slot 0 -- lanes 0-15 axis z, 16-31
            // axis x; slot 1 -- lanes 0-15 axis y (one face node each)
#pragma unroll
            for (int slot = 0; slot < 2; slot++) {
                const int q = slot == 0 ? (lane >> 4) : 2;
                if (slot == 1 && lane >= 16) break;
                const int j = lane & 15, u = j & 3, v = j >> 2;
                const bool lower = (q == 0 ? wz : q == 1 ? wx : wy) == 0;
                int node, ti;
                long long nb = -1;
                if (q == 0) {
                    node = (lower ? 3 : 0) + 4 * u + 16 * v;
                    ti = t8(lower ? -1 : 8, 4 * wx + u, 4 * wy + v);
                    if (present && (lower ? bz > 0 : bz < d.nbz - 1)) nb = b + (lower ? -1 : 1);
                } else if (q == 1) {
                    node = u + (lower ? 12 : 0) + 16 * v;
                    ti = t8(4 * wz + u, lower ? -1 : 8, 4 * wy + v);
                    if (present && (lower ? bx > 0 : bx < d.nbx - 1)) nb = b + (lower ? -d.nbz : d.nbz);
                } else {
                    node = u + 4 * v + (lower ? 48 : 0);
                    ti = t8(4 * wz + u, 4 * wx + v, lower ? -1 : 8);
                    const long long sy = (long long)d.nbz * d.nbx;
                    if (present && (lower ? by > 0 : by < d.nby - 1)) nb = b + (lower ? -sy : sy);
                }
                tile[ti] = nb >= 0 ? __ldcg(p.T + d.t_off + nb * kBrickNodes + node) : kInf;
            }
            if (threadIdx.x == 0) s_face = 0u;
            __syncthreads();  // the tile

            float cA = red0 ? i0 : i1, cB = red0 ? i1 : i0;
            const NodeConst kA = node_const(p.h, red0 ? s0 : s1), kB = node_const(p.h, red0 ? s1 : s0);
            bool more = true;
            int it = 0;
            for (; it < p.max_inner; ++it) {
                bool chA = false;
                if (present) {
                    const float aA = fminf(tile[tA - kT8X], tile[tA + kT8X]);
                    const float gA = fminf(tile[tA - 1], tile[tA + 1]);
                    const float bA = fminf(tile[tA + yA], cB);
                    const float nA = fminf(cA, godunov_jw<kFastSqrt, false>(aA, bA, gA, kA));
                    tile[tA] = nA;
                    chA = nA < cA - p.inner_tol;
                    cA = nA;
                }
                if (!__syncthreads_or(chA) && it > 0) {
                    more = false;
                    ++it;
                    break;
                }
                bool chB = false;
                if (present) {
                    const float aB = fminf(tile[tB - kT8X], tile[tB + kT8X]);
                    const float gB = fminf(tile[tB - 1], tile[tB + 1]);
                    const float bB = fminf(tile[tB - yA], cA);
                    const float nB = fminf(cB, godunov_jw<kFastSqrt, false>(aB, bB, gB, kB));
                    tile[tB] = nB;
                    chB = nB < cB - p.inner_tol;
                    cB = nB;
                }
                if (!__syncthreads_or(chB)) {
                    more = false;
                    ++it;
                    break;
                }
            }
            // the next item's cursor atomic overlaps the epilogue
            if (threadIdx.x == 0) s_next = atomicAdd(cursor, 1u);
            const float c0 = red0 ? cA : cB, c1 = red0 ? cB : cA;
            const bool drop = present && ((c0 < i0) | (c1 < i1));
            if (present && __any_sync(kFull, drop)) {
                __stcg(Tb + n0, c0);
                __stcg(Tb + n0 + 16, c1);
            }
            // outer faces of the group (1 z-, 2 z+, 4 x-, 8 x+, 16 y-, 32 y+): a node that
            // dropped by more than change_tol below the neighbouring halo cell
            const bool d0 = present && c0 < i0 - p.change_tol, d1 = present && c1 < i1 - p.change_tol;
            unsigned fl = 0;
            if (z0 == 0 && ((d0 && c0 < tile[ti0 - 1]) || (d1 && c1 < tile[ti1 - 1]))) fl |= 1u;
            if (z0 == 7 && ((d0 && c0 < tile[ti0 + 1]) || (d1 && c1 < tile[ti1 + 1]))) fl |= 2u;
            if (x0 == 0 && ((d0 && c0 < tile[ti0 - kT8X]) || (d1 && c1 < tile[ti1 - kT8X]))) fl |= 4u;
            if (x0 == 7 && ((d0 && c0 < tile[ti0 + kT8X]) || (d1 && c1 < tile[ti1 + kT8X]))) fl |= 8u;
            if (y0 == 0 && d0 && c0 < tile[ti0 - kT8Y]) fl |= 16u;
            if (y0 == 6 && d1 && c1 < tile[ti1 + kT8Y]) fl |= 32u;
            fl = __reduce_or_sync(kFull, fl);
            if (lane == 0 && fl) atomicOr(&s_face, fl);
            const int any_drop = __syncthreads_or(drop);  // also publishes s_face and s_next
            if (warp == 0) {
                bool want = false;
                unsigned tgt = g;
                if (lane < 6) {
                    const int axis = lane >> 1;
                    const bool up = lane & 1;
                    const int c = axis == 0 ? gz : (axis == 1 ? gx : gy);
                    const int nmax = axis == 0 ? d.gbz8 : (axis == 1 ? d.gbx8 : d.gby8);
                    const unsigned stride = axis == 0 ? 1u : (axis == 1 ? (unsigned)d.gbz8 : (unsigned)(d.gbz8 * d.gbx8));
                    want = ((s_face >> lane) & 1u) && (up ? c < nmax - 1 : c > 0);
                    tgt = up ? g + stride : g - stride;
                } else if (lane == 6) {
                    want = more;
                }
                const unsigned wm = __ballot_sync(kFull, want);
                unsigned pc = s_pcnt;
                if (want) pbuf[pc + __popc(wm & ((1u << lane) - 1u))] = (s << p.local_bits) | tgt;
                pc += __popc(wm);
                __syncwarp();
                if (pc > kPushCap8 - 7u) {
                    flush_pushes8(p, pbuf, pc, round);
                    pc = 0;
                }
                if (lane == 0) {
                    s_pcnt = pc;
                    act += 1;
                    inner += (unsigned long long)it;
                    if (!any_drop) idle += 1;
                }
                __syncwarp();
            }
            const unsigned next = s_next;
            __syncthreads();  // the tile, s_face and s_next are reused by the next item
            i = gridDim.x + next;
        }
        if (warp == 0) {
            const unsigned pc = s_pcnt;
            if (pc) flush_pushes8(p, pbuf, pc, round);
            __syncwarp();
            if (lane == 0) s_pcnt = 0;
        }
        if (!grid_sync(p.ctrl, epoch, p.spin_limit)) {
            ok = false;
            break;
        }
        ++round;
    }
    if (threadIdx.x == 0 && act) {
        atomicAdd(p.stats + 0, act);
        atomicAdd(p.stats + 1, inner);
        atomicAdd(p.stats + 3, idle);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = round;
    if (!ok || p.nrec == 0) return;
    sample_receivers(p.T, p.shots, p.nshots, p.rx, p.ry, p.rz, p.nrec, p.dx, p.dy, p.dz, p.nz, p.t_recv);
}

__global__ void k_fim_seed8(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz,
                            float *T, unsigned *qflag8, unsigned *lists, unsigned local_bits, unsigned *ctrl)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nshots) {
        const ShotDesc d = shots[s];
        const int bz = d.src_brick % d.nbz, t = d.src_brick / d.nbz;
        const int bx = t % d.nbx, by = t / d.nbx;
        const float sl = node_S(S, gbx, gbz, d, bz, bx, by, d.src_node);
        T[d.t_off + (long long)d.src_brick * kBrickNodes + d.src_node] = __fmul_rn(sl, d.src_dist);
        qflag8[d.qbase8 + d.src_brick8] = 1u;
        lists[s] = ((unsigned)s << local_bits) | (unsigned)d.src_brick8;
    }
    if (s == 0) ctrl[kCnt0] = (unsigned)nshots;
}

__global__ void k_receivers(const float *T, const ShotDesc *shots, int nshots, const float *rx, const float *ry,
                            const float *rz, int nrec, float dx, float dy, float dz, int nz, float *t_recv)
{
    sample_receivers(T, shots, nshots, rx, ry, rz, nrec, dx, dy, dz, nz, t_recv);
}

cudaError_t receivers_sample(const float *T, const ShotDesc *shots, int nshots, const float *rx, const float *ry,
                             const float *rz, int nrec, float dx, float dy, float dz, int nz, float *t_recv,
                             cudaStream_t st)
{
    const long long n = (long long)nshots * nrec;
    const int grid = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    k_receivers<<<grid > 0 ? grid : 1, 256, 0, st>>>(T, shots, nshots, rx, ry, rz, nrec, dx, dy, dz, nz, t_recv);
    return cudaGetLastError();
}

// -------------------------------------------------------------------------------------
// Set-up kernels
// -------------------------------------------------------------------------------------
__global__ void k_velocity_to_slowness(const float *v, float *s, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s[i] = __fdiv_rn(1.0f, v[i]);
}

// Largest finite positive value of v (as float bits; positive floats order as unsigned).
__global__ void k_max_positive(const float *v, size_t n, unsigned *out)
{
    unsigned m = 0u;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float x = v[i];
        if (x > 0.f && x < 3.0e38f) m = max(m, __float_as_uint(x));
    }
    m = __reduce_max_sync(kFull, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Pad to the brick multiple by edge replication (Block_FIM::expand_model,
// block_FIM.cpp:8-57, is a clamp of the index) and store brick-major.
__global__ void k_brick_model(const float *slow, float *S, int nx, int ny, int nz, int nxx, int nyy, int nzz)
{
    const int gbz = nzz / kBrick, gbx = nxx / kBrick;
    const size_t total = (size_t)nxx * nyy * nzz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t brick = i / kBrickNodes;
        const int node = (int)(i % kBrickNodes);
        const int bz = (int)(brick % gbz);
        const size_t t = brick / gbz;
        const int bx = (int)(t % gbx), by = (int)(t / gbx);
        const int z = bz * kBrick + (node & 3), x = bx * kBrick + ((node >> 2) & 3), y = by * kBrick + (node >> 4);
        const int zc = min(z, nz - 1), xc = min(x, nx - 1), yc = min(y, ny - 1);
        S[i] = slow[zc + (size_t)xc * nz + (size_t)yc * nx * nz];
    }
}

__global__ void k_fim_init(float4 *T4, size_t n4, unsigned *qflag, size_t nq, unsigned *ctrl,
                           unsigned long long *stats)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const float4 inf4 = make_float4(kInf, kInf, kInf, kInf);
    for (size_t i = t; i < n4; i += stride) __stcg(T4 + i, inf4);
    for (size_t i = t; i < nq; i += stride) qflag[i] = 0u;
    if (t < kCtrlWords) ctrl[t] = 0u;
    if (t < 4) stats[t] = 0ull;
}

__global__ void k_fim_seed(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz,
                           float *T, unsigned *qflag, unsigned *lists, unsigned local_bits, unsigned *ctrl, int async)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nshots) {
        const ShotDesc d = shots[s];
        // Seed value S(seed node) * distance (block_FIM.cpp:315-317); S read from the
        // brick-major slowness at the window's brick.
        const int bz = d.src_brick % d.nbz, t = d.src_brick / d.nbz;
        const int bx = t % d.nbx, by = t / d.nbx;
        const float sl = node_S(S, gbx, gbz, d, bz, bx, by, d.src_node);
        T[d.t_off + (long long)d.src_brick * kBrickNodes + d.src_node] = __fmul_rn(sl, d.src_dist);
        qflag[d.qbase + d.src_brick] = 1u;
        lists[s] = ((unsigned)s << local_bits) | (unsigned)d.src_brick;
    }
    if (s == 0) {
        ctrl[kCnt0] = (unsigned)nshots;           // rounds: items of round 0; async: ring tail
        if (async) ctrl[kCnt1] = (unsigned)nshots;  // async: pending work
    }
}

__global__ void k_unbrick(const float *T, const ShotDesc *shots, int shot, int nz, float *out)
{
    const ShotDesc d = shots[shot];
    const size_t total = (size_t)nz * d.wnx * d.wny;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const size_t r = i / nz;
        const int x = (int)(r % d.wnx), y = (int)(r / d.wnx);
        out[i] = brick_T(T, d, x, y, z);
    }
}

// -------------------------------------------------------------------------------------
// Warm start: ceiling, verification, per-shot reset, export
// -------------------------------------------------------------------------------------
// Grid: x strides over one shot's pool nodes, y = shot.
__device__ __forceinline__ void pool_node(const ShotDesc &d, long long i, int &z, int &x, int &y)
{
    const long long b = i / kBrickNodes;
    const int node = (int)(i % kBrickNodes);
    const int bz = (int)(b % d.nbz);
    const long long t = b / d.nbz;
    const int bx = (int)(t % d.nbx), by = (int)(t / d.nbx);
    z = bz * kBrick + (node & 3);
    x = bx * kBrick + ((node >> 2) & 3);
    y = by * kBrick + (node >> 4);
}

__global__ void k_fim_ceiling(float *T, const ShotDesc *shots, int nz, const float *ceiling, float scale)
{
    const ShotDesc d = shots[blockIdx.y];
    const long long n = (long long)d.nbx * d.nby * d.nbz * kBrickNodes;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int z, x, y;
        pool_node(d, i, z, x, y);
        if (z >= nz || x >= d.wnx || y >= d.wny) continue;
        const float c = __ldg(ceiling + d.v_off + z + (long long)nz * (x + (long long)d.wnx * y));
        if (c > 0.0f && c < kInf) {
            const float u = c * scale;
            if (u < kInf) __stcg(T + d.t_off + i, u);
        }
    }
}

// Two tests per node (source node excepted):
//  * stuck: the node still holds its ceiling value, bit for bit (k_fim_ceiling's product), so
//    the solver never lowered it.  After a converged seeded solve every other node holds a
//    Godunov update of its final neighbours, so if no node is stuck the field solves the
//    discrete equation everywhere but at the source, i.e. it is the plain solution.  A
//    ceiling below the truth always leaves stuck nodes: the wrong node of smallest time
//    has correct upwind neighbours, so it cannot be an update and must hold its ceiling.
//    This holds for smooth deficits of any size, which a per-node test cannot see.
//  * deficit: t is below the update of its final neighbours by more than rel_tol.
template <bool kFastSqrt>
__global__ void k_fim_verify(const float *T, const float *S, const ShotDesc *shots, int gbx, int gbz,
                             float h, float rel_tol, const float *ceiling, float scale, int nz, unsigned long long *viol)
{
    const int s = blockIdx.y;
    const ShotDesc d = shots[s];
    const int ex = d.nbx * kBrick, ey = d.nby * kBrick, ez = d.nbz * kBrick;
    const long long n = (long long)d.nbx * d.nby * d.nbz * kBrickNodes;
    const long long src = (long long)d.src_brick * kBrickNodes + d.src_node;
    unsigned cnt = 0, stuck = 0;
    float worst = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (i == src) continue;
        int z, x, y;
        pool_node(d, i, z, x, y);
        const float t = __ldcg(T + d.t_off + i);
        if (z < nz && x < d.wnx && y < d.wny) {
            const float c = __ldg(ceiling + d.v_off + z + (long long)nz * (x + (long long)d.wnx * y));
            if (c > 0.0f && c < kInf) {
                const float u = c * scale;  // as k_fim_ceiling stored it
                if (u < kInf && __float_as_uint(t) == __float_as_uint(u)) stuck++;
            }
        }
        // neighbours as the solver sees them: nodes of the window's brick grid, INF beyond
        const float xm = x > 0 ? brick_T(T, d, x - 1, y, z) : kInf, xp = x < ex - 1 ? brick_T(T, d, x + 1, y, z) : kInf;
        const float ym = y > 0 ? brick_T(T, d, x, y - 1, z) : kInf, yp = y < ey - 1 ? brick_T(T, d, x, y + 1, z) : kInf;
        const float zm = z > 0 ? brick_T(T, d, x, y, z - 1) : kInf, zp = z < ez - 1 ? brick_T(T, d, x, y, z + 1) : kInf;
        const float sl = node_S(S, gbx, gbz, d, z >> 2, x >> 2, y >> 2, (int)(i % kBrickNodes));
        const float g = godunov_jw<kFastSqrt>(fminf(xm, xp), fminf(ym, yp), fminf(zm, zp), node_const(h, sl));
        if (g < kInf && t < g - rel_tol * g) {
            cnt++;
            worst = fmaxf(worst, (g - t) / g);
        }
    }
    worst = fmaxf(worst, __shfl_xor_sync(kFull, worst, 16));
    worst = fmaxf(worst, __shfl_xor_sync(kFull, worst, 8));
    worst = fmaxf(worst, __shfl_xor_sync(kFull, worst, 4));
    worst = fmaxf(worst, __shfl_xor_sync(kFull, worst, 2));
    worst = fmaxf(worst, __shfl_xor_sync(kFull, worst, 1));
    if ((threadIdx.x & 31) == 0 && worst > 0.0f)  // non-negative floats order as their bits
        atomicMax(viol + gridDim.y + s, (unsigned long long)__float_as_uint(worst));
    // block reductions, one atomic per block and count
    cnt = __reduce_add_sync(kFull, cnt);
    stuck = __reduce_add_sync(kFull, stuck);
    __shared__ unsigned part[32], part_stuck[32];
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = cnt;
        part_stuck[threadIdx.x >> 5] = stuck;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned tot = 0, tot_stuck = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            tot += part[w];
            tot_stuck += part_stuck[w];
        }
        if (tot) atomicAdd(viol + s, (unsigned long long)tot);
        if (tot_stuck) atomicAdd(viol + 2 * gridDim.y + s, (unsigned long long)tot_stuck);
    }
}

__global__ void k_fim_reset_shots(float *T, unsigned *qflag, const ShotDesc *shots)
{
    const ShotDesc d = shots[blockIdx.y];
    const long long nb = (long long)d.nbx * d.nby * d.nbz;
    const float4 inf4 = make_float4(kInf, kInf, kInf, kInf);
    float4 *T4 = reinterpret_cast<float4 *>(T + d.t_off);  // t_off is a multiple of 64 floats
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb * (kBrickNodes / 4);
         i += (long long)gridDim.x * blockDim.x)
        __stcg(T4 + i, inf4);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb; i += (long long)gridDim.x * blockDim.x)
        qflag[d.qbase + i] = 0u;
}

__global__ void k_unbrick_all(const float *T, const ShotDesc *shots, int nz, float *out)
{
    const ShotDesc d = shots[blockIdx.y];
    const long long total = (long long)nz * d.wnx * d.wny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const long long r = i / nz;
        const int x = (int)(r % d.wnx), y = (int)(r / d.wnx);
        out[d.v_off + i] = brick_T(T, d, x, y, z);
    }
}

// -------------------------------------------------------------------------------------
// Launchers
// -------------------------------------------------------------------------------------
static int grid_for(size_t n, int threads)
{
    size_t g = (n + threads - 1) / threads;
    if (g > 148u * 32u) g = 148u * 32u;
    return g < 1 ? 1 : (int)g;
}

cudaError_t max_positive(const float *v, size_t n, unsigned *out_bits, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out_bits, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    k_max_positive<<<grid_for(n, 256), 256, 0, st>>>(v, n, out_bits);
    return cudaGetLastError();
}

cudaError_t velocity_to_slowness(const float *v, float *s, size_t n, cudaStream_t st)
{
    k_velocity_to_slowness<<<grid_for(n, 256), 256, 0, st>>>(v, s, n);
    return cudaGetLastError();
}

cudaError_t fim_brick_model(const float *slow, float *S, int nx, int ny, int nz, int nxx, int nyy,
                            int nzz, cudaStream_t st)
{
    k_brick_model<<<grid_for((size_t)nxx * nyy * nzz, 256), 256, 0, st>>>(slow, S, nx, ny, nz, nxx, nyy, nzz);
    return cudaGetLastError();
}

cudaError_t fim_init(float *T, size_t t_count, unsigned *qflag, size_t q_count, unsigned *ctrl,
                     unsigned long long *stats, cudaStream_t st)
{
    k_fim_init<<<grid_for(t_count / 4, 256), 256, 0, st>>>(reinterpret_cast<float4 *>(T), t_count / 4,
                                                            qflag, q_count, ctrl, stats);
    return cudaGetLastError();
}

cudaError_t fim_seed(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz, float *T,
                     unsigned *qflag, unsigned *lists, unsigned local_bits, unsigned *ctrl, cudaStream_t st,
                     size_t ring_cap)
{
    if (ring_cap) {  // asynchronous schedule: an empty ring, then the seeds in its first slots
        const cudaError_t e = cudaMemsetAsync(lists, 0xff, ring_cap * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
    }
    k_fim_seed<<<(nshots + 127) / 128, 128, 0, st>>>(shots, nshots, S, gbx, gbz, T, qflag, lists, local_bits,
                                                     ctrl, ring_cap ? 1 : 0);
    return cudaGetLastError();
}

// Both schedules run as cooperative launches (every CTA resident): the rounds schedule
// needs it for its grid barrier, the asynchronous one for its waits on other CTAs' pushes.
// The pair schedule (k_fim_pair): per warp two tiles and a push buffer.
template <int MINB, bool kFastSqrt>
static cudaError_t launch_pair(const FimLaunch &p, int block_warps, int *grid_out, cudaStream_t st)
{
    const bool band = p.band > 0.f;
    const void *fn = band ? (p.gather ? (const void *)k_fim_pair_band<MINB, kFastSqrt, true>
                                      : (const void *)k_fim_pair_band<MINB, kFastSqrt, false>)
                          : (p.gather ? (const void *)k_fim_pair<MINB, kFastSqrt, true>
                                      : (const void *)k_fim_pair<MINB, kFastSqrt, false>);
    const int threads = 32 * block_warps;
    // per warp: two tiles, the push buffer, and (time band) the pushes' keys and parked items
    const size_t smem = (size_t)block_warps * (2 * kTileNodes * sizeof(float) + kPushCap * sizeof(unsigned) +
                                               (band ? (kPushCap + kParkCap) * sizeof(unsigned) : 0));
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
    FimLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st);
}

template <int MINB, bool kFastSqrt>
static cudaError_t launch_solve(const FimLaunch &p, int block_warps, bool async, int *grid_out, cudaStream_t st)
{
    const bool band = !async && p.band > 0.f;
    if (!async && p.pair) return launch_pair<MINB, kFastSqrt>(p, block_warps, grid_out, st);
    const void *fn = async          ? (const void *)k_fim_async<MINB, kFastSqrt>
                     : p.gather     ? (band ? (const void *)k_fim_solve<MINB, kFastSqrt, true, true>
                                            : (const void *)k_fim_solve<MINB, kFastSqrt, false, true>)
                     : band         ? (const void *)k_fim_solve<MINB, kFastSqrt, true, false>
                                    : (const void *)k_fim_solve<MINB, kFastSqrt, false, false>;
    if (async && block_warps > 8) block_warps = 8;  // the asynchronous kernel's CTAs hold 8 warps at most
    const int threads = 32 * block_warps;
    // per warp: its tile, its push buffer and (time band) the pushes' keys
    const size_t smem =
        (size_t)block_warps * (kTileNodes * sizeof(float) + (2 * kPushCap + kParkCap) * sizeof(unsigned));
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = nsm * per_sm;
    if (grid_out) *grid_out = grid;
    FimLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, smem, st);
}

template <bool kFastSqrt>
static cudaError_t solve_occ(const FimLaunch &p, int block_warps, int occupancy, bool async, int *grid_out,
                             cudaStream_t st)
{
    switch (occupancy) {
    case 1: return launch_solve<1, kFastSqrt>(p, block_warps, async, grid_out, st);
    case 2: return launch_solve<2, kFastSqrt>(p, block_warps, async, grid_out, st);
    case 3: return launch_solve<3, kFastSqrt>(p, block_warps, async, grid_out, st);
    case 5: return launch_solve<5, kFastSqrt>(p, block_warps, async, grid_out, st);
    case 6: return launch_solve<6, kFastSqrt>(p, block_warps, async, grid_out, st);
    default: return launch_solve<4, kFastSqrt>(p, block_warps, async, grid_out, st);
    }
}

cudaError_t fim_solve(const FimLaunch &p, int block_warps, int occupancy, bool ieee_sqrt, int *grid_out,
                      cudaStream_t st, bool async)
{
    if (block_warps < 1 || block_warps > 16) block_warps = 16;
    return ieee_sqrt ? solve_occ<false>(p, block_warps, occupancy, async, grid_out, st)
                     : solve_occ<true>(p, block_warps, occupancy, async, grid_out, st);
}

template <int MINB, bool kFastSqrt>
static cudaError_t launch_solve8(const FimLaunch &p, int *grid_out, cudaStream_t st)
{
    const void *fn = (const void *)k_fim_solve8<MINB, kFastSqrt>;
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = nsm * per_sm;
    if (grid_out) *grid_out = grid;
    FimLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, 0, st);
}

template <bool kFastSqrt>
static cudaError_t solve8_occ(const FimLaunch &p, int occupancy, int *grid_out, cudaStream_t st)
{
    switch (occupancy) {
    case 2: return launch_solve8<2, kFastSqrt>(p, grid_out, st);
    case 3: return launch_solve8<3, kFastSqrt>(p, grid_out, st);
    case 5: return launch_solve8<5, kFastSqrt>(p, grid_out, st);
    case 6: return launch_solve8<6, kFastSqrt>(p, grid_out, st);
    default: return launch_solve8<4, kFastSqrt>(p, grid_out, st);
    }
}

cudaError_t fim_solve8(const FimLaunch &p, int occupancy, bool ieee_sqrt, int *grid_out, cudaStream_t st)
{
    return ieee_sqrt ? solve8_occ<false>(p, occupancy, grid_out, st) : solve8_occ<true>(p, occupancy, grid_out, st);
}

cudaError_t fim_seed8(const ShotDesc *shots, int nshots, const float *S, int gbx, int gbz, float *T,
                      unsigned *qflag8, unsigned *lists, unsigned local_bits, unsigned *ctrl, cudaStream_t st)
{
    k_fim_seed8<<<(nshots + 127) / 128, 128, 0, st>>>(shots, nshots, S, gbx, gbz, T, qflag8, lists, local_bits,
                                                      ctrl);
    return cudaGetLastError();
}

cudaError_t fim_unbrick(const float *T, const ShotDesc *shots, int shot, int nz, float *out, cudaStream_t st)
{
    k_unbrick<<<148 * 8, 256, 0, st>>>(T, shots, shot, nz, out);
    return cudaGetLastError();
}

static dim3 per_shot_grid(int nshots) { return dim3(nshots >= 64 ? 32 : 128, (unsigned)nshots); }

cudaError_t fim_ceiling(float *T, const ShotDesc *shots, int nshots, int nz, const float *ceiling, float scale,
                        cudaStream_t st)
{
    if (nshots < 1 || nshots > 65535) return cudaErrorInvalidValue;
    k_fim_ceiling<<<per_shot_grid(nshots), 256, 0, st>>>(T, shots, nz, ceiling, scale);
    return cudaGetLastError();
}

cudaError_t fim_verify(const float *T, const float *S, const ShotDesc *shots, int nshots, int gbx,
                       int gbz, float h, float rel_tol, const float *ceiling, float scale, int nz, bool ieee_sqrt,
                       unsigned long long *viol, cudaStream_t st)
{
    if (nshots < 1 || nshots > 65535) return cudaErrorInvalidValue;
    if (ieee_sqrt)
        k_fim_verify<false><<<per_shot_grid(nshots), 256, 0, st>>>(T, S, shots, gbx, gbz, h, rel_tol, ceiling,
                                                                   scale, nz, viol);
    else
        k_fim_verify<true><<<per_shot_grid(nshots), 256, 0, st>>>(T, S, shots, gbx, gbz, h, rel_tol, ceiling,
                                                                  scale, nz, viol);
    return cudaGetLastError();
}

cudaError_t fim_reset_shots(float *T, unsigned *qflag, const ShotDesc *shots, int nshots, cudaStream_t st)
{
    if (nshots < 1 || nshots > 65535) return cudaErrorInvalidValue;
    k_fim_reset_shots<<<per_shot_grid(nshots), 256, 0, st>>>(T, qflag, shots);
    return cudaGetLastError();
}

cudaError_t fim_unbrick_all(const float *T, const ShotDesc *shots, int nshots, int nz, float *out, cudaStream_t st)
{
    if (nshots < 1 || nshots > 65535) return cudaErrorInvalidValue;
    k_unbrick_all<<<per_shot_grid(nshots), 256, 0, st>>>(T, shots, nz, out);
    return cudaGetLastError();
}

}  // namespace tomo
