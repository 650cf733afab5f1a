// C ABI: context, model and batched eikonal solve (include/tomo_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "common.cuh"
#include "context.hpp"
#include "fsm.cuh"
#include "internal.hpp"

using tomo::ShotDesc;

namespace tomo {
int rebrick_model(tomo_ctx *ctx);
int model_buffers(tomo_ctx *ctx);
const char *static_error_text();  // fim_static.cu
}

namespace {

constexpr int kDefaultMaxInner = 16;
// Launch shape of the persistent solve: 16 warps per CTA and occupancy 4 -- 32 warps per
// SM, the register budget (64) of 4 CTAs of 8 warps, i.e. 2 CTAs of 16 -- fastest on config 2.
constexpr int kDefaultOccupancy = 4;
constexpr int kDefaultBlockWarps = 16;
constexpr int kBandBlockWarps = 8, kBandOccupancy = 3;  // banded solves, untuned
#ifndef TOMO_PARK_ROUNDS
#define TOMO_PARK_ROUNDS 6
#endif
// Rounds a put-off brick waits before it is tested again (1..14).  Config-5 starting
// model, banded solve: 1: 503 ms, 2: 472, 4: 404, 6: 396, 8: 397; config 3: 4: 10.8,
// 6 and 8: 10.6 ms.
constexpr int kParkRounds = TOMO_PARK_ROUNDS;
static_assert(kParkRounds >= 1 && kParkRounds + 2 <= 16, "parking lists");
constexpr float kDefaultChangeTol = 1e-6f;
constexpr int kDefaultMaxRounds = 1 << 20;
constexpr int kMaxRounds = 1 << 22;
constexpr unsigned long long kSpinLimit = 1ull << 26;  // default: ~ seconds of polling, then error
// Warm-start check, first test: a node more than this (relative) below the update of its
// final neighbours flags its shot.  The converged FP32 field itself holds such deficits up
// to ~2.7e-7 (rounding of the update, which is monotone only up to a few ulp), so the bar is
// 5e-7.  A deficit spread thinly along a path of n nodes could hide n x 5e-7 from this
// test; the second test (a node that kept its ceiling value, fim_verify) catches any
// ceiling below the truth, smooth or not.
constexpr float kVerifyRelTol = 5e-7f;

int fail(tomo_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(tomo_ctx *c, cudaError_t e, const char *where)
{
    const int code = (e == cudaErrorMemoryAllocation) ? TOMO_ERR_OOM : TOMO_ERR_CUDA;
    return fail(c, code, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);   \
    } while (0)

int pad4(int n) { return n + (tomo::kBrick - n % tomo::kBrick) % tomo::kBrick; }

int upload_model(tomo_ctx *ctx, const float *host, bool is_velocity)
{
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    CK(ctx->slow.ensure(n));
    if (is_velocity) {
        CK(ctx->scratch_v.ensure(n));
        CK(cudaMemcpyAsync(ctx->scratch_v.ptr, host, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        CK(tomo::velocity_to_slowness(ctx->scratch_v.ptr, ctx->slow.ptr, n, ctx->stream));
    } else {
        CK(cudaMemcpyAsync(ctx->slow.ptr, host, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    }
    int rc = tomo::model_buffers(ctx);
    if (rc != TOMO_OK) return rc;
    rc = tomo::rebrick_model(ctx);
    if (rc != TOMO_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->have_model = true;
    return TOMO_OK;
}

// TOMO_OP_NGB: the reference's Accurate_FSM sweeps for every shot (csrc/fsm.cu), written
// into the brick-major pool described by sd, then the receivers.
int launch_ngb(tomo_ctx *ctx, const std::vector<ShotDesc> &sd, const tomo_point *shots, int nshots, int nrec,
               int groups, unsigned long long spin_limit)
{
    const tomo_grid &g = ctx->g;
    std::vector<tomo::FsmShot> fs((size_t)nshots);
    long long total = 0;
    for (int s = 0; s < nshots; s++) {
        tomo::FsmShot &f = fs[(size_t)s];
        const ShotDesc &d = sd[(size_t)s];
        f.wx0 = d.wx0;
        f.wy0 = d.wy0;
        f.wnx = d.wnx;
        f.wny = d.wny;
        const float sx = shots[s].x - (float)d.wx0 * g.dx, sy = shots[s].y - (float)d.wy0 * g.dy, sz = shots[s].z;
        const int nb = 1;
        f.sidx = (int)(sx / g.dx) + nb;
        f.sidy = (int)(sy / g.dy) + nb;
        f.sidz = (int)(sz / g.dz) + nb;
        // the 27 seeded nodes (accurate_FSM.cpp:596-630), including the reference's swap of
        // the (z+1, x-1) and (z-1, x+1) distances (:608-609)
        for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++)
                for (int oz = -1; oz <= 1; oz++) {
                    int fx = ox, fz = oz;
                    if (oy == 0 && oz * ox == -1) {
                        fx = -ox;
                        fz = -oz;
                    }
                    f.seed_dist[(oz + 1) + 3 * (ox + 1) + 9 * (oy + 1)] =
                        sqrtf(powf(((f.sidx - nb) + fx) * g.dx - sx, 2.0f) + powf(((f.sidy - nb) + oy) * g.dy - sy, 2.0f) +
                              powf(((f.sidz - nb) + fz) * g.dz - sz, 2.0f));
                }
        f.t_off = total;
        total += (long long)(g.nz + 2) * (d.wnx + 2) * (d.wny + 2);
    }
    // Schedule: tile by tile (fsm_solve_tiled) unless a source lies on a far face of its
    // window, where the reference's reads cross column edges and only the plane schedule
    // reproduces them; sweep_groups > 0 asks for the plane schedule with that many groups.
    const int nzz = g.nz + 2;
    bool tiled = groups <= 0;
    for (const tomo::FsmShot &f : fs)
        tiled = tiled && f.sidz <= nzz - 3 && f.sidx <= f.wnx - 1 && f.sidy <= f.wny - 1;
    int ngroups = groups > 0 ? groups : 4;  // 4 groups: fastest of 1..16 on the 64-shot batch
    if (ngroups > nshots) ngroups = nshots;
    if (tiled) ngroups = 1;
    std::vector<int> tab;
    std::vector<unsigned> shot_tiles;  // per shot and sweep: the sweep's tile count
    int tab_base[16] = {}, tab_nd[16] = {};
    long long nflags = 0;
    if (tiled) {
        auto cdiv = [](int a, int b) { return (a + b - 1) / b; };
        for (tomo::FsmShot &f : fs) {
            f.flag_off = nflags;
            nflags += (long long)cdiv(nzz - 1, tomo::kFsmTZ) * cdiv(f.wnx + 1, tomo::kFsmTX) *
                      cdiv(f.wny + 1, tomo::kFsmTY);
        }
        // per sweep: first tile of (tile diagonal d, shot s), d-major, and the tile count
        std::vector<int> A((size_t)nshots), B((size_t)nshots), C((size_t)nshots);
        shot_tiles.assign((size_t)nshots * 16, 0u);
        for (int q = 0; q < 16; q++) {
            int nd = 0;
            for (int s = 0; s < nshots; s++) {
                const tomo::FsmShot &f = fs[(size_t)s];
                A[(size_t)s] = cdiv(tomo::fsm_sweep_range(q, tomo::fsm_sign_z(q), nzz, f.sidz).L, tomo::kFsmTZ);
                B[(size_t)s] = cdiv(tomo::fsm_sweep_range(q, tomo::fsm_sign_x(q), f.wnx + 2, f.sidx).L, tomo::kFsmTX);
                C[(size_t)s] = cdiv(tomo::fsm_sweep_range(q, tomo::fsm_sign_y(q), f.wny + 2, f.sidy).L, tomo::kFsmTY);
                nd = std::max(nd, A[(size_t)s] + B[(size_t)s] + C[(size_t)s] - 2);
                shot_tiles[(size_t)s * 16 + q] = (unsigned)(A[(size_t)s] * B[(size_t)s] * C[(size_t)s]);
            }
            tab_base[q] = (int)tab.size();
            tab_nd[q] = nd;
            long long run = 0;
            for (int dg = 0; dg < nd; dg++)
                for (int s = 0; s < nshots; s++) {
                    tab.push_back((int)run);
                    run += tomo::fsm_diag_count(dg, A[(size_t)s], B[(size_t)s], C[(size_t)s]);
                }
            if (run >= (1ll << 31)) return fail(ctx, TOMO_ERR_CAPACITY, "too many sweep tiles for one NGB batch");
            tab.push_back((int)run);
        }
        CK(ctx->fsm_tab.ensure(tab.size() + shot_tiles.size()));
        CK(ctx->fsm_flags.ensure((size_t)nflags));
        CK(cudaMemcpyAsync(ctx->fsm_tab.ptr, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemcpyAsync(ctx->fsm_tab.ptr + tab.size(), shot_tiles.data(), shot_tiles.size() * sizeof(unsigned),
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(ctx->fsm_flags.ptr, 0, (size_t)nflags * sizeof(unsigned), ctx->stream));
    }
    CK(ctx->fsm_T.ensure((size_t)total));
    CK(ctx->fsm_shots.ensure((size_t)nshots));
    CK(ctx->fsm_bar.ensure((size_t)2 * ngroups + 16 + 16 * (size_t)nshots));
    CK(cudaMemcpyAsync(ctx->fsm_shots.ptr, fs.data(), fs.size() * sizeof(tomo::FsmShot), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemsetAsync(ctx->fsm_bar.ptr, 0, (2 * ngroups + 16 + 16 * (size_t)nshots) * sizeof(unsigned),
                       ctx->stream));
    CK(cudaMemsetAsync(ctx->ctrl.ptr, 0, tomo::kCtrlWords * sizeof(unsigned), ctx->stream));
    CK(cudaMemsetAsync(ctx->stats.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
    tomo::FsmLaunch p{};
    p.slow = ctx->slow.ptr;
    p.nx = g.nx;
    p.ny = g.ny;
    p.nz = g.nz;
    p.dx = g.dx;
    p.dy = g.dy;
    p.dz = g.dz;
    // Accurate_FSM::eikonal_equation (accurate_FSM.cpp:632-644), FP32 on the host
    p.dz2i = 1.0f / (g.dz * g.dz);
    p.dx2i = 1.0f / (g.dx * g.dx);
    p.dy2i = 1.0f / (g.dy * g.dy);
    p.dz2dx2 = p.dz2i * p.dx2i;
    p.dz2dy2 = p.dz2i * p.dy2i;
    p.dx2dy2 = p.dx2i * p.dy2i;
    p.dsum = p.dz2i + p.dx2i + p.dy2i;
    p.T = ctx->fsm_T.ptr;
    p.shots = ctx->fsm_shots.ptr;
    p.nshots = nshots;
    p.ngroups = ngroups;
    p.bar = ctx->fsm_bar.ptr;
    p.err = ctx->ctrl.ptr + tomo::kErr;
    p.spin_limit = spin_limit;
    p.Tb = ctx->T.ptr;
    p.desc = ctx->shots_d.ptr;
    if (tiled) {
        p.tab = ctx->fsm_tab.ptr;
        std::memcpy(p.tab_base, tab_base, sizeof(tab_base));
        std::memcpy(p.tab_nd, tab_nd, sizeof(tab_nd));
        p.flags = ctx->fsm_flags.ptr;
        p.cursors = ctx->fsm_bar.ptr + 2;
        p.shot_done = ctx->fsm_bar.ptr + 2 * ngroups + 16;
        p.shot_tiles = reinterpret_cast<const unsigned *>(ctx->fsm_tab.ptr + tab.size());
        p.sweep_barrier = nshots == 1 ? 1 : 0;  // 64 shots: 55.4 ms with the counts, 58.3 with barriers
    }
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    int grid = 0;
    if (tiled)
        CK(tomo::fsm_solve_tiled(p, &grid, ctx->stream));
    else
        CK(tomo::fsm_solve(p, &grid, ctx->stream));
    if (nrec > 0)
        CK(tomo::receivers_sample(ctx->T.ptr, ctx->shots_d.ptr, nshots, ctx->rec.ptr, ctx->rec.ptr + nrec,
                                  ctx->rec.ptr + 2 * nrec, nrec, g.dx, g.dy, g.dz, g.nz, ctx->t_recv.ptr, ctx->stream));
    return TOMO_OK;
}

}  // namespace

namespace tomo {
int model_buffers(tomo_ctx *ctx)
{
    CK(ctx->slow.ensure((size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz));
    CK(ctx->S.ensure((size_t)ctx->nxx * ctx->nyy * ctx->nzz));
    return TOMO_OK;
}

// Bricks the device model (after an upload or a model update; enqueue only, buffers from
// model_buffers).
int rebrick_model(tomo_ctx *ctx)
{
    CK(fim_brick_model(ctx->slow.ptr, ctx->S.ptr, ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->nxx, ctx->nyy, ctx->nzz,
                       ctx->stream));
    return TOMO_OK;
}
}  // namespace tomo

extern "C" {

const char *tomo_status_string(int s)
{
    switch (s) {
    case TOMO_OK: return "ok";
    case TOMO_ERR_INVALID_ARG: return "invalid argument";
    case TOMO_ERR_OOM: return "out of device memory";
    case TOMO_ERR_CUDA: return "CUDA error";
    case TOMO_ERR_NOT_CONVERGED: return "eikonal solve did not converge within the round cap";
    case TOMO_ERR_TIMEOUT: return "device-side wait timed out";
    case TOMO_ERR_STATE: return "call order (missing model, solve or Jacobian)";
    case TOMO_ERR_IO: return "file could not be opened";
    case TOMO_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case TOMO_ERR_CAPACITY: return "device capacity exceeded";
    default: return "unknown status";
    }
}

int tomo_ctx_create_on_stream(const tomo_grid *grid, int device, void *stream, tomo_ctx **out)
{
    if (!out) return TOMO_ERR_INVALID_ARG;
    *out = nullptr;
    if (!grid || grid->nx < 2 || grid->ny < 2 || grid->nz < 2 || !(grid->dx > 0) || !(grid->dy > 0) ||
        !(grid->dz > 0))
        return TOMO_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return TOMO_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return TOMO_ERR_NO_DEVICE;
    if (!prop.cooperativeLaunch) return TOMO_ERR_NO_DEVICE;
    tomo_ctx *ctx = new (std::nothrow) tomo_ctx();
    if (!ctx) return TOMO_ERR_OOM;
    ctx->g = *grid;
    ctx->device = device;
    ctx->nxx = pad4(grid->nx);
    ctx->nyy = pad4(grid->ny);
    ctx->nzz = pad4(grid->nz);
    ctx->gbx = ctx->nxx / tomo::kBrick;
    ctx->gby = ctx->nyy / tomo::kBrick;
    ctx->gbz = ctx->nzz / tomo::kBrick;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) {
        if (stream) {
            ctx->stream = static_cast<cudaStream_t>(stream);
        } else {
            e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
            ctx->own_stream = (e == cudaSuccess);
        }
    }
    for (int i = 0; i < 8 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&ctx->pinned_ctrl), 64 * sizeof(unsigned));
    if (e == cudaSuccess) e = ctx->ctrl.ensure(tomo::kCtrlWords);
    if (e == cudaSuccess) e = ctx->stats.ensure(4);
    if (e != cudaSuccess) {
        tomo_ctx_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? TOMO_ERR_OOM : TOMO_ERR_CUDA;
    }
    *out = ctx;
    return TOMO_OK;
}

int tomo_ctx_create(const tomo_grid *grid, int device, tomo_ctx **out)
{
    return tomo_ctx_create_on_stream(grid, device, nullptr, out);
}

void tomo_release_tomography(tomo_ctx *ctx);  // api_tomography.cpp
void tomo_release_iteration(tomo_ctx *ctx);   // api_iteration.cpp

int tomo_ctx_destroy(tomo_ctx *ctx)
{
    if (!ctx) return TOMO_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    tomo_release_iteration(ctx);
    tomo_release_tomography(ctx);
    ctx->slow.release();
    ctx->vel_stage.release();
    ctx->S.release();
    ctx->scratch_v.release();
    ctx->T.release();
    ctx->qflag.release();
    ctx->qflag8.release();
    ctx->lists.release();
    ctx->ctrl.release();
    ctx->stats.release();
    ctx->shots_d.release();
    ctx->shots_redo.release();
    ctx->viol.release();
    ctx->fsm_T.release();
    ctx->fsm_shots.release();
    ctx->fsm_bar.release();
    ctx->rec.release();
    ctx->t_recv.release();
    for (auto &ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->pinned_ctrl) cudaFreeHost(ctx->pinned_ctrl);
    if (ctx->ev_staged) cudaEventDestroy(ctx->ev_staged);
    if (ctx->ev_stage_free) cudaEventDestroy(ctx->ev_stage_free);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return TOMO_OK;
}

const char *tomo_last_error(const tomo_ctx *ctx) { return ctx ? ctx->err.c_str() : tomo::static_error_text(); }

void *tomo_ctx_stream(tomo_ctx *ctx) { return ctx ? static_cast<void *>(ctx->stream) : nullptr; }

int tomo_set_velocity(tomo_ctx *ctx, const float *velocity)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!velocity) return fail(ctx, TOMO_ERR_INVALID_ARG, "velocity is NULL");
    CK(cudaSetDevice(ctx->device));
    return upload_model(ctx, velocity, true);
}

int tomo_set_slowness(tomo_ctx *ctx, const float *slowness)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!slowness) return fail(ctx, TOMO_ERR_INVALID_ARG, "slowness is NULL");
    CK(cudaSetDevice(ctx->device));
    return upload_model(ctx, slowness, false);
}

int tomo_stage_velocity(tomo_ctx *ctx, const float *velocity)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!velocity) return fail(ctx, TOMO_ERR_INVALID_ARG, "velocity is NULL");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->copy_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->ev_staged, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ev_stage_free, cudaEventDisableTiming));
    }
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    CK(ctx->vel_stage.ensure(n));
    // the staging buffer is rewritten only after the last commit's conversion has read it
    if (ctx->stage_read) CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_stage_free, 0));
    CK(cudaMemcpyAsync(ctx->vel_stage.ptr, velocity, n * sizeof(float), cudaMemcpyHostToDevice, ctx->copy_stream));
    CK(cudaEventRecord(ctx->ev_staged, ctx->copy_stream));
    ctx->staged = true;
    return TOMO_OK;
}

int tomo_commit_velocity(tomo_ctx *ctx)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!ctx->staged) return fail(ctx, TOMO_ERR_STATE, "no staged velocity (tomo_stage_velocity)");
    CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    CK(ctx->slow.ensure(n));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_staged, 0));
    CK(tomo::velocity_to_slowness(ctx->vel_stage.ptr, ctx->slow.ptr, n, ctx->stream));
    CK(cudaEventRecord(ctx->ev_stage_free, ctx->stream));
    ctx->stage_read = true;
    ctx->staged = false;
    int rc = tomo::model_buffers(ctx);
    if (rc != TOMO_OK) return rc;
    rc = tomo::rebrick_model(ctx);
    if (rc != TOMO_OK) return rc;
    ctx->have_model = true;
    return TOMO_OK;
}

int tomo_get_slowness(tomo_ctx *ctx, float *out)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!out) return fail(ctx, TOMO_ERR_INVALID_ARG, "output is NULL");
    if (!ctx->have_model) return fail(ctx, TOMO_ERR_STATE, "no model set");
    CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    CK(cudaMemcpyAsync(out, ctx->slow.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_eik_brick_shapes(int *xyz, int cap)
{
    const int edge[2] = {tomo::kBrick, 2 * tomo::kBrick};  // TOMO_BRICK_4, TOMO_BRICK_8
    for (int i = 0; i < 2 && xyz && i < cap; i++) xyz[3 * i] = xyz[3 * i + 1] = xyz[3 * i + 2] = edge[i];
    return 2;
}

}  // extern "C"

namespace {

// Solver settings of one call (defaults where opts is NULL or a field is 0).
struct SolveCfg {
    int max_inner, max_rounds, block_warps, occupancy;
    float change_tol, inner_tol;
    bool ieee_sqrt;
    bool async;  // asynchronous schedule, else rounds (default)
    bool pair;   // rounds with two bricks per warp (4^3 bricks)
    float time_band;  // rounds schedule: time-band ordering (s), 0 = off
    unsigned long long spin_limit;  // polls of a device-side wait before it gives up
    bool brick8;      // 8^3 bricks (one CTA per 2 x 2 x 2 group of storage bricks)
};

SolveCfg solve_cfg(const tomo_ctx *ctx, const tomo_eik_opts *opts)
{
    SolveCfg c{};
    // fields left 0: the autotuned launch shape if there is one, else the defaults
    const int inner0 = ctx->tuned_max_inner > 0 ? ctx->tuned_max_inner : kDefaultMaxInner;
    const int warps0 = ctx->tuned_block_warps > 0 ? ctx->tuned_block_warps : kDefaultBlockWarps;
    const int occ0 = ctx->tuned_occupancy > 0 ? ctx->tuned_occupancy : kDefaultOccupancy;
    c.max_inner = (opts && opts->max_inner > 0) ? opts->max_inner : inner0;
    c.max_rounds = (opts && opts->max_rounds > 0) ? opts->max_rounds : kDefaultMaxRounds;
    // the round barrier counts arrivals of up to ~1,000 blocks per round in 32 bits
    c.max_rounds = std::min(c.max_rounds, kMaxRounds);
    c.block_warps = (opts && opts->block_warps > 0) ? opts->block_warps : warps0;
    c.occupancy = (opts && opts->occupancy > 0) ? opts->occupancy : occ0;
    // Default: the reference's convergence threshold EPS = 1e-6 s (cuda_kernel.cuh:8).
    c.change_tol = kDefaultChangeTol;
    if (opts && opts->change_tol > 0.f) c.change_tol = opts->change_tol;
    if (opts && opts->change_tol < 0.f) c.change_tol = 0.f;
    // Default: exact in-brick convergence.  Stopping the in-brick relaxation at the face
    // tolerance is 13 % faster on config 2 but raises the error vs the exact fixed point
    // from ~1e-6 to ~2e-5 relative, too close to the 1e-4 budget on larger grids.
    c.inner_tol = (opts && opts->inner_tol > 0.f) ? opts->inner_tol : 0.f;
    c.ieee_sqrt = opts && opts->ieee_sqrt;
    // Rounds by default: the asynchronous schedule relaxes bricks before their upwind
    // neighbours have settled and measured 2.5x slower on config 2 (1.8x the activations).
    c.async = opts && opts->schedule == TOMO_SCHED_ASYNC;
    // Time-band ordering: off by default.  It pays where slow paths reach bricks long
    // before the first arrival does (2.3x on the config-5 starting model at 0.2 s) and
    // costs where they do not (the windowed config-2 batch).  0: the autotuned band, if
    // the autotuner chose one; < 0: off.
    const float band = opts ? opts->time_band : 0.f;
    c.time_band = band > 0.f ? band : (band < 0.f ? 0.f : ctx->tuned_time_band);
    if (c.async) c.time_band = 0.f;
    // Two bricks per warp when asked for, or, with the schedule left to the default, when the
    // autotuner chose it or the solve is banded (time band at 8 warps x 3 CTAs per SM: config
    // 5 starting model 305 vs 435 ms, config 3 9.0 vs 9.8 ms).
    const bool sched_default = !opts || opts->schedule == TOMO_SCHED_DEFAULT;
    c.pair = (opts && opts->schedule == TOMO_SCHED_PAIR) ||
             (sched_default && (ctx->tuned_schedule == TOMO_SCHED_PAIR || c.time_band > 0.f));
    c.spin_limit = (opts && opts->spin_limit > 0) ? opts->spin_limit : kSpinLimit;
    // Brick shape: 4^3 unless asked for (or tuned to) 8^3.  The 8^3 kernel runs the rounds
    // schedule without the time band.
    const int brick = (opts && opts->brick > 0) ? opts->brick : ctx->tuned_brick;
    c.brick8 = brick == TOMO_BRICK_8 && !c.async;
    if (c.brick8) c.time_band = 0.f;
    // Banded solves carry more live state (spills at 64 registers): untuned, they run as
    // 3 CTAs x 8 warps at 80 registers, 1.15x faster than the plain default shape on the
    // config-5 starting model (504 vs 581 ms) and equal on config 3.
    if (c.time_band > 0.f) {
        if (!(opts && opts->block_warps > 0) && ctx->tuned_block_warps == 0) c.block_warps = kBandBlockWarps;
        if (!(opts && opts->occupancy > 0) && ctx->tuned_occupancy == 0) c.occupancy = kBandOccupancy;
    }
    return c;
}

// Validated per-shot descriptors of a batch and the sizes of its device arrays.
struct Batch {
    std::vector<ShotDesc> sd;
    long long t_total = 0;            // traveltime pool (floats)
    long long v_total = 0;            // all window volumes back to back (floats)
    unsigned long long q_total = 0;   // bricks
    unsigned long long q_total8 = 0;  // 8^3 groups
    bool gather = false;              // some window reads its slowness node by node
    unsigned local_bits = 1;
};

int make_batch(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
               const tomo_point *receivers, Batch &bt)
{
    const tomo_grid &g = ctx->g;
    bt.sd.assign((size_t)nshots, ShotDesc{});
    int max_bricks = 1;
    for (int s = 0; s < nshots; s++) {
        tomo_window w{0, g.nx, 0, g.ny};
        if (windows) w = windows[s];
        if (w.x0 < 0 || w.y0 < 0 || w.x1 > g.nx || w.y1 > g.ny || w.x1 - w.x0 < 2 || w.y1 - w.y0 < 2)
            return fail(ctx, TOMO_ERR_INVALID_ARG,
                        "window " + std::to_string(s) + ": must lie inside the model, at least 2 x 2 nodes");
        // A brick-aligned window's bricks are bricks of the shared brick-major model; any other
        // window gathers its slowness node by node from the model, its padding replicating the
        // window's edge like the cropped model (node_S).
        const bool aligned = w.x0 % tomo::kBrick == 0 && w.y0 % tomo::kBrick == 0 &&
                             (w.x1 % tomo::kBrick == 0 || w.x1 == g.nx) && (w.y1 % tomo::kBrick == 0 || w.y1 == g.ny);
        ShotDesc &d = bt.sd[(size_t)s];
        d.wx0 = w.x0;
        d.wy0 = w.y0;
        d.wnx = w.x1 - w.x0;
        d.wny = w.y1 - w.y0;
        d.nbx = pad4(d.wnx) / tomo::kBrick;
        d.nby = pad4(d.wny) / tomo::kBrick;
        d.nbz = ctx->gbz;
        // Source seed in window coordinates (Block_FIM::apply_source_time, block_FIM.cpp:305-317).
        const float sx = shots[s].x - (float)w.x0 * g.dx;
        const float sy = shots[s].y - (float)w.y0 * g.dy;
        const float sz = shots[s].z;
        if (!(sx >= 0.f) || !(sy >= 0.f) || !(sz >= 0.f))
            return fail(ctx, TOMO_ERR_INVALID_ARG, "shot " + std::to_string(s) + " outside its window");
        const int sidx = (int)(sx / g.dx), sidy = (int)(sy / g.dy), sidz = (int)(sz / g.dz);
        if (sidx >= d.wnx || sidy >= d.wny || sidz >= g.nz)
            return fail(ctx, TOMO_ERR_INVALID_ARG, "shot " + std::to_string(s) + " outside its window");
        const float ex = (float)(sidx * g.dx) - sx, ey = (float)(sidy * g.dy) - sy, ez = (float)(sidz * g.dz) - sz;
        d.src_dist = std::sqrt(std::pow(ex, 2.0f) + std::pow(ey, 2.0f) + std::pow(ez, 2.0f));
        d.src_brick = (sidz >> 2) + d.nbz * ((sidx >> 2) + d.nbx * (sidy >> 2));
        d.src_node = (sidz & 3) + 4 * (sidx & 3) + 16 * (sidy & 3);
        const long long nb = (long long)d.nbx * d.nby * d.nbz;
        d.t_off = bt.t_total;
        d.qbase = bt.q_total;
        d.v_off = bt.v_total;
        tomo::set_brick8(d);
        d.qbase8 = bt.q_total8;
        bt.q_total8 += (unsigned long long)d.gbz8 * d.gbx8 * d.gby8;
        d.s_gather = aligned ? 0 : 1;
        bt.gather = bt.gather || !aligned;
        bt.t_total += nb * tomo::kBrickNodes;
        bt.q_total += (unsigned long long)nb;
        bt.v_total += (long long)g.nz * d.wnx * d.wny;
        if (nb > max_bricks) max_bricks = (int)nb;
    }
    bt.local_bits = 1;
    while ((1ll << bt.local_bits) < max_bricks) bt.local_bits++;
    if (bt.local_bits + 1 >= 32 || ((unsigned long long)nshots << bt.local_bits) >= (1ull << 32))
        return fail(ctx, TOMO_ERR_CAPACITY, "too many shots x bricks for one batch; split the batch");
    for (ShotDesc &d : bt.sd) tomo::set_brick_division(d, bt.local_bits);
    for (int r = 0; r < nrec; r++) {
        const tomo_point &p = receivers[r];
        if (!(p.x >= 0.f) || !(p.y >= 0.f) || !(p.z >= 0.f) || p.x > (g.nx - 1) * g.dx || p.y > (g.ny - 1) * g.dy ||
            p.z > (g.nz - 1) * g.dz)
            return fail(ctx, TOMO_ERR_INVALID_ARG, "receiver " + std::to_string(r) + " outside the model");
    }
    return TOMO_OK;
}

// Device buffers of a batch; uploads the descriptors and receiver positions.
int upload_batch(tomo_ctx *ctx, const Batch &bt, int nrec, const tomo_point *receivers)
{
    const int nshots = (int)bt.sd.size();
    CK(ctx->T.ensure((size_t)bt.t_total));
    CK(ctx->qflag.ensure((size_t)bt.q_total));
    CK(ctx->qflag8.ensure((size_t)bt.q_total8));
    CK(ctx->lists.ensure((size_t)bt.q_total * 3));
    // Receivers and shot descriptors equal to what the device buffers already hold (the same
    // survey solved again, as in every iteration of an inversion) are not uploaded again: a
    // copy from pageable memory also waits for the stream's earlier work.  A buffer that is
    // (re)allocated here holds nothing yet.
    if (ctx->shots_d.cap < (size_t)nshots) ctx->sd_up.clear();
    CK(ctx->shots_d.ensure((size_t)nshots));
    if (nrec > 0) {
        if (ctx->rec.cap < (size_t)nrec * 3) ctx->rec_up.clear();
        CK(ctx->rec.ensure((size_t)nrec * 3));
        CK(ctx->t_recv.ensure((size_t)nshots * nrec));
        std::vector<float> rh((size_t)nrec * 3);
        for (int r = 0; r < nrec; r++) {
            rh[(size_t)r] = receivers[r].x;
            rh[(size_t)nrec + r] = receivers[r].y;
            rh[(size_t)2 * nrec + r] = receivers[r].z;
        }
        if (rh != ctx->rec_up) {
            ctx->rec_up.clear();
            CK(cudaMemcpyAsync(ctx->rec.ptr, rh.data(), rh.size() * sizeof(float), cudaMemcpyHostToDevice,
                               ctx->stream));
            ctx->rec_up = std::move(rh);
        }
    }
    const size_t sd_bytes = bt.sd.size() * sizeof(ShotDesc);
    if (ctx->sd_up.size() != bt.sd.size() || std::memcmp(ctx->sd_up.data(), bt.sd.data(), sd_bytes) != 0) {
        ctx->sd_up.clear();
        CK(cudaMemcpyAsync(ctx->shots_d.ptr, bt.sd.data(), sd_bytes, cudaMemcpyHostToDevice, ctx->stream));
        ctx->sd_up = bt.sd;
    }
    return TOMO_OK;
}

tomo::FimLaunch fim_params(tomo_ctx *ctx, const Batch &bt, const SolveCfg &c, int nrec)
{
    const tomo_grid &g = ctx->g;
    tomo::FimLaunch p{};
    p.S = ctx->S.ptr;
    p.T = ctx->T.ptr;
    p.shots = ctx->shots_d.ptr;
    p.nshots = (int)bt.sd.size();
    p.gather = bt.gather ? 1 : 0;
    p.pair = c.pair && !c.brick8 ? 1 : 0;
    p.qflag = c.brick8 ? ctx->qflag8.ptr : ctx->qflag.ptr;
    p.lists = ctx->lists.ptr;
    p.list_cap = (unsigned)(c.brick8 ? bt.q_total8 : bt.q_total);
    p.ctrl = ctx->ctrl.ptr;
    p.stats = ctx->stats.ptr;
    p.gbx = ctx->gbx;
    p.gbz = ctx->gbz;
    p.h = g.dx;  // isotropic spacing h = dx (block_FIM.cpp:173)
    p.max_inner = c.max_inner;
    p.change_tol = c.change_tol;
    p.inner_tol = c.inner_tol;
    p.max_rounds = c.max_rounds;
    p.local_bits = bt.local_bits;
    p.spin_limit = c.spin_limit;
    p.nrec = nrec;
    p.rx = nrec ? ctx->rec.ptr : nullptr;
    p.ry = nrec ? ctx->rec.ptr + nrec : nullptr;
    p.rz = nrec ? ctx->rec.ptr + 2 * nrec : nullptr;
    p.t_recv = nrec ? ctx->t_recv.ptr : nullptr;
    p.dx = g.dx;
    p.dy = g.dy;
    p.dz = g.dz;
    p.nz = g.nz;
    if (c.time_band > 0.f) {  // buffers sized by band_buffers()
        p.band = c.time_band;
        p.keys = ctx->fim_keys.ptr;
        p.band_min = ctx->band_min.ptr;
        p.park = ctx->band_park.ptr;
        p.park_cnt = ctx->band_pcnt.ptr;
        p.park_rounds = kParkRounds;
    }
    return p;
}

// Key and per-shot minimum arrays of the time-band ordering, when the solve uses it.
int band_buffers(tomo_ctx *ctx, const Batch &bt, const SolveCfg &c)
{
    if (c.time_band <= 0.f) return TOMO_OK;
    CK(ctx->fim_keys.ensure((size_t)bt.q_total));
    CK(ctx->band_min.ensure((size_t)3 * bt.sd.size()));
    CK(ctx->band_park.ensure((size_t)(kParkRounds + 2) * bt.q_total));
    CK(ctx->band_pcnt.ensure(16));
    return TOMO_OK;
}

// Every key "none" and every per-shot minimum "none" before a banded solve.
cudaError_t band_reset(tomo_ctx *ctx, const tomo::FimLaunch &p)
{
    if (p.band <= 0.f) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(p.keys, 0xff, (size_t)p.list_cap * sizeof(unsigned), ctx->stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(p.park_cnt, 0, (size_t)(p.park_rounds + 2) * sizeof(unsigned), ctx->stream);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(p.band_min, 0xff, (size_t)3 * p.nshots * sizeof(unsigned), ctx->stream);
}

// Enqueues the pool reset, the source seeds and the persistent JW solve of a batch (4^3 or
// 8^3 bricks, rounds or asynchronous schedule); ev_solve (may be null) is recorded just
// before the persistent launch.
int enqueue_fim(tomo_ctx *ctx, const tomo::FimLaunch &p, size_t t_total, size_t q_total, const SolveCfg &c,
                cudaEvent_t ev_solve)
{
    int grid = 0;
    if (c.brick8) {
        CK(tomo::fim_init(p.T, t_total, p.qflag, (size_t)p.list_cap, p.ctrl, p.stats, ctx->stream));
        CK(tomo::fim_seed8(p.shots, p.nshots, p.S, p.gbx, p.gbz, p.T, p.qflag, p.lists, p.local_bits, p.ctrl,
                           ctx->stream));
        if (ev_solve) CK(cudaEventRecord(ev_solve, ctx->stream));
        CK(tomo::fim_solve8(p, c.occupancy, c.ieee_sqrt, &grid, ctx->stream));
        return TOMO_OK;
    }
    CK(tomo::fim_init(p.T, t_total, p.qflag, q_total, p.ctrl, p.stats, ctx->stream));
    CK(tomo::fim_seed(p.shots, p.nshots, p.S, p.gbx, p.gbz, p.T, p.qflag, p.lists, p.local_bits, p.ctrl,
                      ctx->stream, c.async ? 3 * (size_t)p.list_cap : 0));
    CK(band_reset(ctx, p));
    if (ev_solve) CK(cudaEventRecord(ev_solve, ctx->stream));
    CK(tomo::fim_solve(p, c.block_warps, c.occupancy, c.ieee_sqrt, &grid, ctx->stream, c.async));
    return TOMO_OK;
}

// Reads the control words and counters of the last persistent solve (synchronises).
int read_solve(tomo_ctx *ctx, unsigned &rounds, unsigned long long &act, unsigned long long &inner,
               const SolveCfg &c, unsigned long long *idle = nullptr, unsigned long long *deferred = nullptr)
{
    CK(cudaMemcpyAsync(ctx->pinned_ctrl, ctx->ctrl.ptr, tomo::kCtrlWords * sizeof(unsigned), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaMemcpyAsync(ctx->pinned_ctrl + tomo::kCtrlWords, ctx->stats.ptr, 4 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long st[4];
    std::memcpy(st, ctx->pinned_ctrl + tomo::kCtrlWords, sizeof(st));
    rounds = ctx->pinned_ctrl[tomo::kRounds];
    act = st[0];
    inner = st[1];
    if (idle) *idle = st[3];
    if (deferred) *deferred = st[2];
    const unsigned derr = ctx->pinned_ctrl[tomo::kErr];
    if (derr == tomo::kDevRoundCap)
        return fail(ctx, TOMO_ERR_NOT_CONVERGED,
                    "eikonal solve hit the round cap (" + std::to_string(c.max_rounds) + ")");
    if (derr != tomo::kDevOk) return fail(ctx, TOMO_ERR_TIMEOUT, "eikonal solve: device barrier wait timed out");
    return TOMO_OK;
}

void keep_batch(tomo_ctx *ctx, const Batch &bt, const tomo_point *shots, int nrec, const tomo_point *receivers)
{
    ctx->shots_h = bt.sd;
    ctx->shot_pos.assign(shots, shots + bt.sd.size());
    ctx->rec_h.assign(receivers, receivers + nrec);
    ctx->nshots = (int)bt.sd.size();
    ctx->nrec = nrec;
}

}  // namespace

namespace tomo {

int eik_plan(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
             const tomo_point *receivers, const tomo_eik_opts *opts, EikPlan &plan)
{
    if (nshots < 1 || !shots) return fail(ctx, TOMO_ERR_INVALID_ARG, "nshots must be >= 1 with shot positions");
    if (nrec < 0 || (nrec > 0 && !receivers)) return fail(ctx, TOMO_ERR_INVALID_ARG, "bad receivers");
    if (!ctx->have_model) return fail(ctx, TOMO_ERR_STATE, "no model set (tomo_set_velocity / tomo_set_slowness)");
    if (opts && opts->op != TOMO_OP_JW) return fail(ctx, TOMO_ERR_INVALID_ARG, "the plan runs the JW operator only");
    if (opts && !(std::fabs(opts->time_band) < 1e30f))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "time_band must be finite");
    const SolveCfg cfg = solve_cfg(ctx, opts);
    Batch bt;
    int rc = make_batch(ctx, nshots, shots, windows, nrec, receivers, bt);
    if (rc != TOMO_OK) return rc;
    rc = upload_batch(ctx, bt, nrec, receivers);
    if (rc != TOMO_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));  // host staging of upload_batch
    keep_batch(ctx, bt, shots, nrec, receivers);
    rc = band_buffers(ctx, bt, cfg);
    if (rc != TOMO_OK) return rc;
    plan.p = fim_params(ctx, bt, cfg, nrec);
    plan.block_warps = cfg.block_warps;
    plan.occupancy = cfg.occupancy;
    plan.ieee_sqrt = cfg.ieee_sqrt;
    plan.async = cfg.async;
    plan.brick8 = cfg.brick8;
    plan.t_total = (size_t)bt.t_total;
    plan.q_total = (size_t)bt.q_total;
    return TOMO_OK;
}

int eik_enqueue(tomo_ctx *ctx, const EikPlan &plan)
{
    SolveCfg c{};
    c.block_warps = plan.block_warps;
    c.occupancy = plan.occupancy;
    c.ieee_sqrt = plan.ieee_sqrt;
    c.async = plan.async;
    c.brick8 = plan.brick8;
    return enqueue_fim(ctx, plan.p, plan.t_total, plan.q_total, c, nullptr);
}

}  // namespace tomo

extern "C" {

int tomo_eik_solve(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
                   const tomo_point *receivers, float *t_recv, const tomo_eik_opts *opts,
                   tomo_eik_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (nshots < 1 || !shots) return fail(ctx, TOMO_ERR_INVALID_ARG, "nshots must be >= 1 with shot positions");
    if (nrec < 0 || (nrec > 0 && !receivers)) return fail(ctx, TOMO_ERR_INVALID_ARG, "bad receivers");
    if (!ctx->have_model) return fail(ctx, TOMO_ERR_STATE, "no model set (tomo_set_velocity / tomo_set_slowness)");
    if (opts && opts->op != TOMO_OP_JW && opts->op != TOMO_OP_NGB)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "unknown eikonal operator");
    if (opts && (opts->brick < 0 || opts->brick > TOMO_BRICK_8))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "unknown brick shape (TOMO_BRICK_4 or TOMO_BRICK_8)");
    if (opts && opts->brick == TOMO_BRICK_8 && opts->schedule == TOMO_SCHED_ASYNC)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "8x8x8 bricks run the rounds schedule only");
    if (opts && (opts->schedule < TOMO_SCHED_DEFAULT || opts->schedule > TOMO_SCHED_PAIR))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "unknown work schedule");
    if (opts && !(std::fabs(opts->time_band) < 1e30f))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "time_band must be finite");
    const SolveCfg cfg = solve_cfg(ctx, opts);
    CK(cudaSetDevice(ctx->device));
    Batch bt;
    int rc = make_batch(ctx, nshots, shots, windows, nrec, receivers, bt);
    if (rc != TOMO_OK) return rc;
    ctx->have_solve = false;  // the pool is about to be overwritten
    rc = upload_batch(ctx, bt, nrec, receivers);
    if (rc != TOMO_OK) return rc;
    rc = band_buffers(ctx, bt, cfg);
    if (rc != TOMO_OK) return rc;

    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    if (opts && opts->op == TOMO_OP_NGB) {
        rc = launch_ngb(ctx, bt.sd, shots, nshots, nrec, opts->sweep_groups, cfg.spin_limit);
        if (rc != TOMO_OK) return rc;
    } else {
        const tomo::FimLaunch p = fim_params(ctx, bt, cfg, nrec);
        rc = enqueue_fim(ctx, p, (size_t)bt.t_total, (size_t)bt.q_total, cfg, ctx->ev[3]);
        if (rc != TOMO_OK) return rc;
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    if (t_recv && nrec > 0)
        CK(cudaMemcpyAsync(t_recv, ctx->t_recv.ptr, (size_t)nshots * nrec * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    unsigned rounds = 0;
    unsigned long long act = 0, inner = 0, idle = 0, deferred = 0;
    rc = read_solve(ctx, rounds, act, inner, cfg, &idle, &deferred);
    keep_batch(ctx, bt, shots, nrec, receivers);
    ctx->have_solve = (rc == TOMO_OK);
    if (stats) {
        stats->rounds = rounds;
        stats->activations = (long long)act;
        stats->inner_iterations = (long long)inner;
        stats->idle_activations = (long long)idle;
        stats->deferred = (long long)deferred;
        stats->nodes_per_brick = cfg.brick8 ? 8 * tomo::kBrickNodes : tomo::kBrickNodes;
        cudaEventElapsedTime(&stats->setup_ms, ctx->ev[0], ctx->ev[3]);
        cudaEventElapsedTime(&stats->solve_ms, ctx->ev[3], ctx->ev[1]);
        cudaEventElapsedTime(&stats->total_ms, ctx->ev[0], ctx->ev[2]);
    }
    return rc;
}

int tomo_eik_solve_seeded(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
                          const tomo_point *receivers, float *t_recv, const float *ceiling, float inflate,
                          const tomo_eik_opts *opts, tomo_eik_stats *stats, tomo_seed_stats *seed_stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (nshots < 1 || !shots) return fail(ctx, TOMO_ERR_INVALID_ARG, "nshots must be >= 1 with shot positions");
    if (nshots > 65535) return fail(ctx, TOMO_ERR_CAPACITY, "a warm-started batch holds at most 65535 shots");
    if (nrec < 0 || (nrec > 0 && !receivers)) return fail(ctx, TOMO_ERR_INVALID_ARG, "bad receivers");
    if (!ceiling) return fail(ctx, TOMO_ERR_INVALID_ARG, "ceiling must be a device array");
    if (!(inflate >= 0.f) || !(inflate < 1.f)) return fail(ctx, TOMO_ERR_INVALID_ARG, "inflate must be in [0, 1)");
    if (!ctx->have_model) return fail(ctx, TOMO_ERR_STATE, "no model set (tomo_set_velocity / tomo_set_slowness)");
    if (opts && opts->op != TOMO_OP_JW)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "the warm-started solve runs the JW operator only");
    SolveCfg cfg = solve_cfg(ctx, opts);
    cfg.time_band = 0.f;  // keys start from the ceiling's pool: not used here
    cfg.brick8 = false;   // the warm-started solve and its fallback run 4^3 bricks
    CK(cudaSetDevice(ctx->device));
    Batch bt;
    int rc = make_batch(ctx, nshots, shots, windows, nrec, receivers, bt);
    if (rc != TOMO_OK) return rc;
    ctx->have_solve = false;  // the pool is about to be overwritten
    rc = upload_batch(ctx, bt, nrec, receivers);
    if (rc != TOMO_OK) return rc;
    CK(ctx->viol.ensure((size_t)nshots * 3));
    cudaEvent_t *ev = ctx->ev;

    // 1. pool from the ceiling, source seed, persistent solve (receivers after the check)
    CK(cudaEventRecord(ev[0], ctx->stream));
    CK(tomo::fim_init(ctx->T.ptr, (size_t)bt.t_total, ctx->qflag.ptr, (size_t)bt.q_total, ctx->ctrl.ptr,
                      ctx->stats.ptr, ctx->stream));
    CK(tomo::fim_ceiling(ctx->T.ptr, ctx->shots_d.ptr, nshots, ctx->g.nz, ceiling, 1.0f + inflate, ctx->stream));
    CK(tomo::fim_seed(ctx->shots_d.ptr, nshots, ctx->S.ptr, ctx->gbx, ctx->gbz, ctx->T.ptr, ctx->qflag.ptr,
                      ctx->lists.ptr, bt.local_bits, ctx->ctrl.ptr, ctx->stream, cfg.async ? 3 * (size_t)bt.q_total : 0));
    CK(cudaEventRecord(ev[3], ctx->stream));
    tomo::FimLaunch p = fim_params(ctx, bt, cfg, 0);
    int grid = 0;
    CK(tomo::fim_solve(p, cfg.block_warps, cfg.occupancy, cfg.ieee_sqrt, &grid, ctx->stream, cfg.async));
    CK(cudaEventRecord(ev[4], ctx->stream));
    // 2. check: a node below what its neighbours give came from a ceiling below the truth
    CK(cudaMemsetAsync(ctx->viol.ptr, 0, (size_t)nshots * 3 * sizeof(unsigned long long), ctx->stream));
    CK(tomo::fim_verify(ctx->T.ptr, ctx->S.ptr, ctx->shots_d.ptr, nshots, ctx->gbx, ctx->gbz, ctx->g.dx,
                        kVerifyRelTol, ceiling, 1.0f + inflate, ctx->g.nz, cfg.ieee_sqrt, ctx->viol.ptr,
                        ctx->stream));
    CK(cudaEventRecord(ev[5], ctx->stream));
    std::vector<unsigned long long> viol((size_t)nshots * 3);
    CK(cudaMemcpyAsync(viol.data(), ctx->viol.ptr, viol.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       ctx->stream));
    unsigned rounds = 0, rounds2 = 0;
    unsigned long long act = 0, inner = 0, act2 = 0, inner2 = 0;
    rc = read_solve(ctx, rounds, act, inner, cfg);
    if (rc != TOMO_OK) return rc;

    // 3. fallback: shots with violations are solved again from INF (plain FIM)
    std::vector<ShotDesc> redo;
    long long nviol = 0, nstuck = 0;
    float worst = 0.f;
    for (int s = 0; s < nshots; s++) {
        const unsigned long long deficit = viol[(size_t)s], stuck = viol[(size_t)2 * nshots + s];
        nviol += (long long)deficit;
        nstuck += (long long)stuck;
        float w;
        const unsigned bits = (unsigned)viol[(size_t)nshots + s];
        std::memcpy(&w, &bits, sizeof(w));
        worst = std::max(worst, w);
        if (deficit || stuck) redo.push_back(bt.sd[(size_t)s]);
    }
    const int nredo = (int)redo.size();
    CK(cudaEventRecord(ev[6], ctx->stream));
    if (nredo > 0) {
        CK(ctx->shots_redo.ensure((size_t)nredo));
        CK(cudaMemcpyAsync(ctx->shots_redo.ptr, redo.data(), redo.size() * sizeof(ShotDesc), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(tomo::fim_reset_shots(ctx->T.ptr, ctx->qflag.ptr, ctx->shots_redo.ptr, nredo, ctx->stream));
        CK(tomo::fim_init(nullptr, 0, nullptr, 0, ctx->ctrl.ptr, ctx->stats.ptr, ctx->stream));
        CK(tomo::fim_seed(ctx->shots_redo.ptr, nredo, ctx->S.ptr, ctx->gbx, ctx->gbz, ctx->T.ptr, ctx->qflag.ptr,
                          ctx->lists.ptr, bt.local_bits, ctx->ctrl.ptr, ctx->stream, cfg.async ? 3 * (size_t)bt.q_total : 0));
        tomo::FimLaunch p2 = p;
        p2.shots = ctx->shots_redo.ptr;
        p2.nshots = nredo;
        CK(tomo::fim_solve(p2, cfg.block_warps, cfg.occupancy, cfg.ieee_sqrt, &grid, ctx->stream, cfg.async));
        rc = read_solve(ctx, rounds2, act2, inner2, cfg);
        if (rc != TOMO_OK) return rc;
    }
    CK(cudaEventRecord(ev[7], ctx->stream));
    if (nrec > 0)
        CK(tomo::receivers_sample(ctx->T.ptr, ctx->shots_d.ptr, nshots, ctx->rec.ptr, ctx->rec.ptr + nrec,
                                  ctx->rec.ptr + 2 * nrec, nrec, ctx->g.dx, ctx->g.dy, ctx->g.dz, ctx->g.nz,
                                  ctx->t_recv.ptr, ctx->stream));
    CK(cudaEventRecord(ev[1], ctx->stream));
    if (t_recv && nrec > 0)
        CK(cudaMemcpyAsync(t_recv, ctx->t_recv.ptr, (size_t)nshots * nrec * sizeof(float), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaEventRecord(ev[2], ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    keep_batch(ctx, bt, shots, nrec, receivers);
    ctx->have_solve = true;
    if (stats) {
        stats->rounds = (long long)rounds + rounds2;
        stats->activations = (long long)(act + act2);
        stats->inner_iterations = (long long)(inner + inner2);
        stats->idle_activations = 0;
        stats->deferred = 0;
        stats->nodes_per_brick = tomo::kBrickNodes;
        cudaEventElapsedTime(&stats->setup_ms, ev[0], ev[3]);
        cudaEventElapsedTime(&stats->solve_ms, ev[3], ev[1]);
        cudaEventElapsedTime(&stats->total_ms, ev[0], ev[2]);
    }
    if (seed_stats) {
        seed_stats->violations = nviol;
        seed_stats->stuck = nstuck;
        seed_stats->max_deficit = worst;
        seed_stats->shots_fallback = nredo;
        seed_stats->rounds_seeded = rounds;
        seed_stats->activations_seeded = (long long)act;
        seed_stats->inner_iterations_seeded = (long long)inner;
        cudaEventElapsedTime(&seed_stats->seeded_ms, ev[3], ev[4]);
        cudaEventElapsedTime(&seed_stats->verify_ms, ev[4], ev[5]);
        cudaEventElapsedTime(&seed_stats->fallback_ms, ev[6], ev[7]);
    }
    return TOMO_OK;
}

int tomo_eik_autotune(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int repeats,
                      tomo_eik_opts *best, tomo_tune_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (repeats < 0) return fail(ctx, TOMO_ERR_INVALID_ARG, "repeats must be >= 0");
    if (repeats == 0) repeats = 2;
    // untuned defaults while timing (an earlier tuning must not leak into the trials)
    ctx->tuned_block_warps = ctx->tuned_occupancy = ctx->tuned_max_inner = 0;
    ctx->tuned_brick = 0;
    ctx->tuned_schedule = 0;
    ctx->tuned_time_band = 0.f;
    const int warps[] = {kDefaultBlockWarps, 8, 4};
    const int occs[] = {4, 5, 6, 3};
    const int inners[] = {16, 8, 32};
    tomo_eik_opts o{};
    o.op = TOMO_OP_JW;
    o.brick = TOMO_BRICK_4;
    tomo_eik_stats st{};
    // warm-up (first launch of each kernel variant pays for module loading)
    int rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &o, &st);
    if (rc != TOMO_OK) return rc;
    float best_ms = 0.f, default_ms = 0.f;
    int trials = 0, bw = kDefaultBlockWarps, bo = kDefaultOccupancy, bi = kDefaultMaxInner;
    for (int w : warps)
        for (int oc : occs)
            for (int in : inners) {
                o.block_warps = w;
                o.occupancy = oc;
                o.max_inner = in;
                float ms = 0.f;
                for (int r = 0; r < repeats + 1; r++) {
                    rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &o, &st);
                    if (rc != TOMO_OK) return rc;
                    if (r == 0) continue;  // first launch of this variant: not timed
                    ms = (r == 1) ? st.solve_ms : std::min(ms, st.solve_ms);
                }
                if (trials == 0) default_ms = ms;
                if (trials == 0 || ms < best_ms) {
                    best_ms = ms;
                    bw = w;
                    bo = oc;
                    bi = in;
                }
                ++trials;
            }
    // Two bricks per warp (TOMO_SCHED_PAIR): warps per CTA {8, 4, 16} x CTAs per SM {3, 4}
    // (register budgets 80/64), at the chosen in-brick cap.  Config 2: 8 x 3, 5.02 ms against
    // 5.27 for the one-brick kernel's best shape.
    bool pair_best = false;
    int pw = 0, po = 0;
    {
        tomo_eik_opts op{};
        op.op = TOMO_OP_JW;
        op.brick = TOMO_BRICK_4;
        op.schedule = TOMO_SCHED_PAIR;
        op.max_inner = bi;
        for (int w : {8, 4, 16})
            for (int oc : {3, 4}) {
                op.block_warps = w;
                op.occupancy = oc;
                float ms = 0.f;
                for (int r = 0; r < repeats + 1; r++) {
                    rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &op, &st);
                    if (rc != TOMO_OK) return rc;
                    if (r == 0) continue;
                    ms = (r == 1) ? st.solve_ms : std::min(ms, st.solve_ms);
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    pair_best = true;
                    pw = w;
                    po = oc;
                }
                ++trials;
            }
    }
    // 8^3 bricks: one CTA of 8 warps per brick, CTAs per SM {2, 3, 4, 5} (register
    // budgets 128/80/64/48), in-brick cap {16, 32}.
    int bbrick = TOMO_BRICK_4, bo8 = 0, bi8 = 0;
    float best8 = 0.f;
    {
        tomo_eik_opts o8{};
        o8.op = TOMO_OP_JW;
        o8.brick = TOMO_BRICK_8;
        for (int oc : {4, 3, 5, 2})
            for (int in : {16, 32}) {
                o8.occupancy = oc;
                o8.max_inner = in;
                float ms = 0.f;
                for (int r = 0; r < repeats + 1; r++) {
                    rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &o8, &st);
                    if (rc != TOMO_OK) return rc;
                    if (r == 0) continue;
                    ms = (r == 1) ? st.solve_ms : std::min(ms, st.solve_ms);
                }
                if (bo8 == 0 || ms < best8) {
                    best8 = ms;
                    bo8 = oc;
                    bi8 = in;
                }
                ++trials;
            }
    }
    // Then the time band at the chosen 4^3 shape: multiples of the slowest brick crossing,
    // 4 h s_max (the band is model-relative; no band is the shape loop's own time).
    o.block_warps = bw;
    o.occupancy = bo;
    o.max_inner = bi;
    float bb = 0.f;
    {
        CK(ctx->tune_word.ensure(1));
        CK(tomo::max_positive(ctx->slow.ptr, (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz, ctx->tune_word.ptr,
                              ctx->stream));
        unsigned bits = 0;
        CK(cudaMemcpyAsync(&bits, ctx->tune_word.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        float smax = 0.f;
        std::memcpy(&smax, &bits, sizeof(smax));
        const float crossing = (float)tomo::kBrick * ctx->g.dx * smax;
        for (float mult : {3.f, 6.f, 9.f, 12.f}) {
            if (!(crossing > 0.f)) break;
            o.time_band = mult * crossing;
            float ms = 0.f;
            for (int r = 0; r < repeats + 1; r++) {
                rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &o, &st);
                if (rc != TOMO_OK) return rc;
                if (r == 0) continue;
                ms = (r == 1) ? st.solve_ms : std::min(ms, st.solve_ms);
            }
            if (ms < best_ms) {
                best_ms = ms;
                bb = o.time_band;
                pair_best = false;  // a banded solve runs the one-brick kernel
            }
            ++trials;
        }
    }
    // With a band, the launch shapes again (the banded kernel holds more live state, so
    // its best shape can differ: 3 x 8 warps on the config-5 starting model).
    if (bb > 0.f) {
        o.time_band = bb;
        o.max_inner = bi;
        for (int w : warps)
            for (int oc : occs) {
                o.block_warps = w;
                o.occupancy = oc;
                float ms = 0.f;
                for (int r = 0; r < repeats + 1; r++) {
                    rc = tomo_eik_solve(ctx, nshots, shots, windows, 0, nullptr, nullptr, &o, &st);
                    if (rc != TOMO_OK) return rc;
                    if (r == 0) continue;
                    ms = (r == 1) ? st.solve_ms : std::min(ms, st.solve_ms);
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    bw = w;
                    bo = oc;
                }
                ++trials;
            }
    }
    if (best8 < best_ms) {  // the 8^3 shape beats every 4^3 one (with or without a band)
        bbrick = TOMO_BRICK_8;
        best_ms = best8;
        bo = bo8;
        bi = bi8;
        bb = 0.f;
        pair_best = false;
    }
    if (pair_best) {
        bw = pw;
        bo = po;
    }
    ctx->tuned_brick = bbrick;
    ctx->tuned_schedule = pair_best ? TOMO_SCHED_PAIR : 0;
    ctx->tuned_block_warps = bw;
    ctx->tuned_occupancy = bo;
    ctx->tuned_max_inner = bi;
    ctx->tuned_time_band = bb;
    if (best) {
        *best = tomo_eik_opts{};
        best->op = TOMO_OP_JW;
        best->brick = bbrick;
        best->block_warps = bw;
        best->occupancy = bo;
        best->max_inner = bi;
        best->time_band = bb;
        best->schedule = pair_best ? TOMO_SCHED_PAIR : TOMO_SCHED_DEFAULT;
    }
    if (stats) {
        stats->trials = trials;
        stats->best_ms = best_ms;
        stats->default_ms = default_ms;
    }
    return TOMO_OK;
}

int tomo_eik_volumes(tomo_ctx *ctx, float *dst)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!dst) return fail(ctx, TOMO_ERR_INVALID_ARG, "output is NULL");
    if (!ctx->have_solve) return fail(ctx, TOMO_ERR_STATE, "no eikonal solve");
    CK(cudaSetDevice(ctx->device));
    CK(tomo::fim_unbrick_all(ctx->T.ptr, ctx->shots_d.ptr, ctx->nshots, ctx->g.nz, dst, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_eik_window(tomo_ctx *ctx, int shot, tomo_window *out)
{
    if (!ctx || !out) return TOMO_ERR_INVALID_ARG;
    if (!ctx->have_solve) return fail(ctx, TOMO_ERR_STATE, "no eikonal solve");
    if (shot < 0 || shot >= ctx->nshots) return fail(ctx, TOMO_ERR_INVALID_ARG, "shot index out of range");
    const ShotDesc &d = ctx->shots_h[(size_t)shot];
    *out = tomo_window{d.wx0, d.wx0 + d.wnx, d.wy0, d.wy0 + d.wny};
    return TOMO_OK;
}

int tomo_eik_volume(tomo_ctx *ctx, int shot, float *t_out)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!t_out) return fail(ctx, TOMO_ERR_INVALID_ARG, "output is NULL");
    if (!ctx->have_solve) return fail(ctx, TOMO_ERR_STATE, "no eikonal solve");
    if (shot < 0 || shot >= ctx->nshots) return fail(ctx, TOMO_ERR_INVALID_ARG, "shot index out of range");
    CK(cudaSetDevice(ctx->device));
    const ShotDesc &d = ctx->shots_h[(size_t)shot];
    const size_t n = (size_t)ctx->g.nz * d.wnx * d.wny;
    CK(ctx->scratch_v.ensure(n));
    CK(tomo::fim_unbrick(ctx->T.ptr, ctx->shots_d.ptr, shot, ctx->g.nz, ctx->scratch_v.ptr, ctx->stream));
    CK(cudaMemcpyAsync(t_out, ctx->scratch_v.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

}  // extern "C"
