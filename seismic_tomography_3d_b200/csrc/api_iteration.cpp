// One tomography iteration in one call, replayed from CUDA graphs (include/tomo_b200.h:
// tomo_iteration).  Replaces the body of the reference's iteration loop
// (src/tomography/tomography_main.cpp:19-30: forward_modeling, import_cal_data, converged,
// optimization, model_update) with device-resident stages:
//
//   graph A  eikonal batch solve (+ receiver times) -> ray march -> row lengths (scan)
//            -> non-zero counts and the solver's status words copied to pinned memory
//   host     reads the non-zero count; grows the Jacobian's capacity if it no longer fits
//   graph B  emit rows + Tikhonov rows -> transpose (sorted over the fixed capacity)
//            -> B = [dobs - dcal; 0] -> CGLS -> dm, smoothing, slowness += dm, re-brick
//            -> CGLS status, residual norms copied to pinned memory
//
// The only data-dependent size of an iteration is the Jacobian's non-zero count, hence the
// split: graph B is captured for a capacity (first count x headroom) and replayed while the
// count fits.  Each graph records the device addresses it was captured with; a later call
// whose buffers moved (a larger batch, other options) captures again.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/tomo_b200.h"
#include "common.cuh"
#include "context.hpp"
#include "internal.hpp"

namespace {

int fail(tomo_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                                   \
    do {                                                                                                           \
        const cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess)                                                                                     \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? TOMO_ERR_OOM : TOMO_ERR_CUDA,                       \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                                       \
    } while (0)

// pinned read-back block (64-bit words)
constexpr int kPinSizes = 0;          // csr_sizes[2]
constexpr int kPinEikCtrl = 2;        // eikonal control words (kCtrlWords x u32 = 8 words)
constexpr int kPinEikStats = 10;      // activations, inner iterations
constexpr int kPinCgCtrl = 12;        // CGLS control words (8 words)
constexpr int kPinNorm2 = 20;         // ||dobs - dcal||^2
constexpr int kPinRnorm = 21;         // ||B - A x|| after the last CGLS iteration
constexpr int kPinWords = 32;

template <typename T>
void push(std::vector<char> &key, const T &v)
{
    const char *p = reinterpret_cast<const char *>(&v);
    key.insert(key.end(), p, p + sizeof(T));
}

// Runs `enqueue` either plainly or under stream capture into *exec.  On a capture failure
// the stream leaves capture mode and the work is NOT run (the caller falls back).
template <class F>
int capture(tomo_ctx *ctx, cudaGraphExec_t *exec, F enqueue)
{
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(ctx, TOMO_ERR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
    const int rc = enqueue();
    e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != TOMO_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        return rc != TOMO_OK ? rc : fail(ctx, TOMO_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *exec = nullptr;
        (void)cudaGetLastError();
        return fail(ctx, TOMO_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    return TOMO_OK;
}

}  // namespace

extern "C" void tomo_release_iteration(tomo_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->iter.a) cudaGraphExecDestroy(ctx->iter.a);
    if (ctx->iter.b) cudaGraphExecDestroy(ctx->iter.b);
    if (ctx->iter.pinned) cudaFreeHost(ctx->iter.pinned);
    ctx->iter = tomo::IterGraphs{};
}

extern "C" int tomo_iteration(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows,
                              int nrec, const tomo_point *receivers, const tomo_iteration_opts *opts,
                              tomo_iteration_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!opts) return fail(ctx, TOMO_ERR_INVALID_ARG, "options are required (inversion grid, CGLS iterations)");
    if (nrec < 1) return fail(ctx, TOMO_ERR_INVALID_ARG, "an iteration needs receivers");
    if (opts->cg_iterations < 1) return fail(ctx, TOMO_ERR_INVALID_ARG, "cg_iterations must be >= 1");
    if (!ctx->have_dobs || (long long)ctx->n_dobs != (long long)nshots * nrec)
        return fail(ctx, TOMO_ERR_STATE, "observed data (tomo_set_observed) must hold nshots x nrec picks");
    const float headroom = opts->nnz_headroom >= 1.0f ? opts->nnz_headroom : 1.25f;
    const int nit = opts->cg_iterations;
    tomo::IterGraphs &G = ctx->iter;
    CK(cudaSetDevice(ctx->device));

    // ---- plans and allocations (outside any capture) -----------------------------------
    tomo::EikPlan plan{};
    int rc = tomo::eik_plan(ctx, nshots, shots, windows, nrec, receivers, &opts->eik, plan);
    if (rc != TOMO_OK) return rc;
    ctx->have_solve = true;  // the march below follows the solve on the stream
    tomo::JacGeom jg{};
    rc = tomo::jac_prepare(ctx, &opts->jacobian, jg);
    if (rc == TOMO_OK) {
        ctx->n_rows = (int)jg.N;
        ctx->n_model = (int)jg.M;
        ctx->n_data = (int)jg.nrays;
        ctx->nxt = jg.nxt;
        ctx->nyt = jg.nyt;
        ctx->nzt = jg.nzt;
        ctx->dxt = jg.dx;
        ctx->dyt = jg.dy;
        ctx->dzt = jg.dz;
        rc = tomo::cgls_prepare(ctx, nit);
    }
    if (rc == TOMO_OK) rc = tomo::update_prepare(ctx, &opts->update);
    if (rc != TOMO_OK) {
        ctx->have_solve = false;
        return rc;
    }
    if (!G.pinned) CK(cudaMallocHost(reinterpret_cast<void **>(&G.pinned), kPinWords * sizeof(unsigned long long)));
    unsigned long long *pin = G.pinned;
    const bool graphs = opts->use_graph != 0 && !G.broken;

    auto stage_a = [&]() -> int {
        int r = tomo::eik_enqueue(ctx, plan);
        if (r == TOMO_OK) r = tomo::jac_march(ctx, jg);
        if (r != TOMO_OK) return r;
        CK(cudaMemcpyAsync(pin + kPinSizes, ctx->csr_sizes.ptr, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaMemcpyAsync(pin + kPinEikCtrl, ctx->ctrl.ptr, tomo::kCtrlWords * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(pin + kPinEikStats, ctx->stats.ptr, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           ctx->stream));
        return TOMO_OK;
    };
    long long cap = G.cap;
    auto stage_b = [&]() -> int {
        int r = tomo::jac_emit(ctx, jg, cap);
        if (r == TOMO_OK) r = tomo::cgls_enqueue(ctx, nit);
        if (r == TOMO_OK) r = tomo::update_enqueue(ctx, &opts->update);
        if (r != TOMO_OK) return r;
        CK(cudaMemcpyAsync(pin + kPinCgCtrl, ctx->cg_ctrl.ptr, tomo::kCtrlWords * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(pin + kPinNorm2, ctx->norm2.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(pin + kPinRnorm, ctx->hist.ptr + (nit - 1), sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
        return TOMO_OK;
    };

    // ---- graph A ----------------------------------------------------------------------
    int captured = 0, replayed = graphs ? 1 : 0;
    std::vector<char> key_a;
    push(key_a, plan.p);
    push(key_a, plan.block_warps);
    push(key_a, plan.occupancy);
    push(key_a, plan.ieee_sqrt);
    push(key_a, plan.async);
    push(key_a, plan.t_total);
    push(key_a, plan.q_total);
    push(key_a, jg);
    for (const void *p : {(const void *)ctx->runs.ptr, (const void *)ctx->nuniq.ptr, (const void *)ctx->ray_status.ptr,
                          (const void *)ctx->ray_steps.ptr, (const void *)ctx->final_dist.ptr,
                          (const void *)ctx->spos.ptr, (const void *)ctx->a_ptr.ptr, (const void *)ctx->csr_sizes.ptr,
                          (const void *)ctx->smin.ptr, (const void *)ctx->illum.ptr, (const void *)ctx->slow.ptr,
                          (const void *)ctx->scan_temp.ptr, (const void *)ctx->reduce_temp.ptr, (const void *)pin,
                          (const void *)ctx->ray_keys.ptr, (const void *)ctx->ray_keys_out.ptr,
                          (const void *)ctx->ray_iota.ptr, (const void *)ctx->ray_order.ptr,
                          (const void *)ctx->order_temp.ptr, (const void *)ctx->t_recv.ptr, (const void *)ctx->T.ptr,
                          (const void *)ctx->qflag.ptr, (const void *)ctx->lists.ptr, (const void *)ctx->S.ptr,
                          (const void *)ctx->shots_d.ptr, (const void *)ctx->rec.ptr, (const void *)ctx->qflag8.ptr})
        push(key_a, p);
    push(key_a, plan.brick8);
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    if (graphs && (!G.a || key_a != G.key_a)) {
        if (G.a) cudaGraphExecDestroy(G.a);
        G.a = nullptr;
        G.key_a.clear();
        if (capture(ctx, &G.a, stage_a) == TOMO_OK) {
            G.key_a = key_a;
            captured = 1;
        }
    }
    if (graphs && G.a) {
        CK(cudaGraphLaunch(G.a, ctx->stream));
    } else {
        replayed = 0;
        if (graphs) G.broken = true;  // capture refused: eager from now on
        rc = stage_a();
        if (rc != TOMO_OK) return rc;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    {
        unsigned words[tomo::kCtrlWords];
        std::memcpy(words, pin + kPinEikCtrl, sizeof(words));
        if (words[tomo::kErr] == tomo::kDevRoundCap)
            return fail(ctx, TOMO_ERR_NOT_CONVERGED, "eikonal solve hit the round cap");
        if (words[tomo::kErr] != tomo::kDevOk) return fail(ctx, TOMO_ERR_TIMEOUT, "eikonal: device wait timed out");
    }
    const long long nnz_g = (long long)pin[kPinSizes], nnz = (long long)pin[kPinSizes + 1];

    // ---- capacity and graph B -----------------------------------------------------------
    if (nnz > cap || !graphs) {
        cap = graphs ? (long long)std::ceil((double)nnz * headroom) : nnz;
        rc = tomo::jac_ensure(ctx, jg, cap);
        if (rc != TOMO_OK) return rc;
        G.cap = graphs ? cap : G.cap;
    }
    std::vector<char> key_b;
    push(key_b, jg);
    push(key_b, cap);
    push(key_b, nit);
    push(key_b, opts->update);
    for (const void *p :
         {(const void *)ctx->a_ptr.ptr, (const void *)ctx->a_idx.ptr, (const void *)ctx->a_val.ptr,
          (const void *)ctx->t_ptr.ptr, (const void *)ctx->t_idx.ptr, (const void *)ctx->t_val.ptr,
          (const void *)ctx->sort_keys.ptr, (const void *)ctx->sort_keys_out.ptr, (const void *)ctx->sort_pos.ptr,
          (const void *)ctx->sort_pos_out.ptr, (const void *)ctx->rows_of.ptr, (const void *)ctx->sort_temp.ptr,
          (const void *)ctx->tk_coef.ptr, (const void *)ctx->csr_sizes.ptr, (const void *)ctx->runs.ptr,
          (const void *)ctx->nuniq.ptr, (const void *)ctx->final_dist.ptr, (const void *)ctx->spos.ptr,
          (const void *)ctx->dobs.ptr, (const void *)ctx->t_recv.ptr, (const void *)ctx->rhs.ptr,
          (const void *)ctx->x.ptr, (const void *)ctx->cg_x.ptr, (const void *)ctx->cg_s.ptr,
          (const void *)ctx->cg_r.ptr, (const void *)ctx->cg_p.ptr, (const void *)ctx->cg_q.ptr,
          (const void *)ctx->partials.ptr, (const void *)ctx->hist.ptr, (const void *)ctx->norm2.ptr,
          (const void *)ctx->cg_ctrl.ptr, (const void *)ctx->cg_long.ptr, (const void *)ctx->cg_ltemp.ptr,
          (const void *)ctx->dm.ptr, (const void *)ctx->dm_smooth.ptr,
          (const void *)ctx->gauss_kernel.ptr, (const void *)ctx->slow.ptr, (const void *)ctx->S.ptr,
          (const void *)ctx->T.ptr, (const void *)ctx->shots_d.ptr, (const void *)ctx->rec.ptr, (const void *)pin})
        push(key_b, p);
    if (graphs && (!G.b || key_b != G.key_b)) {
        if (G.b) cudaGraphExecDestroy(G.b);
        G.b = nullptr;
        G.key_b.clear();
        if (capture(ctx, &G.b, stage_b) == TOMO_OK) {
            G.key_b = key_b;
            captured = 1;
        }
    }
    if (graphs && G.b) {
        CK(cudaGraphLaunch(G.b, ctx->stream));
    } else {
        replayed = 0;
        if (graphs) G.broken = true;
        rc = stage_b();
        if (rc != TOMO_OK) return rc;
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    {
        unsigned words[tomo::kCtrlWords];
        std::memcpy(words, pin + kPinCgCtrl, sizeof(words));
        if (words[tomo::kErr] != 0) return fail(ctx, TOMO_ERR_TIMEOUT, "CGLS: device barrier wait timed out");
    }
    tomo::jac_commit(ctx, jg, nnz_g, nnz);
    ctx->have_x = true;
    if (stats) {
        double n2, rn;
        std::memcpy(&n2, pin + kPinNorm2, sizeof(double));
        std::memcpy(&rn, pin + kPinRnorm, sizeof(double));
        stats->residual = std::sqrt(n2);
        stats->cg_rnorm = rn;
        stats->nnz = nnz;
        stats->activations = (long long)pin[kPinEikStats];
        stats->replayed = replayed && !captured;
        stats->captured = captured;
        cudaEventElapsedTime(&stats->ms, ctx->ev[0], ctx->ev[1]);
    }
    return TOMO_OK;
}
