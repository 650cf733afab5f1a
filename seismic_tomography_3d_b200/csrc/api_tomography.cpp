// C ABI: ray tracing into the Jacobian, CGLS and model update (include/tomo_b200.h).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cgls.cuh"
#include "common.cuh"
#include "context.hpp"
#include "internal.hpp"
#include "ray.cuh"

namespace tomo {
int rebrick_model(tomo_ctx *ctx);  // api_eikonal.cpp
}

namespace {

constexpr unsigned long long kSpinLimit = 1ull << 26;
constexpr float kRayLengthFactor = 4.0f;  // default per-ray cap: 4 x (traveltime x v_max)

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

// Least_squares::tk_reg_matrix difference coefficients (least_squares.cpp:380-395):
// order 0 -> [1]; otherwise [-1, 1] differenced tk_order-1 more times.
std::vector<int> tk_coefficients(int order)
{
    if (order == 0) return {1};
    std::vector<int> df((size_t)order + 1, 0);
    df[0] = -1;
    df[1] = 1;
    for (int pass = 1; pass < order; pass++) {
        std::vector<int> shifted((size_t)order + 2, 0);
        for (int k = 0; k <= order; k++) shifted[(size_t)k + 1] = df[(size_t)k];
        for (int k = 0; k <= order; k++) df[(size_t)k] = shifted[(size_t)k] - df[(size_t)k];
    }
    return df;
}

// gaussian() kernel weights (src/utils/smoothing/gaussian.cpp:14-45), host FP32 in the
// reference's order so the device smoothing is bit-identical.
std::vector<float> gaussian_weights(int samples, float stdv)
{
    const int init = samples / 2;
    const int nk = samples * samples * samples;
    std::vector<float> k((size_t)nk, 0.0f);
    const float pi = 4.0f * atanf(1.0f);
    const int mid = samples / 2;
    k[(size_t)(mid + mid * samples + mid * samples * samples)] = 1.0f;
    if (stdv != 0.0f) {
        float sum = 0.0f;
        for (int y = -init; y <= init; y++)
            for (int x = -init; x <= init; x++)
                for (int z = -init; z <= init; z++) {
                    const int index = (z + init) + (x + init) * samples + (y + init) * samples * samples;
                    k[(size_t)index] =
                        1.0f / (2.0f * pi * stdv * stdv) * expf(-((x * x + y * y + z * z) / (2.0f * stdv * stdv)));
                    sum += k[(size_t)index];
                }
        for (int i = 0; i < nk; i++) k[(size_t)i] /= sum;
    }
    return k;
}

int bits_for(long long n)
{
    int b = 1;
    while ((1ll << b) < n) b++;
    return b;
}

// Transposed CSR of (ptr, idx, val) with nrows rows and ncols columns: a stable radix
// sort of the column keys keeps each column's entries in row order (deterministic).  The
// sort runs over a fixed capacity `cap` >= nnz (sizes[1], on the device), the padding keyed
// after every column, so the same launches serve any nnz up to cap.
template <class Ctx>
int transpose_ensure(Ctx *ctx, int ncols, long long cap, tomo::DevBuf<int> &t_ptr, tomo::DevBuf<int> &t_idx,
                     tomo::DevBuf<float> &t_val, tomo::DevBuf<int> &k0, tomo::DevBuf<int> &k1, tomo::DevBuf<int> &p0,
                     tomo::DevBuf<int> &p1, tomo::DevBuf<int> &rows_of, tomo::DevBuf<unsigned char> &temp,
                     cudaStream_t st)
{
    if (cap >= (1ll << 31) - 1) return fail(ctx, TOMO_ERR_CAPACITY, "Jacobian has more than 2^31 non-zeros");
    CK(k0.ensure((size_t)cap));
    CK(k1.ensure((size_t)cap));
    CK(p0.ensure((size_t)cap));
    CK(p1.ensure((size_t)cap));
    CK(rows_of.ensure((size_t)cap));
    CK(t_ptr.ensure((size_t)ncols + 1));
    CK(t_idx.ensure((size_t)cap));
    CK(t_val.ensure((size_t)cap));
    size_t tb = 0;
    CK(tomo::sort_pairs(k0.ptr, k1.ptr, p0.ptr, p1.ptr, cap, bits_for(ncols + 1), nullptr, &tb, st));
    CK(temp.ensure(tb));
    return TOMO_OK;
}

template <class Ctx>
int transpose_enqueue(Ctx *ctx, const int *ptr, const int *idx, const float *val, int nrows, int ncols,
                      const long long *sizes, long long cap, tomo::DevBuf<int> &t_ptr, tomo::DevBuf<int> &t_idx,
                      tomo::DevBuf<float> &t_val, tomo::DevBuf<int> &k0, tomo::DevBuf<int> &k1, tomo::DevBuf<int> &p0,
                      tomo::DevBuf<int> &p1, tomo::DevBuf<int> &rows_of, tomo::DevBuf<unsigned char> &temp,
                      cudaStream_t st)
{
    CK(tomo::csr_transpose_prepare(ptr, idx, nrows, cap, k0.ptr, p0.ptr, rows_of.ptr, st));
    CK(tomo::sort_tail(k0.ptr, p0.ptr, sizes, cap, ncols, st));
    size_t tb = temp.cap;
    CK(tomo::sort_pairs(k0.ptr, k1.ptr, p0.ptr, p1.ptr, cap, bits_for(ncols + 1), temp.ptr, &tb, st));
    CK(tomo::csr_transpose_finish(p1.ptr, rows_of.ptr, val, sizes, cap, ncols, k1.ptr, t_ptr.ptr, t_idx.ptr, t_val.ptr,
                                  st));
    return TOMO_OK;
}

tomo::UpdateMasks reference_masks()
{
    // least_squares.cpp:520 (dm) and :559 (slowness update)
    return tomo::UpdateMasks{11, 2, 15, 16, 15, 15, 16, 15};
}

}  // namespace

extern "C" {

void tomo_release_tomography(tomo_ctx *ctx)
{
    if (!ctx) return;
    ctx->ray_keys.release();
    ctx->ray_keys_out.release();
    ctx->ray_iota.release();
    ctx->ray_order.release();
    ctx->order_temp.release();
    ctx->scan_temp.release();
    ctx->reduce_temp.release();
    ctx->sort_temp.release();
    ctx->csr_sizes.release();
    ctx->smin.release();
    for (auto *b : {&ctx->nuniq, &ctx->ray_status, &ctx->ray_steps, &ctx->a_ptr, &ctx->a_idx, &ctx->t_ptr,
                    &ctx->t_idx, &ctx->sort_keys, &ctx->sort_keys_out, &ctx->sort_pos, &ctx->sort_pos_out,
                    &ctx->rows_of})
        b->release();
    for (auto *b : {&ctx->final_dist, &ctx->spos, &ctx->tk_coef, &ctx->illum, &ctx->a_val, &ctx->t_val, &ctx->dobs,
                    &ctx->rhs, &ctx->x, &ctx->dm, &ctx->dm_smooth,
                    &ctx->vel_out, &ctx->gauss_kernel})
        b->release();
    ctx->runs.release();
    ctx->cub_temp.release();
    ctx->partials.release();
    ctx->hist.release();
    ctx->norm2.release();
    ctx->cg_ctrl.release();
    ctx->cg_long.release();
    ctx->cg_ltemp.release();
    for (auto *b : {&ctx->cg_x, &ctx->cg_s, &ctx->cg_r, &ctx->cg_p, &ctx->cg_q}) b->release();
}

}  // extern "C"

namespace tomo {

int jac_prepare(tomo_ctx *ctx, const tomo_jacobian_opts *opts, JacGeom &jg)
{
    if (!opts || !(opts->dx > 0) || !(opts->dy > 0) || !(opts->dz > 0) || opts->tk_order < 0)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "bad inversion grid / Tikhonov options");
    if (!ctx->have_solve || ctx->nrec < 1) return fail(ctx, TOMO_ERR_STATE, "no eikonal solve with receivers");
    const tomo_grid &g = ctx->g;
    // Least_squares::set_parameters (least_squares.cpp:124-126)
    jg.nzt = (int)((g.nz - 1) * g.dz / opts->dz) + 1;
    jg.nxt = (int)((g.nx - 1) * g.dx / opts->dx) + 1;
    jg.nyt = (int)((g.ny - 1) * g.dy / opts->dy) + 1;
    jg.M = (long long)jg.nxt * jg.nyt * jg.nzt;
    jg.ord = opts->tk_order;
    if (jg.M <= jg.ord || jg.M >= (1ll << 30))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "inversion grid too small or too large");
    jg.nrays = (long long)ctx->nshots * ctx->nrec;
    jg.N = jg.nrays + jg.M - jg.ord;
    if (jg.N >= (1ll << 31) - 1) return fail(ctx, TOMO_ERR_CAPACITY, "too many rows");
    jg.tk_entries = (long long)(jg.ord + 1) * (jg.M - jg.ord);
    jg.rayStep = 0.2f * g.dz;
    const float dmax = std::fmax(g.dx, std::fmax(g.dy, g.dz));
    jg.max_steps = opts->max_ray_steps > 0 ? opts->max_ray_steps
                                           : (int)(20.0f * (g.nx + g.ny + g.nz) * dmax / jg.rayStep);
    // Default cap per ray: the reference marches until the source cell with no cap
    // (least_squares.cpp:216-280), so a ray circling a flat spot of the field never ends.
    // A ray of traveltime T is at most T x v_max long; 4x that (plus 256 steps) leaves
    // every terminating ray untouched and stops circling ones early.
    jg.ray_cap = opts->max_ray_steps <= 0;
    jg.cap_runs = opts->max_cells_per_ray > 0 ? opts->max_cells_per_ray : 1024;
    jg.illum = opts->illumination != 0;
    jg.dx = opts->dx;
    jg.dy = opts->dy;
    jg.dz = opts->dz;
    bool full = true;
    for (const auto &d : ctx->shots_h) full = full && d.wx0 == 0 && d.wy0 == 0 && d.wnx == g.nx && d.wny == g.ny;
    if (jg.illum && !full) return fail(ctx, TOMO_ERR_INVALID_ARG, "illumination needs full-model windows");

    const long long nrays = jg.nrays;
    CK(ctx->runs.ensure((size_t)nrays * jg.cap_runs));
    CK(ctx->nuniq.ensure((size_t)nrays + 1));
    CK(ctx->ray_status.ensure((size_t)nrays));
    CK(ctx->ray_steps.ensure((size_t)nrays));
    CK(ctx->final_dist.ensure((size_t)nrays));
    CK(ctx->spos.ensure((size_t)ctx->nshots * 3));
    CK(ctx->a_ptr.ensure((size_t)jg.N + 1));
    CK(ctx->csr_sizes.ensure(2));
    CK(ctx->smin.ensure(1));
    if (jg.illum) CK(ctx->illum.ensure((size_t)g.nx * g.ny * g.nz));
    std::vector<float> sp((size_t)ctx->nshots * 3);
    for (int s = 0; s < ctx->nshots; s++) {
        sp[(size_t)s] = ctx->shot_pos[(size_t)s].x;
        sp[(size_t)ctx->nshots + s] = ctx->shot_pos[(size_t)s].y;
        sp[(size_t)2 * ctx->nshots + s] = ctx->shot_pos[(size_t)s].z;
    }
    CK(cudaMemcpyAsync(ctx->spos.ptr, sp.data(), sp.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    // Tikhonov rows lambda * df (least_squares.cpp:412-417)
    const std::vector<int> df = tk_coefficients(jg.ord);
    std::vector<float> coef((size_t)jg.ord + 1);
    for (int k = 0; k <= jg.ord; k++) coef[(size_t)k] = opts->tk_param * (float)df[(size_t)k];
    CK(ctx->tk_coef.ensure(coef.size()));
    CK(cudaMemcpyAsync(ctx->tk_coef.ptr, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice,
                       ctx->stream));
    // CUB scratch of the scan and the min-reduction (sizes depend on the counts only)
    size_t tb = 0;
    CK(tomo::scan_exclusive(ctx->nuniq.ptr, ctx->a_ptr.ptr, (int)nrays + 1, nullptr, &tb, ctx->stream));
    CK(ctx->scan_temp.ensure(tb));
    tb = 0;
    CK(tomo::reduce_min(ctx->slow.ptr, nullptr, (size_t)g.nx * g.ny * g.nz, nullptr, &tb, ctx->stream));
    CK(ctx->reduce_temp.ensure(tb));
    CK(ctx->ray_keys.ensure((size_t)nrays));
    CK(ctx->ray_keys_out.ensure((size_t)nrays));
    CK(ctx->ray_iota.ensure((size_t)nrays));
    CK(ctx->ray_order.ensure((size_t)nrays));
    tb = 0;
    CK(tomo::ray_order(ctx->t_recv.ptr, ctx->ray_keys.ptr, ctx->ray_keys_out.ptr, ctx->ray_iota.ptr,
                       ctx->ray_order.ptr, (int)nrays, ctx->nrec, nullptr, &tb, ctx->stream));
    CK(ctx->order_temp.ensure(tb));
    // the sync keeps the host staging vectors alive until the copies are done
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

RayLaunch ray_launch(tomo_ctx *ctx, const JacGeom &jg)
{
    const tomo_grid &g = ctx->g;
    RayLaunch rl{};
    rl.T = ctx->T.ptr;
    rl.shots = ctx->shots_d.ptr;
    rl.nshots = ctx->nshots;
    rl.spos = ctx->spos.ptr;
    rl.rx = ctx->rec.ptr;
    rl.ry = ctx->rec.ptr + ctx->nrec;
    rl.rz = ctx->rec.ptr + 2 * ctx->nrec;
    rl.nrec = ctx->nrec;
    rl.nz = g.nz;
    rl.dx = g.dx;
    rl.dy = g.dy;
    rl.dz = g.dz;
    rl.dxt = jg.dx;
    rl.dyt = jg.dy;
    rl.dzt = jg.dz;
    rl.nxt = jg.nxt;
    rl.nyt = jg.nyt;
    rl.nzt = jg.nzt;
    rl.max_steps = jg.max_steps;
    rl.smin = jg.ray_cap ? ctx->smin.ptr : nullptr;
    rl.length_factor = kRayLengthFactor;
    rl.cap_runs = jg.cap_runs;
    rl.runs = ctx->runs.ptr;
    rl.nuniq = ctx->nuniq.ptr;
    rl.status = ctx->ray_status.ptr;
    rl.steps = ctx->ray_steps.ptr;
    rl.final_dist = ctx->final_dist.ptr;
    rl.illum = jg.illum ? ctx->illum.ptr : nullptr;
    rl.model_nx = g.nx;
    rl.model_ny = g.ny;
    return rl;
}

int jac_march(tomo_ctx *ctx, const JacGeom &jg)
{
    const tomo_grid &g = ctx->g;
    const size_t npts = (size_t)g.nx * g.ny * g.nz;
    if (jg.illum) CK(cudaMemsetAsync(ctx->illum.ptr, 0, npts * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->nuniq.ptr + jg.nrays, 0, sizeof(int), ctx->stream));
    if (jg.ray_cap) {
        size_t tb = ctx->reduce_temp.cap;
        CK(tomo::reduce_min(ctx->slow.ptr, ctx->smin.ptr, npts, ctx->reduce_temp.ptr, &tb, ctx->stream));
    }
    size_t ob = ctx->order_temp.cap;
    CK(tomo::ray_order(ctx->t_recv.ptr, ctx->ray_keys.ptr, ctx->ray_keys_out.ptr, ctx->ray_iota.ptr, ctx->ray_order.ptr,
                       (int)jg.nrays, ctx->nrec, ctx->order_temp.ptr, &ob, ctx->stream));
    RayLaunch rl = ray_launch(ctx, jg);
    rl.order = ctx->ray_order.ptr;
    CK(tomo::ray_march(rl, ctx->stream));
    CK(tomo::ray_sort(rl, ctx->stream));
    size_t tb = ctx->scan_temp.cap;
    CK(tomo::scan_exclusive(ctx->nuniq.ptr, ctx->a_ptr.ptr, (int)jg.nrays + 1, ctx->scan_temp.ptr, &tb, ctx->stream));
    CK(tomo::csr_sizes(ctx->a_ptr.ptr, (int)jg.nrays, jg.tk_entries, ctx->csr_sizes.ptr, ctx->stream));
    return TOMO_OK;
}

int jac_ensure(tomo_ctx *ctx, const JacGeom &jg, long long cap)
{
    CK(ctx->a_idx.ensure((size_t)cap));
    CK(ctx->a_val.ensure((size_t)cap));
    return transpose_ensure(ctx, (int)jg.M, cap, ctx->t_ptr, ctx->t_idx, ctx->t_val, ctx->sort_keys,
                            ctx->sort_keys_out, ctx->sort_pos, ctx->sort_pos_out, ctx->rows_of, ctx->sort_temp,
                            ctx->stream);
}

int jac_emit(tomo_ctx *ctx, const JacGeom &jg, long long cap)
{
    const RayLaunch rl = ray_launch(ctx, jg);
    CK(tomo::ray_emit(rl, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr, ctx->stream));
    CK(tomo::tk_rows((int)jg.nrays, ctx->csr_sizes.ptr, (int)jg.M, jg.ord, ctx->tk_coef.ptr, ctx->a_ptr.ptr,
                     ctx->a_idx.ptr, ctx->a_val.ptr, ctx->stream));
    return transpose_enqueue(ctx, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr, (int)jg.N, (int)jg.M,
                             ctx->csr_sizes.ptr, cap, ctx->t_ptr, ctx->t_idx, ctx->t_val, ctx->sort_keys,
                             ctx->sort_keys_out, ctx->sort_pos, ctx->sort_pos_out, ctx->rows_of, ctx->sort_temp,
                             ctx->stream);
}

void jac_commit(tomo_ctx *ctx, const JacGeom &jg, long long nnz_g, long long nnz)
{
    ctx->n_data = (int)jg.nrays;
    ctx->n_model = (int)jg.M;
    ctx->n_rows = (int)jg.N;
    ctx->tk_order = jg.ord;
    ctx->nxt = jg.nxt;
    ctx->nyt = jg.nyt;
    ctx->nzt = jg.nzt;
    ctx->dxt = jg.dx;
    ctx->dyt = jg.dy;
    ctx->dzt = jg.dz;
    ctx->nnz_g = nnz_g;
    ctx->nnz = nnz;
    ctx->have_jacobian = true;
    ctx->have_illum = jg.illum;
    ctx->have_x = false;
}

}  // namespace tomo

extern "C" {

int tomo_build_jacobian(tomo_ctx *ctx, const tomo_jacobian_opts *opts, tomo_jacobian_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    tomo::JacGeom jg{};
    int rc = tomo::jac_prepare(ctx, opts, jg);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    rc = tomo::jac_march(ctx, jg);
    if (rc != TOMO_OK) return rc;
    long long sizes[2] = {0, 0};
    CK(cudaMemcpyAsync(sizes, ctx->csr_sizes.ptr, sizeof(sizes), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const long long nnz_g = sizes[0], nnz = sizes[1];
    rc = tomo::jac_ensure(ctx, jg, nnz);
    if (rc == TOMO_OK) rc = tomo::jac_emit(ctx, jg, nnz);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    const long long nrays = jg.nrays;
    std::vector<int> st((size_t)nrays), steps((size_t)nrays);
    CK(cudaMemcpyAsync(st.data(), ctx->ray_status.ptr, st.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(steps.data(), ctx->ray_steps.ptr, steps.size() * sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    tomo::jac_commit(ctx, jg, nnz_g, nnz);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nx = jg.nxt;
        stats->ny = jg.nyt;
        stats->nz = jg.nzt;
        stats->rows = jg.N;
        stats->cols = jg.M;
        stats->nnz_rays = nnz_g;
        stats->nnz = nnz;
        stats->rays = nrays;
        long long cnt[6] = {0, 0, 0, 0, 0, 0};
        for (size_t i = 0; i < st.size(); i++) {
            if (st[i] >= 0 && st[i] < 6) cnt[st[i]]++;
            stats->ray_steps += steps[i];
        }
        stats->rays_ok = cnt[0];
        stats->rays_stalled = cnt[1];
        stats->rays_capped = cnt[2];
        stats->rays_nonfinite = cnt[3];
        stats->rays_outside = cnt[4];
        stats->rays_overflow = cnt[5];
        cudaEventElapsedTime(&stats->ms, ctx->ev[0], ctx->ev[1]);
    }
    return TOMO_OK;
}

int tomo_jacobian_copy(tomo_ctx *ctx, int *row_ptr, int *cols, float *vals)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!ctx->have_jacobian) return fail(ctx, TOMO_ERR_STATE, "no Jacobian");
    if (!row_ptr || !cols || !vals) return fail(ctx, TOMO_ERR_INVALID_ARG, "NULL output");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(row_ptr, ctx->a_ptr.ptr, ((size_t)ctx->n_rows + 1) * sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaMemcpyAsync(cols, ctx->a_idx.ptr, (size_t)ctx->nnz * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(vals, ctx->a_val.ptr, (size_t)ctx->nnz * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_ray_status(tomo_ctx *ctx, int *status)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!ctx->have_jacobian) return fail(ctx, TOMO_ERR_STATE, "no Jacobian");
    if (!status) return fail(ctx, TOMO_ERR_INVALID_ARG, "NULL output");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(status, ctx->ray_status.ptr, (size_t)ctx->n_data * sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_illumination(tomo_ctx *ctx, float *out)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!ctx->have_illum) return fail(ctx, TOMO_ERR_STATE, "no illumination (build the Jacobian with illumination=1)");
    if (!out) return fail(ctx, TOMO_ERR_INVALID_ARG, "NULL output");
    CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    CK(cudaMemcpyAsync(out, ctx->illum.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_set_observed(tomo_ctx *ctx, const float *dobs, int n)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!dobs || n < 1) return fail(ctx, TOMO_ERR_INVALID_ARG, "NULL dobs or n < 1");
    CK(cudaSetDevice(ctx->device));
    CK(ctx->dobs.ensure((size_t)n));
    CK(cudaMemcpyAsync(ctx->dobs.ptr, dobs, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->n_dobs = n;
    ctx->have_dobs = true;
    return TOMO_OK;
}

int tomo_data_residual(tomo_ctx *ctx, double *norm)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!norm) return fail(ctx, TOMO_ERR_INVALID_ARG, "NULL output");
    if (!ctx->have_dobs || !ctx->have_solve) return fail(ctx, TOMO_ERR_STATE, "need observed data and a solve");
    if (ctx->n_dobs != ctx->nshots * ctx->nrec)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "observed data size does not match nshots*nrec of the solve");
    CK(cudaSetDevice(ctx->device));
    const int n = ctx->nshots * ctx->nrec;
    CK(ctx->norm2.ensure(1));
    CK(tomo::data_residual(ctx->dobs.ptr, ctx->t_recv.ptr, nullptr, n, n, ctx->norm2.ptr, ctx->stream));
    double v = 0.0;
    CK(cudaMemcpyAsync(&v, ctx->norm2.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *norm = std::sqrt(v);
    return TOMO_OK;
}

}  // extern "C"

namespace {

// Runs the CGLS kernel on prepared device buffers.
template <class Ctx>
int run_cgls(Ctx *ctx, int N, int M, const int *a_ptr, const int *a_idx, const float *a_val, const int *t_ptr,
             const int *t_idx, const float *t_val, const float *B, double *x, double *s, double *r, double *p, double *q,
             float *x32,
             tomo::DevBuf<double> &partials, double *hist, tomo::DevBuf<unsigned> &ctrl,
             tomo::DevBuf<int> &longr, tomo::DevBuf<unsigned char> &ltemp, int nit, double tol, cudaStream_t st,
             int *iters_run)
{
    int grid = 0;
    CK(tomo::cgls_grid(&grid));
    CK(partials.ensure((size_t)grid * 3));
    CK(ctrl.ensure(tomo::kCtrlWords));
    CK(cudaMemsetAsync(ctrl.ptr, 0, tomo::kCtrlWords * sizeof(unsigned), st));
    size_t lbytes = 0;
    CK(tomo::cgls_long_rows(t_ptr, M, nullptr, nullptr, nullptr, &lbytes, st));
    CK(longr.ensure((size_t)M + 1));
    CK(ltemp.ensure(lbytes));
    CK(tomo::cgls_long_rows(t_ptr, M, longr.ptr, longr.ptr + M, ltemp.ptr, &lbytes, st));
    tomo::CglsLaunch cl{};
    cl.long_rows = longr.ptr;
    cl.n_long = longr.ptr + M;
    cl.N = N;
    cl.M = M;
    cl.a_ptr = a_ptr;
    cl.a_idx = a_idx;
    cl.a_val = a_val;
    cl.t_ptr = t_ptr;
    cl.t_idx = t_idx;
    cl.t_val = t_val;
    cl.B = B;
    cl.x = x;
    cl.x32 = x32;
    cl.s = s;
    cl.r = r;
    cl.p = p;
    cl.q = q;
    cl.partials = partials.ptr;
    cl.hist = hist;
    cl.ctrl = ctrl.ptr;
    cl.nit = nit;
    cl.tol = tol;
    cl.spin_limit = kSpinLimit;
    CK(tomo::cgls_run(cl, grid, st));
    unsigned words[tomo::kCtrlWords];
    CK(cudaMemcpyAsync(words, ctrl.ptr, sizeof(words), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (words[tomo::kErr] != 0) return fail(ctx, TOMO_ERR_TIMEOUT, "CGLS: device barrier wait timed out");
    if (iters_run) *iters_run = (int)words[tomo::kRounds];
    return TOMO_OK;
}

struct Plain {
    std::string err;
};
int fail(Plain *c, int code, const std::string &msg)
{
    c->err = msg;
    return code;
}
int cuda_fail(Plain *c, cudaError_t e, const char *where)
{
    c->err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TOMO_ERR_OOM : TOMO_ERR_CUDA;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace tomo {

int cgls_prepare(tomo_ctx *ctx, int iterations)
{
    const int N = ctx->n_rows, M = ctx->n_model;
    CK(ctx->rhs.ensure((size_t)N));
    CK(ctx->x.ensure((size_t)M));
    CK(ctx->cg_x.ensure((size_t)M));
    CK(ctx->cg_s.ensure((size_t)N));
    CK(ctx->cg_q.ensure((size_t)N));
    CK(ctx->cg_r.ensure((size_t)M));
    CK(ctx->cg_p.ensure((size_t)M));
    CK(ctx->hist.ensure((size_t)(iterations > 0 ? iterations : 1)));
    CK(ctx->norm2.ensure(1));
    int grid = 0;
    CK(tomo::cgls_grid(&grid));
    CK(ctx->partials.ensure((size_t)grid * 3));
    CK(ctx->cg_ctrl.ensure(tomo::kCtrlWords));
    size_t lbytes = 0;
    CK(tomo::cgls_long_rows(ctx->t_ptr.ptr, M, nullptr, nullptr, nullptr, &lbytes, ctx->stream));
    CK(ctx->cg_long.ensure((size_t)M + 1));
    CK(ctx->cg_ltemp.ensure(lbytes));
    return TOMO_OK;
}

int cgls_enqueue(tomo_ctx *ctx, int iterations)
{
    const int N = ctx->n_rows, M = ctx->n_model, nd = ctx->n_data;
    // B = [dobs - dcal ; 0] (least_squares.cpp:335-336)
    CK(tomo::data_residual(ctx->dobs.ptr, ctx->t_recv.ptr, ctx->rhs.ptr, nd, N, ctx->norm2.ptr, ctx->stream));
    CK(cudaMemsetAsync(ctx->cg_ctrl.ptr, 0, tomo::kCtrlWords * sizeof(unsigned), ctx->stream));
    int grid = 0;
    CK(tomo::cgls_grid(&grid));
    tomo::CglsLaunch cl{};
    cl.N = N;
    cl.M = M;
    cl.a_ptr = ctx->a_ptr.ptr;
    cl.a_idx = ctx->a_idx.ptr;
    cl.a_val = ctx->a_val.ptr;
    cl.t_ptr = ctx->t_ptr.ptr;
    cl.t_idx = ctx->t_idx.ptr;
    cl.t_val = ctx->t_val.ptr;
    cl.B = ctx->rhs.ptr;
    cl.x = ctx->cg_x.ptr;
    cl.x32 = ctx->x.ptr;
    cl.s = ctx->cg_s.ptr;
    cl.r = ctx->cg_r.ptr;
    cl.p = ctx->cg_p.ptr;
    cl.q = ctx->cg_q.ptr;
    cl.partials = ctx->partials.ptr;
    cl.hist = ctx->hist.ptr;
    cl.ctrl = ctx->cg_ctrl.ptr;
    cl.nit = iterations;
    cl.tol = 0.0;
    cl.spin_limit = kSpinLimit;
    size_t lbytes = ctx->cg_ltemp.cap;
    CK(tomo::cgls_long_rows(ctx->t_ptr.ptr, M, ctx->cg_long.ptr, ctx->cg_long.ptr + M, ctx->cg_ltemp.ptr, &lbytes,
                            ctx->stream));
    cl.long_rows = ctx->cg_long.ptr;
    cl.n_long = ctx->cg_long.ptr + M;
    CK(tomo::cgls_run(cl, grid, ctx->stream));
    return TOMO_OK;
}

int update_prepare(tomo_ctx *ctx, const tomo_update_opts *opts)
{
    const int smooth = opts ? opts->smooth : 1;
    const int samples = opts ? opts->filter_samples : 5;
    const float stdv = opts ? opts->standard_deviation : 2.0f;
    if (smooth && (samples < 1 || samples % 2 == 0))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "filter_samples must be odd and >= 1");
    const tomo_grid &g = ctx->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    CK(ctx->dm.ensure(n));
    if (smooth) {
        const std::vector<float> k = gaussian_weights(samples, stdv);
        CK(ctx->gauss_kernel.ensure(k.size()));
        CK(cudaMemcpyAsync(ctx->gauss_kernel.ptr, k.data(), k.size() * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(ctx->dm_smooth.ensure(n));
        CK(cudaStreamSynchronize(ctx->stream));  // k is a host temporary
    }
    return TOMO_OK;
}

// dm from the CGLS solution, optional smoothing, slowness += dm, re-brick (velocity_out:
// device array or nullptr).
int update_enqueue_v(tomo_ctx *ctx, const tomo_update_opts *opts, float *velocity_out)
{
    const int smooth = opts ? opts->smooth : 1;
    const int samples = opts ? opts->filter_samples : 5;
    const int ref_masks = opts ? opts->use_reference_masks : 1;
    const tomo_grid &g = ctx->g;
    const tomo::UpdateMasks m = ref_masks ? reference_masks() : tomo::UpdateMasks{0, 0, 0, 0, 0, 0, 0, 0};
    CK(tomo::model_dm(ctx->x.ptr, ctx->dm.ptr, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, ctx->dxt, ctx->dyt, ctx->dzt,
                      ctx->nxt, ctx->nyt, ctx->nzt, m, ctx->stream));
    const float *dm = ctx->dm.ptr;
    if (smooth) {
        CK(tomo::gaussian_smooth(ctx->dm.ptr, ctx->dm_smooth.ptr, g.nx, g.ny, g.nz, samples, ctx->gauss_kernel.ptr,
                                 ctx->stream));
        dm = ctx->dm_smooth.ptr;
    }
    CK(tomo::model_apply(ctx->slow.ptr, dm, velocity_out, g.nx, g.ny, g.nz, m, ctx->stream));
    return tomo::rebrick_model(ctx);
}

int update_enqueue(tomo_ctx *ctx, const tomo_update_opts *opts) { return update_enqueue_v(ctx, opts, nullptr); }

}  // namespace tomo

extern "C" {

int tomo_cgls(tomo_ctx *ctx, int iterations, float *x_out, double *history, tomo_cgls_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (iterations < 0) return fail(ctx, TOMO_ERR_INVALID_ARG, "iterations < 0");
    if (!ctx->have_jacobian) return fail(ctx, TOMO_ERR_STATE, "no Jacobian (tomo_build_jacobian)");
    if (!ctx->have_dobs) return fail(ctx, TOMO_ERR_STATE, "no observed data (tomo_set_observed)");
    if (ctx->n_dobs != ctx->n_data)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "observed data size does not match the Jacobian's rays");
    CK(cudaSetDevice(ctx->device));
    const int M = ctx->n_model;
    int rc = tomo::cgls_prepare(ctx, iterations);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    rc = tomo::cgls_enqueue(ctx, iterations);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    std::vector<double> h((size_t)(iterations > 0 ? iterations : 1), 0.0);
    double b2 = 0.0;
    unsigned words[tomo::kCtrlWords];
    CK(cudaMemcpyAsync(words, ctx->cg_ctrl.ptr, sizeof(words), cudaMemcpyDeviceToHost, ctx->stream));
    if (iterations > 0)
        CK(cudaMemcpyAsync(h.data(), ctx->hist.ptr, (size_t)iterations * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaMemcpyAsync(&b2, ctx->norm2.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (x_out) CK(cudaMemcpyAsync(x_out, ctx->x.ptr, (size_t)M * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (words[tomo::kErr] != 0) return fail(ctx, TOMO_ERR_TIMEOUT, "CGLS: device barrier wait timed out");
    if (history && iterations > 0) std::memcpy(history, h.data(), (size_t)iterations * sizeof(double));
    ctx->have_x = true;
    if (stats) {
        stats->iterations = (int)words[tomo::kRounds];
        stats->rnorm0 = std::sqrt(b2);
        stats->rnorm = iterations > 0 ? h[(size_t)iterations - 1] : std::sqrt(b2);
        cudaEventElapsedTime(&stats->ms, ctx->ev[0], ctx->ev[1]);
    }
    return TOMO_OK;
}

int tomo_model_update(tomo_ctx *ctx, const tomo_update_opts *opts, float *velocity_out)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!ctx->have_x) return fail(ctx, TOMO_ERR_STATE, "no CGLS solution (tomo_cgls)");
    CK(cudaSetDevice(ctx->device));
    const size_t n = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    int rc = tomo::update_prepare(ctx, opts);
    if (rc != TOMO_OK) return rc;
    float *vel = nullptr;
    if (velocity_out) {
        CK(ctx->vel_out.ensure(n));
        vel = ctx->vel_out.ptr;
    }
    rc = tomo::update_enqueue_v(ctx, opts, vel);
    if (rc != TOMO_OK) return rc;
    if (velocity_out)
        CK(cudaMemcpyAsync(velocity_out, vel, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TOMO_OK;
}

int tomo_sparse_cgls_gpu(const int *iA, const int *jA, const float *vA, const float *B, float *x, int N, int M,
                         int NNZ, int NIT, float TOL)
{
    if (!iA || !jA || !vA || !B || !x || N < 1 || M < 1 || NNZ < 1 || NIT < 0) return TOMO_ERR_INVALID_ARG;
    for (int k = 0; k < NNZ; k++)
        if (iA[k] < 0 || iA[k] >= N || jA[k] < 0 || jA[k] >= M) return TOMO_ERR_INVALID_ARG;
    // Stable counting sort of the COO rows into CSR (cusparseXcoo2csr needs sorted rows;
    // here any order is accepted and entries keep their order inside a row).
    std::vector<int> ptr((size_t)N + 1, 0), idx((size_t)NNZ);
    std::vector<float> val((size_t)NNZ);
    for (int k = 0; k < NNZ; k++) ptr[(size_t)iA[k] + 1]++;
    for (int r = 0; r < N; r++) ptr[(size_t)r + 1] += ptr[(size_t)r];
    std::vector<int> cur(ptr.begin(), ptr.end() - 1);
    for (int k = 0; k < NNZ; k++) {
        const int pos = cur[(size_t)iA[k]]++;
        idx[(size_t)pos] = jA[k];
        val[(size_t)pos] = vA[k];
    }
    Plain pl;
    Plain *ctx = &pl;
    tomo::DevBuf<int> a_ptr, a_idx, t_ptr, t_idx, k0, k1, p0, p1, rows_of;
    tomo::DevBuf<float> a_val, t_val, dB, dx_;
    tomo::DevBuf<double> x64, s, r, p, q;
    tomo::DevBuf<double> partials;
    tomo::DevBuf<unsigned> ctrl;
    tomo::DevBuf<unsigned char> temp, ltemp;
    tomo::DevBuf<int> longr;
    tomo::DevBuf<long long> sizes;
    cudaStream_t st = nullptr;
    int rc = TOMO_OK;
    auto cleanup = [&]() {
        sizes.release();
        for (auto *b : {&a_ptr, &a_idx, &t_ptr, &t_idx, &k0, &k1, &p0, &p1, &rows_of}) b->release();
        for (auto *b : {&a_val, &t_val, &dB, &dx_}) b->release();
        for (auto *b : {&x64, &s, &r, &p, &q}) b->release();
        partials.release();
        ctrl.release();
        temp.release();
        ltemp.release();
        longr.release();
        if (st) cudaStreamDestroy(st);
    };
    auto body = [&]() -> int {
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CK(a_ptr.ensure((size_t)N + 1));
        CK(a_idx.ensure((size_t)NNZ));
        CK(a_val.ensure((size_t)NNZ));
        CK(dB.ensure((size_t)N));
        CK(dx_.ensure((size_t)M));
        CK(x64.ensure((size_t)M));
        CK(s.ensure((size_t)N));
        CK(q.ensure((size_t)N));
        CK(r.ensure((size_t)M));
        CK(p.ensure((size_t)M));
        CK(cudaMemcpyAsync(a_ptr.ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(a_idx.ptr, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(a_val.ptr, val.data(), val.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(dB.ptr, B, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, st));
        const long long hs[2] = {NNZ, NNZ};
        CK(sizes.ensure(2));
        CK(cudaMemcpyAsync(sizes.ptr, hs, sizeof(hs), cudaMemcpyHostToDevice, st));
        int r2 = transpose_ensure(ctx, M, NNZ, t_ptr, t_idx, t_val, k0, k1, p0, p1, rows_of, temp, st);
        if (r2 == TOMO_OK)
            r2 = transpose_enqueue(ctx, a_ptr.ptr, a_idx.ptr, a_val.ptr, N, M, sizes.ptr, NNZ, t_ptr, t_idx, t_val, k0,
                                   k1, p0, p1, rows_of, temp, st);
        if (r2 != TOMO_OK) return r2;
        r2 = run_cgls(ctx, N, M, a_ptr.ptr, a_idx.ptr, a_val.ptr, t_ptr.ptr, t_idx.ptr, t_val.ptr, dB.ptr, x64.ptr,
                      s.ptr, r.ptr, p.ptr, q.ptr, dx_.ptr, partials, nullptr, ctrl, longr, ltemp, NIT, (double)TOL, st,
                      nullptr);
        if (r2 != TOMO_OK) return r2;
        CK(cudaMemcpyAsync(x, dx_.ptr, (size_t)M * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return TOMO_OK;
    };
    rc = body();
    cleanup();
    return rc;
}

}  // extern "C"
