// C ABI: ray tracing into the Jacobian, CGLS and model update (include/tomo_b200.h).
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cgls.cuh"
#include "common.cuh"
#include "context.hpp"
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
// sort of the column keys keeps each column's entries in row order (deterministic).
template <class Ctx>
int build_transpose(Ctx *ctx, const int *ptr, const int *idx, const float *val, int nrows, int ncols, long long nnz,
                    tomo::DevBuf<int> &t_ptr, tomo::DevBuf<int> &t_idx, tomo::DevBuf<float> &t_val,
                    tomo::DevBuf<int> &k0, tomo::DevBuf<int> &k1, tomo::DevBuf<int> &p0, tomo::DevBuf<int> &p1,
                    tomo::DevBuf<int> &rows_of, tomo::DevBuf<unsigned char> &temp, cudaStream_t st)
{
    CK(k0.ensure((size_t)nnz));
    CK(k1.ensure((size_t)nnz));
    CK(p0.ensure((size_t)nnz));
    CK(p1.ensure((size_t)nnz));
    CK(rows_of.ensure((size_t)nnz));
    CK(t_ptr.ensure((size_t)ncols + 1));
    CK(t_idx.ensure((size_t)nnz));
    CK(t_val.ensure((size_t)nnz));
    CK(tomo::csr_transpose_prepare(ptr, idx, nrows, nnz, k0.ptr, p0.ptr, rows_of.ptr, st));
    size_t tb = 0;
    CK(tomo::sort_pairs(k0.ptr, k1.ptr, p0.ptr, p1.ptr, nnz, bits_for(ncols + 1), nullptr, &tb, st));
    CK(temp.ensure(tb));
    CK(tomo::sort_pairs(k0.ptr, k1.ptr, p0.ptr, p1.ptr, nnz, bits_for(ncols + 1), temp.ptr, &tb, st));
    CK(tomo::csr_transpose_finish(p1.ptr, rows_of.ptr, val, nnz, ncols, k1.ptr, t_ptr.ptr, t_idx.ptr, t_val.ptr, st));
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
    for (auto *b : {&ctx->cg_x, &ctx->cg_s, &ctx->cg_r, &ctx->cg_p, &ctx->cg_q}) b->release();
}

int tomo_build_jacobian(tomo_ctx *ctx, const tomo_jacobian_opts *opts, tomo_jacobian_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (!opts || !(opts->dx > 0) || !(opts->dy > 0) || !(opts->dz > 0) || opts->tk_order < 0)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "bad inversion grid / Tikhonov options");
    if (!ctx->have_solve || ctx->nrec < 1) return fail(ctx, TOMO_ERR_STATE, "no eikonal solve with receivers");
    CK(cudaSetDevice(ctx->device));
    const tomo_grid &g = ctx->g;
    // Least_squares::set_parameters (least_squares.cpp:124-126)
    const int nzt = (int)((g.nz - 1) * g.dz / opts->dz) + 1;
    const int nxt = (int)((g.nx - 1) * g.dx / opts->dx) + 1;
    const int nyt = (int)((g.ny - 1) * g.dy / opts->dy) + 1;
    const long long M = (long long)nxt * nyt * nzt;
    const int ord = opts->tk_order;
    if (M <= ord || M >= (1ll << 30)) return fail(ctx, TOMO_ERR_INVALID_ARG, "inversion grid too small or too large");
    const long long nrays = (long long)ctx->nshots * ctx->nrec;
    const long long N = nrays + M - ord;
    if (N >= (1ll << 31) - 1) return fail(ctx, TOMO_ERR_CAPACITY, "too many rows");
    const float rayStep = 0.2f * g.dz;
    const float dmax = std::fmax(g.dx, std::fmax(g.dy, g.dz));
    const int max_steps = opts->max_ray_steps > 0 ? opts->max_ray_steps
                                                  : (int)(20.0f * (g.nx + g.ny + g.nz) * dmax / rayStep);
    // Default cap per ray: the reference marches until the source cell with no cap
    // (least_squares.cpp:216-280), so a ray circling a flat spot of the field never ends.
    // A ray of traveltime T is at most T x v_max long; 4x that (plus 256 steps) leaves
    // every terminating ray untouched and stops circling ones early.
    float steps_per_second = 0.f;
    if (opts->max_ray_steps <= 0) {
        const size_t nmodel = (size_t)g.nx * g.ny * g.nz;
        size_t tb = 0;
        CK(tomo::reduce_min(ctx->slow.ptr, nullptr, nmodel, nullptr, &tb, ctx->stream));
        const size_t off = (tb + 255) / 256 * 256;
        CK(ctx->cub_temp.ensure(off + sizeof(float)));
        float *smin_d = reinterpret_cast<float *>(ctx->cub_temp.ptr + off);
        CK(tomo::reduce_min(ctx->slow.ptr, smin_d, nmodel, ctx->cub_temp.ptr, &tb, ctx->stream));
        float smin = 0.f;
        CK(cudaMemcpyAsync(&smin, smin_d, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (smin > 0.f && std::isfinite(smin)) steps_per_second = kRayLengthFactor / (smin * rayStep);
    }
    const int cap_runs = opts->max_cells_per_ray > 0 ? opts->max_cells_per_ray : 1024;
    bool full = true;
    for (const auto &d : ctx->shots_h) full = full && d.wx0 == 0 && d.wy0 == 0 && d.wnx == g.nx && d.wny == g.ny;
    if (opts->illumination && !full)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "illumination needs full-model windows");

    CK(ctx->runs.ensure((size_t)nrays * cap_runs));
    CK(ctx->nuniq.ensure((size_t)nrays + 1));
    CK(ctx->ray_status.ensure((size_t)nrays));
    CK(ctx->ray_steps.ensure((size_t)nrays));
    CK(ctx->final_dist.ensure((size_t)nrays));
    CK(ctx->spos.ensure((size_t)ctx->nshots * 3));
    CK(ctx->a_ptr.ensure((size_t)N + 1));
    std::vector<float> sp((size_t)ctx->nshots * 3);
    for (int s = 0; s < ctx->nshots; s++) {
        sp[(size_t)s] = ctx->shot_pos[(size_t)s].x;
        sp[(size_t)ctx->nshots + s] = ctx->shot_pos[(size_t)s].y;
        sp[(size_t)2 * ctx->nshots + s] = ctx->shot_pos[(size_t)s].z;
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    CK(cudaMemcpyAsync(ctx->spos.ptr, sp.data(), sp.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    const size_t npts = (size_t)g.nx * g.ny * g.nz;
    if (opts->illumination) {
        CK(ctx->illum.ensure(npts));
        CK(cudaMemsetAsync(ctx->illum.ptr, 0, npts * sizeof(float), ctx->stream));
    }
    CK(cudaMemsetAsync(ctx->nuniq.ptr + nrays, 0, sizeof(int), ctx->stream));

    tomo::RayLaunch rl{};
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
    rl.dxt = opts->dx;
    rl.dyt = opts->dy;
    rl.dzt = opts->dz;
    rl.nxt = nxt;
    rl.nyt = nyt;
    rl.nzt = nzt;
    rl.max_steps = max_steps;
    rl.steps_per_second = steps_per_second;
    rl.cap_runs = cap_runs;
    rl.runs = ctx->runs.ptr;
    rl.nuniq = ctx->nuniq.ptr;
    rl.status = ctx->ray_status.ptr;
    rl.steps = ctx->ray_steps.ptr;
    rl.final_dist = ctx->final_dist.ptr;
    rl.illum = opts->illumination ? ctx->illum.ptr : nullptr;
    rl.model_nx = g.nx;
    rl.model_ny = g.ny;
    CK(tomo::ray_march(rl, ctx->stream));
    size_t tb = 0;
    CK(tomo::scan_exclusive(ctx->nuniq.ptr, ctx->a_ptr.ptr, (int)nrays + 1, nullptr, &tb, ctx->stream));
    CK(ctx->cub_temp.ensure(tb));
    CK(tomo::scan_exclusive(ctx->nuniq.ptr, ctx->a_ptr.ptr, (int)nrays + 1, ctx->cub_temp.ptr, &tb, ctx->stream));
    int nnz_g = 0;
    CK(cudaMemcpyAsync(&nnz_g, ctx->a_ptr.ptr + nrays, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const long long nL = M - ord;
    const long long nnz = (long long)nnz_g + (long long)(ord + 1) * nL;
    if (nnz >= (1ll << 31) - 1) return fail(ctx, TOMO_ERR_CAPACITY, "Jacobian has more than 2^31 non-zeros");
    CK(ctx->a_idx.ensure((size_t)nnz));
    CK(ctx->a_val.ensure((size_t)nnz));
    CK(tomo::ray_emit(rl, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr, ctx->stream));
    // Tikhonov rows lambda * df (least_squares.cpp:412-417)
    const std::vector<int> df = tk_coefficients(ord);
    std::vector<float> coef((size_t)ord + 1);
    for (int k = 0; k <= ord; k++) coef[(size_t)k] = opts->tk_param * (float)df[(size_t)k];
    CK(ctx->tk_coef.ensure(coef.size()));
    CK(cudaMemcpyAsync(ctx->tk_coef.ptr, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(tomo::tk_rows((int)nrays, nnz_g, (int)M, ord, ctx->tk_coef.ptr, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr,
                     ctx->stream));
    int rc = build_transpose(ctx, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr, (int)N, (int)M, nnz, ctx->t_ptr,
                             ctx->t_idx, ctx->t_val, ctx->sort_keys, ctx->sort_keys_out, ctx->sort_pos,
                             ctx->sort_pos_out, ctx->rows_of, ctx->cub_temp, ctx->stream);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    std::vector<int> st((size_t)nrays), steps((size_t)nrays);
    CK(cudaMemcpyAsync(st.data(), ctx->ray_status.ptr, st.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(steps.data(), ctx->ray_steps.ptr, steps.size() * sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));

    ctx->n_data = (int)nrays;
    ctx->n_model = (int)M;
    ctx->n_rows = (int)N;
    ctx->tk_order = ord;
    ctx->nxt = nxt;
    ctx->nyt = nyt;
    ctx->nzt = nzt;
    ctx->dxt = opts->dx;
    ctx->dyt = opts->dy;
    ctx->dzt = opts->dz;
    ctx->nnz_g = nnz_g;
    ctx->nnz = nnz;
    ctx->have_jacobian = true;
    ctx->have_illum = opts->illumination != 0;
    ctx->have_x = false;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->nx = nxt;
        stats->ny = nyt;
        stats->nz = nzt;
        stats->rows = N;
        stats->cols = M;
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
             tomo::DevBuf<double> &partials, double *hist, tomo::DevBuf<unsigned> &ctrl, int nit, double tol,
             cudaStream_t st, int *iters_run)
{
    int grid = 0;
    CK(tomo::cgls_grid(&grid));
    CK(partials.ensure((size_t)grid * 3));
    CK(ctrl.ensure(tomo::kCtrlWords));
    CK(cudaMemsetAsync(ctrl.ptr, 0, tomo::kCtrlWords * sizeof(unsigned), st));
    tomo::CglsLaunch cl{};
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

int tomo_cgls(tomo_ctx *ctx, int iterations, float *x_out, double *history, tomo_cgls_stats *stats)
{
    if (!ctx) return TOMO_ERR_INVALID_ARG;
    if (iterations < 0) return fail(ctx, TOMO_ERR_INVALID_ARG, "iterations < 0");
    if (!ctx->have_jacobian) return fail(ctx, TOMO_ERR_STATE, "no Jacobian (tomo_build_jacobian)");
    if (!ctx->have_dobs) return fail(ctx, TOMO_ERR_STATE, "no observed data (tomo_set_observed)");
    if (ctx->n_dobs != ctx->n_data)
        return fail(ctx, TOMO_ERR_INVALID_ARG, "observed data size does not match the Jacobian's rays");
    CK(cudaSetDevice(ctx->device));
    const int N = ctx->n_rows, M = ctx->n_model, nd = ctx->n_data;
    CK(ctx->rhs.ensure((size_t)N));
    CK(ctx->x.ensure((size_t)M));
    CK(ctx->cg_x.ensure((size_t)M));
    CK(ctx->cg_s.ensure((size_t)N));
    CK(ctx->cg_q.ensure((size_t)N));
    CK(ctx->cg_r.ensure((size_t)M));
    CK(ctx->cg_p.ensure((size_t)M));
    CK(ctx->hist.ensure((size_t)(iterations > 0 ? iterations : 1)));
    CK(ctx->norm2.ensure(1));
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    // B = [dobs - dcal ; 0] (least_squares.cpp:335-336)
    CK(tomo::data_residual(ctx->dobs.ptr, ctx->t_recv.ptr, ctx->rhs.ptr, nd, N, ctx->norm2.ptr, ctx->stream));
    int iters = 0;
    int rc = run_cgls(ctx, N, M, ctx->a_ptr.ptr, ctx->a_idx.ptr, ctx->a_val.ptr, ctx->t_ptr.ptr, ctx->t_idx.ptr,
                      ctx->t_val.ptr, ctx->rhs.ptr, ctx->cg_x.ptr, ctx->cg_s.ptr, ctx->cg_r.ptr, ctx->cg_p.ptr,
                      ctx->cg_q.ptr, ctx->x.ptr, ctx->partials, ctx->hist.ptr, ctx->cg_ctrl, iterations, 0.0, ctx->stream, &iters);
    if (rc != TOMO_OK) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    std::vector<double> h((size_t)(iterations > 0 ? iterations : 1), 0.0);
    double b2 = 0.0;
    if (iterations > 0)
        CK(cudaMemcpyAsync(h.data(), ctx->hist.ptr, (size_t)iterations * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaMemcpyAsync(&b2, ctx->norm2.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (x_out) CK(cudaMemcpyAsync(x_out, ctx->x.ptr, (size_t)M * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (history && iterations > 0) std::memcpy(history, h.data(), (size_t)iterations * sizeof(double));
    ctx->have_x = true;
    if (stats) {
        stats->iterations = iters;
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
    const int smooth = opts ? opts->smooth : 1;
    const int samples = opts ? opts->filter_samples : 5;
    const float stdv = opts ? opts->standard_deviation : 2.0f;
    const int ref_masks = opts ? opts->use_reference_masks : 1;
    if (smooth && (samples < 1 || samples % 2 == 0))
        return fail(ctx, TOMO_ERR_INVALID_ARG, "filter_samples must be odd and >= 1");
    CK(cudaSetDevice(ctx->device));
    const tomo_grid &g = ctx->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const tomo::UpdateMasks m = ref_masks ? reference_masks() : tomo::UpdateMasks{0, 0, 0, 0, 0, 0, 0, 0};
    CK(ctx->dm.ensure(n));
    CK(tomo::model_dm(ctx->x.ptr, ctx->dm.ptr, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, ctx->dxt, ctx->dyt, ctx->dzt,
                      ctx->nxt, ctx->nyt, ctx->nzt, m, ctx->stream));
    const float *dm = ctx->dm.ptr;
    if (smooth) {
        const std::vector<float> k = gaussian_weights(samples, stdv);
        CK(ctx->gauss_kernel.ensure(k.size()));
        CK(cudaMemcpyAsync(ctx->gauss_kernel.ptr, k.data(), k.size() * sizeof(float), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(ctx->dm_smooth.ensure(n));
        CK(tomo::gaussian_smooth(ctx->dm.ptr, ctx->dm_smooth.ptr, g.nx, g.ny, g.nz, samples, ctx->gauss_kernel.ptr,
                                 ctx->stream));
        dm = ctx->dm_smooth.ptr;
    }
    float *vel = nullptr;
    if (velocity_out) {
        CK(ctx->vel_out.ensure(n));
        vel = ctx->vel_out.ptr;
    }
    CK(tomo::model_apply(ctx->slow.ptr, dm, vel, g.nx, g.ny, g.nz, m, ctx->stream));
    int rc = tomo::rebrick_model(ctx);
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
    tomo::DevBuf<unsigned char> temp;
    cudaStream_t st = nullptr;
    int rc = TOMO_OK;
    auto cleanup = [&]() {
        for (auto *b : {&a_ptr, &a_idx, &t_ptr, &t_idx, &k0, &k1, &p0, &p1, &rows_of}) b->release();
        for (auto *b : {&a_val, &t_val, &dB, &dx_}) b->release();
        for (auto *b : {&x64, &s, &r, &p, &q}) b->release();
        partials.release();
        ctrl.release();
        temp.release();
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
        int r2 = build_transpose(ctx, a_ptr.ptr, a_idx.ptr, a_val.ptr, N, M, NNZ, t_ptr, t_idx, t_val, k0, k1, p0, p1,
                                 rows_of, temp, st);
        if (r2 != TOMO_OK) return r2;
        r2 = run_cgls(ctx, N, M, a_ptr.ptr, a_idx.ptr, a_val.ptr, t_ptr.ptr, t_idx.ptr, t_val.ptr, dB.ptr, x64.ptr,
                      s.ptr, r.ptr, p.ptr, q.ptr, dx_.ptr, partials, nullptr, ctrl, NIT, (double)TOL, st, nullptr);
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
