// Stages of the tomography iteration as enqueue-only steps, shared by the one-call-per-stage
// C ABI (api_eikonal.cpp, api_tomography.cpp) and the graph-captured iteration
// (api_iteration.cpp).  "prepare" steps allocate and upload; "enqueue" steps only put work
// on the context's stream (no allocation, no host synchronisation), so they can be captured.
#pragma once

#include "context.hpp"
#include "ray.cuh"

namespace tomo {

// Geometry of the Jacobian of the current solve (inversion grid, Tikhonov, ray caps).
struct JacGeom {
    int nxt, nyt, nzt, ord;
    long long M, N, nrays, tk_entries;
    int max_steps, cap_runs;
    bool ray_cap, illum;
    float rayStep, dx, dy, dz;
};

int jac_prepare(tomo_ctx *ctx, const tomo_jacobian_opts *opts, JacGeom &jg);
int jac_march(tomo_ctx *ctx, const JacGeom &jg);              // rays, row lengths, csr_sizes
int jac_ensure(tomo_ctx *ctx, const JacGeom &jg, long long cap);
int jac_emit(tomo_ctx *ctx, const JacGeom &jg, long long cap);  // needs nnz <= cap
void jac_commit(tomo_ctx *ctx, const JacGeom &jg, long long nnz_g, long long nnz);

int cgls_prepare(tomo_ctx *ctx, int iterations);
int cgls_enqueue(tomo_ctx *ctx, int iterations);               // B = [dobs - dcal; 0], then CGLS
int update_prepare(tomo_ctx *ctx, const tomo_update_opts *opts);
int update_enqueue(tomo_ctx *ctx, const tomo_update_opts *opts);
int update_enqueue_v(tomo_ctx *ctx, const tomo_update_opts *opts, float *velocity_out);

// The JW batch solve of tomo_eik_solve split the same way.
struct EikPlan {
    FimLaunch p;
    int block_warps, occupancy;
    bool ieee_sqrt, async, brick8;
    size_t t_total, q_total;
};
int eik_plan(tomo_ctx *ctx, int nshots, const tomo_point *shots, const tomo_window *windows, int nrec,
             const tomo_point *receivers, const tomo_eik_opts *opts, EikPlan &plan);
int eik_enqueue(tomo_ctx *ctx, const EikPlan &plan);

}  // namespace tomo
