// CGLS and model-update kernels: shared declarations.
#pragma once

#include <cuda_runtime.h>

namespace tomo {

struct CglsLaunch {
    int N, M;                                               // rows, columns
    const int *a_ptr, *a_idx; const float *a_val;           // A in CSR
    const int *t_ptr, *t_idx; const float *t_val;           // A' in CSR
    const int *long_rows, *n_long;                          // A' rows summed by whole blocks
    const float *B;                                         // right-hand side (N)
    double *x, *s, *r, *p, *q;                              // M, N, M, M, N (FP64 vectors)
    float *x32;                                             // solution rounded to FP32 (M)
    double *partials;                                       // 3 * gridDim.x
    double *hist;                                           // ||s|| per iteration (nit) or nullptr
    unsigned *ctrl;                                         // kCtrlWords (barrier, error, iterations run)
    int nit;
    double tol;                                             // stop when ||r|| < tol (0: never)
    unsigned long long spin_limit;
};

cudaError_t cgls_grid(int *grid);
// The rows of A' (t_ptr, M rows) too long for one 32-lane group, in row order, and their
// count, on the device (temp == nullptr: *temp_bytes = the scratch needed).
cudaError_t cgls_long_rows(const int *t_ptr, int M, int *rows, int *n_long, void *temp, size_t *temp_bytes,
                           cudaStream_t st);
cudaError_t cgls_run(const CglsLaunch &p, int grid, cudaStream_t st);

// Model update (Least_squares::model_update, least_squares.cpp:498-570).
struct UpdateMasks {
    int i_lo, i_hi_off;      // i >= i_lo && i < nz - i_hi_off
    int j_lo, j_hi_off_dm;   // dm mask:     j < nx - j_hi_off_dm (16)
    int j_hi_off_upd;        // update mask: j < nx - j_hi_off_upd (15)
    int k_lo, k_hi_off_dm, k_hi_off_upd;
};

cudaError_t model_dm(const float *xdm, float *dm, int nx, int ny, int nz, float dx, float dy, float dz, float dxt,
                     float dyt, float dzt, int nxt, int nyt, int nzt, UpdateMasks m, cudaStream_t st);
cudaError_t gaussian_smooth(const float *in, float *out, int nx, int ny, int nz, int samples, const float *kernel,
                            cudaStream_t st);
cudaError_t model_apply(float *slowness, const float *dm, float *velocity, int nx, int ny, int nz, UpdateMasks m,
                        cudaStream_t st);
cudaError_t data_residual(const float *dobs, const float *dcal, float *B, int n, int n_total, double *partial,
                          cudaStream_t st);

}  // namespace tomo
