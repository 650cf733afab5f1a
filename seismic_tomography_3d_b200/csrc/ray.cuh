// Ray tracing through the device-resident traveltime fields into the sparse Frechet
// matrix, Tikhonov rows, transpose, CGLS and model update: shared declarations.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fim.cuh"

namespace tomo {

// Ray status (same codes as the CPU oracle).
enum RayStatus : int {
    kRayOk = 0,        // reached the source cell (reference stop rule)
    kRayStalled = 1,   // entered the source node box outside the source cell
    kRayCapped = 2,    // step cap
    kRayNonFinite = 3, // zero gradient -> NaN position
    kRayOutside = 4,   // left the inversion grid / receiver outside the window
    kRayOverflow = 5,  // more distinct cells than the per-ray capacity
};

struct RayLaunch {
    const int *order;     // rays in march order (nullptr: natural order)
    const float *T;
    const ShotDesc *shots;
    int nshots;
    const float *spos;    // 3*nshots: x | y | z (metres)
    const float *rx, *ry, *rz;
    int nrec;
    int nz;               // model nz
    float dx, dy, dz;
    float dxt, dyt, dzt;  // inversion cell size
    int nxt, nyt, nzt;    // inversion grid
    int max_steps;
    const float *smin;       // device: smallest slowness of the model, or nullptr.  Given, a ray
    float length_factor;     // also stops (capped) after length_factor x T(start) / smin / step
                             // + 256 steps -- a ray of traveltime T is at most T x v_max long
    int cap_runs;         // per-ray capacity of distinct cells
    uint2 *runs;          // nrays*cap_runs (cell, count), sorted by cell on exit
    int *nuniq;           // per ray: distinct cells
    int *status, *steps;
    float *final_dist;
    float *illum;         // nz*nx*ny of the model or nullptr (full windows only)
    int model_nx, model_ny;
};

cudaError_t ray_march(const RayLaunch &p, cudaStream_t st);
// per ray: runs sorted by cell with repeated cells merged; nuniq = distinct cells
cudaError_t ray_sort(const RayLaunch &p, cudaStream_t st);
cudaError_t ray_emit(const RayLaunch &p, const int *row_ptr, int *cols, float *vals, cudaStream_t st);
// sizes[0] = row_ptr[n_data_rows] (ray non-zeros), sizes[1] = sizes[0] + tk_entries
cudaError_t csr_sizes(const int *row_ptr, int n_data_rows, long long tk_entries, long long *sizes, cudaStream_t st);
cudaError_t tk_rows(int n_data_rows, const long long *sizes, int n_model, int tk_order, const float *coef, int *row_ptr,
                    int *cols, float *vals, cudaStream_t st);
cudaError_t sort_tail(int *keys, int *pos, const long long *sizes, long long cap, int ncols, cudaStream_t st);
cudaError_t csr_transpose_prepare(const int *row_ptr, const int *cols, int nrows, long long nnz, int *keys,
                                  int *pos, int *rows_of, cudaStream_t st);
// CUB device-wide primitives (temp == nullptr queries *temp_bytes).
cudaError_t scan_exclusive(const int *in, int *out, int n, void *temp, size_t *temp_bytes, cudaStream_t st);
cudaError_t reduce_min(const float *in, float *out, size_t n, void *temp, size_t *temp_bytes, cudaStream_t st);
// order[0..n) = ray indices shot by shot (rays ray = shot * nrec + receiver), by descending
// receiver time within a shot (temp == nullptr queries *temp_bytes)
cudaError_t ray_order(const float *t_recv, unsigned *keys, unsigned *keys_out, int *vals, int *order, int n,
                      int nrec, void *temp, size_t *temp_bytes, cudaStream_t st);
cudaError_t sort_pairs(const int *keys_in, int *keys_out, const int *vals_in, int *vals_out, long long n, int key_bits,
                       void *temp, size_t *temp_bytes, cudaStream_t st);
cudaError_t csr_transpose_finish(const int *sorted_pos, const int *rows_of, const float *vals, const long long *sizes,
                                 long long cap, int ncols, const int *sorted_keys, int *t_ptr, int *t_rows,
                                 float *t_vals, cudaStream_t st);

}  // namespace tomo
