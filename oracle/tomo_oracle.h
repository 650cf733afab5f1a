/*
 * CPU oracle for the tomography hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatements of the reference algorithms (phbastosa/seismic_tomography_3D),
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker.  Nothing in the product library links or calls this code.
 *
 * Index convention (reference): volumes are float32, z fastest, then x, then y:
 *   idx = z + x*nz + y*nx*nz            (src/eikonal/block_FIM/block_FIM.cpp:17)
 */
#ifndef TOMO_ORACLE_H
#define TOMO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Ray status codes (shared meaning with the CUDA ray tracer). */
#define ORACLE_RAY_OK        0  /* reached the source cell (reference stop rule)          */
#define ORACLE_RAY_STALLED   1  /* entered the source node box outside the source cell     */
#define ORACLE_RAY_CAPPED    2  /* hit the step cap                                        */
#define ORACLE_RAY_NONFINITE 3  /* position became NaN/Inf (zero gradient)                 */
#define ORACLE_RAY_OUTSIDE   4  /* left the inversion grid                                 */
#define ORACLE_RAY_OVERFLOW  5  /* more entries than the caller's capacity                 */

/* Jeong-Whitaker Godunov fixed point in FP64 (Block_FIM operator, isotropic h = dx).
 * Pads to a multiple of 4 by edge replication, seeds one node, iterates Gauss-Seidel
 * sweeps in the 8 octant orders until the largest change is <= tol.
 * T_out: nz*nx*ny doubles (cropped).  Returns the number of sweep passes, <0 on error. */
int oracle_fim_jw(int nx, int ny, int nz, float dx, float dy, float dz,
                  const float *slowness, float sx, float sy, float sz,
                  double *T_out, int max_passes, double tol);

/* Noble-Gesret-Belayouni fast sweeping (Accurate_FSM, src/eikonal/accurate_FSM/
 * accurate_FSM.cpp:159-650) restated in FP32 with the reference's operation order.
 * extra_full_sweeps = 0 reproduces the reference (8 source-anchored + 8 full sweeps);
 * > 0 runs that many more full 8-octant passes, or until nothing changes (< 0: no limit).
 * T_out: nz*nx*ny floats (cropped).  Returns the number of extra passes run. */
int oracle_fsm_ngb(int nx, int ny, int nz, float dx, float dy, float dz, const float *slowness,
                   float sx, float sy, float sz, float *T_out, int extra_full_sweeps);

/* Trilinear receiver sampling of a cropped traveltime volume (Block_FIM/Accurate_FSM
 * write_first_arrival), FP32 with the reference's operation order. */
void oracle_first_arrival(int nx, int ny, int nz, float dx, float dy, float dz,
                          const float *T, int nrec, const float *rx, const float *ry,
                          const float *rz, float *out);

/* Least_squares::ray_tracing restated in FP32 (reference operation order), for one
 * shot.  Rows are ray_id + shot_id*nrec.  Per ray, entries are written in increasing
 * column order to cols/vals starting at row_ptr[ray]; row_ptr has nrec+1 entries.
 * illum (nz*nx*ny, may be NULL) accumulates rayStep per step like the reference.
 * Returns total nnz written, or -1 if cap was exceeded (status OVERFLOW set). */
long oracle_raytrace(int nx, int ny, int nz, float dx, float dy, float dz,
                     const float *T, float sx, float sy, float sz,
                     int nrec, const float *rx, const float *ry, const float *rz,
                     float dx_t, float dy_t, float dz_t, int nx_t, int ny_t, int nz_t,
                     int max_steps, long cap, long *row_ptr, int *cols, float *vals,
                     int *status, int *steps, float *illum);

/* Least_squares::tk_reg_matrix coefficients for order tk_order (df[0..tk_order]). */
void oracle_tk_coeffs(int tk_order, int *df);

/* CGLS on the COO system A x = B (Least_squares::sparse_cgls), FP64 everywhere. */
void oracle_cgls_f64(int N, int M, long nnz, const int *iA, const int *jA, const float *vA,
                     const float *B, int nit, double *x, double *rnorm_hist);

/* CGLS with the reference's exact FP32 arithmetic and loop order. */
void oracle_cgls_f32(int N, int M, long nnz, const int *iA, const int *jA, const float *vA,
                     const float *B, int nit, float *x);

/* gaussian() (src/utils/smoothing/gaussian.cpp) FP32, reference order. */
void oracle_gaussian(const float *in, float *out, int nx, int ny, int nz, int samples, float stdv);

/* Least_squares::model_update: trilinear coarse->fine inside the interior mask,
 * optional Gaussian, slowness += dm inside the mask, velocity_out = 1/slowness.
 * slowness is updated in place. */
void oracle_model_update(int nx, int ny, int nz, float dx, float dy, float dz,
                         float dx_t, float dy_t, float dz_t, int nx_t, int ny_t, int nz_t,
                         const float *xdm, int smooth, int samples, float stdv,
                         float *slowness, float *velocity_out);

#ifdef __cplusplus
}
#endif
#endif
