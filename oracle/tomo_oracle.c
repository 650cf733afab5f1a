/*
 * CPU oracle for the tomography hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatements of the reference algorithms, each citing the reference
 * file:line it follows.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this code, always as the checker.  The product library never
 * links it.  Build: oracle/Makefile (-O2 -ffp-contract=off, so FP32 restatements keep
 * the reference's rounding order).
 */
#include "tomo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define O_INF 1e6f /* src/eikonal/block_FIM/cuda_kernel.cuh:7 */

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------------------
 * JW Godunov update in FP64.  Same branch structure as get_time_eikonal
 * (src/eikonal/block_FIM/cuda_kernel.cu:217-248): sort a>=b>=c, 1D, 2D, 3D candidates,
 * each accepted only if it exceeds the next-larger neighbour.
 * ---------------------------------------------------------------------------------- */
static double god_jw64(double a, double b, double c, double h, double s)
{
    double t;
    if (a < b) { t = a; a = b; b = t; }
    if (b < c) { t = b; b = c; c = t; }
    if (a < b) { t = a; a = b; b = t; }
    double ret = 1e6;
    if (c < 1e6) {
        ret = c + h * s;
        if (ret > b) {
            t = ((b + c) + sqrt(2.0 * s * s * h * h - (b - c) * (b - c))) * 0.5;
            if (t > b) ret = t;
            if (ret > a) {
                t = (a + b + c) / 3.0 +
                    sqrt(2.0 * (a * (b - a) + b * (c - b) + c * (a - c)) + 3.0 * s * s * h * h) / 3.0;
                if (t > a) ret = t;
            }
        }
    }
    return ret;
}

/* Block_FIM padding (block_FIM.cpp:142-157, expand_model :8-57): each axis padded to a
 * multiple of 4 by replicating the last sample -- equivalent to clamping the index. */
int oracle_fim_jw(int nx, int ny, int nz, float dx, float dy, float dz,
                  const float *slowness, float sx, float sy, float sz,
                  double *T_out, int max_passes, double tol)
{
    if (nx < 1 || ny < 1 || nz < 1 || !slowness || !T_out) return -1;
    const int nxx = nx + (4 - nx % 4) % 4;
    const int nyy = ny + (4 - ny % 4) % 4;
    const int nzz = nz + (4 - nz % 4) % 4;
    const long n = (long)nxx * nyy * nzz;
    float *S = (float *)malloc(sizeof(float) * n);
    double *T = (double *)malloc(sizeof(double) * n);
    if (!S || !T) { free(S); free(T); return -2; }
    for (int y = 0; y < nyy; y++)
        for (int x = 0; x < nxx; x++)
            for (int z = 0; z < nzz; z++)
                S[z + (long)x * nzz + (long)y * nxx * nzz] =
                    slowness[imin(z, nz - 1) + (long)imin(x, nx - 1) * nz + (long)imin(y, ny - 1) * nx * nz];

    /* Source seed: apply_source_time (block_FIM.cpp:305-317), one node, FP32 t0. */
    const int sidx = (int)(sx / dx), sidy = (int)(sy / dy), sidz = (int)(sz / dz);
    if (sidx < 0 || sidx >= nx || sidy < 0 || sidy >= ny || sidz < 0 || sidz >= nz) {
        free(S); free(T); return -3;
    }
    const long sid = sidz + (long)sidx * nzz + (long)sidy * nxx * nzz;
    const float ex = (float)(sidx * dx) - sx, ey = (float)(sidy * dy) - sy, ez = (float)(sidz * dz) - sz;
    const float t0 = S[sid] * sqrtf(powf(ex, 2.0f) + powf(ey, 2.0f) + powf(ez, 2.0f));
    for (long i = 0; i < n; i++) T[i] = 1e6;
    T[sid] = (double)t0;

    /* Isotropic spacing h = dx for every axis (block_FIM.cpp:173). */
    const double h = (double)dx;
    const long sxs = nzz, sys = (long)nxx * nzz;
    int pass;
    for (pass = 0; pass < max_passes; pass++) {
        double maxchg = 0.0;
        for (int oct = 0; oct < 8; oct++) {
            const int dzr = (oct & 1) ? -1 : 1, dxr = (oct & 2) ? -1 : 1, dyr = (oct & 4) ? -1 : 1;
            for (int yy = 0; yy < nyy; yy++) {
                const int y = dyr > 0 ? yy : nyy - 1 - yy;
                for (int xx = 0; xx < nxx; xx++) {
                    const int x = dxr > 0 ? xx : nxx - 1 - xx;
                    for (int zz = 0; zz < nzz; zz++) {
                        const int z = dzr > 0 ? zz : nzz - 1 - zz;
                        const long i = z + (long)x * sxs + (long)y * sys;
                        /* Missing neighbours at the grid edge act as INF: the reference
                         * uses the node itself as its halo there (cuda_kernel.cu:292-385),
                         * which can never lower the node's own value. */
                        double a = 1e6, b = 1e6, c = 1e6;
                        if (x > 0) a = T[i - sxs];
                        if (x < nxx - 1 && T[i + sxs] < a) a = T[i + sxs];
                        if (y > 0) b = T[i - sys];
                        if (y < nyy - 1 && T[i + sys] < b) b = T[i + sys];
                        if (z > 0) c = T[i - 1];
                        if (z < nzz - 1 && T[i + 1] < c) c = T[i + 1];
                        const double t = god_jw64(a, b, c, h, (double)S[i]);
                        if (t < T[i]) {
                            const double d = T[i] - t;
                            if (d > maxchg) maxchg = d;
                            T[i] = t;
                        }
                    }
                }
            }
        }
        if (maxchg <= tol) { pass++; break; }
    }
    /* reduce_model (block_FIM.cpp:59-69): crop back to nz*nx*ny. */
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++)
                T_out[z + (long)x * nz + (long)y * nx * nz] = T[z + (long)x * sxs + (long)y * sys];
    free(S);
    free(T);
    return pass;
}

/* ------------------------------------------------------------------------------------
 * trilinear (src/utils/interpolation/trilinear.cpp:3-20), FP32 reference order.
 * ---------------------------------------------------------------------------------- */
static float tri32(float c000, float c001, float c100, float c101, float c010, float c011,
                   float c110, float c111, float x0, float x1, float y0, float y1, float z0,
                   float z1, float x, float y, float z)
{
    float xd = (x - x0) / (x1 - x0);
    float yd = (y - y0) / (y1 - y0);
    float zd = (z - z0) / (z1 - z0);
    float c00 = c000 * (1 - xd) + c100 * xd;
    float c01 = c001 * (1 - xd) + c101 * xd;
    float c10 = c010 * (1 - xd) + c110 * xd;
    float c11 = c011 * (1 - xd) + c111 * xd;
    float c0 = c00 * (1 - yd) + c10 * yd;
    float c1 = c01 * (1 - yd) + c11 * yd;
    return (c0 * (1 - zd) + c1 * zd);
}

/* Flattened read with the reference's index arithmetic: an offset that runs past the
 * end of a column wraps into the next one, exactly as in the reference; past the end
 * of the array (undefined in the reference) it reads 0. */
static inline float flat_at(const float *a, long n, long i) { return (i >= 0 && i < n) ? a[i] : 0.0f; }

/* Block_FIM::write_first_arrival (block_FIM.cpp:228-262); identical in Accurate_FSM
 * (accurate_FSM.cpp:541-575). */
void oracle_first_arrival(int nx, int ny, int nz, float dx, float dy, float dz,
                          const float *T, int nrec, const float *rx, const float *ry,
                          const float *rz, float *out)
{
    const long n = (long)nx * ny * nz;
    for (int r = 0; r < nrec; r++) {
        float x = rx[r], y = ry[r], z = rz[r];
        float x0 = floorf(x / dx) * dx, y0 = floorf(y / dy) * dy, z0 = floorf(z / dz) * dz;
        float x1 = floorf(x / dx) * dx + dx, y1 = floorf(y / dy) * dy + dy, z1 = floorf(z / dz) * dz + dz;
        long id = ((int)(z / dz)) + ((long)(int)(x / dx)) * nz + ((long)(int)(y / dy)) * nx * nz;
        long nxz = (long)nx * nz;
        out[r] = tri32(flat_at(T, n, id), flat_at(T, n, id + 1), flat_at(T, n, id + nz),
                       flat_at(T, n, id + 1 + nz), flat_at(T, n, id + nxz), flat_at(T, n, id + 1 + nxz),
                       flat_at(T, n, id + nz + nxz), flat_at(T, n, id + 1 + nz + nxz),
                       x0, x1, y0, y1, z0, z1, x, y, z);
    }
}

/* ------------------------------------------------------------------------------------
 * Least_squares::ray_tracing (src/tomography/least_squares/least_squares.cpp:192-280)
 * over the +1 replicated halo of expand_fdm (:11-67), which equals clamping the index
 * into the cropped volume.  Termination adds three guards the reference lacks (it loops
 * forever in those cases): the source-node-box stall rule, a step cap and a non-finite
 * position check; such rays carry a non-zero status.
 * ---------------------------------------------------------------------------------- */
static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

static inline float texp(const float *T, int nx, int ny, int nz, int i, int j, int k)
{
    /* expanded index (i,j,k) -> cropped (i-1,j-1,k-1), clamped */
    int z = imin(imax(i - 1, 0), nz - 1), x = imin(imax(j - 1, 0), nx - 1), y = imin(imax(k - 1, 0), ny - 1);
    return T[z + (long)x * nz + (long)y * nx * nz];
}

long oracle_raytrace(int nx, int ny, int nz, float dx, float dy, float dz,
                     const float *T, float sx, float sy, float sz,
                     int nrec, const float *rx, const float *ry, const float *rz,
                     float dx_t, float dy_t, float dz_t, int nx_t, int ny_t, int nz_t,
                     int max_steps, long cap, long *row_ptr, int *cols, float *vals,
                     int *status, int *steps, float *illum)
{
    const int sIdz = (int)(sz / dz_t), sIdx = (int)(sx / dx_t), sIdy = (int)(sy / dy_t);
    const int sId = sIdz + sIdx * nz_t + sIdy * nx_t * nz_t;
    const int snz = (int)(sz / dz), snx = (int)(sx / dx), sny = (int)(sy / dy);
    const float rayStep = 0.2f * dz;
    const long npts = (long)nx * ny * nz;
    const int ncell = nx_t * ny_t * nz_t;
    int *idx = (int *)malloc(sizeof(int) * (size_t)(max_steps > 0 ? max_steps : 1));
    long nnz = 0;
    int overflow = 0;
    row_ptr[0] = 0;
    for (int ray = 0; ray < nrec; ray++) {
        float zi = rz[ray], xi = rx[ray], yi = ry[ray];
        int L = 0, st = ORACLE_RAY_CAPPED;
        while (L < max_steps) {
            int i = (int)(zi / dz) + 1, j = (int)(xi / dx) + 1, k = (int)(yi / dy) + 1;
            float dTz = (texp(T, nx, ny, nz, i + 1, j, k) - texp(T, nx, ny, nz, i - 1, j, k)) / (2.0f * dz);
            float dTx = (texp(T, nx, ny, nz, i, j + 1, k) - texp(T, nx, ny, nz, i, j - 1, k)) / (2.0f * dx);
            float dTy = (texp(T, nx, ny, nz, i, j, k + 1) - texp(T, nx, ny, nz, i, j, k - 1)) / (2.0f * dy);
            float norm = sqrtf(dTx * dTx + dTy * dTy + dTz * dTz);
            zi -= rayStep * dTz / norm;
            xi -= rayStep * dTx / norm;
            yi -= rayStep * dTy / norm;
            if (!isfinite(zi) || !isfinite(xi) || !isfinite(yi)) { st = ORACLE_RAY_NONFINITE; break; }
            int im = (int)(zi / dz_t), jm = (int)(xi / dx_t), km = (int)(yi / dy_t);
            if (im < 0 || im >= nz_t || jm < 0 || jm >= nx_t || km < 0 || km >= ny_t) {
                st = ORACLE_RAY_OUTSIDE;
                break;
            }
            int cell = im + jm * nz_t + km * nx_t * nz_t;
            idx[L++] = cell;
            if (illum) {
                long li = i + (long)j * nz + (long)k * nx * nz; /* expanded (i,j,k), cropped strides (:234) */
                if (li >= 0 && li < npts) illum[li] += rayStep;
            }
            if (cell == sId) { st = ORACLE_RAY_OK; break; }
            if ((int)(zi / dz) == snz && (int)(xi / dx) == snx && (int)(yi / dy) == sny) {
                st = ORACLE_RAY_STALLED;
                break;
            }
        }
        (void)ncell;
        if (steps) steps[ray] = L;
        float finalDist = sqrtf(powf(zi - sz, 2.0f) + powf(xi - sx, 2.0f) + powf(yi - sy, 2.0f));
        if (L > 0) {
            qsort(idx, (size_t)L, sizeof(int), cmp_int);
            int current = idx[0];
            float distance = rayStep;
            for (int q = 0; q < L; q++) {
                if (idx[q] == current) {
                    distance += rayStep;
                } else {
                    if (nnz < cap) { cols[nnz] = current; vals[nnz] = (current == sId) ? finalDist : distance; }
                    else overflow = 1;
                    nnz++;
                    distance = rayStep;
                    current = idx[q];
                }
            }
            if (nnz < cap) { cols[nnz] = current; vals[nnz] = (current == sId) ? finalDist : distance; }
            else overflow = 1;
            nnz++;
        }
        if (overflow) st = ORACLE_RAY_OVERFLOW;
        if (status) status[ray] = st;
        row_ptr[ray + 1] = nnz < cap ? nnz : cap;
    }
    free(idx);
    return overflow ? -1 : nnz;
}

/* ------------------------------------------------------------------------------------
 * Least_squares::tk_reg_matrix difference coefficients (least_squares.cpp:380-395).
 * ---------------------------------------------------------------------------------- */
void oracle_tk_coeffs(int tk_order, int *df_out)
{
    int elements = tk_order + 1;
    if (tk_order == 0) { df_out[0] = 1; return; }
    int *df = (int *)calloc(elements, sizeof(int));
    int *df1 = (int *)calloc(elements + 1, sizeof(int));
    int *df2 = (int *)calloc(elements + 1, sizeof(int));
    df[0] = -1;
    df[1] = 1;
    for (int index = 1; index < tk_order; index++) {
        for (int k = 0; k < elements; k++) {
            df2[k] = df[k];
            df1[k + 1] = df[k];
            df[k] = df1[k] - df2[k];
        }
    }
    for (int k = 0; k < elements; k++) df_out[k] = df[k];
    free(df);
    free(df1);
    free(df2);
}

/* ------------------------------------------------------------------------------------
 * Least_squares::sparse_cgls (least_squares.cpp:424-496).
 * ---------------------------------------------------------------------------------- */
void oracle_cgls_f64(int N, int M, long nnz, const int *iA, const int *jA, const float *vA,
                     const float *B, int nit, double *x, double *rnorm_hist)
{
    double *s = (double *)calloc(N, sizeof(double)), *q = (double *)calloc(N, sizeof(double));
    double *r = (double *)calloc(M, sizeof(double)), *p = (double *)calloc(M, sizeof(double));
    for (int i = 0; i < N; i++) s[i] = B[i];
    for (long i = 0; i < nnz; i++) r[jA[i]] += (double)vA[i] * s[iA[i]];
    for (int i = 0; i < M; i++) { p[i] = r[i]; x[i] = 0.0; }
    for (long i = 0; i < nnz; i++) q[iA[i]] += (double)vA[i] * p[jA[i]];
    for (int it = 0; it < nit; it++) {
        double qTq = 0.0, rTr = 0.0;
        for (int k = 0; k < N; k++) qTq += q[k] * q[k];
        for (int k = 0; k < M; k++) rTr += r[k] * r[k];
        double a = rTr / qTq;
        for (int k = 0; k < M; k++) x[k] += a * p[k];
        for (int k = 0; k < N; k++) s[k] -= a * q[k];
        double rd = rTr;
        for (int k = 0; k < M; k++) r[k] = 0.0;
        for (long k = 0; k < nnz; k++) r[jA[k]] += (double)vA[k] * s[iA[k]];
        rTr = 0.0;
        for (int k = 0; k < M; k++) rTr += r[k] * r[k];
        double b = rTr / rd;
        for (int k = 0; k < M; k++) p[k] = r[k] + b * p[k];
        for (int k = 0; k < N; k++) q[k] = 0.0;
        for (long k = 0; k < nnz; k++) q[iA[k]] += (double)vA[k] * p[jA[k]];
        if (rnorm_hist) {
            double ss = 0.0;
            for (int k = 0; k < N; k++) ss += s[k] * s[k];
            rnorm_hist[it] = sqrt(ss);
        }
    }
    free(s); free(q); free(r); free(p);
}

void oracle_cgls_f32(int N, int M, long nnz, const int *iA, const int *jA, const float *vA,
                     const float *B, int nit, float *xdm)
{
    float a, b, qTq, rTr, rd;
    float *s = (float *)calloc(N, sizeof(float)), *q = (float *)calloc(N, sizeof(float));
    float *r = (float *)calloc(M, sizeof(float)), *p = (float *)calloc(M, sizeof(float));
    for (int i = 0; i < N; i++) s[i] = B[i];
    for (long i = 0; i < nnz; i++) r[jA[i]] += vA[i] * s[iA[i]];
    for (int i = 0; i < M; i++) { p[i] = r[i]; xdm[i] = 0.0f; }
    for (long i = 0; i < nnz; i++) q[iA[i]] += vA[i] * p[jA[i]];
    for (int i = 0; i < nit; i++) {
        qTq = 0.0f;
        for (int k = 0; k < N; k++) qTq += q[k] * q[k];
        rTr = 0.0f;
        for (int k = 0; k < M; k++) rTr += r[k] * r[k];
        a = rTr / qTq;
        for (int k = 0; k < M; k++) xdm[k] += a * p[k];
        for (int k = 0; k < N; k++) s[k] -= a * q[k];
        rd = 0.0f;
        for (int k = 0; k < M; k++) rd += r[k] * r[k];
        for (int k = 0; k < M; k++) r[k] = 0.0f;
        for (long k = 0; k < nnz; k++) r[jA[k]] += vA[k] * s[iA[k]];
        rTr = 0.0f;
        for (int k = 0; k < M; k++) rTr += r[k] * r[k];
        b = rTr / rd;
        for (int k = 0; k < M; k++) p[k] = r[k] + b * p[k];
        for (int k = 0; k < N; k++) q[k] = 0.0f;
        for (long k = 0; k < nnz; k++) q[iA[k]] += vA[k] * p[jA[k]];
    }
    free(s); free(q); free(r); free(p);
}

/* ------------------------------------------------------------------------------------
 * gaussian (src/utils/smoothing/gaussian.cpp:5-73).
 * ---------------------------------------------------------------------------------- */
void oracle_gaussian(const float *input, float *output, int nx, int ny, int nz, int samples, float stdv)
{
    int init = samples / 2;
    long nPoints = (long)nx * ny * nz;
    int nKernel = samples * samples * samples;
    float pi = 4.0f * atanf(1.0f);
    float *kernel = (float *)calloc(nKernel, sizeof(float));
    for (long i = 0; i < nPoints; i++) output[i] = input[i];
    int mid = samples / 2;
    kernel[mid + mid * samples + mid * samples * samples] = 1.0f;
    if (stdv != 0.0f) {
        float sum = 0.0f;
        for (int y = -init; y <= init; y++)
            for (int x = -init; x <= init; x++)
                for (int z = -init; z <= init; z++) {
                    int index = (z + init) + (x + init) * samples + (y + init) * samples * samples;
                    kernel[index] = 1.0f / (2.0f * pi * stdv * stdv) * expf(-((x * x + y * y + z * z) / (2.0f * stdv * stdv)));
                    sum += kernel[index];
                }
        for (int i = 0; i < nKernel; i++) kernel[i] /= sum;
    }
    for (int k = init; k < ny - init; k++)
        for (int j = init; j < nx - init; j++)
            for (int i = init; i < nz - init; i++) {
                float accum = 0.0f;
                for (int yk = 0; yk < samples; yk++)
                    for (int xk = 0; xk < samples; xk++)
                        for (int zk = 0; zk < samples; zk++) {
                            int index = zk + xk * samples + yk * samples * samples;
                            long partial = (i - init + zk) + (long)(j - init + xk) * nz + (long)(k - init + yk) * nx * nz;
                            accum += input[partial] * kernel[index];
                        }
                output[i + (long)j * nz + (long)k * nx * nz] = accum;
            }
    free(kernel);
}

/* ------------------------------------------------------------------------------------
 * Least_squares::model_update (least_squares.cpp:498-570).  The interior masks are the
 * reference's hard-coded ones (:520 and :559).
 * ---------------------------------------------------------------------------------- */
void oracle_model_update(int nx, int ny, int nz, float dx, float dy, float dz,
                         float dx_t, float dy_t, float dz_t, int nx_t, int ny_t, int nz_t,
                         const float *xdm, int smooth, int samples, float stdv,
                         float *slowness, float *velocity_out)
{
    long nPoints = (long)nx * ny * nz;
    long nm = (long)nx_t * ny_t * nz_t;
    float *dm = (float *)calloc(nPoints, sizeof(float));
    for (long index = 0; index < nPoints; index++) {
        int k = (int)(index / ((long)nx * nz));
        int j = (int)(index - (long)k * nx * nz) / nz;
        int i = (int)(index - (long)j * nz - (long)k * nx * nz);
        float x = j * dx, y = k * dy, z = i * dz;
        float x0 = floorf(x / dx_t) * dx_t, y0 = floorf(y / dy_t) * dy_t, z0 = floorf(z / dz_t) * dz_t;
        float x1 = floorf(x / dx_t) * dx_t + dx_t, y1 = floorf(y / dy_t) * dy_t + dy_t, z1 = floorf(z / dz_t) * dz_t + dz_t;
        dm[index] = 0.0f;
        if ((i >= 11) && (i < nz - 2) && (j >= 15) && (j < nx - 16) && (k >= 15) && (k < ny - 16)) {
            int idz = (int)(z / dz_t), idx = (int)(x / dx_t), idy = (int)(y / dy_t);
            long m = idz + (long)idx * nz_t + (long)idy * nx_t * nz_t;
            long nzx = (long)nx_t * nz_t;
            float v = tri32(flat_at(xdm, nm, m), flat_at(xdm, nm, m + 1), flat_at(xdm, nm, m + nz_t),
                            flat_at(xdm, nm, m + 1 + nz_t), flat_at(xdm, nm, m + nzx), flat_at(xdm, nm, m + 1 + nzx),
                            flat_at(xdm, nm, m + nz_t + nzx), flat_at(xdm, nm, m + 1 + nz_t + nzx),
                            x0, x1, y0, y1, z0, z1, x, y, z);
            dm[i + (long)j * nz + (long)k * nx * nz] = v;
        }
    }
    float *update = (float *)calloc(nPoints, sizeof(float));
    if (smooth) {
        oracle_gaussian(dm, update, nx, ny, nz, samples, stdv);
        for (long index = 0; index < nPoints; index++) dm[index] = update[index];
    }
    for (long index = 0; index < nPoints; index++) {
        int k = (int)(index / ((long)nx * nz));
        int j = (int)(index - (long)k * nx * nz) / nz;
        int i = (int)(index - (long)j * nz - (long)k * nx * nz);
        if ((i >= 11) && (i < nz - 2) && (j >= 15) && (j < nx - 15) && (k >= 15) && (k < ny - 15))
            slowness[index] += dm[index];
        velocity_out[index] = 1.0f / slowness[index];
    }
    free(update);
    free(dm);
}
