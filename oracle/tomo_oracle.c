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
 * Noble-Gesret-Belayouni fast sweeping (src/eikonal/accurate_FSM/accurate_FSM.cpp),
 * FP32, same operation order as inner_sweep (:159-265).  Grid with a one-node replicated
 * halo (nzz = nz+2, ...).  Neighbour reads use the reference's flattened index, so a read
 * one past a column edge lands in the next column exactly as there; past the array end
 * (undefined in the reference) it reads 1e6.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    int nxx, nyy, nzz;
    long n;
    float dx, dy, dz, dz2i, dx2i, dy2i, dz2dx2, dz2dy2, dx2dy2, dsum;
    float *S, *T;
} Ngb;

static inline float ngb_t(const Ngb *g, long idx) { return (idx >= 0 && idx < g->n) ? g->T[idx] : 1e6f; }
#define NS(ii, jj, kk) (g->S[(ii) + (long)(jj) * g->nzz + (long)(kk) * g->nxx * g->nzz])
static inline float fmin2(float a, float b) { return a < b ? a : b; }   /* std::min(a, b) */
static inline float fmax2(float a, float b) { return a < b ? b : a; }   /* std::max(a, b) */

static int ngb_sweep_point(Ngb *g, int i, int j, int k, int sgntz, int sgntx, int sgnty)
{
    const int nxx = g->nxx, nyy = g->nyy, nzz = g->nzz;
    const long sx = nzz, sy = (long)nxx * nzz;
    const int sgnvz = sgntz == 1, sgnvx = sgntx == 1, sgnvy = sgnty == 1;
    const int i1 = i - sgnvz, j1 = j - sgnvx, k1 = k - sgnvy;
    const float tv = ngb_t(g, (i - sgntz) + j * sx + k * sy);
    const float te = ngb_t(g, i + (j - sgntx) * sx + k * sy);
    const float tn = ngb_t(g, i + j * sx + (k - sgnty) * sy);
    const float tev = ngb_t(g, (i - sgntz) + (j - sgntx) * sx + k * sy);
    const float ten = ngb_t(g, i + (j - sgntx) * sx + (k - sgnty) * sy);
    const float tnv = ngb_t(g, (i - sgntz) + j * sx + (k - sgnty) * sy);
    const float tnve = ngb_t(g, (i - sgntz) + (j - sgntx) * sx + (k - sgnty) * sy);
    const long ijk = i + j * sx + k * sy;
    const int jm = imax(j - 1, 1), jp = imin(j, nxx - 1), km = imax(k - 1, 1), kp = imin(k, nyy - 1);
    const int im = imax(i - 1, 1), ip = imin(i, nzz - 1);
    float t1D1 = tv + g->dz * fmin2(NS(i1, jm, km), fmin2(NS(i1, jm, kp), fmin2(NS(i1, jp, km), NS(i1, jp, kp))));
    float t1D2 = te + g->dx * fmin2(NS(im, j1, km), fmin2(NS(ip, j1, km), fmin2(NS(im, j1, kp), NS(ip, j1, kp))));
    float t1D3 = tn + g->dy * fmin2(NS(im, jm, k1), fmin2(NS(im, jp, k1), fmin2(NS(ip, jm, k1), NS(ip, jp, k1))));
    const float t1D = fmin2(t1D1, fmin2(t1D2, t1D3));
    float t2D1 = 1e6f, t2D2 = 1e6f, t2D3 = 1e6f, ta, tb, tc, Sref;
    const float dz2i = g->dz2i, dx2i = g->dx2i, dy2i = g->dy2i;
    Sref = fmin2(NS(i1, j1, km), NS(i1, j1, kp));
    if ((tv < te + g->dx * Sref) && (te < tv + g->dz * Sref)) {
        ta = tev + te - tv;
        tb = tev - te + tv;
        t2D1 = ((tb * dz2i + ta * dx2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dx2i) - dz2i * dx2i * (ta - tb) * (ta - tb))) / (dz2i + dx2i);
    }
    Sref = fmin2(NS(i1, jm, k1), NS(i1, jp, k1));
    if ((tv < tn + g->dy * Sref) && (tn < tv + g->dz * Sref)) {
        ta = tv - tn + tnv;
        tb = tn - tv + tnv;
        t2D2 = ((ta * dz2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dz2i + dy2i) - dz2i * dy2i * (ta - tb) * (ta - tb))) / (dz2i + dy2i);
    }
    Sref = fmin2(NS(im, j1, k1), NS(ip, j1, k1));
    if ((te < tn + g->dy * Sref) && (tn < te + g->dx * Sref)) {
        ta = te - tn + ten;
        tb = tn - te + ten;
        t2D3 = ((ta * dx2i + tb * dy2i) + sqrtf(4.0f * Sref * Sref * (dx2i + dy2i) - dx2i * dy2i * (ta - tb) * (ta - tb))) / (dx2i + dy2i);
    }
    const float t2D = fmin2(t2D1, fmin2(t2D2, t2D3));
    float t3D = 1e6f;
    Sref = NS(i1, j1, k1);
    ta = te - 0.5f * tn + 0.5f * ten - 0.5f * tv + 0.5f * tev - tnv + tnve;
    tb = tv - 0.5f * tn + 0.5f * tnv - 0.5f * te + 0.5f * tev - ten + tnve;
    tc = tn - 0.5f * te + 0.5f * ten - 0.5f * tv + 0.5f * tnv - tev + tnve;
    if (fmin2(t1D, t2D) > fmax2(tv, fmax2(te, tn))) {
        const float t2 = 9.0f * Sref * Sref * g->dsum;
        const float t3 = g->dz2dx2 * (ta - tb) * (ta - tb) + g->dz2dy2 * (tb - tc) * (tb - tc) + g->dx2dy2 * (ta - tc) * (ta - tc);
        if (t2 >= t3) {
            const float t1 = tb * dz2i + ta * dx2i + tc * dy2i;
            t3D = (t1 + sqrtf(t2 - t3)) / g->dsum;
        }
    }
    const float nv = fmin2(g->T[ijk], fmin2(t1D, fmin2(t2D, t3D)));
    const int changed = nv != g->T[ijk];
    g->T[ijk] = nv;
    return changed;
}

/* One sweep over a box of loop ranges (k outer, j, i inner), each given as first/last. */
static int ngb_sweep(Ngb *g, int sgntz, int sgntx, int sgnty, int i0, int i1, int j0, int j1, int k0, int k1)
{
    int changed = 0;
    const int di = i1 >= i0 ? 1 : -1, dj = j1 >= j0 ? 1 : -1, dk = k1 >= k0 ? 1 : -1;
    for (int k = k0; dk > 0 ? k <= k1 : k >= k1; k += dk)
        for (int j = j0; dj > 0 ? j <= j1 : j >= j1; j += dj)
            for (int i = i0; di > 0 ? i <= i1 : i >= i1; i += di) changed |= ngb_sweep_point(g, i, j, k, sgntz, sgntx, sgnty);
    return changed;
}

int oracle_fsm_ngb(int nx, int ny, int nz, float dx, float dy, float dz, const float *slowness,
                   float sx, float sy, float sz, float *T_out, int extra_full_sweeps)
{
    Ngb G, *g = &G;
    g->nxx = nx + 2;
    g->nyy = ny + 2;
    g->nzz = nz + 2;
    const int nxx = g->nxx, nyy = g->nyy, nzz = g->nzz;
    g->n = (long)nxx * nyy * nzz;
    g->S = (float *)malloc(sizeof(float) * g->n);
    g->T = (float *)malloc(sizeof(float) * g->n);
    /* expand_model (:8-60): replicate one node around (clamp) */
    for (int k = 0; k < nyy; k++)
        for (int j = 0; j < nxx; j++)
            for (int i = 0; i < nzz; i++)
                g->S[i + (long)j * nzz + (long)k * nxx * nzz] =
                    slowness[imin(imax(i - 1, 0), nz - 1) + (long)imin(imax(j - 1, 0), nx - 1) * nz +
                             (long)imin(imax(k - 1, 0), ny - 1) * nx * nz];
    const int nb = 1;
    const int sidx = (int)(sx / dx) + nb, sidy = (int)(sy / dy) + nb, sidz = (int)(sz / dz) + nb;
    const long sId = sidz + (long)sidx * nzz + (long)sidy * nxx * nzz;
    for (long q = 0; q < g->n; q++) g->T[q] = 1e6f;
    /* the source node and its 26 neighbours: analytic time with the source slowness
     * (:596-630).  As in the reference, the nodes at (z+1, x-1) and (z-1, x+1) receive each
     * other's distance (:608-609); identical for a source on a node. */
    for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++)
            for (int oz = -1; oz <= 1; oz++) {
                int fx = ox, fz = oz;
                if (oy == 0 && oz * ox == -1) {
                    fx = -ox;
                    fz = -oz;
                }
                g->T[sId + oz + (long)ox * nzz + (long)oy * nxx * nzz] =
                    g->S[sId] * sqrtf(powf(((sidx - nb) + fx) * dx - sx, 2.0f) + powf(((sidy - nb) + oy) * dy - sy, 2.0f) +
                                      powf(((sidz - nb) + fz) * dz - sz, 2.0f));
            }
    g->dx = dx;
    g->dy = dy;
    g->dz = dz;
    g->dz2i = 1.0f / (dz * dz);
    g->dx2i = 1.0f / (dx * dx);
    g->dy2i = 1.0f / (dy * dy);
    g->dz2dx2 = g->dz2i * g->dx2i;
    g->dz2dy2 = g->dz2i * g->dy2i;
    g->dx2dy2 = g->dx2i * g->dy2i;
    g->dsum = g->dz2i + g->dx2i + g->dy2i;
    /* init_sweep (:267-388): 8 sweeps anchored at the source */
    const int zA = imax(1, sidz), xA = imax(1, sidx), yA = imax(1, sidy);
    ngb_sweep(g, 1, 1, 1, zA, nzz - 1, xA, nxx - 1, yA, nyy - 1);
    ngb_sweep(g, -1, 1, 1, sidz + 1, 0, xA, nxx - 1, yA, nyy - 1);
    ngb_sweep(g, 1, 1, -1, zA, nzz - 1, xA, nxx - 1, sidy + 1, 0);
    ngb_sweep(g, -1, 1, -1, sidz + 1, 0, xA, nxx - 1, sidy + 1, 0);
    ngb_sweep(g, 1, -1, 1, zA, nzz - 1, sidx + 1, 0, yA, nyy - 1);
    ngb_sweep(g, -1, -1, 1, sidz + 1, 0, sidx + 1, 0, yA, nyy - 1);
    ngb_sweep(g, 1, -1, -1, zA, nzz - 1, sidx + 1, 0, sidy + 1, 0);
    ngb_sweep(g, -1, -1, -1, sidz + 1, 0, sidx + 1, 0, sidy + 1, 0);
    /* full_sweep (:390-511) once, then optional extra passes to the fixed point */
    int pass = -1, extra = 0;
    for (;;) {
        int ch = 0;
        ch |= ngb_sweep(g, 1, 1, 1, 1, nzz - 1, 1, nxx - 1, 1, nyy - 1);
        ch |= ngb_sweep(g, -1, 1, 1, nzz - 2, 0, 1, nxx - 1, 1, nyy - 1);
        ch |= ngb_sweep(g, 1, 1, -1, 1, nzz - 1, 1, nxx - 1, nyy - 2, 0);
        ch |= ngb_sweep(g, -1, 1, -1, nzz - 2, 0, 1, nxx - 1, nyy - 2, 0);
        ch |= ngb_sweep(g, 1, -1, 1, 1, nzz - 1, nxx - 2, 0, 1, nyy - 1);
        ch |= ngb_sweep(g, -1, -1, 1, nzz - 2, 0, nxx - 2, 0, 1, nyy - 1);
        ch |= ngb_sweep(g, 1, -1, -1, 1, nzz - 1, nxx - 2, 0, nyy - 2, 0);
        ch |= ngb_sweep(g, -1, -1, -1, nzz - 2, 0, nxx - 2, 0, nyy - 2, 0);
        pass++;
        if (pass > 0) extra++;
        if (extra_full_sweeps == 0 || (extra_full_sweeps > 0 && extra >= extra_full_sweeps) || (pass > 0 && !ch)) break;
    }
    /* reduce_model (:62-72) */
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++)
            for (int z = 0; z < nz; z++)
                T_out[z + (long)x * nz + (long)y * nx * nz] = g->T[(z + 1) + (long)(x + 1) * nzz + (long)(y + 1) * nxx * nzz];
    free(g->S);
    free(g->T);
    return extra;
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
