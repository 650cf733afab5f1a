// Ray tracing through the device-resident traveltime fields into the sparse Frechet
// matrix G, the Tikhonov rows and the transposed matrix (sm_100a).
//
// One thread marches one ray (rows are independent, as in the reference's per-receiver
// loop, src/tomography/least_squares/least_squares.cpp:205-279).  The FP32 arithmetic of
// the march, the binning and the run-length values is restated operation for operation
// with round-to-nearest intrinsics, so with the same traveltime field the Jacobian is
// bit-identical to the reference's COO (iG, jG, vG).  Cells are run-length encoded while
// marching (a ray re-enters a cell rarely), then sorted per ray, which is the reference's
// std::sort + run-length pass without materialising one index per step.
#include <cub/cub.cuh>

#include "common.cuh"
#include "ray.cuh"

namespace tomo {

namespace {

// Traveltime of window-local node (z, x, y) of shot d (brick-major pool).
__device__ __forceinline__ float t_node(const float *T, const ShotDesc &d, int x, int y, int z)
{
    const long long b = (z >> 2) + (long long)d.nbz * ((x >> 2) + (long long)d.nbx * (y >> 2));
    return __ldg(T + d.t_off + b * kBrickNodes + (z & 3) + 4 * (x & 3) + 16 * (y & 3));
}

// expand_fdm (least_squares.cpp:11-67) adds a replicated one-node halo: expanded index
// (i, j, k) reads the cropped node (i-1, j-1, k-1) clamped into the field.  Beyond the
// halo (undefined in the reference) the clamp continues.
__device__ __forceinline__ float t_exp(const float *T, const ShotDesc &d, int nz, int i, int j, int k)
{
    const int z = min(max(i - 1, 0), nz - 1);
    const int x = min(max(j - 1, 0), d.wnx - 1);
    const int y = min(max(k - 1, 0), d.wny - 1);
    return t_node(T, d, x, y, z);
}

__device__ __forceinline__ int trunc_div(float a, float b) { return (int)fdiv(a, b); }

// A window-local node's offset in its shot's brick-major field is a sum of one part per
// axis (t_node's brick index times 64 plus the node in the brick, split by axis).
__device__ __forceinline__ int zpart(int z) { return ((z >> 2) << 6) + (z & 3); }
__device__ __forceinline__ int xpart(const ShotDesc &d, int x) { return (((x >> 2) * d.nbz) << 6) + 4 * (x & 3); }
__device__ __forceinline__ long long ypart(const ShotDesc &d, int y)
{
    return (((long long)(y >> 2) * d.nbz * d.nbx) << 6) + 16 * (y & 3);
}

// The six axis neighbours of expanded node (i, j, k), each read as t_exp reads it (clamped
// per axis), from nine per-axis parts instead of six full index computations.
__device__ __forceinline__ void t_stencil(const float *T, const ShotDesc &d, int nz, int i, int j, int k, float &zm,
                                          float &zp, float &xm, float &xp, float &ym, float &yp)
{
    const float *Tb = T + d.t_off;
    const int z0 = i - 1, x0 = j - 1, y0 = k - 1;
    const int Zc = zpart(min(max(z0, 0), nz - 1)), Zm = zpart(min(max(z0 - 1, 0), nz - 1)),
              Zp = zpart(min(max(z0 + 1, 0), nz - 1));
    const int Xc = xpart(d, min(max(x0, 0), d.wnx - 1)), Xm = xpart(d, min(max(x0 - 1, 0), d.wnx - 1)),
              Xp = xpart(d, min(max(x0 + 1, 0), d.wnx - 1));
    const long long Yc = ypart(d, min(max(y0, 0), d.wny - 1)), Ym = ypart(d, min(max(y0 - 1, 0), d.wny - 1)),
                    Yp = ypart(d, min(max(y0 + 1, 0), d.wny - 1));
    zm = __ldg(Tb + Yc + (Zm + Xc));
    zp = __ldg(Tb + Yc + (Zp + Xc));
    xm = __ldg(Tb + Yc + (Zc + Xm));
    xp = __ldg(Tb + Yc + (Zc + Xp));
    ym = __ldg(Tb + Ym + (Zc + Xc));
    yp = __ldg(Tb + Yp + (Zc + Xc));
}

}  // namespace

__global__ void __launch_bounds__(128) k_ray_march(RayLaunch p)
{
    const long long nrays = (long long)p.nshots * p.nrec;
    const float rayStep = fmul(0.2f, p.dz);  // least_squares.cpp:203
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrays;
         t += (long long)gridDim.x * blockDim.x) {
        // march order (ray_order): shot by shot, longest (largest receiver time) first
        // within a shot; results stay indexed by the ray itself
        const long long ray = p.order ? (long long)p.order[t] : t;
        const int s = (int)(ray / p.nrec), r = (int)(ray % p.nrec);
        const ShotDesc &d = p.shots[s];
        const float ox = fmul((float)d.wx0, p.dx), oy = fmul((float)d.wy0, p.dy);
        const float sxg = p.spos[s], syg = p.spos[p.nshots + s], sz = p.spos[2 * p.nshots + s];
        const float sx = fsub(sxg, ox), sy = fsub(syg, oy);
        // source cell (least_squares.cpp:197-201) and source floor node (stall guard)
        const int sId = trunc_div(sz, p.dzt) + trunc_div(sxg, p.dxt) * p.nzt + trunc_div(syg, p.dyt) * p.nxt * p.nzt;
        const int snz = trunc_div(sz, p.dz), snx = trunc_div(sx, p.dx), sny = trunc_div(sy, p.dy);

        float zi = p.rz[r], xi = fsub(p.rx[r], ox), yi = fsub(p.ry[r], oy);
        uint2 *runs = p.runs + ray * (long long)p.cap_runs;
        int nr = 0, L = 0, st = kRayCapped;
        bool overflow = false;
        unsigned cur = 0xffffffffu, cnt = 0;
        int ci = -1;  // run that collects the steps in cell `cur`
        // The four cells most recently entered and their runs: a ray running along a cell
        // face alternates between two or three cells, and their steps go to one run each
        // instead of a new run per re-entry (the per-cell totals are the same).
        unsigned c0 = 0xffffffffu, c1 = 0xffffffffu, c2 = 0xffffffffu, c3 = 0xffffffffu;
        int r0 = -1, r1 = -1, r2 = -1, r3 = -1;
        if (xi < 0.0f || yi < 0.0f || xi > fmul((float)(d.wnx - 1), p.dx) || yi > fmul((float)(d.wny - 1), p.dy)) {
            st = kRayOutside;  // receiver outside this shot's window
            L = p.max_steps;   // skip the march
        }
        // grid node of the current position (least_squares.cpp:215-217 less the halo offset):
        // the stall test of one step and the gradient stencil of the next use the same one
        int iz = trunc_div(zi, p.dz), ix = trunc_div(xi, p.dx), iy = trunc_div(yi, p.dy);
        int cap = p.max_steps;
        if (p.smin && L == 0) {
            const float t0 = t_exp(p.T, d, p.nz, iz + 1, ix + 1, iy + 1);
            const float smin = *p.smin;
            if (smin > 0.0f) {
                const float c = t0 * (p.length_factor / (smin * rayStep)) + 256.0f;
                if (c < (float)cap) cap = (int)c;
            }
        }
        const float two_dz = fmul(2.0f, p.dz), two_dx = fmul(2.0f, p.dx), two_dy = fmul(2.0f, p.dy);
        while (L < cap) {
            const int i = iz + 1, j = ix + 1, k = iy + 1;
            float tzm, tzp, txm, txp, tym, typ;
            t_stencil(p.T, d, p.nz, i, j, k, tzm, tzp, txm, txp, tym, typ);
            const float dTz = fdiv(fsub(tzp, tzm), two_dz);
            const float dTx = fdiv(fsub(txp, txm), two_dx);
            const float dTy = fdiv(fsub(typ, tym), two_dy);
            const float norm = __fsqrt_rn(fadd(fadd(fmul(dTx, dTx), fmul(dTy, dTy)), fmul(dTz, dTz)));
            zi = fsub(zi, fdiv(fmul(rayStep, dTz), norm));
            xi = fsub(xi, fdiv(fmul(rayStep, dTx), norm));
            yi = fsub(yi, fdiv(fmul(rayStep, dTy), norm));
            if (!isfinite(zi) || !isfinite(xi) || !isfinite(yi)) {
                st = kRayNonFinite;
                break;
            }
            iz = trunc_div(zi, p.dz);
            ix = trunc_div(xi, p.dx);
            iy = trunc_div(yi, p.dy);
            const int im = trunc_div(zi, p.dzt), jm = trunc_div(fadd(xi, ox), p.dxt), km = trunc_div(fadd(yi, oy), p.dyt);
            if (im < 0 || im >= p.nzt || jm < 0 || jm >= p.nxt || km < 0 || km >= p.nyt) {
                st = kRayOutside;
                break;
            }
            const unsigned cell = (unsigned)(im + jm * p.nzt + km * p.nxt * p.nzt);
            ++L;
            if (cell == cur) {
                ++cnt;
            } else {
                if (cnt && ci >= 0) runs[ci].y += cnt;
                int hit = cell == c0 ? r0 : cell == c1 ? r1 : cell == c2 ? r2 : cell == c3 ? r3 : -1;
                if (hit < 0) {
                    if (nr < p.cap_runs) {
                        runs[nr] = make_uint2(cell, 0u);
                        hit = nr++;
                        c3 = c2; r3 = r2;
                        c2 = c1; r2 = r1;
                        c1 = c0; r1 = r0;
                        c0 = cell; r0 = hit;
                    } else {
                        overflow = true;
                    }
                }
                ci = hit;
                cur = cell;
                cnt = 1;
            }
            if (p.illum) {  // expanded (i,j,k) with cropped strides (least_squares.cpp:234)
                const long long li = i + (long long)j * p.nz + (long long)k * p.model_nx * p.nz;
                if (li >= 0 && li < (long long)p.nz * p.model_nx * p.model_ny) atomicAdd(p.illum + li, rayStep);
            }
            if ((int)cell == sId) {
                st = kRayOk;
                break;
            }
            if (iz == snz && ix == snx && iy == sny) {
                st = kRayStalled;
                break;
            }
        }
        if (cnt && ci >= 0) runs[ci].y += cnt;
        if (overflow) {
            st = kRayOverflow;
            nr = 0;
        }
        p.nuniq[ray] = nr;  // raw run count; k_ray_sort sorts, merges and rewrites it
        p.status[ray] = st;
        p.steps[ray] = L;
        const float ez = fsub(zi, sz), ex = fsub(xi, sx), ey = fsub(yi, sy);
        p.final_dist[ray] = __fsqrt_rn(fadd(fadd(fmul(ez, ez), fmul(ex, ex)), fmul(ey, ey)));
    }
}


// Sorts each ray's runs by cell and merges repeated cells -- the reference's std::sort of
// the step cells and run-length count (least_squares.cpp:241-263), on the runs recorded
// while marching.  One warp per ray: a bitonic sort in shared memory over the next power
// of two of the run count, then one lane merges equal cells (their step counts add).
// Rays with more runs than the shared buffer (possible only with max_cells_per_ray > 1024)
// are sorted by one lane in place.
constexpr int kSortWarps = 4;
constexpr int kSortCap = 1024;

__global__ void __launch_bounds__(32 * kSortWarps) k_ray_sort(RayLaunch p)
{
    __shared__ uint2 sbuf[kSortWarps][kSortCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint2 *buf = sbuf[warp];
    const long long nrays = (long long)p.nshots * p.nrec;
    for (long long ray = blockIdx.x * (long long)kSortWarps + warp; ray < nrays;
         ray += (long long)gridDim.x * kSortWarps) {
        uint2 *runs = p.runs + ray * (long long)p.cap_runs;
        const int n = p.nuniq[ray];
        if (n <= 1) continue;
        if (n > kSortCap) {
            if (lane == 0) {
                for (int a = 1; a < n; a++) {
                    const uint2 key = runs[a];
                    int b = a - 1;
                    while (b >= 0 && runs[b].x > key.x) {
                        runs[b + 1] = runs[b];
                        --b;
                    }
                    runs[b + 1] = key;
                }
                int w = 0;
                for (int a = 0; a < n; a++) {
                    const uint2 e = runs[a];
                    if (w > 0 && runs[w - 1].x == e.x) runs[w - 1].y += e.y;
                    else runs[w++] = e;
                }
                p.nuniq[ray] = w;
            }
            __syncwarp();
            continue;
        }
        int P = 2;
        while (P < n) P <<= 1;
        for (int i = lane; i < P; i += 32) buf[i] = i < n ? runs[i] : make_uint2(0xffffffffu, 0u);
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const uint2 a = buf[i], b = buf[ixj];
                        if ((a.x > b.x) == ((i & k) == 0)) {
                            buf[i] = b;
                            buf[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        // Merge equal cells, 32 sorted entries at a time: an entry that starts a new cell sums
        // the step counts of the equal entries after it (integers: the order does not matter)
        // and goes to the slot that the cells before it leave.
        int w = 0;
        for (int b = 0; b < n; b += 32) {
            const int i = b + lane;
            const uint2 e = i < n ? buf[i] : make_uint2(0xffffffffu, 0u);
            const bool head = i < n && (i == 0 || buf[i - 1].x != e.x);
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (head) {
                unsigned y = e.y;
                for (int j = i + 1; j < n && buf[j].x == e.x; ++j) y += buf[j].y;
                runs[w + __popc(hm & ((1u << lane) - 1u))] = make_uint2(e.x, y);
            }
            w += __popc(hm);
        }
        if (lane == 0) p.nuniq[ray] = w;
        __syncwarp();
    }
}

// Values of the run-length entries: the reference accumulates rayStep once per step by
// repeated FP32 addition, starting from rayStep; the first (smallest) cell gets one extra
// step and the source cell gets the final distance to the source (:243-276).
// One warp per ray, a lane per run: each run's chain of additions is its own, so the values
// are those of a serial pass, and the run reads and row writes are contiguous.
__global__ void __launch_bounds__(128) k_ray_emit(RayLaunch p, const int *row_ptr, int *cols, float *vals)
{
    const long long nrays = (long long)p.nshots * p.nrec;
    const float rayStep = fmul(0.2f, p.dz);
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long ray = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; ray < nrays; ray += nwarps) {
        const int s = (int)(ray / p.nrec);
        const float sxg = p.spos[s], syg = p.spos[p.nshots + s], sz = p.spos[2 * p.nshots + s];
        const int sId = trunc_div(sz, p.dzt) + trunc_div(sxg, p.dxt) * p.nzt + trunc_div(syg, p.dyt) * p.nxt * p.nzt;
        const uint2 *runs = p.runs + ray * (long long)p.cap_runs;
        const int n = p.nuniq[ray];
        const int base = row_ptr[ray];
        const float fd = p.final_dist[ray];
        for (int k = lane; k < n; k += 32) {
            const uint2 e = runs[k];
            float v = rayStep;
            const unsigned adds = (k == 0) ? e.y : e.y - 1u;
            for (unsigned t = 0; t < adds; t++) v = fadd(v, rayStep);
            cols[base + k] = (int)e.x;
            vals[base + k] = ((int)e.x == sId) ? fd : v;
        }
    }
}

// Least_squares::tk_reg_matrix (:358-422): row n_data + t holds lambda*df[k] at column t+k.
// sizes[0] = ray non-zeros (the scan total), sizes[1] = all non-zeros with the Tikhonov rows
__global__ void k_csr_sizes(const int *row_ptr, int n_data_rows, long long tk_entries, long long *sizes)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sizes[0] = row_ptr[n_data_rows];
        sizes[1] = sizes[0] + tk_entries;
    }
}

__global__ void k_tk_rows(int n_data_rows, const long long *sizes, int n_model, int tk_order, const float *coef,
                          int *row_ptr, int *cols, float *vals)
{
    const long long nnz_g = sizes[0];
    const int e = tk_order + 1;
    const int nL = n_model - tk_order;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= nL; t += gridDim.x * blockDim.x) {
        row_ptr[n_data_rows + t] = (int)(nnz_g + (long long)e * t);
        if (t < nL)
            for (int k = 0; k < e; k++) {
                cols[nnz_g + (long long)e * t + k] = t + k;
                vals[nnz_g + (long long)e * t + k] = coef[k];
            }
    }
}

// One warp per row, lanes over its entries (contiguous stores).
__global__ void k_transpose_prepare(const int *row_ptr, const int *cols, int nrows, int *keys, int *pos, int *rows_of)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrows; r += nwarps) {
        const int e = row_ptr[r + 1];
        for (int k = row_ptr[r] + lane; k < e; k += 32) {
            keys[k] = cols[k];
            pos[k] = k;
            rows_of[k] = (int)r;
        }
    }
}

// Sort padding: entries [nnz, cap) get the key ncols (after every column) and their own
// position, so a sort over a fixed capacity leaves the real entries in front, in order.
__global__ void k_sort_tail(int *keys, int *pos, const long long *sizes, long long cap, int ncols)
{
    for (long long k = sizes[1] + blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cap;
         k += (long long)gridDim.x * blockDim.x) {
        keys[k] = ncols;
        pos[k] = (int)k;
    }
}

__global__ void k_transpose_finish(const int *sorted_pos, const int *rows_of, const float *vals,
                                   const long long *sizes, int ncols, const int *sorted_keys, int *t_ptr, int *t_rows,
                                   float *t_vals)
{
    const long long nnz = sizes[1];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
        const int src = sorted_pos[k];
        t_rows[k] = rows_of[src];
        t_vals[k] = vals[src];
        const int c = sorted_keys[k];
        const int prev = (k == 0) ? -1 : sorted_keys[k - 1];
        for (int q = prev + 1; q <= c; q++) t_ptr[q] = (int)k;
        if (k == nnz - 1)
            for (int q = c + 1; q <= ncols; q++) t_ptr[q] = (int)nnz;
    }
    if (nnz == 0 && blockIdx.x == 0)
        for (int q = threadIdx.x; q <= ncols; q += blockDim.x) t_ptr[q] = 0;
}

static int grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 32) g = 148LL * 32;
    return g < 1 ? 1 : (int)g;
}

cudaError_t ray_march(const RayLaunch &p, cudaStream_t st)
{
    k_ray_march<<<grid_for((long long)p.nshots * p.nrec, 128), 128, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t ray_sort(const RayLaunch &p, cudaStream_t st)
{
    const long long nrays = (long long)p.nshots * p.nrec;
    long long g = (nrays + kSortWarps - 1) / kSortWarps;
    if (g > 148LL * 16) g = 148LL * 16;
    k_ray_sort<<<(int)(g > 0 ? g : 1), 32 * kSortWarps, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t ray_emit(const RayLaunch &p, const int *row_ptr, int *cols, float *vals, cudaStream_t st)
{
    k_ray_emit<<<grid_for(32LL * p.nshots * p.nrec, 128), 128, 0, st>>>(p, row_ptr, cols, vals);
    return cudaGetLastError();
}

cudaError_t csr_sizes(const int *row_ptr, int n_data_rows, long long tk_entries, long long *sizes, cudaStream_t st)
{
    k_csr_sizes<<<1, 32, 0, st>>>(row_ptr, n_data_rows, tk_entries, sizes);
    return cudaGetLastError();
}

cudaError_t tk_rows(int n_data_rows, const long long *sizes, int n_model, int tk_order, const float *coef, int *row_ptr,
                    int *cols, float *vals, cudaStream_t st)
{
    k_tk_rows<<<grid_for(n_model + 1, 256), 256, 0, st>>>(n_data_rows, sizes, n_model, tk_order, coef, row_ptr, cols,
                                                          vals);
    return cudaGetLastError();
}

cudaError_t sort_tail(int *keys, int *pos, const long long *sizes, long long cap, int ncols, cudaStream_t st)
{
    k_sort_tail<<<grid_for(cap > 0 ? cap : 1, 256), 256, 0, st>>>(keys, pos, sizes, cap, ncols);
    return cudaGetLastError();
}

cudaError_t csr_transpose_prepare(const int *row_ptr, const int *cols, int nrows, long long nnz, int *keys, int *pos,
                                  int *rows_of, cudaStream_t st)
{
    (void)nnz;
    k_transpose_prepare<<<grid_for(32LL * nrows, 256), 256, 0, st>>>(row_ptr, cols, nrows, keys, pos, rows_of);
    return cudaGetLastError();
}

cudaError_t csr_transpose_finish(const int *sorted_pos, const int *rows_of, const float *vals, const long long *sizes,
                                 long long cap, int ncols, const int *sorted_keys, int *t_ptr, int *t_rows,
                                 float *t_vals, cudaStream_t st)
{
    k_transpose_finish<<<grid_for(cap > 0 ? cap : 1, 256), 256, 0, st>>>(sorted_pos, rows_of, vals, sizes, ncols,
                                                                        sorted_keys, t_ptr, t_rows, t_vals);
    return cudaGetLastError();
}

// CUB device primitives (scan, stable radix sort) used for the CSR set-up.
cudaError_t scan_exclusive(const int *in, int *out, int n, void *temp, size_t *temp_bytes, cudaStream_t st)
{
    return cub::DeviceScan::ExclusiveSum(temp, *temp_bytes, in, out, n, st);
}

// March order: shot by shot, and within a shot by descending receiver time.  The key is
// the shot index in the top shot_bits bits and the top 32 - shot_bits bits of the time
// (non-negative floats order as their bits, sign bit 0), values the ray index.  Rays of
// one shot in one warp read the same traveltime field and converge on the same source
// (1.9x faster marching on the config-5 model than one global time order, 1.3x on
// config 3); similar times keep the lanes' path lengths alike.
__global__ void k_ray_order_init(const float *t_recv, unsigned *keys, int *vals, int n, int nrec, int shot_bits)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float t = t_recv[i];
        const unsigned tb = t > 0.0f ? __float_as_uint(t) : 0u;
        keys[i] = shot_bits ? ((unsigned)(i / nrec) << (32 - shot_bits)) | (tb >> shot_bits) : tb;
        vals[i] = i;
    }
}

cudaError_t ray_order(const float *t_recv, unsigned *keys, unsigned *keys_out, int *vals, int *order, int n,
                      int nrec, void *temp, size_t *temp_bytes, cudaStream_t st)
{
    if (temp) {
        if (nrec < 1 || n % nrec) return cudaErrorInvalidValue;
        int shot_bits = 0;
        while (shot_bits < 31 && (1LL << shot_bits) < (long long)(n / nrec)) ++shot_bits;
        k_ray_order_init<<<grid_for(n, 256), 256, 0, st>>>(t_recv, keys, vals, n, nrec, shot_bits);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cub::DeviceRadixSort::SortPairsDescending(temp, *temp_bytes, keys, keys_out, vals, order, n, 0, 32, st);
}

cudaError_t reduce_min(const float *in, float *out, size_t n, void *temp, size_t *temp_bytes, cudaStream_t st)
{
    return cub::DeviceReduce::Min(temp, *temp_bytes, in, out, (long long)n, st);
}

cudaError_t sort_pairs(const int *keys_in, int *keys_out, const int *vals_in, int *vals_out, long long n, int key_bits,
                       void *temp, size_t *temp_bytes, cudaStream_t st)
{
    return cub::DeviceRadixSort::SortPairs(temp, *temp_bytes, keys_in, keys_out, vals_in, vals_out, (int)n, 0, key_bits,
                                           st);
}

}  // namespace tomo
