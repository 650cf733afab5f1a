// CGLS for the Tikhonov-regularised tomography system A x = B on the device (sm_100a).
//
// Same recurrence as Least_squares::sparse_cgls (src/tomography/least_squares/
// least_squares.cpp:424-496) -- s = B, r = A's, p = r, q = A p, then per iteration
// a = r'r/q'q, x += a p, s -= a q, r = A's, b = r'r/r'r_old, p = r + b p, q = A p --
// with the FP32 matrix in CSR (A) and CSR of the transpose (A', so both
// products are gathers, no atomics), and FP64 for every inner product, the step lengths
// and the row sums.  One cooperative persistent launch runs all iterations; the four
// grid-wide dependencies per iteration are software grid barriers with bounded waits.
// Reductions are deterministic: fixed row-to-thread mapping, fixed-order block and grid
// sums computed identically by every block.
//
// A' has very uneven rows: a model cell is crossed by anything from no ray to thousands
// (config 3: median 3 non-zeros, maximum 3,206; config 5: 778 on average).  Rows longer
// than long_row_limit -- 8 x the mean row length, at least kLongRow -- are listed once per
// call (cgls_long_rows, in row order) and each is summed by a whole block; the 32-lane
// groups take the rest, so the longest row no longer sets the length of A's.  A fixed
// limit of kLongRow sent nearly every config-5 row to a block, one row at a time per block:
// 2.26 ms per iteration there against 1.83 ms with the relative limit and the unrolled
// gathers (config 3: 0.111 -> 0.094 ms).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"
#include "cgls.cuh"

namespace tomo {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kLongRow = 256;  // A' rows with more non-zeros are summed by a whole block

// Block-wide FP64 sum in a fixed order; result valid in every thread.
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < kWarps; i++) t += sh[i];
    return t;
}

// Sum of the per-block partials (same order in every block).
__device__ __forceinline__ double grid_sum(const double *partials, int nb, double *sh)
{
    double v = 0.0;
    if (threadIdx.x < 32) {
        for (int i = threadIdx.x; i < nb; i += 32) v += __ldcg(partials + i);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        if (threadIdx.x == 0) sh[kWarps] = v;
    }
    __syncthreads();
    v = sh[kWarps];
    __syncthreads();
    return v;
}

// Rows of A' longer than this are summed by whole blocks (t_ptr[M] = the non-zero count).
__device__ __forceinline__ int long_row_limit(const int *t_ptr, int M)
{
    const long long mean8 = 8ll * t_ptr[M] / (M > 0 ? M : 1);
    return mean8 > kLongRow ? (int)mean8 : kLongRow;
}

// y = M x for a CSR matrix with `G` lanes per row: FP32 matrix values, FP64 vectors and
// row sums.  Returns this thread's share of y'y.  kSkipLong: rows longer than long_row
// are left to spmv_long.  The gathers are unrolled 4 deep (same summation order).
template <int G, bool kSkipLong = false>
__device__ __forceinline__ double spmv(const int *ptr, const int *idx, const float *val, const double *x, double *y,
                                       int nrows, int long_row = 0)
{
    const int lane = threadIdx.x & 31;
    const int sub = lane % G;
    const long long gthread = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long groups = (long long)gridDim.x * blockDim.x / G;
    const long long iters = (nrows + groups - 1) / groups;  // warp-uniform trip count
    double local = 0.0;
    for (long long it = 0; it < iters; it++) {
        const long long row = gthread / G + it * groups;
        double acc = 0.0;
        bool mine = row < nrows;
        if (mine) {
            const int b = __ldg(ptr + row), e = __ldg(ptr + row + 1);
            mine = !kSkipLong || e - b <= long_row;
            if (mine) {
#pragma unroll 4
                for (int k = b + sub; k < e; k += G) acc += (double)__ldg(val + k) * __ldcg(x + __ldg(idx + k));
            }
        }
        for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o, G);
        if (mine && sub == 0) {
            y[row] = acc;
            local += acc * acc;
        }
    }
    return local;
}

// The listed long rows of y = M x, one block per row (block i takes rows i, i + grid, ...
// of the list).  Returns this thread's share of y'y (thread 0 holds it).
__device__ __forceinline__ double spmv_long(const int *ptr, const int *idx, const float *val, const double *x,
                                            double *y, const int *rows, const int *nrows_long, double *sh)
{
    double local = 0.0;
    const int nl = __ldcg(nrows_long);
    for (int i = blockIdx.x; i < nl; i += gridDim.x) {
        const int row = __ldcg(rows + i);
        const int b = __ldg(ptr + row), e = __ldg(ptr + row + 1);
        double acc = 0.0;
        for (int k = b + (int)threadIdx.x; k < e; k += blockDim.x)
            acc += (double)__ldg(val + k) * __ldcg(x + __ldg(idx + k));
        acc = block_sum(acc, sh);
        if (threadIdx.x == 0) {
            y[row] = acc;
            local += acc * acc;
        }
    }
    return local;
}

// r = A' s: long rows by blocks, the rest by 32-lane groups.
__device__ __forceinline__ double spmv_t(const CglsLaunch &p, const double *x, double *y, double *sh)
{
    const double l = spmv_long(p.t_ptr, p.t_idx, p.t_val, x, y, p.long_rows, p.n_long, sh);
    return l + spmv<32, true>(p.t_ptr, p.t_idx, p.t_val, x, y, p.M, long_row_limit(p.t_ptr, p.M));
}

}  // namespace

__global__ void __launch_bounds__(kThreads) k_cgls(CglsLaunch p)
{
    __shared__ double sh[kWarps + 1];
    const int nb = gridDim.x;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nth = (long long)gridDim.x * blockDim.x;
    double *pa = p.partials, *pb = p.partials + nb, *pc = p.partials + 2 * nb;

    // s = B, x = 0
    for (long long i = tid; i < p.N; i += nth) p.s[i] = (double)p.B[i];
    for (long long i = tid; i < p.M; i += nth) p.x[i] = 0.0;
    if (!grid_barrier(p.ctrl, p.spin_limit)) return;
    // r = A' s
    double v = block_sum(spmv_t(p, p.s, p.r, sh), sh);
    if (threadIdx.x == 0) pa[blockIdx.x] = v;
    if (!grid_barrier(p.ctrl, p.spin_limit)) return;
    // p = r, q = A r (= A p)
    for (long long i = tid; i < p.M; i += nth) p.p[i] = p.r[i];
    v = block_sum(spmv<8>(p.a_ptr, p.a_idx, p.a_val, p.r, p.q, p.N), sh);
    if (threadIdx.x == 0) pb[blockIdx.x] = v;
    if (!grid_barrier(p.ctrl, p.spin_limit)) return;
    double rTr = grid_sum(pa, nb, sh);
    double qTq = grid_sum(pb, nb, sh);

    for (int it = 0; it < p.nit; it++) {
        const double a = rTr / qTq;
        double ss = 0.0;
        for (long long i = tid; i < p.M; i += nth) p.x[i] += a * __ldcg(p.p + i);
        for (long long i = tid; i < p.N; i += nth) {
            const double si = __ldcg(p.s + i) - a * __ldcg(p.q + i);
            p.s[i] = si;
            ss += si * si;
        }
        v = block_sum(ss, sh);
        if (threadIdx.x == 0) pc[blockIdx.x] = v;
        if (!grid_barrier(p.ctrl, p.spin_limit)) return;
        if (p.hist) {
            const double sn = grid_sum(pc, nb, sh);
            if (blockIdx.x == 0 && threadIdx.x == 0) p.hist[it] = sqrt(sn);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) p.ctrl[kRounds] = (unsigned)(it + 1);
        // sparse_cgls_gpu's exit test on the r of this iteration (src/utils/cgls/cgls.cu:102)
        if (p.tol > 0.0 && sqrt(rTr) < p.tol) break;
        // r = A' s
        v = block_sum(spmv_t(p, p.s, p.r, sh), sh);
        if (threadIdx.x == 0) pa[blockIdx.x] = v;
        if (!grid_barrier(p.ctrl, p.spin_limit)) return;
        const double rTr_new = grid_sum(pa, nb, sh);
        const double b = rTr_new / rTr;
        rTr = rTr_new;
        for (long long i = tid; i < p.M; i += nth) p.p[i] = __ldcg(p.r + i) + b * __ldcg(p.p + i);
        if (!grid_barrier(p.ctrl, p.spin_limit)) return;
        // q = A p
        v = block_sum(spmv<8>(p.a_ptr, p.a_idx, p.a_val, p.p, p.q, p.N), sh);
        if (threadIdx.x == 0) pb[blockIdx.x] = v;
        if (!grid_barrier(p.ctrl, p.spin_limit)) return;
        qTq = grid_sum(pb, nb, sh);
    }
    // the model update consumes the solution in FP32, as the reference's xdm
    for (long long i = tid; i < p.M; i += nth) p.x32[i] = (float)p.x[i];
}

cudaError_t cgls_grid(int *grid)
{
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cgls, kThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *grid = nsm * (per_sm < 4 ? per_sm : 4);
    return cudaSuccess;
}

namespace {
struct IsLongRow {
    const int *ptr;
    int M;
    __device__ bool operator()(int r) const { return ptr[r + 1] - ptr[r] > long_row_limit(ptr, M); }
};
}  // namespace

cudaError_t cgls_long_rows(const int *t_ptr, int M, int *rows, int *n_long, void *temp, size_t *temp_bytes,
                           cudaStream_t st)
{
    return cub::DeviceSelect::If(temp, *temp_bytes, thrust::counting_iterator<int>(0), rows, n_long, M,
                                 IsLongRow{t_ptr, M}, st);
}

cudaError_t cgls_run(const CglsLaunch &p, int grid, cudaStream_t st)
{
    CglsLaunch pp = p;
    void *args[] = {&pp};
    return cudaLaunchCooperativeKernel((const void *)k_cgls, dim3(grid), dim3(kThreads), args, 0, st);
}

}  // namespace tomo
