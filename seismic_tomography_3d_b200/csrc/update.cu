// Model update on the device (sm_100a): trilinear coarse-to-fine of the CGLS solution,
// 3D Gaussian smoothing, masked slowness update, velocity output, and the data residual.
// FP32 arithmetic follows the reference operation order with round-to-nearest intrinsics
// (no FMA contraction), so results are bit-identical to Least_squares::model_update
// (src/tomography/least_squares/least_squares.cpp:498-570) and gaussian
// (src/utils/smoothing/gaussian.cpp:5-73).
#include "cgls.cuh"
#include "common.cuh"

namespace tomo {

namespace {

__device__ __forceinline__ float flat_at(const float *a, long long n, long long i)
{
    return (i >= 0 && i < n) ? __ldg(a + i) : 0.0f;
}

int grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 32) g = 148LL * 32;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

__global__ void k_model_dm(const float *xdm, float *dm, int nx, int ny, int nz, float dx, float dy, float dz, float dxt,
                           float dyt, float dzt, int nxt, int nyt, int nzt, UpdateMasks m)
{
    const long long n = (long long)nx * ny * nz;
    const long long nm = (long long)nxt * nyt * nzt;
    for (long long index = blockIdx.x * (long long)blockDim.x + threadIdx.x; index < n;
         index += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(index / ((long long)nx * nz));
        const int j = (int)((index - (long long)k * nx * nz) / nz);
        const int i = (int)(index - (long long)j * nz - (long long)k * nx * nz);
        float v = 0.0f;
        if (i >= m.i_lo && i < nz - m.i_hi_off && j >= m.j_lo && j < nx - m.j_hi_off_dm && k >= m.k_lo &&
            k < ny - m.k_hi_off_dm) {
            const float x = fmul((float)j, dx), y = fmul((float)k, dy), z = fmul((float)i, dz);
            const float fx = floorf(fdiv(x, dxt)), fy = floorf(fdiv(y, dyt)), fz = floorf(fdiv(z, dzt));
            const float x0 = fmul(fx, dxt), y0 = fmul(fy, dyt), z0 = fmul(fz, dzt);
            const float x1 = fadd(fmul(fx, dxt), dxt), y1 = fadd(fmul(fy, dyt), dyt), z1 = fadd(fmul(fz, dzt), dzt);
            const long long im = (long long)(int)fdiv(z, dzt) + (long long)(int)fdiv(x, dxt) * nzt +
                                 (long long)(int)fdiv(y, dyt) * nxt * nzt;
            const long long sx = nzt, sy = (long long)nxt * nzt;
            v = trilinear_ref(flat_at(xdm, nm, im), flat_at(xdm, nm, im + 1), flat_at(xdm, nm, im + sx),
                              flat_at(xdm, nm, im + 1 + sx), flat_at(xdm, nm, im + sy), flat_at(xdm, nm, im + 1 + sy),
                              flat_at(xdm, nm, im + sx + sy), flat_at(xdm, nm, im + 1 + sx + sy), x0, x1, y0, y1, z0,
                              z1, x, y, z);
        }
        dm[index] = v;
    }
}

// One output node per thread; taps summed in the reference's (y, x, z) loop order.
__global__ void k_gaussian(const float *in, float *out, int nx, int ny, int nz, int samples, const float *kernel)
{
    const long long n = (long long)nx * ny * nz;
    const int init = samples / 2;
    for (long long index = blockIdx.x * (long long)blockDim.x + threadIdx.x; index < n;
         index += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(index / ((long long)nx * nz));
        const int j = (int)((index - (long long)k * nx * nz) / nz);
        const int i = (int)(index - (long long)j * nz - (long long)k * nx * nz);
        if (k < init || k >= ny - init || j < init || j >= nx - init || i < init || i >= nz - init) {
            out[index] = __ldg(in + index);
            continue;
        }
        float accum = 0.0f;
        for (int yk = 0; yk < samples; yk++)
            for (int xk = 0; xk < samples; xk++) {
                const float *row = in + (i - init) + (long long)(j - init + xk) * nz + (long long)(k - init + yk) * nx * nz;
                const float *kr = kernel + xk * samples + yk * samples * samples;
                for (int zk = 0; zk < samples; zk++) accum = fadd(accum, fmul(__ldg(row + zk), __ldg(kr + zk)));
            }
        out[index] = accum;
    }
}

__global__ void k_model_apply(float *slowness, const float *dm, float *velocity, int nx, int ny, int nz, UpdateMasks m)
{
    const long long n = (long long)nx * ny * nz;
    for (long long index = blockIdx.x * (long long)blockDim.x + threadIdx.x; index < n;
         index += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(index / ((long long)nx * nz));
        const int j = (int)((index - (long long)k * nx * nz) / nz);
        const int i = (int)(index - (long long)j * nz - (long long)k * nx * nz);
        float s = slowness[index];
        if (i >= m.i_lo && i < nz - m.i_hi_off && j >= m.j_lo && j < nx - m.j_hi_off_upd && k >= m.k_lo &&
            k < ny - m.k_hi_off_upd) {
            s = fadd(s, dm[index]);
            slowness[index] = s;
        }
        if (velocity) velocity[index] = fdiv(1.0f, s);
    }
}

// B = [dobs - dcal ; 0] and ||dobs - dcal||^2 in FP64 (one block: fixed summation order).
__global__ void k_residual_norm(const float *dobs, const float *dcal, int n, double *out)
{
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = (double)dobs[i] - (double)dcal[i];
        acc += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
        *out = t;
    }
}

__global__ void k_rhs(const float *dobs, const float *dcal, float *B, int n, int n_total)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_total; i += gridDim.x * blockDim.x)
        B[i] = i < n ? fsub(dobs[i], dcal[i]) : 0.0f;
}

cudaError_t model_dm(const float *xdm, float *dm, int nx, int ny, int nz, float dx, float dy, float dz, float dxt,
                     float dyt, float dzt, int nxt, int nyt, int nzt, UpdateMasks m, cudaStream_t st)
{
    k_model_dm<<<grid_for((long long)nx * ny * nz, 256), 256, 0, st>>>(xdm, dm, nx, ny, nz, dx, dy, dz, dxt, dyt, dzt,
                                                                       nxt, nyt, nzt, m);
    return cudaGetLastError();
}

cudaError_t gaussian_smooth(const float *in, float *out, int nx, int ny, int nz, int samples, const float *kernel,
                            cudaStream_t st)
{
    k_gaussian<<<grid_for((long long)nx * ny * nz, 256), 256, 0, st>>>(in, out, nx, ny, nz, samples, kernel);
    return cudaGetLastError();
}

cudaError_t model_apply(float *slowness, const float *dm, float *velocity, int nx, int ny, int nz, UpdateMasks m,
                        cudaStream_t st)
{
    k_model_apply<<<grid_for((long long)nx * ny * nz, 256), 256, 0, st>>>(slowness, dm, velocity, nx, ny, nz, m);
    return cudaGetLastError();
}

cudaError_t data_residual(const float *dobs, const float *dcal, float *B, int n, int n_total, double *norm2,
                          cudaStream_t st)
{
    if (B) k_rhs<<<grid_for(n_total, 256), 256, 0, st>>>(dobs, dcal, B, n, n_total);
    if (norm2) k_residual_norm<<<1, 1024, 0, st>>>(dobs, dcal, n, norm2);
    return cudaGetLastError();
}

}  // namespace tomo
