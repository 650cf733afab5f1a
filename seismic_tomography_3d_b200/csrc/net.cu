// Surrogate network kernels (sm_100a): the weight gradient of the 3x3x3 convolutions,
// resampling, head/loss, Adam, and the feature / target / data kernels.  The convolution
// forward (also used for dgrad, on flipped and transposed weights) runs on the tcgen05
// tensor cores (net_tc.cu).
//
// wgrad tiling.  Voxel tiles of 4 x 8 x 8 (256 voxels); the input halo of a 16-channel
// chunk (6 x 10 x 10 voxels, 32 B each) is staged in shared memory, and dW = dY^T X_shift
// is accumulated over the tiles with mma.sync.m16n8k16 (BF16 in, FP32 accumulate) and
// ldmatrix(.trans) operand loads: a tap shift is just a different row address into the
// halo.  The partial sums are added into the FP32 gradient with atomics once per CTA.
#include <cmath>

#include "net.cuh"

namespace tomo {
namespace net {

namespace {

constexpr int TD = 4, TH = 8, TW = 8;                       // output tile
constexpr int HD = TD + 2, HH = TH + 2, HW = TW + 2;        // halo tile
constexpr int kHalo = HD * HH * HW;                         // 600 voxels
constexpr int kTileVox = TD * TH * TW;                      // 256 voxels

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4_t(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct TileCoord {
    int b, d0, h0, w0;
};

__device__ __forceinline__ TileCoord tile_of(long long t, const Vol &v)
{
    const int nw = (v.W + TW - 1) / TW, nh = (v.H + TH - 1) / TH, nd = (v.D + TD - 1) / TD;
    TileCoord c;
    c.w0 = (int)(t % nw) * TW;
    t /= nw;
    c.h0 = (int)(t % nh) * TH;
    t /= nh;
    c.d0 = (int)(t % nd) * TD;
    t /= nd;
    c.b = (int)t;
    return c;
}

__host__ __device__ inline long long tiles_of(const Vol &v)
{
    return (long long)v.B * ((v.D + TD - 1) / TD) * ((v.H + TH - 1) / TH) * ((v.W + TW - 1) / TW);
}

// Channels [ci0, ci0 + 16) of the halo tile (zero outside the volume): 2 x 16 B per voxel.
__device__ __forceinline__ void stage_halo(const bf16 *x, const Vol &v, int cin, int ci0, const TileCoord &tc,
                                           uint4 *dst)
{
    for (int i = threadIdx.x; i < kHalo * 2; i += blockDim.x) {
        const int hv = i >> 1, half = i & 1;
        const int hw = hv % HW, hh = (hv / HW) % HH, hd = hv / (HW * HH);
        const int d = tc.d0 + hd - 1, h = tc.h0 + hh - 1, w = tc.w0 + hw - 1;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (d >= 0 && d < v.D && h >= 0 && h < v.H && w >= 0 && w < v.W) {
            const long long vox = (((long long)tc.b * v.D + d) * v.H + h) * v.W + w;
            val = __ldg(reinterpret_cast<const uint4 *>(x + vox * cin + ci0) + half);
        }
        dst[i] = val;
    }
}

__device__ __forceinline__ int halo_index(int m, int dd, int dh, int dw)
{
    const int ww = m % TW, wh = (m / TW) % TH, wd = m / (TW * TH);
    return ((wd + dd) * HH + (wh + dh)) * HW + (ww + dw);
}

// wgrad: 9 warps, warp w owns taps 3w .. 3w+2; CTA owns 16 input channels (blockIdx.y) and
// NM output channels (blockIdx.z), and loops over voxel tiles (blockIdx.x strided).
template <int NM>
__global__ void __launch_bounds__(288) k_conv_wgrad(const bf16 *x, const bf16 *dy, float *dw, Vol v, int cin,
                                                    int cout)
{
    constexpr int MT = NM / 16;
    constexpr int DYS = NM + 8;  // padded row (elements): ldmatrix rows fall on distinct banks
    extern __shared__ uint4 sm[];
    uint4 *s_in = sm;
    bf16 *s_dy = reinterpret_cast<bf16 *>(sm + kHalo * 2);
    const int ci0 = blockIdx.y * 16, co0 = blockIdx.z * NM;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = lane >> 3;
    float acc[3][MT][2][4];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < MT; b++)
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc[a][b][c][e] = 0.f;
    const unsigned s_in_b = smem_u32(s_in);
    const long long ntiles = tiles_of(v);
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileCoord tc = tile_of(t, v);
        __syncthreads();
        stage_halo(x, v, cin, ci0, tc, s_in);
        for (int i = threadIdx.x; i < kTileVox * (NM / 8); i += blockDim.x) {
            const int r = i / (NM / 8), part = i % (NM / 8);
            const int ww = r % TW, wh = (r / TW) % TH, wd = r / (TW * TH);
            const int d = tc.d0 + wd, h = tc.h0 + wh, ws = tc.w0 + ww;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (d < v.D && h < v.H && ws < v.W && co0 + part * 8 < cout) {
                const long long vox = (((long long)tc.b * v.D + d) * v.H + h) * v.W + ws;
                val = __ldg(reinterpret_cast<const uint4 *>(dy + vox * cout + co0 + part * 8));
            }
            *reinterpret_cast<uint4 *>(s_dy + r * DYS + part * 8) = val;
        }
        __syncthreads();
#pragma unroll 1
        for (int kk = 0; kk < kTileVox / 16; kk++) {
            unsigned a[MT][4];
#pragma unroll
            for (int mt = 0; mt < MT; mt++) {
                const int row = kk * 16 + (q >> 1) * 8 + (lane & 7);
                const int col = mt * 16 + (q & 1) * 8;
                ldsm_x4_t(smem_u32(s_dy + row * DYS + col), a[mt][0], a[mt][1], a[mt][2], a[mt][3]);
            }
            const int m = kk * 16 + (q & 1) * 8 + (lane & 7);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int tap = warp * 3 + j;
                const int hidx = halo_index(m, tap / 9, (tap / 3) % 3, tap % 3);
                unsigned b0, b1, b2, b3;
                ldsm_x4_t(s_in_b + (hidx * 16 + (q >> 1) * 8) * 2, b0, b1, b2, b3);
#pragma unroll
                for (int mt = 0; mt < MT; mt++) {
                    mma16816(acc[j][mt][0], a[mt], b0, b1);
                    mma16816(acc[j][mt][1], a[mt], b2, b3);
                }
            }
        }
    }
    const int g = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int tap = warp * 3 + j;
#pragma unroll
        for (int mt = 0; mt < MT; mt++)
#pragma unroll
            for (int nt = 0; nt < 2; nt++)
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int co = co0 + mt * 16 + g + (r >= 2 ? 8 : 0);
                    const int ci = ci0 + nt * 8 + c2 + (r & 1);
                    if (co < cout) atomicAdd(dw + ((long long)co * 27 + tap) * cin + ci, acc[j][mt][nt][r]);
                }
    }
}

__global__ void k_bias_grad(const bf16 *dy, float *db, long long n, int c)
{
    __shared__ float part[128];
    for (int i = threadIdx.x; i < c; i += blockDim.x) part[i] = 0.f;
    __syncthreads();
    const long long nth = (long long)gridDim.x * blockDim.x;
    const long long stride = nth - nth % c;  // a multiple of c: each thread keeps one channel
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t < stride) {
        float s = 0.f;
        for (long long e = t; e < n; e += stride) s += __bfloat162float(dy[e]);
        atomicAdd(&part[t % c], s);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < c; i += blockDim.x) atomicAdd(db + i, part[i]);
}

__global__ void k_flip_weights(const float *w, bf16 *wt, int cin, int cout)
{
    const long long n = (long long)cin * 27 * cout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(e % cout);
        const int tap = (int)((e / cout) % 27);
        const int ci = (int)(e / ((long long)cout * 27));
        wt[e] = __float2bfloat16_rn(w[((long long)co * 27 + (26 - tap)) * cin + ci]);
    }
}

__global__ void k_to_bf16(const float *a, bf16 *b, long long n)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        b[e] = __float2bfloat16_rn(a[e]);
}

__global__ void k_relu_bwd(const bf16 *y, bf16 *dy, long long n)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        if (!(__bfloat162float(y[e]) > 0.f)) dy[e] = __float2bfloat16_rn(0.f);
}

__global__ void k_add_into(bf16 *a, const bf16 *b, long long n)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        a[e] = __float2bfloat16_rn(__bfloat162float(a[e]) + __bfloat162float(b[e]));
}

// coarse voxel index -> its 8 fine children
__device__ __forceinline__ long long fine_index(const Vol &f, long long cv, int k)
{
    const int cw = f.W / 2, ch = f.H / 2, cd = f.D / 2;
    const int w = (int)(cv % cw);
    long long r = cv / cw;
    const int h = (int)(r % ch);
    r /= ch;
    const int d = (int)(r % cd);
    const int b = (int)(r / cd);
    return (((long long)b * f.D + 2 * d + (k >> 2)) * f.H + 2 * h + ((k >> 1) & 1)) * f.W + 2 * w + (k & 1);
}

__global__ void k_pool_fwd(const bf16 *x, bf16 *y, Vol f, int c)
{
    const long long n = f.voxels() / 8 * c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long cv = e / c;
        const int ch = (int)(e % c);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++) s += __bfloat162float(x[fine_index(f, cv, k) * c + ch]);
        y[e] = __float2bfloat16_rn(0.125f * s);
    }
}

__global__ void k_pool_bwd(const bf16 *dy, bf16 *dx, Vol f, int c)
{
    const long long n = f.voxels() / 8 * c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long cv = e / c;
        const int ch = (int)(e % c);
        const bf16 g = __float2bfloat16_rn(0.125f * __bfloat162float(dy[e]));
#pragma unroll
        for (int k = 0; k < 8; k++) dx[fine_index(f, cv, k) * c + ch] = g;
    }
}

__global__ void k_up_fwd(const bf16 *x, bf16 *y, Vol f, int c)
{
    const long long n = f.voxels() / 8 * c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long cv = e / c;
        const int ch = (int)(e % c);
        const bf16 val = x[e];
#pragma unroll
        for (int k = 0; k < 8; k++) y[fine_index(f, cv, k) * c + ch] = val;
    }
}

__global__ void k_up_bwd(const bf16 *dy, bf16 *dx, Vol f, int c)
{
    const long long n = f.voxels() / 8 * c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long cv = e / c;
        const int ch = (int)(e % c);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; k++) s += __bfloat162float(dy[fine_index(f, cv, k) * c + ch]);
        dx[e] = __float2bfloat16_rn(s);
    }
}

// 8 channels (16 B) per element
__global__ void k_concat_fwd(const uint4 *a, int ca8, const uint4 *b, int cb8, uint4 *y, long long vox)
{
    const int c8 = ca8 + cb8;
    const long long n = vox * c8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long v = e / c8;
        const int k = (int)(e % c8);
        y[e] = k < ca8 ? a[v * ca8 + k] : b[v * cb8 + (k - ca8)];
    }
}

__global__ void k_concat_bwd(const uint4 *dy, uint4 *da, int ca8, uint4 *db, int cb8, long long vox)
{
    const int c8 = ca8 + cb8;
    const long long n = vox * c8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long v = e / c8;
        const int k = (int)(e % c8);
        if (k < ca8) da[v * ca8 + k] = dy[e];
        else db[v * cb8 + (k - ca8)] = dy[e];
    }
}

__device__ __forceinline__ double block_sum(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    __syncthreads();
    return s;
}

__global__ void k_head_fwd(const bf16 *y, const float *wh, const float *bh, float *tau, const float *target,
                           long long n, int c, double *acc)
{
    __shared__ double sh[32];
    double se = 0.0, cnt = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float s = 1.0f + bh[0];
        for (int k = 0; k < c; k++) s += wh[k] * __bfloat162float(y[v * c + k]);
        tau[v] = s;
        if (target && target[v] > 0.f) {
            const double d = (double)s - (double)target[v];
            se += d * d;
            cnt += 1.0;
        }
    }
    if (!target) return;
    se = block_sum(se, sh);
    cnt = block_sum(cnt, sh);
    if (threadIdx.x == 0) {
        atomicAdd(acc, se);
        atomicAdd(acc + 1, cnt);
    }
}

__global__ void k_head_bwd(const bf16 *y, const float *wh, const float *tau, const float *target, const double *acc,
                           bf16 *dy, float *dwh, float *dbh, long long n, int c)
{
    __shared__ float sw[64];
    __shared__ float sb;
    for (int k = threadIdx.x; k < c; k += blockDim.x) sw[k] = 0.f;
    if (threadIdx.x == 0) sb = 0.f;
    __syncthreads();
    const float scale = acc[1] > 0.0 ? (float)(2.0 / acc[1]) : 0.f;
    float lb = 0.f;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const float g = target[v] > 0.f ? scale * (tau[v] - target[v]) : 0.f;
        lb += g;
        for (int k = 0; k < c; k++) {
            dy[v * c + k] = __float2bfloat16_rn(g * wh[k]);
            if (g != 0.f) atomicAdd(&sw[k], g * __bfloat162float(y[v * c + k]));
        }
    }
    atomicAdd(&sb, lb);
    __syncthreads();
    for (int k = threadIdx.x; k < c; k += blockDim.x) atomicAdd(dwh + k, sw[k]);
    if (threadIdx.x == 0) atomicAdd(dbh, sb);
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float gr = g[e];
        const float mm = b1 * m[e] + (1.f - b1) * gr;
        const float vv = b2 * v[e] + (1.f - b2) * gr * gr;
        m[e] = mm;
        v[e] = vv;
        p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

struct JobGeo {
    int y, x, z;      // clamped window node
    bool inside;
    float dist, s, s_src;
};

__device__ __forceinline__ JobGeo job_geo(const Job &j, long long i, float h)
{
    JobGeo q;
    const int w = (int)(i % j.pw);
    const long long r = i / j.pw;
    const int hh = (int)(r % j.ph), d = (int)(r / j.ph);
    const int k = j.stride;  // network voxel (d, hh, w) samples window node (k d, k hh, k w)
    q.inside = d * k < j.wny && hh * k < j.wnx && w * k < j.nz;
    q.y = min(d * k, j.wny - 1);
    q.x = min(hh * k, j.wnx - 1);
    q.z = min(w * k, j.nz - 1);
    const float ex = q.x * h - j.sx, ey = q.y * h - j.sy, ez = q.z * h - j.sz;
    q.dist = sqrtf(ex * ex + ey * ey + ez * ez);
    const long long mstride = (long long)j.nz * j.model_nx;
    q.s = __ldg(j.slow + q.z + (long long)j.nz * (j.wx0 + q.x) + mstride * (j.wy0 + q.y));
    const int sz = min((int)(j.sz / h), j.nz - 1), sx = min((int)(j.sx / h), j.wnx - 1),
              sy = min((int)(j.sy / h), j.wny - 1);
    q.s_src = __ldg(j.slow + sz + (long long)j.nz * (j.wx0 + sx) + mstride * (j.wy0 + sy));
    return q;
}

__global__ void k_features(const Job *jobs, float h, bf16 *x16)
{
    const Job j = jobs[blockIdx.y];
    const long long n = (long long)j.pd * j.ph * j.pw;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const JobGeo q = job_geo(j, i, h);
        __align__(16) bf16 f[16];
#pragma unroll
        for (int k = 0; k < 16; k++) f[k] = __float2bfloat16_rn(0.f);
        f[0] = __float2bfloat16_rn(q.s / q.s_src - 1.0f);
        f[1] = __float2bfloat16_rn(q.dist / (64.0f * h * (float)j.stride));
        uint4 *dst = reinterpret_cast<uint4 *>(x16 + (j.out_off + i) * 16);
        dst[0] = reinterpret_cast<const uint4 *>(f)[0];
        dst[1] = reinterpret_cast<const uint4 *>(f)[1];
    }
}

__global__ void k_tau_target(const Job *jobs, float h, float *tau)
{
    const Job j = jobs[blockIdx.y];
    const long long n = (long long)j.pd * j.ph * j.pw;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const JobGeo q = job_geo(j, i, h);
        float t = 0.f;
        if (q.inside && q.dist >= h) {
            const float tt = j.T[q.z + (long long)j.nz * (q.x + (long long)j.wnx * q.y)];
            t = tt / (q.s_src * q.dist);
        }
        tau[j.out_off + i] = t;
    }
}

__global__ void k_tau_to_time(const Job *jobs, float h, const float *tau, float *t_out)
{
    const Job j = jobs[blockIdx.y];
    const long long n = (long long)j.pd * j.ph * j.pw;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const JobGeo q = job_geo(j, i, h);
        if (!q.inside) continue;
        const float t = q.dist >= h ? tau[j.out_off + i] * q.s_src * q.dist : 0.f;
        t_out[j.nat_off + q.z + (long long)j.nz * (q.x + (long long)j.wnx * q.y)] = t;
    }
}

// Strided prediction: tau at every window node, trilinear between the sampled nodes (node
// c of an axis sits at min(c k, n - 1)), then T = tau s_src distance as k_tau_to_time.
__device__ __forceinline__ void axis_weight(int x, int k, int n, int &c0, int &c1, float &t)
{
    const int nc = (n + k - 1) / k;
    c0 = min(x / k, nc - 1);
    c1 = min(c0 + 1, nc - 1);
    const int p0 = c0 * k, p1 = min(c1 * k, n - 1);
    t = p1 > p0 ? (float)(x - p0) / (float)(p1 - p0) : 0.f;
}

__global__ void k_tau_to_time_strided(const Job *jobs, float h, const float *tau, float *t_out)
{
    const Job j = jobs[blockIdx.y];
    const int k = j.stride;
    const long long n = (long long)j.nz * j.wnx * j.wny;
    const int sz = min((int)(j.sz / h), j.nz - 1), sx = min((int)(j.sx / h), j.wnx - 1),
              sy = min((int)(j.sy / h), j.wny - 1);
    const float s_src =
        __ldg(j.slow + sz + (long long)j.nz * (j.wx0 + sx) + (long long)j.nz * j.model_nx * (j.wy0 + sy));
    const float *tj = tau + j.out_off;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i % j.nz);
        const long long r = i / j.nz;
        const int x = (int)(r % j.wnx), y = (int)(r / j.wnx);
        const float ex = x * h - j.sx, ey = y * h - j.sy, ez = z * h - j.sz;
        const float dist = sqrtf(ex * ex + ey * ey + ez * ez);
        float t = 0.f;
        if (dist >= h) {
            int z0, z1, x0, x1, y0, y1;
            float tz, tx, ty;
            axis_weight(z, k, j.nz, z0, z1, tz);
            axis_weight(x, k, j.wnx, x0, x1, tx);
            axis_weight(y, k, j.wny, y0, y1, ty);
            auto T = [&](int a, int b, int c) { return tj[a + (long long)j.pw * (b + (long long)j.ph * c)]; };
            const float c00 = T(z0, x0, y0) * (1.f - tz) + T(z1, x0, y0) * tz;
            const float c01 = T(z0, x0, y1) * (1.f - tz) + T(z1, x0, y1) * tz;
            const float c10 = T(z0, x1, y0) * (1.f - tz) + T(z1, x1, y0) * tz;
            const float c11 = T(z0, x1, y1) * (1.f - tz) + T(z1, x1, y1) * tz;
            const float c0 = c00 * (1.f - tx) + c10 * tx, c1 = c01 * (1.f - tx) + c11 * tx;
            t = (c0 * (1.f - ty) + c1 * ty) * s_src * dist;
        }
        t_out[j.nat_off + i] = t;
    }
}

__global__ void k_random_models(const TileModel *tiles, float *slow, int nx, int ny, int nz)
{
    const TileModel &tm = tiles[blockIdx.y];
    const long long n = (long long)tm.n * tm.n * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz);
        const long long r = i / nz;
        const int x = (int)(r % tm.n), y = (int)(r / tm.n);
        int layer = 0;
        for (int k = 0; k < tm.nlayers - 1; k++)
            if ((float)z > tm.z0[k] + tm.gx[k] * x + tm.gy[k] * y) layer = k + 1;
        float v = tm.vel[layer];
        for (int a = 0; a < tm.nanom; a++) {
            const float dx = x - tm.ax[a], dy = y - tm.ay[a], dz = z - tm.az[a];
            v *= 1.0f + tm.aamp[a] * expf(-(dx * dx + dy * dy + dz * dz) / (2.0f * tm.asig[a] * tm.asig[a]));
        }
        const int gx = tm.x0 + x, gy = tm.y0 + y;
        if (gx < nx && gy < ny) slow[z + (long long)nz * (gx + (long long)nx * gy)] = 1.0f / v;
    }
}

int grid1(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 64) g = 148LL * 64;
    return g < 1 ? 1 : (int)g;
}

template <int NM>
cudaError_t launch_wgrad(const bf16 *x, const bf16 *dy, float *dw, Vol v, int cin, int cout, cudaStream_t st)
{
    const size_t smem = (size_t)kHalo * 2 * sizeof(uint4) + (size_t)kTileVox * (NM + 8) * sizeof(bf16);
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad<NM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long nt = tiles_of(v);
    const int ny = cin / 16, nz = (cout + NM - 1) / NM;
    long long gx = (2LL * 148 + ny * nz - 1) / (ny * nz);
    if (gx > nt) gx = nt;
    if (gx < 1) gx = 1;
    k_conv_wgrad<NM><<<dim3((unsigned)gx, (unsigned)ny, (unsigned)nz), 288, smem, st>>>(x, dy, dw, v, cin, cout);
    return cudaGetLastError();
}

}  // namespace

cudaError_t conv_fwd(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout, int relu,
                     cudaStream_t st)
{
    // the tcgen05 kernel (net_tc.cu); it reproduces the earlier mma.sync kernel's outputs bit
    // for bit (same FP32 accumulation order per output) at 1.2-1.6x its speed
    return conv_fwd_tc(x, w, bias, y, v, cin, cout, relu, st);
}

cudaError_t conv_wgrad(const bf16 *x, const bf16 *dy, float *dw, Vol v, int cin, int cout, cudaStream_t st)
{
    if (cin % 16 || cout % 16 || cin < 16 || cout < 16) return cudaErrorInvalidValue;
    switch (cout >= 64 ? 64 : cout) {
    case 16: return launch_wgrad<16>(x, dy, dw, v, cin, cout, st);
    case 32: return launch_wgrad<32>(x, dy, dw, v, cin, cout, st);
    case 48: return launch_wgrad<48>(x, dy, dw, v, cin, cout, st);
    default: return launch_wgrad<64>(x, dy, dw, v, cin, cout, st);
    }
}

cudaError_t bias_grad(const bf16 *dy, float *db, long long voxels, int c, cudaStream_t st)
{
    if (c > 128) return cudaErrorInvalidValue;
    k_bias_grad<<<grid1(voxels * c / 64, 256), 256, 0, st>>>(dy, db, voxels * c, c);
    return cudaGetLastError();
}

cudaError_t flip_weights(const float *w, bf16 *wt, int cin, int cout, cudaStream_t st)
{
    k_flip_weights<<<grid1((long long)cin * 27 * cout, 256), 256, 0, st>>>(w, wt, cin, cout);
    return cudaGetLastError();
}

cudaError_t to_bf16(const float *a, bf16 *b, long long n, cudaStream_t st)
{
    k_to_bf16<<<grid1(n, 256), 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

cudaError_t relu_bwd(const bf16 *y, bf16 *dy, long long n, cudaStream_t st)
{
    k_relu_bwd<<<grid1(n, 256), 256, 0, st>>>(y, dy, n);
    return cudaGetLastError();
}

cudaError_t add_into(bf16 *a, const bf16 *b, long long n, cudaStream_t st)
{
    k_add_into<<<grid1(n, 256), 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

cudaError_t pool_fwd(const bf16 *x, bf16 *y, Vol f, int c, cudaStream_t st)
{
    if (f.D % 2 || f.H % 2 || f.W % 2) return cudaErrorInvalidValue;
    k_pool_fwd<<<grid1(f.voxels() / 8 * c, 256), 256, 0, st>>>(x, y, f, c);
    return cudaGetLastError();
}

cudaError_t pool_bwd(const bf16 *dy, bf16 *dx, Vol f, int c, cudaStream_t st)
{
    if (f.D % 2 || f.H % 2 || f.W % 2) return cudaErrorInvalidValue;
    k_pool_bwd<<<grid1(f.voxels() / 8 * c, 256), 256, 0, st>>>(dy, dx, f, c);
    return cudaGetLastError();
}

cudaError_t up_fwd(const bf16 *x, bf16 *y, Vol f, int c, cudaStream_t st)
{
    if (f.D % 2 || f.H % 2 || f.W % 2) return cudaErrorInvalidValue;
    k_up_fwd<<<grid1(f.voxels() / 8 * c, 256), 256, 0, st>>>(x, y, f, c);
    return cudaGetLastError();
}

cudaError_t up_bwd(const bf16 *dy, bf16 *dx, Vol f, int c, cudaStream_t st)
{
    if (f.D % 2 || f.H % 2 || f.W % 2) return cudaErrorInvalidValue;
    k_up_bwd<<<grid1(f.voxels() / 8 * c, 256), 256, 0, st>>>(dy, dx, f, c);
    return cudaGetLastError();
}

cudaError_t concat_fwd(const bf16 *a, int ca, const bf16 *b, int cb, bf16 *y, long long voxels, cudaStream_t st)
{
    if (ca % 8 || cb % 8) return cudaErrorInvalidValue;
    k_concat_fwd<<<grid1(voxels * (ca + cb) / 8, 256), 256, 0, st>>>(reinterpret_cast<const uint4 *>(a), ca / 8,
                                                                    reinterpret_cast<const uint4 *>(b), cb / 8,
                                                                    reinterpret_cast<uint4 *>(y), voxels);
    return cudaGetLastError();
}

cudaError_t concat_bwd(const bf16 *dy, bf16 *da, int ca, bf16 *db, int cb, long long voxels, cudaStream_t st)
{
    if (ca % 8 || cb % 8) return cudaErrorInvalidValue;
    k_concat_bwd<<<grid1(voxels * (ca + cb) / 8, 256), 256, 0, st>>>(reinterpret_cast<const uint4 *>(dy),
                                                                    reinterpret_cast<uint4 *>(da), ca / 8,
                                                                    reinterpret_cast<uint4 *>(db), cb / 8, voxels);
    return cudaGetLastError();
}

cudaError_t head_fwd(const bf16 *y, const float *wh, const float *bh, float *tau, const float *target, long long voxels,
                     int c, double *acc, cudaStream_t st)
{
    k_head_fwd<<<grid1(voxels, 256), 256, 0, st>>>(y, wh, bh, tau, target, voxels, c, acc);
    return cudaGetLastError();
}

cudaError_t head_bwd(const bf16 *y, const float *wh, const float *tau, const float *target, const double *acc, bf16 *dy,
                     float *dwh, float *dbh, long long voxels, int c, cudaStream_t st)
{
    if (c > 64) return cudaErrorInvalidValue;
    k_head_bwd<<<grid1(voxels, 256), 256, 0, st>>>(y, wh, tau, target, acc, dy, dwh, dbh, voxels, c);
    return cudaGetLastError();
}

cudaError_t adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                 int t, cudaStream_t st)
{
    const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
    k_adam<<<grid1(n, 256), 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t features(const Job *jobs, int njobs, float h, bf16 *x16, long long max_vox, cudaStream_t st)
{
    if (njobs < 1 || njobs > 65535) return cudaErrorInvalidValue;
    k_features<<<dim3((unsigned)grid1(max_vox, 256) / 8 + 1, (unsigned)njobs), 256, 0, st>>>(jobs, h, x16);
    return cudaGetLastError();
}

cudaError_t tau_target(const Job *jobs, int njobs, float h, float *tau, long long max_vox, cudaStream_t st)
{
    if (njobs < 1 || njobs > 65535) return cudaErrorInvalidValue;
    k_tau_target<<<dim3((unsigned)grid1(max_vox, 256) / 8 + 1, (unsigned)njobs), 256, 0, st>>>(jobs, h, tau);
    return cudaGetLastError();
}

cudaError_t tau_to_time(const Job *jobs, int njobs, float h, const float *tau, float *t_out, long long max_vox,
                        cudaStream_t st)
{
    if (njobs < 1 || njobs > 65535) return cudaErrorInvalidValue;
    k_tau_to_time<<<dim3((unsigned)grid1(max_vox, 256) / 8 + 1, (unsigned)njobs), 256, 0, st>>>(jobs, h, tau, t_out);
    return cudaGetLastError();
}

cudaError_t tau_to_time_strided(const Job *jobs, int njobs, float h, const float *tau, float *t_out, long long max_nat,
                                cudaStream_t st)
{
    if (njobs < 1 || njobs > 65535) return cudaErrorInvalidValue;
    k_tau_to_time_strided<<<dim3((unsigned)grid1(max_nat, 256) / 8 + 1, (unsigned)njobs), 256, 0, st>>>(jobs, h, tau,
                                                                                                        t_out);
    return cudaGetLastError();
}

cudaError_t random_models(const TileModel *tiles, int ntiles, float *slow, int nx, int ny, int nz, cudaStream_t st)
{
    if (ntiles < 1 || ntiles > 65535) return cudaErrorInvalidValue;
    k_random_models<<<dim3(64, (unsigned)ntiles), 256, 0, st>>>(tiles, slow, nx, ny, nz);
    return cudaGetLastError();
}

}  // namespace net
}  // namespace tomo
