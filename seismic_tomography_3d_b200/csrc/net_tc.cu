// 3x3x3 convolution forward on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Implicit GEMM with the accumulators in tensor memory: a CTA of 4 warps owns DS slices of
// 128 output voxels -- 8 along W (the model's z) x 16 along H (x), DS consecutive along D
// (y) -- and N = NT output channels, one M128 x N accumulator per slice.  For each
// 16-channel slice of the input channels, the CTA stages into shared memory
//   * the 10 x 18 x (DS + 2) input halo, as [8-channel half][halo voxel][8 channels],
//   * the 27 taps' weights, as [tap][8-channel half][output channel][8 channels],
// both in the canonical K-major, unswizzled operand layout (8 rows x 16 B core matrices),
// and one thread issues 27 x DS tcgen05.mma (M128 x N x K16, BF16 in, FP32 accumulate):
// the weights staged once serve all DS slices.  A tap and a slice are only a different
// start address: output row (w, h) of slice s reads halo voxel
// (w + dw) + 10 (h + dh) + 180 (s + dd), so the rows of each 8-row core matrix (w = 0..7)
// are consecutive halo voxels and the core matrices (h) sit 10 voxels = 160 B apart -- the
// operand's row-group stride.  The MMAs' completion arrives on an mbarrier
// (tcgen05.commit); the epilogue reads the accumulators back with tcgen05.ld (each warp its
// 32 lanes = 32 output voxels of each slice), adds the bias, applies ReLU and stores BF16
// channels-last.
//
// Every wait is bounded: on a timeout the kernel records kConvTimeout in its error word,
// still frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "net.cuh"

namespace tomo {
namespace net {

__device__ unsigned g_conv_tc_error;  // 0, or kConvTimeout after a wait ran out

namespace {

constexpr unsigned kConvTimeout = 1u;
constexpr int TW = 8, TH = 16;                          // output tile (W, H) of one slice
constexpr int HW = TW + 2, HH = TH + 2;                 // input halo (W, H); D: DS + 2

// One 8-channel half of the input halo of a CTA with DS slices (bytes).
__host__ __device__ constexpr unsigned half_bytes(int ds) { return (unsigned)(HW * HH * (ds + 2)) * 16u; }
constexpr long long kWaitLimit = 1ll << 22;             // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle -- in 16-byte units the layout
// ((8 rows, n), 2 halves of K) : ((1, sbo), lbo) -- descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t operand_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N = n, M = 128.
__host__ __device__ constexpr uint32_t instr_desc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// 16-byte asynchronous global -> shared copy; src_bytes 0 fills the 16 bytes with zeros.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase)
{
    for (long long i = 0; i < kWaitLimit; i++) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

struct TcTile {
    int b, d0, h0, w0;
};

template <int DS>
__device__ __forceinline__ TcTile tc_tile(long long t, const Vol &v)
{
    const int nw = (v.W + TW - 1) / TW, nh = (v.H + TH - 1) / TH, nd = (v.D + DS - 1) / DS;
    TcTile c;
    c.w0 = (int)(t % nw) * TW;
    t /= nw;
    c.h0 = (int)(t % nh) * TH;
    t /= nh;
    c.d0 = (int)(t % nd) * DS;
    c.b = (int)(t / nd);
    return c;
}

template <int NT, int DS>
__global__ void __launch_bounds__(128) k_conv_fwd_tc(const bf16 *x, const bf16 *w, const float *bias, bf16 *y,
                                                     Vol v, int cin, int cout, int relu)
{
    constexpr int kHalo = HW * HH * (DS + 2);
    constexpr unsigned kHalfBytes = half_bytes(DS);
    // TMEM columns for DS accumulators of NT columns: a power of two >= 32
    constexpr uint32_t kCols = DS * NT <= 32 ? 32u : DS * NT <= 64 ? 64u : DS * NT <= 128 ? 128u : 256u;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *s_a = smem;                                  // 2 x kHalfBytes
    unsigned char *s_b = smem + 2 * kHalfBytes;                 // 27 x 2 x NT x 16 B
    uint64_t *bar = reinterpret_cast<uint64_t *>(s_b + 27 * 2 * NT * 16);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TcTile tc = tc_tile<DS>(blockIdx.x, v);
    const int co0 = blockIdx.y * NT;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t bar_a = smem_addr(bar), a_base = smem_addr(s_a), b_base = smem_addr(s_b);
    constexpr uint32_t idesc = instr_desc(NT);
    bool ok = true;
    uint32_t phase = 0;

    for (int ci0 = 0; ci0 < cin && ok; ci0 += 16) {
        // Stage the halo slice ([half][halo voxel][8 channels], zero outside the volume) and
        // the weights ([tap][half][output channel][8 channels]) with 16-byte asynchronous
        // copies, all of a thread's copies in flight at once.
        for (int i = threadIdx.x; i < kHalo * 2; i += blockDim.x) {
            const int hv = i >> 1, half = i & 1;
            const int hw = hv % HW, hh = (hv / HW) % HH, hd = hv / (HW * HH);
            const int d = tc.d0 + hd - 1, h = tc.h0 + hh - 1, ws = tc.w0 + hw - 1;
            const bool in = d >= 0 && d < v.D && h >= 0 && h < v.H && ws >= 0 && ws < v.W;
            const long long vox = in ? (((long long)tc.b * v.D + d) * v.H + h) * v.W + ws : 0;
            cp_async16(a_base + half * kHalfBytes + hv * 16, x + vox * cin + ci0 + 8 * half, in ? 16u : 0u);
        }
        for (int i = threadIdx.x; i < 27 * 2 * NT; i += blockDim.x) {
            const int co = i % NT, half = (i / NT) & 1, tap = i / (2 * NT);
            const bool in = co0 + co < cout;
            const long long src = in ? ((long long)(co0 + co) * 27 + tap) * cin + ci0 + 8 * half : 0;
            cp_async16(b_base + i * 16, w + src, in ? 16u : 0u);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        // the tensor cores read shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int tap = 0; tap < 27; tap++) {
                const int dd = tap / 9, dh = (tap / 3) % 3, dw = tap % 3;
                const uint64_t bd = operand_desc(b_base + (uint32_t)tap * 2u * NT * 16u, NT * 16u, 128u);
#pragma unroll
                for (int sl = 0; sl < DS; sl++) {
                    const uint32_t a_off = (uint32_t)(dw + HW * dh + HW * HH * (dd + sl)) * 16u;
                    const uint64_t ad = operand_desc(a_base + a_off, kHalfBytes, HW * 16u);
                    mma_bf16(tmem + (uint32_t)(sl * NT), ad, bd, idesc, (ci0 > 0 || tap > 0) ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                         : "memory");
        }
        // the next slice may overwrite the operands only once these MMAs have read them; one
        // answer for the whole block, so that no thread leaves the loop alone
        const bool done = mbar_wait(bar_a, phase);
        ok = __syncthreads_and(done) != 0;
        if (!ok && threadIdx.x == 0) atomicExch(&g_conv_tc_error, kConvTimeout);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }

    // epilogue: row m = 32 warp + lane of slice sl's accumulator is output voxel
    // (w, h, d) = (m % 8, m / 8, d0 + sl)
    const int m = 32 * warp + lane;
    const int h = tc.h0 + m / TW, ws = tc.w0 + m % TW;
#pragma unroll 1
    for (int sl = 0; sl < DS && ok; sl++) {
        const int d = tc.d0 + sl;
        const bool inside = h < v.H && ws < v.W && d < v.D;
        const long long vox = (((long long)tc.b * v.D + d) * v.H + h) * v.W + ws;
#pragma unroll
        for (int c = 0; c < NT; c += 16) {
            float acc[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(sl * NT + c), acc);
            if (!inside || co0 + c >= cout) continue;
            uint32_t packed[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                float v0 = acc[2 * j], v1 = acc[2 * j + 1];
                if (bias) {
                    v0 += __ldg(bias + co0 + c + 2 * j);
                    v1 += __ldg(bias + co0 + c + 2 * j + 1);
                }
                if (relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                const __nv_bfloat162 p2 = __floats2bfloat162_rn(v0, v1);
                packed[j] = *reinterpret_cast<const uint32_t *>(&p2);
            }
            uint4 *dst = reinterpret_cast<uint4 *>(y + vox * cout + co0 + c);
            dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
    }
}

template <int NT, int DS>
cudaError_t launch_fwd_tc(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout, int relu,
                          long long tiles, cudaStream_t st)
{
    const size_t smem = 2 * (size_t)half_bytes(DS) + 27 * 2 * NT * 16 + 16;
    cudaError_t e = cudaFuncSetAttribute(k_conv_fwd_tc<NT, DS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)tiles, (unsigned)((cout + NT - 1) / NT));
    k_conv_fwd_tc<NT, DS><<<grid, 128, smem, st>>>(x, w, bias, y, v, cin, cout, relu);
    return cudaGetLastError();
}

long long tc_tiles(const Vol &v, int ds)
{
    return (long long)v.B * ((v.D + ds - 1) / ds) * ((v.H + TH - 1) / TH) * ((v.W + TW - 1) / TW);
}

// Slices per CTA: as many as keep about two CTAs per SM busy (more slices share one weight
// staging; fewer give small volumes enough CTAs).
template <int NT>
cudaError_t launch_fwd_tc_ds(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout,
                             int relu, cudaStream_t st)
{
    const long long chunks = (cout + NT - 1) / NT, want = 2LL * 148;
    if (tc_tiles(v, 1) >= (1LL << 31)) return cudaErrorInvalidValue;
    if (tc_tiles(v, 4) * chunks >= want) return launch_fwd_tc<NT, 4>(x, w, bias, y, v, cin, cout, relu, tc_tiles(v, 4), st);
    if (tc_tiles(v, 2) * chunks >= want) return launch_fwd_tc<NT, 2>(x, w, bias, y, v, cin, cout, relu, tc_tiles(v, 2), st);
    return launch_fwd_tc<NT, 1>(x, w, bias, y, v, cin, cout, relu, tc_tiles(v, 1), st);
}

}  // namespace

cudaError_t conv_fwd_tc(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout, int relu,
                        cudaStream_t st)
{
    if (cin % 16 || cout % 16 || cin < 16 || cout < 16) return cudaErrorInvalidValue;
    switch (cout >= 64 ? 64 : cout) {
    case 16: return launch_fwd_tc_ds<16>(x, w, bias, y, v, cin, cout, relu, st);
    case 32: return launch_fwd_tc_ds<32>(x, w, bias, y, v, cin, cout, relu, st);
    case 48: return launch_fwd_tc_ds<48>(x, w, bias, y, v, cin, cout, relu, st);
    default: return launch_fwd_tc_ds<64>(x, w, bias, y, v, cin, cout, relu, st);
    }
}

cudaError_t conv_tc_error(unsigned *err, bool reset, cudaStream_t st)
{
    cudaError_t e = cudaMemcpyFromSymbolAsync(err, g_conv_tc_error, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess || !reset || *err == 0) return e;
    const unsigned zero = 0;
    return cudaMemcpyToSymbolAsync(g_conv_tc_error, &zero, sizeof(unsigned), 0, cudaMemcpyHostToDevice, st);
}

}  // namespace net
}  // namespace tomo
