// Surrogate of the factored traveltime tau = T / T0 (learned warm start): device kernels.
//
// Tensors are channels-last BF16 volumes [B][D][H][W][C] (C a multiple of 16); a volume
// of the model maps D = y, H = x, W = z, so channels-last order follows the model's
// z-fastest layout.  Weights of a 3x3x3 convolution are BF16 [Cout][27][Cin] with
// tap = (dd*3 + dh)*3 + dw (offsets -1..1); master weights, gradients and optimiser state
// are FP32.  Convolutions are implicit GEMMs on the tensor cores with BF16 operands and
// FP32 accumulation -- the forward on tcgen05 (accumulator in tensor memory), the weight
// gradient on mma.sync -- zero padding, same-size output.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tomo {
namespace net {

typedef __nv_bfloat16 bf16;

struct Vol {
    int B, D, H, W;
    __host__ __device__ long long voxels() const { return (long long)B * D * H * W; }
};

// y = act(conv3x3x3(x, w) + bias); relu: 0/1; bias may be nullptr.
cudaError_t conv_fwd(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout, int relu,
                     cudaStream_t st);
// The same convolution on the tcgen05 tensor cores (net_tc.cu): M = 128 voxels per CTA,
// accumulator in tensor memory.
cudaError_t conv_fwd_tc(const bf16 *x, const bf16 *w, const float *bias, bf16 *y, Vol v, int cin, int cout, int relu,
                        cudaStream_t st);
// The tcgen05 convolution's error word (0, or 1 after a bounded wait ran out); synchronises
// the stream; reset: clear it after reading.
cudaError_t conv_tc_error(unsigned *err, bool reset, cudaStream_t st);
// dW[co][tap][ci] += sum_v dy[v][co] * x[v + tap][ci]  (FP32, accumulated with atomics)
cudaError_t conv_wgrad(const bf16 *x, const bf16 *dy, float *dw, Vol v, int cin, int cout, cudaStream_t st);
// db[co] += sum_v dy[v][co]
cudaError_t bias_grad(const bf16 *dy, float *db, long long voxels, int c, cudaStream_t st);
// wt[ci][26 - tap][co] = w[co][tap][ci]: the weights of dgrad run as a forward conv
cudaError_t flip_weights(const float *w, bf16 *wt, int cin, int cout, cudaStream_t st);
cudaError_t to_bf16(const float *a, bf16 *b, long long n, cudaStream_t st);

// elementwise and resampling (channels-last, c channels)
cudaError_t relu_bwd(const bf16 *y, bf16 *dy, long long n, cudaStream_t st);      // dy *= (y > 0)
cudaError_t add_into(bf16 *a, const bf16 *b, long long n, cudaStream_t st);       // a += b
cudaError_t pool_fwd(const bf16 *x, bf16 *y, Vol fine, int c, cudaStream_t st);   // 2x2x2 mean
cudaError_t pool_bwd(const bf16 *dy, bf16 *dx, Vol fine, int c, cudaStream_t st);
cudaError_t up_fwd(const bf16 *x, bf16 *y, Vol fine, int c, cudaStream_t st);     // nearest x2
cudaError_t up_bwd(const bf16 *dy, bf16 *dx, Vol fine, int c, cudaStream_t st);
cudaError_t concat_fwd(const bf16 *a, int ca, const bf16 *b, int cb, bf16 *y, long long voxels, cudaStream_t st);
cudaError_t concat_bwd(const bf16 *dy, bf16 *da, int ca, bf16 *db, int cb, long long voxels, cudaStream_t st);

// Head: tau[v] = 1 + sum_c wh[c] y[v][c] + bh[0].  With a target (target[v] > 0 marks the
// voxels of the loss), acc[0] += sum (tau - target)^2 and acc[1] += count.
cudaError_t head_fwd(const bf16 *y, const float *wh, const float *bh, float *tau, const float *target, long long voxels,
                     int c, double *acc, cudaStream_t st);
// Gradients of loss = acc[0] / acc[1]: dy[v][c] = g wh[c], dwh[c] += sum g y[v][c],
// dbh += sum g, with g = 2 (tau - target) / acc[1] on the loss voxels, else 0.
cudaError_t head_bwd(const bf16 *y, const float *wh, const float *tau, const float *target, const double *acc, bf16 *dy,
                     float *dwh, float *dbh, long long voxels, int c, cudaStream_t st);

// Adam on n FP32 parameters (bias-corrected, step t >= 1)
cudaError_t adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2, float eps,
                 int t, cudaStream_t st);

// One volume of a batch: a window of a slowness model and its source.
struct Job {
    const float *slow;   // model slowness, natural layout (z fastest, then x, then y)
    int model_nx, nz;    // strides of that model
    int wx0, wy0;        // window origin (nodes)
    int wnx, wny;        // window size (nodes); depth is nz
    int pd, ph, pw;      // padded network volume: D = y, H = x, W = z (multiples of 8)
    float sx, sy, sz;    // source, window coordinates (m)
    long long out_off;   // voxel offset of the padded volume in the batch tensors
    long long nat_off;   // offset of the window volume in back-to-back natural outputs
    const float *T;      // the window's traveltimes (natural layout) for training targets
    int stride;          // the network volume samples every stride-th window node (1: all)
};
// Input features: channel 0 = s / s_src - 1, channel 1 = distance / (64 h stride),
// channels 2..15 = 0.  Padding voxels repeat the nearest window voxel.
cudaError_t features(const Job *jobs, int njobs, float h, bf16 *x16, long long max_vox, cudaStream_t st);
// tau = T / (s_src * distance) inside the window at distance >= h, else 0 (not in the loss)
cudaError_t tau_target(const Job *jobs, int njobs, float h, float *tau, long long max_vox, cudaStream_t st);
// predicted traveltime tau * s_src * distance into the back-to-back natural layout (0 at
// distance < h: no ceiling there); jobs with stride > 1 interpolate tau trilinearly between
// the sampled nodes first (max_nat: the largest window volume)
cudaError_t tau_to_time(const Job *jobs, int njobs, float h, const float *tau, float *t_out, long long max_vox,
                        cudaStream_t st);
cudaError_t tau_to_time_strided(const Job *jobs, int njobs, float h, const float *tau, float *t_out,
                                long long max_nat, cudaStream_t st);

// Seeded random layered models (training data): one 64^3-like tile per entry of `tiles`,
// written as slowness into the natural-layout model of size nz x nx x ny.
struct TileModel {
    int x0, y0, n;             // tile origin and edge (nodes)
    int nlayers;               // 3..6
    float z0[6], gx[6], gy[6]; // interface k: depth z0 + gx (x - x0) + gy (y - y0) (nodes), k < nlayers - 1
    float vel[6];              // layer velocities (m/s)
    int nanom;                 // 0..12
    float ax[12], ay[12], az[12], asig[12], aamp[12];  // Gaussian anomalies (nodes, relative)
};
cudaError_t random_models(const TileModel *tiles, int ntiles, float *slow, int nx, int ny, int nz, cudaStream_t st);

}  // namespace net
}  // namespace tomo
