// C ABI of the traveltime surrogate (learned warm start): a 3D U-Net predicting the
// factored traveltime tau = T / T0, trained on the device by its own forward and backward
// kernels (net.cu).  No counterpart in the reference, which has no learned component.
//
// Network (4 levels, 16-32-48-64 channels, 3x3x3 convolutions + ReLU, 2x2x2 mean pooling,
// nearest upsampling, skip concatenation, linear 1x1x1 head with tau = 1 + output):
//   enc1  in16->16->16     @1      dec3  (64 up + 48)=112 -> 48 -> 48   @1/4
//   enc2  16->32->32       @1/2    dec2  (48 up + 32)=80  -> 32 -> 32   @1/2
//   enc3  32->48->48       @1/4    dec1  (32 up + 16)=48  -> 16 -> 16   @1
//   bott  48->64->64       @1/8    head  16 -> 1
// Inputs: channel 0 = s / s_src - 1, channel 1 = distance / (64 h) (net.cuh: features).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/tomo_b200.h"
#include "context.hpp"
#include "net.cuh"

using tomo::net::bf16;
using tomo::net::Vol;

namespace {

struct ConvSpec {
    int cin, cout;
    long long w_off, b_off;    // FP32 parameter offsets
    long long wb_off;          // BF16 weight offsets (forward and flipped share the layout size)
};

// conv order: e1a e1b e2a e2b e3a e3b ba bb d3a d3b d2a d2b d1a d1b
constexpr int kConvs = 14;
constexpr int kSpec[kConvs][2] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 48}, {48, 48}, {48, 64},
                                  {64, 64}, {112, 48}, {48, 48}, {80, 32}, {32, 32}, {48, 16}, {16, 16}};
// level of each conv (0 = full resolution)
constexpr int kLevel[kConvs] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0};

template <typename T>
using Buf = tomo::DevBuf<T>;

}  // namespace

struct tomo_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    ConvSpec conv[kConvs];
    long long n_params = 0, n_wb = 0, head_off = 0;
    Buf<float> p, g, m, v;         // FP32 parameters, gradients, Adam moments
    Buf<bf16> wb, wf;              // BF16 forward / flipped (dgrad) weights
    int step = 0;
    // activations (BF16) and their gradients, sized for `cap_vox` full-resolution voxels
    long long cap_vox = 0;
    // forward: x, e1a, e1, p1, e2a, e2, p2, e3a, e3, p3, ba, b, u3, c3, d3a, d3, u2, c2, d2a, d2, u1, c1, d1a, d1
    Buf<bf16> act[24];
    Buf<bf16> grad[24];
    Buf<float> tau, target;
    Buf<double> acc;
    Buf<tomo::net::Job> jobs;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

namespace {

int fail(tomo_net *n, int code, const std::string &msg)
{
    if (n) n->err = msg;
    return code;
}

#define NK(call)                                                                                                    \
    do {                                                                                                            \
        const cudaError_t e_ = (call);                                                                              \
        if (e_ != cudaSuccess)                                                                                      \
            return fail(net, e_ == cudaErrorMemoryAllocation ? TOMO_ERR_OOM : TOMO_ERR_CUDA,                        \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                                        \
    } while (0)

// activation slots
enum Slot {
    X, E1A, E1, P1, E2A, E2, P2, E3A, E3, P3, BA, BB, U3, C3, D3A, D3, U2, C2, D2A, D2, U1, C1, D1A, D1, NSLOT
};
// channels and level of each slot
constexpr int kSlotC[NSLOT] = {16, 16, 16, 16, 32, 32, 32, 48, 48, 48, 64, 64,
                               64, 112, 48, 48, 48, 80, 32, 32, 32, 48, 16, 16};
constexpr int kSlotL[NSLOT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 2, 1, 1, 1, 1, 0, 0, 0, 0};

int ensure_acts(tomo_net *net, long long vox)
{
    if (vox <= net->cap_vox) return TOMO_OK;
    for (int s = 0; s < NSLOT; s++) {
        const long long n = (vox >> (3 * kSlotL[s])) * kSlotC[s];
        NK(net->act[s].ensure((size_t)n));
        NK(net->grad[s].ensure((size_t)n));
    }
    NK(net->tau.ensure((size_t)vox));
    NK(net->target.ensure((size_t)vox));
    net->cap_vox = vox;
    return TOMO_OK;
}

Vol level(Vol v, int l)
{
    return Vol{v.B, v.D >> l, v.H >> l, v.W >> l};
}

// conv layer i: input slot -> output slot (ReLU)
int conv_forward(tomo_net *net, int i, int in, int out, Vol v0)
{
    const ConvSpec &c = net->conv[i];
    const Vol v = level(v0, kLevel[i]);
    NK(tomo::net::conv_fwd(net->act[in].ptr, net->wb.ptr + c.wb_off, net->p.ptr + c.b_off, net->act[out].ptr, v, c.cin,
                           c.cout, 1, net->stream));
    return TOMO_OK;
}

int forward(tomo_net *net, Vol v, bool with_target)
{
    const cudaStream_t st = net->stream;
    int rc;
#define FWD(i, a, b)                                   \
    if ((rc = conv_forward(net, i, a, b, v)) != TOMO_OK) \
        return rc;
    FWD(0, X, E1A) FWD(1, E1A, E1)
    NK(tomo::net::pool_fwd(net->act[E1].ptr, net->act[P1].ptr, level(v, 0), 16, st));
    FWD(2, P1, E2A) FWD(3, E2A, E2)
    NK(tomo::net::pool_fwd(net->act[E2].ptr, net->act[P2].ptr, level(v, 1), 32, st));
    FWD(4, P2, E3A) FWD(5, E3A, E3)
    NK(tomo::net::pool_fwd(net->act[E3].ptr, net->act[P3].ptr, level(v, 2), 48, st));
    FWD(6, P3, BA) FWD(7, BA, BB)
    NK(tomo::net::up_fwd(net->act[BB].ptr, net->act[U3].ptr, level(v, 2), 64, st));
    NK(tomo::net::concat_fwd(net->act[U3].ptr, 64, net->act[E3].ptr, 48, net->act[C3].ptr, level(v, 2).voxels(), st));
    FWD(8, C3, D3A) FWD(9, D3A, D3)
    NK(tomo::net::up_fwd(net->act[D3].ptr, net->act[U2].ptr, level(v, 1), 48, st));
    NK(tomo::net::concat_fwd(net->act[U2].ptr, 48, net->act[E2].ptr, 32, net->act[C2].ptr, level(v, 1).voxels(), st));
    FWD(10, C2, D2A) FWD(11, D2A, D2)
    NK(tomo::net::up_fwd(net->act[D2].ptr, net->act[U1].ptr, level(v, 0), 32, st));
    NK(tomo::net::concat_fwd(net->act[U1].ptr, 32, net->act[E1].ptr, 16, net->act[C1].ptr, level(v, 0).voxels(), st));
    FWD(12, C1, D1A) FWD(13, D1A, D1)
#undef FWD
    if (with_target) NK(cudaMemsetAsync(net->acc.ptr, 0, 2 * sizeof(double), st));
    NK(tomo::net::head_fwd(net->act[D1].ptr, net->p.ptr + net->head_off, net->p.ptr + net->head_off + 16, net->tau.ptr,
                           with_target ? net->target.ptr : nullptr, v.voxels(), 16, net->acc.ptr, st));
    return TOMO_OK;
}

// conv layer i backward: dy (grad slot of its output) -> weight/bias gradients and, if
// gin >= 0, the gradient of its input into grad slot gin
int conv_backward(tomo_net *net, int i, int in, int out, int gin, Vol v0)
{
    const ConvSpec &c = net->conv[i];
    const Vol v = level(v0, kLevel[i]);
    const cudaStream_t st = net->stream;
    bf16 *dy = net->grad[out].ptr;
    NK(tomo::net::relu_bwd(net->act[out].ptr, dy, v.voxels() * c.cout, st));
    NK(tomo::net::conv_wgrad(net->act[in].ptr, dy, net->g.ptr + c.w_off, v, c.cin, c.cout, st));
    NK(tomo::net::bias_grad(dy, net->g.ptr + c.b_off, v.voxels(), c.cout, st));
    if (gin >= 0)
        NK(tomo::net::conv_fwd(dy, net->wf.ptr + c.wb_off, nullptr, net->grad[gin].ptr, v, c.cout, c.cin, 0, st));
    return TOMO_OK;
}

int backward(tomo_net *net, Vol v)
{
    const cudaStream_t st = net->stream;
    int rc;
    NK(cudaMemsetAsync(net->g.ptr, 0, (size_t)net->n_params * sizeof(float), st));
    NK(tomo::net::head_bwd(net->act[D1].ptr, net->p.ptr + net->head_off, net->tau.ptr, net->target.ptr, net->acc.ptr,
                           net->grad[D1].ptr, net->g.ptr + net->head_off, net->g.ptr + net->head_off + 16, v.voxels(), 16,
                           st));
#define BWD(i, a, b, gin)                                        \
    if ((rc = conv_backward(net, i, a, b, gin, v)) != TOMO_OK) \
        return rc;
    BWD(13, D1A, D1, D1A) BWD(12, C1, D1A, C1)
    NK(tomo::net::concat_bwd(net->grad[C1].ptr, net->grad[U1].ptr, 32, net->grad[E1].ptr, 16, level(v, 0).voxels(), st));
    NK(tomo::net::up_bwd(net->grad[U1].ptr, net->grad[D2].ptr, level(v, 0), 32, st));
    BWD(11, D2A, D2, D2A) BWD(10, C2, D2A, C2)
    NK(tomo::net::concat_bwd(net->grad[C2].ptr, net->grad[U2].ptr, 48, net->grad[E2].ptr, 32, level(v, 1).voxels(), st));
    NK(tomo::net::up_bwd(net->grad[U2].ptr, net->grad[D3].ptr, level(v, 1), 48, st));
    BWD(9, D3A, D3, D3A) BWD(8, C3, D3A, C3)
    NK(tomo::net::concat_bwd(net->grad[C3].ptr, net->grad[U3].ptr, 64, net->grad[E3].ptr, 48, level(v, 2).voxels(), st));
    NK(tomo::net::up_bwd(net->grad[U3].ptr, net->grad[BB].ptr, level(v, 2), 64, st));
    BWD(7, BA, BB, BA) BWD(6, P3, BA, P3)
    // E3's gradient: skip path (already in grad[E3]) + pooling path
    NK(tomo::net::pool_bwd(net->grad[P3].ptr, net->grad[E3A].ptr, level(v, 2), 48, st));
    NK(tomo::net::add_into(net->grad[E3].ptr, net->grad[E3A].ptr, level(v, 2).voxels() * 48, st));
    BWD(5, E3A, E3, E3A) BWD(4, P2, E3A, P2)
    NK(tomo::net::pool_bwd(net->grad[P2].ptr, net->grad[E2A].ptr, level(v, 1), 32, st));
    NK(tomo::net::add_into(net->grad[E2].ptr, net->grad[E2A].ptr, level(v, 1).voxels() * 32, st));
    BWD(3, E2A, E2, E2A) BWD(2, P1, E2A, P1)
    NK(tomo::net::pool_bwd(net->grad[P1].ptr, net->grad[E1A].ptr, level(v, 0), 16, st));
    NK(tomo::net::add_into(net->grad[E1].ptr, net->grad[E1A].ptr, level(v, 0).voxels() * 16, st));
    BWD(1, E1A, E1, E1A) BWD(0, X, E1A, -1)
#undef BWD
    return TOMO_OK;
}

int refresh_weights(tomo_net *net)
{
    for (int i = 0; i < kConvs; i++) {
        const ConvSpec &c = net->conv[i];
        NK(tomo::net::to_bf16(net->p.ptr + c.w_off, net->wb.ptr + c.wb_off, 27LL * c.cin * c.cout, net->stream));
        NK(tomo::net::flip_weights(net->p.ptr + c.w_off, net->wf.ptr + c.wb_off, c.cin, c.cout, net->stream));
    }
    return TOMO_OK;
}

int pad8(int n) { return (n + 7) / 8 * 8; }

// Jobs of a batch (one padded volume per sample, all of the same padded size).
// stride k: the network volume holds every k-th window node (ceil(n / k) per axis, padded)
int make_jobs(tomo_net *net, int n, const tomo_net_sample *s, float h, Vol &v, std::vector<tomo::net::Job> &jobs,
              int stride = 1)
{
    int pd = 0, ph = 0, pw = 0;
    auto ck = [stride](int m) { return (m + stride - 1) / stride; };
    for (int i = 0; i < n; i++) {
        const tomo_window &w = s[i].window;
        if (!s[i].slow || w.x0 < 0 || w.y0 < 0 || w.x1 > s[i].model_nx || w.y1 > s[i].model_ny || w.x1 - w.x0 < 2 ||
            w.y1 - w.y0 < 2 || s[i].nz < 2)
            return fail(net, TOMO_ERR_INVALID_ARG, "sample " + std::to_string(i) + ": bad model or window");
        pd = std::max(pd, pad8(ck(w.y1 - w.y0)));
        ph = std::max(ph, pad8(ck(w.x1 - w.x0)));
        pw = std::max(pw, pad8(ck(s[i].nz)));
    }
    v = Vol{n, pd, ph, pw};
    jobs.resize((size_t)n);
    long long nat = 0;
    for (int i = 0; i < n; i++) {
        const tomo_window &w = s[i].window;
        tomo::net::Job &j = jobs[(size_t)i];
        j.slow = s[i].slow;
        j.model_nx = s[i].model_nx;
        j.nz = s[i].nz;
        j.wx0 = w.x0;
        j.wy0 = w.y0;
        j.wnx = w.x1 - w.x0;
        j.wny = w.y1 - w.y0;
        j.pd = pd;
        j.ph = ph;
        j.pw = pw;
        j.sx = s[i].source.x - w.x0 * h;
        j.sy = s[i].source.y - w.y0 * h;
        j.sz = s[i].source.z;
        if (!(j.sx >= 0.f) || !(j.sy >= 0.f) || !(j.sz >= 0.f) || j.sx > (j.wnx - 1) * h || j.sy > (j.wny - 1) * h ||
            j.sz > (j.nz - 1) * h)
            return fail(net, TOMO_ERR_INVALID_ARG, "sample " + std::to_string(i) + ": source outside its window");
        j.out_off = (long long)i * pd * ph * pw;
        j.nat_off = nat;
        j.T = s[i].T;
        j.stride = stride;
        nat += (long long)j.nz * j.wnx * j.wny;
    }
    NK(net->jobs.ensure((size_t)n));
    NK(cudaMemcpyAsync(net->jobs.ptr, jobs.data(), jobs.size() * sizeof(tomo::net::Job), cudaMemcpyHostToDevice,
                       net->stream));
    return ensure_acts(net, v.voxels());
}

int load_batch(tomo_net *net, int n, const tomo_net_sample *s, float h, bool targets, Vol &v)
{
    std::vector<tomo::net::Job> jobs;
    int rc = make_jobs(net, n, s, h, v, jobs);
    if (rc != TOMO_OK) return rc;
    const long long per = (long long)v.D * v.H * v.W;
    NK(tomo::net::features(net->jobs.ptr, n, h, net->act[X].ptr, per, net->stream));
    if (targets) {
        for (int i = 0; i < n; i++)
            if (!s[i].T) return fail(net, TOMO_ERR_INVALID_ARG, "sample " + std::to_string(i) + ": no traveltimes");
        NK(tomo::net::tau_target(net->jobs.ptr, n, h, net->target.ptr, per, net->stream));
    }
    return TOMO_OK;
}

// The tensor-core convolutions' error word (synchronises the stream): a bounded wait that
// ran out is reported, and the word cleared, instead of returning garbage.
int check_convolutions(tomo_net *net)
{
    unsigned err = 0;
    NK(tomo::net::conv_tc_error(&err, true, net->stream));
    if (err) return fail(net, TOMO_ERR_TIMEOUT, "tensor-core convolution: a device wait timed out");
    return TOMO_OK;
}

int read_loss(tomo_net *net, double *loss)
{
    double a[2];
    NK(cudaMemcpyAsync(a, net->acc.ptr, sizeof(a), cudaMemcpyDeviceToHost, net->stream));
    NK(cudaStreamSynchronize(net->stream));
    const int rc = check_convolutions(net);
    if (rc != TOMO_OK) return rc;
    if (loss) *loss = a[1] > 0 ? a[0] / a[1] : 0.0;
    return TOMO_OK;
}

}  // namespace

extern "C" {

int tomo_net_create(int device, void *stream, unsigned long long seed, tomo_net **out)
{
    if (!out) return TOMO_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return TOMO_ERR_NO_DEVICE;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return TOMO_ERR_NO_DEVICE;
    tomo_net *net = new tomo_net;
    net->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) {
        if (stream) {
            net->stream = static_cast<cudaStream_t>(stream);
        } else {
            e = cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking);
            net->own_stream = e == cudaSuccess;
        }
    }
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreate(&net->ev[i]);
    // parameter layout: per conv [w (cout x 27 x cin), b (cout)], then head [wh (16), bh (1)]
    long long off = 0, wb = 0;
    for (int i = 0; i < kConvs; i++) {
        ConvSpec &c = net->conv[i];
        c.cin = kSpec[i][0];
        c.cout = kSpec[i][1];
        c.w_off = off;
        off += 27LL * c.cin * c.cout;
        c.b_off = off;
        off += c.cout;
        c.wb_off = wb;
        wb += 27LL * c.cin * c.cout;
    }
    net->head_off = off;
    off += 17;
    net->n_params = off;
    net->n_wb = wb;
    if (e == cudaSuccess) e = net->p.ensure((size_t)off);
    if (e == cudaSuccess) e = net->g.ensure((size_t)off);
    if (e == cudaSuccess) e = net->m.ensure((size_t)off);
    if (e == cudaSuccess) e = net->v.ensure((size_t)off);
    if (e == cudaSuccess) e = net->wb.ensure((size_t)wb);
    if (e == cudaSuccess) e = net->wf.ensure((size_t)wb);
    if (e == cudaSuccess) e = net->acc.ensure(2);
    if (e != cudaSuccess) {
        tomo_net_destroy(net);
        return e == cudaErrorMemoryAllocation ? TOMO_ERR_OOM : TOMO_ERR_CUDA;
    }
    // He-uniform initialisation (bound sqrt(6 / fan_in)), zero biases, small head
    std::vector<float> h((size_t)off, 0.f);
    std::mt19937_64 rng(seed);
    for (int i = 0; i < kConvs; i++) {
        const ConvSpec &c = net->conv[i];
        const float bound = std::sqrt(6.0f / (27.0f * c.cin));
        std::uniform_real_distribution<float> u(-bound, bound);
        for (long long k = 0; k < 27LL * c.cin * c.cout; k++) h[(size_t)(c.w_off + k)] = u(rng);
    }
    std::uniform_real_distribution<float> uh(-0.01f, 0.01f);
    for (int k = 0; k < 16; k++) h[(size_t)(net->head_off + k)] = uh(rng);
    const int rc = tomo_net_set_params(net, h.data());
    if (rc != TOMO_OK) {
        tomo_net_destroy(net);
        return rc;
    }
    *out = net;
    return TOMO_OK;
}

int tomo_net_destroy(tomo_net *net)
{
    if (!net) return TOMO_OK;
    cudaSetDevice(net->device);
    if (net->stream) cudaStreamSynchronize(net->stream);
    net->p.release();
    net->g.release();
    net->m.release();
    net->v.release();
    net->wb.release();
    net->wf.release();
    for (auto &b : net->act) b.release();
    for (auto &b : net->grad) b.release();
    net->tau.release();
    net->target.release();
    net->acc.release();
    net->jobs.release();
    for (auto &e : net->ev)
        if (e) cudaEventDestroy(e);
    if (net->own_stream && net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return TOMO_OK;
}

const char *tomo_net_last_error(const tomo_net *net) { return net ? net->err.c_str() : ""; }

long long tomo_net_param_count(const tomo_net *net) { return net ? net->n_params : 0; }

int tomo_net_get_params(tomo_net *net, float *out)
{
    if (!net || !out) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    NK(cudaMemcpyAsync(out, net->p.ptr, (size_t)net->n_params * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    NK(cudaStreamSynchronize(net->stream));
    return TOMO_OK;
}

int tomo_net_set_params(tomo_net *net, const float *in)
{
    if (!net || !in) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    NK(cudaMemcpyAsync(net->p.ptr, in, (size_t)net->n_params * sizeof(float), cudaMemcpyHostToDevice, net->stream));
    NK(cudaMemsetAsync(net->m.ptr, 0, (size_t)net->n_params * sizeof(float), net->stream));
    NK(cudaMemsetAsync(net->v.ptr, 0, (size_t)net->n_params * sizeof(float), net->stream));
    net->step = 0;
    const int rc = refresh_weights(net);
    if (rc != TOMO_OK) return rc;
    NK(cudaStreamSynchronize(net->stream));
    return TOMO_OK;
}

int tomo_net_gradients(tomo_net *net, int n, const tomo_net_sample *samples, float h, double *loss, float *grads)
{
    if (!net || n < 1 || !samples || !(h > 0)) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    Vol v{};
    int rc = load_batch(net, n, samples, h, true, v);
    if (rc == TOMO_OK) rc = forward(net, v, true);
    if (rc == TOMO_OK) rc = backward(net, v);
    if (rc != TOMO_OK) return rc;
    if (grads)
        NK(cudaMemcpyAsync(grads, net->g.ptr, (size_t)net->n_params * sizeof(float), cudaMemcpyDeviceToHost,
                           net->stream));
    return read_loss(net, loss);
}

int tomo_net_train_step(tomo_net *net, int n, const tomo_net_sample *samples, float h, float lr, double *loss)
{
    if (!net || n < 1 || !samples || !(h > 0) || !(lr > 0)) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    Vol v{};
    int rc = load_batch(net, n, samples, h, true, v);
    if (rc == TOMO_OK) rc = forward(net, v, true);
    if (rc == TOMO_OK) rc = backward(net, v);
    if (rc != TOMO_OK) return rc;
    net->step++;
    NK(tomo::net::adam(net->p.ptr, net->g.ptr, net->m.ptr, net->v.ptr, net->n_params, lr, 0.9f, 0.999f, 1e-8f,
                       net->step, net->stream));
    rc = refresh_weights(net);
    if (rc != TOMO_OK) return rc;
    return read_loss(net, loss);
}

int tomo_net_evaluate(tomo_net *net, int n, const tomo_net_sample *samples, float h, double *loss)
{
    if (!net || n < 1 || !samples || !(h > 0)) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    Vol v{};
    int rc = load_batch(net, n, samples, h, true, v);
    if (rc == TOMO_OK) rc = forward(net, v, true);
    if (rc != TOMO_OK) return rc;
    return read_loss(net, loss);
}

int tomo_net_predict(tomo_net *net, int n, const tomo_net_sample *samples, float h, float *t_pred, float *ms)
{
    return tomo_net_predict_strided(net, n, samples, h, 1, t_pred, ms);
}

int tomo_net_predict_strided(tomo_net *net, int n, const tomo_net_sample *samples, float h, int stride, float *t_pred,
                             float *ms)
{
    if (!net || n < 1 || !samples || !(h > 0) || !t_pred || stride < 1 || stride > 16) return TOMO_ERR_INVALID_ARG;
    NK(cudaSetDevice(net->device));
    NK(cudaEventRecord(net->ev[0], net->stream));
    long long nat = 0;
    auto ck = [stride](int m) { return (m + stride - 1) / stride; };
    for (int i0 = 0; i0 < n;) {
        // as many samples per pass as fit in one window's worth of activations x 8
        int cnt = 1;
        Vol v{};
        std::vector<tomo::net::Job> jobs;
        {
            const tomo_window &w = samples[i0].window;
            const long long one =
                (long long)pad8(ck(w.y1 - w.y0)) * pad8(ck(w.x1 - w.x0)) * pad8(ck(samples[i0].nz));
            cnt = (int)std::max(1LL, std::min<long long>(n - i0, (8LL << 20) / std::max(one, 1LL)));
        }
        int rc = make_jobs(net, cnt, samples + i0, h, v, jobs, stride);
        if (rc != TOMO_OK) return rc;
        const long long per = (long long)v.D * v.H * v.W;
        NK(tomo::net::features(net->jobs.ptr, cnt, h, net->act[X].ptr, per, net->stream));
        rc = forward(net, v, false);
        if (rc != TOMO_OK) return rc;
        long long max_nat = 0;
        for (const auto &j : jobs) max_nat = std::max(max_nat, (long long)j.nz * j.wnx * j.wny);
        if (stride == 1)
            NK(tomo::net::tau_to_time(net->jobs.ptr, cnt, h, net->tau.ptr, t_pred + nat, per, net->stream));
        else
            NK(tomo::net::tau_to_time_strided(net->jobs.ptr, cnt, h, net->tau.ptr, t_pred + nat, max_nat, net->stream));
        for (const auto &j : jobs) nat += (long long)j.nz * j.wnx * j.wny;
        i0 += cnt;
    }
    NK(cudaEventRecord(net->ev[1], net->stream));
    NK(cudaStreamSynchronize(net->stream));
    if (ms) cudaEventElapsedTime(ms, net->ev[0], net->ev[1]);
    return check_convolutions(net);
}

}  // extern "C"

// ----------------------------------------------------------------------------------------
// Training data: seeded random layered tiles written into a context's model.
// ----------------------------------------------------------------------------------------
namespace tomo {
int rebrick_model(tomo_ctx *ctx);
int model_buffers(tomo_ctx *ctx);
}

extern "C" int tomo_random_tiles(tomo_ctx *ctx, int tile, unsigned long long seed)
{
    if (!ctx || tile < 8) return TOMO_ERR_INVALID_ARG;
    const tomo_grid &g = ctx->g;
    if (g.nx % tile || g.ny % tile) {
        ctx->err = "model width and length must be multiples of the tile edge";
        return TOMO_ERR_INVALID_ARG;
    }
    const int tx = g.nx / tile, ty = g.ny / tile;
    std::vector<tomo::net::TileModel> tm((size_t)tx * ty);
    std::mt19937_64 rng(seed);
    auto U = [&](float a, float b) { return std::uniform_real_distribution<float>(a, b)(rng); };
    for (int j = 0; j < ty; j++)
        for (int i = 0; i < tx; i++) {
            tomo::net::TileModel &t = tm[(size_t)j * tx + i];
            t = tomo::net::TileModel{};
            t.x0 = i * tile;
            t.y0 = j * tile;
            t.n = tile;
            t.nlayers = 3 + (int)(rng() % 4);  // 3..6 layers
            std::vector<float> z(t.nlayers - 1);
            for (auto &zz : z) zz = U(0.08f, 0.92f) * g.nz;
            std::sort(z.begin(), z.end());
            for (int k = 0; k < t.nlayers - 1; k++) {
                t.z0[k] = z[(size_t)k];
                t.gx[k] = U(-0.15f, 0.15f);  // dips up to ~8.5 degrees
                t.gy[k] = U(-0.15f, 0.15f);
                t.z0[k] -= t.gx[k] * tile * 0.5f + t.gy[k] * tile * 0.5f;  // depth z[k] at the tile centre
            }
            for (int k = 0; k < t.nlayers; k++) t.vel[k] = U(1500.f, 4500.f);
            t.nanom = (int)(rng() % 13);  // 0..12
            for (int a = 0; a < t.nanom; a++) {
                t.ax[a] = U(0.f, (float)tile);
                t.ay[a] = U(0.f, (float)tile);
                t.az[a] = U(0.f, (float)g.nz);
                t.asig[a] = U(0.04f, 0.15f) * tile;
                t.aamp[a] = U(-0.15f, 0.15f);
            }
        }
    tomo::DevBuf<tomo::net::TileModel> d;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = d.ensure(tm.size());
    if (e == cudaSuccess) e = ctx->slow.ensure((size_t)g.nx * g.ny * g.nz);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.ptr, tm.data(), tm.size() * sizeof(tomo::net::TileModel), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = tomo::net::random_models(d.ptr, (int)tm.size(), ctx->slow.ptr, g.nx, g.ny, g.nz, ctx->stream);
    if (e != cudaSuccess) {
        ctx->err = std::string("tomo_random_tiles: ") + cudaGetErrorString(e);
        d.release();
        return TOMO_ERR_CUDA;
    }
    int rc = tomo::model_buffers(ctx);
    if (rc == TOMO_OK) rc = tomo::rebrick_model(ctx);
    if (rc == TOMO_OK) {
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            ctx->err = std::string("tomo_random_tiles: ") + cudaGetErrorString(e);
            rc = TOMO_ERR_CUDA;
        }
    }
    d.release();
    ctx->have_model = rc == TOMO_OK;
    return rc;
}

extern "C" const float *tomo_ctx_slowness_device(tomo_ctx *ctx) { return ctx ? ctx->slow.ptr : nullptr; }
