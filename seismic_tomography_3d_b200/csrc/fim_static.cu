// Allocation-free single-shot eikonal solve: tomo_eik_solve_static (include/tomo_b200.h).
//
// For callers that cannot call cudaMalloc -- a host application whose framework has
// already reserved the GPU's memory for its own pool, or a processing loop that must run
// within a fixed device-memory budget without going back to the driver's allocator.  The
// caller passes device input (slowness) and output (traveltimes); the solver's own
// working memory -- the brick-major slowness and traveltime copies, the work lists, the
// queue flags and the control words -- lives in the file-scope device array below, whose
// size is fixed at compile time.  No cudaMalloc, cudaFree or allocating library routine
// is called.
//
// Limits and sharing:
//  * at most kStaticNodes padded nodes (each axis padded to a multiple of 4): 4,194,304,
//    e.g. 160 x 160 x 160 or the 101 x 101 x 51 single-shot survey;
//  * the array (about 34.6 MB) is reserved on every GPU where the library's code is
//    loaded, and stays reserved until the process exits;
//  * every call on a device shares the one array and leaves its contents behind; each
//    call re-initialises everything it reads, but calls whose GPU work overlaps (on
//    different streams or host threads) race on the array and corrupt each other;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//    with that device current; make that first call before any stream capture.  Later
//    calls look it up again unless their stream is capturing (after cudaDeviceReset the
//    module is loaded anew and the array may sit at another address);
//  * the call blocks: it reads the solver's error word back and synchronises the stream.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/tomo_b200.h"
#include "common.cuh"
#include "fim.cuh"

namespace tomo {
namespace {

constexpr size_t kStaticNodes = size_t(1) << 22;
constexpr size_t kStaticBricks = kStaticNodes / kBrickNodes;
// byte offsets inside the array (all multiples of 256)
constexpr size_t kOffS = 0;                                   // brick-major slowness
constexpr size_t kOffT = kOffS + 4 * kStaticNodes;            // brick-major traveltimes
constexpr size_t kOffQ = kOffT + 4 * kStaticNodes;            // queue flags, one per brick
constexpr size_t kOffL = kOffQ + 4 * kStaticBricks;           // 3 work lists
constexpr size_t kOffC = kOffL + 3 * 4 * kStaticBricks;       // control words
constexpr size_t kOffStats = kOffC + 256;                     // activation counters
constexpr size_t kOffDesc = kOffStats + 256;                  // the shot descriptor
constexpr size_t kStaticBytes = kOffDesc + 256;
static_assert(kCtrlWords * sizeof(unsigned) <= 256, "control words overflow their slot");
static_assert(4 * sizeof(unsigned long long) <= 256, "activation counters overflow their slot");
static_assert(sizeof(ShotDesc) <= 256, "shot descriptor overflows its slot");

static __device__ __align__(256) unsigned char g_eik_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices] = {};
thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

// Device address of the array on device `dev` (current).  Looked up on the first call on a
// device and again on every call whose stream is not capturing, since a device reset loads
// the module anew; a capturing call uses the address of the last lookup.
int scratch_on(int dev, cudaStream_t st, unsigned char **out)
{
    if (dev < 0 || dev >= kMaxDevices) return fail(TOMO_ERR_NO_DEVICE, "device index out of range");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess)
        return fail(TOMO_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev] || cap == cudaStreamCaptureStatusNone) {
        if (cap != cudaStreamCaptureStatusNone)
            return fail(TOMO_ERR_STATE, "first call on this device made during a stream capture");
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_eik_scratch);
        if (e != cudaSuccess)
            return fail(TOMO_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_addr[dev];
    return TOMO_OK;
}

__global__ void k_store_desc(ShotDesc d, ShotDesc *dst) { *dst = d; }

int pad4(int n) { return n + (kBrick - n % kBrick) % kBrick; }

}  // namespace

const char *static_error_text() { return g_err.c_str(); }

}  // namespace tomo

#define CKS(call)                                                                                          \
    do {                                                                                                   \
        const cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return tomo::fail(TOMO_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

extern "C" int tomo_eik_solve_static(const float *slowness, int nx, int ny, int nz, float dx, float dy, float dz,
                                     float sx, float sy, float sz, float *t_out, void *stream)
{
    using namespace tomo;
    if (!slowness || !t_out) return fail(TOMO_ERR_INVALID_ARG, "slowness and t_out must be device pointers");
    if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0))
        return fail(TOMO_ERR_INVALID_ARG, "grid must be at least 2x2x2 with positive spacing");
    // Each axis is checked before any product is formed, so that none can wrap: a padded
    // axis is then at most 2^22 + 3, the product of two below 2^45, and the triple product
    // is only formed once the first two are known to be at most 2^22.
    const int lim = (int)kStaticNodes;
    const bool axis_ok = nx <= lim && ny <= lim && nz <= lim;
    const size_t padx = axis_ok ? (size_t)pad4(nx) : 0, pady = axis_ok ? (size_t)pad4(ny) : 0,
                 padz = axis_ok ? (size_t)pad4(nz) : 0;
    if (!axis_ok || padx * pady > kStaticNodes || padx * pady * padz > kStaticNodes)
        return fail(TOMO_ERR_CAPACITY, "grid of " + std::to_string(nx) + " x " + std::to_string(ny) + " x " +
                                           std::to_string(nz) + " nodes exceeds the " +
                                           std::to_string(kStaticNodes) +
                                           " padded nodes of the allocation-free solver; use tomo_eik_solve");
    // source seed as in Block_FIM::apply_source_time (block_FIM.cpp:305-317)
    const int sidx = (int)(sx / dx), sidy = (int)(sy / dy), sidz = (int)(sz / dz);
    if (!(sx >= 0.f) || !(sy >= 0.f) || !(sz >= 0.f) || sidx >= nx || sidy >= ny || sidz >= nz)
        return fail(TOMO_ERR_INVALID_ARG, "source outside the model");
    int dev = 0;
    CKS(cudaGetDevice(&dev));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *base = nullptr;
    int rc = scratch_on(dev, st, &base);
    if (rc != TOMO_OK) return rc;

    ShotDesc d{};
    d.wx0 = d.wy0 = 0;
    d.wnx = nx;
    d.wny = ny;
    d.nbx = pad4(nx) / kBrick;
    d.nby = pad4(ny) / kBrick;
    d.nbz = pad4(nz) / kBrick;
    const float ex = (float)(sidx * dx) - sx, ey = (float)(sidy * dy) - sy, ez = (float)(sidz * dz) - sz;
    d.src_dist = std::sqrt(std::pow(ex, 2.0f) + std::pow(ey, 2.0f) + std::pow(ez, 2.0f));
    d.src_brick = (sidz >> 2) + d.nbz * ((sidx >> 2) + d.nbx * (sidy >> 2));
    d.src_node = (sidz & 3) + 4 * (sidx & 3) + 16 * (sidy & 3);
    d.t_off = 0;
    d.qbase = 0;
    d.s_gather = 0;  // the whole grid: its bricks are the array's model bricks
    const long long nbricks = (long long)d.nbx * d.nby * d.nbz;
    unsigned local_bits = 1;
    while ((1ll << local_bits) < nbricks) local_bits++;
    set_brick_division(d, local_bits);

    float *S = reinterpret_cast<float *>(base + kOffS);
    float *T = reinterpret_cast<float *>(base + kOffT);
    unsigned *qflag = reinterpret_cast<unsigned *>(base + kOffQ);
    unsigned *lists = reinterpret_cast<unsigned *>(base + kOffL);
    unsigned *ctrl = reinterpret_cast<unsigned *>(base + kOffC);
    unsigned long long *stats = reinterpret_cast<unsigned long long *>(base + kOffStats);
    ShotDesc *desc = reinterpret_cast<ShotDesc *>(base + kOffDesc);

    k_store_desc<<<1, 1, 0, st>>>(d, desc);
    CKS(cudaGetLastError());
    CKS(fim_brick_model(slowness, S, nx, ny, nz, pad4(nx), pad4(ny), pad4(nz), st));
    // everything the solve reads is re-initialised: traveltimes, queue flags, control words
    CKS(fim_init(T, (size_t)nbricks * kBrickNodes, qflag, (size_t)nbricks, ctrl, stats, st));
    CKS(fim_seed(desc, 1, S, d.nbx, d.nbz, T, qflag, lists, local_bits, ctrl, st));
    FimLaunch p{};
    p.S = S;
    p.T = T;
    p.shots = desc;
    p.nshots = 1;
    p.qflag = qflag;
    p.lists = lists;
    p.list_cap = (unsigned)nbricks;
    p.ctrl = ctrl;
    p.stats = stats;
    p.gbx = d.nbx;
    p.gbz = d.nbz;
    p.h = dx;  // isotropic h = dx (block_FIM.cpp:173)
    p.max_inner = 16;
    p.max_rounds = 1 << 20;
    p.change_tol = 1e-6f;  // the reference's EPS (cuda_kernel.cuh:8)
    p.inner_tol = 0.f;
    p.local_bits = local_bits;
    p.spin_limit = 1ull << 26;
    CKS(fim_solve(p, 8, 4, false, nullptr, st));
    CKS(fim_unbrick(T, desc, 0, nz, t_out, st));
    unsigned err_word = 0;
    CKS(cudaMemcpyAsync(&err_word, ctrl + kErr, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    if (err_word == kDevRoundCap) return fail(TOMO_ERR_NOT_CONVERGED, "eikonal solve hit the round cap");
    if (err_word != kDevOk) return fail(TOMO_ERR_TIMEOUT, "device barrier wait timed out");
    return TOMO_OK;
}
