// Device context behind the C ABI: owns the stream, the model and every device buffer.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/tomo_b200.h"
#include "fim.cuh"

namespace tomo {

// Grow-only device buffer.
template <typename T>
struct DevBuf {
    T *ptr = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&ptr), (n ? n : 1) * sizeof(T));
        if (e == cudaSuccess) cap = n;
        return e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

struct Jacobian;  // ray tracing output (ray.cu)

}  // namespace tomo

struct tomo_ctx {
    tomo_grid g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    // padded model (multiple of the brick edge) and its brick grid
    int nxx = 0, nyy = 0, nzz = 0, gbx = 0, gby = 0, gbz = 0;
    tomo::DevBuf<float> slow;      // natural layout, nz*nx*ny (the model state)
    tomo::DevBuf<float> S;         // brick-major padded slowness
    tomo::DevBuf<float> scratch_v; // staging for uploads / unbrick
    bool have_model = false;

    // last eikonal solve
    tomo::DevBuf<float> T;
    tomo::DevBuf<unsigned> qflag, lists, ctrl;
    tomo::DevBuf<unsigned long long> stats;
    tomo::DevBuf<tomo::ShotDesc> shots_d;
    std::vector<tomo::ShotDesc> shots_h;
    std::vector<tomo_point> shot_pos;
    tomo::DevBuf<float> rec;       // 3*nrec: x | y | z
    tomo::DevBuf<float> t_recv;    // nshots*nrec
    std::vector<tomo_point> rec_h;
    int nshots = 0, nrec = 0;
    bool have_solve = false;

    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    unsigned *pinned_ctrl = nullptr;  // kCtrlWords + stats
};
