// Shared device helpers for the tomography kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tomo {

constexpr float kInf = 1e6f;  // "not reached" value (src/eikonal/block_FIM/cuda_kernel.cuh:7)
constexpr unsigned kFull = 0xffffffffu;

// Device-side error word values (ctrl[kErr]).
enum DevErr : unsigned {
    kDevOk = 0,
    kDevBarrierTimeout = 1,
    kDevRoundCap = 2,
    kDevCapacity = 3,
};

// Control-block layout shared by the persistent kernels.
enum CtrlSlot : int {
    kCnt0 = 0, kCnt1 = 1, kCnt2 = 2,  // work-list counters (3-way rotation)
    kBarCount = 3, kBarGen = 4,       // grid barrier
    kErr = 5,                         // DevErr
    kRounds = 6,                      // rounds run (written by block 0)
    kCur0 = 7, kCur1 = 8, kCur2 = 9,  // per-round fetch cursors (3-way rotation)
    kCtrlWords = 16,
};

#ifdef __CUDACC__
__device__ __forceinline__ unsigned ld_volatile(const unsigned *p)
{
    return *reinterpret_cast<const volatile unsigned *>(p);
}

// Software grid barrier for a cooperatively launched (co-resident) grid.  The wait is
// bounded: after `spin_limit` polls it records kDevBarrierTimeout and returns false, so a
// lost block can never hang the GPU.  Returns false if any block recorded an error; every
// thread of a block gets the same answer (thread 0's read of the error word), so a block
// never splits over an error raised while it passes the barrier.
__device__ __forceinline__ bool grid_barrier(unsigned *ctrl, unsigned long long spin_limit)
{
    __shared__ unsigned err;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
        const unsigned gen = ld_volatile(ctrl + kBarGen);
        __threadfence();
        const unsigned arrived = atomicAdd(ctrl + kBarCount, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(ctrl + kBarCount, 0u);
            __threadfence();
            atomicAdd(ctrl + kBarGen, 1u);
        } else {
            unsigned long long spins = 0;
            while (ld_volatile(ctrl + kBarGen) == gen) {
                if (++spins > spin_limit) {
                    atomicCAS(ctrl + kErr, 0u, (unsigned)kDevBarrierTimeout);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        err = ld_volatile(ctrl + kErr);
    }
    __syncthreads();
    return err == 0u;
}

// Grid-wide barrier on a monotone arrival counter: the k-th barrier of a launch (k = epoch,
// counted by every block) completes when ctrl[kBarCount] reaches (k + 1) * blocks.  There is
// no reset and no generation word, so the last block to arrive does no extra atomics.  The
// counter starts at 0 for the launch; the waits are bounded as in grid_barrier.
__device__ __forceinline__ bool grid_sync(unsigned *ctrl, unsigned &epoch, unsigned long long spin_limit)
{
    __shared__ unsigned err;  // the error word as thread 0 read it: one answer for the block
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        const unsigned target = epoch * (gridDim.x * gridDim.y * gridDim.z);
        __threadfence();
        atomicAdd(ctrl + kBarCount, 1u);
        unsigned long long spins = 0;
        while (ld_volatile(ctrl + kBarCount) < target) {
            if (++spins > spin_limit) {
                atomicCAS(ctrl + kErr, 0u, (unsigned)kDevBarrierTimeout);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        err = ld_volatile(ctrl + kErr);
    }
    __syncthreads();
    return err == 0u;
}

// IEEE FP32 arithmetic that the compiler may not contract into FMAs: used wherever the
// reference's FP32 operation order is restated bit for bit.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// trilinear (src/utils/interpolation/trilinear.cpp:3-20), same operation order.
__device__ __forceinline__ float trilinear_ref(float c000, float c001, float c100, float c101,
                                               float c010, float c011, float c110, float c111,
                                               float x0, float x1, float y0, float y1, float z0,
                                               float z1, float x, float y, float z)
{
    const float xd = fdiv(fsub(x, x0), fsub(x1, x0));
    const float yd = fdiv(fsub(y, y0), fsub(y1, y0));
    const float zd = fdiv(fsub(z, z0), fsub(z1, z0));
    const float c00 = fadd(fmul(c000, fsub(1.0f, xd)), fmul(c100, xd));
    const float c01 = fadd(fmul(c001, fsub(1.0f, xd)), fmul(c101, xd));
    const float c10 = fadd(fmul(c010, fsub(1.0f, xd)), fmul(c110, xd));
    const float c11 = fadd(fmul(c011, fsub(1.0f, xd)), fmul(c111, xd));
    const float c0 = fadd(fmul(c00, fsub(1.0f, yd)), fmul(c10, yd));
    const float c1 = fadd(fmul(c01, fsub(1.0f, yd)), fmul(c11, yd));
    return fadd(fmul(c0, fsub(1.0f, zd)), fmul(c1, zd));
}

#endif  // __CUDACC__

}  // namespace tomo
