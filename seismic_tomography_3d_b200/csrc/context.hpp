// Device context behind the C ABI: owns the stream, the model and every device buffer.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/tomo_b200.h"
#include "fim.cuh"
#include "fsm.cuh"

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

// CUDA graphs of tomo_iteration (api_iteration.cpp) and what they were captured with.
struct IterGraphs {
    cudaGraphExec_t a = nullptr, b = nullptr;
    std::vector<char> key_a, key_b;  // options, sizes and device addresses baked in
    long long cap = 0;               // Jacobian capacity graph B was built for
    unsigned long long *pinned = nullptr;
    bool broken = false;             // capture refused once: run eagerly from then on
};

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
    // staged velocity uploads (tomo_stage_velocity / tomo_commit_velocity)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_staged = nullptr;      // the staged copy has landed
    cudaEvent_t ev_stage_free = nullptr;  // the last commit has read the staging buffer
    tomo::DevBuf<float> vel_stage;
    bool staged = false, stage_read = false;
    tomo::DevBuf<float> S;         // brick-major padded slowness
    tomo::DevBuf<float> scratch_v; // staging for uploads / unbrick
    bool have_model = false;

    // last eikonal solve
    tomo::DevBuf<float> T;
    tomo::DevBuf<unsigned> qflag, lists, ctrl;
    tomo::DevBuf<unsigned> qflag8;  // queue flags of the 8^3 groups (TOMO_BRICK_8 solves)
    tomo::DevBuf<unsigned> fim_keys, band_min, band_park, band_pcnt;  // time-band ordering (per brick keys,
                                                                      // per-shot minima, parking lists, counts)
    tomo::DevBuf<unsigned> tune_word;            // autotuner scratch (largest slowness)
    tomo::DevBuf<float> fsm_T;                      // TOMO_OP_NGB sweep grids (with halo)
    tomo::DevBuf<tomo::FsmShot> fsm_shots;
    tomo::DevBuf<unsigned> fsm_bar;                 // barrier words (+ the tiled schedule's cursors)
    tomo::DevBuf<int> fsm_tab;                      // tiled schedule: tile-diagonal tables
    tomo::DevBuf<unsigned> fsm_flags;               // tiled schedule: per-tile sweep flags
    tomo::DevBuf<unsigned long long> stats;
    tomo::DevBuf<tomo::ShotDesc> shots_d;
    tomo::DevBuf<tomo::ShotDesc> shots_redo;        // warm start: shots solved again from INF
    tomo::DevBuf<unsigned long long> viol;          // warm start: per-shot check counts
    std::vector<tomo::ShotDesc> shots_h;
    std::vector<tomo_point> shot_pos;
    tomo::DevBuf<float> rec;       // 3*nrec: x | y | z
    tomo::DevBuf<float> t_recv;    // nshots*nrec
    std::vector<tomo_point> rec_h;
    // what `rec` and `shots_d` hold on the device (as last uploaded), so that a batch with
    // the same receivers or descriptors as the previous call is not uploaded again
    std::vector<float> rec_up;
    std::vector<tomo::ShotDesc> sd_up;
    int nshots = 0, nrec = 0;
    bool have_solve = false;
    // launch shape chosen by tomo_eik_autotune (0: not tuned)
    int tuned_block_warps = 0, tuned_occupancy = 0, tuned_max_inner = 0;
    int tuned_brick = 0;          // 0: none chosen (4^3); TOMO_BRICK_4 / TOMO_BRICK_8
    int tuned_schedule = 0;       // 0: none chosen (rounds); TOMO_SCHED_PAIR
    float tuned_time_band = 0.f;  // 0: none chosen (off)

    cudaEvent_t ev[8] = {};
    unsigned *pinned_ctrl = nullptr;  // kCtrlWords + stats

    // ---- tomography (api_tomography.cpp) -----------------------------------------------
    // ray tracing scratch
    tomo::DevBuf<uint2> runs;
    tomo::DevBuf<int> nuniq, ray_status, ray_steps;
    tomo::DevBuf<float> final_dist, spos, tk_coef, illum;
    // A = [G ; lambda L] in CSR and its transpose
    tomo::DevBuf<int> a_ptr, a_idx, t_ptr, t_idx;
    tomo::DevBuf<float> a_val, t_val;
    tomo::DevBuf<int> sort_keys, sort_keys_out, sort_pos, sort_pos_out, rows_of;
    tomo::DevBuf<unsigned char> cub_temp, scan_temp, reduce_temp, sort_temp;
    tomo::DevBuf<long long> csr_sizes;  // [0] ray non-zeros, [1] all non-zeros (device side)
    tomo::DevBuf<float> smin;           // smallest slowness of the model (per-ray cap)
    tomo::DevBuf<unsigned> ray_keys, ray_keys_out;  // march order of the rays
    tomo::DevBuf<int> ray_iota, ray_order;
    tomo::DevBuf<unsigned char> order_temp;
    int n_data = 0, n_model = 0, n_rows = 0, tk_order = 0;
    int nxt = 0, nyt = 0, nzt = 0;
    float dxt = 0, dyt = 0, dzt = 0;
    long long nnz_g = 0, nnz = 0;
    bool have_jacobian = false, have_illum = false;
    // CGLS and model update
    tomo::DevBuf<float> dobs, rhs, x;                 // x: CGLS solution in FP32
    tomo::DevBuf<double> cg_x, cg_s, cg_r, cg_p, cg_q;  // CGLS vectors (FP64)
    tomo::DevBuf<double> partials, hist, norm2;
    tomo::DevBuf<unsigned> cg_ctrl;
    tomo::DevBuf<int> cg_long;                // long rows of A' (M) and their count (last entry)
    tomo::DevBuf<unsigned char> cg_ltemp;     // scratch of the long-row selection
    tomo::DevBuf<float> dm, dm_smooth, vel_out, gauss_kernel;
    bool have_dobs = false, have_x = false;
    int n_dobs = 0;
    tomo::IterGraphs iter;
};
