// TEST INFRASTRUCTURE ONLY -- drives the reference's own Eikonal classes
// (phbastosa/seismic_tomography_3D, compiled unmodified from its sources by
// oracle/Makefile into oracle/_ref/) through their public API:
//   parameters -> set_parameters() -> prepare_volumes() -> eikonal_equation() -> travel_time
// (src/eikonal/eikonal.hpp:15-58, src/eikonal/eikonal_main.cpp:18-33).
// Used by tests/ (parity pins) and bench.py's reference / CPU-baseline legs only.
//
// The shot position is changed between solves through the public Geometry arrays
// (shots->x/y/z, src/geometry/geometry.hpp:21-24), so one instance per thread solves
// many shots without re-reading the model.

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "eikonal/accurate_FSM/accurate_FSM.hpp"
#include "eikonal/classic/classic.hpp"
#ifdef REF_WITH_FIM
#include "eikonal/block_FIM/block_FIM.hpp"
#endif

namespace {

std::string write_params(const std::string &dir, int tag, int type, int nx, int ny, int nz, float dx,
                         float dy, float dz, float sx, float sy, float sz)
{
    const std::string path = dir + "/ref_params_" + std::to_string(tag) + ".txt";
    std::ofstream f(path);
    // Unquoted values: catch_parameter strips spaces and cuts at '#'
    // (src/utils/file_manager/file_manager.cpp:74-120).
    f << "x_samples = " << nx << "\n"
      << "y_samples = " << ny << "\n"
      << "z_samples = " << nz << "\n";
    f.precision(9);
    f << "x_spacing = " << dx << "\n"
      << "y_spacing = " << dy << "\n"
      << "z_spacing = " << dz << "\n"
      << "vp_file = " << dir << "/ref_model.bin\n"
      << "reciprocity = False\n"
      << "shots_geometry_type = 0\n"
      << "nodes_geometry_type = 0\n"
      << "shots_elevation = " << sz << "\n"
      << "nodes_elevation = 0\n"
      << "shots_topography = False\n"
      << "nodes_topography = False\n"
      << "shots_topography_file = none\n"
      << "nodes_topography_file = none\n"
      << "shots_output_file = " << dir << "/ref_shots_" << tag << ".txt\n"
      << "nodes_output_file = " << dir << "/ref_nodes_" << tag << ".txt\n"
      << "shots_n_xline = 1\n"
      << "shots_n_yline = 1\n"
      << "shots_SW = " << sx << "," << sy << "\n"
      << "shots_NW = " << sx << "," << sy << "\n"
      << "shots_SE = " << sx << "," << sy << "\n"
      << "nodes_n_xline = 1\n"
      << "nodes_n_yline = 1\n"
      << "nodes_SW = 0,0\n"
      << "nodes_NW = 0,0\n"
      << "nodes_SE = 0,0\n"
      << "eikonal_type = " << type << "\n"
      << "export_time_volume = False\n"
      << "export_first_arrival = False\n"
      << "time_volume_folder = " << dir << "/\n"
      << "first_arrival_folder = " << dir << "/\n";
    return path;
}

Eikonal *make_solver(int type)
{
    switch (type) {
    case 0: return new Classic();
    case 2: return new Accurate_FSM();
#ifdef REF_WITH_FIM
    case 1: return new Block_FIM();
#endif
    default: return nullptr;
    }
}

}  // namespace

extern "C" {

// Solve nshots shots of the reference solver `type` (0 Podvin-Lecomte, 1 Block_FIM [GPU
// build only], 2 Accurate_FSM) on the model `velocity` (nz*nx*ny, z fastest), with
// nthreads host threads, one solver instance per thread.  T_out (nshots*nz*nx*ny floats)
// may be NULL to only time.  solve_seconds[s] receives the eikonal_equation() wall time
// of shot s.  Returns 0 on success.
int ref_eikonal_solve(int type, const char *workdir, int nx, int ny, int nz, float dx, float dy,
                      float dz, const float *velocity, int nshots, const float *sx, const float *sy,
                      const float *sz, float *T_out, double *solve_seconds, int nthreads)
{
    const std::string dir(workdir);
    {
        std::ofstream m(dir + "/ref_model.bin", std::ios::binary);
        if (!m) return -1;
        m.write(reinterpret_cast<const char *>(velocity), sizeof(float) * (size_t)nx * ny * nz);
    }
    if (nthreads < 1) nthreads = 1;
    if (nthreads > nshots) nthreads = nshots > 0 ? nshots : 1;
    std::atomic<int> next(0), err(0);
    const size_t npts = (size_t)nx * ny * nz;
    auto worker = [&](int tid) {
        Eikonal *e = make_solver(type);
        if (!e) { err = -2; return; }
        e->parameters = write_params(dir, tid, type, nx, ny, nz, dx, dy, dz, sx[0], sy[0], sz[0]);
        e->set_parameters();
        e->prepare_volumes();
        for (;;) {
            const int s = next.fetch_add(1);
            if (s >= nshots) break;
            e->shots->x[0] = sx[s];
            e->shots->y[0] = sy[s];
            e->shots->z[0] = sz[s];
            e->shot_id = 0;
            auto t0 = std::chrono::steady_clock::now();
            e->eikonal_equation();
            auto t1 = std::chrono::steady_clock::now();
            if (solve_seconds) solve_seconds[s] = std::chrono::duration<double>(t1 - t0).count();
            if (T_out) std::memcpy(T_out + (size_t)s * npts, e->travel_time, sizeof(float) * npts);
        }
        e->destroy_volumes();
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++) pool.emplace_back(worker, t);
    for (auto &th : pool) th.join();
    return err.load();
}

// The reference's own catch_parameter (src/utils/file_manager/file_manager.cpp:74-120).
int ref_catch_parameter(const char *key, const char *file, char *out, int cap)
{
    const std::string v = catch_parameter(key, file);
    if ((int)v.size() + 1 > cap) return -1;
    std::memcpy(out, v.c_str(), v.size() + 1);
    return (int)v.size();
}

// The reference's own Regular / Circular set_geometry (src/geometry/).
int ref_geometry(const char *file, const char *name, int type, float *xyz, int cap)
{
    Geometry *g = type == 0 ? static_cast<Geometry *>(new Regular()) : static_cast<Geometry *>(new Circular());
    g->set_geometry(file, name);
    for (int i = 0; i < g->all && i < cap; i++) {
        xyz[3 * i] = g->x[i];
        xyz[3 * i + 1] = g->y[i];
        xyz[3 * i + 2] = g->z[i];
    }
    return g->all;
}

int ref_has_block_fim(void)
{
#ifdef REF_WITH_FIM
    return 1;
#else
    return 0;
#endif
}

}  // extern "C"
