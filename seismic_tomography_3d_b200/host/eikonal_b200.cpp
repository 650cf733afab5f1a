// Eikonal_B200: see eikonal_b200.hpp.  Parameter keys, reciprocity handling and output
// file names are those of the reference solvers (src/eikonal/block_FIM/block_FIM.cpp:71-262).
#include "eikonal_b200.hpp"

#include <algorithm>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>

void Eikonal_B200::check(int status, const char *what)
{
    if (status != TOMO_OK) {
        const char *msg = ctx ? tomo_last_error(ctx) : tomo_status_string(status);
        throw std::runtime_error(std::string("Eikonal_B200 ") + what + ": " + tomo_status_string(status) + " (" +
                                 msg + ")");
    }
}

void Eikonal_B200::set_parameters()
{
    name = "fim";  // the Jeong-Whitaker operator of Block_FIM: same output file prefix

    nx = std::stoi(catch_parameter("x_samples", parameters));
    ny = std::stoi(catch_parameter("y_samples", parameters));
    nz = std::stoi(catch_parameter("z_samples", parameters));
    nPoints = nx * ny * nz;

    dx = std::stof(catch_parameter("x_spacing", parameters));
    dy = std::stof(catch_parameter("y_spacing", parameters));
    dz = std::stof(catch_parameter("z_spacing", parameters));

    slowness = new float[(size_t)nPoints]();
    read_binary_float(catch_parameter("vp_file", parameters), slowness, nPoints);
    for (int i = 0; i < nPoints; i++) slowness[i] = 1.0f / slowness[i];

    shots_type = std::stoi(catch_parameter("shots_geometry_type", parameters));
    nodes_type = std::stoi(catch_parameter("nodes_geometry_type", parameters));
    auto make = [](int t) -> Geometry * {
        if (t == 0) return new Regular();
        if (t == 1) return new Circular();
        throw std::invalid_argument("geometry type must be 0 (regular) or 1 (circular)");
    };
    shots = make(shots_type);
    nodes = make(nodes_type);
    shots->set_geometry(parameters, "shots");
    nodes->set_geometry(parameters, "nodes");
    geometry_ready = true;

    reciprocity = str2bool(catch_parameter("reciprocity", parameters));
    if (reciprocity) {
        std::swap(shots->x, nodes->x);
        std::swap(shots->y, nodes->y);
        std::swap(shots->z, nodes->z);
        std::swap(shots->all, nodes->all);
    }
    total_shots = shots->all;
    total_nodes = nodes->all;

    // Optional (no key in the reference's files): time-band ordering of the batched solve,
    // in seconds.  Full-grid shots on smooth starting models solve 1.2-2.3x faster with
    // about 0.2 s; absent or empty keeps it off.
    const std::string band = catch_parameter("eikonal_time_band", parameters);
    time_band = band.empty() ? 0.f : std::stof(band);
    // Optional: the local operator.  "fim" (default) is Block_FIM's Jeong-Whitaker update;
    // "fsm" runs Accurate_FSM's Noble-Gesret-Belayouni sweeps on the device, bit for bit,
    // and names the outputs as Accurate_FSM does (fsm_*), so that its results can stand in
    // for those of the reference's eikonal_type = 2.
    const std::string op = catch_parameter("eikonal_operator", parameters);
    if (op == "fsm")
        ngb = true;
    else if (!op.empty() && op != "fim")
        throw std::invalid_argument("eikonal_operator must be fim or fsm");
    if (ngb) name = "fsm";

    export_time_volume = str2bool(catch_parameter("export_time_volume", parameters));
    export_first_arrival = str2bool(catch_parameter("export_first_arrival", parameters));
    time_volume_folder = catch_parameter("time_volume_folder", parameters);
    first_arrival_folder = catch_parameter("first_arrival_folder", parameters);

    travel_time = new float[(size_t)nPoints]();
    first_arrival = new float[(size_t)total_nodes]();

    // device context (optional key gpu_device, default 0)
    const std::string dev = catch_parameter("gpu_device", parameters);
    const tomo_grid g{nx, ny, nz, dx, dy, dz};
    check(tomo_ctx_create(&g, dev.empty() ? 0 : std::stoi(dev), &ctx), "context");
}

void Eikonal_B200::prepare_volumes()
{
    // The caller may have changed `slowness` (the tomography updates it in place between
    // iterations): upload it and forget the previous batch.
    nxx = nx + (4 - nx % 4) % 4;
    nyy = ny + (4 - ny % 4) % 4;
    nzz = nz + (4 - nz % 4) % 4;
    nPointsB = nxx * nyy * nzz;
    check(tomo_set_slowness(ctx, slowness), "model upload");
    batch_ready = false;
}

void Eikonal_B200::info_message()
{
    std::cout << "3D eikonal equation solver\n\n";
    std::cout << "Total x model length = " << (nx - 1) * dx << " m\n";
    std::cout << "Total Y model length = " << (ny - 1) * dy << " m\n";
    std::cout << "Total Z model length = " << (nz - 1) * dz << " m\n\n";
    std::cout << (reciprocity ? "Reciprocity = True\n\n" : "Reciprocity = False\n\n");
    std::cout << "Shot " << shot_id + 1 << " of " << total_shots << "\n";
    std::cout << "Position (x,y,z) = (" << shots->x[shot_id] << ", " << shots->y[shot_id] << ", " << shots->z[shot_id]
              << ") m\n\n";
    std::cout << (ngb ? "Solving eikonal equation with the Noble, Gesret and Belayouni (2014) formulation, "
                        "batched on B200\n\n"
                      : "Solving eikonal equation with the Jeong & Whitaker (2008) formulation, batched on B200\n\n");
}

void Eikonal_B200::solve_batch()
{
    std::vector<tomo_point> sp((size_t)total_shots), rp((size_t)total_nodes);
    for (int i = 0; i < total_shots; i++) sp[(size_t)i] = tomo_point{shots->x[i], shots->y[i], shots->z[i]};
    for (int i = 0; i < total_nodes; i++) rp[(size_t)i] = tomo_point{nodes->x[i], nodes->y[i], nodes->z[i]};
    recv_times.assign((size_t)total_shots * total_nodes, 0.0f);
    tomo_eik_opts opts{};  // defaults, plus the optional operator and time band
    opts.op = ngb ? TOMO_OP_NGB : TOMO_OP_JW;
    opts.time_band = time_band;
    check(tomo_eik_solve(ctx, total_shots, sp.data(), nullptr, total_nodes, rp.data(), recv_times.data(), &opts,
                         nullptr),
          "batched solve");
    batch_ready = true;
}

void Eikonal_B200::eikonal_equation()
{
    if (!batch_ready) solve_batch();
    check(tomo_eik_volume(ctx, shot_id, travel_time), "traveltime copy");
}

// Files go to the background writer (same bytes, path and message as write_binary_float);
// the call returns before the disk write.
void Eikonal_B200::write_time_volume()
{
    if (export_time_volume)
        tomo_io::AsyncWriter::instance().write_floats(time_volume_folder + name + "_eikonal_nz" + std::to_string(nz) +
                                                          "_nx" + std::to_string(nx) + "_ny" + std::to_string(ny) +
                                                          "_shot_" + std::to_string(shot_id + 1) + ".bin",
                                                      travel_time, (size_t)nPoints);
}

void Eikonal_B200::write_first_arrival()
{
    if (!batch_ready) solve_batch();
    // receiver times were sampled on the device with the reference's trilinear rule
    std::memcpy(first_arrival, recv_times.data() + (size_t)shot_id * total_nodes, sizeof(float) * total_nodes);
    if (export_first_arrival)
        tomo_io::AsyncWriter::instance().write_floats(first_arrival_folder + name + "_times_nr" +
                                                          std::to_string(total_nodes) + "_shot_" +
                                                          std::to_string(shot_id + 1) + ".bin",
                                                      first_arrival, (size_t)total_nodes);
}

void Eikonal_B200::destroy_volumes() { batch_ready = false; }

Eikonal_B200::Eikonal_B200()
{
    slowness = travel_time = first_arrival = nullptr;
    shots = nodes = nullptr;
    shot_id = total_shots = total_nodes = 0;
}

Eikonal_B200::~Eikonal_B200()
{
    if (ctx) tomo_ctx_destroy(ctx);
    delete[] slowness;
    delete[] travel_time;
    delete[] first_arrival;
    if (geometry_ready)  // coordinate arrays exist (swapped, never shared, under reciprocity)
        for (Geometry *g : {shots, nodes}) {
            delete[] g->x;
            delete[] g->y;
            delete[] g->z;
        }
    // as the concrete type: deleting through Geometry * would skip Circular's members
    auto destroy = [](Geometry *g, int type) {
        if (type == 1)
            delete static_cast<Circular *>(g);
        else
            delete static_cast<Regular *>(g);
    };
    destroy(shots, shots_type);  // reciprocity swaps the coordinate arrays, not the objects
    destroy(nodes, nodes_type);
}
