// Least_squares_B200: see least_squares_b200.hpp.  Mirrors Least_squares
// (src/tomography/least_squares/least_squares.cpp) step for step, device-resident.
#include "least_squares_b200.hpp"

#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {
void check(tomo_ctx *ctx, int status, const char *what)
{
    if (status != TOMO_OK)
        throw std::runtime_error(std::string("Least_squares_B200 ") + what + ": " + tomo_status_string(status) + " (" +
                                 (ctx ? tomo_last_error(ctx) : "") + ")");
}
}  // namespace

void Least_squares_B200::info_message()
{
    eikonal->info_message();
    if (iteration == max_iteration)
        std::cout << "------- Checking final residuo ------------\n\n";
    else
        std::cout << "------- Computing iteration " << iteration + 1 << " of " << max_iteration << " ------------\n\n";
    if (iteration > 0) std::cout << "Previous iteration residuo: " << residuo[(size_t)iteration - 1] << "\n\n";
}

void Least_squares_B200::set_parameters()
{
    const int type = std::stoi(catch_parameter("eikonal_type", parameters));
    if (type != 3)
        throw std::invalid_argument("Least_squares_B200 runs the device eikonal solver: set eikonal_type = 3");
    b200 = new Eikonal_B200();
    eikonal = b200;
    eikonal->parameters = parameters;
    eikonal->set_parameters();

    n_data = eikonal->total_shots * eikonal->total_nodes;
    max_iteration = std::stoi(catch_parameter("max_iteration", parameters));
    lambda = std::stof(catch_parameter("tk_param", parameters));
    tk_order = (int)std::stof(catch_parameter("tk_order", parameters));
    smooth = str2bool(catch_parameter("smooth", parameters));
    window = std::stoi(catch_parameter("filter_samples", parameters));
    stdv = std::stof(catch_parameter("standard_deviation", parameters));
    dx_tomo = std::stof(catch_parameter("dx_tomo", parameters));
    dy_tomo = std::stof(catch_parameter("dy_tomo", parameters));
    dz_tomo = std::stof(catch_parameter("dz_tomo", parameters));
    nz_tomo = (int)((eikonal->nz - 1) * eikonal->dz / dz_tomo) + 1;
    nx_tomo = (int)((eikonal->nx - 1) * eikonal->dx / dx_tomo) + 1;
    ny_tomo = (int)((eikonal->ny - 1) * eikonal->dy / dy_tomo) + 1;
    n_model = nx_tomo * ny_tomo * nz_tomo;

    obs_data_folder = catch_parameter("dobs_folder", parameters);
    cal_data_folder = catch_parameter("first_arrival_folder", parameters);
    convergency_folder = catch_parameter("convergency_folder", parameters);
    estimated_model_folder = catch_parameter("estimated_models_folder", parameters);
    const std::string cg = catch_parameter("cg_iterations", parameters);
    cg_iterations = cg.empty() ? 10 : std::stoi(cg);
    illumination_folder = catch_parameter("illumination_folder", parameters);
    if (illumination_folder.empty()) illumination_folder = "../outputs/illumination/";

    iteration = 0;
    dobs = new float[(size_t)n_data]();
    dcal = new float[(size_t)n_data]();
    dm = new float[(size_t)eikonal->nPoints]();
}

void Least_squares_B200::import_obs_data()
{
    std::vector<float> data((size_t)eikonal->total_nodes);
    for (int shot = 0; shot < eikonal->total_shots; shot++) {
        read_binary_float(obs_data_folder + "obsData_" + std::to_string(eikonal->total_nodes) + "_samples_shot_" +
                              std::to_string(shot + 1) + ".bin",
                          data.data(), eikonal->total_nodes);
        for (int r = 0; r < eikonal->total_nodes; r++) dobs[(size_t)shot * eikonal->total_nodes + r] = data[(size_t)r];
    }
}

void Least_squares_B200::forward_modeling()
{
    eikonal->prepare_volumes();
    for (int i = 0; i < eikonal->total_shots; i++) {
        eikonal->shot_id = i;
        info_message();
        // The first call solves every shot in one launch; the field copy per shot keeps
        // travel_time meaningful for callers of the reference interface.
        eikonal->eikonal_equation();
        eikonal->write_first_arrival();
    }
    // Ray tracing of all shots on the device, from the device-resident fields.
    tomo_jacobian_opts o{};
    o.dx = dx_tomo;
    o.dy = dy_tomo;
    o.dz = dz_tomo;
    o.tk_order = tk_order;
    o.tk_param = lambda;
    o.illumination = 1;
    tomo_jacobian_stats st{};
    check(b200->context(), tomo_build_jacobian(b200->context(), &o, &st), "Jacobian");
    if (st.rays_ok != st.rays)
        std::cout << "Ray tracing: " << st.rays - st.rays_ok << " of " << st.rays
                  << " rays cut (stalled next to the source: " << st.rays_stalled << ")\n";
    std::vector<float> illum((size_t)eikonal->nPoints);
    check(b200->context(), tomo_illumination(b200->context(), illum.data()), "illumination");
    tomo_io::AsyncWriter::instance().write_floats(illumination_folder + eikonal->name + "_illumination_iteration_" +
                                                      std::to_string(iteration) + ".bin",
                                                  illum.data(), (size_t)eikonal->nPoints);
    eikonal->destroy_volumes();
}

void Least_squares_B200::import_cal_data()
{
    // The receiver times this iteration's forward_modeling() wrote to the first-arrival
    // files are still in memory: take them from there (the same floats, bit for bit) and
    // let the files finish in the background.  Without them, read the files back as the
    // reference does, once every queued write is on disk.
    const std::vector<float> &rt = b200->receiver_times();
    if (rt.size() == (size_t)n_data) {
        std::copy(rt.begin(), rt.end(), dcal);
        return;
    }
    tomo_io::AsyncWriter::instance().drain();
    std::vector<float> data((size_t)eikonal->total_nodes);
    for (int shot = 0; shot < eikonal->total_shots; shot++) {
        read_binary_float(cal_data_folder + eikonal->name + "_times_nr" + std::to_string(eikonal->total_nodes) +
                              "_shot_" + std::to_string(shot + 1) + ".bin",
                          data.data(), eikonal->total_nodes);
        for (int r = 0; r < eikonal->total_nodes; r++) dcal[(size_t)shot * eikonal->total_nodes + r] = data[(size_t)r];
    }
}

bool Least_squares_B200::converged()
{
    // FP32 accumulation as the reference (least_squares.cpp:303-307)
    float r = 0.0f;
    for (int i = 0; i < n_data; i++) r += powf(dobs[i] - dcal[i], 2.0f);
    residuo.push_back(sqrtf(r));
    if (iteration >= max_iteration) {
        std::cout << "\nFinal residuo: " << sqrtf(r) << std::endl;
        return true;
    }
    iteration += 1;
    return false;
}

void Least_squares_B200::optimization()
{
    std::cout << "Solving linear system using Tikhonov regularization with order " + std::to_string(tk_order) + "\n\n";
    tomo_ctx *ctx = b200->context();
    check(ctx, tomo_set_observed(ctx, dobs, n_data), "observed data");
    check(ctx, tomo_cgls(ctx, cg_iterations, nullptr, nullptr, nullptr), "CGLS");
}

void Least_squares_B200::model_update()
{
    tomo_ctx *ctx = b200->context();
    tomo_update_opts o{};
    o.smooth = smooth ? 1 : 0;
    o.filter_samples = window;
    o.standard_deviation = stdv;
    o.use_reference_masks = 1;
    std::vector<float> velocity((size_t)eikonal->nPoints);
    check(ctx, tomo_model_update(ctx, &o, velocity.data()), "model update");
    // the host slowness stays the model state, as Eikonal::slowness in the reference
    check(ctx, tomo_get_slowness(ctx, eikonal->slowness), "slowness copy");
    tomo_io::AsyncWriter::instance().write_floats(estimated_model_folder + eikonal->name + "_model_iteration_" +
                                                      std::to_string(iteration) + ".bin",
                                                  velocity.data(), (size_t)eikonal->nPoints);
}

void Least_squares_B200::export_convergency()
{
    std::ofstream f(convergency_folder + eikonal->name + "_convergency.txt", std::ios::out);
    for (float r : residuo) f << r << "\n";
    // the run ends here: every model, illumination and first-arrival file is on disk
    tomo_io::AsyncWriter::instance().drain();
}

Least_squares_B200::Least_squares_B200()
{
    // the interface's raw pointers start out empty so that an exception thrown by
    // set_parameters() leaves a destructible object
    dm = dobs = dcal = nullptr;
    eikonal = nullptr;
    iteration = 0;
}

Least_squares_B200::~Least_squares_B200()
{
    delete b200;
    delete[] dobs;
    delete[] dcal;
    delete[] dm;
}
