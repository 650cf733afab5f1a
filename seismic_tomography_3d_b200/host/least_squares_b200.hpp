// Least_squares_B200: the reference's Tomography plug-in interface
// (src/tomography/tomography.hpp:11-56) implemented over the libtomo_b200 C ABI with the
// whole iteration on the device: batched eikonal solve, ray tracing into the Jacobian,
// Tikhonov CGLS and model update.  Parameter keys, the iteration logic of
// tomography_main.cpp:19-30 and every file the reference reads or writes are kept:
//   <dobs_folder>obsData_<nodes>_samples_shot_<k>.bin          (read)
//   <first_arrival_folder><name>_times_nr<nodes>_shot_<k>.bin  (written; the same values are
//                                                                then taken from memory)
//   <illumination_folder><name>_illumination_iteration_<i>.bin (written; default folder
//                                                                ../outputs/illumination/)
//   <estimated_models_folder><name>_model_iteration_<i>.bin    (written, velocity)
//   <convergency_folder><name>_convergency.txt                 (written)
// Extra optional keys: cg_iterations (default 10, the reference's hard-coded count) and
// illumination_folder.  The binary files are written by a background thread
// (async_writer.hpp) while the iteration goes on; export_convergency() waits for all of them.
#ifndef LEAST_SQUARES_B200_HPP
#define LEAST_SQUARES_B200_HPP

#include "eikonal_b200.hpp"

#ifdef TOMO_B200_REFERENCE_TREE
#include "../tomography.hpp"
#endif

class Least_squares_B200 : public Tomography {
private:
    int tk_order = 2;
    float lambda = 0.0f;
    float dx_tomo = 0, dy_tomo = 0, dz_tomo = 0;
    int nx_tomo = 0, ny_tomo = 0, nz_tomo = 0;
    int cg_iterations = 10;
    std::string illumination_folder;
    Eikonal_B200 *b200 = nullptr;

    void info_message();

public:
    void set_parameters();
    void import_obs_data();

    void forward_modeling();
    void import_cal_data();

    bool converged();

    void optimization();
    void model_update();

    void export_convergency();
    Least_squares_B200();
    ~Least_squares_B200();
};

#endif
