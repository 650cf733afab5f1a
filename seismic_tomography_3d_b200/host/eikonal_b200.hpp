// Eikonal_B200: the reference's Eikonal plug-in interface (src/eikonal/eikonal.hpp:15-58)
// implemented over the libtomo_b200 C ABI.  Selected by eikonal_type = 3.
//
// Behaviour seen by the caller is that of the reference solvers: after set_parameters()
// the public fields (slowness, shots, nodes, travel_time, first_arrival, ...) exist;
// prepare_volumes() is called once per tomography iteration; per shot the caller sets
// shot_id and calls eikonal_equation(), after which travel_time holds the nz*nx*ny field,
// and write_first_arrival() fills first_arrival and writes
// <first_arrival_folder><name>_times_nr<N>_shot_<k>.bin.
//
// Underneath, the first eikonal_equation() after prepare_volumes() solves ALL shots in one
// persistent device launch; later calls copy the requested shot's field back.
#ifndef EIKONAL_B200_HPP
#define EIKONAL_B200_HPP

#include <vector>

#ifdef TOMO_B200_REFERENCE_TREE
#include "../eikonal.hpp"
#else
#include "tomo_b200_interface.hpp"
#endif
#include "async_writer.hpp"
#include "tomo_b200.h"

class Eikonal_B200 final : public Eikonal {
protected:
    tomo_ctx *ctx = nullptr;
    bool batch_ready = false;
    float time_band = 0.f;  // optional key eikonal_time_band (s): time-band ordering, 0 = off
    bool ngb = false;       // optional key eikonal_operator = fsm: Accurate_FSM's operator
    bool geometry_ready = false;
    int shots_type = 0, nodes_type = 0;  // 0 Regular, 1 Circular: deleted as that type (the
                                         // reference's Geometry has no virtual destructor)
    std::vector<float> recv_times;  // total_shots x total_nodes, trilinear receiver times

    void expand_model() {}  // padding to whole bricks happens on the device
    void reduce_model() {}  // fields are cropped on the device (tomo_eik_volume)
    void solve_batch();
    void check(int status, const char *what);

public:
    void set_parameters();
    void prepare_volumes();

    void info_message();
    void eikonal_equation();
    void write_time_volume();
    void write_first_arrival();

    void destroy_volumes();
    Eikonal_B200();
    ~Eikonal_B200();

    // for the device-resident tomography
    tomo_ctx *context() { return ctx; }
    const std::vector<float> &receiver_times() const { return recv_times; }
};

#endif
