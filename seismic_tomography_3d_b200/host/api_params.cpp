// C ABI over the parameters.txt reader and the geometry generators (include/tomo_b200.h).
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "tomo_b200.h"
#include "tomo_b200_interface.hpp"

extern "C" {

int tomo_catch_parameter(const char *key, const char *parameter_file, char *out, int cap)
{
    if (!key || !parameter_file || !out || cap < 1) return TOMO_ERR_INVALID_ARG;
    const std::string v = catch_parameter(key, parameter_file);
    if ((int)v.size() + 1 > cap) return TOMO_ERR_INVALID_ARG;
    std::memcpy(out, v.c_str(), v.size() + 1);
    return (int)v.size();
}

int tomo_geometry(const char *parameter_file, const char *name, int type, float *xyz, int cap)
{
    if (!parameter_file || !name || (type != 0 && type != 1) || cap < 0) return TOMO_ERR_INVALID_ARG;
    try {
        // held as the concrete type (the reference's Geometry has no virtual destructor)
        std::unique_ptr<Regular> reg(type == 0 ? new Regular() : nullptr);
        std::unique_ptr<Circular> circ(type == 1 ? new Circular() : nullptr);
        Geometry *g = reg ? static_cast<Geometry *>(reg.get()) : static_cast<Geometry *>(circ.get());
        g->set_geometry(parameter_file, name);
        const int n = g->all;
        for (int i = 0; i < n && i < cap && xyz; i++) {
            xyz[3 * i + 0] = g->x[i];
            xyz[3 * i + 1] = g->y[i];
            xyz[3 * i + 2] = g->z[i];
        }
        delete[] g->x;
        delete[] g->y;
        delete[] g->z;
        return n;
    } catch (const std::exception &) {
        return TOMO_ERR_IO;
    }
}

}  // extern "C"
