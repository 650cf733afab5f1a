// Acquisition geometry from parameters.txt: the reference's two generators with the same
// keys, point order and float arithmetic (src/geometry/regular/regular.cpp:6-125,
// src/geometry/circular/circular.cpp:5-93), so shot/node coordinates are bit-identical.
#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>

#include "tomo_b200_interface.hpp"

namespace {

// n points from a to b inclusive: a + (float)(step * i) with step = (b - a) / (n - 1).
std::vector<float> evenly(float a, float b, int n)
{
    std::vector<float> v;
    if (n <= 0) return v;
    if (n == 1) return {a};
    const float step = (b - a) / (float)(n - 1);
    v.reserve((size_t)n);
    for (int i = 0; i < n; i++) v.push_back(a + (float)(step * i));
    return v;
}

void read_pair(const std::string &value, float out[2])
{
    const std::vector<std::string> p = split(value, ',');
    if (p.size() < 2) throw std::invalid_argument("Error: expected an (x, y) pair");
    out[0] = std::stof(p[0]);
    out[1] = std::stof(p[1]);
}

void write_xyz(const std::string &path, int n, const float *x, const float *y, const float *z)
{
    std::ofstream f(path, std::ios::out);
    if (!f.is_open()) throw std::invalid_argument("Error: file could not be opened!");
    for (int i = 0; i < n; i++) f << x[i] << ", " << y[i] << ", " << z[i] << std::endl;
    std::cout << "Geometry file " + path + " was succesfully written." << std::endl;
}

void elevations(bool topo, const std::string &file, float elevation, int n, float *z)
{
    if (topo) {
        std::vector<std::string> lines;
        read_text_file(file, lines);
        for (int i = 0; i < n; i++) z[i] = std::stof(lines[(size_t)i]);
    } else {
        for (int i = 0; i < n; i++) z[i] = elevation;
    }
}

}  // namespace

void Regular::set_geometry(std::string parameters, std::string name)
{
    elevation = std::stof(catch_parameter(name + "_elevation", parameters));
    topography = str2bool(catch_parameter(name + "_topography", parameters));
    topo_file = catch_parameter(name + "_topography_file", parameters);
    output_file = catch_parameter(name + "_output_file", parameters);
    lines_x = std::stoi(catch_parameter(name + "_n_xline", parameters));
    lines_y = std::stoi(catch_parameter(name + "_n_yline", parameters));
    read_pair(catch_parameter(name + "_SW", parameters), sw);
    read_pair(catch_parameter(name + "_NW", parameters), nw);
    read_pair(catch_parameter(name + "_SE", parameters), se);
    build_geometry();
    set_topography();
    write_geometry();
}

void Regular::build_geometry()
{
    all = lines_x * lines_y;
    x = new float[(size_t)all]();
    y = new float[(size_t)all]();
    z = new float[(size_t)all]();
    const std::vector<float> xs = evenly(sw[0], se[0], lines_x);
    const std::vector<float> ys = evenly(sw[1], nw[1], lines_y);
    // point k + j*lines_y is (xs[j], ys[k])  (regular.cpp:95-98)
    for (size_t k = 0; k < ys.size(); k++)
        for (size_t j = 0; j < xs.size(); j++) {
            x[k + j * (size_t)lines_y] = xs[j];
            y[k + j * (size_t)lines_y] = ys[k];
        }
}

void Regular::set_topography() { elevations(topography, topo_file, elevation, all, z); }
void Regular::write_geometry() { write_xyz(output_file, all, x, y, z); }

void Circular::set_geometry(std::string parameters, std::string name)
{
    elevation = std::stof(catch_parameter(name + "_elevation", parameters));
    topo_file = catch_parameter(name + "_topography_file", parameters);
    topography = str2bool(catch_parameter(name + "_topography", parameters));
    output_file = catch_parameter(name + "_output_file", parameters);
    cx = std::stof(catch_parameter(name + "_xcenter", parameters));
    cy = std::stof(catch_parameter(name + "_ycenter", parameters));
    arc = std::stof(catch_parameter(name + "_spacing", parameters));
    radii.clear();
    for (const std::string &r : split(catch_parameter(name + "_offsets", parameters), ',')) radii.push_back(std::stof(r));
    build_geometry();
    set_topography();
    write_geometry();
}

void Circular::build_geometry()
{
    // Points every `arc` metres of chord on each ring.  The reference evaluates the
    // trigonometry in double (::sin/::cos/::acos/::atan of float arguments) and stores
    // float; the same promotions are kept so the coordinates are bit-identical.
    std::vector<float> xs, ys;
    const double two_pi = (double)(2.0f * 4.0f) * std::atan(1.0);
    for (float r : radii) {
        float theta = 0.0f;
        while ((double)theta < two_pi) {
            xs.push_back((float)((double)r * std::sin((double)theta) + (double)cx));
            ys.push_back((float)((double)r * std::cos((double)theta) + (double)cy));
            const float c = 1.0f - powf(arc, 2.0f) / (2.0f * powf(r, 2.0f));
            theta = (float)((double)theta + std::acos((double)c));
        }
    }
    all = (int)xs.size();
    x = new float[(size_t)all]();
    y = new float[(size_t)all]();
    z = new float[(size_t)all]();
    for (int i = 0; i < all; i++) {
        x[i] = xs[(size_t)i];
        y[i] = ys[(size_t)i];
    }
}

void Circular::set_topography() { elevations(topography, topo_file, elevation, all, z); }
void Circular::write_geometry() { write_xyz(output_file, all, x, y, z); }
