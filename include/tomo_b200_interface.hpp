// C++ plug-in interface of the reference, mirrored member for member so that the
// B200 classes (seismic_tomography_3d_b200/host/) compile either against this header
// (this repository's own executables) or against the reference's own headers
// (src/eikonal/eikonal.hpp, src/tomography/tomography.hpp) when dropped into its tree
// with -DTOMO_B200_REFERENCE_TREE.  Like the reference's, the classes declare no virtual
// destructors, so both builds give them the same virtual tables.  The shapes follow:
//   Geometry   src/geometry/geometry.hpp:8-30
//   Eikonal    src/eikonal/eikonal.hpp:15-58
//   Tomography src/tomography/tomography.hpp:11-56
#ifndef TOMO_B200_INTERFACE_HPP
#define TOMO_B200_INTERFACE_HPP

#include <string>
#include <vector>

// ---- file_manager (src/utils/file_manager/file_manager.hpp) -----------------------------
bool str2bool(std::string s);
void read_binary_float(std::string path, float *array, int n);
void write_binary_float(std::string path, float *array, int n);
void read_text_file(std::string path, std::vector<std::string> &elements);
std::string catch_parameter(std::string target, std::string file);
std::vector<std::string> split(std::string s, char delimiter);

// ---- trilinear (src/utils/interpolation/trilinear.hpp) -----------------------------------
float trilinear(float c000, float c001, float c100, float c101, float c010, float c011, float c110, float c111,
                float x0, float x1, float y0, float y1, float z0, float z1, float x, float y, float z);

// ---- Geometry --------------------------------------------------------------------------
class Geometry {
protected:
    bool topography;
    float elevation;
    std::string topo_file;
    std::string output_file;

    virtual void set_topography() = 0;
    virtual void build_geometry() = 0;
    virtual void write_geometry() = 0;

public:
    int all;

    float *x;
    float *y;
    float *z;

    virtual void set_geometry(std::string parameters, std::string name) = 0;
};

// Regular grid of points between the SW, NW and SE corners (regular/regular.cpp).
class Regular final : public Geometry {
private:
    float sw[2] = {0, 0}, nw[2] = {0, 0}, se[2] = {0, 0};
    int lines_x = 0, lines_y = 0;
    void set_topography();
    void build_geometry();
    void write_geometry();

public:
    void set_geometry(std::string parameters, std::string name);
};

// Rings of points around a centre (circular/circular.cpp).
class Circular final : public Geometry {
private:
    float cx = 0, cy = 0, arc = 0;
    std::vector<float> radii;
    void set_topography();
    void build_geometry();
    void write_geometry();

public:
    void set_geometry(std::string parameters, std::string name);
};

// ---- Eikonal ---------------------------------------------------------------------------
class Eikonal {
protected:
    bool reciprocity;
    bool export_time_volume;
    bool export_first_arrival;

    std::string time_volume_folder;
    std::string first_arrival_folder;

    virtual void expand_model() = 0;
    virtual void reduce_model() = 0;

public:
    float dx, dy, dz;
    int nx, ny, nz, nPoints;
    int nxx, nyy, nzz, nPointsB;

    float *slowness;
    float *travel_time;
    float *first_arrival;

    Geometry *shots;
    Geometry *nodes;

    std::string name;
    std::string parameters;

    int shot_id;
    int total_shots;
    int total_nodes;

    virtual void set_parameters() = 0;
    virtual void prepare_volumes() = 0;

    virtual void info_message() = 0;
    virtual void eikonal_equation() = 0;
    virtual void write_time_volume() = 0;
    virtual void write_first_arrival() = 0;

    virtual void destroy_volumes() = 0;
};

// ---- Tomography ------------------------------------------------------------------------
class Tomography {
protected:
    int max_iteration;

    int window;
    float stdv;
    bool smooth;

    float *dm;
    float *dobs;
    float *dcal;

    int n_data;
    int n_model;

    std::string obs_data_folder;
    std::string cal_data_folder;
    std::string convergency_folder;
    std::string estimated_model_folder;

    std::vector<float> residuo;

    Eikonal *eikonal;

    virtual void info_message() = 0;

public:
    int iteration;
    std::string parameters;

    virtual void set_parameters() = 0;
    virtual void import_obs_data() = 0;

    virtual void forward_modeling() = 0;
    virtual void import_cal_data() = 0;

    virtual bool converged() = 0;

    virtual void optimization() = 0;
    virtual void model_update() = 0;

    virtual void export_convergency() = 0;
};

#endif
