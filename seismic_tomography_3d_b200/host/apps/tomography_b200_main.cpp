// tomography_b200 <parameters.txt>: the reference's tomography.exe loop
// (src/tomography/tomography_main.cpp:7-43) with the device-resident Least_squares_B200.
#include <chrono>
#include <exception>
#include <iostream>

#include "../least_squares_b200.hpp"

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " parameters.txt\n";
        return 2;
    }
    try {
        const auto ti = std::chrono::system_clock::now();
        Least_squares_B200 tomography;
        tomography.parameters = argv[1];
        tomography.set_parameters();
        tomography.import_obs_data();
        while (true) {
            tomography.forward_modeling();
            tomography.import_cal_data();
            if (tomography.converged()) break;
            tomography.optimization();
            tomography.model_update();
        }
        tomography.export_convergency();
        const std::chrono::duration<double> dt = std::chrono::system_clock::now() - ti;
        std::cout << "\nTomography run time: " << dt.count() << " s." << std::endl;
    } catch (const std::exception &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    return 0;
}
