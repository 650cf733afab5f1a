// eikonal_b200 <parameters.txt>: the reference's eikonal.exe flow
// (src/eikonal/eikonal_main.cpp:10-50) with the B200 solver, eikonal_type = 3.
#include <chrono>
#include <exception>
#include <iostream>

#include "../eikonal_b200.hpp"

int main(int argc, char **argv)
{
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " parameters.txt\n";
        return 2;
    }
    try {
        const int type = std::stoi(catch_parameter("eikonal_type", argv[1]));
        if (type != 3) {
            std::cerr << "this build provides eikonal_type = 3 (B200 batched FIM); got " << type << "\n";
            return 2;
        }
        Eikonal_B200 eik;
        eik.parameters = argv[1];
        eik.set_parameters();
        eik.prepare_volumes();
        const auto t0 = std::chrono::system_clock::now();
        for (int i = 0; i < eik.total_shots; i++) {
            eik.shot_id = i;
            eik.info_message();
            eik.eikonal_equation();
            eik.write_time_volume();
            eik.write_first_arrival();
        }
        const std::chrono::duration<double> dt = std::chrono::system_clock::now() - t0;
        std::cout << "Run time = " << dt.count() << "s.\n";
        eik.destroy_volumes();
    } catch (const std::exception &e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    return 0;
}
