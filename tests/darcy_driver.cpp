// darcy_driver.cpp -- TEST INFRASTRUCTURE: drives the DEM class with Darcy
// flow on (the darcyflow argument of DEM::DEM, src/sphere.h:254), which the
// reference's command line never sets (src/main.cpp constructs DEM without
// it).  Usage: darcy_driver <input.bin> <initCuda: 0 stops after set-up, 1 runs>
#include <cstdlib>

#include "sphere.h"

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    const int run = std::atoi(argv[2]);
    DEM dem(argv[1], 0, 1, 0, run, 1, 1);
    if (run) dem.startTime();
    return 0;
}
