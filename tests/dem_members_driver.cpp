// dem_members_driver.cpp -- TEST INFRASTRUCTURE: calls the DEM class's
// analysis members (minPos, maxPos, findOverlaps) and the Darcy array
// printers on a state file, without a device, and writes what they return.
// Usage: dem_members_driver <input.bin> <output directory> <Darcy grid nodes>
#include <cstdio>
#include <string>
#include <vector>

#include "sphere.h"

int main(int argc, char **argv)
{
    if (argc < 4) return 2;
    const std::string out = argv[2];
    DEM dem(argv[1], 0, 0, 0, 0, 1, 0);
    FILE *f = fopen((out + "/minmax.txt").c_str(), "w");
    if (!f) return 3;
    const Float3 lo = dem.minPos(), hi = dem.maxPos();
    fprintf(f, "%.17g %.17g %.17g\n%.17g %.17g %.17g\n", lo.x, lo.y, lo.z, hi.x, hi.y, hi.z);
    fclose(f);
    std::vector<std::vector<unsigned int>> ij;
    std::vector<double> delta;
    dem.findOverlaps(ij, delta);
    f = fopen((out + "/overlaps.txt").c_str(), "w");
    if (!f) return 3;
    for (size_t k = 0; k < ij.size(); ++k) fprintf(f, "%u %u %.17g\n", ij[k][0], ij[k][1], delta[k]);
    fclose(f);
    // a seeded field over the (num + 2)^3 nodes of the Darcy grid
    const size_t nodes = (size_t)std::stoul(argv[3]);
    std::vector<double> s(nodes);
    std::vector<Float3> v(nodes);
    for (size_t k = 0; k < nodes; ++k) {
        s[k] = (double)((k * 2654435761ull) % 1000003ull) / 1000.0 - 500.0;
        v[k] = Float3{s[k], -0.5 * s[k], 0.25 * (double)k};
    }
    dem.writeDarcyArray(s.data(), (out + "/scalar.txt").c_str());
    dem.writeDarcyArray(v.data(), (out + "/vector.txt").c_str());
    dem.printDarcyArray(stdout, s.data(), "scalar field");
    return 0;
}
