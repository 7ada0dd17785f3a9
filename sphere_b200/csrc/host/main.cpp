// main.cpp -- the `sphere` executable: the command line of the reference
// (src/main.cpp:27-182) over the DEM class.  For every input binary it builds
// a DEM (read, check, upload) and runs the time loop, writing
// output/<sid>.outputNNNNN.bin and output/<sid>.status.dat.
//
// Flags: -h/--help, -V/--version, -q/--quiet, -n/--dry, -dc/--dont-check,
// -r/--render (render the input files to img_out/<sid>.ppm instead of
// simulating) and -m/--method <method> [<maxval> [-l <cutoff>]] (the colour
// map: normal, pres, vel, angvel, xdisp, angpos).
#include <cstdlib>
#include <iostream>
#include <string>

#include "sphere.h"

int main(const int argc, const char *argv[])
{
    int verbose = 1, checkVals = 1, dry = 0, render = 0, nfiles = 0, method = 0;
    float max_val = 0.0f, lower_cutoff = 0.0f;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        if (a == "-h" || a == "--help") {
            std::cout << argv[0] << ": particle dynamics simulator\n"
                      << "Usage: " << argv[0] << " [OPTION[S]]... [FILE1 ...]\nOptions:\n"
                      << "-h, --help\t\tprint help\n"
                      << "-V, --version\t\tprint version information and exit\n"
                      << "-q, --quiet\t\tsuppress status messages to stdout\n"
                      << "-n, --dry\t\tshow key experiment parameters and quit\n"
                      << "-r, --render\t\trender input files instead of simulating temporal evolution\n"
                      << "-dc, --dont-check\tdon't check values before running\n"
                      << "\nRaytracer (-r) specific options:\n"
                      << "-m <method> <maxval> [-l <lower cutoff val>], or\n"
                      << "--method <method> <maxval> [-l <lower cutoff val>]\n"
                      << "\tcolor visualization method, possible values:\n"
                      << "\tnormal, pres, vel, angvel, xdisp, angpos\n"
                      << "\tif -l is appended, don't render particles with value below\n"
                      << std::endl;
            return 0;
        } else if (a == "-V" || a == "--version") {
            std::cout << "sphere (B200 DEM step), libsphk ABI version " << sph_version()
                      << "\n A discrete element method particle dynamics simulator.\n";
            return 0;
        } else if (a == "-q" || a == "--quiet") {
            verbose = 0;
        } else if (a == "-n" || a == "--dry") {
            dry = 1;
        } else if (a == "-dc" || a == "--dont-check") {
            checkVals = 0;
        } else if (a == "-r" || a == "--render") {
            render = 1;
            checkVals = 0;
        } else if (a == "-m" || a == "--method") {
            // src/main.cpp:97-134
            render = 1;
            const std::string m = (i + 1 < argc) ? argv[i + 1] : "";
            if (m == "normal") method = 0;
            else if (m == "pres") method = 1;
            else if (m == "vel") method = 2;
            else if (m == "angvel") method = 3;
            else if (m == "xdisp") method = 4;
            else if (m == "angpos") method = 5;
            else {
                std::cerr << "Visualization method not understood. See `" << argv[0]
                          << " --help` for more information." << std::endl;
                return 1;
            }
            if (method != 0) {
                max_val = (i + 2 < argc) ? (float)std::atof(argv[i + 2]) : 0.0f;
                if (i + 4 < argc && std::string(argv[i + 3]) == "-l") {
                    lower_cutoff = (float)std::atof(argv[i + 4]);
                    i += 4;
                } else {
                    i += 2;
                }
            } else {
                i += 1;
            }
        } else {
            ++nfiles;
            if (verbose == 1) std::cout << argv[0] << ": processing input file: " << a << std::endl;
            DEM dem(a, verbose, checkVals, dry, 1, nfiles == 1 ? 1 : 0);
            if (render == 1)
                dem.render(method, max_val, lower_cutoff);
            else
                dem.startTime();
        }
    }
    if (argc == 1 || nfiles == 0) {
        std::cerr << argv[0] << ": missing input binary file\n"
                  << "See `" << argv[0] << " --help` for more information" << std::endl;
        return 1;
    }
    return 0;
}
