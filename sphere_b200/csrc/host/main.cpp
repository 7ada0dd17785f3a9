// main.cpp -- the `sphere` executable: the command line of the reference
// (src/main.cpp:27-182) over the DEM class.  For every input binary it builds
// a DEM (read, check, upload) and runs the time loop, writing
// output/<sid>.outputNNNNN.bin and output/<sid>.status.dat.
//
// Flags: -h/--help, -V/--version, -q/--quiet, -n/--dry, -dc/--dont-check,
// and -r/--render, -m/--method, which name the reference's ray tracer; the
// renderer is not part of this DEM step, so those report that and exit 1.
#include <cstdlib>
#include <iostream>
#include <string>

#include "sphere.h"

int main(const int argc, const char *argv[])
{
    int verbose = 1, checkVals = 1, dry = 0, render = 0, nfiles = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        if (a == "-h" || a == "--help") {
            std::cout << argv[0] << ": particle dynamics simulator\n"
                      << "Usage: " << argv[0] << " [OPTION[S]]... [FILE1 ...]\nOptions:\n"
                      << "-h, --help\t\tprint help\n"
                      << "-V, --version\t\tprint version information and exit\n"
                      << "-q, --quiet\t\tsuppress status messages to stdout\n"
                      << "-n, --dry\t\tshow key experiment parameters and quit\n"
                      << "-r, --render\t\t(renderer not part of this build)\n"
                      << "-dc, --dont-check\tdon't check values before running\n"
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
        } else if (a == "-r" || a == "--render" || a == "-m" || a == "--method") {
            render = 1;
            break;
        } else {
            ++nfiles;
            if (verbose == 1) std::cout << argv[0] << ": processing input file: " << a << std::endl;
            DEM dem(a, verbose, checkVals, dry, 1, nfiles == 1 ? 1 : 0);
            dem.startTime();
        }
    }
    if (render) {
        std::cerr << argv[0] << ": the ray-traced renderer is not part of this build" << std::endl;
        return 1;
    }
    if (argc == 1 || nfiles == 0) {
        std::cerr << argv[0] << ": missing input binary file\n"
                  << "See `" << argv[0] << " --help` for more information" << std::endl;
        return 1;
    }
    return 0;
}
