// sphere.h -- the DEM class: the reference's host-side driver API
// (src/sphere.h:12-322) over libsphk's C ABI (include/sphk.h).
//
// Public interface kept from the reference (src/sphere.h:244-273):
// constructor DEM(inputbin, verbosity, checkVals, dry, initCuda,
// transferConstMem, darcyflow), readbin, writebin, checkValues,
// reportValues, startTime, and the destructor.  The state is held in the
// reference's host layout (Float4 rows, src/datatypes.h:17-33) and moved to
// and from the device with sph_upload / sph_download.  With darcyflow = 1 and
// nu > 0 the Darcy flow runs with the step (src/darcy.cpp, src/darcy.cuh):
// its grid is read from and written to the files' fluid section, set up by
// sph_darcy_init and stepped on the device.  render() draws the current
// state with the reference's ray tracer (sph_render) and writePPM saves it
// into img_out/<sid>.ppm.  The analysis members minPos, maxPos and
// findOverlaps and the Darcy array printers (src/sphere.cpp:487-602,
// src/darcy.cpp:483-528,801-824) work on the host state.  The
// lattice-Boltzmann coupling (nu > 0 without darcyflow) and the porosity and
// force-chain tools are not part of this build: they report that and exit.
#ifndef SPHERE_B200_SPHERE_H_
#define SPHERE_B200_SPHERE_H_

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "sphk.h"

// The reference's Float3 in its double-precision build (src/datatypes.h).
struct Float3 {
    double x, y, z;
};

class DEM {
  public:
    DEM(std::string inputbin, const int verbosity = 1, const int checkVals = 1,
        const int dry = 0, const int initCuda = 1, const int transferConstMem = 1,
        const int darcyflow = 0);
    ~DEM();

    // binary state file, src/file_io.cpp:29-490
    void readbin(const char *target);
    void writebin(const char *target);

    // pre-flight checks and parameter report, src/sphere.cpp:104-341
    void checkValues();
    void reportValues();

    // time loop, src/device.cu:576-1299
    void startTime();

    // outside the DEM step (renderer, analysis tools)
    void render(const int method = 1, const float maxval = 1.0e3f,
                const float lower_cutoff = 0.0f, const float focalLength = 1.0f,
                const unsigned int img_width = 800, const unsigned int img_height = 800);
    void porosity(const int z_slices = 10);
    void forcechains(const std::string format = "interactive", const int threedim = 1,
                     const double lower_cutoff = 0.0, const double upper_cutoff = 1.0e9);

    // the image of the last render() as binary PPM, src/file_io.cpp:493-516
    void writePPM(const char *target);

    // smallest / largest particle coordinate in each dimension, each
    // starting from 0 as the reference's do (src/sphere.cpp:487-551)
    Float3 minPos();
    Float3 maxPos();

    // every overlapping pair i < j in (i, j) order with its delta_n < 0,
    // src/sphere.cpp:556-602
    void findOverlaps(std::vector<std::vector<unsigned int>> &ij, std::vector<double> &delta_n_ij);

    // a field over the Darcy cell grid (ghost nodes included, the layout of
    // the fluid section) as text, src/darcy.cpp:483-528,801-824
    void printDarcyArray(FILE *stream, double *arr);
    void printDarcyArray(FILE *stream, double *arr, std::string desc);
    void printDarcyArray(FILE *stream, Float3 *arr);
    void printDarcyArray(FILE *stream, Float3 *arr, std::string desc);
    void writeDarcyArray(double *array, const char *filename);
    void writeDarcyArray(Float3 *array, const char *filename);

  private:
    std::string inputbin_, sid_;
    int verbose_ = 1;
    int darcy_ = 0;

    // time (src/datatypes.h:62-68)
    double dt_ = 0.0, current_ = 0.0, total_ = 0.0, file_dt_ = 0.0;
    uint32_t step_count_ = 0;

    // configuration and state in the reference host layout
    sph_config cfg_{};
    std::vector<double> x_, xysum_, vel_, force_, angpos_, angvel_, torque_;
    std::vector<double> es_dot_, es_, ev_dot_, ev_, p_;
    std::vector<double> walls_nx_, walls_mvfd_;
    std::vector<uint32_t> bonds_;
    std::vector<double> bonds_delta_, bonds_omega_;
    double nu_ = 0.0;
    std::vector<char> fluid_trailer_;   // carried unchanged when nu > 0 without Darcy flow

    // Darcy grid (DEM::d, src/darcy.cpp:17-38): (num+2)^3 nodes with ghosts
    std::vector<double> d_H_, d_H_new_, d_V_, d_dH_, d_K_, d_T_, d_Ss_, d_W_, d_phi_, d_dphi_;
    bool darcyOn() const { return nu_ > 0.0 && darcy_ == 1; }
    size_t darcyNode(int x, int y, int z) const;
    void initDarcyMem();
    void initDarcy();
    void endDarcy();
    sph_darcy_state darcyState();

    sph_ctx *ctx_ = nullptr;

    // the last render(): RGBA bytes, width_ x height_
    std::vector<unsigned char> img_;
    unsigned int width_ = 0, height_ = 0;

    void initDevice();
    void upload();
    void download();
    void fail(int rc, const char *where);
    sph_host_state hostState();
};

#endif
