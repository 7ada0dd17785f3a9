// sphere.cpp -- DEM class: construction, pre-flight checks, parameter report
// and the time loop, over libsphk's C ABI.
//
// Behaviour follows the reference host driver: DEM::DEM (src/sphere.cpp:16-77),
// checkValues (:104-246), reportValues (:249-341) and DEM::startTime
// (src/device.cu:576-1299) -- output file numbering, status.dat, the
// `float` file-interval clock (device.cu:594) and the loop condition
// time.current <= time.total.  Instead of one launch sequence and one device
// synchronisation per step, the steps between two output files are handed
// to sph_step in one call and errors are checked once per output interval.
#include "sphere.h"

#include <chrono>
#include <cmath>
#include <fstream>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <iostream>

DEM::DEM(std::string inputbin, const int verbosity, const int checkVals, const int dry,
         const int initCuda, const int transferConstMem, const int darcyflow)
    : inputbin_(inputbin), verbose_(verbosity), darcy_(darcyflow)
{
    (void)transferConstMem;   // parameters live in per-context device memory
    const size_t dotpos = inputbin.rfind('.');
    const size_t slashpos = inputbin.rfind('/');
    const size_t start = (slashpos == std::string::npos) ? 0 : slashpos + 1;
    if (dotpos == std::string::npos || dotpos < start) {
        std::cerr << "Error! Unable to extract simulation id from input file name.\n";
        sid_ = inputbin.substr(start);
    } else {
        sid_ = inputbin.substr(start, dotpos - start);
    }
    readbin(inputbin.c_str());
    if (checkVals == 1) checkValues();
    if (dry == 1) {
        reportValues();
        exit(0);
    }
    if (darcyOn()) initDarcy();   // src/sphere.cpp:52-54
    if (initCuda == 1) initDevice();
}

// ---- Darcy flow: the host side of src/darcy.cpp -----------------------------

size_t DEM::darcyNode(int x, int y, int z) const
{
    const size_t nx2 = (size_t)cfg_.num[0] + 2, ny2 = (size_t)cfg_.num[1] + 2;
    return (size_t)(x + 1) + nx2 * (size_t)(y + 1) + nx2 * ny2 * (size_t)(z + 1);
}

// initDarcyMem (src/darcy.cpp:17-38) with the cell grid; the values the
// reference leaves unset are zero here
void DEM::initDarcyMem()
{
    const size_t n = (size_t)(cfg_.num[0] + 2) * (cfg_.num[1] + 2) * (cfg_.num[2] + 2);
    for (auto *v : {&d_H_, &d_H_new_, &d_K_, &d_Ss_, &d_W_, &d_phi_, &d_dphi_}) v->assign(n, 0.0);
    for (auto *v : {&d_V_, &d_dH_, &d_T_}) v->assign(3 * n, 0.0);
}

sph_darcy_state DEM::darcyState()
{
    sph_darcy_state s{};
    s.H = d_H_.data();
    s.H_new = d_H_new_.data();
    s.V = d_V_.data();
    s.dH = d_dH_.data();
    s.K = d_K_.data();
    s.T = d_T_.data();
    s.Ss = d_Ss_.data();
    s.W = d_W_.data();
    s.phi = d_phi_.data();
    s.dphi = d_dphi_.data();
    return s;
}

// initDarcy (src/darcy.cpp:760-798)
void DEM::initDarcy()
{
    const double dx = cfg_.L[0] / cfg_.num[0], dy = cfg_.L[1] / cfg_.num[1],
                 dz = cfg_.L[2] / cfg_.num[2];
    if (verbose_ == 1) {
        std::cout << "  - Fluid grid dimensions: " << cfg_.num[0] << "*" << cfg_.num[1] << "*"
                  << cfg_.num[2] << std::endl;
        std::cout << "  - Fluid grid cell size: " << dx << "*" << dy << "*" << dz << std::endl;
    }
    sph_darcy_state s = darcyState();
    double value = 0.0;
    const int rc = sph_darcy_init(&cfg_, nu_, x_.data(), &s, &value);
    if (rc == SPH_ERR_UNSTABLE) {
        std::cerr << "Error! The explicit Darcy solution will be unstable.\n"
                  << " Reason: (" << value << " > 0.5)" << std::endl;
        exit(1);
    }
    if (rc != SPH_OK) {
        std::cerr << "Error in initDarcy. The dynamic viscosity (params.nu) should be larger "
                     "than 0.0, but is "
                  << nu_ << std::endl;
        exit(1);
    }
}

// endDarcy (src/darcy.cpp:826-836): porosity and conductivity of every cell
void DEM::endDarcy()
{
    writeDarcyArray(d_phi_.data(), "d_phi.txt");
    writeDarcyArray(d_K_.data(), "d_K.txt");
}

// printDarcyArray (src/darcy.cpp:483-528): the cells of the grid, x fastest,
// a tab after each value, a line per (y, z) row and an empty line per z
// slice; the ghost nodes are not printed.  The described forms write their
// heading to standard output whatever the stream, as the reference's do.
void DEM::printDarcyArray(FILE *stream, double *arr)
{
    for (uint32_t z = 0; z < cfg_.num[2]; ++z) {
        for (uint32_t y = 0; y < cfg_.num[1]; ++y) {
            for (uint32_t x = 0; x < cfg_.num[0]; ++x)
                fprintf(stream, "%f\t", arr[darcyNode((int)x, (int)y, (int)z)]);
            fprintf(stream, "\n");
        }
        fprintf(stream, "\n");
    }
}

void DEM::printDarcyArray(FILE *stream, double *arr, std::string desc)
{
    std::cout << "\n" << desc << ":\n";
    printDarcyArray(stream, arr);
}

void DEM::printDarcyArray(FILE *stream, Float3 *arr)
{
    for (uint32_t z = 0; z < cfg_.num[2]; ++z) {
        for (uint32_t y = 0; y < cfg_.num[1]; ++y) {
            for (uint32_t x = 0; x < cfg_.num[0]; ++x) {
                const Float3 &v = arr[darcyNode((int)x, (int)y, (int)z)];
                fprintf(stream, "%f,%f,%f\t", v.x, v.y, v.z);
            }
            fprintf(stream, "\n");
        }
        fprintf(stream, "\n");
    }
}

void DEM::printDarcyArray(FILE *stream, Float3 *arr, std::string desc)
{
    std::cout << "\n" << desc << ":\n";
    printDarcyArray(stream, arr);
}

// writeDarcyArray (src/darcy.cpp:801-824)
void DEM::writeDarcyArray(double *array, const char *filename)
{
    FILE *file = fopen(filename, "w");
    if (file) {
        printDarcyArray(file, array);
        fclose(file);
    } else {
        fprintf(stderr, "Error, could not open %s.\n", filename);
    }
}

void DEM::writeDarcyArray(Float3 *array, const char *filename)
{
    FILE *file = fopen(filename, "w");
    if (file) {
        printDarcyArray(file, array);
        fclose(file);
    } else {
        fprintf(stderr, "Error, could not open %s.\n", filename);
    }
}

DEM::~DEM()
{
    if (ctx_) sph_destroy(ctx_);
    if (verbose_ == 1) std::cout << "Freeing host memory:                             Done" << std::endl;
}

void DEM::fail(int rc, const char *where)
{
    const char *msg = ctx_ ? sph_last_error(ctx_) : "";
    std::cerr << "\nDevice error detected, checkpoint: " << where << "\nError string: " << msg
              << " (status " << rc << ")" << std::endl;
    if (rc == SPH_ERR_OUT_OF_GRID)
        std::cerr << "One or more particles moved outside the grid.\n"
                     "This could possibly be caused by a numerical instability.\n"
                     "Is the computational time step too large?" << std::endl;
    exit(EXIT_FAILURE);
}

sph_host_state DEM::hostState()
{
    sph_host_state h{};
    h.x = x_.data();
    h.xysum = xysum_.data();
    h.vel = vel_.data();
    h.force = force_.data();
    h.angpos = angpos_.data();
    h.angvel = angvel_.data();
    h.torque = torque_.data();
    h.es_dot = es_dot_.data();
    h.es = es_.data();
    h.ev_dot = ev_dot_.data();
    h.ev = ev_.data();
    h.p = p_.data();
    h.bonds = bonds_.empty() ? nullptr : bonds_.data();
    h.bonds_delta = bonds_delta_.empty() ? nullptr : bonds_delta_.data();
    h.bonds_omega = bonds_omega_.empty() ? nullptr : bonds_omega_.data();
    h.walls_nx = walls_nx_.empty() ? nullptr : walls_nx_.data();
    h.walls_mvfd = walls_mvfd_.empty() ? nullptr : walls_mvfd_.data();
    h.t_current = current_;
    return h;
}

void DEM::initDevice()
{
    if (nu_ > 0.0 && !darcyOn()) {
        std::cerr << "Error: the lattice-Boltzmann fluid coupling (nu > 0 without Darcy flow) "
                     "is not part of this DEM step implementation." << std::endl;
        exit(1);
    }
    cfg_.device = 0;
    int rc = sph_create(&cfg_, &ctx_);
    if (rc != SPH_OK) fail(rc, "sph_create");
    if (verbose_ == 1) std::cout << "  Allocating global device memory:                Done\n";
    upload();
}

void DEM::upload()
{
    sph_host_state h = hostState();
    int rc = sph_upload(ctx_, &h);
    if (rc != SPH_OK) fail(rc, "sph_upload");
    if (darcyOn()) {
        sph_darcy_state s = darcyState();
        rc = sph_darcy_upload(ctx_, nu_, &s);
        if (rc != SPH_OK) fail(rc, "sph_darcy_upload");
    }
    if (verbose_ == 1) std::cout << "  Transfering data to the device:                 Done\n";
}

void DEM::download()
{
    sph_host_state h = hostState();
    int rc = sph_download(ctx_, &h);
    if (rc != SPH_OK) fail(rc, "sph_download");
    if (darcyOn()) {
        sph_darcy_state s = darcyState();
        rc = sph_darcy_download(ctx_, &s);
        if (rc != SPH_OK) fail(rc, "sph_darcy_download");
    }
}

void DEM::checkValues()
{
    using std::cerr;
    if (cfg_.np < 1) {
        cerr << "Error: np = " << cfg_.np << '\n';
        exit(1);
    }
    if (current_ > total_ || current_ < 0.0) {
        cerr << "Error: time.current = " << current_ << " s, time.total = " << total_ << " s\n";
        exit(1);
    }
    if (cfg_.origo[0] < 0.0 || cfg_.origo[1] < 0.0 || cfg_.origo[2] < 0.0) {
        cerr << "Error: Negative values in grid.origo are known to cause problems. \n"
             << "grid.origo[0] = " << cfg_.origo[0] << " m, grid.origo[1] = " << cfg_.origo[1]
             << " m, grid.origo[2] = " << cfg_.origo[2] << " m.\n";
        exit(1);
    }
    if (cfg_.L[0] <= 0.0 || cfg_.L[1] <= 0.0 || cfg_.L[2] <= 0.0) {
        cerr << "Error: grid.L[0] = " << cfg_.L[0] << " m, grid.L[1] = " << cfg_.L[1]
             << " m, grid.L[2] = " << cfg_.L[2] << " m.\n";
        exit(1);
    }
    if (cfg_.num[0] == 0 || cfg_.num[1] == 0 || cfg_.num[2] == 0) {
        cerr << "Error: grid.num[0] = " << cfg_.num[0] << ", grid.num[1] = " << cfg_.num[1]
             << ", grid.num[2] = " << cfg_.num[2] << ".\n";
        exit(1);
    }
    if (cfg_.periodic == 2 && cfg_.num[0] < 3) {
        cerr << "Error: When 1st dimension boundaries are periodic, "
             << "there must be at least 3 cells in that dimension.";
        exit(1);
    }
    if (cfg_.periodic == 1 && (cfg_.num[0] < 3 || cfg_.num[1] < 3)) {
        cerr << "Error: When 1st and 2nd dimension boundaries are periodic, "
             << "there must be at least 3 cells in each of those dimensions.";
        exit(1);
    }
    for (uint32_t i = 0; i < cfg_.np; ++i) {
        const double *x = &x_[4 * (size_t)i];
        if (x[3] <= 0.0) {
            cerr << "Error: Particle " << i << " has a radius of " << x[3] << " m." << std::endl;
            exit(1);
        }
        if (x[0] < cfg_.origo[0] || x[1] < cfg_.origo[1] || x[2] < cfg_.origo[2] ||
            x[0] > cfg_.L[0] || x[1] > cfg_.L[1] || x[2] > cfg_.L[2]) {
            cerr << "Error: Particle " << i << " is outside of the computational grid\n"
                 << "k.x[i] = [" << x[0] << ", " << x[1] << ", " << x[2] << "]\n"
                 << "grid.origo = [" << cfg_.origo[0] << ", " << cfg_.origo[1] << ", "
                 << cfg_.origo[2] << "], grid.L = [" << cfg_.L[0] << ", " << cfg_.L[1] << ", "
                 << cfg_.L[2] << "]." << std::endl;
            exit(1);
        }
    }
    if (cfg_.nw > 0) {
        double z_max = 0.0;
        for (uint32_t i = 0; i < cfg_.np; ++i) z_max = std::max(z_max, x_[4 * (size_t)i + 2]);
        if (walls_nx_[3] < z_max) {
            cerr << "Error: One or more particles have centres above the upper, dynamic wall";
            exit(1);
        }
    }
    if (cfg_.k_n <= 0.0) {
        cerr << "Error: k_n = " << cfg_.k_n << " N/m\n";
        exit(1);
    }
    if (cfg_.rho <= 0.0) {
        cerr << "Error: rho = " << cfg_.rho << " kg/m3\n";
        exit(1);
    }
}

void DEM::reportValues()
{
    using std::cout;
    cout << "  - Number of dimensions: nd = 3\n"
         << "  - Number of particles:  np = " << cfg_.np << "\n"
         << "  - Compiled for double precision\n"
         << "  - Timestep length:      time.dt         = " << dt_ << " s\n"
         << "  - Start at time:        time.current    = " << current_ << " s\n"
         << "  - Total sim. time:      time.total      = " << total_ << " s\n"
         << "  - File output interval: time.file_dt    = " << file_dt_ << " s\n"
         << "  - Start at step count:  time.step_count = " << step_count_ << std::endl;
    if (cfg_.contactmodel == 1)
        cout << "  - Contact model: Linear-elastic-viscous (n), visco-frictional (t)\n";
    else if (cfg_.contactmodel == 2)
        cout << "  - Contact model: Linear-elastic-visco-frictional\n";
    else if (cfg_.contactmodel == 3)
        cout << "  - Contact model: Nonlinear-elastic-visco-frictional\n";
    else {
        std::cerr << "Error: Contact model value (" << cfg_.contactmodel << ") not understood.\n";
        exit(1);
    }
    cout << "  - Number of dynamic walls: " << cfg_.nw << '\n';
    if (cfg_.periodic == 1)
        cout << "  - 1st and 2nd dim. boundaries: Periodic\n";
    else if (cfg_.periodic == 2)
        cout << "  - 1st dim. boundaries: Visco-frictional walls\n";
    else
        cout << "  - 1st and 2nd dim. boundaries: Visco-frictional walls\n";
    if (cfg_.nw > 0) {
        cout << "  - Top BC: ";
        if (cfg_.wmode[0] == 0) cout << "Fixed\n";
        else if (cfg_.wmode[0] == 1) cout << "Deviatoric stress, " << walls_mvfd_[3] << " Pa\n";
        else if (cfg_.wmode[0] == 2) cout << "Velocity, " << walls_mvfd_[1] << " m/s\n";
        else {
            std::cerr << "Top BC not recognized!\n";
            exit(1);
        }
    }
    cout << "  - Grid: " << cfg_.num[0] << " * " << cfg_.num[1] << " * " << cfg_.num[2]
         << " cells\n"
         << "  - Domain size: " << cfg_.L[0] << " * " << cfg_.L[1] << " * " << cfg_.L[2]
         << " m\n"
         << "  - No. of particle bonds: " << cfg_.nb0 << std::endl;
}

static void write_status(const std::string &sid, double current, double total, uint32_t count)
{
    const std::string fn = "output/" + sid + ".status.dat";
    FILE *fp = fopen(fn.c_str(), "w");
    if (!fp) {
        std::cerr << "Could not write " << fn << std::endl;
        exit(1);
    }
    fprintf(fp, "%2.4e %2.4e %d\n", current, 100.0 * current / total, count);
    fclose(fp);
}

void DEM::startTime()
{
    if (!ctx_) initDevice();
    writebin(("output/" + sid_ + ".output00000.bin").c_str());
    write_status(sid_, current_, total_, step_count_);
    const auto tic = std::chrono::steady_clock::now();
    float filetimeclock = 0.0f;   // float in the reference (src/device.cu:594)
    uint64_t pending = 0, iter = 0;
    char file[512];
    if (verbose_ == 1) std::cout << "  Current simulation time: " << current_ << " s.";
    while (current_ <= total_) {
        ++pending;
        ++iter;
        current_ += dt_;
        filetimeclock += dt_;
        if (filetimeclock >= file_dt_) {
            int rc = sph_step(ctx_, pending, nullptr);
            if (rc == SPH_OK) rc = sph_sync(ctx_);
            if (rc != SPH_OK) fail(rc, "time loop");
            pending = 0;
            download();
            step_count_ += 1;
            snprintf(file, sizeof file, "output/%s.output%05d.bin", sid_.c_str(), step_count_);
            writebin(file);
            write_status(sid_, current_, total_, step_count_);
            filetimeclock = 0.0f;
            if (verbose_ == 1)
                std::cout << "\r  Current simulation time: " << current_ << "/" << total_
                          << " s.        " << std::flush;
        }
    }
    if (pending) {
        int rc = sph_step(ctx_, pending, nullptr);
        if (rc == SPH_OK) rc = sph_sync(ctx_);
        if (rc != SPH_OK) fail(rc, "time loop");
        download();
    }
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - tic).count();
    if (verbose_ == 1) {
        std::cout << "\nSimulation ended. Statistics:\n"
                  << "  - Last output file number: " << step_count_ << "\n"
                  << "  - Wall time spent: " << secs << " s\n"
                  << "  - Mean duration of iteration:\n"
                  << "      " << (iter ? secs / (double)iter : 0.0) << " s" << std::endl;
    }
    if (darcyOn()) endDarcy();   // src/device.cu:1292-1297
}

// DEM::render (src/raytracer.cuh:303-553) through sph_render, then
// writePPM (src/file_io.cpp:493-516).  focalLength is unused there too.
void DEM::render(const int method, const float maxval, const float lower_cutoff, const float,
                 const unsigned int img_width, const unsigned int img_height)
{
    if (!ctx_) initDevice();
    if (verbose_ == 1 && method != 0) {
        static const char *desc[] = {"", "Pressure", "Linear velocity", "Angular velocity",
                                     "X-axis displacement", "Angular positions"};
        static const char *unit[] = {"", "Pa", "m/s", "rad/s", "m", "rad"};
        if (method > 0 && method < 6)
            std::cout << "  " << desc[method] << " color map range: [0, " << maxval << "] "
                      << unit[method] << std::endl;
    }
    sph_render_opts o{};
    o.method = method;
    o.maxval = maxval;
    o.lower_cutoff = lower_cutoff;
    o.width = img_width;
    o.height = img_height;
    img_.assign((size_t)img_width * img_height * 4, 0);
    width_ = img_width;
    height_ = img_height;
    const int rc = sph_render(ctx_, &o, img_.data());
    if (rc != SPH_OK) fail(rc, "sph_render");
    writePPM(("img_out/" + sid_ + ".ppm").c_str());
}

// writePPM (src/file_io.cpp:493-516): header, then r, g, b of every pixel
void DEM::writePPM(const char *target)
{
    std::ofstream ofs(target, std::ios_base::binary);
    if (!ofs) {
        std::cerr << "Could not create output PPM file '" << target << std::endl;
        exit(1);
    }
    if (verbose_ == 1) std::cout << "  Saving image: " << target << std::endl;
    ofs << "P6 " << width_ << " " << height_ << " 255\n";
    for (size_t i = 0; i < (size_t)width_ * height_; ++i)
        ofs << img_[4 * i] << img_[4 * i + 1] << img_[4 * i + 2];
}

// minPos / maxPos (src/sphere.cpp:487-551): the reference reduces per
// thread and then across threads, every partial starting from 0, with
// std::min / std::max (a NaN coordinate is never taken, and 0 and -0
// compare equal, so the first value kept stays): the order of the
// comparisons does not change the result.
Float3 DEM::minPos()
{
    Float3 m{0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < cfg_.np; ++i) {
        m.x = std::min(m.x, x_[4 * (size_t)i]);
        m.y = std::min(m.y, x_[4 * (size_t)i + 1]);
        m.z = std::min(m.z, x_[4 * (size_t)i + 2]);
    }
    return m;
}

Float3 DEM::maxPos()
{
    Float3 m{0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < cfg_.np; ++i) {
        m.x = std::max(m.x, x_[4 * (size_t)i]);
        m.y = std::max(m.y, x_[4 * (size_t)i + 1]);
        m.z = std::max(m.z, x_[4 * (size_t)i + 2]);
    }
    return m;
}

// findOverlaps (src/sphere.cpp:556-602).  The reference tests all pairs
// i < j.  A pair overlaps only when it is closer than r_i + r_j <= 2 r_max,
// so the candidates here come from a grid of cells a little wider than
// 2 r_max (two such particles lie in the same or adjacent cells); each is
// tested with the reference's arithmetic (x_j - x_i, the squares summed x,
// y, z, sqrt, less r_i + r_j) and the pairs are put in the reference's
// (i, j) order.  A particle with a coordinate or radius that is not finite
// overlaps nothing there (delta_n is NaN) and is left out.
void DEM::findOverlaps(std::vector<std::vector<unsigned int>> &ij, std::vector<double> &delta_n_ij)
{
    const uint32_t n = cfg_.np;
    auto finite = [&](uint32_t i) {
        const double *p = &x_[4 * (size_t)i];
        return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]) &&
               std::isfinite(p[3]);
    };
    double rmax = 0.0, lo[3] = {0.0, 0.0, 0.0};
    bool any = false;
    for (uint32_t i = 0; i < n; ++i) {
        if (!finite(i)) continue;
        const double *p = &x_[4 * (size_t)i];
        rmax = std::max(rmax, p[3]);
        for (int d = 0; d < 3; ++d) lo[d] = any ? std::min(lo[d], p[d]) : p[d];
        any = true;
    }
    // r_i + r_j <= 0 leaves delta_n = |x_ij| - (r_i + r_j) >= 0
    if (!any || !(rmax > 0.0)) return;
    const double edge = 2.0 * rmax * (1.0 + 1e-6);
    std::vector<std::pair<uint64_t, uint32_t>> keyed;   // (cell key, particle)
    std::vector<int64_t> cell(3 * (size_t)n);
    auto key_of = [](int64_t cx, int64_t cy, int64_t cz) {
        return ((uint64_t)(cx & 0x1fffff) << 42) | ((uint64_t)(cy & 0x1fffff) << 21) |
               (uint64_t)(cz & 0x1fffff);
    };
    for (uint32_t i = 0; i < n; ++i) {
        if (!finite(i)) continue;
        const double *p = &x_[4 * (size_t)i];
        for (int d = 0; d < 3; ++d) cell[3 * (size_t)i + d] = (int64_t)std::floor((p[d] - lo[d]) / edge);
        keyed.emplace_back(key_of(cell[3 * (size_t)i], cell[3 * (size_t)i + 1], cell[3 * (size_t)i + 2]), i);
    }
    std::sort(keyed.begin(), keyed.end());
    std::vector<std::pair<std::pair<uint32_t, uint32_t>, double>> found;
    for (const auto &ki : keyed) {
        const uint32_t i = ki.second;
        const double *xi = &x_[4 * (size_t)i];
        for (int64_t dz = -1; dz <= 1; ++dz)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dx = -1; dx <= 1; ++dx) {
                    const uint64_t k = key_of(cell[3 * (size_t)i] + dx, cell[3 * (size_t)i + 1] + dy,
                                              cell[3 * (size_t)i + 2] + dz);
                    auto it = std::lower_bound(keyed.begin(), keyed.end(),
                                               std::make_pair(k, (uint32_t)0));
                    for (; it != keyed.end() && it->first == k; ++it) {
                        const uint32_t j = it->second;
                        if (j <= i) continue;
                        const double *xj = &x_[4 * (size_t)j];
                        // the 21-bit keys wrap; a far particle sharing a key is no neighbour
                        if (std::abs(cell[3 * (size_t)j] - cell[3 * (size_t)i]) > 1 ||
                            std::abs(cell[3 * (size_t)j + 1] - cell[3 * (size_t)i + 1]) > 1 ||
                            std::abs(cell[3 * (size_t)j + 2] - cell[3 * (size_t)i + 2]) > 1)
                            continue;
                        const double ax = xj[0] - xi[0], ay = xj[1] - xi[1], az = xj[2] - xi[2];
                        const double len = std::sqrt(ax * ax + ay * ay + az * az);
                        const double delta_n = len - (xi[3] + xj[3]);
                        if (delta_n < 0.0) found.push_back({{i, j}, delta_n});
                    }
                }
    }
    std::sort(found.begin(), found.end(),
              [](const auto &a, const auto &b) { return a.first < b.first; });
    for (const auto &f : found) {
        ij.push_back({f.first.first, f.first.second});
        delta_n_ij.push_back(f.second);
    }
}

void DEM::porosity(const int)
{
    std::cerr << "Error: the porosity tool is not part of this DEM step implementation."
              << std::endl;
    exit(1);
}

void DEM::forcechains(const std::string, const int, const double, const double)
{
    std::cerr << "Error: the force-chain tool is not part of this DEM step implementation."
              << std::endl;
    exit(1);
}
