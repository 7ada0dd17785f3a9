// darcy.cu -- Darcy flow through the packing (src/darcy.cuh:169-779, launched
// at src/device.cu:913-1021) and its host-side initialisation
// (src/darcy.cpp:69-798).
//
// The reference runs six kernels per step, each over the fluid grid (the
// cell grid): porosity, transmissivity, ghost nodes, explicit pressure step,
// pressure gradient, velocity.  Here they are four:
//   k_darcy_porosity  porosity of every node from the cell list of the
//                     step's start positions, and from it the node's
//                     conductivity and transmissivity (a per-node function,
//                     so fusing changes no value);
//   k_darcy_ghosts    the boundary nodes copied onto the opposite ghost
//                     nodes, one thread per face node instead of a thread
//                     per node of the whole grid;
//   k_darcy_explicit  the explicit step of the pressure;
//   k_darcy_grad_vel  pressure gradient and pore velocity (per node again).
// Every expression keeps the reference's operands and order (FP64, no
// contraction), so the results are the reference's bit for bit.  The
// kernels read the step's start positions and the cell list, which the
// contact-force kernel leaves untouched, and write only the fluid grid.
#include "sphk_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

#include "sphk.h"

namespace sphk {

constexpr int DARCY_BLOCK = 128;
constexpr double D_PI = 3.14159265358979323846;   // M_PI, which src/darcy.cuh uses

// node (x, y, z) with ghost nodes at -1 and num (src/darcy.cuh:125-135)
__host__ __device__ __forceinline__ size_t dnode(uint32_t nx, uint32_t ny, int x, int y, int z)
{
    const size_t nx2 = (size_t)nx + 2, ny2 = (size_t)ny + 2;
    return (size_t)(x + 1) + nx2 * (size_t)(y + 1) + nx2 * ny2 * (size_t)(z + 1);
}

// findDistMod (src/contactsearch.cuh:12-74): false for a neighbour cell
// beyond a non-periodic boundary; otherwise wraps periodic axes and adds
// the +-L shift to dm
__device__ __forceinline__ bool neighbour_cell(const Params &P, int &cx, int &cy, int cz, d3 &dm)
{
    const int nx = (int)P.num[0], ny = (int)P.num[1], nz = (int)P.num[2];
    if (P.periodic == 1 || P.periodic == 2) {
        if (cx < 0) { cx = nx - 1; dm = add(dm, mk(P.L[0], 0.0, 0.0)); }
        if (cx == nx) { cx = 0; dm = sub(dm, mk(P.L[0], 0.0, 0.0)); }
    } else if (cx < 0 || cx == nx) {
        return false;
    }
    if (P.periodic == 1) {
        if (cy < 0) { cy = ny - 1; dm = add(dm, mk(0.0, P.L[1], 0.0)); }
        if (cy == ny) { cy = 0; dm = sub(dm, mk(0.0, P.L[1], 0.0)); }
    } else if (cy < 0 || cy == ny) {
        return false;
    }
    return !(cz < 0 || cz == nz);
}

// findPorositiesSphericalDev (src/darcy.cuh:338-477) and
// findDarcyTransmissivitiesDev (src/darcy.cuh:480-538) for one node.  The
// void fraction of a sphere of radius min(dx,dy,dz)/2 at the cell centre
// (measured from the origin, as the reference does, not from origo), less
// the lens-shaped parts of the particles of the 27 neighbour cells, which
// are visited z, y, x outermost to innermost and in cell-list order within a
// cell; clamped to [0.1, 0.9].  Its change is zero in the first step.
//
// Most particles of the 27 cells miss the cell sphere.  They are ruled out
// from the float position copy in cell-list order (xs, the one contact
// detection culls with): one 16-byte load at the list position and a few
// float operations.  The cull is conservative: it skips a particle only
// when its float distance exceeds (R + r)(1 + 1e-5) plus a bound on the
// float rounding of the positions (1e-6 of the coordinates' magnitudes), so
// every particle the reference's test (dd < R + r) would take goes through
// the exact FP64 path, in order.
__global__ void __launch_bounds__(DARCY_BLOCK)
k_darcy_porosity(Dev d, DarcyDev f, int A)
{
    const Params &P = *d.prm;
    const uint32_t nx = P.num[0], ny = P.num[1], nz = P.num[2];
    const uint32_t i = blockIdx.x * DARCY_BLOCK + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const uint32_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    const double dx = P.L[0] / nx, dy = P.L[1] / ny, dz = P.L[2] / nz;
    const double R = fmin(dx, fmin(dy, dz)) * 0.5;
    const double cell_volume = 4.0 / 3.0 * D_PI * R * R * R;
    double void_volume = cell_volume;
    const d3 X = mk(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
    const size_t me = dnode(nx, ny, (int)x, (int)y, (int)z);
    const double phi_0 = f.phi[me];
    const double4 *__restrict__ xr = d.xr[A];
    const float4 *__restrict__ xs = d.xs[A];
    const float Xx = (float)X.x, Xy = (float)X.y, Xz = (float)X.z;
    const float Rf = (float)R;
    const float err = 1e-6f * (2.0f * (fabsf(Xx) + fabsf(Xy) + fabsf(Xz)) + (float)P.L[0] +
                               (float)P.L[1] + (float)P.L[2] + Rf);
    for (int oz = -1; oz < 2; ++oz)
        for (int oy = -1; oy < 2; ++oy)
            for (int ox = -1; ox < 2; ++ox) {
                int cx = (int)x + ox, cy = (int)y + oy;
                const int cz = (int)z + oz;
                d3 dm = mk(0.0, 0.0, 0.0);
                if (!neighbour_cell(P, cx, cy, cz, dm)) continue;
                const uint32_t c = (uint32_t)cx + (uint32_t)cy * nx + (nx * ny) * (uint32_t)cz;
                const uint32_t beg = d.cell_start[c], end = d.cell_start[c + 1];
                const float sx = (float)dm.x, sy = (float)dm.y, sz = (float)dm.z;
                for (uint32_t k = beg; k < end; ++k) {
                    const float4 q = __ldg(&xs[k]);
                    const float fx = (Xx - q.x) + sx, fy = (Xy - q.y) + sy, fz = (Xz - q.z) + sz;
                    const float thr = (Rf + q.w) * 1.00001f + err;
                    if (fx * fx + fy * fy + fz * fz > thr * thr * 1.00001f) continue;
                    const double4 p = xr[d.cellorder[k]];
                    const double r = p.w;
                    const d3 dist = add(mk(X.x - p.x, X.y - p.y, X.z - p.z), dm);
                    const double dd = flen(dist);
                    if ((R - r) < dd && dd < (R + r))
                        void_volume -= 1.0 / (12.0 * dd) *
                                       (D_PI * (R + r - dd) * (R + r - dd) *
                                        (dd * dd + 2.0 * dd * r - 3.0 * r * r + 2.0 * dd * R +
                                         6.0 * r * R - 3.0 * R * R));
                    if (dd <= R - r) void_volume -= 4.0 / 3.0 * D_PI * r * r * r;
                }
            }
    const double phi = fmin(0.9, fmax(0.1, void_volume / cell_volume));
    f.phi[me] = phi;
    f.dphi[me] = (*f.first) ? 0.0 : phi - phi_0;
    // Kozeny-Carman conductivity and the transmissivity K * (dx, dy, dz)
    const double rho = 1000.0;
    const double kk = phi * phi * phi / ((1.0 - phi) * (1.0 - phi)) * f.d_factor;
    const double K = kk * rho * -P.g[2] / f.nu;
    f.K[me] = K;
    f.T[3 * me + 0] = K * dx;
    f.T[3 * me + 1] = K * dy;
    f.T[3 * me + 2] = K * dz;
}

// copyDarcyValsDev (src/darcy.cuh:137-166): every field of node `from` onto
// node `to`
__device__ __forceinline__ void copy_node(const DarcyDev &f, size_t from, size_t to)
{
    f.H[0][to] = f.H[0][from];
    f.H[1][to] = f.H[1][from];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        f.V[3 * to + c] = f.V[3 * from + c];
        f.dH[3 * to + c] = f.dH[3 * from + c];
        f.T[3 * to + c] = f.T[3 * from + c];
    }
    f.K[to] = f.K[from];
    f.Ss[to] = f.Ss[from];
    f.W[to] = f.W[from];
    f.phi[to] = f.phi[from];
    f.dphi[to] = f.dphi[from];
}

// setDarcyGhostNodesDev (src/darcy.cuh:169-261): a node on a face of the
// grid is copied onto the ghost node beyond the opposite face.  Edge and
// corner ghosts are never written (nor read).  Threads [0, ny nz) take the
// x faces, then [.., + nx nz) the y faces, then [.., + nx ny) the z faces;
// every ghost node is written by one thread, and no thread reads a ghost.
__global__ void __launch_bounds__(DARCY_BLOCK)
k_darcy_ghosts(const Params *prm, DarcyDev f)
{
    const Params &P = *prm;
    const int nx = (int)P.num[0], ny = (int)P.num[1], nz = (int)P.num[2];
    uint32_t t = blockIdx.x * DARCY_BLOCK + threadIdx.x;
    const uint32_t nyz = (uint32_t)(ny * nz), nxz = (uint32_t)(nx * nz), nxy = (uint32_t)(nx * ny);
    const uint32_t ux = (uint32_t)nx, uy = (uint32_t)ny;
    if (t < nyz) {
        const int y = (int)(t % uy), z = (int)(t / uy);
        copy_node(f, dnode(ux, uy, 0, y, z), dnode(ux, uy, nx, y, z));
        copy_node(f, dnode(ux, uy, nx - 1, y, z), dnode(ux, uy, -1, y, z));
        return;
    }
    t -= nyz;
    if (t < nxz) {
        const int x = (int)(t % ux), z = (int)(t / ux);
        copy_node(f, dnode(ux, uy, x, 0, z), dnode(ux, uy, x, ny, z));
        copy_node(f, dnode(ux, uy, x, ny - 1, z), dnode(ux, uy, x, -1, z));
        return;
    }
    t -= nxz;
    if (t < nxy) {
        const int x = (int)(t % ux), y = (int)(t / ux);
        copy_node(f, dnode(ux, uy, x, y, 0), dnode(ux, uy, x, y, nz));
        copy_node(f, dnode(ux, uy, x, y, nz - 1), dnode(ux, uy, x, y, -1));
    }
}

__device__ __forceinline__ double hmean(double a, double b) { return (2.0 * a * b) / (a + b); }

// explDarcyStepDev (src/darcy.cuh:604-725): explicit finite-difference
// step of the pressure from H into Hn, with harmonic-mean transmissivities
// between nodes and no flux through the z faces
__global__ void __launch_bounds__(DARCY_BLOCK)
k_darcy_explicit(const Params *prm, DarcyDev f, const double *__restrict__ H, double *Hn)
{
    const Params &P = *prm;
    const uint32_t nx = P.num[0], ny = P.num[1], nz = P.num[2];
    const uint32_t i = blockIdx.x * DARCY_BLOCK + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / (nx * ny));
    const double dx = P.L[0] / nx, dy = P.L[1] / ny, dz = P.L[2] / nz;
    const double *__restrict__ T = f.T;
    const size_t me = dnode(nx, ny, x, y, z);
    const size_t xn = dnode(nx, ny, x - 1, y, z), xp = dnode(nx, ny, x + 1, y, z);
    const size_t yn = dnode(nx, ny, x, y - 1, z), yp = dnode(nx, ny, x, y + 1, z);
    const size_t zn = dnode(nx, ny, x, y, z - 1), zp = dnode(nx, ny, x, y, z + 1);
    const double Ss = f.Ss[me], Q = f.W[me], dphi = f.dphi[me], Hc = H[me];
    const double TdH_xn = hmean(T[3 * me + 0], T[3 * xn + 0]) * (H[xn] - Hc) / (dx * dx);
    const double TdH_xp = hmean(T[3 * me + 0], T[3 * xp + 0]) * (H[xp] - Hc) / (dx * dx);
    const double TdH_yn = hmean(T[3 * me + 1], T[3 * yn + 1]) * (H[yn] - Hc) / (dy * dy);
    const double TdH_yp = hmean(T[3 * me + 1], T[3 * yp + 1]) * (H[yp] - Hc) / (dy * dy);
    double TdH_zn = hmean(T[3 * me + 2], T[3 * zn + 2]) * (H[zn] - Hc) / (dz * dz);
    double TdH_zp = hmean(T[3 * me + 2], T[3 * zp + 2]) * (H[zp] - Hc) / (dz * dz);
    const double dx_bar = (dx + dy + dz) / 3.0;
    if (z == 0) TdH_zn = 0.0;
    if ((uint32_t)z == nz - 1) TdH_zp = 0.0;
    const double laplacianH = TdH_xn + TdH_xp + TdH_yn + TdH_yp + TdH_zn + TdH_zp;
    const double porevol = -dx_bar * dphi / P.dt;
    const double deltaH = P.dt / (Ss * dx * dy * dz) * (laplacianH + Q + porevol);
    Hn[me] = fmax(0.0, Hc + deltaH);
}

// findDarcyGradientsDev + findDarcyVelocitiesDev (src/darcy.cuh:541-598,
// 728-776): central-difference gradient of the new pressure H (its ghost
// nodes still hold what the ghost copy put there before the step), flux
// -K/nu dH and pore velocity flux / phi
__global__ void __launch_bounds__(DARCY_BLOCK)
k_darcy_grad_vel(const Params *prm, DarcyDev f, const double *__restrict__ H)
{
    const Params &P = *prm;
    const uint32_t nx = P.num[0], ny = P.num[1], nz = P.num[2];
    const uint32_t i = blockIdx.x * DARCY_BLOCK + threadIdx.x;
    if (i >= nx * ny * nz) return;
    if (i == 0) *f.first = 0u;   // the porosity of this step has read it
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / (nx * ny));
    const double dx = P.L[0] / nx, dy = P.L[1] / ny, dz = P.L[2] / nz;
    const size_t me = dnode(nx, ny, x, y, z);
    const double gx = (H[dnode(nx, ny, x + 1, y, z)] - H[dnode(nx, ny, x - 1, y, z)]) / (2.0 * dx);
    const double gy = (H[dnode(nx, ny, x, y + 1, z)] - H[dnode(nx, ny, x, y - 1, z)]) / (2.0 * dy);
    const double gz = (H[dnode(nx, ny, x, y, z + 1)] - H[dnode(nx, ny, x, y, z - 1)]) / (2.0 * dz);
    f.dH[3 * me + 0] = gx;
    f.dH[3 * me + 1] = gy;
    f.dH[3 * me + 2] = gz;
    const double nu = f.nu, K = f.K[me], phi = f.phi[me];
    const double qx = -K / nu * gx, qy = -K / nu * gy, qz = -K / nu * gz;
    f.V[3 * me + 0] = qx / phi;
    f.V[3 * me + 1] = qy / phi;
    f.V[3 * me + 2] = qz / phi;
}

// The Darcy block of one step: `a` is the particle buffer of the step's
// start positions, `hs` the pressure buffer they go with.
void launch_darcy(const Dev &d, const DarcyDev &f, const Params &hp, int a, int hs, cudaStream_t st)
{
    const uint64_t n = (uint64_t)hp.num[0] * hp.num[1] * hp.num[2];
    const uint64_t faces = (uint64_t)hp.num[1] * hp.num[2] + (uint64_t)hp.num[0] * hp.num[2] +
                           (uint64_t)hp.num[0] * hp.num[1];
    k_darcy_porosity<<<div_up(n, DARCY_BLOCK), DARCY_BLOCK, 0, st>>>(d, f, a);
    k_darcy_ghosts<<<div_up(faces, DARCY_BLOCK), DARCY_BLOCK, 0, st>>>(d.prm, f);
    k_darcy_explicit<<<div_up(n, DARCY_BLOCK), DARCY_BLOCK, 0, st>>>(d.prm, f, f.H[hs], f.H[hs ^ 1]);
    k_darcy_grad_vel<<<div_up(n, DARCY_BLOCK), DARCY_BLOCK, 0, st>>>(d.prm, f, f.H[hs ^ 1]);
}

}  // namespace sphk

// ---- host-side initialisation: DEM::initDarcy (src/darcy.cpp:760-798) ------

namespace {

inline size_t hnode(const sph_config &c, int x, int y, int z)
{
    return sphk::dnode(c.num[0], c.num[1], x, y, z);
}

}  // namespace

extern "C" int sph_darcy_init(const sph_config *cfg, double nu, const double *x,
                              sph_darcy_state *st, double *stability)
{
    if (!cfg || !x || !st || !st->H || !st->phi || !st->dphi || !st->K || !st->T || !st->Ss ||
        !st->W)
        return SPH_ERR_BAD_INPUT;
    // src/darcy.cpp:762-766
    if (!(nu > 0.0)) return SPH_ERR_BAD_INPUT;
    const sph_config &c = *cfg;
    const int nx = (int)c.num[0], ny = (int)c.num[1], nz = (int)c.num[2];
    if (nx <= 0 || ny <= 0 || nz <= 0) return SPH_ERR_BAD_INPUT;
    const double dx = c.L[0] / nx, dy = c.L[1] / ny, dz = c.L[2] / nz;

    // initDarcyVals (src/darcy.cpp:69-104): every node, ghosts included
    for (int ix = -1; ix <= nx; ++ix)
        for (int iy = -1; iy <= ny; ++iy)
            for (int iz = -1; iz <= nz; ++iz) {
                const size_t k = hnode(c, ix, iy, iz);
                st->Ss[k] = 1.0;
                st->W[k] = 0.0;
            }

    // findPorosities / cellPorosity (src/darcy.cpp:600-644): the particles
    // whose centres lie in [x*dx, (x+1)*dx) x ... of a cell, subtracted from
    // its volume one by one in particle order.  The reference loops over all
    // particles per cell; each particle lies in at most one such box (the
    // boxes' bounds are the same products on both sides), so one pass over
    // the particles in order gives every cell the same subtractions.
    const double cell_volume = dx * dy * dz;
    std::vector<double> void_volume((size_t)nx * ny * nz, cell_volume);
    auto box_of = [](double p, double h, int n) {
        // the index b with b*h <= p < (b+1)*h, or -1 when there is none
        if (!(p >= 0.0)) return -1;
        double fb = std::floor(p / h);
        if (fb > (double)n) fb = (double)n;
        int b = (int)fb;
        while (b > 0 && b * h > p) --b;
        while (b < n && (b + 1) * h <= p) ++b;
        return (b < n && b * h <= p && p < (b + 1) * h) ? b : -1;
    };
    for (uint32_t i = 0; i < c.np; ++i) {
        const double *xr = x + 4 * (size_t)i;
        const int bx = box_of(xr[0], dx, nx), by = box_of(xr[1], dy, ny), bz = box_of(xr[2], dz, nz);
        if (bx < 0 || by < 0 || bz < 0) continue;
        double &v = void_volume[(size_t)bx + (size_t)nx * by + (size_t)nx * ny * bz];
        v -= 4.0 / 3.0 * sphk::D_PI * xr[3] * xr[3] * xr[3];
    }
    // meanRadius (src/darcy.cpp:646-653), the sum started from zero, and the
    // host's grain-size factor (src/darcy.cpp:184-187)
    double r_sum = 0.0;
    for (uint32_t i = 0; i < c.np; ++i) r_sum += x[4 * (size_t)i + 3];
    const double r_bar2 = r_sum / (double)c.np * 2.0 * 1.0e-6;
    const double d_factor = r_bar2 * r_bar2 / 180.0;
    // findDarcyTransmissivities (src/darcy.cpp:177-221), dphi := 0
    // (src/darcy.cpp:788-795)
    const double rho = 1000.0;
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int iz = 0; iz < nz; ++iz) {
                const size_t k = hnode(c, ix, iy, iz);
                const double phi = std::fmin(
                    0.99, std::fmax(0.01, void_volume[(size_t)ix + (size_t)nx * iy +
                                                      (size_t)nx * ny * iz] /
                                              cell_volume));
                st->phi[k] = phi;
                const double kk = phi * phi * phi / ((1.0 - phi) * (1.0 - phi)) * d_factor;
                const double K = kk * rho * -c.g[2] / nu;
                st->K[k] = K;
                st->T[3 * k + 0] = K * dx;
                st->T[3 * k + 1] = K * dy;
                st->T[3 * k + 2] = K * dz;
                st->dphi[k] = 0.0;
            }
    // checkDarcyTimestep (src/darcy.cpp:692-758)
    double T_max = -1.0e13, Ss_min = 1.0e13;
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int iz = 0; iz < nz; ++iz) {
                const size_t k = hnode(c, ix, iy, iz);
                for (int q = 0; q < 3; ++q)
                    if (st->T[3 * k + q] > T_max) T_max = st->T[3 * k + q];
                if (st->Ss[k] < Ss_min) Ss_min = st->Ss[k];
            }
    const double S_min = Ss_min * dx * dy * dz;
    const double value =
        T_max / S_min * (c.dt / (dx * dx) + c.dt / (dy * dy) + c.dt / (dz * dz));
    if (stability) *stability = value;
    return value > 0.5 ? SPH_ERR_UNSTABLE : SPH_OK;
}
