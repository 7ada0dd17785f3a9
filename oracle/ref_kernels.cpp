/*
 * oracle/ref_kernels.cpp -- the reference's hot-path kernels as host C++,
 * driven in the order of the reference time loop (src/device.cu:731-1109).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/oracle.h): this file holds no physics
 * of its own.  It compiles the reference's src/sorting.cuh,
 * src/contactmodels.cuh, src/cohesion.cuh and src/contactsearch.cuh
 * unchanged from where they lie (the include path points at the reference's
 * src/), launches every kernel with one-thread blocks, replaces
 * thrust::sort_by_key (src/device.cu:763-765) with std::stable_sort of the
 * same (cellID, index) pairs, and runs bondsLinear serially in bond order.
 *
 * Build flags (oracle/Makefile) mirror the reference's arithmetic:
 * -ffp-contract=off for --fmad=false, and -ftrivial-auto-var-init=zero so the
 * uninitialised locals and host arrays the reference leaves unset read as 0.
 */
#include "ref_shim.h"

#include "vector_arithmetic.h"
#include "constants.cuh"
#include "sorting.cuh"
#include "contactmodels.cuh"
#include "cohesion.cuh"
#include "contactsearch.cuh"
#include "darcy.cuh"

#include "oracle.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
dim3 blockDim(1, 1, 1);
dim3 gridDim(1, 1, 1);

/* storage behind reorderArrays' `extern __shared__` (one-thread blocks) */
unsigned int shared_data[2];

/* oracle/ref_integration.cpp */
void ref_integrate_one(Float4 *, Float4 *, Float4 *, Float4 *, Float4 *, Float4 *, Float4 *,
                       Float4 *, Float4 *, Float4 *, Float4 *, Float4 *, Float4 *, Float2 *,
                       unsigned int *, unsigned int);
void ref_summation_blocks(Float *in, Float *out, unsigned int nblocks);
void ref_integrate_walls(Float4 *, Float4 *, int *, Float *, Float *, unsigned int, Float,
                         unsigned int);

/* Up to this particle count (default 0: never) summation() runs with 256
 * host threads per block; above it the wall-force block tree is evaluated in the
 * same order by harness code instead of 256 host threads per block (the
 * threaded form is exact but too slow for a timed baseline). */
static unsigned int g_threaded_summation_max = 0;

extern "C" void orc_set_threaded_summation_max(unsigned int n) { g_threaded_summation_max = n; }

static void summation_same_order(const Float *in, Float *out, unsigned int np,
                                 unsigned int nblocks)
{
    Float cache[256];
    for (unsigned int b = 0; b < nblocks; ++b) {
        for (unsigned int t = 0; t < 256; ++t) {
            unsigned int idx = t + b * 256;
            Float temp = 0.0f;
            while (idx < np) { temp += in[idx]; idx += 256 * nblocks; }
            cache[t] = temp;
        }
        for (unsigned int i = 128; i != 0; i /= 2)
            for (unsigned int t = 0; t < i; ++t) cache[t] += cache[t + i];
        out[b] = cache[0];
    }
}

/* src/darcy.cuh also holds DEM's Darcy memory-transfer methods, which the
 * harness never calls; these stand-ins resolve the CUDA runtime and utility
 * symbols they name, and stay private to this library. */
#define REF_HIDDEN __attribute__((visibility("hidden")))
extern "C" REF_HIDDEN cudaError_t cudaMalloc(void **, size_t) { return cudaErrorNotSupported; }
extern "C" REF_HIDDEN cudaError_t cudaFree(void *) { return cudaErrorNotSupported; }
extern "C" REF_HIDDEN cudaError_t cudaMemcpy(void *, const void *, size_t, cudaMemcpyKind)
{
    return cudaErrorNotSupported;
}
REF_HIDDEN void checkForCudaErrors(const char *) {}

extern "C" int orc_kind(void) { return 2; }

extern "C" int orc_threads(int nthreads)
{
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

static inline void launch1(unsigned int i)
{
    blockIdx.x = i;
    threadIdx.x = 0;
}

/* one-thread block (x, y, z) of a 3-D launch */
static inline void launch3(unsigned int x, unsigned int y, unsigned int z)
{
    blockIdx.x = x; blockIdx.y = y; blockIdx.z = z;
    threadIdx.x = 0; threadIdx.y = 0; threadIdx.z = 0;
}

extern "C" int orc_step(orc_scene *s, uint64_t nsteps, int nthreads)
{
    if (!s || s->np == 0 || s->nw > ORC_MAXWALLS) return ORC_ERR_BAD_INPUT;
    if (s->contactmodel < 1 || s->contactmodel > 3) return ORC_ERR_BAD_INPUT;
    const unsigned int np = s->np;
    const unsigned long long nc64 = (unsigned long long)s->num[0] * s->num[1] * s->num[2];
    if (nc64 == 0 || nc64 >= 0xffffffffull) return ORC_ERR_BAD_INPUT;
    const unsigned int ncells = (unsigned int)nc64;

    /* __constant__ memory, src/device.cu:214-220 */
    devC_nd = 3;
    devC_np = np;
    devC_nw = s->nw;
    devC_nc = ORC_NC;
    devC_dt = s->dt;
    devC_nb0 = s->nb0;
    for (int d = 0; d < 3; ++d) {
        devC_grid.origo[d] = s->origo[d];
        devC_grid.L[d] = s->L[d];
        devC_grid.num[d] = s->num[d];
        devC_params.g[d] = s->g[d];
    }
    devC_grid.periodic = s->periodic;
    Params &P = devC_params;
    P.k_n = s->k_n; P.k_t = s->k_t; P.k_r = s->k_r;
    P.gamma_n = s->gamma_n; P.gamma_t = s->gamma_t; P.gamma_r = s->gamma_r;
    P.mu_s = s->mu_s; P.mu_d = s->mu_d; P.mu_r = s->mu_r;
    P.gamma_wn = s->gamma_wn; P.gamma_wt = s->gamma_wt;
    P.mu_ws = s->mu_ws; P.mu_wd = s->mu_wd; P.rho = s->rho;
    P.contactmodel = s->contactmodel;
    P.kappa = s->kappa; P.db = s->db; P.V_b = s->V_b;
    P.lambda_bar = s->lambda_bar; P.nb0 = s->nb0;
    P.sigma_b = s->sigma_b; P.tau_b = s->tau_b;
    P.devs_A = s->devs_A; P.devs_f = s->devs_f; P.nu = s->nu;

    /* The host build cannot reproduce the device's saturating conversion of
     * floor(negative) (src/sorting.cuh:12-14), and a cell id past the grid
     * makes reorderArrays write out of bounds: refuse such states. */
    auto inside = [&](void) {
        for (unsigned int i = 0; i < np; ++i)
            for (int d = 0; d < 3; ++d) {
                double f = floor((s->x[4 * (size_t)i + d] - s->origo[d]) /
                                 (s->L[d] / s->num[d]));
                if (!(f >= 0.0) || f >= (double)s->num[d]) return false;
            }
        return true;
    };

    Float4 *x = (Float4 *)s->x, *vel = (Float4 *)s->vel, *vel0 = (Float4 *)s->vel0;
    Float4 *acc = (Float4 *)s->acc, *force = (Float4 *)s->force;
    Float4 *angpos = (Float4 *)s->angpos, *angvel = (Float4 *)s->angvel;
    Float4 *angvel0 = (Float4 *)s->angvel0, *angacc = (Float4 *)s->angacc;
    Float4 *torque = (Float4 *)s->torque;
    Float2 *xysum = (Float2 *)s->xysum;
    Float4 *distmod = (Float4 *)s->distmod, *delta_t = (Float4 *)s->delta_t;
    uint2 *bonds = (uint2 *)s->bonds;
    Float4 *bonds_delta = (Float4 *)s->bonds_delta, *bonds_omega = (Float4 *)s->bonds_omega;
    Float4 *walls_nx = (Float4 *)s->walls_nx, *walls_mvfd = (Float4 *)s->walls_mvfd;

    std::vector<unsigned int> cellid(np), index(np);
    std::vector<Float4> x_sorted(np), vel_sorted(np), angvel_sorted(np);
    std::vector<Float> walls_force_pp((size_t)std::max(1u, s->nw) * np, 0.0);
    const unsigned int nblocks = (np + 255) / 256;
    std::vector<Float> partial(nblocks, 0.0);
    std::vector<int> wmode(ORC_MAXWALLS);
    for (int w = 0; w < ORC_MAXWALLS; ++w) wmode[w] = s->wmode[w];
    std::vector<std::pair<unsigned int, unsigned int>> kv(np);
    const int nt = orc_threads(nthreads);

    for (uint64_t step = 0; step < nsteps; ++step) {
        if (!inside()) return ORC_ERR_OUT_OF_GRID;
        blockDim = dim3(1, 1, 1);
        gridDim = dim3(np, 1, 1);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (long i = 0; i < (long)np; ++i) {
            launch1((unsigned int)i);
            calcParticleCellID(cellid.data(), index.data(), x);
        }
        for (unsigned int i = 0; i < np; ++i)
            if (cellid[i] >= ncells) return ORC_ERR_OUT_OF_GRID;
        /* thrust::sort_by_key is a stable radix sort of (key, value) */
        for (unsigned int i = 0; i < np; ++i) kv[i] = {cellid[i], index[i]};
        std::stable_sort(kv.begin(), kv.end(),
                         [](const auto &a, const auto &b) { return a.first < b.first; });
        for (unsigned int i = 0; i < np; ++i) { cellid[i] = kv[i].first; index[i] = kv[i].second; }
        memset(s->cell_start, 0xff, sizeof(unsigned int) * (size_t)ncells);
        for (unsigned int i = 0; i < np; ++i) {
            launch1(i);
            reorderArrays(s->cell_start, s->cell_end, cellid.data(), index.data(), x, vel,
                          angvel, x_sorted.data(), vel_sorted.data(), angvel_sorted.data());
        }
        /* contact history only for models 2 and 3 (src/device.cu:805) */
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
        for (long i = 0; i < (long)(s->contactmodel == 1 ? 0u : np); ++i) {
            launch1((unsigned int)i);
            topology(s->cell_start, s->cell_end, index.data(), x_sorted.data(), s->contacts,
                     distmod);
        }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
        for (long i = 0; i < (long)np; ++i) {
            launch1((unsigned int)i);
            interact(index.data(), s->cell_start, s->cell_end, x, x_sorted.data(),
                     vel_sorted.data(), angvel_sorted.data(), vel, angvel, force, torque,
                     s->es_dot, s->ev_dot, s->es, s->ev, s->p, walls_nx, walls_mvfd,
                     walls_force_pp.data(), s->contacts, distmod, delta_t);
        }
        if (s->nb0 > 0) {
            gridDim = dim3(s->nb0, 1, 1);
            for (unsigned int b = 0; b < s->nb0; ++b) {
                launch1(b);
                bondsLinear(bonds, bonds_delta, bonds_omega, x, vel, angvel, force, torque);
            }
            gridDim = dim3(np, 1, 1);
        }
        if (s->darcy == 1 && s->nu > 0.0) {
            /* src/device.cu:913-1021: one-thread blocks over the fluid grid */
            const unsigned int fx = s->num[0], fy = s->num[1], fz = s->num[2];
            const long nfl = (long)fx * fy * fz;
            blockDim = dim3(1, 1, 1);
            gridDim = dim3(fx, fy, fz);
            Float *H = s->d_Hbuf[s->d_hsel], *Hn = s->d_Hbuf[1 - s->d_hsel];
            Float3 *V = (Float3 *)s->d_V, *dH = (Float3 *)s->d_dH, *T = (Float3 *)s->d_T;
            auto at = [&](long i) {
                launch3((unsigned int)(i % fx), (unsigned int)(i / fx % fy),
                        (unsigned int)(i / ((long)fx * fy)));
            };
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
            for (long i = 0; i < nfl; ++i) {
                at(i);
                findPorositiesSphericalDev(s->cell_start, s->cell_end, x_sorted.data(), s->d_phi,
                                           s->d_dphi, s->iteration);
            }
            for (long i = 0; i < nfl; ++i) {
                at(i);
                findDarcyTransmissivitiesDev(s->d_K, T, s->d_phi, s->d_factor);
            }
            for (long i = 0; i < nfl; ++i) {
                at(i);
                setDarcyGhostNodesDev(H, Hn, V, dH, s->d_K, T, s->d_Ss, s->d_W, s->d_phi,
                                      s->d_dphi);
            }
            for (long i = 0; i < nfl; ++i) {
                at(i);
                explDarcyStepDev(H, Hn, T, s->d_Ss, s->d_W, s->d_dphi);
            }
            s->d_hsel ^= 1u;   /* the pointer swap of src/device.cu:991-994 */
            std::swap(H, Hn);
            for (long i = 0; i < nfl; ++i) {
                at(i);
                findDarcyGradientsDev(H, dH);
            }
            for (long i = 0; i < nfl; ++i) {
                at(i);
                findDarcyVelocitiesDev(H, dH, V, s->d_phi, s->d_K);
            }
            gridDim = dim3(np, 1, 1);
        }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (long i = 0; i < (long)np; ++i)
            ref_integrate_one(x_sorted.data(), vel_sorted.data(), angvel_sorted.data(), x, vel,
                              angvel, force, torque, angpos, acc, angacc, vel0, angvel0, xysum,
                              index.data(), (unsigned int)i);
        if (s->nw > 0) {
            if (np <= g_threaded_summation_max)
                ref_summation_blocks(walls_force_pp.data(), partial.data(), nblocks);
            else
                summation_same_order(walls_force_pp.data(), partial.data(), np, nblocks);
            ref_integrate_walls(walls_nx, walls_mvfd, wmode.data(), partial.data(),
                                s->walls_vel0, nblocks, s->t_current, s->nw);
        }
        s->t_current += s->dt;
        s->iteration++;
    }
    for (unsigned int i = 0; i < np; ++i) { s->cell_sorted[i] = cellid[i]; s->perm[i] = index[i]; }
    if (s->wall0_force) memcpy(s->wall0_force, walls_force_pp.data(), sizeof(double) * np);
    return 0;
}
