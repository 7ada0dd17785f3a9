// noalloc.cu -- the cell list of device-resident positions without any
// device allocation (sph_cell_list_noalloc in include/sphk.h).
//
// Some callers cannot allocate device memory: a plugin whose host owns the
// whole device memory pool through its own allocator and forbids cudaMalloc,
// or a latency-critical loop that must not pay the implicit device-wide
// synchronisation of cudaMalloc/cudaFree.  This entry point computes the same
// cell list as the rest of libsphk (cell id of every particle, the stable
// (cell, particle index) order, cell start/end) using only the caller's
// input and output arrays and one fixed scratch array that lives in the
// library image: a file-scope __device__ array, which every GPU that loads
// the library holds until the process exits.
//
// The host never passes the array's name to a kernel (in host code that
// name is a host-side stand-in, not a device address); it asks the runtime
// for the device address with cudaGetSymbolAddress once per device, with
// that device current, and passes that pointer.  All calls share the one
// scratch array, so calls that overlap on the GPU race; the array keeps the
// last call's contents, so the counters that must start at zero are cleared
// at the start of every call.
#include "sphk_internal.cuh"
#include "../../include/sphk.h"

#include <mutex>

namespace sphk {

// fixed capacity of the scratch array
constexpr uint32_t NA_MAX_NP = SPHK_NOALLOC_MAX_PARTICLES;
constexpr uint32_t NA_MAX_CELLS = SPHK_NOALLOC_MAX_CELLS;
// layout in 32-bit words: cell id per particle, per-cell counters (one extra
// bucket for positions outside the grid), per-cell start (+2)
constexpr size_t NA_OFF_CELLID = 0;
constexpr size_t NA_OFF_COUNT = NA_OFF_CELLID + NA_MAX_NP;
constexpr size_t NA_OFF_START = NA_OFF_COUNT + NA_MAX_CELLS + 1;
constexpr size_t NA_WORDS = NA_OFF_START + NA_MAX_CELLS + 2;

static __device__ __align__(256) uint32_t g_na_scratch[NA_WORDS];

struct NaGrid {
    uint32_t np, ncells, num[3];
    double origo[3], cellsize[3];
};

__device__ __forceinline__ uint32_t na_cell(const NaGrid &g, double x, double y, double z)
{
    const uint32_t ix = __double2uint_rz(floor((x - g.origo[0]) / g.cellsize[0]));
    const uint32_t iy = __double2uint_rz(floor((y - g.origo[1]) / g.cellsize[1]));
    const uint32_t iz = __double2uint_rz(floor((z - g.origo[2]) / g.cellsize[2]));
    return (iz * g.num[1]) * g.num[0] + iy * g.num[0] + ix;
}

__global__ void k_na_zero(uint32_t *scratch, uint32_t ncells)
{
    uint32_t *count = scratch + NA_OFF_COUNT;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += gridDim.x * blockDim.x)
        count[c] = 0u;
}

__global__ void k_na_hash(uint32_t *scratch, NaGrid g, const double4 *x)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.np) return;
    const double4 p = x[i];
    uint32_t c = na_cell(g, p.x, p.y, p.z);
    if (c >= g.ncells) c = g.ncells;   // outside the grid: the last bucket
    scratch[NA_OFF_CELLID + i] = c;
    atomicAdd(&scratch[NA_OFF_COUNT + c], 1u);
}

// one block: exclusive scan of the ncells + 1 counters into start[]
__global__ void __launch_bounds__(1024) k_na_scan(uint32_t *scratch, uint32_t ncells, uint32_t np)
{
    __shared__ uint32_t warp_tot[32];
    const uint32_t *count = scratch + NA_OFF_COUNT;
    uint32_t *start = scratch + NA_OFF_START;
    const uint32_t n = ncells + 1;
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(n, b + per);
    uint32_t sum = 0;
    for (uint32_t c = b; c < e; ++c) sum += count[c];
    const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (unsigned)o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t woff = 0;
    for (unsigned int w = 0; w < warp; ++w) woff += warp_tot[w];
    uint32_t run = woff + inc - sum;
    for (uint32_t c = b; c < e; ++c) {
        start[c] = run;
        run += count[c];
    }
    if (threadIdx.x == 0) start[n] = np;
}

__global__ void k_na_scatter(uint32_t *scratch, uint32_t np, uint32_t *perm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const uint32_t c = scratch[NA_OFF_CELLID + i];
    const uint32_t k = atomicSub(&scratch[NA_OFF_COUNT + c], 1u) - 1u;
    perm[scratch[NA_OFF_START + c] + k] = i;
}

// per cell: members by particle index (stable order), then the outputs
__global__ void k_na_cells(const uint32_t *scratch, uint32_t ncells, uint32_t *perm,
                           uint32_t *cell_sorted, uint32_t *cell_start, uint32_t *cell_end)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > ncells) return;
    const uint32_t beg = scratch[NA_OFF_START + c], end = scratch[NA_OFF_START + c + 1];
    for (uint32_t i = beg + 1; i < end; ++i) {
        const uint32_t v = perm[i];
        uint32_t j = i;
        while (j > beg && perm[j - 1] > v) {
            perm[j] = perm[j - 1];
            --j;
        }
        perm[j] = v;
    }
    const uint32_t label = (c < ncells) ? c : 0xffffffffu;
    for (uint32_t k = beg; k < end; ++k) cell_sorted[k] = label;
    if (c < ncells) {
        cell_start[c] = (beg == end) ? 0xffffffffu : beg;
        cell_end[c] = (beg == end) ? 0u : end;
    }
}

// device address of the scratch array, looked up once per device
static std::mutex g_na_mutex;
static uint32_t *g_na_ptr[64] = {};

static int na_scratch_for_current_device(uint32_t **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SPH_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p) return SPH_ERR_CUDA;
        g_na_ptr[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_na_ptr[dev];
    return SPH_OK;
}

}  // namespace sphk

using namespace sphk;

extern "C" int sph_cell_list_noalloc(const sph_config *cfg, const double *x_dev,
                                     uint32_t *cell_sorted, uint32_t *perm, uint32_t *cell_start,
                                     uint32_t *cell_end, void *stream)
{
    if (!cfg || !x_dev || !cell_sorted || !perm || !cell_start || !cell_end) return SPH_ERR_BAD_INPUT;
    const uint64_t ncells = (uint64_t)cfg->num[0] * cfg->num[1] * cfg->num[2];
    if (cfg->np == 0 || ncells == 0) return SPH_ERR_BAD_INPUT;
    if (cfg->np > NA_MAX_NP || ncells > NA_MAX_CELLS) return SPH_ERR_TOO_LARGE;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return SPH_ERR_CUDA;
    uint32_t *scratch = nullptr;
    int rc = na_scratch_for_current_device(&scratch);
    if (rc != SPH_OK) return rc;
    NaGrid g{};
    g.np = cfg->np;
    g.ncells = (uint32_t)ncells;
    for (int k = 0; k < 3; ++k) {
        g.num[k] = cfg->num[k];
        g.origo[k] = cfg->origo[k];
        g.cellsize[k] = cfg->L[k] / (double)cfg->num[k];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const unsigned int pb = div_up(g.np, 256), cb = div_up((unsigned long long)g.ncells + 1, 256);
    k_na_zero<<<cb, 256, 0, st>>>(scratch, g.ncells);
    k_na_hash<<<pb, 256, 0, st>>>(scratch, g, reinterpret_cast<const double4 *>(x_dev));
    k_na_scan<<<1, 1024, 0, st>>>(scratch, g.ncells, g.np);
    k_na_scatter<<<pb, 256, 0, st>>>(scratch, g.np, perm);
    k_na_cells<<<cb, 256, 0, st>>>(scratch, g.ncells, perm, cell_sorted, cell_start, cell_end);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}
