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
// The order is made by a stable least-significant-digit radix sort of the
// particles' bucket ids (the cell id, or one bucket after the last cell for
// a position outside the grid or not finite), 8 bits a pass, the particle
// index as the value: every pass keeps equal digits in their order, so
// equal ids stay in particle-index order, and the work is linear in the
// number of particles whatever their spread over the cells.  The caller's
// two np-long outputs (sorted ids, permutation) are one of the sort's two
// buffer pairs, the scratch array the other.
//
// The host never passes the array's name to a kernel (in host code that
// name is a host-side stand-in, not a device address); it asks the runtime
// for the device address with cudaGetSymbolAddress once per device, with
// that device current, and passes that pointer.  All calls share the one
// scratch array, so calls that overlap on the GPU race; the array keeps the
// last call's contents, and every call overwrites what it reads before
// reading it.
#include "sphk_internal.cuh"
#include "../../include/sphk.h"

#include <mutex>

namespace sphk {

// fixed capacity of the scratch array
constexpr uint32_t NA_MAX_NP = SPHK_NOALLOC_MAX_PARTICLES;
constexpr uint32_t NA_MAX_CELLS = SPHK_NOALLOC_MAX_CELLS;
// radix sort: 8-bit digits, tiles of 2048 particles (256 threads x 8)
constexpr int NA_BLOCK = 256;
constexpr int NA_ITEMS = 8;
constexpr uint32_t NA_TILE = NA_BLOCK * NA_ITEMS;
constexpr uint32_t NA_BINS = 256;
constexpr uint32_t NA_MAX_TILES = (NA_MAX_NP + NA_TILE - 1) / NA_TILE;
// layout in 32-bit words: the second key/value buffer pair, then the
// digit counts of every tile (digit-major), scanned in place
constexpr size_t NA_OFF_KEYS = 0;
constexpr size_t NA_OFF_VALS = NA_OFF_KEYS + NA_MAX_NP;
constexpr size_t NA_OFF_HIST = NA_OFF_VALS + NA_MAX_NP;
constexpr size_t NA_WORDS = NA_OFF_HIST + (size_t)NA_BINS * NA_MAX_TILES;

static __device__ __align__(256) uint32_t g_na_scratch[NA_WORDS];

struct NaGrid {
    uint32_t np, ncells, num[3];
    double origo[3], cellsize[3];
};

// empty cells: start 0xffffffff, end 0 (src/device.cu:776-777)
__global__ void k_na_clear(uint32_t *cell_start, uint32_t *cell_end, uint32_t ncells)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        cell_start[c] = 0xffffffffu;
        cell_end[c] = 0u;
    }
}

// the bucket of every particle (the cell list's rule: grid_cell) and the
// identity permutation, the sort's first keys and values
__global__ void k_na_hash(NaGrid g, const double4 *x, uint32_t *keys, uint32_t *vals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.np) return;
    const double4 p = x[i];
    uint32_t c;
    keys[i] = grid_cell(g, p.x, p.y, p.z, c) ? c : g.ncells;
    vals[i] = i;
}

// digit counts of one tile: hist[digit * ntiles + tile]
__global__ void __launch_bounds__(NA_BLOCK) k_na_hist(const uint32_t *keys, uint32_t n,
                                                      uint32_t shift, uint32_t *hist,
                                                      uint32_t ntiles)
{
    __shared__ uint32_t cnt[NA_BINS];
    cnt[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t base = blockIdx.x * NA_TILE;
#pragma unroll
    for (int k = 0; k < NA_ITEMS; ++k) {
        const uint32_t i = base + k * NA_BLOCK + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// one block: exclusive scan of the n counts in place (digit-major, so a
// tile's digit d starts after every smaller digit and after d in the tiles
// before it)
__global__ void __launch_bounds__(1024) k_na_scan(uint32_t *hist, uint32_t n)
{
    __shared__ uint32_t warp_tot[32];
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(n, b + per);
    uint32_t sum = 0;
    for (uint32_t c = b; c < e; ++c) sum += hist[c];
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
        const uint32_t v = hist[c];
        hist[c] = run;
        run += v;
    }
}

// Stable scatter of one tile by the digit at `shift`.  Warp w takes the
// tile's w-th run of 256 particles, 32 at a time in order; a particle's
// place is the tile's start for its digit (from the scan), plus the
// particles with that digit in the earlier runs, plus those before it in
// its own run (the lanes of its step that share the digit, then its lower
// lanes among them).
__global__ void __launch_bounds__(NA_BLOCK) k_na_scatter(const uint32_t *kin, const uint32_t *vin,
                                                         uint32_t *kout, uint32_t *vout,
                                                         uint32_t n, uint32_t shift,
                                                         const uint32_t *hist, uint32_t ntiles)
{
    constexpr int WARPS = NA_BLOCK / 32;
    __shared__ uint32_t run_cnt[WARPS][NA_BINS];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    for (uint32_t k = threadIdx.x; k < WARPS * NA_BINS; k += NA_BLOCK) (&run_cnt[0][0])[k] = 0u;
    __syncthreads();
    const uint32_t run0 = blockIdx.x * NA_TILE + w * (NA_TILE / WARPS);
    // the digit counts of each warp's run
#pragma unroll
    for (int k = 0; k < NA_ITEMS; ++k) {
        const uint32_t i = run0 + k * 32u + lane;
        if (i < n) atomicAdd(&run_cnt[w][(kin[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    // each run's first place for every digit
    {
        const uint32_t dgt = threadIdx.x;
        uint32_t at = hist[dgt * ntiles + blockIdx.x];
        for (int r = 0; r < WARPS; ++r) {
            const uint32_t c = run_cnt[r][dgt];
            run_cnt[r][dgt] = at;
            at += c;
        }
    }
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < NA_ITEMS; ++k) {
        const uint32_t i = run0 + k * 32u + lane;
        const bool ok = i < n;
        const uint32_t key = ok ? kin[i] : 0u;
        const uint32_t dgt = ok ? ((key >> shift) & 0xffu) : NA_BINS;
        const uint32_t peers = __match_any_sync(0xffffffffu, dgt);
        const uint32_t at = ok ? run_cnt[w][dgt] : 0u;
        __syncwarp();
        if (ok) {
            const uint32_t dst = at + __popc(peers & lt);
            kout[dst] = key;
            vout[dst] = vin[i];
            if ((peers & lt) == 0u) run_cnt[w][dgt] = at + __popc(peers);
        }
        __syncwarp();
    }
}

// cell start/end from the sorted buckets; the out-of-grid bucket has none
__global__ void k_na_bounds(const uint32_t *keys, uint32_t np, uint32_t ncells,
                            uint32_t *cell_start, uint32_t *cell_end)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const uint32_t c = keys[k];
    if (c >= ncells) return;
    if (k == 0 || keys[k - 1] != c) cell_start[c] = k;
    if (k + 1 == np || keys[k + 1] != c) cell_end[c] = k + 1;
}

// the sorted ids and permutation into the outputs; the out-of-grid bucket
// is labelled 0xffffffff, as sph_get_cells reports it
__global__ void k_na_out(const uint32_t *keys, const uint32_t *vals, uint32_t np, uint32_t ncells,
                         uint32_t *cell_sorted, uint32_t *perm)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const uint32_t c = keys[k];
    const uint32_t v = vals[k];
    cell_sorted[k] = (c < ncells) ? c : 0xffffffffu;
    perm[k] = v;
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

static int na_run(const sph_config *cfg, const double *x_dev, uint32_t *cell_sorted,
                  uint32_t *perm, uint32_t *cell_start, uint32_t *cell_end, cudaStream_t st)
{
    uint32_t *scratch = nullptr;
    const int rc = na_scratch_for_current_device(&scratch);
    if (rc != SPH_OK) return rc;
    NaGrid g{};
    g.np = cfg->np;
    g.ncells = cfg->num[0] * cfg->num[1] * cfg->num[2];
    for (int k = 0; k < 3; ++k) {
        g.num[k] = cfg->num[k];
        g.origo[k] = cfg->origo[k];
        g.cellsize[k] = cfg->L[k] / (double)cfg->num[k];
    }
    const uint32_t np = g.np;
    const uint32_t ntiles = div_up(np, NA_TILE);
    // the buckets run to ncells (out of the grid): passes for its bits
    uint32_t passes = 0;
    for (uint32_t top = g.ncells; top; top >>= 8) ++passes;
    if (passes == 0) passes = 1;
    uint32_t *keys[2] = {cell_sorted, scratch + NA_OFF_KEYS};
    uint32_t *vals[2] = {perm, scratch + NA_OFF_VALS};
    uint32_t *hist = scratch + NA_OFF_HIST;
    const unsigned int pb = div_up(np, 256);
    k_na_clear<<<div_up(g.ncells, 256), 256, 0, st>>>(cell_start, cell_end, g.ncells);
    k_na_hash<<<pb, 256, 0, st>>>(g, reinterpret_cast<const double4 *>(x_dev), keys[0], vals[0]);
    int cur = 0;
    for (uint32_t p = 0; p < passes; ++p) {
        const uint32_t shift = 8u * p;
        k_na_hist<<<ntiles, NA_BLOCK, 0, st>>>(keys[cur], np, shift, hist, ntiles);
        k_na_scan<<<1, 1024, 0, st>>>(hist, NA_BINS * ntiles);
        k_na_scatter<<<ntiles, NA_BLOCK, 0, st>>>(keys[cur], vals[cur], keys[cur ^ 1],
                                                 vals[cur ^ 1], np, shift, hist, ntiles);
        cur ^= 1;
    }
    k_na_bounds<<<pb, 256, 0, st>>>(keys[cur], np, g.ncells, cell_start, cell_end);
    // in place when the last pass wrote the outputs (each thread reads its
    // own entries before writing them)
    k_na_out<<<pb, 256, 0, st>>>(keys[cur], vals[cur], np, g.ncells, cell_sorted, perm);
    // a launch error of these kernels, without clearing one left by the
    // caller's own work (which is then reported too)
    return cudaPeekAtLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
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
    // the caller's current device is put back before returning
    int caller_dev = 0;
    if (cudaGetDevice(&caller_dev) != cudaSuccess) return SPH_ERR_CUDA;
    if (cfg->device != caller_dev && cudaSetDevice(cfg->device) != cudaSuccess) return SPH_ERR_CUDA;
    const int rc = na_run(cfg, x_dev, cell_sorted, perm, cell_start, cell_end,
                          static_cast<cudaStream_t>(stream));
    if (cfg->device != caller_dev && cudaSetDevice(caller_dev) != cudaSuccess) return SPH_ERR_CUDA;
    return rc;
}
