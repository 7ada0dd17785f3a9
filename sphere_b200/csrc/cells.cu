// cells.cu -- the cell list of libsphk: hash, sort, cell start/end, relayout.
//
// The reference hashes every particle to a cell (calcParticleCellID,
// src/sorting.cuh:24-43), sorts (cellID, index) pairs with thrust's stable
// radix sort (src/device.cu:763-765) and marks cell ranges
// (reorderArrays, src/sorting.cuh:49-121).  The sorted order is "by cell, then
// by particle index".  Here the same order comes from a one-pass counting
// sort with the cell id as the radix:
//   k_count    histogram of cell ids                  (atomics in L2)
//   k_scan_*   exclusive scan of the histogram        (two launches, no waits)
//   k_scatter  each particle claims a position in its cell's range
//   k_cellsort each cell orders its few members by particle index
//   k_post_sort inverse order and the float position copy in list order
// The cell of every particle is computed by the step kernel from its new
// position, which also raises `rebuild` when any particle changed cell; all
// the kernels above return at once when it is clear, so an unchanged cell
// list costs only their empty launches.
//
// Particles are stored in cell order (relayout), so neighbours are close in
// memory; k_relayout_* re-establish that order on demand.
#include "sphk_internal.cuh"

namespace sphk {

constexpr int CELL_BLOCK = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = CELL_BLOCK * SCAN_ITEMS;   // 2048 counters per block

__global__ void k_cell_init(Dev d, int A)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.np_all) return;
    const Params &P = prm_of(d, s);
    const double4 x = d.xr[A][s];
    d.outside[s] = cell_outside(P, x.x, x.y, x.z) ? 1 : 0;
    uint32_t c;
    if (!grid_cell(P, x.x, x.y, x.z, c)) {
        atomicOr(d.status, ST_OUT_OF_GRID);
        c = d.ncells_all;
    } else {
        c += P.cell_base;
    }
    d.cell[s] = c;
}

__global__ void k_count(Dev d)
{
    if (*d.rebuild == 0u) return;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) *d.alias_any = 0u;   // recomputed by k_post_sort
    if (s >= d.np_all) return;
    atomicAdd(&d.cell_fill[d.cell[s]], 1u);
}

// block-wide exclusive scan of one value per thread; returns the block total
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t &excl)
{
    __shared__ uint32_t warp_tot[CELL_BLOCK / 32];
    const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= (unsigned)o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    uint32_t woff = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < CELL_BLOCK / 32; ++w) {
        const uint32_t t = warp_tot[w];
        if ((unsigned)w < warp) woff += t;
        tot += t;
    }
    __syncthreads();
    excl = woff + inc - v;
    return tot;
}

// pass 1: per-tile totals of cell_fill[0 .. ncells] (ncells + 1 buckets)
__global__ void k_scan_tiles(Dev d)
{
    if (*d.rebuild == 0u) return;
    const uint32_t n = d.ncells_all + 1;
    const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
        if (base + i < n) sum += d.cell_fill[base + i];
    uint32_t excl;
    const uint32_t tot = block_exclusive_scan(sum, excl);
    if (threadIdx.x == 0) d.scan_tiles[blockIdx.x] = tot;
}

// pass 2: every block adds up the totals of the tiles before it, then writes
// cell_start for its own tile; cell_start[ncells + 1] = np
__global__ void k_scan_apply(Dev d)
{
    if (*d.rebuild == 0u) return;
    const uint32_t n = d.ncells_all + 1;
    uint32_t pre = 0;
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += CELL_BLOCK) pre += d.scan_tiles[b];
    // block reduction of pre
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, o);
    __shared__ uint32_t red[CELL_BLOCK / 32];
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = pre;
    __syncthreads();
    uint32_t tile_off = 0;
#pragma unroll
    for (int w = 0; w < CELL_BLOCK / 32; ++w) tile_off += red[w];
    __syncthreads();
    const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = (base + i < n) ? d.cell_fill[base + i] : 0u;
        sum += v[i];
    }
    uint32_t excl;
    (void)block_exclusive_scan(sum, excl);
    uint32_t run = tile_off + excl;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (base + i < n) d.cell_start[base + i] = run;
        run += v[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) d.cell_start[n] = d.np_all;
}

// each particle takes a slot of its cell's range; counters return to zero
__global__ void k_scatter(Dev d)
{
    if (*d.rebuild == 0u) return;
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= d.np_all) return;
    const uint32_t c = d.cell[s];
    const uint32_t k = atomicSub(&d.cell_fill[c], 1u) - 1u;
    d.cellorder[d.cell_start[c] + k] = s;
}

// order the members of each cell by particle index (insertion sort)
__global__ void k_cellsort(Dev d)
{
    if (*d.rebuild == 0u) return;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > d.ncells_all) return;
    const uint32_t beg = d.cell_start[c], end = d.cell_start[c + 1];
    for (uint32_t i = beg + 1; i < end; ++i) {
        const uint32_t s = d.cellorder[i];
        const uint32_t key = d.uid[s];
        uint32_t j = i;
        while (j > beg) {
            const uint32_t o = d.cellorder[j - 1];
            if (d.uid[o] <= key) break;
            d.cellorder[j] = o;
            --j;
        }
        d.cellorder[j] = s;
    }
}

// inverse of the new order and the float copy of the positions in list order
__global__ void k_post_sort(Dev d, int A)
{
    if (*d.rebuild == 0u) return;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.np_all) return;
    const uint32_t s = d.cellorder[k];
    const Params &P = prm_of(d, s);
    d.pos[s] = k;
    const double4 x = d.xr[A][s];
    d.xs[A][k] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    // a particle whose floored coordinates leave the grid sits outside its
    // cell's box (saturated or aliased cell id): contact search must then
    // not prune cells by geometry
    const double f0 = cell_floor(P, 0, x.x), f1 = cell_floor(P, 1, x.y), f2 = cell_floor(P, 2, x.z);
    if (!(f0 >= 0.0 && f0 < (double)P.num[0] && f1 >= 0.0 && f1 < (double)P.num[1] &&
          f2 >= 0.0 && f2 < (double)P.num[2]))
        atomicOr(d.alias_any, 1u);
}

// Verlet lists: every cell of the 27-cell neighbourhood of a cell that
// gained or lost a member is stamped with this step's number; particles in
// stamped cells re-sweep their stencil (their list's membership or order may
// have changed).  Periodic axes wrap as in findDistMod.
__global__ void k_mark_dirty(Dev d)
{
    if (*d.rebuild == 0u) return;
    Verlet &V = *d.vs;
    const uint32_t n = min(V.nmovers, MOVER_CAP);
    if (blockIdx.x == 0 && threadIdx.x == 0) V.rebuilds += 1u;
    if (blockIdx.x == 0 && threadIdx.x == 0 && V.movers_overflow) {
        V.all_rebuild = 1u;
        V.dmax_bits = 0u;
    }
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * n; e += gridDim.x * blockDim.x) {
        const uint2 mv = d.movers[e >> 1];
        const uint32_t cg = (e & 1u) ? mv.y : mv.x;
        if (cg >= d.ncells_all) continue;
        // the instance owning global cell cg (batched contexts)
        uint32_t inst = 0;
        if (d.inst) {
            uint32_t lo = 0, hi = d.ninst;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (d.inst_cell_base[mid] <= cg) lo = mid; else hi = mid;
            }
            inst = lo;
        }
        const Params &P = d.prm[inst];
        const uint32_t c = cg - P.cell_base;
        const uint32_t nx = P.num[0], ny = P.num[1], nz = P.num[2];
        const int32_t cx = (int32_t)(c % nx), cy = (int32_t)((c / nx) % ny), cz = (int32_t)(c / (nx * ny));
        for (int oz = -1; oz < 2; ++oz) {
            const int32_t z = cz + oz;
            if (z < 0 || z >= (int32_t)nz) continue;
            for (int oy = -1; oy < 2; ++oy) {
                int32_t y = cy + oy;
                if (y < 0 || y >= (int32_t)ny) {
                    if (P.periodic != 1) continue;
                    y = (y + (int32_t)ny) % (int32_t)ny;
                }
                for (int ox = -1; ox < 2; ++ox) {
                    int32_t x = cx + ox;
                    if (x < 0 || x >= (int32_t)nx) {
                        if (P.periodic != 1 && P.periodic != 2) continue;
                        x = (x + (int32_t)nx) % (int32_t)nx;
                    }
                    d.dirty[P.cell_base + (uint32_t)x + (uint32_t)y * nx + (nx * ny) * (uint32_t)z] = V.step;
                    V.dirty_step = V.step;
                }
            }
        }
    }
}

// Graph gate of the rebuild: the six rebuild kernels and the flag reset form
// the body of a conditional graph node that runs only when the step before
// moved a particle to another cell; this kernel sets the node's condition.
__global__ void k_rebuild_gate(cudaGraphConditionalHandle h, const uint32_t *rebuild)
{
    cudaGraphSetConditional(h, *rebuild ? 1u : 0u);
}

void launch_rebuild_gate(cudaGraphConditionalHandle h, const uint32_t *rebuild, cudaStream_t st)
{
    k_rebuild_gate<<<1, 1, 0, st>>>(h, rebuild);
}

void launch_cell_init(const Dev &d, uint32_t np, int a, cudaStream_t st)
{
    k_cell_init<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d, a);
}

// A Verlet epoch from scratch after a state was put back: the cell list is
// rebuilt and every particle sweeps in the next step.
__global__ void k_epoch_reset(Dev d)
{
    Verlet V{};
    V.step = 1;
    V.all_rebuild = 1;
    *d.vs = V;
    *d.rebuild = 1u;
}

void launch_epoch_reset(const Dev &d, cudaStream_t st)
{
    k_epoch_reset<<<1, 1, 0, st>>>(d);
}

void launch_rebuild(const Dev &d, uint32_t np, uint32_t ncells, int a, cudaStream_t st)
{
    const unsigned int ntiles = div_up((unsigned long long)ncells + 1, SCAN_TILE);
    k_count<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d);
    k_scan_tiles<<<ntiles, CELL_BLOCK, 0, st>>>(d);
    k_scan_apply<<<ntiles, CELL_BLOCK, 0, st>>>(d);
    k_scatter<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d);
    k_cellsort<<<div_up((unsigned long long)ncells + 1, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d);
    k_post_sort<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d, a);
    k_mark_dirty<<<64, CELL_BLOCK, 0, st>>>(d);
    cudaMemsetAsync(d.rebuild, 0, sizeof(uint32_t), st);
}

unsigned int scan_tile_count(uint32_t ncells)
{
    return div_up((unsigned long long)ncells + 1, SCAN_TILE);
}

// ---- relayout: storage order := current cell order -----------------------
// inv[old storage index] = new storage index
__global__ void k_relayout_inv(Dev d, uint32_t *inv)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.np_all) return;
    inv[d.cellorder[k]] = k;
}

template <typename T>
__global__ void k_gather(const T *__restrict__ src, T *__restrict__ dst, const uint32_t *order,
                         uint32_t n)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[order[k]];
}

// contact rows: move the row and translate partner indices
// Tiled slot entries into the new storage order: entry e of the new tiles
// takes the old particle's entry, partners renamed through `inv` (empty
// slots keep whatever they held: an empty slot's entry is never read).
__device__ __forceinline__ bool tile_entry(uint64_t e, uint32_t np, uint32_t &s, uint32_t &i)
{
    s = (uint32_t)((e / (32ull * NC)) * 32ull + (e & 31ull));
    i = (uint32_t)((e >> 5) % NC);
    return s < np;
}

__global__ void k_gather_rows(const uint32_t *src, uint32_t *dst, const uint32_t *order,
                              const uint32_t *inv, uint32_t np)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= tiled_size(np, NC)) return;
    uint32_t s, i;
    if (!tile_entry(e, np, s, i)) return;
    const uint32_t v = src[tile_at(order[s], i, NC)];
    dst[e] = (v < np) ? inv[v] : np;
}

__global__ void k_gather_dt(const P3 *src, P3 *dst, const uint32_t *order, uint32_t np)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= tiled_size(np, NC)) return;
    uint32_t s, i;
    if (!tile_entry(e, np, s, i)) return;
    dst[e] = src[tile_at(order[s], i, NC)];
}

__global__ void k_relayout_finish(Dev d, int A)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.np_all) return;
    d.cellorder[k] = k;
    d.pos[k] = k;
    d.sidx[d.uid[k]] = k;
    if (k == 0) {
        // storage indices changed: every Verlet list is stale
        d.vs->all_rebuild = 1u;
        d.vs->dmax_bits = 0u;
    }
    const double4 x = d.xr[A][k];
    d.xs[A][k] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
}

template <typename T>
static void gather_back(T *arr, void *scratch, const uint32_t *order, uint32_t n, cudaStream_t st)
{
    T *tmp = static_cast<T *>(scratch);
    k_gather<T><<<div_up(n, CELL_BLOCK), CELL_BLOCK, 0, st>>>(arr, tmp, order, n);
    cudaMemcpyAsync(arr, tmp, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, st);
}

// Permute every per-particle array into the order of d.cellorder (which the
// rebuild kernels must have brought up to date).  `scratch` holds at least
// tiled_size(np, NC) * sizeof(P3) bytes plus np * sizeof(uint32_t) for the
// inverse.
void relayout(const Dev &d, uint32_t np, int a, void *scratch, cudaStream_t st)
{
    uint32_t *inv = reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) +
                                                 tiled_size(np, NC) * sizeof(P3));
    const uint32_t *order = d.cellorder;
    k_relayout_inv<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d, inv);
    gather_back(d.xr[a], scratch, order, np, st);
    gather_back(d.vel[a], scratch, order, np, st);
    gather_back(d.angvel[a], scratch, order, np, st);
    gather_back(d.vel0, scratch, order, np, st);
    gather_back(d.angvel0, scratch, order, np, st);
    gather_back(d.angpos, scratch, order, np, st);
    gather_back(d.xysum, scratch, order, np, st);
    gather_back(d.esv, scratch, order, np, st);
    gather_back(d.force, scratch, order, np, st);
    gather_back(d.torque, scratch, order, np, st);
    gather_back(d.acc, scratch, order, np, st);
    gather_back(d.angacc, scratch, order, np, st);
    gather_back(d.edp, scratch, order, np, st);
    gather_back(d.uid, scratch, order, np, st);
    gather_back(d.cell, scratch, order, np, st);
    gather_back(d.fixed, scratch, order, np, st);
    gather_back(d.outside, scratch, order, np, st);
    gather_back(d.cmask, scratch, order, np, st);
    gather_back(d.dmc, scratch, order, np, st);
    gather_back(d.wtouch, scratch, order, np, st);
    if (d.inst) gather_back(d.inst, scratch, order, np, st);
    const size_t ntile = tiled_size(np, NC);
    const unsigned int rows = div_up(ntile, CELL_BLOCK);
    {
        uint32_t *tmp = static_cast<uint32_t *>(scratch);
        k_gather_rows<<<rows, CELL_BLOCK, 0, st>>>(d.contacts, tmp, order, inv, np);
        cudaMemcpyAsync(d.contacts, tmp, sizeof(uint32_t) * ntile, cudaMemcpyDeviceToDevice, st);
    }
    {
        P3 *tmp = static_cast<P3 *>(scratch);
        k_gather_dt<<<rows, CELL_BLOCK, 0, st>>>(d.delta_t, tmp, order, np);
        cudaMemcpyAsync(d.delta_t, tmp, sizeof(P3) * ntile, cudaMemcpyDeviceToDevice, st);
    }
    k_relayout_finish<<<div_up(np, CELL_BLOCK), CELL_BLOCK, 0, st>>>(d, a);
}

}  // namespace sphk
