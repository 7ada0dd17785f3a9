// sphk_internal.cuh -- device-side layout and exact-order arithmetic shared by
// the kernels of libsphk (the B200 DEM step).
//
// Numerics.  Every kernel here must reproduce the reference's double-precision
// results bit for bit (src/CMakeLists.txt:16-22 builds the reference with
// --fmad=false).  libsphk is therefore compiled with --fmad=false, and the
// helpers below keep the operand order of the reference's vector operators
// (src/vector_arithmetic.h): scalar*vector is (s*a.x, s*a.y, s*a.z),
// vector*scalar is (a.x*s, ...), dot() sums left to right, and length()
// narrows the dot product to float and takes a correctly rounded float square
// root (src/vector_arithmetic.h:317-320).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sphk {

constexpr int NC = 32;           // contact slots per particle, src/constants.h:24
constexpr int MAXWALLS = 6;      // src/constants.h:11
constexpr double REF_PI = 3.14159265358979;   // src/constants.h:14

// device status bits (OR-ed into Ctx::status)
constexpr uint32_t ST_NC_OVERFLOW = 1u;   // a contact would land past slot NC-1
constexpr uint32_t ST_OUT_OF_GRID = 2u;   // a cell index fell outside the grid
constexpr uint32_t ST_BOND_ALIAS = 4u;    // a broken bond's marker aliases a particle
constexpr uint32_t ST_TIMEOUT = 8u;       // a bounded device wait gave up

struct d3 { double x, y, z; };

__device__ __forceinline__ d3 mk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 add(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ d3 smul(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ d3 muls(d3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ d3 divs(d3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ d3 adds(d3 a, double s) { return mk(a.x + s, a.y + s, a.z + s); }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// length(): float square root of the narrowed dot product
__device__ __forceinline__ double flen(d3 a)
{
    return (double)__fsqrt_rn(__double2float_rn(dot(a, a)));
}
__device__ __forceinline__ double fsqrt_of(double v) { return (double)__fsqrt_rn(__double2float_rn(v)); }
__device__ __forceinline__ d3 xyz(double4 v) { return mk(v.x, v.y, v.z); }

// Static scene parameters, resident in device memory for the whole run.
struct Params {
    uint32_t np, nw, nb0, contactmodel;
    int32_t periodic;
    uint32_t num[3];
    uint32_t ncells;
    double origo[3], L[3], cellsize[3];   // cellsize = L / num, computed once
    double dt;
    double g[3], k_n, k_t, k_r, gamma_n, gamma_t, gamma_r, mu_s, mu_d, mu_r;
    double gamma_wn, gamma_wt, mu_ws, mu_wd, rho, kappa, db, V_b;
    double lambda_bar, sigma_b, tau_b, devs_A, devs_f;
    int32_t wmode[MAXWALLS];
    float cull_eps;     // absolute FP32 slack of the neighbour cull (metres)
    double rmax;        // largest radius of the scene (set at upload)
    double prune_pad;   // absolute slack of the cell-level distance test (metres)
    double skin;        // Verlet-list skin (metres); 0 disables the lists
    double reach_extra; // model 1: db, the capillary reach beyond contact (metres)
    uint32_t esv_skip;  // no es/ev is -0.0: adding a zero rate may be skipped exactly
    uint32_t cell_base; // batched contexts: first global cell id of this instance
    uint32_t uid_base;  // batched contexts: first global particle index of this instance
};

// The scene constants the force kernel reads for every particle, passed by
// value to single-scene launches (read from the constant bank, never
// reloaded after a store); the same fields as in Params.  skin and esv_skip
// change at upload: a context captures its step graphs again when any field
// changes.
struct ForceConsts {
    uint32_t nw, nb0, ncells, cell_base;
    int32_t periodic;
    uint32_t num[3];
    uint32_t esv_skip;
    uint32_t pad;
    double origo[3], L[3], cellsize[3];
    double dt, g[3], rho, skin;
};
inline ForceConsts force_consts(const Params &P)
{
    ForceConsts c{};
    c.nw = P.nw;
    c.nb0 = P.nb0;
    c.ncells = P.ncells;
    c.cell_base = P.cell_base;
    c.periodic = P.periodic;
    c.esv_skip = P.esv_skip;
    for (int i = 0; i < 3; ++i) {
        c.num[i] = P.num[i];
        c.origo[i] = P.origo[i];
        c.L[i] = P.L[i];
        c.cellsize[i] = P.cellsize[i];
        c.g[i] = P.g[i];
    }
    c.dt = P.dt;
    c.rho = P.rho;
    c.skin = P.skin;
    return c;
}

constexpr int VL_CAP = 32;              // candidates kept per particle
constexpr uint8_t VL_NONE = 0xff;       // no usable list: sweep the stencil
constexpr uint32_t MOVER_CAP = 1u << 16;

// State of the Verlet-list epoch, device resident.  An epoch starts with a
// full sweep of every particle; lists stay exact while 4 * dmax < skin, where
// dmax bounds how far any particle moved since the epoch started.
struct Verlet {
    uint32_t step;          // number of the step about to run (dirty stamps)
    uint32_t all_rebuild;   // every particle sweeps in this step
    uint32_t dmax_bits;     // float bits of the displacement bound (atomicMax)
    uint32_t nmovers;       // particles that changed cell in the last step
    uint32_t movers_overflow;
    uint32_t dirty_step;    // the last step in which any cell was stamped dirty
    uint32_t rebuilds;      // cell-list rebuilds performed since upload
    uint32_t pad;
};

// Wall state (src/datatypes.h:95-100), device resident.
struct Walls {
    double4 nx[MAXWALLS];     // normal xyz, position w
    double4 mvfd[MAXWALLS];   // mass, velocity, force, deviatoric stress
    double vel0[MAXWALLS];    // half-step velocities
    double t_current;         // simulation time at the start of the next step
    uint32_t done_blocks;     // last-block counter of the wall reduction
    uint32_t pad;
};

// Three doubles (24 bytes): rows whose fourth lane a step never reads.
struct P3 {
    double x, y, z;
};

// The fourth lanes of the host's four-double rows that the device keeps as
// three doubles; a step never changes them.
constexpr int W_VEL0 = 0, W_ANGVEL0 = 1, W_ANGPOS = 2, W_ANGVEL = 3, W_VEL = 4, WLANES = 5;

// A P3 row as a double4 with a zero fourth lane.
__device__ __forceinline__ double4 ld4(const P3 *a, uint32_t i)
{
    const P3 v = a[i];
    return make_double4(v.x, v.y, v.z, 0.0);
}
__device__ __forceinline__ P3 p3of(double4 v) { return P3{v.x, v.y, v.z}; }

// Device pointers of one simulation.  Per-particle arrays are indexed by the
// storage index s (particles are kept in cell order); uid[s] is the caller's
// particle index and sidx[uid] its inverse.  Contact rows store partners as
// storage indices, np marks an empty slot.
struct Dev {
    // sizes of the whole context: one scene, or every instance of a batch
    uint32_t np_all, ncells_all, ninst;
    uint32_t shape;       // block shapes of the contact search and forces (SPH_OPT_BLOCK_SHAPES)
    uint32_t topo_span;   // list decisions per thread of the contact search (0: by size)
    // batched contexts: instance of each storage index and the first global
    // cell id of each instance (ninst + 1 entries); nullptr for one scene
    uint32_t *inst;
    uint32_t *inst_cell_base;
    // double-buffered kinematics read by neighbours: [0]/[1]
    double4 *xr[2];       // x, y, z, radius
    P3 *vel[2];           // vx, vy, vz (fixvel in `fixed`, the host lane in w_user)
    P3 *angvel[2];        // wx, wy, wz (the host lane in w_user)
    float4 *xs[2];        // float copy of xr in cell-list order, for the neighbour cull
    // private per-particle state (updated in place); three doubles each, the
    // fourth lane of the host rows (never changed by a step) is kept apart in
    // w_user
    P3 *vel0, *angvel0, *angpos;
    double *w_user;       // [np][WLANES] fourth host lanes, by caller index (W_* below)
    uint8_t *fixed;       // fixvel > 0: x/y acceleration and spin held (integration.cuh:65-77)
    double2 *xysum;
    double2 *esv;         // es, ev
    // per-step outputs
    double4 *force, *torque, *acc, *angacc;
    double4 *edp;         // es_dot, ev_dot, p, 0
    uint32_t *uid, *sidx;
    uint32_t *cell;       // cell id (calcCellID semantics) of the current positions
    uint8_t *outside;     // the position's floored cell coordinates leave the grid
    // contacts
    uint32_t *contacts;   // tiled, NC per particle (tile_at)
    ulonglong2 *dmc;      // [np] 4-bit periodic shift code of each of the NC slots
    P3 *delta_t;          // tiled, NC per particle; the reference's fourth lane is always 0
    uint32_t *cmask;      // [np] occupied-slot bit mask
    // [ceil(np / 32)] the chunk of 32 storage indices may hold a contact
    // (1), or, between k_contact and k_force_tiles, was visited by k_contact
    // (2: a slot is still held, 3: none is)
    uint8_t *cflag;
    // contact models 2 and 3: the slot sums k_contact leaves for k_force_tiles (F
    // xyz and p; T xyz and ev_dot; es_dot)
    double4 *csum_f, *csum_t;
    double *csum_es;
    // cell list (cell order sorted by uid inside each cell)
    uint32_t *cell_start; // [ncells + 2]
    uint32_t *cellorder;  // [np] cell-list position -> storage index
    uint32_t *pos;        // [np] storage index -> cell-list position
    uint32_t *cell_fill;  // [ncells + 1] scratch
    uint32_t *scan_tiles; // scratch for the scan
    uint32_t *alias_any;  // some particle sits outside its cell's box (set by the rebuild)
    // Verlet lists
    uint32_t *vl;         // tiled, VL_CAP per particle: candidate storage indices, in visiting order
    uint32_t *vl_meta;    // tiled, VL_CAP per particle: vl_meta_of(stencil cell, shift code, gap)
    uint8_t *vl_len;      // [np] list length or VL_NONE
    float *vl_gap;        // [np] lower bound of the smallest gap to a listed candidate
    float *disp;          // [np] displacement bound since the epoch started
    uint8_t *settled;     // [np] every candidate of the valid list holds its slot (k_topo sets
                          // it; a freed slot, a new list, upload or relayout clears it)
    uint2 *movers;        // [MOVER_CAP] (old cell, new cell) of the last step
    uint32_t *dirty;      // [ncells + 1] step stamp: a neighbour cell changed members
    Verlet *vs;
    // walls
    double *wf_pp;        // [np] wall-0 force by uid
    uint8_t *wtouch;      // [np] by storage index: wall-0 force was nonzero
    double *wf_partial;   // [ceil(np/256)]
    uint8_t *wf_flag;     // [ceil(np/256)] a wall-0 force of the 256-block was written
    Walls *walls;
    // bonds (user indices, as the reference stores them)
    uint2 *bonds;
    double4 *bonds_delta, *bonds_omega;
    double4 *bond_f, *bond_t;   // per-bond force on x and torque on y
    uint32_t *bond_xu;          // user index that received +f this step, or ~0u
    uint2 *bond_s;              // the bond's particles as storage indices (set at relayout)
    uint32_t *bond_ptr;         // [np + 1] CSR by uid
    uint32_t *bond_list;        // [2 nb0] (bond << 1) | role (0: x, 1: y)
    // contact model 1: contact force xyz and pressure summed by k_topo
    double4 *c1acc;
    // differentiable step: per-particle friction and the tape of one segment
    // ([step][np] rows; partner and history rows [step][np][NC], written for
    // evaluated slots only)
    double *mu_p;
    double4 *tp_x, *tp_v, *tp_w;
    P3 *tp_dt0;             // tape_slot_at: starting history of each evaluated slot
    uint32_t *tp_mask, *tp_partner;   // tp_partner: tape_slot_at
    ulonglong2 *tp_dmc;
    // status
    uint32_t *status;
    uint32_t *rebuild;          // cell list must be rebuilt before the next step
    Params *prm;
};

// Parameters of the scene that storage index s belongs to.  Dev::prm holds
// one Params per instance; a single-scene context has exactly one.
__device__ __forceinline__ const Params &prm_of(const Dev &d, uint32_t s)
{
    return d.inst ? d.prm[d.inst[s]] : *d.prm;
}

// The same, with the kind of context fixed at compile time (the step
// kernels are instantiated for each, so a single scene's kernels carry no
// instance lookup).
template <bool BATCH>
__device__ __forceinline__ const Params &prm_at(const Dev &d, uint32_t s)
{
    if constexpr (BATCH) return d.prm[d.inst[s]];
    else return *d.prm;
}

// The force-law constants of one scene (contact models 2 and 3), fixed when
// a context is created.  Single-scene contexts pass them to the contact
// kernel by value, where the law reads them as constant operands.
struct LawParams {
    double k_n, k_t, gamma_n, gamma_t, gamma_r, mu_s, mu_d, mu_r, kappa, dt;
    double L[2];
};

// periodic shift code: bits 0-1 x (1: +L, 2: -L), bits 2-3 y.  PR is Params
// or LawParams.
template <class PR>
__device__ __forceinline__ d3 decode_dm(uint32_t code, const PR &P)
{
    // reproduces (0,0,0) += (L,0,0) / -= (L,0,0) etc. of findDistMod
    double dx = 0.0, dy = 0.0, dz = 0.0;
    if (code & 1u) { dx = dx + P.L[0]; dy = dy + 0.0; dz = dz + 0.0; }
    if (code & 2u) { dx = dx - P.L[0]; dy = dy - 0.0; dz = dz - 0.0; }
    if (code & 4u) { dx = dx + 0.0; dy = dy + P.L[1]; dz = dz + 0.0; }
    if (code & 8u) { dx = dx - 0.0; dy = dy - P.L[1]; dz = dz - 0.0; }
    return mk(dx, dy, dz);
}

// (x - origo) / (L / num), floored (src/sorting.cuh:12-14).  G is any grid
// with origo[3], cellsize[3], num[3] and ncells (Params among them).
template <class G>
__device__ __forceinline__ double cell_floor(const G &P, int d, double v)
{
    return floor((v - P.origo[d]) / P.cellsize[d]);
}

// calcCellID with the device's saturating float->unsigned conversion
template <class G>
__device__ __forceinline__ uint32_t cell_id(const G &P, double x, double y, double z)
{
    uint32_t ix = __double2uint_rz(cell_floor(P, 0, x));
    uint32_t iy = __double2uint_rz(cell_floor(P, 1, y));
    uint32_t iz = __double2uint_rz(cell_floor(P, 2, z));
    return (iz * P.num[1]) * P.num[0] + iy * P.num[0] + ix;
}

// The cell of a position for the cell list: calcCellID's id in c, and
// whether it lies in the grid.  A position that is not finite is outside
// whatever its float-to-integer conversion gives; every cell list here puts
// such a particle, like one whose id is past the grid, in one bucket after
// the last cell.
template <class G>
__device__ __forceinline__ bool grid_cell(const G &P, double x, double y, double z, uint32_t &c)
{
    c = cell_id(P, x, y, z);
    return c < P.ncells && isfinite(x + y + z);
}

// Whether some floored cell coordinate of the position lies outside
// [0, num): the particle is not inside its own cell's box (contact search
// takes the reference's stencil from the floored coordinates, not the id).
template <class G>
__device__ __forceinline__ bool cell_outside(const G &P, double x, double y, double z)
{
    const double f0 = cell_floor(P, 0, x), f1 = cell_floor(P, 1, y), f2 = cell_floor(P, 2, z);
    return !(f0 >= 0.0 && f0 < (double)P.num[0] && f1 >= 0.0 && f1 < (double)P.num[1] &&
             f2 >= 0.0 && f2 < (double)P.num[2]);
}

// Tiles of 32 storage indices.  The contact slots (partners and tangential
// history) and the Verlet lists hold `width` entries per particle, stored
// tile by tile: entry i of particle s sits at ((s / 32) width + i) 32 +
// s % 32.  The lanes of a warp that touch entry i of their 32 particles touch
// one contiguous run, and the few entries a particle uses (its occupied
// slots, its short list) cost no more than their own bytes, where rows of
// `width` entries per particle cost whole cache lines.
__host__ __device__ __forceinline__ size_t tile_at(uint32_t s, uint32_t i, uint32_t width)
{
    return ((size_t)(s >> 5) * width + i) * 32u + (s & 31u);
}
// Asks the copy engine to bring `bytes` at `p` into L2 (a hint: nothing is
// waited for, no register is held).  `p` and `bytes` are multiples of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Bulk copies into shared memory that complete on an mbarrier (the copy
// engine moves the bytes; the issuing thread holds no register for them).
// Addresses and sizes are multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised barriers visible to the copy engine
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// the issuing thread's arrival, announcing `bytes` of copies to complete
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// orders this thread's earlier shared-memory accesses (and those a barrier
// made it wait for) before the copies it issues next
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits until phase `parity` of `bar` completes, for at most limit_ns
// nanoseconds; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}
// The per-particle arrays that the force kernel copies in tiles are
// allocated in whole multiples of ROW_PAD rows, so that a tile's copy never
// reads past its array.
constexpr uint32_t ROW_PAD = 128;
__host__ __device__ constexpr size_t padded_rows(size_t n) { return (n + ROW_PAD - 1) / ROW_PAD * ROW_PAD; }

// How long a kernel waits for a bulk copy before it reports ST_TIMEOUT.
constexpr uint64_t BULK_WAIT_NS = 1000000000ull;

// The slot rule fills the last empty slot first (src/contactsearch.cuh:
// 252-271), so a particle's few contacts sit in the top slots: the tile rows
// worth fetching ahead are the top PF_SLOTS.  Six: a dense packing holds
// four to six contacts a sphere (the jammed column exactly six), and rows
// fetched for empty slots only take L2 bandwidth from the ones used
// (4, 5, 6 and 8 slots measured on the 1M column: 6 fastest).
#ifndef SPHK_PF_SLOTS
#define SPHK_PF_SLOTS 6
#endif
constexpr uint32_t PF_SLOTS = SPHK_PF_SLOTS;

// The metadata of a Verlet-list entry: bits 0-4 the stencil cell (0..26),
// 5-15 the periodic shift code, 16-31 the top half of the float gap to the
// candidate when the list was recorded (a lower bound: the float's low half
// is dropped, toward zero, and a negative gap is kept as 0).
__device__ __forceinline__ uint32_t vl_meta_of(uint32_t slot, uint32_t code, float gap)
{
    const uint32_t g = __float_as_uint(fmaxf(gap, 0.0f)) & 0xffff0000u;
    return slot | (code << 5) | g;
}
__device__ __forceinline__ uint32_t vl_code(uint32_t meta) { return (meta & 0xffffu) >> 5; }
__device__ __forceinline__ float vl_gap_of(uint32_t meta) { return __uint_as_float(meta & 0xffff0000u); }

// Entry e of particle s's Verlet list (Dev::vl, Dev::vl_meta): tiled like
// the slots, or (SPHK_VL_ROWS) one row of VL_CAP entries per particle.
#ifdef SPHK_VL_ROWS
__host__ __device__ __forceinline__ size_t vl_at(uint32_t s, uint32_t e)
{
    return (size_t)s * VL_CAP + e;
}
#else
__host__ __device__ __forceinline__ size_t vl_at(uint32_t s, uint32_t e)
{
    return tile_at(s, e, VL_CAP);
}
#endif
// Entries of a tiled array for np particles (the last tile is padded).
__host__ __device__ __forceinline__ size_t tiled_size(size_t np, uint32_t width)
{
    return ((np + 31) / 32) * 32 * (size_t)width;
}

// Slot i of particle s in row j of the differentiable step's tape: the slot
// tiles of every step one after another, so that a warp's accesses to one
// slot of its 32 particles are one contiguous run, as in the state's slots.
__host__ __device__ __forceinline__ size_t tape_slot_at(uint32_t j, uint32_t np, uint32_t s, uint32_t i)
{
    return (size_t)j * tiled_size(np, NC) + tile_at(s, i, NC);
}

inline unsigned int div_up(unsigned long long a, unsigned int b)
{
    return (unsigned int)((a + b - 1) / b);
}

// Darcy flow state (src/darcy.cuh): the fluid grid is the cell grid with one
// ghost node on every side, (num[0]+2)(num[1]+2)(num[2]+2) nodes, x fastest,
// laid out as the reference's host arrays so that upload and download are
// plain copies.  V, dH and T hold three doubles per node.
struct DarcyDev {
    double *H[2];          // pressure buffers; a step reads H[hs], writes H[hs ^ 1]
    double *V, *dH, *T;
    double *K, *Ss, *W, *phi, *dphi;
    uint32_t *first;       // 1 until the first step after upload has run
    double nu;             // dynamic viscosity
    double d_factor;       // grain-size factor of the Kozeny-Carman relation
};

}  // namespace sphk
