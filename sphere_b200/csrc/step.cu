// step.cu -- the per-particle DEM step of libsphk, in three launches.
//
// k_topo   contact detection into the persistent slots (topology,
//          src/contactsearch.cuh:181-355): a lane's list decisions for one
//          to four particles, then a search for each particle they do not
//          settle.  Candidates come from a float copy of the positions kept
//          in cell-list order (Dev::xs), so the three cells of each x-row of
//          the 27-cell stencil are three adjacent runs of one array and a
//          candidate costs one coalesced 16-byte load; the particle's own slot
//          row is fetched only when an overlap is found.
// k_contact the force laws of the occupied slots (interact's slot loop,
//          src/contactsearch.cuh:468-543), one lane per directed contact;
//          each particle's sums, in slot order, are left for k_force_tiles.
// k_force_tiles  everything per particle after it (src/device.cu:829-1058):
//          the slot sums, the walls (interact, contactsearch.cuh:578-663),
//          the per-bond forces of bondsLinear (cohesion.cuh:8-233, computed
//          by bonds.cu and gathered here in bond order), and the half-step
//          leapfrog (integrate, integration.cuh:9-187).  A resident grid over
//          tiles of 128 particles whose rows arrive by bulk copies.  The
//          differentiable step runs k_force_diff instead of k_contact and
//          k_force_tiles.
// Kinematics of step n are read from buffer A and step n+1 is written to
// buffer B, so neighbours always see start-of-step values.
//
// Parity: every expression keeps the reference's operation order; see
// sphk_internal.cuh.  Candidates are first culled with a conservative FP32
// distance test (Params::cull_eps bounds the float rounding), then the
// reference's own predicate float_sqrt(dot) - (ra + rb) < 0 decides.  The
// visiting order is the reference's: stencil cells z, y, x, members of a cell
// by particle index.
#include <algorithm>

#include "sphk_internal.cuh"
#include "diff_step.cuh"

namespace sphk {

// Threads per block, and resident blocks per SM that the register
// allocation must allow (the __launch_bounds__ minimum), from sweeps of
// block shapes and caps at 1M spheres.
#ifndef SPHK_FORCE_BLOCK
#define SPHK_FORCE_BLOCK 128
#endif
constexpr int FORCE_BLOCK = SPHK_FORCE_BLOCK;
#ifndef SPHK_FORCE_MIN_BLOCKS
#define SPHK_FORCE_MIN_BLOCKS 8
#endif
// The contact search and the contact forces are compiled in two block
// shapes each, and a context picks one pair (Dev::shape, SPH_OPT_BLOCK_SHAPES;
// the ensemble's autotuner times both).  Shape 0, the default: k_topo in
// blocks of 64 threads, 16 per SM, whose threads leave at different times;
// k_contact in blocks of 4 warps, 5 per SM.  Shape 1: k_topo in 128 x 8,
// k_contact in 2 warps x 10.  The threads resident per SM are the same.
#ifndef SPHK_TOPO_THREADS_PER_SM
#define SPHK_TOPO_THREADS_PER_SM 1024
#endif
constexpr int TOPO_THREADS_PER_SM = SPHK_TOPO_THREADS_PER_SM;
#ifndef SPHK_CONTACT_THREADS_PER_SM
#define SPHK_CONTACT_THREADS_PER_SM 640
#endif
constexpr int CONTACT_THREADS_PER_SM = SPHK_CONTACT_THREADS_PER_SM;
__host__ __device__ constexpr int topo_block(uint32_t shape) { return shape ? 128 : 64; }
__host__ __device__ constexpr int contact_block(uint32_t shape) { return shape ? 64 : 128; }

// What one law adds to a particle's sums.  The laws return their terms by
// value and the caller adds them: each reference update `s += term` is the
// caller's `s + term`, the same operation.  (The wall law is out of line;
// a reference into the caller's sums would put them in local memory for the
// whole kernel.)
struct WallOut {
    d3 f, t;       // F += f, T += t
    double pr;     // p += pr
    double fn;     // the normal force along n (walls_force_pp)
};
struct LawOut {
    d3 f, t;           // F += f, T += t
    double pr, ev;     // p += pr, ev_dot += ev
    double es;         // es_dot += es, where es_set
    bool es_set;
    double4 dt4;       // the slot's new tangential history
};

// contactLinear_wall, src/contactmodels.cuh:10-109.  Inlined into
// wall_forces, its one caller.
__device__ __forceinline__ WallOut contact_wall(const Params &P, double ra, double4 vel_a,
                                             double4 angvel_a, d3 n, double delta, double wvel)
{
    const d3 linvel = xyz(vel_a), angvel = xyz(angvel_a);
    const d3 vel = adds(add(linvel, smul(ra, cross(n, angvel))), wvel);
    const double vel_n = dot(vel, n);
    const d3 vel_t = sub(vel, muls(n, dot(vel, n)));
    const double vel_t_length = flen(vel_t);
    d3 f_n = smul(-P.k_n * delta - P.gamma_wn * vel_n, n);
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    const double f_n_length = flen(f_n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    const d3 T_res = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.f) {
        const double f_t_visc = P.gamma_wt * vel_t_length;
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = P.mu_wd * f_n_length;
        else f_t_limit = P.mu_ws * f_n_length;
        if (f_t_visc < f_t_limit) f_t = divs(smul(-1.0f * f_t_visc, vel_t), vel_t_length);
        else f_t = divs(smul(-1.0f * f_t_limit, vel_t), vel_t_length);
    }
    WallOut o;
    o.f = add(f_n, f_t);
    o.t = add(smul(-ra, cross(n, f_t)), T_res);
    o.pr = f_n_length / (4.0f * REF_PI * ra * ra);
    o.fn = dot(f_n, n);
    return o;
}

// The walls interact visits, in its order (src/contactsearch.cuh:578-663,
// defaults :416-427): 0 the top wall (dynamic wall 0, else z = L.z), 1 the
// floor at origo.z, then with periodic == 0 the x walls (dynamic walls 1 and
// 2, else x = L.x and x = 0), and with periodic == 0 or 2 the y walls
// (dynamic walls 3 and 4, else y = L.y and y = 0).  Wall k's gap, normal and
// velocity; a dynamic wall replaces the default in order.
template <class PS>
__device__ __forceinline__ double wall_gap(const PS &P, const Walls &W, int k, double4 xa)
{
    auto wpos = [&](int j, double dflt) { return ((uint32_t)j < P.nw) ? W.nx[j].w : dflt; };
    const double ra = xa.w;
    switch (k) {
    case 0: return wpos(0, P.L[2]) - (xa.z + ra);
    case 1: return xa.z - ra - P.origo[2];
    case 2: return wpos(1, P.L[0]) - (xa.x + ra);
    case 3: return xa.x - ra - wpos(2, 0.0);
    case 4: return wpos(3, P.L[1]) - (xa.y + ra);
    default: return xa.y - ra - wpos(4, 0.0);
    }
}

// Bit k: the particle touches wall k (its gap is negative).
template <class PS>
__device__ __forceinline__ uint32_t wall_touch(const PS &P, const Walls &W, double4 xa)
{
    const int nwall = (P.periodic == 0) ? 6 : ((P.periodic == 2) ? 6 : 2);
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (k >= nwall || (P.periodic == 2 && (k == 2 || k == 3))) continue;
        if (wall_gap(P, W, k, xa) < 0.0f) m |= 1u << k;
    }
    return m;
}

struct WallSums {
    d3 F, T;
    double p;
    double w0f;   // the normal force of wall 0 (walls_force_pp)
};

// The wall terms of the touched walls, added in interact's order to the slot
// sums (F, T, p).  Out of line: only particles touching a wall call it.
__device__ __noinline__ WallSums wall_forces(const Params &P, const Walls &W, uint32_t touch,
                                             double4 xa, double4 vel_a, double4 angvel_a, d3 F,
                                             d3 T, double p)
{
    WallSums r{F, T, p, 0.0};
    for (int k = 0; k < 6; ++k) {
        if (!((touch >> k) & 1u)) continue;
        const int j = (k == 0) ? 0 : k - 1;    // the dynamic wall that replaces wall k
        const bool dyn = k != 1 && (uint32_t)j < P.nw;
        d3 n;
        switch (k) {
        case 0: n = mk(0.0, 0.0, -1.0); break;
        case 1: n = mk(0.0, 0.0, 1.0); break;
        case 2: n = mk(-1.0, 0.0, 0.0); break;
        case 3: n = mk(1.0, 0.0, 0.0); break;
        case 4: n = mk(0.0, -1.0, 0.0); break;
        default: n = mk(0.0, 1.0, 0.0); break;
        }
        if (dyn) n = xyz(W.nx[j]);
        const double wv = dyn ? W.mvfd[j].y : ((k == 1) ? (double)0.0f : 0.0);
        const WallOut o = contact_wall(P, xa.w, vel_a, angvel_a, n, wall_gap(P, W, k, xa), wv);
        r.F = add(r.F, o.f);
        r.T = add(r.T, o.t);
        r.p += o.pr;
        if (k == 0) r.w0f = o.fn;
    }
    return r;
}

// contactLinear, src/contactmodels.cuh:283-493 (contact model 2).  Inlined
// into k_contact, the one kernel that evaluates it.
template <class PR>
__device__ __forceinline__ LawOut contact_linear(const PR &P, double4 vel_a, d3 angvel_a,
                                              double4 vel_b4, double4 angvel_b4, double ra,
                                              double rb, d3 x, double x_length, double delta,
                                              double4 dt4)
{
    LawOut o;
    o.es = 0.0;
    o.es_set = false;
    const double dt = P.dt;
    const d3 vel_b = xyz(vel_b4), angvel_b = xyz(angvel_b4);
    const d3 dt0u = xyz(dt4);
    const d3 n = divs(x, x_length);
    const d3 vel_linear = mk(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    const d3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                       smul(rb + delta / 2.0, cross(n, angvel_b)));
    const double vel_n = -dot(vel_linear, n);
    const d3 vel_t = sub(vel, muls(n, dot(n, vel)));
    const double vel_t_length = flen(vel_t);
    const d3 delta_t0 = sub(dt0u, muls(n, dot(n, dt0u)));
    const double delta_t0_length = flen(delta_t0);
    d3 delta_t = mk(0.0, 0.0, 0.0);   // the reference leaves it unset when unused
    d3 f_n = smul(-P.k_n * delta - P.gamma_n * vel_n, n);
    o.ev = P.gamma_n * vel_n * vel_n;
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    const double f_n_length = flen(f_n);
    const d3 f_c = smul(-P.kappa * fsqrt_of(ra * rb), n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = add(delta_t0, muls(vel_t, dt));
        const d3 f_t_elast = smul(-P.k_t, delta_t);
        const d3 f_t_visc = smul(-P.gamma_t, vel_t);
        f_t = add(f_t_elast, f_t_visc);
        const double f_t_length = flen(f_t);
        const double f_t_limit = P.mu_s * flen(sub(f_n, f_c));
        if (f_t_length > f_t_limit) {
            const d3 t = divs(f_t, flen(f_t));
            f_t = smul(f_t_limit, t);
            delta_t = smul(-1.0 / P.k_t,
                           add(smul(P.mu_d * flen(sub(f_n, f_c)), t), smul(P.gamma_t, vel_t)));
            o.es = flen(muls(smul(flen(f_t), vel_t), dt)) / dt;
            o.es_set = true;
        }
    }
    o.f = add(add(f_n, f_t), f_c);
    o.t = cross(smul(-(ra + delta * 0.5), n), f_t);
    o.pr = f_n_length / (4.0f * REF_PI * ra * ra);
    o.dt4 = make_double4(delta_t.x, delta_t.y, delta_t.z, 0.0f);
    return o;
}

// The FP32 transcendentals of the force laws (expf in capillaryCohesion_exp,
// powf in contactHertz), evaluated as the float nearest to the
// double-precision result.  The reference's GPU build used its fast-math
// intrinsics and its host build the C library's functions; neither is
// correctly rounded, so these are the one place where this path follows
// neither bit for bit (the oracle computes the same nearest float).
__device__ __forceinline__ double f32_expf(double x)
{
    return (double)__double2float_rn(exp((double)__double2float_rn(x)));
}
__device__ __forceinline__ double f32_powf(double x, float y)
{
    return (double)__double2float_rn(pow((double)__double2float_rn(x), (double)y));
}

// contactLinearViscous, src/contactmodels.cuh:114-253 (contact model 1): no
// tangential history, and the torque is left alone (its update is commented
// out in the reference, :244).
__device__ __noinline__ void contact_viscous(const Params &P, d3 &F, double &p, double4 vel_a,
                                                double4 vel_b, d3 angvel_a, d3 angvel_b,
                                                double ra, double rb, d3 x_ab,
                                                double x_ab_length, double delta)
{
    const d3 n = divs(x_ab, x_ab_length);
    const d3 vel_linear = mk(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    const d3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                       smul(rb + delta / 2.0, cross(n, angvel_b)));
    const double vel_n = dot(vel_linear, n);
    const d3 vel_t = sub(vel, muls(n, dot(vel, n)));
    const double vel_t_length = flen(vel_t);
    d3 f_n = smul(-P.k_n * delta - P.gamma_n * vel_n, n);
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    const double f_n_length = flen(f_n);
    const d3 f_c = smul(-P.kappa * fsqrt_of(ra * rb), n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0) {
        const double f_t_visc = P.gamma_t * vel_t_length;
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = P.mu_d * flen(sub(f_n, f_c));
        else f_t_limit = P.mu_s * flen(sub(f_n, f_c));
        if (f_t_visc < f_t_limit) f_t = divs(smul(-f_t_visc, vel_t), vel_t_length);
        else f_t = divs(smul(-f_t_limit, vel_t), vel_t_length);
    }
    F = add(F, add(add(f_n, f_t), f_c));
    p += f_n_length / (4.0f * REF_PI * ra * ra);
}

// capillaryCohesion_exp, src/cohesion.cuh:314-350
__device__ __noinline__ void capillary_exp(const Params &P, d3 &F, double ra, double rb,
                                              double delta, d3 x_ab, double x_ab_length)
{
    const d3 n = divs(x_ab, x_ab_length);
    double r;
    if ((ra / rb) > (rb / ra)) r = ra / rb;
    else r = rb / ra;
    const double h = -fsqrt_of(r);
    const double R_har = (2.0f * ra * rb) / (ra + rb);
    const double R_geo = fsqrt_of(ra * rb);
    const double lambda = 0.9f * h * fsqrt_of(P.V_b / R_har);
    const d3 f_c = smul(-P.kappa * R_geo * f32_expf(-delta / lambda), n);
    F = add(F, f_c);
}

// contactHertz, src/contactmodels.cuh:499-666 (contact model 3).  As in the
// reference, delta is the (negative) overlap, so its fractional powers are
// NaN and so are the forces of every touching pair.  Inlined into k_contact.
template <class PR>
__device__ __forceinline__ LawOut contact_hertz(const PR &P, double4 vel_a, d3 angvel_a,
                                             double4 vel_b4, double4 angvel_b4, double ra,
                                             double rb, d3 x, double x_length, double delta,
                                             double4 dt4)
{
    LawOut o;
    o.es = 0.0;
    o.es_set = false;
    const double dt = P.dt;
    const d3 vel_b = xyz(vel_b4), angvel_b = xyz(angvel_b4);
    const d3 dt0u = xyz(dt4);
    const d3 n = divs(x, x_length);
    const d3 vel_linear = mk(vel_a.x - vel_b.x, vel_a.y - vel_b.y, vel_a.z - vel_b.z);
    const d3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                       smul(rb + delta / 2.0, cross(n, angvel_b)));
    const d3 angvel_ab = sub(angvel_a, angvel_b);
    const double angvel_ab_length = flen(angvel_ab);
    const double vel_n = dot(vel_linear, n);
    const d3 vel_t = sub(vel, muls(n, dot(vel, n)));
    const double vel_t_length = flen(vel_t);
    const d3 delta_t0 = sub(dt0u, muls(n, dot(dt0u, n)));
    const double delta_t0_length = flen(delta_t0);
    d3 delta_t = mk(0.0, 0.0, 0.0);   // the reference leaves it unset when unused
    d3 f_n = smul(-P.k_n * f32_powf(delta, 3.0f / 2.0f)
                      - P.gamma_n * f32_powf(delta, 1.0f / 4.0f) * vel_n, n);
    o.ev = P.gamma_n * vel_n * vel_n;
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    const double f_n_length = flen(f_n);
    const d3 f_c = smul(-P.kappa * fsqrt_of(ra * rb), n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    d3 T_res = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.f || vel_t_length > 0.f) {
        const d3 f_t_elast = smul(-P.k_t * f32_powf(delta, 1.0f / 2.0f), delta_t0);
        const d3 f_t_visc = smul(-P.gamma_t * f32_powf(delta, 1.0f / 4.0f), vel_t);
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = P.mu_d * flen(sub(f_n, f_c));
        else f_t_limit = P.mu_s * flen(sub(f_n, f_c));
        f_t = add(f_t_elast, f_t_visc);
        const double f_t_length = flen(f_t);
        if (f_t_length > f_t_limit) {
            f_t = muls(f_t, f_t_limit / f_t_length);
            delta_t = divs(add(f_t, smul(P.gamma_t * f32_powf(delta, 1.0f / 4.0f), vel_t)),
                           -P.k_t * f32_powf(delta, 1.0f / 2.0f));
            o.es = flen(sub(delta_t0, delta_t)) * P.k_t / dt;
            o.es_set = true;
        } else {
            delta_t = add(delta_t0, muls(vel_t, dt));
        }
    }
    if (angvel_ab_length > 0.f) {
        T_res = divs(smul(-1.0f * fmin(P.gamma_r * ra * angvel_ab_length,
                                       P.mu_r * ra * f_n_length),
                          angvel_ab),
                     angvel_ab_length);
    }
    o.f = add(add(f_n, f_t), f_c);
    o.t = add(smul(-(ra + delta / 2.0), cross(n, f_t)), T_res);
    o.pr = f_n_length / (4.0f * REF_PI * ra * ra);
    o.dt4 = make_double4(delta_t.x, delta_t.y, delta_t.z, 0.0f);
    return o;
}

__device__ __forceinline__ uint32_t dm_get(unsigned long long lo, unsigned long long hi, int i)
{
    return (uint32_t)((i < 16 ? (lo >> (4 * i)) : (hi >> (4 * (i - 16)))) & 0xFull);
}
__device__ __forceinline__ void dm_set(unsigned long long &lo, unsigned long long &hi, int i,
                                       uint32_t code)
{
    if (i < 16) {
        lo = (lo & ~(0xFull << (4 * i))) | ((unsigned long long)code << (4 * i));
    } else {
        hi = (hi & ~(0xFull << (4 * (i - 16)))) | ((unsigned long long)code << (4 * (i - 16)));
    }
}


// findDistMod for one axis that may be periodic (src/contactsearch.cuh:12-74):
// wraps -1 -> num-1 (shift +L, code bit lo) and num -> 0 (shift -L, bit hi).
__device__ __forceinline__ void wrap_axis(int32_t &c, uint32_t num, uint32_t &code,
                                          uint32_t bit_lo, uint32_t bit_hi)
{
    if (c < 0) { c = (int32_t)(num - 1); code |= bit_lo; }
    if ((uint32_t)c == num) { c = 0; code |= bit_hi; }
}

// Slot state of one particle during contact detection.
struct TopoSlots {
    uint32_t occ;                    // occupied-slot mask
    uint32_t occ0;                   // the mask before this step's search
    uint32_t err;
    unsigned long long dm_lo, dm_hi; // periodic shift code of each slot
    int nc;                          // contacts found this step
    bool loaded;                     // row copied to shared memory
    bool dirty;                      // row changed
};

// Copies the partners of the particle's occupied slots to shared memory and
// its shift codes to registers (once); the other entries are neither
// searched nor written back.
template <int TB>
__device__ __forceinline__ void topo_load_row(const Dev &d, uint32_t *srow, int tid, uint32_t s,
                                              TopoSlots &ts)
{
    if (ts.loaded) return;
    if (ts.occ) {
        for (uint32_t m = ts.occ; m; m &= m - 1u) {
            const uint32_t i = (uint32_t)(__ffs(m) - 1);
            srow[i * TB + tid] = d.contacts[tile_at(s, i, NC)];
        }
        const ulonglong2 c2 = d.dmc[s];
        ts.dm_lo = c2.x;
        ts.dm_hi = c2.y;
    }
    ts.loaded = true;
}

// Whether candidate t already holds a slot of the (loaded) row through the
// periodic image `code`.
template <int TB>
__device__ __forceinline__ bool in_slot(const uint32_t *srow, int tid, const TopoSlots &ts,
                                        uint32_t t, uint32_t code)
{
    for (uint32_t m = ts.occ; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        if (srow[i * TB + tid] == t) return dm_get(ts.dm_lo, ts.dm_hi, i) == code;
    }
    return false;
}

// Overlapping candidate t (storage index) reached through a stencil cell
// with shift `code`: the slot choice.  Returns false once nc > NC, which ends
// the current cell (the reference returns from findContactsInCell).  Kept
// out of line: it runs for the few overlaps of a particle, and inlining it
// would raise the register count of the whole candidate loop.
template <int TB>
__device__ __noinline__ bool topo_insert(const Dev &d, uint32_t *srow, int tid, uint32_t s,
                                         uint32_t t, uint32_t code, TopoSlots &ts)
{
    topo_load_row<TB>(d, srow, tid, s, ts);
    // slot choice, src/contactsearch.cuh:252-271: a slot already holding t
    // wins, else the last empty slot, else position nc
    int cpos = -1;
    for (uint32_t m = ts.occ; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        if (srow[i * TB + tid] == t) { cpos = i; break; }
    }
    if (cpos >= 0) {
        // already in its slot: the reference writes the slot again, which
        // changes the row only where the partner is now seen through
        // another periodic image
        if (dm_get(ts.dm_lo, ts.dm_hi, cpos) != code) {
            dm_set(ts.dm_lo, ts.dm_hi, cpos, code);
            ts.dirty = true;
        }
    } else {
        const uint32_t empty = ~ts.occ;
        cpos = empty ? 31 - __clz(empty) : ts.nc;
        if (cpos < NC) {
            ts.occ |= 1u << cpos;
            srow[cpos * TB + tid] = t;
            dm_set(ts.dm_lo, ts.dm_hi, cpos, code);
            ts.dirty = true;
        } else {
            ts.err |= ST_NC_OVERFLOW;
        }
    }
    return ++ts.nc <= NC;
}

// The reference's overlap predicate, float_sqrt(dot) - (ra + rb) < 0, for
// candidate t through a stencil cell with shift `code`
// (src/contactsearch.cuh:233-248).
__device__ __forceinline__ bool overlaps(const Params &P, const double4 *xr, uint32_t t,
                                         uint32_t code, double4 xa)
{
    const double4 xb = xr[t];
    const d3 dm = decode_dm(code, P);
    const d3 xab = add(mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z), dm);
    const double delta = flen(xab) - (xa.w + xb.w);
    return delta < 0.0f;
}

// Contact model 1 processes each candidate as soon as it is found
// (findAndProcessContactsInCell, src/contactsearch.cuh:81-175): overlap ->
// contactLinearViscous, else a gap below db -> capillaryCohesion_exp.  Out of
// line, with every operand loaded here, so the candidate loop stays lean.
__device__ __noinline__ void visc_pair(const Dev &d, int A, uint32_t s, uint32_t t,
                                       uint32_t code, d3 &F, double &p)
{
    const Params &P = prm_of(d, s);
    const double4 xa = d.xr[A][s], xb = d.xr[A][t];
    const d3 dm = decode_dm(code, P);
    const d3 xab = add(mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z), dm);
    const double len = flen(xab);
    const double delta = len - (xa.w + xb.w);
    if (delta < 0.0f) {
        contact_viscous(P, F, p, ld4(d.vel[A], s), ld4(d.vel[A], t), xyz(ld4(d.angvel[A], s)),
                        xyz(ld4(d.angvel[A], t)), xa.w, xb.w, xab, len, delta);
    } else if (delta < P.db) {
        capillary_exp(P, F, xa.w, xb.w, delta, xab, len);
    }
}

// How far particle s and any partner can have closed their gap since s's list
// was recorded: its own displacement bound plus the largest of any particle,
// rounded up.  While that stays below the list's smallest gap (Dev::vl_gap)
// no listed candidate can overlap, and the list need not be tested.
__device__ __forceinline__ float moved_bound(const Dev &d, uint32_t s, const Verlet &V)
{
    return __fadd_ru(d.disp[s], __uint_as_float(V.dmax_bits));
}

// k_topo: one thread per particle s (storage order, which relayout keeps close
// to cell order); its cell-list position k = pos[s] locates it in the runs.
//
// List mode: while the particle's Verlet list is valid (no epoch restart, no
// cell of its neighbourhood changed members this step) only the listed
// candidates are tested, in their recorded order.  The list holds, in the
// reference's visiting order, every member of the stencil cells that was
// within ra + rb + skin when it was recorded; a pair missing from it is at
// least skin - 4 dmax > 0 apart now, so it cannot overlap.
//
// Sweep mode: the 27 stencil cells are scanned as in the reference (z, y, x;
// members by particle index) and the list is recorded on the way.
//
// VISC (contact model 1): no slots; every candidate within ra + rb + db is
// processed in visiting order and the contact force and pressure sums are
// left in Dev::c1acc for k_force_tiles.
// The contact search of one particle s whose list decision (k_topo) did not
// settle it: list_ok, its Verlet list is valid; held, Dev::settled[s].
template <bool VISC, bool BATCH, int TB>
__device__ __forceinline__ void topo_search(const Dev &d, int A, uint32_t s, int tid, uint32_t *srow,
                                            bool list_ok, bool held)
{
    const Params &P = prm_at<BATCH>(d, s);
    const uint32_t len = d.vl_len[s];
    // After a position left the grid (the step reports SPH_ERR_OUT_OF_GRID)
    // the scene has come apart: saturated cell ids pile its particles into
    // the edge cells, where the stencil sweep grows with the square of their
    // count.  The search stays off until an upload clears the status.  A
    // batch goes on, since its other scenes are still sound.  Tested only
    // here, past the list decision, so that the particles the decision
    // settles do not wait for the status word.
    // The slot mask and the position are loaded with the status word, so
    // the three wait out one memory latency together.
    const uint32_t occ_in = d.cmask[s];
    const double4 xa = d.xr[A][s];
    if (!BATCH && (*(volatile const uint32_t *)d.status & ST_OUT_OF_GRID)) return;
    const double ra = xa.w;
    const double4 *__restrict__ xr = d.xr[A];
    TopoSlots ts{occ_in, occ_in, 0u, 0ull, 0ull, 0, false, false};
    const uint32_t nx = P.num[0], ny = P.num[1], nz = P.num[2];
    int32_t gp[3];
    gp[0] = __double2int_rz(cell_floor(P, 0, xa.x));
    gp[1] = __double2int_rz(cell_floor(P, 1, xa.y));
    gp[2] = __double2int_rz(cell_floor(P, 2, xa.z));
    const bool gp_in = gp[0] >= 0 && (uint32_t)gp[0] < nx && gp[1] >= 0 && (uint32_t)gp[1] < ny &&
                       gp[2] >= 0 && (uint32_t)gp[2] < nz;
    const bool use_lists = P.skin > 0.0 && gp_in;
    d3 F1 = mk(0.0, 0.0, 0.0);   // model 1 sums
    double p1 = 0.0f;

    if (VISC && list_ok) {
        for (uint32_t e = 0; e < len; ++e) {
            const size_t at = vl_at(s, e);
            visc_pair(d, A, s, d.vl[at], vl_code(d.vl_meta[at]), F1, p1);
        }
    } else if (list_ok) {
        // the list is read four entries at a time, so that their loads are
        // in flight together
        // A candidate that already holds a slot through the same image needs
        // no test: overlapping or not, the reference's topology leaves its
        // slot as it is (a separated one is freed by the force pass).  The
        // test only feeds the count nc, which matters once a row fills up;
        // while the occupied slots plus the list length stay within NC, no
        // row can fill, so the filter changes nothing.
        const bool filter = ts.occ != 0u && len + (uint32_t)__popc(ts.occ) <= (uint32_t)NC;
        // A candidate whose own recorded gap exceeds the displacement bound
        // cannot overlap (nor hold a slot taken since the list was
        // recorded): its position is not fetched.  Skipping it leaves the
        // order of the others, and so the slot choice, unchanged.
        const float bound = moved_bound(d, s, *d.vs);
        uint32_t tv[4], mv[4];
        auto load4 = [&](uint32_t e0) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const size_t at = vl_at(s, min(e0 + (uint32_t)j, (uint32_t)len - 1u));
                tv[j] = d.vl[at];
                mv[j] = d.vl_meta[at];
            }
        };
        load4(0);   // the first four entries are in flight with the slot row
        if (filter) topo_load_row<TB>(d, srow, tid, s, ts);
        int skip_slot = -1;
        uint32_t found = 0;   // candidates found in their slots
        for (uint32_t e0 = 0; e0 < len; e0 += 4) {
            if (e0) load4(e0);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (e0 + (uint32_t)j >= len) break;
                const uint32_t meta = mv[j];
                const int slot = (int)(meta & 31u);
                if (slot == skip_slot) continue;   // nc > NC: rest of that cell
                const uint32_t t = tv[j], code = vl_code(meta);
                if (filter && in_slot<TB>(srow, tid, ts, t, code)) {
                    ++found;
                    continue;
                }
                if (vl_gap_of(meta) > bound) continue;
                if (overlaps(P, xr, t, code, xa) && !topo_insert<TB>(d, srow, tid, s, t, code, ts))
                    skip_slot = slot;
            }
        }
        // every candidate already held its slot: settled until a slot is
        // freed (k_contact) or the list is recorded again
        if (!VISC && filter && found == len && len != 0) d.settled[s] = 1;
    } else {
        if (held) d.settled[s] = 0;   // the list is recorded again
        const float4 *__restrict__ xs = d.xs[A];
        const uint32_t k = d.pos[s];
        const float4 xaf = xs[k];
        const float Lf0 = (float)P.L[0], Lf1 = (float)P.L[1];
        const float eps = P.cull_eps;
        const float skinf = (float)P.skin;
        const float extraf = (float)P.reach_extra;
        uint32_t nlist = 0;
        bool list_overflow = false;
        float gmin = 3.0e38f;   // smallest gap to a listed candidate, bounded below

        // A run [beg, end) of cell-list positions (one cell, or the three
        // cells of an x-row whose inner boundaries are bnd1 <= bnd2, stencil
        // slots slot0 .. slot0 + 2), culled four candidates at a time so the
        // four loads are in flight together; hits are handled in list order.
        auto scan_run = [&](uint32_t beg, uint32_t end, uint32_t code, uint32_t bnd1,
                            uint32_t bnd2, uint32_t slot0) {
            const float sx = (code & 1u) ? Lf0 : ((code & 2u) ? -Lf0 : 0.0f);
            const float sy = (code & 4u) ? Lf1 : ((code & 8u) ? -Lf1 : 0.0f);
            uint32_t base = beg;
            while (base < end) {
                const uint32_t last = end - 1;
                float4 c[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) c[j] = __ldg(&xs[min(base + (uint32_t)j, last)]);
                uint32_t near = 0, hit = 0;
                float gj[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float fx = (xaf.x - c[j].x) + sx;
                    const float fy = (xaf.y - c[j].y) + sy;
                    const float fz = xaf.z - c[j].z;
                    const float d2 = __fmaf_rn(fx, fx, __fmaf_rn(fy, fy, fz * fz));
                    const float rsum = VISC ? (xaf.w + c[j].w + extraf) : (xaf.w + c[j].w);
                    const float rr = rsum * 1.000004f + eps;
                    const float rs = (rsum + skinf) * 1.000004f + eps;
                    const uint32_t k2 = base + (uint32_t)j;
                    const bool ok = k2 < end && k2 != k;
                    if (ok && d2 < rs * rs) {
                        near |= 1u << j;
                        // the gap, with the cull's float slack taken against
                        // it (over every near candidate: at least the listed)
                        gj[j] = __fsub_rd(__fmul_rd(__fsqrt_rd(d2), 0.999996f), rr);
                        gmin = fminf(gmin, gj[j]);
                    }
                    if (ok && d2 < rr * rr) hit |= 1u << j;
                }
                uint32_t next = base + 4;
                while (near) {
                    const int j = __ffs(near) - 1;
                    near &= near - 1;
                    const uint32_t k2 = base + (uint32_t)j;
                    const uint32_t t = __ldg(&d.cellorder[k2]);
                    const uint32_t slot = slot0 + ((k2 < bnd1) ? 0u : ((k2 < bnd2) ? 1u : 2u));
                    if (!use_lists) {
                    } else if (nlist < VL_CAP) {
                        const size_t at = vl_at(s, nlist);
                        d.vl[at] = t;
                        d.vl_meta[at] = vl_meta_of(slot, code, gj[j]);
                        ++nlist;
                    } else {
                        list_overflow = true;
                    }
                    if (VISC) {
                        if ((hit >> j) & 1u) visc_pair(d, A, s, t, code, F1, p1);
                    } else if ((hit >> j) & 1u) {
                        if (overlaps(P, xr, t, code, xa) &&
                            !topo_insert<TB>(d, srow, tid, s, t, code, ts)) {
                            // nc > NC: skip the rest of this cell; the list
                            // would not describe the skipped part
                            next = (k2 < bnd1) ? bnd1 : ((k2 < bnd2) ? bnd2 : end);
                            near = 0;
                            list_overflow = true;
                        }
                    }
                }
                base = next;
            }
        };

        // Cell-level pruning: a stencil cell whose box lies farther from the
        // particle than ra + rmax + skin (plus the float slack of the
        // predicate) holds neither a contact nor a list candidate; skipping
        // it leaves the visiting order of the others unchanged.  Used only
        // while the particle's own cell is inside the grid and every
        // particle sits inside its cell's box (alias_any clear).
        const bool prune = gp_in && (*d.alias_any == 0u);
        float flo[3], fhi[3];
        {
            const double xc[3] = {xa.x, xa.y, xa.z};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const double lo = xc[q] - (P.origo[q] + (double)gp[q] * P.cellsize[q]);
                const double hi = (P.origo[q] + (double)(gp[q] + 1) * P.cellsize[q]) - xc[q];
                flo[q] = lo > 0.0 ? (float)(lo * lo) * 0.99999f : 0.0f;
                fhi[q] = hi > 0.0 ? (float)(hi * hi) * 0.99999f : 0.0f;
            }
        }
        const double extra = VISC ? P.reach_extra : 0.0;
        const float reach = (float)((ra + P.rmax + P.skin + extra) * (1.0 + 1e-5) + P.prune_pad);
        const float reach2 = prune ? reach * reach : 3.0e38f;

        for (int oz = -1; oz < 2; ++oz) {
            const int32_t cz = (int32_t)((uint32_t)gp[2] + (uint32_t)oz);
            if (cz < 0 || (uint32_t)cz == nz) continue;
            const float dz2 = oz < 0 ? flo[2] : (oz > 0 ? fhi[2] : 0.0f);
            if (dz2 > reach2) continue;
            for (int oy = -1; oy < 2; ++oy) {
                const float dyz2 = dz2 + (oy < 0 ? flo[1] : (oy > 0 ? fhi[1] : 0.0f));
                if (dyz2 > reach2) continue;
                int32_t cy = (int32_t)((uint32_t)gp[1] + (uint32_t)oy);
                uint32_t ycode = 0;
                if (P.periodic == 1) {
                    wrap_axis(cy, ny, ycode, 4u, 8u);
                } else if (cy < 0 || (uint32_t)cy == ny) {
                    continue;
                }
                const uint32_t rowbase = (uint32_t)cy * nx + (nx * ny) * (uint32_t)cz;
                const uint32_t slot0 = (uint32_t)((oz + 1) * 9 + (oy + 1) * 3);
                const int32_t c0 = gp[0] - 1;
                if (c0 >= 0 && (uint32_t)c0 + 2 < nx) {
                    // the three x cells are consecutive ids: one run of xs
                    const uint32_t cid0 = (uint32_t)c0 + rowbase;
                    if (cid0 + 2 >= P.ncells) { ts.err |= ST_OUT_OF_GRID; continue; }
                    const uint32_t g0 = cid0 + P.cell_base;
                    const uint32_t b0 = d.cell_start[g0], b1 = d.cell_start[g0 + 1];
                    const uint32_t b2 = d.cell_start[g0 + 2], b3 = d.cell_start[g0 + 3];
                    const uint32_t lo = (dyz2 + flo[0] <= reach2) ? b0 : b1;
                    const uint32_t hi = (dyz2 + fhi[0] <= reach2) ? b3 : b2;
                    scan_run(lo, hi, ycode, b1, b2, slot0);
                } else {
                    for (int ox = -1; ox < 2; ++ox) {
                        if (dyz2 + (ox < 0 ? flo[0] : (ox > 0 ? fhi[0] : 0.0f)) > reach2) continue;
                        int32_t cx = (int32_t)((uint32_t)gp[0] + (uint32_t)ox);
                        uint32_t code = ycode;
                        if (P.periodic == 1 || P.periodic == 2) {
                            wrap_axis(cx, nx, code, 1u, 2u);
                        } else if (cx < 0 || (uint32_t)cx == nx) {
                            continue;
                        }
                        const uint32_t cid = (uint32_t)cx + rowbase;
                        if (cid >= P.ncells) { ts.err |= ST_OUT_OF_GRID; continue; }
                        const uint32_t g = cid + P.cell_base;
                        const uint32_t e = d.cell_start[g + 1];
                        scan_run(d.cell_start[g], e, code, e, e, slot0 + (uint32_t)(ox + 1));
                    }
                }
            }
        }
        d.vl_len[s] = (use_lists && !list_overflow) ? (uint8_t)nlist : VL_NONE;
        if (use_lists) d.vl_gap[s] = gmin;
    }

    if (VISC) d.c1acc[s] = make_double4(F1.x, F1.y, F1.z, p1);
    if (ts.dirty) {
        // the search only fills empty slots (and may change a code): the
        // partners of the newly occupied slots are the entries to write;
        // an empty slot's entry is never read
        const uint32_t occ = ts.occ;
        for (uint32_t m = occ & ~ts.occ0; m; m &= m - 1u) {
            const uint32_t i = (uint32_t)(__ffs(m) - 1);
            d.contacts[tile_at(s, i, NC)] = srow[i * TB + tid];
        }
        d.cmask[s] = occ;
        d.dmc[s] = make_ulonglong2(ts.dm_lo, ts.dm_hi);
        if (occ) d.cflag[s >> 5] = 1;
    }
    if (ts.err) atomicOr(d.status, ts.err);
}

// Most particles whose list decision each lane of k_topo makes in one go.
constexpr uint32_t TOPO_SPAN_MAX = 4;

// k_topo: the contact search, one warp per span x 32 consecutive storage
// indices (storage order, which relayout keeps close to cell order), span
// <= TOPO_SPAN_MAX.  First every lane makes the list decision of its span
// particles (particle base + 32 j + lane), their loads in flight together;
// the particles it does not settle are then dealt to the warp's lanes in
// order, 32 at a time, each searched by topo_search.
//
// List mode: while the particle's Verlet list is valid (no epoch restart, no
// cell of its neighbourhood changed members this step) only the listed
// candidates are tested, in their recorded order.  The list holds, in the
// reference's visiting order, every member of the stencil cells that was
// within ra + rb + skin when it was recorded; a pair missing from it is at
// least skin - 4 dmax > 0 apart now, so it cannot overlap.
//
// Sweep mode: the 27 stencil cells are scanned as in the reference (z, y, x;
// members by particle index) and the list is recorded on the way.
//
// VISC (contact model 1): no slots; every candidate within ra + rb + db is
// processed in visiting order and the contact force and pressure sums are
// left in Dev::c1acc for k_force_tiles.
template <bool VISC, bool BATCH, int TB>
__global__ void __launch_bounds__(TB, TOPO_THREADS_PER_SM / TB)
k_topo(Dev d, int A, uint32_t span)
{
    constexpr uint32_t FULL = 0xffffffffu;
    __shared__ uint32_t srow[NC * TB];
    const uint32_t np = d.np_all;
    const int tid = threadIdx.x;
    const uint32_t lane = (uint32_t)tid & 31u;
    const uint32_t base = ((blockIdx.x * TB + (uint32_t)tid) >> 5) * (32u * span);
    if (blockIdx.x == 0 && tid == 0) {
        // the movers of the last step have been consumed by the rebuild
        d.vs->nmovers = 0u;
        d.vs->movers_overflow = 0u;
    }
    const Verlet &V = *d.vs;
    // bit j: particle base + 32 j + lane needs the search / has a valid
    // list / is marked settled
    uint32_t need = 0, lok = 0, hld = 0;
#pragma unroll
    for (uint32_t j = 0; j < TOPO_SPAN_MAX; ++j) {
        const uint32_t s = base + 32u * j + lane;
        if (j >= span) break;
        if (s >= np) continue;
        const Params &P = prm_at<BATCH>(d, s);
        // The list decision, from a few bytes: a valid list whose gap bound
        // rules out every contact ends the particle's work here.  Its
        // per-particle loads are unconditional so that they (and those of
        // the lane's other particles) are in flight together.
        const uint8_t len = d.vl_len[s];
        const uint8_t outs = d.outside[s];
        const float gap = d.vl_gap[s];
        const uint8_t held = VISC ? 0 : d.settled[s];
        const float bound = moved_bound(d, s, V);
        bool list_ok = P.skin > 0.0 && !V.all_rebuild && len != VL_NONE && outs == 0;
        if (list_ok && V.dirty_step == V.step) list_ok = d.dirty[d.cell[s]] != V.step;
        // A valid list whose candidates all hold their slots (Dev::settled) is
        // settled too: the reference's topology would find every overlap among
        // them (the list holds every possible one) already in its slot and
        // change nothing.
        if (list_ok && (gap > bound || held)) {
            if (VISC) d.c1acc[s] = make_double4(0.0, 0.0, 0.0, 0.0);
            continue;
        }
        need |= 1u << j;
        if (list_ok) lok |= 1u << j;
        if (held) hld |= 1u << j;
    }
    // the warp's particles that need the search, in (j, lane) order: the
    // k-th goes to lane k % 32 in round k / 32
    uint32_t m[TOPO_SPAN_MAX], ml[TOPO_SPAN_MAX], mh[TOPO_SPAN_MAX];
    uint32_t total = 0;
#pragma unroll
    for (uint32_t j = 0; j < TOPO_SPAN_MAX; ++j) {
        // need, lok and hld have no bit j >= span: those masks are zero
        m[j] = __ballot_sync(FULL, (need >> j) & 1u);
        ml[j] = __ballot_sync(FULL, (lok >> j) & 1u);
        mh[j] = __ballot_sync(FULL, (hld >> j) & 1u);
        total += (uint32_t)__popc(m[j]);
    }
    for (uint32_t k = lane; k < total; k += 32u) {
        uint32_t rem = k, sel = 0, selj = 0, sel_l = 0, sel_h = 0;
        bool got = false;
#pragma unroll
        for (uint32_t j = 0; j < TOPO_SPAN_MAX; ++j) {
            const uint32_t c = (uint32_t)__popc(m[j]);
            if (!got) {
                if (rem < c) {
                    sel = m[j];
                    sel_l = ml[j];
                    sel_h = mh[j];
                    selj = j;
                    got = true;
                } else {
                    rem -= c;
                }
            }
        }
        const uint32_t bit = __fns(sel, 0, (int)rem + 1);
        const uint32_t s = base + 32u * selj + bit;
        topo_search<VISC, BATCH, TB>(d, A, s, tid, srow, (sel_l >> bit) & 1u, (sel_h >> bit) & 1u);
    }
}

struct ForceArgs {
    Dev d;
    int a;              // read buffer (start of step); the kernel writes buffer 1-a
    int write_outputs;  // store force/torque/acc/angacc/edp of this step
    int tape_step;      // differentiable step: tape row to record, or -1
    ForceConsts fc;     // single-scene contexts: the scene's constants
};

// Where the force kernels read a particle's own start-of-step rows: global
// memory (GlobalRows) or a tile of rows staged in shared memory (TileRows).
struct GlobalRows {
    const Dev &d;
    int A;
    uint32_t s;
    __device__ double4 xr() const { return d.xr[A][s]; }
    __device__ double4 vel() const { return ld4(d.vel[A], s); }
    __device__ double4 angvel() const { return ld4(d.angvel[A], s); }
    __device__ P3 angpos() const { return d.angpos[s]; }
    __device__ P3 angvel0() const { return d.angvel0[s]; }
    __device__ P3 vel0() const { return d.vel0[s]; }
    __device__ double2 xysum() const { return d.xysum[s]; }
    __device__ uint32_t pos() const { return d.pos[s]; }
    __device__ float disp() const { return d.disp[s]; }
    __device__ uint32_t cell() const { return d.cell[s]; }
    __device__ uint8_t fixed() const { return d.fixed[s]; }
    __device__ uint8_t wtouch() const { return d.wtouch[s]; }
};

// Particles per tile of the tiled force kernel (one thread each), a multiple
// of 32; the per-particle arrays it stages are allocated in whole tiles.
#ifndef SPHK_FORCE_TILE
#define SPHK_FORCE_TILE 128
#endif
constexpr uint32_t FT_TILE = SPHK_FORCE_TILE;
static_assert(FT_TILE % 32 == 0 && ROW_PAD % FT_TILE == 0, "force tiles are whole warps of a padded array");
// Resident blocks per SM: two stages of a tile are ~45.5 KB of shared memory.
#ifndef SPHK_FORCE_TILE_BLOCKS
#define SPHK_FORCE_TILE_BLOCKS (512 / SPHK_FORCE_TILE)
#endif

// The start-of-step rows of FT_TILE consecutive particles, each array one
// bulk copy (every member a multiple of 16 bytes).
struct __align__(16) ForceTile {
    double4 xr[FT_TILE];
    P3 vel[FT_TILE], angvel[FT_TILE], angpos[FT_TILE], angvel0[FT_TILE], vel0[FT_TILE];
    double2 xysum[FT_TILE];
    uint32_t pos[FT_TILE], cell[FT_TILE];
    float disp[FT_TILE];
    uint8_t fixed[FT_TILE], wtouch[FT_TILE];
};
static_assert(sizeof(ForceTile) % 16 == 0 && (FT_TILE % 16) == 0, "bulk copies are multiples of 16 bytes");

struct TileRows {
    const ForceTile &T;
    uint32_t r;
    __device__ double4 xr() const { return T.xr[r]; }
    __device__ double4 vel() const
    {
        const P3 v = T.vel[r];
        return make_double4(v.x, v.y, v.z, 0.0);
    }
    __device__ double4 angvel() const
    {
        const P3 v = T.angvel[r];
        return make_double4(v.x, v.y, v.z, 0.0);
    }
    __device__ P3 angpos() const { return T.angpos[r]; }
    __device__ P3 angvel0() const { return T.angvel0[r]; }
    __device__ P3 vel0() const { return T.vel0[r]; }
    __device__ double2 xysum() const { return T.xysum[r]; }
    __device__ uint32_t pos() const { return T.pos[r]; }
    __device__ float disp() const { return T.disp[r]; }
    __device__ uint32_t cell() const { return T.cell[r]; }
    __device__ uint8_t fixed() const { return T.fixed[r]; }
    __device__ uint8_t wtouch() const { return T.wtouch[r]; }
};

// MODEL: the contact model (1, 2 or 3), a template argument so that each
// model's kernel carries only its own force law.
// DIFF: the differentiable step (contact model 2 in exact FP64 with
// per-particle friction, implicit walls only, no bonds), recording the tape
// row args.tape_step when it is >= 0.  Energy rates and pressure are not
// computed in this variant.
// Everything per particle after the slot sums (F, T, p, ev_dot, es_dot):
// the walls, the bonds, the energy sums, the half-step leapfrog, the
// displacement bound and the cell of the new position.  xa, vel_a and
// angvel_a4 are the particle's start-of-step rows of buffer A, R reads its
// other rows; the new state goes to buffer 1 - A.
// P: the particle's scene constants (Params, or a launch's ForceConsts);
// restart: this step starts a Verlet epoch (Verlet::all_rebuild).
template <bool BATCH, bool DIFF, class Rows, class PS>
__device__ __forceinline__ void particle_tail(const Dev &d, const PS &P, uint32_t s, int A,
                                              int write_outputs, bool restart, double4 xa,
                                              double4 vel_a, double4 angvel_a4, d3 F, d3 T,
                                              double p, double ev_dot, double es_dot,
                                              const Rows &R)
{
    const int B = 1 - A;
    const double ra = xa.w;
    uint32_t err = 0;
    // ---- walls, src/contactsearch.cuh:578-663 (defaults :416-427) ----------
    double w0f = 0.0;
    if constexpr (DIFF) {
        WallHits wh;
        implicit_walls(P, xa, wh);
        const dl::WallLaw wl{P.k_n, P.gamma_wn, P.gamma_wt, P.mu_ws, P.mu_wd};
        for (int k = 0; k < wh.count; ++k) {
            dl::V3 fw, tw;
            dl::wall_fwd(wl, ra, dl::v3(vel_a.x, vel_a.y, vel_a.z),
                         dl::v3(angvel_a4.x, angvel_a4.y, angvel_a4.z), wh.n[k], wh.delta[k], 0.0,
                         fw, tw);
            F = add(F, mk(fw.x, fw.y, fw.z));
            T = add(T, mk(tw.x, tw.y, tw.z));
        }
    } else {
        // the six wall gaps first, inline; a particle touching no wall
        // (nearly all) takes no call
        const uint32_t touch = wall_touch(P, *d.walls, xa);
        if (touch) {
            const WallSums ws = wall_forces(prm_at<BATCH>(d, s), *d.walls, touch, xa, vel_a,
                                            angvel_a4, F, T, p);
            F = ws.F;
            T = ws.T;
            p = ws.p;
            w0f = ws.w0f;
        }
    }

    // ---- bonds: per-bond contributions in bond order (bondsLinear's serial
    // scatter order, cohesion.cuh:220-226) ------------------------------------
    if (P.nb0 > 0) {
        const uint32_t u = d.uid[s];
        const uint32_t e0 = d.bond_ptr[u], e1 = d.bond_ptr[u + 1];
        for (uint32_t e = e0; e < e1; ++e) {
            const uint32_t ent = d.bond_list[e];
            const uint32_t b = ent >> 1;
            const uint32_t xu = d.bond_xu[b];
            if (xu == 0xffffffffu) continue;
            const double4 f = d.bond_f[b];
            const double4 tj = d.bond_t[b];
            if ((ent & 1u) == 0u) {
                if (xu != u) continue;
                F = mk(F.x + f.x, F.y + f.y, F.z + f.z);
                T = mk(T.x - tj.x, T.y - tj.y, T.z - tj.z);
            } else {
                F = mk(F.x - f.x, F.y - f.y, F.z - f.z);
                T = mk(T.x + tj.x, T.y + tj.y, T.z + tj.z);
            }
        }
    }

    const double dt = P.dt;
    // es += es_dot dt, ev += ev_dot dt; a zero rate adds +0.0, which leaves
    // the sums unchanged unless one is -0.0 (esv_skip clear)
    if (es_dot != 0.0 || ev_dot != 0.0 || !P.esv_skip) {
        const double2 e = d.esv[s];
        d.esv[s] = make_double2(e.x + es_dot * dt, e.y + ev_dot * dt);
    }
    // the outputs of the call's last step, each stored once it is final, so
    // that no sum stays live through the integration for them
    if (write_outputs) {
        d.force[s] = make_double4(F.x, F.y, F.z, 0.0f);
        d.edp[s] = make_double4(es_dot, ev_dot, p, 0.0);
    }
    if (P.nw > 0) {
        const uint8_t touched = R.wtouch();
        if (w0f != 0.0 || touched) {
            const uint32_t u = d.uid[s];
            d.wf_pp[u] = w0f;
            d.wf_flag[u / 256u] = 1;
            d.wtouch[s] = (w0f != 0.0) ? 1 : 0;
        }
    }

    // ---- integrate, src/integration.cuh:9-187 -------------------------------
    // The rotation and the translation are independent; each is finished and
    // stored before the other starts, so fewer values are live at once.
    // Every expression keeps the reference's operands and order.
    const double radius = xa.w;
    const double m = 4.0 / 3.0 * REF_PI * radius * radius * radius * P.rho;
    const bool fixed = R.fixed() != 0;   // fixvel > 0
    {
        P3 angpos = R.angpos(), angvel0 = R.angvel0();
        double4 angacc;
        angacc.x = T.x * 1.0 / (2.0 / 5.0 * m * radius * radius);
        angacc.y = T.y * 1.0 / (2.0 / 5.0 * m * radius * radius);
        angacc.z = T.z * 1.0 / (2.0 / 5.0 * m * radius * radius);
        angacc.w = 0.0;
        if (fixed) angacc = make_double4(0.0f, 0.0f, 0.0f, 0.0f);
        angvel0.x += angacc.x * dt;
        angvel0.y += angacc.y * dt;
        angvel0.z += angacc.z * dt;
        angpos.x += angvel0.x * dt;
        angpos.y += angvel0.y * dt;
        angpos.z += angvel0.z * dt;
        P3 angvel;
        angvel.x = angvel0.x + 0.5 * angacc.x * dt;
        angvel.y = angvel0.y + 0.5 * angacc.y * dt;
        angvel.z = angvel0.z + 0.5 * angacc.z * dt;
        d.angvel[B][s] = angvel;
        d.angvel0[s] = angvel0;
        d.angpos[s] = angpos;
        if (write_outputs) {
            d.torque[s] = make_double4(T.x, T.y, T.z, 0.0f);
            d.angacc[s] = angacc;
        }
    }
    double4 x = xa, vel = vel_a;
    P3 vel0 = R.vel0();
    double4 acc;
    acc.x = F.x / m;
    acc.y = F.y / m;
    acc.z = F.z / m;
    acc.w = 0.0;
    acc.x += P.g[0];
    acc.y += P.g[1];
    acc.z += P.g[2];
    if (fixed) {
        acc.x = 0.0;
        acc.y = 0.0;
        acc.z -= P.g[2];
    }
    if (write_outputs) d.acc[s] = acc;
    if (P.periodic == 1) {
        if (x.x < P.origo[0]) x.x += P.L[0];
        if (x.x > P.L[0]) x.x -= P.L[0];
        if (x.y < P.origo[1]) x.y += P.L[1];
        if (x.y > P.L[1]) x.y -= P.L[1];
    } else if (P.periodic == 2) {
        if (x.x < P.origo[0]) x.x += P.L[0];
        if (x.x > P.L[0]) x.x -= P.L[0];
    }
    vel0.x += acc.x * dt;
    vel0.y += acc.y * dt;
    vel0.z += acc.z * dt;
    x.x += vel0.x * dt;
    x.y += vel0.y * dt;
    x.z += vel0.z * dt;
    vel.x = vel0.x + 0.5 * acc.x * dt;
    vel.y = vel0.y + 0.5 * acc.y * dt;
    vel.z = vel0.z + 0.5 * acc.z * dt;
    double2 xys = make_double2(0.0f, 0.0f);
    xys.x += vel.x * dt;
    xys.y += vel.y * dt;
    {
        const double2 o = R.xysum();
        d.xysum[s] = make_double2(o.x + xys.x, o.y + xys.y);
    }
    d.xr[B][s] = x;
    d.vel[B][s] = p3of(vel);
    d.vel0[s] = vel0;
    // float copy for the next step's contact search, at this particle's
    // cell-list position (rewritten by the rebuild when the order changes)
    d.xs[B][R.pos()] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);

    // ---- displacement bound since the Verlet epoch started ----------------
    Verlet &V = *d.vs;
    if (P.skin > 0.0) {
        const double ix = vel0.x * dt, iy = vel0.y * dt, iz = vel0.z * dt;
        const float inc = __fadd_ru(__fmul_ru((float)sqrt(ix * ix + iy * iy + iz * iz), 1.0001f), 1e-15f);
        const float dnew = __fadd_ru(restart ? 0.0f : R.disp(), inc);
        d.disp[s] = dnew;
        const uint32_t bits = __reduce_max_sync(__activemask(), __float_as_uint(dnew));
        if ((threadIdx.x & 31u) == (uint32_t)(__ffs(__activemask()) - 1)) atomicMax(&V.dmax_bits, bits);
    }

    // ---- cell of the new position, for the next step's cell list -----------
    // a position that is not finite (NaN forces, contact model 3) is
    // outside the grid whatever its float-to-integer conversion gives
    uint32_t c;
    if (!grid_cell(P, x.x, x.y, x.z, c)) { err |= ST_OUT_OF_GRID; c = d.ncells_all; }
    else c += P.cell_base;
    d.outside[s] = cell_outside(P, x.x, x.y, x.z) ? 1 : 0;
    const uint32_t c_old = R.cell();
    if (c != c_old) {
        d.cell[s] = c;
        *d.rebuild = 1u;
        if (P.skin > 0.0) {
            const uint32_t m = atomicAdd(&V.nmovers, 1u);
            if (m < MOVER_CAP) d.movers[m] = make_uint2(c_old, c);
            else V.movers_overflow = 1u;
        }
    }
    if (err) atomicOr(d.status, err);
}

// Everything of one particle s after the contact search, outside the
// differentiable step: its slot sums (k_contact's, or k_topo's for model 1)
// and particle_tail.  f: the chunk flag of s (Dev::cflag[s / 32], read by
// the caller ahead of the rows); restart: Verlet::all_rebuild.
template <int MODEL, bool BATCH, class Rows>
__device__ __forceinline__ void force_row(const ForceArgs &args, uint32_t s, const Rows &R,
                                          uint8_t f, bool restart)
{
    const Dev &d = args.d;
    // A chunk k_contact visited (flag 2: a contact remains, 3: none does)
    // has the slot sums of its particles in Dev::csum_*; its flag goes back
    // to 1 or 0 for the next step's search.  A warp is one chunk, so the
    // flag is the warp's.
    bool visited = false;
    if constexpr (MODEL != 1) {
        visited = f >= 2;
        if (visited) {
            __syncwarp(__activemask());
            if ((s & 31u) == 0) d.cflag[s >> 5] = (f == 2) ? 1 : 0;
        }
    }
    const double4 xa = R.xr();
    const double4 vel_a = R.vel();
    const double4 angvel_a4 = R.angvel();
    d3 F = mk(0.0, 0.0, 0.0), T = mk(0.0, 0.0, 0.0);
    double es_dot = 0.0f, ev_dot = 0.0f, p = 0.0f;
    if (MODEL == 1) {
        const double4 c = d.c1acc[s];
        F = mk(c.x, c.y, c.z);
        p = c.w;
    } else if (visited && d.cmask[s] != 0u) {
        // the sums of a particle that still holds a slot (with every slot
        // freed nothing was added: the sums are zero)
        const double4 cf = d.csum_f[s], ct = d.csum_t[s];
        F = mk(cf.x, cf.y, cf.z);
        p = cf.w;
        T = mk(ct.x, ct.y, ct.z);
        ev_dot = ct.w;
        es_dot = d.csum_es[s];
    }
    if constexpr (BATCH)
        particle_tail<true, false>(d, prm_at<true>(d, s), s, args.a, args.write_outputs, restart, xa,
                                   vel_a, angvel_a4, F, T, p, ev_dot, es_dot, R);
    else
        particle_tail<false, false>(d, args.fc, s, args.a, args.write_outputs, restart, xa, vel_a,
                                    angvel_a4, F, T, p, ev_dot, es_dot, R);
}

// The differentiable step's force kernel: one thread per particle, rows
// read from global memory, its own slot laws (contact model 2 in exact FP64
// with per-particle friction), recording the tape.
__global__ void __launch_bounds__(FORCE_BLOCK, SPHK_FORCE_MIN_BLOCKS)
k_force_diff(ForceArgs args)
{
    const Dev &d = args.d;
    const uint32_t np = d.np_all;
    const uint32_t s = blockIdx.x * FORCE_BLOCK + threadIdx.x;
    if (s >= np) return;
#ifndef SPHK_NO_PREFETCH
    // The state the integration reads comes after the contact work and
    // after stores the compiler may not move loads across, so each of its
    // loads would wait out a full DRAM latency in turn.  Lane 0 of every
    // warp whose 32 rows all exist asks for the warp's rows of it up front.
    if ((threadIdx.x & 31u) == 0 && s + 32 <= np) {
        bulk_prefetch_l2(d.angpos + s, 32 * sizeof(P3));
        bulk_prefetch_l2(d.angvel0 + s, 32 * sizeof(P3));
        bulk_prefetch_l2(d.vel0 + s, 32 * sizeof(P3));
        bulk_prefetch_l2(d.xysum + s, 32 * sizeof(double2));
        bulk_prefetch_l2(d.pos + s, 32 * sizeof(uint32_t));
        bulk_prefetch_l2(d.disp + s, 32 * sizeof(float));
        bulk_prefetch_l2(d.cell + s, 32 * sizeof(uint32_t));
        bulk_prefetch_l2(d.fixed + s, 32);
        bulk_prefetch_l2(d.wtouch + s, 32);
    }
#endif
    const GlobalRows R{d, args.a, s};
    const bool restart = d.vs->all_rebuild != 0u;
    {
        const Params &P = *d.prm;
        const int A = args.a;
        const double4 xa = d.xr[A][s];
        const double ra = xa.w;
        const double4 vel_a = ld4(d.vel[A], s);
        const double4 angvel_a4 = ld4(d.angvel[A], s);
        d3 F = mk(0.0, 0.0, 0.0), T = mk(0.0, 0.0, 0.0);
        double es_dot = 0.0f, ev_dot = 0.0f, p = 0.0f;
        // ---- interact: occupied slots in slot order ----------------------
        uint32_t occ = d.cmask[s];
        const int j = args.tape_step;
        const size_t row = (j >= 0) ? ((size_t)j * np + s) : 0;
        uint32_t lawmask = 0;
        const ulonglong2 dmw = d.dmc[s];
        const uint32_t occ0 = occ;
        for (uint32_t m = occ0; m; m &= m - 1) {
            const int i = __ffs(m) - 1;
            const size_t at = tile_at(s, (uint32_t)i, NC);
            const uint32_t t = d.contacts[at];
            const d3 dm = decode_dm(dm_get(dmw.x, dmw.y, i), P);
            const double4 xb = d.xr[A][t];
            dl::PairIn in;
            in.xab = dl::v3(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            in.ra = ra;
            in.rb = xb.w;
            if (dl::len(in.xab) - (ra + xb.w) < 0.0) {
                const P3 d0p = d.delta_t[at];
                const double4 vb = ld4(d.vel[A], t), wb = ld4(d.angvel[A], t);
                const double4 d0 = make_double4(d0p.x, d0p.y, d0p.z, 0.0);
                in.va = dl::v3(vel_a.x, vel_a.y, vel_a.z);
                in.vb = dl::v3(vb.x, vb.y, vb.z);
                in.wa = dl::v3(angvel_a4.x, angvel_a4.y, angvel_a4.z);
                in.wb = dl::v3(wb.x, wb.y, wb.z);
                in.d0u = dl::v3(d0.x, d0.y, d0.z);
                const dl::Law law{P.k_n, P.k_t, P.gamma_n, P.gamma_t,
                                  0.5 * (d.mu_p[s] + d.mu_p[t]), P.kappa, P.dt};
                dl::PairOut o;
                dl::pair_fwd(law, in, o);
                F = add(F, mk(o.F.x, o.F.y, o.F.z));
                T = add(T, mk(o.T.x, o.T.y, o.T.z));
                d.delta_t[at] = P3{o.dtn.x, o.dtn.y, o.dtn.z};
                lawmask |= 1u << i;
                if (j >= 0) {
                    const size_t ts = tape_slot_at((uint32_t)j, np, s, (uint32_t)i);
                    d.tp_partner[ts] = t;
                    d.tp_dt0[ts] = d0p;
                }
            } else {
                occ &= ~(1u << i);
                d.contacts[at] = np;
                d.delta_t[at] = P3{0.0, 0.0, 0.0};
            }
        }
        if (occ != occ0) {
            d.cmask[s] = occ;
            d.settled[s] = 0;   // a listed candidate left its slot
        }
        if (j >= 0) {
            d.tp_x[row] = xa;
            d.tp_v[row] = make_double4(vel_a.x, vel_a.y, vel_a.z, d.fixed[s] ? 1.0 : 0.0);
            d.tp_w[row] = angvel_a4;
            d.tp_mask[row] = lawmask;
            d.tp_dmc[row] = dmw;
        }
        particle_tail<false, true>(d, P, s, A, args.write_outputs, restart, xa, vel_a, angvel_a4, F,
                                   T, p, ev_dot, es_dot, R);
    }
}

// Issues the bulk copies of tile t's rows into T, completing on `bar`.
__device__ __forceinline__ void stage_force_tile(const Dev &d, int A, uint32_t t, ForceTile &T,
                                                 uint64_t *bar)
{
    const size_t s0 = (size_t)t * FT_TILE;
    mbar_expect_tx(bar, (uint32_t)sizeof(ForceTile));
    bulk_load(T.xr, d.xr[A] + s0, sizeof(T.xr), bar);
    bulk_load(T.vel, d.vel[A] + s0, sizeof(T.vel), bar);
    bulk_load(T.angvel, d.angvel[A] + s0, sizeof(T.angvel), bar);
    bulk_load(T.angpos, d.angpos + s0, sizeof(T.angpos), bar);
    bulk_load(T.angvel0, d.angvel0 + s0, sizeof(T.angvel0), bar);
    bulk_load(T.vel0, d.vel0 + s0, sizeof(T.vel0), bar);
    bulk_load(T.xysum, d.xysum + s0, sizeof(T.xysum), bar);
    bulk_load(T.pos, d.pos + s0, sizeof(T.pos), bar);
    bulk_load(T.cell, d.cell + s0, sizeof(T.cell), bar);
    bulk_load(T.disp, d.disp + s0, sizeof(T.disp), bar);
    bulk_load(T.fixed, d.fixed + s0, sizeof(T.fixed), bar);
    bulk_load(T.wtouch, d.wtouch + s0, sizeof(T.wtouch), bar);
}

// Shared-memory stages of k_force_tiles: tiles a block has in flight.
#ifndef SPHK_FORCE_STAGES
#define SPHK_FORCE_STAGES 2
#endif
constexpr uint32_t FT_STAGES = SPHK_FORCE_STAGES;

// k_force_tiles: force_row over tiles of FT_TILE particles, a resident grid
// of blocks (one thread per particle of a tile), each taking tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...  The particle's own rows (372 of
// the 372 + 189 bytes a particle moves) arrive by bulk copies into a ring of
// FT_STAGES shared-memory stages: while a block integrates one tile, the
// copy engine fetches its next ones, so the bytes in flight do not depend on
// how many threads are resident.  A stage is refilled, FT_STAGES tiles
// ahead, once the block's barrier shows its tile consumed.  The
// per-particle arrays are allocated in whole tiles (ROW_PAD), so every copy
// is a whole tile.  A copy that has not landed after BULK_WAIT_NS stops the
// block with ST_TIMEOUT, after the copies it issued have landed.
template <int MODEL, bool BATCH>
__global__ void __launch_bounds__(FT_TILE, SPHK_FORCE_TILE_BLOCKS)
k_force_tiles(ForceArgs args)
{
    __shared__ ForceTile tiles[FT_STAGES];
    __shared__ uint64_t full[FT_STAGES];
    const Dev &d = args.d;
    const uint32_t np = d.np_all;
    const uint32_t ntiles = (np + FT_TILE - 1) / FT_TILE;
    const uint32_t tid = threadIdx.x;
    const int A = args.a;
    if (tid == 0) {
        for (uint32_t k = 0; k < FT_STAGES; ++k) mbar_init(&full[k], 1);
        mbar_init_fence();
        // the block's first FT_STAGES tiles
        for (uint32_t k = 0; k < FT_STAGES; ++k) {
            const uint32_t tk = blockIdx.x + k * gridDim.x;
            if (tk < ntiles) stage_force_tile(d, A, tk, tiles[k], &full[k]);
        }
    }
    __syncthreads();
    const bool restart = d.vs->all_rebuild != 0u;
    uint32_t t = blockIdx.x;
    for (uint32_t it = 0; t < ntiles; t += gridDim.x, ++it) {
        const uint32_t k = it % FT_STAGES;
        const uint32_t s = t * FT_TILE + tid;
        // the chunk flag comes from global memory: asked for before the wait
        const uint8_t f = (MODEL != 1 && s < np) ? d.cflag[s >> 5] : (uint8_t)0;
        const bool ready = mbar_wait(&full[k], (it / FT_STAGES) & 1u, BULK_WAIT_NS);
        if (ready && s < np) force_row<MODEL, BATCH>(args, s, TileRows{tiles[k], tid}, f, restart);
        if (__syncthreads_or(!ready)) {
            if (tid == 0) {
                atomicOr(d.status, ST_TIMEOUT);
                // this tile's copies and those issued for the next ones land
                // before the block leaves
                for (uint32_t q = 0; q < FT_STAGES; ++q) {
                    const uint32_t iq = it + q;
                    if (t + q * gridDim.x < ntiles)
                        mbar_wait(&full[iq % FT_STAGES], (iq / FT_STAGES) & 1u, BULK_WAIT_NS);
                }
            }
            return;
        }
        // every thread is past its reads of stage k: it takes the tile
        // FT_STAGES rounds ahead
        const uint32_t tn = t + FT_STAGES * gridDim.x;
        if (tid == 0 && tn < ntiles) {
            fence_proxy_async_smem();
            stage_force_tile(d, A, tn, tiles[k], &full[k]);
        }
    }
}

struct ContactArgs {
    Dev d;
    int a;               // read buffer (start of step)
    int write_outputs;   // store force/torque/acc/angacc/edp of this step
    LawParams lp;        // single-scene contexts; a batch reads each scene's Params
};

// Contacts of one chunk whose law terms a warp holds at once (a multiple of 32).
#ifndef SPHK_CONTACT_CAP
#define SPHK_CONTACT_CAP 64
#endif
constexpr uint32_t CT_CAP = SPHK_CONTACT_CAP;

// k_contact: interact's slot loop (src/contactsearch.cuh:468-543) for
// contact models 2 and 3, one lane per directed contact.
//
// The unit of work is a chunk of 32 consecutive storage indices, and a chunk
// is visited only while its flag (Dev::cflag) says it may hold a contact:
// the contact search sets the flag when it writes a row with an occupied
// slot, and this kernel clears it when the chunk ends without one.  The grid
// is resident (a few blocks per SM); warp g takes chunks g, g + W, g + 2W,
// ... of the W warps, reading the flags of 32 of them in one load, so a
// contact-free scene costs about one memory latency.
//
// In a chunk, the occupied slots form a list of directed contacts, written
// once into shared memory as (lane, slot) pairs in slot-major order.  The
// list is evaluated 32 contacts at a time, one per lane, so every lane runs
// a force law whatever the spread of contact counts, and the terms of up to
// CT_CAP contacts are kept in shared memory.  Then every particle's own lane
// adds its terms in slot order, the reference's summation order, all lanes
// at once, and at the end stores the sums for k_force_tiles.  A slot whose partner
// no longer overlaps is freed and its history zeroed, as in the reference.
// A chunk's rows are contiguous, its slot tiles too, and a round's lanes
// mostly read one slot of consecutive particles, so their loads coalesce.
template <int MODEL, bool BATCH, int CB>
__global__ void __launch_bounds__(CB, CONTACT_THREADS_PER_SM / CB)
k_contact(ContactArgs args)
{
    constexpr uint32_t FULL = 0xffffffffu;
    constexpr int WARPS = CB / 32;
    // per warp: the law terms of the contacts held (F xyz, T xyz, p, ev_dot,
    // es_dot), the chunk's list of (lane | slot << 5), and which held
    // contacts overlapped (hits) and slipped
    __shared__ double terms[WARPS][9][CT_CAP];
    __shared__ uint16_t expand[WARPS][32 * NC];
    __shared__ uint32_t hitw[WARPS][CT_CAP / 32], slipw[WARPS][CT_CAP / 32];
    __shared__ double sums[WARPS][9][32];   // each particle's running sums
    __shared__ uint16_t sbase[WARPS][NC];    // first list entry of each slot
    __shared__ uint32_t smask[WARPS][NC];    // the particles holding each slot
    const Dev &d = args.d;
    const int A = args.a;
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t np = d.np_all;
    const uint32_t nchunk = (np + 31u) >> 5;
    const uint32_t gw = blockIdx.x * WARPS + w, nwarps = gridDim.x * WARPS;
    double (*tm)[CT_CAP] = terms[w];
    double (*sm)[32] = sums[w];
    uint16_t *ex = expand[w];
    // A chunk's rows are contiguous (its slot tiles too), so one lane asks
    // the copy engine to bring a chunk that is coming up into L2 while the
    // warp works: the chain of loads of each round then waits on L2, not on
    // DRAM.  Only whole chunks, so that no request passes an array's end.
    auto prefetch_chunk = [&](uint32_t ch) {
        const uint32_t b = ch << 5;
        if (lane != 0 || b + 32u > np) return;
        bulk_prefetch_l2(d.cmask + b, 32 * sizeof(uint32_t));
        bulk_prefetch_l2(d.dmc + b, 32 * sizeof(ulonglong2));
        bulk_prefetch_l2(d.xr[A] + b, 32 * sizeof(double4));
        bulk_prefetch_l2(d.vel[A] + b, 32 * sizeof(P3));
        bulk_prefetch_l2(d.angvel[A] + b, 32 * sizeof(P3));
        bulk_prefetch_l2(d.contacts + tile_at(b, NC - PF_SLOTS, NC), PF_SLOTS * 32 * sizeof(uint32_t));
        bulk_prefetch_l2(d.delta_t + tile_at(b, NC - PF_SLOTS, NC), PF_SLOTS * 32 * sizeof(P3));
    };

    for (uint32_t g = gw; g < nchunk; g += 32u * nwarps) {
        // the flags of this warp's next 32 chunks: g, g + W, ..., one a lane
        const uint32_t mine = g + lane * nwarps;
        uint32_t todo = __ballot_sync(FULL, mine < nchunk && d.cflag[mine] != 0);
        if (todo) prefetch_chunk(g + (uint32_t)(__ffs(todo) - 1) * nwarps);
        while (todo) {
            const uint32_t chunk = g + (uint32_t)(__ffs(todo) - 1) * nwarps;
            todo &= todo - 1u;
            if (todo) prefetch_chunk(g + (uint32_t)(__ffs(todo) - 1) * nwarps);
            const uint32_t s0 = chunk << 5;
            const uint32_t s = s0 + lane;
            const uint32_t occ0 = (s < np) ? d.cmask[s] : 0u;
            const uint32_t n = __popc(occ0);
            const uint32_t total = __reduce_add_sync(FULL, n);   // the chunk's contacts
            // The list in slot-major order: slot by slot, and within a slot
            // by particle.  The lanes of a round then mostly share a slot and
            // touch consecutive particles: consecutive entries of the slot
            // tiles and consecutive particle rows.  A particle's contacts stay
            // in ascending slot order along the list; slot i's first entry is
            // sbase[i], and a particle finds its own entry of slot i from
            // smask[i], the particles holding it.
            {
                const uint32_t lt = (1u << lane) - 1u;
                uint32_t k = 0;
                for (uint32_t u = __reduce_or_sync(FULL, occ0); u; u &= u - 1u) {
                    const uint32_t i = (uint32_t)(__ffs(u) - 1);
                    const uint32_t m = __ballot_sync(FULL, (occ0 >> i) & 1u);
                    if ((occ0 >> i) & 1u) ex[k + __popc(m & lt)] = (uint16_t)(lane | (i << 5));
                    if (lane == 0) {
                        sbase[w][i] = (uint16_t)k;
                        smask[w][i] = m;
                    }
                    k += __popc(m);
                }
            }
            __syncwarp();

            // the particle's running sums live in shared memory between the
            // passes, so no register holds them while the laws run
            if (n) {
#pragma unroll
                for (int f = 0; f < 9; ++f) sm[f][lane] = 0.0;
            }
            uint32_t occ = occ0;   // slots still held after this step
            uint32_t rem = occ0;   // slots whose terms are still to be added
            // the partner of this lane's contact, loaded a round ahead
            uint32_t t_next = 0;
            if (lane < total) {
                const uint32_t x = ex[lane];
                t_next = d.contacts[tile_at(s0 + (x & 31u), x >> 5, NC)];
            }
            for (uint32_t base = 0; base < total; base += 32u) {
                const uint32_t c = base + lane;
                const uint32_t t = t_next;
                if (c + 32u < total) {
                    const uint32_t x = ex[c + 32u];
                    t_next = d.contacts[tile_at(s0 + (x & 31u), x >> 5, NC)];
                }
                const uint32_t pb = base - base % CT_CAP;   // first contact of this pass
                bool hit = false, slip = false;
                if (c < total) {
                    const uint32_t x = ex[c];
                    const uint32_t sq = s0 + (x & 31u), i = x >> 5;
                    const size_t e = tile_at(sq, i, NC);
                    const ulonglong2 dmw = d.dmc[sq];
                    const P3 dtp = d.delta_t[e];
                    const double4 dt0 = make_double4(dtp.x, dtp.y, dtp.z, 0.0);
                    const double4 xa = d.xr[A][sq];
                    const double4 vel_a = ld4(d.vel[A], sq);
                    const d3 angvel_a = xyz(ld4(d.angvel[A], sq));
                    const double4 xb = d.xr[A][t];
                    const double4 vel_b = ld4(d.vel[A], t), angvel_b = ld4(d.angvel[A], t);
                    LawOut o;
                    bool touch;
                    auto eval = [&](const auto &P) {
                        const d3 dm = decode_dm(dm_get(dmw.x, dmw.y, (int)i), P);
                        const double ra = xa.w, rb = xb.w;
                        const d3 xab = mk(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y,
                                          xa.z - xb.z + dm.z);
                        const double xlen = flen(xab);
                        const double delta_n = xlen - (ra + rb);
                        touch = delta_n < 0.0f;
                        if (touch) {
                            o = (MODEL == 2)
                                ? contact_linear(P, vel_a, angvel_a, vel_b, angvel_b, ra, rb, xab,
                                                 xlen, delta_n, dt0)
                                : contact_hertz(P, vel_a, angvel_a, vel_b, angvel_b, ra, rb, xab,
                                                xlen, delta_n, dt0);
                        }
                    };
                    if constexpr (BATCH) eval(prm_at<true>(d, sq));
                    else eval(args.lp);
                    if (touch) {
                        const uint32_t k = c - pb;
                        d.delta_t[e] = P3{o.dt4.x, o.dt4.y, o.dt4.z};
                        tm[0][k] = o.f.x;
                        tm[1][k] = o.f.y;
                        tm[2][k] = o.f.z;
                        tm[3][k] = o.t.x;
                        tm[4][k] = o.t.y;
                        tm[5][k] = o.t.z;
                        tm[6][k] = o.pr;
                        tm[7][k] = o.ev;
                        tm[8][k] = o.es;
                        hit = true;
                        slip = o.es_set;
                    } else {
                        // separated: free the slot and zero its history
                        d.contacts[e] = np;
                        d.delta_t[e] = P3{0.0, 0.0, 0.0};
                    }
                }
                const uint32_t hb = __ballot_sync(FULL, hit);
                const uint32_t sb = __ballot_sync(FULL, slip);
                if (lane == 0) {
                    hitw[w][(base - pb) >> 5] = hb;
                    slipw[w][(base - pb) >> 5] = sb;
                }
                const uint32_t pe = min(total, pb + CT_CAP);
                if (base + 32u < pe) continue;
                __syncwarp();
                // the pass is complete: every particle adds its terms of the
                // pass, in slot order
                const uint32_t lt = (1u << lane) - 1u;
                auto entry = [&](uint32_t i) { return (uint32_t)sbase[w][i] + __popc(smask[w][i] & lt); };
                if (rem && entry((uint32_t)(__ffs(rem) - 1)) < pe) {
                    d3 F = mk(sm[0][lane], sm[1][lane], sm[2][lane]);
                    d3 T = mk(sm[3][lane], sm[4][lane], sm[5][lane]);
                    double p = sm[6][lane], ev_dot = sm[7][lane], es_dot = sm[8][lane];
                    while (rem) {
                        const uint32_t i = (uint32_t)(__ffs(rem) - 1);
                        const uint32_t j = entry(i);
                        if (j >= pe) break;   // in a later pass
                        const uint32_t k = j - pb;
                        rem &= rem - 1u;
                        if ((hitw[w][k >> 5] >> (k & 31u)) & 1u) {
                            F = add(F, mk(tm[0][k], tm[1][k], tm[2][k]));
                            T = add(T, mk(tm[3][k], tm[4][k], tm[5][k]));
                            p += tm[6][k];
                            ev_dot += tm[7][k];
                            if ((slipw[w][k >> 5] >> (k & 31u)) & 1u) es_dot += tm[8][k];
                        } else {
                            occ &= ~(1u << i);
                        }
                    }
                    sm[0][lane] = F.x;
                    sm[1][lane] = F.y;
                    sm[2][lane] = F.z;
                    sm[3][lane] = T.x;
                    sm[4][lane] = T.y;
                    sm[5][lane] = T.z;
                    sm[6][lane] = p;
                    sm[7][lane] = ev_dot;
                    sm[8][lane] = es_dot;
                }
                __syncwarp();
            }
            if (n) {
                d.csum_f[s] = make_double4(sm[0][lane], sm[1][lane], sm[2][lane], sm[6][lane]);
                d.csum_t[s] = make_double4(sm[3][lane], sm[4][lane], sm[5][lane], sm[7][lane]);
                d.csum_es[s] = sm[8][lane];
                if (occ != occ0) {
                    d.cmask[s] = occ;
                    d.settled[s] = 0;   // a listed candidate left its slot
                }
            }
            // visited (2: a slot is still held, 3: none is); k_force_tiles reads
            // the sums of a visited chunk and sets its flag back to 1 or 0
            // for the next step's search
            const bool held = __any_sync(FULL, occ != 0u);
            if (lane == 0) d.cflag[chunk] = held ? 2 : 3;
        }
    }
}

// A resident grid of k_contact: the SMs times the blocks of this
// instantiation that fit on one (looked up once per instantiation).
template <int MODEL, bool BATCH, int CB>
static unsigned contact_grid(uint32_t np)
{
    static int resident = 0;
    if (resident == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contact<MODEL, BATCH, CB>, CB, 0);
        resident = std::max(1, sms) * std::max(1, per_sm);
    }
    const uint64_t chunks = div_up(np, 32);
    return (unsigned)std::min<uint64_t>((uint64_t)resident, div_up(chunks, CB / 32));
}

// Particles per lane of k_topo's list decisions: 4 once the scene is four
// times the threads the device holds at once (one decision round then
// hides the latency of four), 2 from twice, else 1, so that a smaller
// scene's searches run on as many lanes as it has particles.
static uint32_t topo_span(uint32_t np)
{
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (nsm < 1) nsm = 1;
    }
    const uint64_t resident = (uint64_t)nsm * TOPO_THREADS_PER_SM;
    return (uint64_t)np >= 4 * resident ? 4u : ((uint64_t)np >= 2 * resident ? 2u : 1u);
}

template <int TB>
static void launch_topo_as(const Dev &d, uint32_t np, bool visc, int a, cudaStream_t st)
{
    // one warp per span x 32 particles
    const uint32_t span = d.topo_span ? d.topo_span : topo_span(np);
    const unsigned grid = div_up(div_up(np, 32u * span), (uint32_t)TB / 32u);
    if (d.inst)   // batched contexts: contact model 2 only
        k_topo<false, true, TB><<<grid, TB, 0, st>>>(d, a, span);
    else if (visc)
        k_topo<true, false, TB><<<grid, TB, 0, st>>>(d, a, span);
    else
        k_topo<false, false, TB><<<grid, TB, 0, st>>>(d, a, span);
}

template <int CB>
static void launch_contact_as(const ContactArgs &args, uint32_t np, int model, cudaStream_t st)
{
    if (args.d.inst)   // batched contexts: contact model 2 only
        k_contact<2, true, CB><<<contact_grid<2, true, CB>(np), CB, 0, st>>>(args);
    else if (model == 3)
        k_contact<3, false, CB><<<contact_grid<3, false, CB>(np), CB, 0, st>>>(args);
    else
        k_contact<2, false, CB><<<contact_grid<2, false, CB>(np), CB, 0, st>>>(args);
}

void launch_topo(const Dev &d, uint32_t np, bool visc, int a, cudaStream_t st)
{
    if (d.shape) launch_topo_as<topo_block(1)>(d, np, visc, a, st);
    else launch_topo_as<topo_block(0)>(d, np, visc, a, st);
}

// Blocks of k_force_tiles: as many as fit on the device at once, no more
// than there are tiles.
template <int MODEL, bool BATCH>
static void launch_force_tiles(const ForceArgs &args, uint32_t np, cudaStream_t st)
{
    static int per_sm = 0, nsm = 0;
    if (per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_force_tiles<MODEL, BATCH>, FT_TILE, 0);
        if (per_sm < 1) per_sm = 1;
    }
    const uint32_t ntiles = div_up(np, FT_TILE);
    const uint32_t grid = std::min<uint32_t>(ntiles, (uint32_t)(per_sm * nsm));
    if (grid) k_force_tiles<MODEL, BATCH><<<grid, FT_TILE, 0, st>>>(args);
}

void launch_force(const Dev &d, const Params &hp, uint32_t np, int model, int a, int write_outputs,
                  cudaStream_t st)
{
    ForceArgs args{d, a, write_outputs, -1, force_consts(hp)};
    if (d.inst) {   // batched contexts: contact model 2 only
        launch_force_tiles<2, true>(args, np, st);
    } else if (d.mu_p) {   // the differentiable step
        k_force_diff<<<div_up(np, FORCE_BLOCK), FORCE_BLOCK, 0, st>>>(args);
    } else if (model == 1) {
        launch_force_tiles<1, false>(args, np, st);
    } else if (model == 3) {
        launch_force_tiles<3, false>(args, np, st);
    } else {
        launch_force_tiles<2, false>(args, np, st);
    }
}

// The differentiable step, recording tape row `tape_step`.
void launch_force_tape(const Dev &d, uint32_t np, int a, int tape_step, cudaStream_t st)
{
    ForceArgs args{d, a, 0, tape_step, ForceConsts{}};
    k_force_diff<<<div_up(np, FORCE_BLOCK), FORCE_BLOCK, 0, st>>>(args);
}

// The slot forces of contact models 2 and 3; model 1 has no slots (k_topo
// sums its forces) and the differentiable step evaluates its own law in
// k_force_diff, recording the tape.
void launch_contact(const Dev &d, const Params &hp, uint32_t np, int model, int a,
                    int write_outputs, cudaStream_t st)
{
    if (model == 1 || d.mu_p) return;
    ContactArgs args{d, a, write_outputs,
                     LawParams{hp.k_n, hp.k_t, hp.gamma_n, hp.gamma_t, hp.gamma_r, hp.mu_s, hp.mu_d,
                               hp.mu_r, hp.kappa, hp.dt, {hp.L[0], hp.L[1]}}};
    if (d.shape) launch_contact_as<contact_block(1)>(args, np, model, st);
    else launch_contact_as<contact_block(0)>(args, np, model, st);
}

}  // namespace sphk
