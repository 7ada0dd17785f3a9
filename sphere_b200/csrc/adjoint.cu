// adjoint.cu -- the reverse pass of the differentiable step.
//
// The differentiable step is contact model 2 in exact FP64 with
// per-particle friction (k_force_diff, step.cu).  Going backwards
// through one step j needs the step's inputs, which the forward re-run of a
// checkpoint segment records in the tape (Dev::tp_*): positions, velocities
// and spins of every particle, and for each contact slot the law was
// evaluated on (tp_mask) its partner, periodic shift code and the stored
// tangential displacement it started from.  The reverse of step j is two
// launches:
//   k_rev_integ     the leapfrog in reverse: adjoints of the next state ->
//                   adjoints of force and torque, and of the state carried
//                   through (positions, half-step velocities and spins);
//   k_rev_contacts  the wall and pair laws in reverse (diff_law.h): the
//                   particle's own adjoints, its partners' (atomically), the
//                   adjoint of every slot's starting tangential displacement,
//                   and the parameter adjoints.
// A slot's tangential displacement at the start of step j came from step
// j - 1 exactly when the law was evaluated on that slot in step j - 1 (a slot
// holding a partner keeps it; a slot the law did not evaluate ends the step
// empty with zero history), so the adjoint written for slot i in step j is
// consumed by step j - 1 only if step j - 1's mask has slot i.
#include "diff_step.cuh"

namespace sphk {

constexpr int REV_BLOCK = 128;
// Resident blocks per SM that k_rev_contacts' register allocation must allow.
#ifndef SPHK_REV_MIN_BLOCKS
#define SPHK_REV_MIN_BLOCKS 2
#endif

__device__ __forceinline__ dl::V3 v3of(double4 a) { return dl::v3(a.x, a.y, a.z); }
__device__ __forceinline__ double4 d4of(dl::V3 a) { return make_double4(a.x, a.y, a.z, 0.0); }

__device__ __forceinline__ void atomic_add3(double4 *p, dl::V3 v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}

// The leapfrog of the force kernels (src/integration.cuh:9-187) is linear in force,
// torque and the carried state:
//   acc = F / m + g, angacc = T / (2/5 m r^2)   (zero under fixvel, except acc.z)
//   vel0' = vel0 + acc dt,  x' = x + vel0' dt,  vel' = vel0' + acc dt / 2
// and the same for the spins; the periodic wrap adds a constant.
__global__ void k_rev_integ(Dev d, AdjDev a, int j)
{
    const uint32_t np = d.np_all;
    const uint32_t s = blockIdx.x * REV_BLOCK + threadIdx.x;
    if (s >= np) return;
    const Params &P = *d.prm;
    const size_t row = (size_t)j * np + s;
    const double4 x = d.tp_x[row], v = d.tp_v[row];
    const double r = x.w, dt = P.dt;
    const double m = 4.0 / 3.0 * REF_PI * r * r * r * P.rho;
    const double I = 2.0 / 5.0 * m * r * r;
    const dl::V3 xb = v3of(a.xb[s]), vb = v3of(a.vb[s]), wb = v3of(a.wb[s]);
    const dl::V3 v0b = v3of(a.v0b[s]), w0b = v3of(a.w0b[s]);
    const dl::V3 v0tot = (v0b + dt * xb) + vb;
    const dl::V3 accb = dt * v0tot + (0.5 * dt) * vb;
    const dl::V3 w0tot = w0b + wb;
    const dl::V3 angaccb = dt * w0tot + (0.5 * dt) * wb;
    dl::V3 Fb = accb / m, Tb = angaccb / I;
    if (v.w > 0.0f) {   // fixvel: x and y acceleration and the spin are held
        Fb.x = 0.0;
        Fb.y = 0.0;
        Tb = dl::v3(0.0, 0.0, 0.0);
    }
    a.Fb[s] = d4of(Fb);
    a.Tb[s] = d4of(Tb);
    a.v0b[s] = d4of(v0tot);
    a.w0b[s] = d4of(w0tot);
    a.vb[s] = make_double4(0.0, 0.0, 0.0, 0.0);
    a.wb[s] = make_double4(0.0, 0.0, 0.0, 0.0);
}

__global__ void __launch_bounds__(REV_BLOCK, SPHK_REV_MIN_BLOCKS)
k_rev_contacts(Dev d, AdjDev a, int j)
{
    const uint32_t np = d.np_all;
    const uint32_t s = blockIdx.x * REV_BLOCK + threadIdx.x;
    double knb = 0.0, ktb = 0.0, gnb = 0.0;
    if (s < np) {
        const Params &P = *d.prm;
        const size_t row = (size_t)j * np + s;
        const double4 xa = d.tp_x[row], va4 = d.tp_v[row], wa4 = d.tp_w[row];
        const dl::V3 va = v3of(va4), wa = v3of(wa4);
        const dl::V3 Fb = v3of(a.Fb[s]), Tb = v3of(a.Tb[s]);
        dl::V3 xbs = dl::v3(0.0, 0.0, 0.0), vbs = xbs, wbs = xbs;
        double mubs = 0.0;   // the particle's own share of its contacts' friction adjoints

        // walls
        WallHits wh;
        implicit_walls(P, xa, wh);
        const dl::WallLaw wl{P.k_n, P.gamma_wn, P.gamma_wt, P.mu_ws, P.mu_wd};
        for (int k = 0; k < wh.count; ++k) {
            dl::V3 vab, wab;
            double deltab, kb;
            dl::wall_rev(wl, xa.w, va, wa, wh.n[k], wh.delta[k], 0.0, Fb, Tb, vab, wab, deltab, kb);
            vbs += vab;
            wbs += wab;
            const double g = wh.sign[k] * deltab;
            if (wh.axis[k] == 0) xbs.x += g;
            else if (wh.axis[k] == 1) xbs.y += g;
            else xbs.z += g;
            knb += kb;
        }

        // contact slots the law was evaluated on; a slot outside them starts
        // the step with constant (zero) history, so its adjoint is cleared
        // -- only where an earlier (later-in-time) step left one
        const uint32_t mask = d.tp_mask[row];
        const ulonglong2 dmw = d.tp_dmc[row];
        for (uint32_t m = a.dtb_mask[s] & ~mask; m; m &= m - 1)
            a.dtb[tile_at(s, (uint32_t)(__ffs(m) - 1), NC)] = P3{0.0, 0.0, 0.0};
        if (a.dtb_mask[s] != mask) a.dtb_mask[s] = mask;
        for (uint32_t m = mask; m; m &= m - 1) {
            const int i = __ffs(m) - 1;
            const size_t ts = tape_slot_at((uint32_t)j, np, s, (uint32_t)i);
            const size_t si = tile_at(s, (uint32_t)i, NC);
            const uint32_t t = d.tp_partner[ts];
            const size_t rt = (size_t)j * np + t;
            const double4 xb = d.tp_x[rt];
            const uint32_t code = (uint32_t)((i < 16 ? (dmw.x >> (4 * i)) : (dmw.y >> (4 * (i - 16)))) & 0xFull);
            const d3 dm = decode_dm(code, P);
            dl::PairIn in;
            in.xab = dl::v3(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            in.ra = xa.w;
            in.rb = xb.w;
            in.va = va;
            in.vb = v3of(d.tp_v[rt]);
            in.wa = wa;
            in.wb = v3of(d.tp_w[rt]);
            const P3 d0 = d.tp_dt0[ts];
            in.d0u = dl::v3(d0.x, d0.y, d0.z);
            const dl::Law law{P.k_n, P.k_t, P.gamma_n, P.gamma_t, 0.5 * (d.mu_p[s] + d.mu_p[t]),
                              P.kappa, P.dt};
            dl::PairBar ib;
            dl::LawBar lb{0.0, 0.0, 0.0, 0.0};
            const P3 dtbi = a.dtb[si];
            dl::pair_rev(law, in, Fb, Tb, dl::v3(dtbi.x, dtbi.y, dtbi.z), ib, lb);
            xbs += ib.xab;
            vbs += ib.va;
            wbs += ib.wa;
            atomic_add3(&a.xb[t], -ib.xab);
            atomic_add3(&a.vb[t], ib.vb);
            atomic_add3(&a.wb[t], ib.wb);
            a.dtb[si] = P3{ib.d0u.x, ib.d0u.y, ib.d0u.z};
            knb += lb.kn;
            ktb += lb.kt;
            gnb += lb.gn;
            mubs += 0.5 * lb.mu;
            atomicAdd(&a.mub[t], 0.5 * lb.mu);
        }
        if (mask != 0u || wh.count > 0) {   // nothing to add otherwise
            atomic_add3(&a.xb[s], xbs);
            atomic_add3(&a.vb[s], vbs);
            atomic_add3(&a.wb[s], wbs);
        }
        if (mask != 0u) atomicAdd(&a.mub[s], mubs);
    }
    // parameter adjoints: warp sums, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        knb += __shfl_down_sync(0xffffffffu, knb, o);
        ktb += __shfl_down_sync(0xffffffffu, ktb, o);
        gnb += __shfl_down_sync(0xffffffffu, gnb, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (knb != 0.0) atomicAdd(&a.theta_b[0], knb);
        if (ktb != 0.0) atomicAdd(&a.theta_b[1], ktb);
        if (gnb != 0.0) atomicAdd(&a.theta_b[2], gnb);
    }
}

// storage order <-> the caller's particle order
__global__ void k_user_to_storage3(const double *src, double4 *dst, const uint32_t *uid, uint32_t n)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t u = uid[s];
    dst[s] = src ? make_double4(src[3 * (size_t)u], src[3 * (size_t)u + 1], src[3 * (size_t)u + 2], 0.0)
                 : make_double4(0.0, 0.0, 0.0, 0.0);
}

__global__ void k_user_to_storage1(const double *src, double *dst, const uint32_t *uid, double dflt,
                                   uint32_t n)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = src ? src[uid[s]] : dflt;
}

__global__ void k_storage_to_user3(const double4 *a, const double4 *b, double *dst,
                                   const uint32_t *sidx, uint32_t n)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    double4 v = a[sidx[u]];
    if (b) {
        const double4 w = b[sidx[u]];
        v.x += w.x;
        v.y += w.y;
        v.z += w.z;
    }
    dst[3 * (size_t)u] = v.x;
    dst[3 * (size_t)u + 1] = v.y;
    dst[3 * (size_t)u + 2] = v.z;
}

__global__ void k_storage_to_user1(const double *src, double *dst, const uint32_t *sidx, uint32_t n)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) dst[u] = src[sidx[u]];
}

void launch_rev_step(const Dev &d, const AdjDev &a, uint32_t np, int j, cudaStream_t st)
{
    const unsigned grid = div_up(np, REV_BLOCK);
    k_rev_integ<<<grid, REV_BLOCK, 0, st>>>(d, a, j);
    k_rev_contacts<<<grid, REV_BLOCK, 0, st>>>(d, a, j);
}

void launch_user_to_storage3(const double *src, double4 *dst, const uint32_t *uid, uint32_t n,
                             cudaStream_t st)
{
    k_user_to_storage3<<<div_up(n, 256), 256, 0, st>>>(src, dst, uid, n);
}

void launch_user_to_storage1(const double *src, double *dst, const uint32_t *uid, double dflt,
                             uint32_t n, cudaStream_t st)
{
    k_user_to_storage1<<<div_up(n, 256), 256, 0, st>>>(src, dst, uid, dflt, n);
}

void launch_storage_to_user3(const double4 *a, const double4 *b, double *dst, const uint32_t *sidx,
                             uint32_t n, cudaStream_t st)
{
    k_storage_to_user3<<<div_up(n, 256), 256, 0, st>>>(a, b, dst, sidx, n);
}

void launch_storage_to_user1(const double *src, double *dst, const uint32_t *sidx, uint32_t n,
                             cudaStream_t st)
{
    k_storage_to_user1<<<div_up(n, 256), 256, 0, st>>>(src, dst, sidx, n);
}

}  // namespace sphk
