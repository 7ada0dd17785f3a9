// bonds.cu -- parallel-bond forces (bondsLinear, src/cohesion.cuh:8-233).
//
// One thread per bond computes the beam model exactly as the reference and
// stores the force on the first particle and the torque on the second in
// per-bond slots.  The step kernel then gathers them per particle in bond
// order, which is the order in which the reference's (racy, non-atomic)
// scatter adds them when bonds are processed one after another.  The result
// is deterministic and needs no atomics.
#include "sphk_internal.cuh"

namespace sphk {

constexpr int BOND_BLOCK = 256;

// The constants of bondsLinear, fixed when a context is created: passed by
// value (the constant bank) rather than read through Params after a store.
struct BondConsts {
    uint32_t nb0, np;
    double dt, lambda_bar, k_n, k_t, gamma_n, gamma_t, sigma_b, tau_b;
};

// The bonds' particles as storage indices: bond_s follows bonds (by caller
// index) through sidx.  Storage order changes only at a relayout, after
// which this runs; a bond already broken (marker x >= np) keeps a pair that
// is never read.
__global__ void k_bond_storage(Dev d, uint32_t nb0, uint32_t np)
{
    const uint32_t b = blockIdx.x * BOND_BLOCK + threadIdx.x;
    if (b >= nb0) return;
    const uint2 bond = d.bonds[b];
    d.bond_s[b] = make_uint2(bond.x < np ? d.sidx[bond.x] : 0u, d.sidx[bond.y]);
}

__global__ void __launch_bounds__(BOND_BLOCK)
k_bonds(Dev d, int A, BondConsts P)
{
    const uint32_t idx = blockIdx.x * BOND_BLOCK + threadIdx.x;
    if (idx >= P.nb0) return;
    // the bond and its storage pair before any store, so that the two loads
    // and then the particle rows are each one memory latency
    const uint2 bond = d.bonds[idx];
    const uint2 bs = d.bond_s[idx];
    d.bond_xu[idx] = 0xffffffffu;
    if (!(bond.x < P.np)) return;     // erased bond (marker nb0 >= np)
    const uint32_t si = bs.x, sj = bs.y;
    const double dt = P.dt;
    const double4 d0 = d.bonds_delta[idx], o0 = d.bonds_omega[idx];
    d3 delta0_t = xyz(d0);
    const double delta0_n = d0.w;
    d3 omega0_t = xyz(o0);
    const double omega0_n = o0.w;
    const double4 xi = d.xr[A][si], xj = d.xr[A][sj];
    const double4 vi = ld4(d.vel[A], si), vj = ld4(d.vel[A], sj);
    const d3 wi = xyz(ld4(d.angvel[A], si)), wj = xyz(ld4(d.angvel[A], sj));
    const double R_bar = P.lambda_bar * fmin(xi.w, xj.w);
    const double Ab = REF_PI * R_bar * R_bar;
    const double I = 0.25 * REF_PI * R_bar * R_bar * R_bar * R_bar;
    const double J = I * 2.0;
    const d3 x = mk(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
    const double x_length = flen(x);
    const double overlap = fmin(0.0, x_length - (xi.w + xj.w));
    const d3 n = divs(x, x_length);
    delta0_t = sub(delta0_t, muls(n, dot(n, delta0_t)));
    const d3 ddelta = muls(add(add(mk(vi.x - vj.x, vi.y - vj.y, vi.z - vj.z),
                                   smul(xi.w + overlap / 2.0, cross(n, wi))),
                               smul(xj.w + overlap / 2.0, cross(n, wj))),
                           dt);
    const double ddelta_n = -dot(ddelta, n);
    const double delta_n = delta0_n + ddelta_n;
    const d3 ddelta_t = sub(ddelta, muls(n, dot(n, ddelta)));
    const d3 delta_t = add(delta0_t, ddelta_t);
    const d3 f_n = smul(P.k_n * Ab * delta_n + P.gamma_n * ddelta_n / dt, n);
    const d3 f_t = sub(smul(-P.k_t * Ab, delta_t), divs(smul(P.gamma_t, ddelta_t), dt));
    const d3 f = add(f_n, f_t);
    const d3 mn = mk(-n.x, -n.y, -n.z);
    omega0_t = sub(omega0_t, muls(mn, dot(omega0_t, mn)));
    const d3 domega = muls(mk(wj.x - wi.x, wj.y - wi.y, wj.z - wi.z), dt);
    const double domega_n = dot(domega, mn);
    const double omega_n = omega0_n + domega_n;
    const d3 domega_t = sub(domega, smul(domega_n, mn));
    const d3 omega_t = add(omega0_t, domega_t);
    const d3 t_n = smul(-P.k_t * J * omega_n, mn);
    const d3 t_t = smul(-P.k_n * I, omega_t);
    const d3 t_j = add(t_n, t_t);
    const double sigma_max = flen(f_n) / Ab + flen(t_t) * R_bar / I;
    const double tau_max = flen(f_t) / Ab + flen(t_n) * R_bar / J;
    if (sigma_max >= P.sigma_b || tau_max >= P.tau_b) {
        d.bonds[idx].x = P.nb0;
        // the reference re-reads the marker as a live particle index when
        // nb0 < np; such a bond would then act on particle nb0
        if (P.nb0 < P.np) atomicOr(d.status, ST_BOND_ALIAS);
        return;
    }
    d.bonds_delta[idx] = make_double4(delta_t.x, delta_t.y, delta_t.z, delta_n);
    d.bonds_omega[idx] = make_double4(omega_t.x, omega_t.y, omega_t.z, omega_n);
    d.bond_f[idx] = make_double4(f.x, f.y, f.z, 0.0);
    d.bond_t[idx] = make_double4(t_j.x, t_j.y, t_j.z, 0.0);
    d.bond_xu[idx] = bond.x;
}

void launch_bonds(const Dev &d, const Params &hp, uint32_t nb0, int a, cudaStream_t st)
{
    if (nb0 == 0) return;
    const BondConsts bc{hp.nb0,     hp.np,     hp.dt,      hp.lambda_bar, hp.k_n,
                        hp.k_t,     hp.gamma_n, hp.gamma_t, hp.sigma_b,   hp.tau_b};
    k_bonds<<<div_up(nb0, BOND_BLOCK), BOND_BLOCK, 0, st>>>(d, a, bc);
}

void launch_bond_storage(const Dev &d, uint32_t nb0, uint32_t np, cudaStream_t st)
{
    if (nb0 == 0) return;
    k_bond_storage<<<div_up(nb0, BOND_BLOCK), BOND_BLOCK, 0, st>>>(d, nb0, np);
}

}  // namespace sphk
