// diff_law.h -- the contact laws of the differentiable step and their reverse
// (adjoint) passes, for host and device.
//
// The differentiable step is contact model 2 (contactLinear,
// src/contactmodels.cuh:283-493, with the wall law contactLinear_wall,
// :10-109) evaluated in exact FP64: vector lengths are full double square
// roots, not the reference's float-narrowed ones, so the step is smooth
// enough for finite differences to check it.  Friction is per particle; a
// pair uses the mean of its two coefficients for both mu_s and mu_d.
//
// Each law has a forward function and a reverse function.  The reverse takes
// the adjoints ("bars") of the law's outputs and returns the adjoints of its
// inputs and parameters; it recomputes the forward intermediates itself, so
// nothing but the inputs has to be stored.  Branches (clipped normal force,
// sliding) are taken as in the forward: the derivative is that of the branch
// the forward took.  This header compiles as plain C++ too, so the reverse
// passes are checked against central differences of the forward on the host.
#ifndef SPHK_DIFF_LAW_H_
#define SPHK_DIFF_LAW_H_

#include <math.h>

#ifdef __CUDACC__
#define DL_HD __host__ __device__ __forceinline__
#else
#define DL_HD inline
#endif

namespace dl {

struct V3 {
    double x, y, z;
};

DL_HD V3 v3(double x, double y, double z) { return V3{x, y, z}; }
DL_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
DL_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
DL_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
DL_HD V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
DL_HD V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
DL_HD V3 &operator+=(V3 &a, V3 b) { a = a + b; return a; }
DL_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DL_HD V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
DL_HD double len(V3 a) { return sqrt(dot(a, a)); }

// Parameters of one contact: stiffnesses, damping, the pair's friction,
// cohesion factor, time step.
struct Law {
    double kn, kt, gn, gt, mu, kappa, dt;
};

// Adjoints of the differentiable parameters.
struct LawBar {
    double kn, kt, gn, mu;
};

// Particle-particle contact: inputs are the branch vector xab = xa - xb
// (+ periodic shift), radii, velocities, spins and the stored tangential
// displacement d0u; outputs are the force and torque on a and the new
// tangential displacement.
struct PairIn {
    V3 xab;
    double ra, rb;
    V3 va, vb, wa, wb, d0u;
};
struct PairOut {
    V3 F, T, dtn;
};
struct PairBar {
    V3 xab, va, vb, wa, wb, d0u;
};

DL_HD void pair_fwd(const Law &P, const PairIn &in, PairOut &out)
{
    const double L = len(in.xab);
    const double delta = L - (in.ra + in.rb);
    const V3 n = in.xab / L;
    const V3 vl = in.va - in.vb;
    const double ha = in.ra + delta / 2.0, hb = in.rb + delta / 2.0;
    const V3 vel = (vl + ha * cross(n, in.wa)) + hb * cross(n, in.wb);
    const double vn = -dot(vl, n);
    const V3 vt = vel - dot(n, vel) * n;
    const double Lt = len(vt);
    const V3 d0 = in.d0u - dot(n, in.d0u) * n;
    const double L0 = len(d0);
    const double sfn = -P.kn * delta - P.gn * vn;
    V3 fn = sfn * n;
    if (dot(fn, n) < 0.0) fn = v3(0.0, 0.0, 0.0);
    const double cfc = -P.kappa * sqrt(in.ra * in.rb);
    const V3 fc = cfc * n;
    V3 ft = v3(0.0, 0.0, 0.0), dtn = v3(0.0, 0.0, 0.0);
    if (L0 > 0.0 || Lt > 0.0) {
        const V3 dtn1 = d0 + P.dt * vt;
        const V3 ft1 = -P.kt * dtn1 - P.gt * vt;
        const double Lft = len(ft1);
        const double Lg = len(fn - fc);
        const double lim = P.mu * Lg;
        if (Lft > lim) {
            const V3 t = ft1 / Lft;
            ft = lim * t;
            dtn = (-1.0 / P.kt) * (P.mu * Lg * t + P.gt * vt);
        } else {
            ft = ft1;
            dtn = dtn1;
        }
    }
    out.F = (fn + ft) + fc;
    out.T = cross(-(in.ra + delta * 0.5) * n, ft);
    out.dtn = dtn;
}

// Reverse of pair_fwd: from the adjoints of F, T and dtn, the adjoints of
// the inputs (stored into ib) and of the parameters (added to pb).
DL_HD void pair_rev(const Law &P, const PairIn &in, V3 Fb, V3 Tb, V3 dtnb, PairBar &ib,
                    LawBar &pb)
{
    // ---- forward, keeping what the reverse needs ----
    const double L = len(in.xab);
    const double delta = L - (in.ra + in.rb);
    const V3 n = in.xab / L;
    const V3 vl = in.va - in.vb;
    const double ha = in.ra + delta / 2.0, hb = in.rb + delta / 2.0;
    const V3 ca = cross(n, in.wa), cb = cross(n, in.wb);
    const V3 vel = (vl + ha * ca) + hb * cb;
    const double vn = -dot(vl, n);
    const double s1 = dot(n, vel);
    const V3 vt = vel - s1 * n;
    const double Lt = len(vt);
    const double s0 = dot(n, in.d0u);
    const V3 d0 = in.d0u - s0 * n;
    const double L0 = len(d0);
    const double sfn = -P.kn * delta - P.gn * vn;
    V3 fn = sfn * n;
    const bool clip = dot(fn, n) < 0.0;
    if (clip) fn = v3(0.0, 0.0, 0.0);
    const double cfc = -P.kappa * sqrt(in.ra * in.rb);
    const V3 fc = cfc * n;
    // The forward skips the tangential law when both d0 and vt vanish; there
    // the sticking branch gives the same values (zero force, zero
    // displacement) and its derivative is the true one, so the reverse always
    // takes the law.
    (void)L0;
    (void)Lt;
    const bool active = true;
    V3 ft = v3(0.0, 0.0, 0.0), dtn1 = v3(0.0, 0.0, 0.0), ft1 = v3(0.0, 0.0, 0.0);
    V3 t = v3(0.0, 0.0, 0.0), g = v3(0.0, 0.0, 0.0);
    double Lft = 0.0, Lg = 0.0, lim = 0.0;
    bool slip = false;
    if (active) {
        dtn1 = d0 + P.dt * vt;
        ft1 = -P.kt * dtn1 - P.gt * vt;
        Lft = len(ft1);
        g = fn - fc;
        Lg = len(g);
        lim = P.mu * Lg;
        slip = Lft > lim;
        if (slip) {
            t = ft1 / Lft;
            ft = lim * t;
        } else {
            ft = ft1;
        }
    }
    const double hT = -(in.ra + delta * 0.5);
    const V3 u = hT * n;

    // ---- reverse ----
    V3 nb = v3(0.0, 0.0, 0.0), ftb, fnb, vtb = v3(0.0, 0.0, 0.0), d0b = v3(0.0, 0.0, 0.0);
    double deltab = 0.0;
    // T = cross(u, ft)
    const V3 ub = cross(ft, Tb);
    ftb = cross(Tb, u);
    deltab += -0.5 * dot(ub, n);
    nb += hT * ub;
    // F = fn + ft + fc
    fnb = Fb;
    ftb += Fb;
    nb += cfc * Fb;
    if (active) {
        V3 ft1b, dtn1b = v3(0.0, 0.0, 0.0);
        double Lgb = 0.0;
        if (slip) {
            const V3 q = P.mu * Lg * t + P.gt * vt;
            const V3 qb = (-1.0 / P.kt) * dtnb;
            pb.kt += dot(dtnb, q) / (P.kt * P.kt);
            pb.mu += Lg * dot(qb, t);
            Lgb += P.mu * dot(qb, t);
            V3 tb = (P.mu * Lg) * qb;
            vtb += P.gt * qb;
            const double limb = dot(ftb, t);
            tb += lim * ftb;
            ft1b = (tb - dot(t, tb) * t) / Lft;
            pb.mu += Lg * limb;
            Lgb += P.mu * limb;
        } else {
            ft1b = ftb;
            dtn1b = dtnb;
        }
        // Lg = |fn - fc|
        if (Lg > 0.0) {
            const V3 gb = (Lgb / Lg) * g;
            fnb += gb;
            nb += cfc * (-gb);
        }
        // ft1 = -kt dtn1 - gt vt
        pb.kt += -dot(ft1b, dtn1);
        dtn1b += -P.kt * ft1b;
        vtb += -P.gt * ft1b;
        // dtn1 = d0 + dt vt
        d0b = dtn1b;
        vtb += P.dt * dtn1b;
    }
    double vnb = 0.0;
    if (!clip) {
        const double sfnb = dot(fnb, n);
        nb += sfn * fnb;
        pb.kn += -delta * sfnb;
        deltab += -P.kn * sfnb;
        pb.gn += -vn * sfnb;
        vnb = -P.gn * sfnb;
    }
    // d0 = d0u - (n . d0u) n
    const double s0b = -dot(d0b, n);
    ib.d0u = d0b + s0b * n;
    nb += (-s0) * d0b + s0b * in.d0u;
    // vt = vel - (n . vel) n
    const double s1b = -dot(vtb, n);
    V3 velb = vtb + s1b * n;
    nb += (-s1) * vtb + s1b * vel;
    // vn = -(vl . n)
    V3 vlb = (-vnb) * n;
    nb += (-vnb) * vl;
    // vel = vl + ha ca + hb cb
    vlb += velb;
    deltab += 0.5 * (dot(velb, ca) + dot(velb, cb));
    const V3 cab = ha * velb, cbb = hb * velb;
    nb += cross(in.wa, cab) + cross(in.wb, cbb);
    ib.wa = cross(cab, n);
    ib.wb = cross(cbb, n);
    ib.va = vlb;
    ib.vb = -vlb;
    // n = xab / L, L = |xab| (through delta)
    ib.xab = (nb - dot(n, nb) * n) / L + deltab * n;
}

// Wall contact (contactLinear_wall): wall normal n, overlap delta (negative
// when touching), wall velocity wvel added to every component.  Outputs the
// force and torque on the particle.
struct WallLaw {
    double kn, gwn, gwt, mus, mud;
};

DL_HD void wall_fwd(const WallLaw &W, double ra, V3 va, V3 wa, V3 n, double delta, double wvel,
                    V3 &F, V3 &T)
{
    const V3 vel0 = va + ra * cross(n, wa);
    const V3 vel = v3(vel0.x + wvel, vel0.y + wvel, vel0.z + wvel);
    const double vn = dot(vel, n);
    const V3 vt = vel - dot(vel, n) * n;
    const double Lt = len(vt);
    V3 fn = (-W.kn * delta - W.gwn * vn) * n;
    if (dot(fn, n) < 0.0) fn = v3(0.0, 0.0, 0.0);
    const double Lfn = len(fn);
    V3 ft = v3(0.0, 0.0, 0.0);
    if (Lt > 0.0) {
        const double visc = W.gwt * Lt;
        const double lim = (Lt > 0.001f ? W.mud : W.mus) * Lfn;
        if (visc < lim) ft = (-visc * vt) / Lt;
        else ft = (-lim * vt) / Lt;
    }
    F = fn + ft;
    T = (-ra) * cross(n, ft);
}

// Reverse of wall_fwd: adjoints of va, wa, delta and of k_n.
DL_HD void wall_rev(const WallLaw &W, double ra, V3 va, V3 wa, V3 n, double delta, double wvel,
                    V3 Fb, V3 Tb, V3 &vab, V3 &wab, double &deltab, double &knb)
{
    const V3 vel0 = va + ra * cross(n, wa);
    const V3 vel = v3(vel0.x + wvel, vel0.y + wvel, vel0.z + wvel);
    const double vn = dot(vel, n);
    const V3 vt = vel - dot(vel, n) * n;
    const double Lt = len(vt);
    const double sfn = -W.kn * delta - W.gwn * vn;
    V3 fn = sfn * n;
    const bool clip = dot(fn, n) < 0.0;
    if (clip) fn = v3(0.0, 0.0, 0.0);
    const double Lfn = len(fn);
    V3 fnb = Fb;
    const V3 ftb = Fb + (-ra) * cross(Tb, n);
    V3 vtb = v3(0.0, 0.0, 0.0);
    if (Lt == 0.0) {
        // at rest in the tangent plane the forward skips the law; the
        // sticking branch (when the normal force allows friction) has the
        // same value there and gives the derivative
        if (0.0 < W.mus * Lfn) vtb += -W.gwt * ftb;
    } else {
        const double visc = W.gwt * Lt;
        const double mu = (Lt > 0.001f ? W.mud : W.mus);
        const double lim = mu * Lfn;
        if (visc < lim) {
            // ft = -gwt vt (visc / Lt = gwt)
            vtb += -W.gwt * ftb;
        } else {
            const V3 th = vt / Lt;
            const double limb = -dot(ftb, th);
            vtb += (-lim / Lt) * (ftb - dot(th, ftb) * th);
            if (Lfn > 0.0) fnb += (mu * limb / Lfn) * fn;
        }
    }
    double vnb = 0.0;
    deltab = 0.0;
    knb = 0.0;
    if (!clip) {
        const double sfnb = dot(fnb, n);
        knb = -delta * sfnb;
        deltab = -W.kn * sfnb;
        vnb = -W.gwn * sfnb;
    }
    const V3 velb = (vtb - dot(n, vtb) * n) + vnb * n;
    vab = velb;
    wab = ra * cross(velb, n);
}

}  // namespace dl

#endif
