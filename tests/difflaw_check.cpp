// Host build of sphere_b200/csrc/diff_law.h for tests/test_adjoint_laws.py:
// flat C entry points around the forward and reverse contact laws, so the
// reverse passes can be checked against central differences of the forward.
#include "diff_law.h"

using namespace dl;

static V3 ld(const double *p) { return v3(p[0], p[1], p[2]); }
static void st(double *p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

static Law law_of(const double *q)
{
    return Law{q[0], q[1], q[2], q[3], q[4], q[5], q[6]};
}

// in: xab(3) ra rb va(3) vb(3) wa(3) wb(3) d0u(3) = 20 doubles
static PairIn pair_of(const double *q)
{
    PairIn in;
    in.xab = ld(q);
    in.ra = q[3];
    in.rb = q[4];
    in.va = ld(q + 5);
    in.vb = ld(q + 8);
    in.wa = ld(q + 11);
    in.wb = ld(q + 14);
    in.d0u = ld(q + 17);
    return in;
}

extern "C" void pair_fwd_c(const double *law, const double *in, double *out)
{
    PairOut o;
    pair_fwd(law_of(law), pair_of(in), o);
    st(out, o.F);
    st(out + 3, o.T);
    st(out + 6, o.dtn);
}

// bars: F(3) T(3) dtn(3); inbar: xab va vb wa wb d0u (18); lawbar: kn kt gn mu
extern "C" void pair_rev_c(const double *law, const double *in, const double *bars, double *inbar,
                           double *lawbar)
{
    PairBar ib;
    LawBar lb{0.0, 0.0, 0.0, 0.0};
    pair_rev(law_of(law), pair_of(in), ld(bars), ld(bars + 3), ld(bars + 6), ib, lb);
    st(inbar, ib.xab);
    st(inbar + 3, ib.va);
    st(inbar + 6, ib.vb);
    st(inbar + 9, ib.wa);
    st(inbar + 12, ib.wb);
    st(inbar + 15, ib.d0u);
    lawbar[0] = lb.kn;
    lawbar[1] = lb.kt;
    lawbar[2] = lb.gn;
    lawbar[3] = lb.mu;
}

// wall law: w = kn gwn gwt mus mud; q = ra va(3) wa(3) n(3) delta wvel
extern "C" void wall_fwd_c(const double *w, const double *q, double *out)
{
    V3 F, T;
    wall_fwd(WallLaw{w[0], w[1], w[2], w[3], w[4]}, q[0], ld(q + 1), ld(q + 4), ld(q + 7), q[10],
             q[11], F, T);
    st(out, F);
    st(out + 3, T);
}

// out: va_bar(3) wa_bar(3) delta_bar kn_bar
extern "C" void wall_rev_c(const double *w, const double *q, const double *bars, double *out)
{
    V3 vab, wab;
    double deltab, knb;
    wall_rev(WallLaw{w[0], w[1], w[2], w[3], w[4]}, q[0], ld(q + 1), ld(q + 4), ld(q + 7), q[10],
             q[11], ld(bars), ld(bars + 3), vab, wab, deltab, knb);
    st(out, vab);
    st(out + 3, wab);
    out[6] = deltab;
    out[7] = knb;
}
