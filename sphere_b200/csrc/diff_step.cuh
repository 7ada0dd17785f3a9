// diff_step.cuh -- shared pieces of the differentiable step (k_force_diff in
// step.cu) and of its reverse (adjoint.cu).
#ifndef SPHK_DIFF_STEP_CUH_
#define SPHK_DIFF_STEP_CUH_

#include "sphk_internal.cuh"
#include "diff_law.h"

namespace sphk {

// The implicit walls of a scene without dynamic walls (defaults of
// src/contactsearch.cuh:416-427, tests :578-663) that particle xa touches,
// in the order the step applies them: outward normal n, overlap delta, the
// axis of the position it depends on and the sign of that dependence.
struct WallHits {
    int count;          // at most 6: top, floor, two in x, two in y
    dl::V3 n[6];
    double delta[6];
    int axis[6];
    double sign[6];
};

__device__ __forceinline__ void implicit_walls(const Params &P, double4 xa, WallHits &h)
{
    const double ra = xa.w;
    h.count = 0;
    auto add = [&](dl::V3 n, double delta, int axis, double sign) {
        if (delta < 0.0f) {
            h.n[h.count] = n;
            h.delta[h.count] = delta;
            h.axis[h.count] = axis;
            h.sign[h.count] = sign;
            ++h.count;
        }
    };
    add(dl::v3(0.0, 0.0, -1.0), P.L[2] - (xa.z + ra), 2, -1.0);
    add(dl::v3(0.0, 0.0, 1.0), xa.z - ra - P.origo[2], 2, 1.0);
    if (P.periodic == 0) {
        add(dl::v3(-1.0, 0.0, 0.0), P.L[0] - (xa.x + ra), 0, -1.0);
        add(dl::v3(1.0, 0.0, 0.0), xa.x - ra - 0.0, 0, 1.0);
    }
    if (P.periodic == 0 || P.periodic == 2) {
        add(dl::v3(0.0, -1.0, 0.0), P.L[1] - (xa.y + ra), 1, -1.0);
        add(dl::v3(0.0, 1.0, 0.0), xa.y - ra - 0.0, 1, 1.0);
    }
}

// Adjoint arrays of the reverse pass (adjoint.cu), storage-indexed.
struct AdjDev {
    double4 *xb, *vb, *wb, *v0b, *w0b;  // adjoints of the state, xyz used
    double4 *Fb, *Tb;                   // adjoints of force and torque, per step
    P3 *dtb;                            // adjoint of the slot history, tiled (tile_at)
    uint32_t *dtb_mask;                 // [np] slots whose dtb entry may be nonzero
    double *mub;                        // [np] adjoint of per-particle friction
    double *theta_b;                    // [3] adjoints of k_n, k_t, gamma_n
};

}  // namespace sphk

#endif
