/*
 * oracle/dem_oracle.c -- plain-C restatement of sphere's per-timestep DEM
 * step (the time-loop body of src/device.cu:731-1109).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the path
 * itself.  It is loaded by tests/, __graft_entry__.smoke() and the CPU
 * baseline of bench.py.  Its results are pinned against the reference's own
 * kernel bodies (oracle/_ref, built by oracle/Makefile) and against the
 * fixtures under tests/golden/.
 *
 * Every floating-point expression keeps the reference's operation order,
 * because the CUDA path is checked against this file bit for bit:
 *   - double arithmetic with no contraction (build with -ffp-contract=off,
 *     the reference is built with --fmad=false, src/CMakeLists.txt:16-22);
 *   - length() narrows to float and calls sqrtf (src/vector_arithmetic.h:317);
 *   - float literals (0.001f, 4.0f) are widened exactly as in the reference.
 * Float-to-integer conversions follow the device semantics (saturating), the
 * behaviour of the GPU build the reference targets.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PI of src/constants.h:14 (not M_PI) */
static const double REF_PI = 3.14159265358979;

typedef struct { double x, y, z; } v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
/* scalar * vector: (s*a.x, ...) as vector_arithmetic.h:153-156 */
static inline v3 smul(double s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
/* vector * scalar: (a.x*s, ...) as vector_arithmetic.h:149-152 */
static inline v3 muls(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 adds(v3 a, double s) { return mk(a.x + s, a.y + s, a.z + s); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* src/vector_arithmetic.h:317-320: sqrtf of the narrowed dot product */
static inline double vlen(v3 a) { return (double)sqrtf((float)dot(a, a)); }
static inline v3 cross(v3 a, v3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 ld3(const double *p) { return mk(p[0], p[1], p[2]); }

/* device float->unsigned conversion (saturating, NaN -> 0) */
static inline uint32_t sat_u32(double f)
{
    if (!(f > 0.0)) return 0u;
    if (f >= 4294967295.0) return 0xffffffffu;
    return (uint32_t)f;
}
/* device float->int conversion (saturating, NaN -> 0) */
static inline int32_t sat_i32(double f)
{
    if (f != f) return 0;
    if (f <= -2147483648.0) return INT32_MIN;
    if (f >= 2147483647.0) return INT32_MAX;
    return (int32_t)f;
}
static inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

/* (x - origo) / (L / num), floored: src/sorting.cuh:12-14, contactsearch.cuh:336-338 */
static inline double cell_floor(const orc_scene *s, int d, double xd)
{
    return floor((xd - s->origo[d]) / (s->L[d] / (double)s->num[d]));
}

/* calcCellID, src/sorting.cuh:7-19 (unsigned arithmetic, wraps mod 2^32) */
static uint32_t cell_id(const orc_scene *s, const double *x)
{
    uint32_t ix = sat_u32(cell_floor(s, 0, x[0]));
    uint32_t iy = sat_u32(cell_floor(s, 1, x[1]));
    uint32_t iz = sat_u32(cell_floor(s, 2, x[2]));
    return (iz * s->num[1]) * s->num[0] + iy * s->num[0] + ix;
}

/* findDistMod, src/contactsearch.cuh:12-74.  Returns -1 when the target cell
 * lies outside a non-periodic boundary; otherwise wraps periodic axes and
 * accumulates the +/-L shift into *dm. */
static int dist_mod(const orc_scene *s, int32_t c[3], v3 *dm)
{
    const uint32_t nx = s->num[0], ny = s->num[1], nz = s->num[2];
    if (s->periodic == 1) {
        if (c[0] < 0) { c[0] = (int32_t)(nx - 1); *dm = add(*dm, mk(s->L[0], 0.0, 0.0)); }
        if ((uint32_t)c[0] == nx) { c[0] = 0; *dm = sub(*dm, mk(s->L[0], 0.0, 0.0)); }
        if (c[1] < 0) { c[1] = (int32_t)(ny - 1); *dm = add(*dm, mk(0.0, s->L[1], 0.0)); }
        if ((uint32_t)c[1] == ny) { c[1] = 0; *dm = sub(*dm, mk(0.0, s->L[1], 0.0)); }
    } else if (s->periodic == 2) {
        if (c[0] < 0) { c[0] = (int32_t)(nx - 1); *dm = add(*dm, mk(s->L[0], 0.0, 0.0)); }
        if ((uint32_t)c[0] == nx) { c[0] = 0; *dm = sub(*dm, mk(s->L[0], 0.0, 0.0)); }
        if (c[1] < 0 || (uint32_t)c[1] == ny) return -1;
    } else {
        if (c[0] < 0 || (uint32_t)c[0] == nx) return -1;
        if (c[1] < 0 || (uint32_t)c[1] == ny) return -1;
    }
    if (c[2] < 0 || (uint32_t)c[2] == nz) return -1;
    return 0;
}

/* working arrays that live across steps */
typedef struct {
    uint32_t np, ncells;
    uint32_t *cellid;   /* per original index */
    uint32_t *count;    /* ncells + 1 (last bucket: out-of-grid keys) */
    double *x_s, *vel_s, *angvel_s; /* sorted copies, 4 doubles each */
    double *wf_pp;      /* wall-0 force per original index */
} work_t;

static void work_free(work_t *w)
{
    free(w->cellid); free(w->count); free(w->x_s); free(w->vel_s);
    free(w->angvel_s); free(w->wf_pp);
    memset(w, 0, sizeof(*w));
}

static int work_alloc(work_t *w, uint32_t np, uint32_t ncells)
{
    memset(w, 0, sizeof(*w));
    w->np = np; w->ncells = ncells;
    w->cellid = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)np);
    w->count = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)ncells + 1));
    w->x_s = (double *)malloc(sizeof(double) * 4 * (size_t)np);
    w->vel_s = (double *)malloc(sizeof(double) * 4 * (size_t)np);
    w->angvel_s = (double *)malloc(sizeof(double) * 4 * (size_t)np);
    w->wf_pp = (double *)calloc((size_t)np, sizeof(double));
    if (!w->cellid || !w->count || !w->x_s || !w->vel_s || !w->angvel_s || !w->wf_pp) {
        work_free(w);
        return -1;
    }
    return 0;
}

/* ---- cell list: calcParticleCellID + stable sort + reorderArrays ------- */
/* src/sorting.cuh:24-43 (cell of every particle), src/device.cu:763-765
 * (stable sort of (cellID, index); a counting sort is stable by
 * construction), src/device.cu:776-777 (cellStart := 0xffffffff) and
 * src/sorting.cuh:49-121 (cellStart/cellEnd and the gathered copies). */
static int build_cells(orc_scene *s, work_t *w)
{
    const uint32_t np = s->np, nc = w->ncells;
    int err = 0;
    for (uint32_t i = 0; i < np; ++i) {
        const double *xi = &s->x[4 * (size_t)i];
        uint32_t c = cell_id(s, xi);
        /* a position that is not finite lies outside the grid */
        if (c >= nc || !isfinite(xi[0] + xi[1] + xi[2])) { err |= ORC_ERR_OUT_OF_GRID; c = nc; }
        w->cellid[i] = c;
    }
    memset(w->count, 0, sizeof(uint32_t) * ((size_t)nc + 1));
    for (uint32_t i = 0; i < np; ++i) w->count[w->cellid[i]]++;
    uint32_t run = 0;
    for (uint32_t c = 0; c <= nc; ++c) { uint32_t k = w->count[c]; w->count[c] = run; run += k; }
    for (uint32_t i = 0; i < np; ++i) {
        uint32_t c = w->cellid[i];
        uint32_t k = w->count[c]++;
        s->perm[k] = i;
        s->cell_sorted[k] = (c == nc) ? 0xffffffffu : cell_id(s, &s->x[4 * (size_t)i]);
    }
    for (uint32_t c = 0; c < nc; ++c) s->cell_start[c] = 0xffffffffu;
    for (uint32_t k = 0; k < np; ++k) {
        uint32_t c = w->cellid[s->perm[k]];
        uint32_t prev = k > 0 ? w->cellid[s->perm[k - 1]] : 0;
        if (c < nc && (k == 0 || c != prev)) s->cell_start[c] = k;
        if (k > 0 && c != prev && prev < nc) s->cell_end[prev] = k;
        if (k == np - 1 && c < nc) s->cell_end[c] = k + 1;
        const size_t o = 4 * (size_t)s->perm[k];
        memcpy(&w->x_s[4 * (size_t)k], &s->x[o], 4 * sizeof(double));
        memcpy(&w->vel_s[4 * (size_t)k], &s->vel[o], 4 * sizeof(double));
        memcpy(&w->angvel_s[4 * (size_t)k], &s->angvel[o], 4 * sizeof(double));
    }
    return err;
}

/* ---- topology: src/contactsearch.cuh:181-355 ---------------------------- */
static int topology_one(orc_scene *s, work_t *w, uint32_t a)
{
    const uint32_t np = s->np;
    const double *xa = &w->x_s[4 * (size_t)a];
    const double ra = xa[3];
    const uint32_t a_orig = s->perm[a];
    uint32_t *row = &s->contacts[(size_t)a_orig * ORC_NC];
    double *dmrow = &s->distmod[(size_t)a_orig * ORC_NC * 4];
    int err = 0;
    int nc = 0;
    int32_t gp[3];
    for (int d = 0; d < 3; ++d) gp[d] = sat_i32(cell_floor(s, d, xa[d]));
    for (int oz = -1; oz < 2; ++oz)
        for (int oy = -1; oy < 2; ++oy)
            for (int ox = -1; ox < 2; ++ox) {
                int32_t c[3] = {wrap_add(gp[0], ox), wrap_add(gp[1], oy), wrap_add(gp[2], oz)};
                v3 dm = mk(0.0, 0.0, 0.0);
                if (dist_mod(s, c, &dm) == -1) continue;
                uint32_t cid = (uint32_t)c[0] + (uint32_t)c[1] * s->num[0]
                    + (s->num[0] * s->num[1]) * (uint32_t)c[2];
                if (cid >= w->ncells) { err |= ORC_ERR_OUT_OF_GRID; continue; }
                uint32_t start = s->cell_start[cid];
                if (start == 0xffffffffu) continue;
                uint32_t end = s->cell_end[cid];
                for (uint32_t b = start; b < end; ++b) {
                    if (b == a) continue;
                    const double *xb = &w->x_s[4 * (size_t)b];
                    const double rb = xb[3];
                    const uint32_t b_orig = s->perm[b];
                    v3 xab = add(mk(xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]), dm);
                    double len = vlen(xab);
                    double delta = len - (ra + rb);
                    if (delta < 0.0f) {
                        /* slot choice, contactsearch.cuh:252-265: a slot that
                         * already holds b wins; otherwise the last empty slot;
                         * otherwise position nc */
                        int cpos = nc;
                        for (int i = 0; i < ORC_NC; ++i) {
                            uint32_t v = row[i];
                            if (v == np) cpos = i;
                            else if (v == b_orig) { cpos = i; break; }
                        }
                        if (cpos >= ORC_NC) {
                            err |= ORC_ERR_NC_OVERFLOW;
                        } else {
                            row[cpos] = b_orig;
                            double *d = &dmrow[4 * cpos];
                            d[0] = dm.x; d[1] = dm.y; d[2] = dm.z; d[3] = rb;
                        }
                        ++nc;
                        if (nc > ORC_NC) break; /* returns from this cell only */
                    }
                }
            }
    return err;
}

/* ---- contact laws: src/contactmodels.cuh -------------------------------- */

/* contactLinear_wall, src/contactmodels.cuh:10-109 */
static double contact_wall(const orc_scene *s, v3 *F, v3 *T, double *p,
                           double ra, const double *vel_a, const double *angvel_a,
                           v3 n, double delta, double wvel)
{
    v3 linvel = ld3(vel_a), angvel = ld3(angvel_a);
    v3 vel = adds(add(linvel, smul(ra, cross(n, angvel))), wvel);
    double vel_n = dot(vel, n);
    v3 vel_t = sub(vel, muls(n, dot(vel, n)));
    double vel_t_length = vlen(vel_t);
    v3 f_n = smul(-s->k_n * delta - s->gamma_wn * vel_n, n);
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(f_n);
    v3 f_t = mk(0.0, 0.0, 0.0);
    v3 T_res = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.f) {
        double f_t_visc = s->gamma_wt * vel_t_length;
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = s->mu_wd * f_n_length;
        else f_t_limit = s->mu_ws * f_n_length;
        if (f_t_visc < f_t_limit) f_t = divs(smul(-1.0f * f_t_visc, vel_t), vel_t_length);
        else f_t = divs(smul(-1.0f * f_t_limit, vel_t), vel_t_length);
    }
    *F = add(*F, add(f_n, f_t));
    *T = add(*T, add(smul(-ra, cross(n, f_t)), T_res));
    *p += f_n_length / (4.0f * REF_PI * ra * ra);
    return dot(f_n, n);
}

/* contactLinear, src/contactmodels.cuh:283-493 (contact model 2) */
static void contact_linear(const orc_scene *s, v3 *F, v3 *T, double *es_dot,
                           double *ev_dot, double *p, uint32_t b_orig,
                           const double *vel_a4, v3 angvel_a, double ra, double rb,
                           v3 x, double x_length, double delta, double *dt4)
{
    const double dt = s->dt;
    v3 vel_b = ld3(&s->vel[4 * (size_t)b_orig]);
    v3 angvel_b = ld3(&s->angvel[4 * (size_t)b_orig]);
    v3 dt0u = ld3(dt4);
    v3 n = divs(x, x_length);
    v3 vel_linear = mk(vel_a4[0] - vel_b.x, vel_a4[1] - vel_b.y, vel_a4[2] - vel_b.z);
    v3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                 smul(rb + delta / 2.0, cross(n, angvel_b)));
    double vel_n = -dot(vel_linear, n);
    v3 vel_t = sub(vel, muls(n, dot(n, vel)));
    double vel_t_length = vlen(vel_t);
    v3 delta_t0 = sub(dt0u, muls(n, dot(n, dt0u)));
    double delta_t0_length = vlen(delta_t0);
    v3 delta_t = mk(0.0, 0.0, 0.0); /* left unset by the reference when unused */
    v3 f_n = smul(-s->k_n * delta - s->gamma_n * vel_n, n);
    *ev_dot += s->gamma_n * vel_n * vel_n;
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(f_n);
    v3 f_c = smul(-s->kappa * (double)sqrtf((float)(ra * rb)), n);
    v3 f_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = add(delta_t0, muls(vel_t, dt));
        v3 f_t_elast = smul(-s->k_t, delta_t);
        v3 f_t_visc = smul(-s->gamma_t, vel_t);
        f_t = add(f_t_elast, f_t_visc);
        double f_t_length = vlen(f_t);
        double f_t_limit = s->mu_s * vlen(sub(f_n, f_c));
        delta_t = add(delta_t0, muls(vel_t, dt));
        if (f_t_length > f_t_limit) {
            v3 t = divs(f_t, vlen(f_t));
            f_t = smul(f_t_limit, t);
            delta_t = smul(-1.0 / s->k_t,
                           add(smul(s->mu_d * vlen(sub(f_n, f_c)), t), smul(s->gamma_t, vel_t)));
            *es_dot += vlen(muls(smul(vlen(f_t), vel_t), dt)) / dt;
        }
    }
    *F = add(*F, add(add(f_n, f_t), f_c));
    *T = add(*T, cross(smul(-(ra + delta * 0.5), n), f_t));
    *p += f_n_length / (4.0f * REF_PI * ra * ra);
    dt4[0] = delta_t.x; dt4[1] = delta_t.y; dt4[2] = delta_t.z; dt4[3] = 0.0f;
}

/* The FP32 transcendentals of the force laws: expf in capillaryCohesion_exp
 * and powf in contactHertz.  By default each is evaluated as the float
 * nearest to the double-precision result, which is also what the CUDA path
 * computes; orc_set_libm_float_math(1) switches to the C library's expf and
 * powf, which is what the reference's host build calls. */
static int g_libm_float = 0;
void orc_set_libm_float_math(int on) { g_libm_float = on; }

static inline double f32_expf(double x)
{
    const float xf = (float)x;
    return g_libm_float ? (double)expf(xf) : (double)(float)exp((double)xf);
}

static inline double f32_powf(double x, float y)
{
    const float xf = (float)x;
    return g_libm_float ? (double)powf(xf, y) : (double)(float)pow((double)xf, (double)y);
}

/* contactLinearViscous, src/contactmodels.cuh:114-253 (contact model 1):
 * no tangential history; the torque is not changed (its update is commented
 * out in the reference, :244) */
static void contact_viscous(const orc_scene *s, v3 *F, double *p, const double *vel_a,
                            const double *vel_b, v3 angvel_a, v3 angvel_b, double ra,
                            double rb, v3 x_ab, double x_ab_length, double delta, double kappa)
{
    v3 n = divs(x_ab, x_ab_length);
    v3 vel_linear = mk(vel_a[0] - vel_b[0], vel_a[1] - vel_b[1], vel_a[2] - vel_b[2]);
    v3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                 smul(rb + delta / 2.0, cross(n, angvel_b)));
    double vel_n = dot(vel_linear, n);
    v3 vel_t = sub(vel, muls(n, dot(vel, n)));
    double vel_t_length = vlen(vel_t);
    v3 f_n = smul(-s->k_n * delta - s->gamma_n * vel_n, n);
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(f_n);
    v3 f_c = smul(-kappa * (double)sqrtf((float)(ra * rb)), n);
    v3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0) {
        double f_t_visc = s->gamma_t * vel_t_length;
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = s->mu_d * vlen(sub(f_n, f_c));
        else f_t_limit = s->mu_s * vlen(sub(f_n, f_c));
        if (f_t_visc < f_t_limit) f_t = divs(smul(-f_t_visc, vel_t), vel_t_length);
        else f_t = divs(smul(-f_t_limit, vel_t), vel_t_length);
    }
    *F = add(*F, add(add(f_n, f_t), f_c));
    *p += f_n_length / (4.0f * REF_PI * ra * ra);
}

/* capillaryCohesion_exp, src/cohesion.cuh:314-350 */
static void capillary_exp(const orc_scene *s, v3 *F, double ra, double rb, double delta,
                          v3 x_ab, double x_ab_length, double kappa)
{
    v3 n = divs(x_ab, x_ab_length);
    double r;
    if ((ra / rb) > (rb / ra)) r = ra / rb;
    else r = rb / ra;
    double h = -(double)sqrtf((float)r);
    double R_har = (2.0f * ra * rb) / (ra + rb);
    double R_geo = (double)sqrtf((float)(ra * rb));
    double lambda = 0.9f * h * (double)sqrtf((float)(s->V_b / R_har));
    v3 f_c = smul(-kappa * R_geo * f32_expf(-delta / lambda), n);
    *F = add(*F, f_c);
}

/* contactHertz, src/contactmodels.cuh:499-666 (contact model 3).  The
 * overlap delta is negative here, as in the reference, so the fractional
 * powers of it are NaN. */
static void contact_hertz(const orc_scene *s, v3 *F, v3 *T, double *es_dot, double *ev_dot,
                          double *p, uint32_t b_orig, const double *vel_a4, v3 angvel_a,
                          double ra, double rb, v3 x, double x_length, double delta,
                          double *dt4)
{
    const double dt = s->dt;
    v3 vel_b = ld3(&s->vel[4 * (size_t)b_orig]);
    v3 angvel_b = ld3(&s->angvel[4 * (size_t)b_orig]);
    v3 dt0u = ld3(dt4);
    v3 n = divs(x, x_length);
    v3 vel_linear = mk(vel_a4[0] - vel_b.x, vel_a4[1] - vel_b.y, vel_a4[2] - vel_b.z);
    v3 vel = add(add(vel_linear, smul(ra + delta / 2.0, cross(n, angvel_a))),
                 smul(rb + delta / 2.0, cross(n, angvel_b)));
    v3 angvel_ab = sub(angvel_a, angvel_b);
    double angvel_ab_length = vlen(angvel_ab);
    double vel_n = dot(vel_linear, n);
    v3 vel_t = sub(vel, muls(n, dot(vel, n)));
    double vel_t_length = vlen(vel_t);
    v3 delta_t0 = sub(dt0u, muls(n, dot(dt0u, n)));
    double delta_t0_length = vlen(delta_t0);
    v3 delta_t = mk(0.0, 0.0, 0.0); /* left unset by the reference when unused */
    v3 f_n = smul(-s->k_n * f32_powf(delta, 3.0f / 2.0f)
                      - s->gamma_n * f32_powf(delta, 1.0f / 4.0f) * vel_n, n);
    *ev_dot += s->gamma_n * vel_n * vel_n;
    if (dot(f_n, n) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(f_n);
    v3 f_c = smul(-s->kappa * (double)sqrtf((float)(ra * rb)), n);
    v3 f_t = mk(0.0, 0.0, 0.0);
    v3 T_res = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.f || vel_t_length > 0.f) {
        v3 f_t_elast = smul(-s->k_t * f32_powf(delta, 1.0f / 2.0f), delta_t0);
        v3 f_t_visc = smul(-s->gamma_t * f32_powf(delta, 1.0f / 4.0f), vel_t);
        double f_t_limit;
        if (vel_t_length > 0.001f) f_t_limit = s->mu_d * vlen(sub(f_n, f_c));
        else f_t_limit = s->mu_s * vlen(sub(f_n, f_c));
        f_t = add(f_t_elast, f_t_visc);
        double f_t_length = vlen(f_t);
        if (f_t_length > f_t_limit) {
            f_t = muls(f_t, f_t_limit / f_t_length);
            delta_t = divs(add(f_t, smul(s->gamma_t * f32_powf(delta, 1.0f / 4.0f), vel_t)),
                           -s->k_t * f32_powf(delta, 1.0f / 2.0f));
            *es_dot += vlen(sub(delta_t0, delta_t)) * s->k_t / dt;
        } else {
            delta_t = add(delta_t0, muls(vel_t, dt));
        }
    }
    if (angvel_ab_length > 0.f) {
        T_res = divs(smul(-1.0f * fmin(s->gamma_r * ra * angvel_ab_length,
                                       s->mu_r * ra * f_n_length),
                          angvel_ab),
                     angvel_ab_length);
    }
    *F = add(*F, add(add(f_n, f_t), f_c));
    *T = add(*T, add(smul(-(ra + delta / 2.0), cross(n, f_t)), T_res));
    *p += f_n_length / (4.0f * REF_PI * ra * ra);
    dt4[0] = delta_t.x; dt4[1] = delta_t.y; dt4[2] = delta_t.z; dt4[3] = 0.0f;
}

/* Model 1 finds and processes contacts in one pass over the 27 stencil cells
 * (contactsearch.cuh:548-576 and findAndProcessContactsInCell, :81-175),
 * over the sorted copies. */
static int sweep_viscous(orc_scene *s, work_t *w, uint32_t a, v3 *F, double *p)
{
    const double *xa = &w->x_s[4 * (size_t)a];
    const double ra = xa[3];
    const double *vel_a = &w->vel_s[4 * (size_t)a];
    const v3 angvel_a = ld3(&w->angvel_s[4 * (size_t)a]);
    int err = 0;
    int32_t gp[3];
    for (int d = 0; d < 3; ++d) gp[d] = sat_i32(cell_floor(s, d, xa[d]));
    for (int oz = -1; oz < 2; ++oz)
        for (int oy = -1; oy < 2; ++oy)
            for (int ox = -1; ox < 2; ++ox) {
                int32_t c[3] = {wrap_add(gp[0], ox), wrap_add(gp[1], oy), wrap_add(gp[2], oz)};
                v3 dm = mk(0.0, 0.0, 0.0);
                if (dist_mod(s, c, &dm) == -1) continue;
                uint32_t cid = (uint32_t)c[0] + (uint32_t)c[1] * s->num[0]
                    + (s->num[0] * s->num[1]) * (uint32_t)c[2];
                if (cid >= w->ncells) { err |= ORC_ERR_OUT_OF_GRID; continue; }
                uint32_t start = s->cell_start[cid];
                if (start == 0xffffffffu) continue;
                uint32_t end = s->cell_end[cid];
                for (uint32_t b = start; b < end; ++b) {
                    if (b == a) continue;
                    const double *xb = &w->x_s[4 * (size_t)b];
                    const double rb = xb[3];
                    v3 xab = add(mk(xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]), dm);
                    double len = vlen(xab);
                    double delta = len - (ra + rb);
                    if (delta < 0.0f)
                        contact_viscous(s, F, p, vel_a, &w->vel_s[4 * (size_t)b], angvel_a,
                                        ld3(&w->angvel_s[4 * (size_t)b]), ra, rb, xab, len,
                                        delta, s->kappa);
                    else if (delta < s->db)
                        capillary_exp(s, F, ra, rb, delta, xab, len, s->kappa);
                }
            }
    return err;
}

/* ---- interact: src/contactsearch.cuh:369-689 (contact models 2/3) ------- */
static int interact_one(orc_scene *s, work_t *w, uint32_t a)
{
    int err = 0;
    const uint32_t np = s->np;
    const uint32_t a_orig = s->perm[a];
    const double *xa = &w->x_s[4 * (size_t)a];
    const double ra = xa[3];
    const v3 origo = mk(s->origo[0], s->origo[1], s->origo[2]);
    const v3 L = mk(s->L[0], s->L[1], s->L[2]);
    /* default walls, contactsearch.cuh:416-427 */
    double wnx[5][4] = {{0.0, 0.0, -1.0, L.z}, {-1.0, 0.0, 0.0, L.x}, {1.0, 0.0, 0.0, 0.0},
                        {0.0, -1.0, 0.0, L.y}, {0.0, 1.0, 0.0, 0.0}};
    double wmvfd[5][4] = {{0}};
    for (uint32_t k = 0; k < s->nw && k < 5; ++k) {
        memcpy(wnx[k], &s->walls_nx[4 * k], 4 * sizeof(double));
        memcpy(wmvfd[k], &s->walls_mvfd[4 * k], 4 * sizeof(double));
    }
    double es_dot = 0.0f, ev_dot = 0.0f, p = 0.0f;
    v3 F = mk(0.0, 0.0, 0.0), T = mk(0.0, 0.0, 0.0);
    const double *vel_a = &w->vel_s[4 * (size_t)a];
    const double *angvel_a4 = &w->angvel_s[4 * (size_t)a];
    v3 angvel_a = ld3(angvel_a4);
    if (s->contactmodel == 2 || s->contactmodel == 3) {
        for (int i = 0; i < ORC_NC; ++i) {
            size_t mp = (size_t)a_orig * ORC_NC + (size_t)i;
            uint32_t b_orig = s->contacts[mp];
            double *dt4 = &s->delta_t[4 * mp];
            if (b_orig != np) {
                const double *dm = &s->distmod[4 * mp];
                const double *xb = &s->x[4 * (size_t)b_orig];
                double rb = xb[3];
                v3 xab = mk(xa[0] - xb[0] + dm[0], xa[1] - xb[1] + dm[1], xa[2] - xb[2] + dm[2]);
                double xlen = vlen(xab);
                double delta_n = xlen - (ra + rb);
                if (delta_n < 0.0f) {
                    if (s->contactmodel == 2)
                        contact_linear(s, &F, &T, &es_dot, &ev_dot, &p, b_orig, vel_a,
                                       angvel_a, ra, rb, xab, xlen, delta_n, dt4);
                    else
                        contact_hertz(s, &F, &T, &es_dot, &ev_dot, &p, b_orig, vel_a,
                                      angvel_a, ra, rb, xab, xlen, delta_n, dt4);
                } else {
                    s->contacts[mp] = np;
                    dt4[0] = dt4[1] = dt4[2] = dt4[3] = 0.0;
                }
            } else {
                dt4[0] = dt4[1] = dt4[2] = dt4[3] = 0.0;
            }
        }
    } else if (s->contactmodel == 1) {
        err |= sweep_viscous(s, w, a, &F, &p);
    }
    /* walls, contactsearch.cuh:578-663 */
    double w0f = 0.0;
    double dw;
    dw = wnx[0][3] - (xa[2] + ra);
    if (dw < 0.0f)
        w0f = contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[0]), dw, wmvfd[0][1]);
    dw = xa[2] - ra - origo.z;
    if (dw < 0.0f)
        (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, mk(0.0, 0.0, 1.0), dw, 0.0f);
    if (s->periodic == 0) {
        dw = wnx[1][3] - (xa[0] + ra);
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[1]), dw, wmvfd[1][1]);
        dw = xa[0] - ra - wnx[2][3];
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[2]), dw, wmvfd[2][1]);
        dw = wnx[3][3] - (xa[1] + ra);
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[3]), dw, wmvfd[3][1]);
        dw = xa[1] - ra - wnx[4][3];
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[4]), dw, wmvfd[4][1]);
    } else if (s->periodic == 2) {
        dw = wnx[3][3] - (xa[1] + ra);
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[3]), dw, wmvfd[3][1]);
        dw = xa[1] - ra - wnx[4][3];
        if (dw < 0.0f) (void)contact_wall(s, &F, &T, &p, ra, vel_a, angvel_a4, ld3(wnx[4]), dw, wmvfd[4][1]);
    }
    /* writes at the original index, contactsearch.cuh:670-687 */
    double *f = &s->force[4 * (size_t)a_orig];
    double *t = &s->torque[4 * (size_t)a_orig];
    f[0] = F.x; f[1] = F.y; f[2] = F.z; f[3] = 0.0f;
    t[0] = T.x; t[1] = T.y; t[2] = T.z; t[3] = 0.0f;
    s->es_dot[a_orig] = es_dot;
    s->ev_dot[a_orig] = ev_dot;
    s->es[a_orig] += es_dot * s->dt;
    s->ev[a_orig] += ev_dot * s->dt;
    s->p[a_orig] = p;
    w->wf_pp[a_orig] = w0f;
    return err;
}

/* ---- bondsLinear: src/cohesion.cuh:8-233, bonds in index order ---------- */
static void bond_one(orc_scene *s, uint32_t idx)
{
    const double dt = s->dt;
    uint32_t bi = s->bonds[2 * (size_t)idx], bj = s->bonds[2 * (size_t)idx + 1];
    if (!(bi < s->np)) return;
    const double *d0 = &s->bonds_delta[4 * (size_t)idx];
    const double *o0 = &s->bonds_omega[4 * (size_t)idx];
    v3 delta0_t = ld3(d0);
    const double delta0_n = d0[3];
    v3 omega0_t = ld3(o0);
    const double omega0_n = o0[3];
    const double *xi = &s->x[4 * (size_t)bi], *xj = &s->x[4 * (size_t)bj];
    const double *vi = &s->vel[4 * (size_t)bi], *vj = &s->vel[4 * (size_t)bj];
    v3 wi = ld3(&s->angvel[4 * (size_t)bi]), wj = ld3(&s->angvel[4 * (size_t)bj]);
    const double R_bar = s->lambda_bar * fmin(xi[3], xj[3]);
    const double A = REF_PI * R_bar * R_bar;
    const double I = 0.25 * REF_PI * R_bar * R_bar * R_bar * R_bar;
    const double J = I * 2.0;
    const v3 x = mk(xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]);
    const double x_length = vlen(x);
    const double overlap = fmin(0.0, x_length - (xi[3] + xj[3]));
    v3 n = divs(x, x_length);
    delta0_t = sub(delta0_t, muls(n, dot(n, delta0_t)));
    const v3 ddelta = muls(add(add(mk(vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]),
                                   smul(xi[3] + overlap / 2.0, cross(n, wi))),
                               smul(xj[3] + overlap / 2.0, cross(n, wj))),
                           dt);
    const double ddelta_n = -dot(ddelta, n);
    const double delta_n = delta0_n + ddelta_n;
    const v3 ddelta_t = sub(ddelta, muls(n, dot(n, ddelta)));
    const v3 delta_t = add(delta0_t, ddelta_t);
    const v3 f_n = smul(s->k_n * A * delta_n + s->gamma_n * ddelta_n / dt, n);
    const v3 f_t = sub(smul(-s->k_t * A, delta_t), divs(smul(s->gamma_t, ddelta_t), dt));
    const v3 f = add(f_n, f_t);
    const v3 mn = mk(-n.x, -n.y, -n.z);
    omega0_t = sub(omega0_t, muls(mn, dot(omega0_t, mn)));
    const v3 domega = muls(mk(wj.x - wi.x, wj.y - wi.y, wj.z - wi.z), dt);
    const double domega_n = dot(domega, mn);
    const double omega_n = omega0_n + domega_n;
    const v3 domega_t = sub(domega, smul(domega_n, mn));
    const v3 omega_t = add(omega0_t, domega_t);
    const v3 t_n = smul(-s->k_t * J * omega_n, mn);
    const v3 t_t = smul(-s->k_n * I, omega_t);
    const v3 t_j = add(t_n, t_t);
    const double sigma_max = vlen(f_n) / A + vlen(t_t) * R_bar / I;
    const double tau_max = vlen(f_t) / A + vlen(t_n) * R_bar / J;
    if (sigma_max >= s->sigma_b || tau_max >= s->tau_b) {
        s->bonds[2 * (size_t)idx] = s->nb0;
        return;
    }
    double *bd = &s->bonds_delta[4 * (size_t)idx], *bo = &s->bonds_omega[4 * (size_t)idx];
    bd[0] = delta_t.x; bd[1] = delta_t.y; bd[2] = delta_t.z; bd[3] = delta_n;
    bo[0] = omega_t.x; bo[1] = omega_t.y; bo[2] = omega_t.z; bo[3] = omega_n;
    double *fi = &s->force[4 * (size_t)bi], *fj = &s->force[4 * (size_t)bj];
    double *ti = &s->torque[4 * (size_t)bi], *tj = &s->torque[4 * (size_t)bj];
    fi[0] += f.x; fi[1] += f.y; fi[2] += f.z; fi[3] += 0.0;
    fj[0] -= f.x; fj[1] -= f.y; fj[2] -= f.z; fj[3] -= 0.0;
    ti[0] -= t_j.x; ti[1] -= t_j.y; ti[2] -= t_j.z; ti[3] -= 0.0;
    tj[0] += t_j.x; tj[1] += t_j.y; tj[2] += t_j.z; tj[3] += 0.0;
}

/* ---- integrate: src/integration.cuh:9-187 ------------------------------- */
static void integrate_one(orc_scene *s, work_t *w, uint32_t k)
{
    const uint32_t o = s->perm[k];
    const size_t q = 4 * (size_t)o;
    const double *force = &s->force[q], *torque = &s->torque[q];
    double angpos[4], acc[4], angacc[4], vel0[4], angvel0[4], x[4], vel[4], angvel[4];
    memcpy(angpos, &s->angpos[q], sizeof angpos);
    memcpy(acc, &s->acc[q], sizeof acc);
    memcpy(angacc, &s->angacc[q], sizeof angacc);
    memcpy(vel0, &s->vel0[q], sizeof vel0);
    memcpy(angvel0, &s->angvel0[q], sizeof angvel0);
    memcpy(x, &w->x_s[4 * (size_t)k], sizeof x);
    memcpy(vel, &w->vel_s[4 * (size_t)k], sizeof vel);
    memcpy(angvel, &w->angvel_s[4 * (size_t)k], sizeof angvel);
    const double radius = x[3];
    double xysum[2] = {0.0f, 0.0f};
    const double dt = s->dt;
    const double m = 4.0 / 3.0 * REF_PI * radius * radius * radius * s->rho;
    acc[0] = force[0] / m;
    acc[1] = force[1] / m;
    acc[2] = force[2] / m;
    angacc[0] = torque[0] * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc[1] = torque[1] * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc[2] = torque[2] * 1.0 / (2.0 / 5.0 * m * radius * radius);
    acc[0] += s->g[0];
    acc[1] += s->g[1];
    acc[2] += s->g[2];
    if (vel[3] > 0.0f) {
        acc[0] = 0.0;
        acc[1] = 0.0;
        acc[2] -= s->g[2];
        angacc[0] = angacc[1] = angacc[2] = angacc[3] = 0.0f;
    }
    if (s->periodic == 1) {
        if (x[0] < s->origo[0]) x[0] += s->L[0];
        if (x[0] > s->L[0]) x[0] -= s->L[0];
        if (x[1] < s->origo[1]) x[1] += s->L[1];
        if (x[1] > s->L[1]) x[1] -= s->L[1];
    } else if (s->periodic == 2) {
        if (x[0] < s->origo[0]) x[0] += s->L[0];
        if (x[0] > s->L[0]) x[0] -= s->L[0];
    }
    for (int d = 0; d < 3; ++d) vel0[d] += acc[d] * dt;
    for (int d = 0; d < 3; ++d) angvel0[d] += angacc[d] * dt;
    for (int d = 0; d < 3; ++d) x[d] += vel0[d] * dt;
    for (int d = 0; d < 3; ++d) angpos[d] += angvel0[d] * dt;
    for (int d = 0; d < 3; ++d) vel[d] = vel0[d] + 0.5 * acc[d] * dt;
    for (int d = 0; d < 3; ++d) angvel[d] = angvel0[d] + 0.5 * angacc[d] * dt;
    xysum[0] += vel[0] * dt;
    xysum[1] += vel[1] * dt;
    s->xysum[2 * (size_t)o] += xysum[0];
    s->xysum[2 * (size_t)o + 1] += xysum[1];
    memcpy(&s->acc[q], acc, sizeof acc);
    memcpy(&s->angacc[q], angacc, sizeof angacc);
    memcpy(&s->angvel[q], angvel, sizeof angvel);
    memcpy(&s->angvel0[q], angvel0, sizeof angvel0);
    memcpy(&s->vel[q], vel, sizeof vel);
    memcpy(&s->vel0[q], vel0, sizeof vel0);
    memcpy(&s->angpos[q], angpos, sizeof angpos);
    memcpy(&s->x[q], x, sizeof x);
}

/* ---- summation + integrateWalls: src/integration.cuh:191-295 ------------ */
/* The wall-0 force is summed exactly as the reference GPU kernels do: blocks
 * of 256 particles reduced by a halving tree (integration.cuh:197-216), then
 * the block partials added in block order (integration.cuh:249-252). */
static double wall_force_sum(const work_t *w)
{
    const uint32_t np = w->np;
    const uint32_t nblk = (np + 255u) / 256u;
    double total = 0.0;
    double cache[256];
    for (uint32_t b = 0; b < nblk; ++b) {
        for (uint32_t t = 0; t < 256; ++t) {
            uint32_t idx = b * 256u + t;
            double temp = 0.0f;
            if (idx < np) temp += w->wf_pp[idx];
            cache[t] = temp;
        }
        for (uint32_t i = 128; i != 0; i /= 2)
            for (uint32_t t = 0; t < i; ++t) cache[t] += cache[t + i];
        total += cache[0];
    }
    return total;
}

static void integrate_walls(orc_scene *s, const work_t *w, double t_current)
{
    if (s->nw == 0) return;
    const double fsum = wall_force_sum(w);
    for (uint32_t i = 0; i < s->nw; ++i) {
        double *nx = &s->walls_nx[4 * i], *mvfd = &s->walls_mvfd[4 * i];
        int wmode = s->wmode[i];
        double vel0 = s->walls_vel0[i];
        if (wmode == 0) continue;
        mvfd[2] = 0.0;
        mvfd[2] += fsum;
        const double dt = s->dt;
        double sigma_0 = mvfd[3] + s->devs_A * sin(2.0 * 3.141596654 * s->devs_f * t_current);
        double N = -sigma_0 * s->L[0] * s->L[1];
        double acc = (mvfd[2] + N) / mvfd[0];
        if (wmode == 2) acc = 0.0;
        vel0 += acc * dt;
        nx[3] += vel0 * dt;
        mvfd[1] = vel0 + 0.5 * acc * dt;
        s->walls_vel0[i] = vel0;
    }
}

/* ---- Darcy flow: src/darcy.cuh ------------------------------------------
 * The six kernels the time loop runs between bondsLinear and integrate when
 * darcy == 1 and nu > 0 (src/device.cu:913-1021), each over the interior
 * nodes, in that order.  The fluid grid is the cell grid plus one ghost node
 * on every side. */
static const double D_PI = 3.14159265358979323846;   /* M_PI */

/* node (x, y, z) with ghosts at -1 and num; src/darcy.cuh:125-135 */
static inline size_t d_idx(const orc_scene *s, int x, int y, int z)
{
    const size_t nx2 = (size_t)s->num[0] + 2, ny2 = (size_t)s->num[1] + 2;
    return (size_t)(x + 1) + nx2 * (size_t)(y + 1) + nx2 * ny2 * (size_t)(z + 1);
}

/* findPorositiesSphericalDev, src/darcy.cuh:338-477: the void fraction of a
 * sphere of radius min(dx,dy,dz)/2 at the cell centre (measured from the
 * origin, not from origo), from the lens-shaped overlaps of the particles of
 * the 27 neighbour cells, visited z, y, x outermost to innermost and in
 * sorted order within a cell; clamped to [0.1, 0.9].  The change is zero in
 * the run's first step. */
static void darcy_porosity(orc_scene *s, const work_t *w, uint32_t x, uint32_t y, uint32_t z)
{
    const uint32_t nx = s->num[0], ny = s->num[1], nz = s->num[2];
    const double dx = s->L[0] / nx, dy = s->L[1] / ny, dz = s->L[2] / nz;
    const double R = fmin(dx, fmin(dy, dz)) * 0.5;
    const double cell_volume = 4.0 / 3.0 * D_PI * R * R * R;
    double void_volume = cell_volume;
    const v3 X = mk(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
    const size_t me = d_idx(s, (int)x, (int)y, (int)z);
    const double phi_0 = s->d_phi[me];
    for (int oz = -1; oz < 2; ++oz)
        for (int oy = -1; oy < 2; ++oy)
            for (int ox = -1; ox < 2; ++ox) {
                int32_t c[3] = {(int32_t)x + ox, (int32_t)y + oy, (int32_t)z + oz};
                v3 dm = mk(0.0, 0.0, 0.0);
                if (dist_mod(s, c, &dm) == -1) continue;
                const uint32_t cid = (uint32_t)c[0] + (uint32_t)c[1] * nx + (nx * ny) * (uint32_t)c[2];
                const uint32_t beg = s->cell_start[cid];
                if (beg == 0xffffffffu) continue;
                const uint32_t end = s->cell_end[cid];
                for (uint32_t i = beg; i < end; ++i) {
                    const double *xr = &w->x_s[4 * (size_t)i];
                    const double r = xr[3];
                    const v3 dist = add(mk(X.x - xr[0], X.y - xr[1], X.z - xr[2]), dm);
                    const double d = vlen(dist);
                    if ((R - r) < d && d < (R + r))
                        void_volume -= 1.0 / (12.0 * d) *
                                       (D_PI * (R + r - d) * (R + r - d) *
                                        (d * d + 2.0 * d * r - 3.0 * r * r + 2.0 * d * R +
                                         6.0 * r * R - 3.0 * R * R));
                    if (d <= R - r) void_volume -= 4.0 / 3.0 * D_PI * r * r * r;
                }
            }
    const double phi = fmin(0.9, fmax(0.1, void_volume / cell_volume));
    s->d_phi[me] = phi;
    s->d_dphi[me] = (s->iteration == 0) ? 0.0 : phi - phi_0;
}

/* findDarcyTransmissivitiesDev, src/darcy.cuh:480-538: Kozeny-Carman
 * conductivity from the porosity, and the transmissivity K * (dx, dy, dz). */
static void darcy_transmissivity(orc_scene *s, uint32_t x, uint32_t y, uint32_t z)
{
    const double dx = s->L[0] / s->num[0], dy = s->L[1] / s->num[1], dz = s->L[2] / s->num[2];
    const double rho = 1000.0;
    const size_t me = d_idx(s, (int)x, (int)y, (int)z);
    const double phi = s->d_phi[me];
    const double k = phi * phi * phi / ((1.0 - phi) * (1.0 - phi)) * s->d_factor;
    const double K = k * rho * -s->g[2] / s->nu;
    s->d_K[me] = K;
    s->d_T[3 * me + 0] = K * dx;
    s->d_T[3 * me + 1] = K * dy;
    s->d_T[3 * me + 2] = K * dz;
}

/* copyDarcyValsDev, src/darcy.cuh:137-166: every field of node `from`
 * onto node `to` */
static void darcy_copy_node(orc_scene *s, size_t from, size_t to)
{
    double *H = s->d_Hbuf[s->d_hsel], *Hn = s->d_Hbuf[1 - s->d_hsel];
    H[to] = H[from];
    Hn[to] = Hn[from];
    for (int c = 0; c < 3; ++c) {
        s->d_V[3 * to + c] = s->d_V[3 * from + c];
        s->d_dH[3 * to + c] = s->d_dH[3 * from + c];
        s->d_T[3 * to + c] = s->d_T[3 * from + c];
    }
    s->d_K[to] = s->d_K[from];
    s->d_Ss[to] = s->d_Ss[from];
    s->d_W[to] = s->d_W[from];
    s->d_phi[to] = s->d_phi[from];
    s->d_dphi[to] = s->d_dphi[from];
}

/* setDarcyGhostNodesDev, src/darcy.cuh:169-261: a boundary node is copied
 * onto the ghost node on the opposite side of the grid (faces only) */
static void darcy_ghosts(orc_scene *s, uint32_t x, uint32_t y, uint32_t z)
{
    const int nx = (int)s->num[0], ny = (int)s->num[1], nz = (int)s->num[2];
    const int X = (int)x, Y = (int)y, Z = (int)z;
    const size_t me = d_idx(s, X, Y, Z);
    if (X == 0) darcy_copy_node(s, me, d_idx(s, nx, Y, Z));
    if (X == nx - 1) darcy_copy_node(s, me, d_idx(s, -1, Y, Z));
    if (Y == 0) darcy_copy_node(s, me, d_idx(s, X, ny, Z));
    if (Y == ny - 1) darcy_copy_node(s, me, d_idx(s, X, -1, Z));
    if (Z == 0) darcy_copy_node(s, me, d_idx(s, X, Y, nz));
    if (Z == nz - 1) darcy_copy_node(s, me, d_idx(s, X, Y, -1));
}

static inline double d_hmean(double a, double b) { return (2.0 * a * b) / (a + b); }

/* explDarcyStepDev, src/darcy.cuh:604-725: explicit finite-difference step
 * of the pressure into H_new, with zero flux through the z faces */
static void darcy_explicit(orc_scene *s, uint32_t x, uint32_t y, uint32_t z)
{
    const uint32_t nz = s->num[2];
    const double dx = s->L[0] / s->num[0], dy = s->L[1] / s->num[1], dz = s->L[2] / s->num[2];
    const int X = (int)x, Y = (int)y, Z = (int)z;
    const double *H = s->d_Hbuf[s->d_hsel];
    double *Hn = s->d_Hbuf[1 - s->d_hsel];
    const double *T = s->d_T;
    const size_t me = d_idx(s, X, Y, Z);
    const size_t xn = d_idx(s, X - 1, Y, Z), xp = d_idx(s, X + 1, Y, Z);
    const size_t yn = d_idx(s, X, Y - 1, Z), yp = d_idx(s, X, Y + 1, Z);
    const size_t zn = d_idx(s, X, Y, Z - 1), zp = d_idx(s, X, Y, Z + 1);
    const double Ss = s->d_Ss[me], Q = s->d_W[me], dphi = s->d_dphi[me], Hc = H[me];
    const double TdH_xn = d_hmean(T[3 * me + 0], T[3 * xn + 0]) * (H[xn] - Hc) / (dx * dx);
    const double TdH_xp = d_hmean(T[3 * me + 0], T[3 * xp + 0]) * (H[xp] - Hc) / (dx * dx);
    const double TdH_yn = d_hmean(T[3 * me + 1], T[3 * yn + 1]) * (H[yn] - Hc) / (dy * dy);
    const double TdH_yp = d_hmean(T[3 * me + 1], T[3 * yp + 1]) * (H[yp] - Hc) / (dy * dy);
    double TdH_zn = d_hmean(T[3 * me + 2], T[3 * zn + 2]) * (H[zn] - Hc) / (dz * dz);
    double TdH_zp = d_hmean(T[3 * me + 2], T[3 * zp + 2]) * (H[zp] - Hc) / (dz * dz);
    const double dx_bar = (dx + dy + dz) / 3.0;
    if (z == 0) TdH_zn = 0.0;
    if (z == nz - 1) TdH_zp = 0.0;
    const double laplacianH = TdH_xn + TdH_xp + TdH_yn + TdH_yp + TdH_zn + TdH_zp;
    const double porevol = -dx_bar * dphi / s->dt;
    const double deltaH = s->dt / (Ss * dx * dy * dz) * (laplacianH + Q + porevol);
    Hn[me] = fmax(0.0, Hc + deltaH);
}

/* findDarcyGradientsDev + findDarcyVelocitiesDev, src/darcy.cuh:541-598 and
 * 728-776: central-difference pressure gradient (after the swap, so from the
 * new pressure and the ghost values set before the step), flux -K/nu dH and
 * the pore velocity flux / phi */
static void darcy_grad_vel(orc_scene *s, uint32_t x, uint32_t y, uint32_t z)
{
    const double dx = s->L[0] / s->num[0], dy = s->L[1] / s->num[1], dz = s->L[2] / s->num[2];
    const int X = (int)x, Y = (int)y, Z = (int)z;
    const double *H = s->d_Hbuf[s->d_hsel];
    const size_t me = d_idx(s, X, Y, Z);
    const double gx = (H[d_idx(s, X + 1, Y, Z)] - H[d_idx(s, X - 1, Y, Z)]) / (2.0 * dx);
    const double gy = (H[d_idx(s, X, Y + 1, Z)] - H[d_idx(s, X, Y - 1, Z)]) / (2.0 * dy);
    const double gz = (H[d_idx(s, X, Y, Z + 1)] - H[d_idx(s, X, Y, Z - 1)]) / (2.0 * dz);
    s->d_dH[3 * me + 0] = gx;
    s->d_dH[3 * me + 1] = gy;
    s->d_dH[3 * me + 2] = gz;
    const double nu = s->nu, K = s->d_K[me], phi = s->d_phi[me];
    const double qx = -K / nu * gx, qy = -K / nu * gy, qz = -K / nu * gz;
    s->d_V[3 * me + 0] = qx / phi;
    s->d_V[3 * me + 1] = qy / phi;
    s->d_V[3 * me + 2] = qz / phi;
}

/* the Darcy block of one step, src/device.cu:913-1021 */
static void darcy_step(orc_scene *s, const work_t *w, int nt)
{
    const int64_t nx = s->num[0], ny = s->num[1], nz = s->num[2], n = nx * ny * nz;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i)
        darcy_porosity(s, w, (uint32_t)(i % nx), (uint32_t)(i / nx % ny), (uint32_t)(i / (nx * ny)));
    for (int64_t i = 0; i < n; ++i)
        darcy_transmissivity(s, (uint32_t)(i % nx), (uint32_t)(i / nx % ny), (uint32_t)(i / (nx * ny)));
    for (int64_t i = 0; i < n; ++i)
        darcy_ghosts(s, (uint32_t)(i % nx), (uint32_t)(i / nx % ny), (uint32_t)(i / (nx * ny)));
    for (int64_t i = 0; i < n; ++i)
        darcy_explicit(s, (uint32_t)(i % nx), (uint32_t)(i / nx % ny), (uint32_t)(i / (nx * ny)));
    s->d_hsel ^= 1u;
    for (int64_t i = 0; i < n; ++i)
        darcy_grad_vel(s, (uint32_t)(i % nx), (uint32_t)(i / nx % ny), (uint32_t)(i / (nx * ny)));
}

int orc_kind(void) { return 1; }

int orc_threads(int nthreads)
{
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

int orc_step(orc_scene *s, uint64_t nsteps, int nthreads)
{
    if (!s || s->np == 0 || s->nw > ORC_MAXWALLS) return ORC_ERR_BAD_INPUT;
    if (s->contactmodel < 1 || s->contactmodel > 3) return ORC_ERR_BAD_INPUT;
    const uint64_t nc64 = (uint64_t)s->num[0] * s->num[1] * s->num[2];
    if (nc64 == 0 || nc64 >= 0xffffffffull) return ORC_ERR_BAD_INPUT;
    work_t w;
    if (work_alloc(&w, s->np, (uint32_t)nc64) != 0) return ORC_ERR_BAD_INPUT;
    const int nt = orc_threads(nthreads);
    int err = 0;
    for (uint64_t step = 0; step < nsteps; ++step) {
        err |= build_cells(s, &w);
        int e_topo = 0, e_int = 0;
        /* models 2 and 3 keep contact history (device.cu:805) */
        if (s->contactmodel != 1) {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(| : e_topo)
            for (int64_t a = 0; a < (int64_t)s->np; ++a)
                e_topo |= topology_one(s, &w, (uint32_t)a);
        }
        err |= e_topo;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(| : e_int)
        for (int64_t a = 0; a < (int64_t)s->np; ++a) e_int |= interact_one(s, &w, (uint32_t)a);
        err |= e_int;
        for (uint32_t b = 0; b < s->nb0; ++b) bond_one(s, b);
        if (s->darcy == 1 && s->nu > 0.0) darcy_step(s, &w, nt);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t k = 0; k < (int64_t)s->np; ++k) integrate_one(s, &w, (uint32_t)k);
        integrate_walls(s, &w, s->t_current);
        s->t_current += s->dt;
        s->iteration++;
    }
    if (s->wall0_force) memcpy(s->wall0_force, w.wf_pp, sizeof(double) * s->np);
    work_free(&w);
    return err;
}
