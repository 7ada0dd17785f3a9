/*
 * oracle/render_oracle.c -- plain-C restatement of the reference's ray
 * tracer (src/raytracer.cuh:14-553, DEM::render) for one image.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA renderer, never the
 * renderer itself; pinned against the reference's own kernels compiled for
 * the host (oracle/_ref).  Brute force as in the reference: every pixel
 * tests every sphere in particle order.
 *
 * Arithmetic: IEEE single precision, no contraction (built with
 * -ffp-contract=off), every expression in the reference's operand order.
 * The reference's GPU build used --use_fast_math, whose approximate
 * division, square root and reciprocal square root are not reproduced; a
 * vector is normalised as v * (1 / sqrt(v.v)), the host form of the
 * helper_math normalize() the reference calls.
 */
#include "oracle.h"

#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float x, y, z; } f3;

static inline f3 f3mk(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 f3add(f3 a, f3 b) { return f3mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 f3sub(f3 a, f3 b) { return f3mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 f3neg(f3 a) { return f3mk(-a.x, -a.y, -a.z); }
static inline f3 f3smul(float s, f3 a) { return f3mk(s * a.x, s * a.y, s * a.z); }
static inline f3 f3muls(f3 a, float s) { return f3mk(a.x * s, a.y * s, a.z * s); }
static inline f3 f3divs(f3 a, float s) { return f3mk(a.x / s, a.y / s, a.z / s); }
static inline f3 f3mulv(f3 a, f3 b) { return f3mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float f3dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float f3len(f3 a) { return sqrtf(f3dot(a, a)); }
static inline f3 f3cross(f3 a, f3 b)
{
    return f3mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline f3 f3norm(f3 v) { return f3muls(v, 1.0f / sqrtf(f3dot(v, v))); }

/* blue-white-red colour map, src/colorbar.h:7-20 */
static inline float cb_red(float r)
{
    return fminf(1.0f, 0.209f * r * r * r - 2.49f * r * r + 3.0f * r + 0.0109f);
}
static inline float cb_green(float r) { return fminf(1.0f, -2.44f * r * r + 2.15f * r + 0.369f); }
static inline float cb_blue(float r) { return fminf(1.0f, -2.21f * r * r + 1.61f * r + 0.573f); }

void orc_render_camera(const orc_render *r, orc_camera *cam)
{
    /* DEM::render (src/raytracer.cuh:351-367): image-plane width 1.35 L0,
     * eye at (2.3 L0, -5 L1, 1.3 L2), looking at half the largest
     * coordinates (DEM::maxPos, src/sphere.cpp:520-548, starting from 0) */
    const float imgw = (float)(r->L[0] * (double)1.35f);
    double mx = 0.0, my = 0.0, mz = 0.0;
    for (uint32_t i = 0; i < r->np; ++i) {
        const double *p = &r->x[4 * (size_t)i];
        if (p[0] > mx) mx = p[0];
        if (p[1] > my) my = p[1];
        if (p[2] > mz) mz = p[2];
    }
    const f3 lookat = f3divs(f3mk((float)mx, (float)my, (float)mz), 2.0f);
    const f3 eye = f3mk((float)(r->L[0] * (double)2.3f), (float)(r->L[1] * (double)-5.0f),
                        (float)(r->L[2] * (double)1.3f));
    /* DEM::cameraInit (src/raytracer.cuh:269-300); height/width divide as
     * unsigned integers there */
    const float hw_ratio = (float)(r->height / r->width);
    cam->imgplane[0] = -0.5f * imgw;
    cam->imgplane[1] = 0.5f * imgw;
    cam->imgplane[2] = -0.5f * imgw * hw_ratio;
    cam->imgplane[3] = 0.5f * imgw * hw_ratio;
    const f3 view = f3sub(eye, lookat);
    const f3 up = f3mk(0.0f, 0.0f, 1.0f);
    const f3 w = f3divs(f3neg(view), f3len(view));
    const f3 uc = f3cross(up, w);
    const f3 u = f3divs(uc, f3len(f3cross(up, w)));
    const f3 v = f3cross(w, u);
    const float d = f3len(view) * 0.8f;
    const f3 light = f3norm(f3mulv(f3smul(-1.0f, eye), f3mk(1.0f, 0.2f, 0.6f)));
    const f3 *src[5] = {&u, &v, &w, &eye, &light};
    float *dst[5] = {cam->u, cam->v, cam->w, cam->eye, cam->light};
    for (int k = 0; k < 5; ++k) {
        dst[k][0] = src[k]->x;
        dst[k][1] = src[k]->y;
        dst[k][2] = src[k]->z;
    }
    cam->d = d;
}

void orc_render_values(int method, uint32_t np, const double *vel, const double *angvel,
                       const double *angpos, const double *xysum, const double *p, double *out)
{
    /* DEM::render's colour-map arrays (src/raytracer.cuh:396-452) */
    for (uint32_t i = 0; i < np; ++i) {
        const double *a;
        switch (method) {
        case 1: out[i] = p[i]; break;
        case 2: a = &vel[4 * (size_t)i]; out[i] = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); break;
        case 3: a = &angvel[4 * (size_t)i]; out[i] = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); break;
        case 4: out[i] = xysum[2 * (size_t)i]; break;
        case 5: a = &angpos[4 * (size_t)i]; out[i] = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); break;
        default: out[i] = 0.0; break;
        }
    }
}

int orc_render_image(const orc_render *r, const orc_camera *cam, uint8_t *rgba, int nthreads)
{
    return orc_render_rows(r, cam, rgba, 0, r ? r->height : 0, nthreads);
}

int orc_render_rows(const orc_render *r, const orc_camera *cam, uint8_t *rgba, uint32_t row0,
                    uint32_t nrows, int nthreads)
{
    if (!r || !cam || !rgba || r->width == 0 || r->height == 0) return ORC_ERR_BAD_INPUT;
    if (r->method < 0 || r->method > 5 || (r->method > 0 && !r->values)) return ORC_ERR_BAD_INPUT;
    if (row0 > r->height || nrows > r->height - row0) return ORC_ERR_BAD_INPUT;
    const uint32_t W = r->width, H = r->height;
    const int64_t first = (int64_t)row0 * W, pixels = (int64_t)nrows * W;
    const f3 U = f3mk(cam->u[0], cam->u[1], cam->u[2]);
    const f3 V = f3mk(cam->v[0], cam->v[1], cam->v[2]);
    const f3 Wv = f3mk(cam->w[0], cam->w[1], cam->w[2]);
    const f3 e = f3mk(cam->eye[0], cam->eye[1], cam->eye[2]);
    const f3 light = f3mk(cam->light[0], cam->light[1], cam->light[2]);
    const int nt = orc_threads(nthreads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t q = 0; q < pixels; ++q) {
        const int64_t m = first + q;
        /* imageInit (src/raytracer.cuh:14-24): white background */
        uint8_t *px = &rgba[4 * (size_t)m];
        px[0] = px[1] = px[2] = 255;
        px[3] = 0;
        /* rayInitPerspective (src/raytracer.cuh:27-51); the row index wraps
         * modulo the width there */
        const uint32_t i = (uint32_t)(m % W);
        const uint32_t j = (uint32_t)((int)floorf((float)m / W) % (int)W);
        const float p_u = cam->imgplane[0] + (cam->imgplane[1] - cam->imgplane[0]) * (i + 0.5f) / W;
        const float p_v = cam->imgplane[2] + (cam->imgplane[3] - cam->imgplane[2]) * (j + 0.5f) / H;
        const f3 d = f3add(f3add(f3smul(-cam->d, Wv), f3smul(p_u, U)), f3smul(p_v, V));
        /* rayIntersectSpheres / rayIntersectSpheresColormap
         * (src/raytracer.cuh:55-263) */
        float tdist = 1e10f;
        f3 n = f3mk(0.0f, 0.0f, 0.0f);
        uint32_t hit = 0;
        for (uint32_t s = 0; s < r->np; ++s) {
            const double *xs = &r->x[4 * (size_t)s];
            const f3 c = f3mk((float)xs[0], (float)xs[1], (float)xs[2]);
            const float R = (float)xs[3];
            const f3 ec = f3sub(e, c);
            const float Delta = (2.0f * f3dot(d, ec)) * (2.0f * f3dot(d, ec)) -
                                4.0f * f3dot(d, d) * (f3dot(ec, ec) - R * R);
            int take = Delta > 0.0f;
            if (r->method > 0 && r->lower_cutoff > 0.0) {
                const float val = (float)r->values[s];
                const float fixvel = (float)r->vel[4 * (size_t)s + 3];
                take = take && val > r->lower_cutoff && fixvel == 0.f;
            }
            if (!take) continue;
            const float t_minus =
                ((f3dot(f3neg(d), ec) -
                  sqrtf(f3dot(d, ec) * f3dot(d, ec) - f3dot(d, d) * (f3dot(ec, ec) - R * R))) /
                 f3dot(d, d));
            if (fabsf(t_minus) < tdist) {
                const f3 p = f3add(e, f3smul(t_minus, d));
                tdist = fabsf(t_minus);
                n = f3norm(f3smul(2.0f, f3sub(p, c)));
                hit = s;
            }
        }
        if (!(tdist < 1e10f)) continue;
        const float dotprod = fmaxf(0.0f, f3dot(n, light));
        const float I_d = 40.0f, k_d = 5.0f, k_a = 10.0f, I_a = 5.0f;
        if (r->method == 0) {
            px[0] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.48f);
            px[1] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.41f);
            px[2] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.27f);
        } else {
            const float fixvel = (float)r->vel[4 * (size_t)hit + 3];
            float ratio = (float)(r->values[hit] / (double)r->maxval);
            if (ratio < 0.01f) ratio = 0.01f;
            if (ratio > 0.99f) ratio = 0.99f;
            float redv = cb_red(ratio), greenv = cb_green(ratio), bluev = cb_blue(ratio);
            if (fixvel > 0.f) redv = greenv = bluev = 0.5f;
            px[0] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * redv);
            px[1] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * greenv);
            px[2] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * bluev);
        }
    }
    return ORC_OK;
}
