// render.cu -- the reference's ray tracer (src/raytracer.cuh:14-553,
// DEM::render) on the context's current particle state.
//
// The reference shades each pixel by the sphere its viewing line meets
// nearest to the eye, testing every sphere for every pixel (np x pixels
// tests, in particle order, keeping a strictly smaller |t|: the lowest
// particle index wins a tie).  Here each sphere is splatted onto the pixels
// it can touch, and each pixel keeps the smallest 64-bit key
// (float bits of |t|, particle index), which is that same choice:
//   k_rt_values   the colour-map value of every particle (methods 1-5);
//   k_rt_splat    one thread per particle: a conservative pixel box, then,
//                 for each pixel in it, the reference's ray and
//                 discriminant arithmetic and an atomicMin of the key;
//   k_rt_resolve  one thread per pixel: the winner's hit point, normal and
//                 shading, or the white background.
// Arithmetic is IEEE single precision without contraction, in the
// reference's operand order; the reference's GPU build used --use_fast_math,
// whose approximate division and square roots are not reproduced, and a
// vector is normalised as v * (1 / sqrt(v.v)), the host form of the
// normalize() it calls.
//
// The pixel box.  For the float vectors d (ray direction) and ec = e - c
// the reference draws the sphere where its discriminant
//   4 (d.ec)^2 - 4 (d.d) (ec.ec - R^2)
// evaluates positive.  In exact arithmetic that is dist^2 < R^2, dist the
// distance from c to the line e + t d.  The float evaluation errs by at most
// 4 |d|^2 (16 u |ec|^2 + 6 u R^2) to first order (u = 2^-24: three-term dot
// products, two squarings, a subtraction), so a positive result needs
//   dist^2 < R^2 (1 + 6u) + 16 u |ec|^2.
// The box is the image of the ball around c with radius
//   sqrt(R^2 (1 + 1e-6) + 4e-6 |ec|^2) + 2e-6 (|e| + |c| + |ec| (1 + P / D)),
// about four times those bounds plus the rounding of c, e and d (P: the
// image-plane half extent, D: the focal distance), projected through the
// eye onto the image plane, widened by two pixels.  A ball that reaches the
// plane through the eye parallel to the image plane projects without bound:
// such a sphere is tested against every pixel.
#include "sphk_internal.cuh"

#include <cmath>
#include <vector>

#include "sphk.h"

namespace sphk {

constexpr int RT_BLOCK = 128;

struct Camera {
    float u[3], v[3], w[3], eye[3], light[3];
    float imgplane[4];   // l, r, b, t
    float d;             // focal distance
};

struct RenderArgs {
    Camera cam;
    uint32_t W, H;
    int method;
    float maxval, lower_cutoff;
};

struct fl3 { float x, y, z; };
__device__ __forceinline__ fl3 f3(float x, float y, float z) { return fl3{x, y, z}; }
__device__ __forceinline__ fl3 operator+(fl3 a, fl3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ fl3 operator-(fl3 a, fl3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ fl3 operator-(fl3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ fl3 operator*(float s, fl3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float fdot(fl3 a, fl3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ fl3 fnorm(fl3 v)
{
    const float s = 1.0f / sqrtf(fdot(v, v));
    return f3(v.x * s, v.y * s, v.z * s);
}

// rayInitPerspective (src/raytracer.cuh:27-51) for pixel m: the row index
// is the quotient modulo the width there
__device__ __forceinline__ fl3 ray_dir(const RenderArgs &g, uint32_t m)
{
    const uint32_t i = m % g.W;
    const uint32_t j = (uint32_t)((int)floorf((float)m / g.W) % (int)g.W);
    const float *ip = g.cam.imgplane;
    const float p_u = ip[0] + (ip[1] - ip[0]) * (i + 0.5f) / g.W;
    const float p_v = ip[2] + (ip[3] - ip[2]) * (j + 0.5f) / g.H;
    const fl3 U = f3(g.cam.u[0], g.cam.u[1], g.cam.u[2]);
    const fl3 V = f3(g.cam.v[0], g.cam.v[1], g.cam.v[2]);
    const fl3 Wv = f3(g.cam.w[0], g.cam.w[1], g.cam.w[2]);
    return (-g.cam.d * Wv + p_u * U) + p_v * V;
}

// The reference's direction is ((-D w) + p_u u) + p_v v (rayInitPerspective,
// in that order): the first sum depends on the column only, the last term on
// the (wrapped) row only.  They are tabulated once per image with the same
// float operations, so a pixel's direction is A[column] + B[row], exactly.
__global__ void __launch_bounds__(RT_BLOCK) k_rt_rays(RenderArgs g, fl3 *A, fl3 *B)
{
    const uint32_t t = blockIdx.x * RT_BLOCK + threadIdx.x;
    if (t >= g.W) return;
    const float *ip = g.cam.imgplane;
    const fl3 U = f3(g.cam.u[0], g.cam.u[1], g.cam.u[2]);
    const fl3 V = f3(g.cam.v[0], g.cam.v[1], g.cam.v[2]);
    const fl3 Wv = f3(g.cam.w[0], g.cam.w[1], g.cam.w[2]);
    const float p_u = ip[0] + (ip[1] - ip[0]) * (t + 0.5f) / g.W;
    A[t] = -g.cam.d * Wv + p_u * U;
    const float p_v = ip[2] + (ip[3] - ip[2]) * (t + 0.5f) / g.H;
    B[t] = p_v * V;
}

// the reference's intersection (src/raytracer.cuh:84-108): true when the
// discriminant is positive and |t_minus| < 1e10, with |t_minus| in *t
__device__ __forceinline__ bool intersect(fl3 d, fl3 ec, float R, float *t)
{
    const float Delta = (2.0f * fdot(d, ec)) * (2.0f * fdot(d, ec)) -
                        4.0f * fdot(d, d) * (fdot(ec, ec) - R * R);
    if (!(Delta > 0.0f)) return false;
    const float t_minus =
        ((fdot(-d, ec) - sqrtf(fdot(d, ec) * fdot(d, ec) - fdot(d, d) * (fdot(ec, ec) - R * R))) /
         fdot(d, d));
    *t = fabsf(t_minus);
    if (!(*t < 1e10f)) return false;   // NaN, or beyond the initial distance
    return true;
}

// DEM::render's colour-map values (src/raytracer.cuh:396-452), by storage index
__global__ void __launch_bounds__(RT_BLOCK) k_rt_values(Dev d, int A, int method, double *out)
{
    const uint32_t s = blockIdx.x * RT_BLOCK + threadIdx.x;
    if (s >= d.np_all) return;
    double v = 0.0;
    P3 a;
    switch (method) {
    case 1: v = d.edp[s].z; break;
    case 2: a = d.vel[A][s]; v = sqrt(a.x * a.x + a.y * a.y + a.z * a.z); break;
    case 3: a = d.angvel[A][s]; v = sqrt(a.x * a.x + a.y * a.y + a.z * a.z); break;
    case 4: v = d.xysum[s].x; break;
    case 5: a = d.angpos[s]; v = sqrt(a.x * a.x + a.y * a.y + a.z * a.z); break;
    default: break;
    }
    out[s] = v;
}

// DEM::maxPos (src/sphere.cpp:520-548): the largest coordinate on each axis,
// starting from zero; a max is order-free, so any reduction order gives it
__global__ void __launch_bounds__(RT_BLOCK) k_rt_maxpos(Dev d, int A, unsigned long long *mx)
{
    const uint32_t s = blockIdx.x * RT_BLOCK + threadIdx.x;
    double m[3] = {0.0, 0.0, 0.0};
    if (s < d.np_all) {
        const double4 x = d.xr[A][s];
        m[0] = x.x > 0.0 ? x.x : 0.0;
        m[1] = x.y > 0.0 ? x.y : 0.0;
        m[2] = x.z > 0.0 ? x.z : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = m[k];
        for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        // non-negative doubles order as their bit patterns
        if ((threadIdx.x & 31u) == 0) atomicMax(&mx[k], (unsigned long long)__double_as_longlong(v));
    }
}

__global__ void __launch_bounds__(RT_BLOCK)
k_rt_splat(Dev d, int A, RenderArgs g, const double *values, const fl3 *__restrict__ colA,
           const fl3 *__restrict__ rowB, unsigned long long *keys)
{
    const uint32_t s = blockIdx.x * RT_BLOCK + threadIdx.x;
    if (s >= d.np_all) return;
    const double4 x = d.xr[A][s];
    const uint32_t uid = d.uid[s];
    if (g.method > 0 && g.lower_cutoff > 0.0) {
        // rayIntersectSpheresColormap's filter (src/raytracer.cuh:185-199)
        const float val = (float)values[s];
        const float fixvel = (float)d.w_user[(size_t)uid * WLANES + W_VEL];
        if (!(val > g.lower_cutoff && fixvel == 0.f)) return;
    }
    const fl3 c = f3((float)x.x, (float)x.y, (float)x.z);
    const float R = (float)x.w;
    const fl3 e = f3(g.cam.eye[0], g.cam.eye[1], g.cam.eye[2]);
    const fl3 ec = e - c;
    const uint64_t idx = uid;

    // ---- the pixel box (double precision; see the top of the file) ----
    const double qx = (double)c.x - e.x, qy = (double)c.y - e.y, qz = (double)c.z - e.z;
    const double nb = sqrt(qx * qx + qy * qy + qz * qz);
    const double ne = sqrt((double)e.x * e.x + (double)e.y * e.y + (double)e.z * e.z);
    const double nc = sqrt((double)c.x * c.x + (double)c.y * c.y + (double)c.z * c.z);
    const double D = g.cam.d;
    const float *ip = g.cam.imgplane;
    const double P = fmax(fmax(fabs((double)ip[0]), fabs((double)ip[1])),
                          fmax(fabs((double)ip[2]), fabs((double)ip[3])));
    const double rho = sqrt((double)R * R * (1.0 + 1e-6) + 4e-6 * nb * nb) +
                       2e-6 * (ne + nc + nb * (1.0 + P / D));
    const double a0 = qx * g.cam.u[0] + qy * g.cam.u[1] + qz * g.cam.u[2];
    const double b0 = qx * g.cam.v[0] + qy * g.cam.v[1] + qz * g.cam.v[2];
    const double c0 = qx * g.cam.w[0] + qy * g.cam.w[1] + qz * g.cam.w[2];
    if (!isfinite(rho) || !isfinite(a0) || !isfinite(b0) || !isfinite(c0)) return;   // no hit
    const int W = (int)g.W;
    int i0 = 0, i1 = W - 1, j0 = 0, j1 = W - 1;   // j: the wrapped row index
    const double r2 = rho * (1.0 + 1e-6);
    if (c0 * c0 > r2 * r2) {
        // image-plane coordinate -D * (along / depth) over the ball
        auto range = [&](double p0, double lo_img, double hi_img, int n, int &lo, int &hi) {
            const double den = c0 * c0 - r2 * r2;
            const double root = r2 * sqrt(p0 * p0 + c0 * c0 - r2 * r2);
            const double k1 = (p0 * c0 + root) / den, k2 = (p0 * c0 - root) / den;
            const double pa = -D * k1, pb = -D * k2;
            if (!isfinite(pa) || !isfinite(pb)) return;   // keep the whole range
            const double plo = fmin(pa, pb), phi = fmax(pa, pb);
            const double span = hi_img - lo_img;
            if (span == 0.0) {
                // every column (row) has the same coordinate
                if (lo_img < plo - 1e-6 * (fabs(plo) + D) || lo_img > phi + 1e-6 * (fabs(phi) + D)) {
                    lo = 1; hi = 0;
                }
                return;
            }
            const double f_lo = (plo - lo_img) * n / span - 0.5, f_hi = (phi - lo_img) * n / span - 0.5;
            if (!isfinite(f_lo) || !isfinite(f_hi)) return;
            const double a = fmin(f_lo, f_hi), b = fmax(f_lo, f_hi);
            lo = (int)fmax(-1.0, fmin((double)n, floor(a) - 2.0));
            hi = (int)fmax(-1.0, fmin((double)n, ceil(b) + 2.0));
        };
        range(a0, ip[0], ip[1], (int)g.W, i0, i1);
        range(b0, ip[2], ip[3], (int)g.H, j0, j1);
        i0 = max(i0, 0);
        i1 = min(i1, W - 1);
        j0 = max(j0, 0);
        j1 = min(j1, W - 1);
    }
    if (i0 > i1 || j0 > j1) return;
    // rows y whose wrapped index y mod W lies within [j0 - 1, j1 + 1]; the
    // exact row index of each pixel is recomputed as the reference does
    const uint32_t H = g.H;
    for (uint32_t base = 0; base < H; base += (uint32_t)W) {
        const int ylo = (int)base + max(j0 - 1, 0), yhi = (int)base + min(j1 + 1, W - 1);
        for (int y = ylo; y <= yhi && y < (int)H; ++y) {
            // the row index floor((float)m / W) mod W does not decrease with
            // m: equal at both ends of the box's row, it is the row's own
            const uint32_t mrow = (uint32_t)y * g.W;
            const uint32_t ja = (uint32_t)((int)floorf((float)(mrow + i0) / g.W) % (int)g.W);
            const uint32_t jb = (uint32_t)((int)floorf((float)(mrow + i1) / g.W) % (int)g.W);
            const fl3 Bj = rowB[ja];
            for (int xi = i0; xi <= i1; ++xi) {
                const uint32_t m = mrow + (uint32_t)xi;
                fl3 dir;
                if (ja == jb) {
                    dir = colA[xi] + Bj;
                } else {
                    const uint32_t j = (uint32_t)((int)floorf((float)m / g.W) % (int)g.W);
                    dir = colA[xi] + rowB[j];
                }
                float t;
                if (!intersect(dir, ec, R, &t)) continue;
                const unsigned long long key = ((unsigned long long)__float_as_uint(t) << 32) | idx;
                atomicMin(&keys[m], key);
            }
        }
    }
}

// blue-white-red colour map, src/colorbar.h:7-20
__device__ __forceinline__ float cb_red(float r)
{
    return fminf(1.0f, 0.209f * r * r * r - 2.49f * r * r + 3.0f * r + 0.0109f);
}
__device__ __forceinline__ float cb_green(float r) { return fminf(1.0f, -2.44f * r * r + 2.15f * r + 0.369f); }
__device__ __forceinline__ float cb_blue(float r) { return fminf(1.0f, -2.21f * r * r + 1.61f * r + 0.573f); }

__global__ void __launch_bounds__(RT_BLOCK)
k_rt_resolve(Dev d, int A, RenderArgs g, const double *values, const unsigned long long *keys,
             uchar4 *img)
{
    const uint32_t m = blockIdx.x * RT_BLOCK + threadIdx.x;
    if (m >= g.W * g.H) return;
    const unsigned long long key = keys[m];
    if (key == ~0ull) {
        img[m] = make_uchar4(255, 255, 255, 0);   // imageInit's background
        return;
    }
    const uint32_t uid = (uint32_t)(key & 0xffffffffu);
    const uint32_t s = d.sidx[uid];
    const double4 x = d.xr[A][s];
    const fl3 c = f3((float)x.x, (float)x.y, (float)x.z);
    const float R = (float)x.w;
    const fl3 e = f3(g.cam.eye[0], g.cam.eye[1], g.cam.eye[2]);
    const fl3 ec = e - c;
    const fl3 dir = ray_dir(g, m);
    const float t_minus =
        ((fdot(-dir, ec) - sqrtf(fdot(dir, ec) * fdot(dir, ec) - fdot(dir, dir) * (fdot(ec, ec) - R * R))) /
         fdot(dir, dir));
    const fl3 p = e + t_minus * dir;
    const fl3 n = fnorm(2.0f * (p - c));
    const fl3 light = f3(g.cam.light[0], g.cam.light[1], g.cam.light[2]);
    const float dotprod = fmaxf(0.0f, fdot(n, light));
    const float I_d = 40.0f, k_d = 5.0f, k_a = 10.0f, I_a = 5.0f;
    float cr, cg, cb;
    if (g.method == 0) {
        cr = 0.48f; cg = 0.41f; cb = 0.27f;
    } else {
        const float fixvel = (float)d.w_user[(size_t)uid * WLANES + W_VEL];
        float ratio = (float)(values[s] / (double)g.maxval);
        if (ratio < 0.01f) ratio = 0.01f;
        if (ratio > 0.99f) ratio = 0.99f;
        cr = cb_red(ratio); cg = cb_green(ratio); cb = cb_blue(ratio);
        if (fixvel > 0.f) cr = cg = cb = 0.5f;
    }
    img[m] = make_uchar4((unsigned char)((k_d * I_d * dotprod + k_a * I_a) * cr),
                         (unsigned char)((k_d * I_d * dotprod + k_a * I_a) * cg),
                         (unsigned char)((k_d * I_d * dotprod + k_a * I_a) * cb), 0);
}

void launch_maxpos(const Dev &d, uint32_t np, int a, unsigned long long *mx, cudaStream_t st)
{
    k_rt_maxpos<<<div_up(np, RT_BLOCK), RT_BLOCK, 0, st>>>(d, a, mx);
}

// DEM::render's camera (src/raytracer.cuh:351-367) and DEM::cameraInit
// (src/raytracer.cuh:266-300), in single precision on the host
Camera make_camera(const double L[3], const double maxpos[3], uint32_t W, uint32_t H)
{
    struct h3 { float x, y, z; };
    auto mk3 = [](float x, float y, float z) { return h3{x, y, z}; };
    auto sub = [&](h3 a, h3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); };
    auto dot = [](h3 a, h3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
    auto len = [&](h3 a) { return sqrtf(dot(a, a)); };
    auto divs = [&](h3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); };
    auto cross = [&](h3 a, h3 b) {
        return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    };
    const float imgw = (float)(L[0] * (double)1.35f);
    const h3 lookat = divs(mk3((float)maxpos[0], (float)maxpos[1], (float)maxpos[2]), 2.0f);
    const h3 eye = mk3((float)(L[0] * (double)2.3f), (float)(L[1] * (double)-5.0f),
                       (float)(L[2] * (double)1.3f));
    const float hw_ratio = (float)(H / W);   // unsigned division, as the reference
    Camera c{};
    c.imgplane[0] = -0.5f * imgw;
    c.imgplane[1] = 0.5f * imgw;
    c.imgplane[2] = -0.5f * imgw * hw_ratio;
    c.imgplane[3] = 0.5f * imgw * hw_ratio;
    const h3 view = sub(eye, lookat);
    const h3 up = mk3(0.0f, 0.0f, 1.0f);
    const h3 w = divs(mk3(-view.x, -view.y, -view.z), len(view));
    const h3 u = divs(cross(up, w), len(cross(up, w)));
    const h3 v = cross(w, u);
    const float dist = len(view) * 0.8f;
    const h3 ml = mk3(-1.0f * eye.x * 1.0f, -1.0f * eye.y * 0.2f, -1.0f * eye.z * 0.6f);
    const float inv = 1.0f / sqrtf(dot(ml, ml));
    const h3 light = mk3(ml.x * inv, ml.y * inv, ml.z * inv);
    const h3 *src[5] = {&u, &v, &w, &eye, &light};
    float *dst[5] = {c.u, c.v, c.w, c.eye, c.light};
    for (int k = 0; k < 5; ++k) {
        dst[k][0] = src[k]->x;
        dst[k][1] = src[k]->y;
        dst[k][2] = src[k]->z;
    }
    c.d = dist;
    return c;
}

// One image: the colour-map values, the direction tables, the splat and
// the resolve.  `keys` must hold all ones (no hit) for every pixel; `rays`
// holds 2 * width directions.
int render_image(const Dev &d, uint32_t np, int a, const double L[3], const double maxpos[3],
                 const sph_render_opts &o, double *values, unsigned long long *keys, uchar4 *img,
                 float *rays, cudaStream_t st)
{
    RenderArgs g{};
    g.cam = make_camera(L, maxpos, o.width, o.height);
    g.W = o.width;
    g.H = o.height;
    g.method = o.method;
    g.maxval = o.maxval;
    g.lower_cutoff = o.lower_cutoff;
    const unsigned gp = div_up(np, RT_BLOCK);
    fl3 *colA = reinterpret_cast<fl3 *>(rays), *rowB = colA + g.W;
    if (g.method > 0) k_rt_values<<<gp, RT_BLOCK, 0, st>>>(d, a, g.method, values);
    k_rt_rays<<<div_up(g.W, RT_BLOCK), RT_BLOCK, 0, st>>>(g, colA, rowB);
    k_rt_splat<<<gp, RT_BLOCK, 0, st>>>(d, a, g, values, colA, rowB, keys);
    k_rt_resolve<<<div_up((uint64_t)g.W * g.H, RT_BLOCK), RT_BLOCK, 0, st>>>(d, a, g, values, keys, img);
    return 0;
}

}  // namespace sphk
