/*
 * oracle/ref_render.cpp -- the reference's ray-tracer kernels
 * (src/raytracer.cuh:14-263) driven over one image.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/oracle.h).  oracle/Makefile compiles
 * the kernels from the reference's own file into _ref/raytracer_kernels.o:
 * the file's host part (DEM::cameraInit onwards, which launches the kernels
 * with <<< >>> syntax) is cut off in the pipe to the compiler.  Here they
 * run in one-thread blocks, one block per pixel, after the camera of
 * *cam is put into their __constant__ values.  The camera itself comes from
 * the caller (the plain-C restatement computes it).
 */
#define REF_CONSTANT_EXTERN
#include "ref_shim.h"

#include "vector_arithmetic.h"
#include "constants.cuh"

#include "oracle.h"

#include <vector>

/* the reference's kernels, src/raytracer.cuh:14-263 */
void imageInit(unsigned char *dev_img, unsigned int pixels);
void rayInitPerspective(float4 *dev_ray_origo, float4 *dev_ray_direction, float4 eye,
                        unsigned int width, unsigned int height);
void rayIntersectSpheres(float4 *dev_ray_origo, float4 *dev_ray_direction, Float4 *dev_x,
                         unsigned char *dev_img);
void rayIntersectSpheresColormap(float4 *dev_ray_origo, float4 *dev_ray_direction, Float4 *dev_x,
                                 Float4 *dev_vel, Float *dev_linarr, float max_val,
                                 float lower_cutoff, unsigned char *dev_img);

extern "C" int orc_render_rows(const orc_render *r, const orc_camera *cam, uint8_t *rgba,
                               uint32_t row0, uint32_t nrows, int nthreads);

extern "C" int orc_render_image(const orc_render *r, const orc_camera *cam, uint8_t *rgba,
                                int nthreads)
{
    return orc_render_rows(r, cam, rgba, 0, r ? r->height : 0, nthreads);
}

extern "C" int orc_render_rows(const orc_render *r, const orc_camera *cam, uint8_t *rgba,
                               uint32_t row0, uint32_t nrows, int nthreads)
{
    if (!r || !cam || !rgba || r->width == 0 || r->height == 0) return ORC_ERR_BAD_INPUT;
    if (r->method < 0 || r->method > 5 || (r->method > 0 && !r->values)) return ORC_ERR_BAD_INPUT;
    if (row0 > r->height || nrows > r->height - row0) return ORC_ERR_BAD_INPUT;
    const unsigned int W = r->width, H = r->height, pixels = W * H;
    const long first = (long)row0 * W, last = first + (long)nrows * W;
    /* DEM::cameraInit's cudaMemcpyToSymbol calls (src/raytracer.cuh:290-297) */
    devC_u = make_float3(cam->u[0], cam->u[1], cam->u[2]);
    devC_v = make_float3(cam->v[0], cam->v[1], cam->v[2]);
    devC_w = make_float3(cam->w[0], cam->w[1], cam->w[2]);
    devC_eye = make_float3(cam->eye[0], cam->eye[1], cam->eye[2]);
    devC_imgplane = make_float4(cam->imgplane[0], cam->imgplane[1], cam->imgplane[2],
                                cam->imgplane[3]);
    devC_d = cam->d;
    devC_light = make_float3(cam->light[0], cam->light[1], cam->light[2]);
    devC_pixels = pixels;
    devC_np = r->np;
    std::vector<float4> origo(pixels), dir(pixels);
    std::vector<unsigned char> img((size_t)pixels * 4, 0);
    Float4 *x = (Float4 *)const_cast<double *>(r->x);
    Float4 *vel = (Float4 *)const_cast<double *>(r->vel);
    Float *values = const_cast<double *>(r->values);
    const int nt = orc_threads(nthreads);
    blockDim = dim3(1, 1, 1);
    gridDim = dim3(pixels, 1, 1);
    auto at = [](long m) {
        blockIdx.x = (unsigned int)m;
        threadIdx.x = 0;
    };
    /* the reference's bound test lets thread `pixels` through
     * (src/raytracer.cuh:19, 36, 62); only the image's own pixels run here */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long m = first; m < last; ++m) {
        at(m);
        imageInit(img.data(), pixels);
        rayInitPerspective(origo.data(), dir.data(),
                           make_float4(cam->eye[0], cam->eye[1], cam->eye[2], 0.0f), W, H);
    }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (long m = first; m < last; ++m) {
        at(m);
        if (r->method == 0)
            rayIntersectSpheres(origo.data(), dir.data(), x, img.data());
        else
            rayIntersectSpheresColormap(origo.data(), dir.data(), x, vel, values, r->maxval,
                                        r->lower_cutoff, img.data());
    }
    for (size_t m = (size_t)first; m < (size_t)last; ++m) {
        rgba[4 * m + 0] = img[4 * m + 0];
        rgba[4 * m + 1] = img[4 * m + 1];
        rgba[4 * m + 2] = img[4 * m + 2];
        rgba[4 * m + 3] = 0;
    }
    return ORC_OK;
}
