/*
 * oracle/ref_inc/helper_math.h -- stand-in for the CUDA samples' helper_math.h
 * (TEST INFRASTRUCTURE ONLY).
 *
 * The reference includes <helper_math.h> (src/device.cu:7, src/darcy.cuh:11)
 * but does not ship it.  Its Darcy kernels use none of it (their vector
 * arithmetic is the reference's own src/vector_arithmetic.h, and int3
 * addition comes from oracle/ref_shim.h); its ray tracer
 * (src/raytracer.cuh) uses the float3 operators below and make_float4 from a
 * float3, written here from
 * their plain definitions: component-wise arithmetic, dot product summed x,
 * y, z in that order, length = sqrtf(dot), and normalize as
 * v * (1 / sqrtf(v . v)), the form the samples' header takes on the host.
 */
#ifndef SPHERE_ORACLE_HELPER_MATH_STANDIN_H_
#define SPHERE_ORACLE_HELPER_MATH_STANDIN_H_

#include <math.h>
#include <vector_functions.h>
#include <vector_types.h>

inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(float3 v) { return sqrtf(dot(v, v)); }
inline float3 normalize(float3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
inline float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

#endif
