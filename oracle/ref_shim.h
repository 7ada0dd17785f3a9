/*
 * oracle/ref_shim.h -- lets the reference's CUDA kernel bodies compile as
 * host C++ (TEST INFRASTRUCTURE ONLY; see oracle/oracle.h).
 *
 * The kernels are launched one thread per block (blockDim.x == 1) from the
 * harness, so every __syncthreads() is trivially satisfied, except for
 * summation(), which the harness can run with real 256-thread blocks
 * (oracle/ref_integration.cpp).
 *
 * Defines:
 *   __global__, __shared__, __constant__  as storage-class shims;
 *   threadIdx/blockIdx (thread-local, so OpenMP threads can launch kernels
 *   concurrently), blockDim/gridDim;
 *   int3 operator+ (normally from the CUDA samples' helper_math.h, which the
 *   reference includes in src/device.cu:7 but does not ship).
 */
#ifndef SPHERE_REF_SHIM_H_
#define SPHERE_REF_SHIM_H_

#include <vector_types.h>
#include <vector_functions.h>
#include <math.h>

#undef __global__
#define __global__
#undef __shared__
#ifdef REF_SHARED_STATIC
#define __shared__ static
#else
#define __shared__
#endif
#undef __constant__
#ifdef REF_CONSTANT_EXTERN
#define __constant__ extern
#else
#define __constant__
#endif

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern dim3 blockDim;
extern dim3 gridDim;

/* block barrier: a no-op for one-thread blocks, a real barrier while the
 * harness runs a multi-thread block */
void ref_block_barrier(void);
inline void __syncthreads(void) { ref_block_barrier(); }

inline int3 operator+(int3 a, int3 b) { return make_int3(a.x + b.x, a.y + b.y, a.z + b.z); }

#endif
