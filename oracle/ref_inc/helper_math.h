/*
 * oracle/ref_inc/helper_math.h -- empty stand-in (TEST INFRASTRUCTURE ONLY).
 *
 * The reference's src/darcy.cuh includes <helper_math.h> from the CUDA
 * samples, which the reference does not ship.  None of the float3/int3
 * helpers it declares are used by the Darcy kernels the oracle harness
 * compiles (their vector arithmetic is the reference's own
 * src/vector_arithmetic.h; int3 addition comes from oracle/ref_shim.h), so
 * an empty header on the include path is enough.
 */
#ifndef SPHERE_ORACLE_HELPER_MATH_STANDIN_H_
#define SPHERE_ORACLE_HELPER_MATH_STANDIN_H_
#endif
