/* mpc_cuda.cuh -- drop-in umbrella for the fixed-precision path.
 *
 * Code written against the mpc_cuda umbrella (reference include/mpc_cuda.cuh:
 * 37-55) for its fixed-precision types and their elementary functions keeps
 * compiling unchanged:
 *
 *   #include "mpc_cuda.cuh"
 *   cu_fp::cu_freal<256> a = 1.5, b = x, c = a * b + a;
 *   cu_fp::cu_fcomplex<1024> z = za * zx + zy;
 *
 * Only the fixed-precision surface (cu_fp::cu_freal / cu_fcomplex) is provided;
 * the reference's runtime-precision MPFR/MPC device port is not part of this
 * engine.  Host code that works on whole arrays calls the C ABI in mpb.h.
 */
#ifndef MPB_DROPIN_UMBRELLA_CUH
#define MPB_DROPIN_UMBRELLA_CUH
#include "mpc_cuda/cu_freal.cuh"
#include "mpc_cuda/cu_fcomplex.cuh"
#include "mpc_cuda/cu_fmath.cuh"
#include "mpc_cuda/cu_fcmath.cuh"
#endif
