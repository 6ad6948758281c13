// CPU ORACLE — test infrastructure, not product code.
//
// Host build of the reference's own 3x3 SVD: this translation unit includes
// simulation/helper_math.cuh from the reference tree UNMODIFIED (the include
// path is given by oracle/Makefile; nothing of it is copied here) and supplies
// host definitions of the CUDA names it uses. The shims follow IEEE-754
// semantics, not CUDA internals:
//   __fadd_rn / __fsub_rn : one correctly rounded float add / subtract
//                           (this file is compiled with -ffp-contract=off)
//   __frsqrt_rn           : correctly rounded float 1/sqrt(x), via one
//                           rounding from 64-bit extended precision
//   max(float, float)     : fmaxf
// The exported ref_svd3x3 mirrors the reference's wrapper svd3x3
// (simulation/mpm_kernels.cuh:585-601): row-major A, U, V; S the singular
// values.
#include <cmath>

#define __device__
#define __forceinline__ inline

static inline float __fadd_rn(float a, float b) { return a + b; }
static inline float __fsub_rn(float a, float b) { return a - b; }
static inline float __frsqrt_rn(float x) { return (float)(1.0L / sqrtl((long double)x)); }
static inline float max(float a, float b) { return std::fmax(a, b); }

#include "helper_math.cuh"

extern "C" void ref_svd3x3(const double A[9], double U[9], double S[3], double V[9]) {
    svd<double>(A[0], A[1], A[2], A[3], A[4], A[5], A[6], A[7], A[8],
                U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], U[8],
                S[0], S[1], S[2],
                V[0], V[1], V[2], V[3], V[4], V[5], V[6], V[7], V[8]);
}
