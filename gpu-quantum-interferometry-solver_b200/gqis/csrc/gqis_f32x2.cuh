// gqis_f32x2.cuh - packed FP32 primitives of sm_100a: one fma/add/mul/sub.rn.f32x2 instruction on a
// pair of FP32 lanes, each lane rounded as the scalar instruction would round it.
//
// Used by the two-points-per-thread reduced form (gqis_packed.cuh: the lanes are two points) and by
// the tensor-core epilogue (gqis_matrix_tc.cuh: the lanes are the real and imaginary part of one
// density-matrix element).
#pragma once

#include <cuda_runtime.h>

namespace gq {

__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
    unsigned long long A = *reinterpret_cast<unsigned long long*>(&a);
    unsigned long long B = *reinterpret_cast<unsigned long long*>(&b);
    unsigned long long D;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(D) : "l"(A), "l"(B));
    return *reinterpret_cast<float2*>(&D);
}
// Sign flip of both lanes. Literal coefficients fold at compile time; a runtime operand becomes an
// operand of the consuming packed instruction.
__device__ __forceinline__ float2 f2_neg(float2 a) { return make_float2(-a.x, -a.y); }

// Compensated y += h*a per lane (h = h_hi + h_lo to about FP64 accuracy) with the correction kept
// negated (cn = -c of the scalar Kahan update), so every step is one packed instruction:
// v = a*h_hi + (a*h_lo + cn); s = y + v; cn = v - (s - y); y = s. Per lane the result is bit for bit
// that of FormFP32::accumulate (negation is exact and round-to-nearest is symmetric).
__device__ __forceinline__ void f2_kahan(float2& y, float2& cn, float2 a, float2 h_hi, float2 h_lo) {
    const float2 v = f2_fma(a, h_hi, f2_fma(a, h_lo, cn));
    const float2 s = f2_add(y, v);
    cn = f2_sub(v, f2_sub(s, y));
    y = s;
}

}  // namespace gq
