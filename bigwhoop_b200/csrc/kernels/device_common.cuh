// Device-side helpers shared by the kernels: exactly rounded arithmetic in the codec's
// floating-point type (no FMA contraction, so results match the reference's x86 build bit for
// bit) and launch-geometry helpers.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "kernels.hpp"

namespace bwcb {
namespace dev {

__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ bwc_raw as_raw(bwc_float f) {
#ifdef BWC_SINGLE_PRECISION
  return __float_as_uint(f);
#else
  return (bwc_raw)__double_as_longlong(f);
#endif
}
__device__ __forceinline__ bwc_float as_float(bwc_raw r) {
#ifdef BWC_SINGLE_PRECISION
  return __uint_as_float(r);
#else
  return __longlong_as_double((long long)r);
#endif
}

// truncating float -> unsigned conversion of the quantiser, (bwc_raw)(x)
__device__ __forceinline__ bwc_raw to_raw_rz(bwc_float x) {
#ifdef BWC_SINGLE_PRECISION
  return __float2uint_rz(x);
#else
  return __double2ull_rz(x);
#endif
}

// round-to-nearest unsigned 64-bit -> codec float conversion, (bwc_float)u
__device__ __forceinline__ bwc_float from_u64_rn(uint64_t u) {
#ifdef BWC_SINGLE_PRECISION
  return __ull2float_rn(u);
#else
  return __ull2double_rn(u);
#endif
}

constexpr int kNumSMs = 148;

}  // namespace dev
}  // namespace bwcb

#define BWCB_CUDA_CHECK_LAUNCH() ((void)0)
