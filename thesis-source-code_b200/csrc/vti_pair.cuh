// Packed FP32 pairs for sm_100 (add/sub/mul/fma .rn.f32x2). Each lane is
// rounded as the scalar instruction with the same rounding (__fadd_rn,
// __fsub_rn, __fmul_rn, __fmaf_rn), so a pair computes exactly what two
// scalar evaluations of the same operation sequence compute.
#pragma once

#include <cuda_runtime.h>

namespace vti {

#define VTI_PAIR_OP2(op)                                                              \
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t" op \
      " rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"                                     \
      : "=f"(d.x), "=f"(d.y)                                                           \
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y))
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 d;
  VTI_PAIR_OP2("add.rn.f32x2");
  return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  float2 d;
  VTI_PAIR_OP2("sub.rn.f32x2");
  return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 d;
  VTI_PAIR_OP2("mul.rn.f32x2");
  return d;
}
#undef VTI_PAIR_OP2
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 splat(float v) { return make_float2(v, v); }

}  // namespace vti
