// Shared device helpers: complex float2/double2 arithmetic and status codes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define HB_DEV __host__ __device__ __forceinline__

namespace hb {

// Complex add/subtract as one packed FP32x2 instruction on sm_100 (same IEEE results
// as two scalar adds).  Packed multiplies are not used: they need the operands
// broadcast or swapped within the pair, which costs more than the scalar FMAs.
#if defined(__CUDA_ARCH__)
HB_DEV float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
HB_DEV float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
HB_DEV float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#else
HB_DEV float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HB_DEV float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
HB_DEV float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
#endif
HB_DEV float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
HB_DEV float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
HB_DEV float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (DIR = -1) or +i (DIR = +1)
template <int DIR>
HB_DEV float2 rot90(float2 a) {
  return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
// a * w where w is given by (c, s) = (cos, DIR*sin)
HB_DEV float2 crot(float2 a, float c, float s) {
  return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
}

// ---- asynchronous global -> shared copies (cp.async, completion by groups) ----
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// wait until at most n groups are pending (n is small; the switch keeps it immediate)
__device__ __forceinline__ void cp_async_wait_dyn(int n) {
  switch (n) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    case 3: cp_async_wait<3>(); break;
    default: cp_async_wait<4>(); break;
  }
}

}  // namespace hb
