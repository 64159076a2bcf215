// tile_common.cuh -- device helpers shared by the tiled stage kernel
// (transport_tile.cu) and its transpose (transport_adjoint.cu): 16-byte
// asynchronous copies into shared memory, four tracers per lane as two
// packed float2 pairs (FFMA2 / FADD2 / FMUL2), grad_z_quadratic faces.
#pragma once
#include <cuda_runtime.h>

namespace olamgpu {

// ---- 16-byte asynchronous copies into shared memory ------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// four tracers of a lane as two packed pairs
struct F4 {
  float2 a, b;
};
__device__ __forceinline__ F4 zero4() { return F4{make_float2(0.f, 0.f), make_float2(0.f, 0.f)}; }
__device__ __forceinline__ F4 lds4(const char* base, int off) {
  const float4 v = *reinterpret_cast<const float4*>(base + off);
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ F4 ldg4(const float* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void stg4(float* p, F4 v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
__device__ __forceinline__ F4 add4(F4 x, F4 y) { return F4{__fadd2_rn(x.a, y.a), __fadd2_rn(x.b, y.b)}; }
__device__ __forceinline__ F4 sub4(F4 x, F4 y) {
  return F4{__fadd2_rn(x.a, make_float2(-y.a.x, -y.a.y)), __fadd2_rn(x.b, make_float2(-y.b.x, -y.b.y))};
}
// acc + w * x
__device__ __forceinline__ F4 fma4s(float w, F4 x, F4 acc) {
  const float2 w2 = make_float2(w, w);
  return F4{__ffma2_rn(w2, x.a, acc.a), __ffma2_rn(w2, x.b, acc.b)};
}
__device__ __forceinline__ F4 scale4(float w, F4 x) {
  const float2 w2 = make_float2(w, w);
  return F4{__fmul2_rn(w2, x.a), __fmul2_rn(w2, x.b)};
}
__device__ __forceinline__ F4 sel4(bool p, F4 x, F4 y) { return p ? x : y; }

// grad_z_quadratic (bounded, zero-gradient BCs) at level lev from rows
// a = S(lev-1), b = S(lev), c = S(lev+1); aw holds a_w(lev,1:2,1:2).
// Rows outside the column are never used (the select drops them).
__device__ __forceinline__ float2 zface_t(const float* aw, int mza, int kb, int lev, bool want_bot, float2 a,
                                          float2 b, float2 c) {
  const bool top = (lev > mza - 2), bot = (lev < kb + 1);
  const float c1 = aw[want_bot ? 0 : 2], c2 = aw[want_bot ? 1 : 3];
  float2 r;
  float dsk = top ? 0.f : (c.x - b.x), dskm1 = bot ? 0.f : (b.x - a.x);
  r.x = b.x + dsk * c1 + dskm1 * c2;
  dsk = top ? 0.f : (c.y - b.y); dskm1 = bot ? 0.f : (b.y - a.y);
  r.y = b.y + dsk * c1 + dskm1 * c2;
  return r;
}
__device__ __forceinline__ F4 zface4(const float* aw, int mza, int kb, int lev, bool want_bot, F4 a, F4 b, F4 c) {
  return F4{zface_t(aw, mza, kb, lev, want_bot, a.a, b.a, c.a), zface_t(aw, mza, kb, lev, want_bot, a.b, b.b, c.b)};
}

}  // namespace olamgpu
