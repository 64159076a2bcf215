// tile_common.cuh -- device helpers shared by the tiled stage kernel
// (transport_tile.cu) and its transpose (transport_adjoint.cu): 16-byte
// asynchronous copies into shared memory, four tracers per lane as two
// packed float2 pairs (FFMA2 / FADD2 / FMUL2).
#pragma once
#include <cuda.h>
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
// bring the line at p into L2 ahead of a later load (no register held)
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
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

// ---- mbarriers and TMA row gathers ---------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// make the initialised barriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase with the given parity; false if it did not complete
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, unsigned limit) {
  for (unsigned i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// four rows y0..y3 of a 2-D tensor (box: one row of the map's box width,
// from column x) into consecutive rows at dst, completing on bar
__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, int x, int y0, int y1, int y2, int y3,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace olamgpu
