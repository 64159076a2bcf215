// transport_tile.cu -- the fused RK stage of update_scalar in tiles, for
// grids without terrain (lpw = lpv = 2 everywhere).
//
// Restates, fused into one pass over the batched layout Q[iw][kd][ntp],
// omodel/scalar_transport_rk.F90:
//   grad_t2d / grad_t2d_quadratic (grad_lib.f90:236-341)  gradient planes
//   scalar_v_column (474-534)                             upwind V-face value
//   grad_z_quadratic (grad_lib.f90:166-229),
//   scalar_w_column (537-612)                             vertical faces, flux
//                                                         divergence, update
// Work mapping.  A block owns a tile of consecutive prognostic columns and a
// group of 64 tracers, and sweeps the levels bottom to top.  Per level:
//   staging  the tracer rows of the tile's two-ring neighbourhood U (tile
//            columns, their neighbours, the neighbours' neighbours) are
//            copied into shared memory with cp.async, 256 B per row;
//   phase A  one warp per ring-1 cell (tile + first ring) forms the gradient
//            planes from U, in the reference's operation order, into G;
//   phase B  one warp per tile column takes the upwind face value of each V
//            face from U and G (its own side for outflow, the neighbour's
//            side for inflow), adds the vertical quadratic upwind faces and
//            writes the updated tracer.
// A warp handles one column for 64 tracers (a float2 per lane), so every
// table read and branch is warp-uniform; each gradient is formed once per
// tile and each tracer row crosses HBM once per stage.
#include "transport_kernels.cuh"

namespace olamgpu {

struct TileArgs {
  int mza, ntp, nrk, istage, kb, ntiles, T, nu_max, mwa, mva;
  float dtr;
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const float* __restrict__ amat;   // slot weights, TILE_AW per tile column
  const int* __restrict__ tc;
  const float* __restrict__ a_w;    // Fortran (mza, 2, 2)
  const float* __restrict__ volti;
  const float* __restrict__ vmasc;
  const float* __restrict__ wmasc;
  const float* __restrict__ rhos;   // rhos(:,:,nrk)
  const float* __restrict__ ff;     // (mwa, nrk)
  const float* __restrict__ S;
  const float* __restrict__ S0;
  const float* __restrict__ SCT;
  float* __restrict__ OUT;
  int* err;                         // device status record
};

#define TILE_THREADS 256
#define TILE_NW (TILE_THREADS / 32)
// per tile column and level: vmasc of the 6 faces, wmasc(k-1), wmasc(k),
// volti, dtr / rhos, 1 - ff, pad
#define TILE_LV 12

// ---- 16-byte asynchronous copies into shared memory ------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// acc + w * a on both tracers of a lane (one packed FFMA2)
__device__ __forceinline__ float2 fma2s(float w, float2 a, float2 acc) {
  return __ffma2_rn(make_float2(w, w), a, acc);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// grad_z_quadratic (bounded, zero-gradient BCs) at level lev from rows
// a = S(lev-1), b = S(lev), c = S(lev+1); aw holds a_w(lev,1:2,1:2).
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

// four tracers of a lane as two packed pairs
struct F4 {
  float2 a, b;
};
__device__ __forceinline__ F4 zero4() { return F4{make_float2(0.f, 0.f), make_float2(0.f, 0.f)}; }
__device__ __forceinline__ F4 lds4(const char* base, int off) {
  const float4 v = *reinterpret_cast<const float4*>(base + off);
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void sts4(const char* base, int off, F4 v) {
  *reinterpret_cast<float4*>(const_cast<char*>(base) + off) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
__device__ __forceinline__ F4 ldg4(const float* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void stg4(float* p, F4 v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
__device__ __forceinline__ F4 add4(F4 x, F4 y) { return F4{__fadd2_rn(x.a, y.a), __fadd2_rn(x.b, y.b)}; }
__device__ __forceinline__ F4 neg4(F4 x) { return F4{make_float2(-x.a.x, -x.a.y), make_float2(-x.b.x, -x.b.y)}; }
// acc + w * x
__device__ __forceinline__ F4 fma4s(float w, F4 x, F4 acc) {
  const float2 w2 = make_float2(w, w);
  return F4{__ffma2_rn(w2, x.a, acc.a), __ffma2_rn(w2, x.b, acc.b)};
}
// x * w + acc (acc a vector)
__device__ __forceinline__ F4 fma4v(F4 x, float w, F4 acc) { return fma4s(w, x, acc); }
__device__ __forceinline__ F4 scale4(float w, F4 x) {
  const float2 w2 = make_float2(w, w);
  return F4{__fmul2_rn(w2, x.a), __fmul2_rn(w2, x.b)};
}
__device__ __forceinline__ F4 sel4(bool p, F4 x, F4 y) { return p ? x : y; }
// grad_z_quadratic on four tracers (zface_t per pair)
__device__ __forceinline__ F4 zface4(const float* aw, int mza, int kb, int lev, bool want_bot, F4 a, F4 b, F4 c) {
  return F4{zface_t(aw, mza, kb, lev, want_bot, a.a, b.a, c.a), zface_t(aw, mza, kb, lev, want_bot, a.b, b.b, c.b)};
}

// Work per level: phase W forms, for every tile column, the weights of its
// slot columns in the horizontal flux divergence from the level's vmasc
// (one thread per (column, slot), shared by all tracers); phase B computes,
// per column and tracer,
//   fluxdiv = SW * (S - S0) + sum_j W_j (S(slot j) - S)
// with SW = sum_f dirv*vmasc, which is update_scalar's sum over the faces of
// dirv*vmasc*(upwind face value - S0) with the reconstruction folded into W.
__global__ void __launch_bounds__(TILE_THREADS, 2) k_tile(TileArgs A) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int tile = blockIdx.x % A.ntiles, grp = blockIdx.x / A.ntiles;
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nT = h.w;
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  unsigned char* p = smraw;
  p += 16;   // reserved
  float2* U = reinterpret_cast<float2*>(p);  p += al((size_t)A.nu_max * 256);
  float2* Q0 = reinterpret_cast<float2*>(p); p += al((size_t)A.T * 2 * 256);   // scp0, sct rows of the tile
  int* TC = reinterpret_cast<int*>(p);       p += al((size_t)A.T * TILE_TCW * 4);
  float* AM = reinterpret_cast<float*>(p);   p += al((size_t)A.T * TILE_AW * 4);
  float* WW = reinterpret_cast<float*>(p);   p += al((size_t)A.T * 24 * 4);    // W[0..20), SW at 20
  float* LV = reinterpret_cast<float*>(p);   p += al((size_t)A.T * TILE_LV * 4);
  int* UIW = reinterpret_cast<int*>(p);      p += al((size_t)A.nu_max * 4);
  float* AW = reinterpret_cast<float*>(p);   // a_w at levels kd-1, kd, kd+1 (4 each)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // tables of this tile, checked once: every index must address the arrays
  // it is used on (a failure is recorded and the block does nothing)
  int bad = (nU > A.nu_max || nT > A.T || nT > nU) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nT * TILE_TCW; i += TILE_THREADS) {
      const int v = __ldg(A.tc + (size_t)tile * A.T * TILE_TCW + i), f = i % TILE_TCW;
      if (f == TILE_TC_IW && (v < 1 || v >= A.mwa)) bad = 4;
      if (f == TILE_TC_NP && (v < 3 || v > 6)) bad = 5;
      if (f >= TILE_TC_SLOT && f < TILE_TC_SLOT + TILE_NS && ((unsigned)v >= (unsigned)nU * 256u || (v & 255)))
        bad = 6;
      if (f >= TILE_TC_EV && f < TILE_TC_EV + 6 && (unsigned)v >= (unsigned)A.mva) bad = 7;
      TC[i] = v;
    }
    for (int i = tid; i < nT * TILE_AW; i += TILE_THREADS) AM[i] = __ldg(A.amat + (size_t)tile * A.T * TILE_AW + i);
    for (int i = tid; i < nU; i += TILE_THREADS) {
      const int v = __ldg(A.ulist + u_off + i);
      if (v < 1 || v >= A.mwa) bad = 8;
      UIW[i] = v;
    }
  }
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }

  const int mza = A.mza, ntp = A.ntp, kb = A.kb;
  const int t0 = grp * 64;
  const int seg = min(64, ntp - t0);  // tracers of this group (a multiple of 4)
  // a half warp per column: lane hl of half h holds tracers 4 hl .. 4 hl + 3
  const int half = lane >> 4, hl = lane & 15;
  const bool act = 4 * hl < seg;
  const int nrow = nU + 2 * nT;

  // staging of level kd: 16-byte asynchronous copies of the U rows, then
  // of the tile's scp0 / sct rows (a row is 16 chunks); per-level values; a_w
  const int nch = seg >> 2;
  auto stage = [&](int kd) {
    for (int i = tid; i < nrow * 16; i += TILE_THREADS) {
      const int r = i >> 4, ch = i & 15;
      if (ch >= nch) continue;
      const float* src;
      char* dst;
      if (r < nU) {
        src = A.S + ((size_t)UIW[r] * mza + kd) * ntp + t0;
        dst = reinterpret_cast<char*>(U) + r * 256;
      } else {
        const int j = r - nU;   // 2 * cell + (0: scp0, 1: sct)
        src = ((j & 1) ? A.SCT : A.S0) + ((size_t)UIW[j >> 1] * mza + kd) * ntp + t0;
        dst = reinterpret_cast<char*>(Q0) + j * 256;
      }
      cp_async16(dst + ch * 16, src + ch * 4);
    }
    cp_async_commit();
    for (int i = tid; i < nT * TILE_LV; i += TILE_THREADS) {
      const int c = i / TILE_LV, f = i - c * TILE_LV;
      const int* w = TC + c * TILE_TCW;
      const int iw = w[TILE_TC_IW];
      const size_t x = (size_t)iw * mza + kd;
      float v = 0.f;
      if (f < 6) { if (f < w[TILE_TC_NP]) v = __ldg(A.vmasc + (size_t)w[TILE_TC_EV + f] * mza + kd); }
      else if (f == 6) v = __ldg(A.wmasc + x - 1);
      else if (f == 7) v = __ldg(A.wmasc + x);
      else if (f == 8) v = __ldg(A.volti + x);
      else if (f == 9) v = A.dtr / __ldg(A.rhos + x);
      else if (f == 10) v = 1.0f - __ldg(A.ff + (size_t)iw * A.nrk + A.istage - 1);
      LV[i] = v;
    }
    if (tid < 12) {
      const int lev = kd - 1 + tid / 4, m = tid & 3;
      AW[tid] = (lev >= 0 && lev < mza) ? __ldg(A.a_w + lev + m * mza) : 0.f;
    }
  };

  const char* Ul = reinterpret_cast<const char*>(U) + hl * 16;
  stage(kb);
  for (int kd = kb; kd < mza; ++kd) {
    cp_async_wait_all();
    __syncthreads();
    // ---- phase W: slot weights of this level, a thread per (column, slot)
    for (int i = tid; i < nT * TILE_NS; i += TILE_THREADS) {
      const int c = i / TILE_NS, j = i - c * TILE_NS;
      const int* w = TC + c * TILE_TCW;
      const float* lv = LV + c * TILE_LV;
      const float* am = AM + c * TILE_AW;
      const int side = w[TILE_TC_SIDE];
      float acc = 0.f;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const float vm = lv[f];
        const int k = ((vm < 0.f ? 1 : 0) != ((side >> f) & 1)) ? 1 : 0;   // 1: the neighbour is upwind
        acc = fmaf(__int_as_float(w[TILE_TC_DV + f]) * vm, am[(f * 2 + k) * TILE_NS + j], acc);
      }
      WW[c * 24 + j] = acc;
    }
    __syncthreads();
    // ---- phase B: horizontal and vertical fluxes, the update of the tile columns
    const float* aw = AW;
    for (int c = 2 * warp + half; c < nT; c += 2 * TILE_NW) {
      const float* lv = LV + c * TILE_LV;
      const int* w = TC + c * TILE_TCW;
      const int iw = w[TILE_TC_IW];
      const float4 l1 = reinterpret_cast<const float4*>(lv)[1];
      const float4 l2 = reinterpret_cast<const float4*>(lv)[2];
      const float wkm1 = l1.z, wk0 = l1.w, vt = l2.x, rinv = l2.y, fexpl = l2.z;
      const size_t row = ((size_t)iw * mza + kd) * ntp + t0 + 4 * hl;
      const size_t lvl = (size_t)ntp;
      // the column's values two levels either side (the level's own range
      // checks are the same for the whole block)
      const F4 s0 = lds4(Ul, c * 256);
      F4 sm1 = s0, sp1 = s0;
      if (act && kd - 1 >= kb) sm1 = ldg4(A.S + row - lvl);
      if (act && kd + 1 < mza) sp1 = ldg4(A.S + row + lvl);
      F4 sm2 = sm1, sp2 = sp1;
      if (act && kd - 2 >= kb) sm2 = ldg4(A.S + row - 2 * lvl);
      if (act && kd + 2 < mza) sp2 = ldg4(A.S + row + 2 * lvl);
      const F4 s00 = lds4(reinterpret_cast<const char*>(Q0) + hl * 16, (2 * c) * 256);
      const F4 st = lds4(reinterpret_cast<const char*>(Q0) + hl * 16, (2 * c + 1) * 256);
      const F4 ns0 = neg4(s0), ns00 = neg4(s00);
      const float* wc = WW + c * 24;
      float sw = 0.f;   // sum over the faces of dirv * vmasc
#pragma unroll
      for (int f = 0; f < 6; ++f) sw = fmaf(__int_as_float(w[TILE_TC_DV + f]), lv[f], sw);
      F4 fd = scale4(sw, add4(s0, ns00));
#pragma unroll
      for (int q = 0; q < TILE_NS / 4; ++q) {
        const int4 so4 = reinterpret_cast<const int4*>(w + TILE_TC_SLOT)[q];
        const float4 w4 = reinterpret_cast<const float4*>(wc)[q];
        fd = fma4s(w4.x, add4(lds4(Ul, so4.x), ns0), fd);
        fd = fma4s(w4.y, add4(lds4(Ul, so4.y), ns0), fd);
        fd = fma4s(w4.z, add4(lds4(Ul, so4.z), ns0), fd);
        fd = fma4s(w4.w, add4(lds4(Ul, so4.w), ns0), fd);
      }
      // vertical upwind faces kd-1 and kd (grad_z_quadratic, bounded): the
      // upwind level's stencil is selected, then reconstructed once
      F4 up_lo, up_hi;
      if (kd == kb) {
        up_lo = s0;                                                   // scp_upw(kb-1) = scp(kb)
      } else {
        const bool dn = wkm1 < 0.f;   // scpb(kd) from (kd-1, kd, kd+1), else scpt(kd-1) from (kd-2, kd-1, kd)
        up_lo = zface4(dn ? aw + 4 : aw, mza, kb, dn ? kd : kd - 1, dn, sel4(dn, sm1, sm2), sel4(dn, s0, sm1),
                       sel4(dn, sp1, s0));
      }
      if (kd == mza - 1) {
        up_hi = s0;                                                   // scp_upw(mza) = scp(mza)
      } else {
        const bool dn = wk0 < 0.f;    // scpb(kd+1) from (kd, kd+1, kd+2), else scpt(kd) from (kd-1, kd, kd+1)
        up_hi = zface4(dn ? aw + 8 : aw + 4, mza, kb, dn ? kd + 1 : kd, dn, sel4(dn, s0, sm1), sel4(dn, sp1, s0),
                       sel4(dn, sp2, sp1));
      }
      // scp = scp0 + dtr * (sct + volti * (fluxdiv + fexpl * vertical)) / rhos
      const F4 v = scale4(fexpl, add4(scale4(wkm1, add4(up_lo, ns00)), scale4(-wk0, add4(up_hi, ns00))));
      const F4 o = fma4v(add4(st, scale4(vt, add4(fd, v))), rinv, s00);
      if (act) {
        stg4(A.OUT + row, o);
        if (kd == kb)
          for (int k2 = 0; k2 < kb; ++k2) stg4(A.OUT + ((size_t)iw * mza + k2) * ntp + t0 + 4 * hl, o);
      }
    }
    __syncthreads();
    if (kd + 1 < mza) stage(kd + 1);
  }
}

bool tile_stage_available(const DevGrid& d, const Transport& tp, int order) {
  return tp.flat && d.tile_T > 0 && d.tile_order == order;
}

int launch_tile_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                      const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr,
                      const float* rhos, int* status, cudaStream_t s) {
  TileArgs A;
  A.mza = d.mza; A.ntp = ntp; A.nrk = nrk; A.istage = istage; A.kb = 1;
  A.ntiles = d.ntiles; A.T = d.tile_T; A.nu_max = d.tile_nu_max;
  A.mwa = d.mwa; A.mva = d.mva;
  A.dtr = dtr;
  A.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  A.ulist = d.tile_u.p; A.amat = d.tile_a.p; A.tc = d.tile_tc.p;
  A.a_w = d.a_w.p; A.volti = d.volti.p; A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p;
  A.rhos = rhos; A.ff = tp.ff.p;
  A.S = S; A.S0 = S0; A.SCT = SCT; A.OUT = OUT;
  A.err = status;
  const size_t smem = tile_smem_bytes(d.tile_T, d.tile_nu_max);
  const unsigned ngrp = (unsigned)((ntp + 63) / 64);
  const unsigned nblk = (unsigned)d.ntiles * ngrp;
  OG_CUDA(cudaFuncSetAttribute(k_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_tile<<<nblk, TILE_THREADS, smem, s>>>(A);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

}  // namespace olamgpu
