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
  int mza, ntp, nrk, istage, kb, ntiles, T, nu_max, nr1_max, mwa, mva;
  float dtr;
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const int* __restrict__ r1;
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

// ---- bulk copies into shared memory, completed on an mbarrier -------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// the single arrival of a phase, announcing the bytes its copies will deliver
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// waits for the phase with the given parity to complete; gives up after
// about a second of clock (returns false)
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  const long long t_start = clock64();
  while (true) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t_start > (1ll << 31)) return false;
  }
}

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
// grad_z_quadratic on four tracers (zface_t per pair)
__device__ __forceinline__ F4 zface4(const float* aw, int mza, int kb, int lev, bool want_bot, F4 a, F4 b, F4 c) {
  return F4{zface_t(aw, mza, kb, lev, want_bot, a.a, b.a, c.a), zface_t(aw, mza, kb, lev, want_bot, a.b, b.b, c.b)};
}

template <int ORDER>
__global__ void __launch_bounds__(TILE_THREADS, 2) k_tile(TileArgs A) {
  constexpr int NPL = ORDER == 2 ? 2 : 5;     // gradient planes (and face offsets)
  constexpr int R1W = TILE_R1W(ORDER), TCW = TILE_TCW(ORDER);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int tile = blockIdx.x % A.ntiles, grp = blockIdx.x / A.ntiles;
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nR1 = h.z, nT = h.w;
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  unsigned char* p = smraw;
  unsigned long long* MB = reinterpret_cast<unsigned long long*>(p);  p += 16;
  float2* U = reinterpret_cast<float2*>(p);  p += al((size_t)A.nu_max * 256);
  float2* G = reinterpret_cast<float2*>(p);  p += al((size_t)A.nr1_max * NPL * 256);
  float2* Q0 = reinterpret_cast<float2*>(p); p += al((size_t)A.T * 2 * 256);   // scp0, sct rows of the tile
  int* R1 = reinterpret_cast<int*>(p);       p += al((size_t)A.nr1_max * R1W * 4);
  int* TC = reinterpret_cast<int*>(p);       p += al((size_t)A.T * TCW * 4);
  float* LV = reinterpret_cast<float*>(p);   p += al((size_t)A.T * TILE_LV * 4);
  int* UIW = reinterpret_cast<int*>(p);      p += al((size_t)A.nu_max * 4);
  float* AW = reinterpret_cast<float*>(p);   // a_w at levels kd-1, kd, kd+1 (4 each)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned bar = smem_addr(MB);

  // tables of this tile, checked once: every index must address the arrays
  // it is used on (a failure is recorded and the block does nothing)
  int bad = (nU > A.nu_max || nR1 > A.nr1_max || nT > A.T || nR1 > nU || nT > nR1) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nR1 * R1W; i += TILE_THREADS) {
      const int v = __ldg(A.r1 + (size_t)u_off * R1W + i), f = i % R1W;
      if (f < 6 && ((unsigned)v >= (unsigned)nU * 256u || (v & 255))) bad = 2;
      if (f == TILE_R1_NP && (v < 3 || v > 6)) bad = 3;
      R1[i] = v;
    }
    for (int i = tid; i < nT * TCW; i += TILE_THREADS) {
      const int v = __ldg(A.tc + (size_t)tile * A.T * TCW + i), f = i % TCW;
      if (f == TILE_TC_IW && (v < 1 || v >= A.mwa)) bad = 4;
      if (f == TILE_TC_NP && (v < 3 || v > 6)) bad = 5;
      if (f >= TILE_TC_NBU && f < TILE_TC_NBU + 6 && ((unsigned)v >= (unsigned)nR1 * 256u || (v & 255))) bad = 6;
      if (f >= TILE_TC_NBG && f < TILE_TC_NBG + 6 && ((unsigned)v >= (unsigned)nR1 * NPL * 256u || (v & 255)))
        bad = 9;
      if (f >= TILE_TC_EV && f < TILE_TC_EV + 6 && (unsigned)v >= (unsigned)A.mva) bad = 7;
      TC[i] = v;
    }
    for (int i = tid; i < nU; i += TILE_THREADS) {
      const int v = __ldg(A.ulist + u_off + i);
      if (v < 1 || v >= A.mwa) bad = 8;
      UIW[i] = v;
    }
  }
  if (tid == 0) mbar_init(bar, 1);
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
  const unsigned rowbytes = (unsigned)seg * 4u;

  // staging of level kd: one bulk copy per row (the U rows, then the
  // tile's scp0 / sct rows) completing on the mbarrier, whose arrival with
  // the byte count thread 0 has made beforehand; raw LV values; a_w
  auto stage = [&](int kd) {
    for (int i = tid; i < nrow; i += TILE_THREADS) {
      const float* src;
      unsigned dst;
      if (i < nU) {
        src = A.S + ((size_t)UIW[i] * mza + kd) * ntp + t0;
        dst = smem_addr(reinterpret_cast<char*>(U) + i * 256);
      } else {
        const int j = i - nU;   // 2 * cell + (0: scp0, 1: sct)
        src = ((j & 1) ? A.SCT : A.S0) + ((size_t)UIW[j >> 1] * mza + kd) * ntp + t0;
        dst = smem_addr(reinterpret_cast<char*>(Q0) + j * 256);
      }
      bulk_g2s(dst, src, rowbytes, bar);
    }
    for (int i = tid; i < nT * TILE_LV; i += TILE_THREADS) {
      const int c = i / TILE_LV, f = i - c * TILE_LV;
      const int* w = TC + c * TCW;
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
  const char* Gl = reinterpret_cast<const char*>(G) + hl * 16;
  if (tid == 0) mbar_expect(bar, (unsigned)nrow * rowbytes);
  __syncthreads();
  stage(kb);
  for (int kd = kb; kd < mza; ++kd) {
    const bool arrived = mbar_wait(bar, (unsigned)((kd - kb) & 1));
    if (__syncthreads_or(!arrived)) {
      // the copies did not complete: record it, give them a second bound, leave
      if (tid == 0 && atomicCAS(A.err, 0, 200) == 0) { A.err[1] = kd; A.err[2] = blockIdx.x; A.err[3] = tile; }
      mbar_wait(bar, (unsigned)((kd - kb) & 1));
      return;
    }
    // the next level's arrival; its copies start after phase B
    if (tid == 0 && kd + 1 < mza) mbar_expect(bar, (unsigned)nrow * rowbytes);
    // ---- phase A: gradient planes of the ring-1 cells (grad_t2d order:
    // differences to the cell, summed over the neighbours in table order)
    for (int r = 2 * warp + half; r < nR1; r += 2 * TILE_NW) {
      const int4* w4 = reinterpret_cast<const int4*>(R1 + r * R1W);
      const int4 na = w4[0], nb = w4[1];
      const int nbo[6] = {na.x, na.y, na.z, na.w, nb.x, nb.y};   // byte offsets of the U rows
      float cf[6 * NPL];
      const float4* c4 = reinterpret_cast<const float4*>(R1 + r * R1W + TILE_R1_C);
#pragma unroll
      for (int q = 0; q < (6 * NPL) / 4; ++q) {
        const float4 v = c4[q];
        cf[4 * q] = v.x; cf[4 * q + 1] = v.y; cf[4 * q + 2] = v.z; cf[4 * q + 3] = v.w;
      }
      if ((6 * NPL) % 4) {
        const float2 v = reinterpret_cast<const float2*>(c4 + (6 * NPL) / 4)[0];
        cf[6 * NPL - 2] = v.x; cf[6 * NPL - 1] = v.y;
      }
      const F4 nsc = neg4(lds4(Ul, r * 256));
      F4 g[NPL];
#pragma unroll
      for (int m = 0; m < NPL; ++m) g[m] = zero4();
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        const F4 d = add4(lds4(Ul, nbo[n]), nsc);
#pragma unroll
        for (int m = 0; m < NPL; ++m) g[m] = fma4s(cf[m * 6 + n], d, g[m]);
      }
#pragma unroll
      for (int m = 0; m < NPL; ++m) sts4(Gl, (r * NPL + m) * 256, g[m]);
    }
    __syncthreads();
    // ---- phase B: faces, vertical fluxes and the update of the tile columns
    const float* aw = AW;
    for (int c = 2 * warp + half; c < nT; c += 2 * TILE_NW) {
      const float* lv = LV + c * TILE_LV;
      const int* w = TC + c * TCW;
      const int iw = w[TILE_TC_IW], side = w[TILE_TC_SIDE];
      const float4 l1 = reinterpret_cast<const float4*>(lv)[1];
      const float4 l2 = reinterpret_cast<const float4*>(lv)[2];
      const float wkm1 = l1.z, wk0 = l1.w, vt = l2.x, rinv = l2.y, fexpl = l2.z;
      const size_t row = ((size_t)iw * mza + kd) * ntp + t0 + 4 * hl;
      const size_t lvl = (size_t)ntp;
      const F4 s0 = lds4(Ul, c * 256);
      const F4 s00 = lds4(reinterpret_cast<const char*>(Q0) + hl * 16, (2 * c) * 256);
      const F4 st = lds4(reinterpret_cast<const char*>(Q0) + hl * 16, (2 * c + 1) * 256);
      F4 sm1 = s0, sp1 = s0;
      const bool need_m2 = kd != kb && !(wkm1 < 0.f);
      const bool need_p2 = kd != mza - 1 && wk0 < 0.f;
      if (act) {
        if (kd - 1 >= kb) sm1 = ldg4(A.S + row - lvl);
        if (kd + 1 < mza) sp1 = ldg4(A.S + row + lvl);
      }
      F4 sm2 = sm1, sp2 = sp1;
      if (act && need_m2 && kd - 2 >= kb) sm2 = ldg4(A.S + row - 2 * lvl);
      if (act && need_p2 && kd + 2 < mza) sp2 = ldg4(A.S + row + 2 * lvl);
      const F4 ns00 = neg4(s00);
      // the six faces across lanes 0..5 of the half warp: dirv*vmasc, upwind
      // side, and the outflow faces' sums (their share of the flux divergence
      // is so * (S - S0) + sum_m sm[m] * grad_m(cell))
      const int nf = hl < 6 ? hl : 0;
      const float vmf = hl < 6 ? lv[nf] : 0.f;
      const float dvvm = __int_as_float(w[TILE_TC_DV + nf]) * vmf;
      const bool inflow = hl < 6 && ((vmf < 0.f ? 1 : 0) != ((side >> nf) & 1));
      float so = inflow ? 0.f : dvvm, sm[NPL];
      {
        const float* oo = reinterpret_cast<const float*>(w + TILE_TC_OFF + nf * NPL);
#pragma unroll
        for (int m = 0; m < NPL; ++m) sm[m] = so * oo[m];
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        so += __shfl_xor_sync(0xffffffffu, so, o, 16);
#pragma unroll
        for (int m = 0; m < NPL; ++m) sm[m] += __shfl_xor_sync(0xffffffffu, sm[m], o, 16);
      }
      unsigned inmask = (__ballot_sync(0xffffffffu, inflow) >> (16 * half)) & 0x3fu;
      F4 fd = scale4(so, add4(s0, ns00));
#pragma unroll
      for (int m = 0; m < NPL; ++m) fd = fma4s(sm[m], lds4(Gl, (c * NPL + m) * 256), fd);
      // inflow faces: the upwind neighbour's reconstruction
      const float dvsrc = dvvm;
      while (__any_sync(0xffffffffu, inmask != 0)) {
        const int f = inmask ? __ffs(inmask) - 1 : 0;
        const float coef = __shfl_sync(0xffffffffu, dvsrc, f, 16);
        if (inmask) {
          inmask &= inmask - 1;
          const int su = w[TILE_TC_NBU + f], sg = w[TILE_TC_NBG + f];
          const float* of = reinterpret_cast<const float*>(w + TILE_TC_OFF + (6 + f) * NPL);
          F4 val = lds4(Ul, su);
#pragma unroll
          for (int m = 0; m < NPL; ++m) val = fma4s(of[m], lds4(Gl, sg + m * 256), val);
          fd = fma4s(coef, add4(val, ns00), fd);
        }
      }
      // vertical upwind faces kd-1 and kd (grad_z_quadratic, bounded)
      F4 up_lo, up_hi;
      if (kd == kb) up_lo = s0;                                                    // scp_upw(kb-1) = scp(kb)
      else if (wkm1 < 0.f) up_lo = zface4(aw + 4, mza, kb, kd, true, sm1, s0, sp1);       // scpb(kd)
      else up_lo = zface4(aw, mza, kb, kd - 1, false, sm2, sm1, s0);                      // scpt(kd-1)
      if (kd == mza - 1) up_hi = s0;                                               // scp_upw(mza) = scp(mza)
      else if (wk0 < 0.f) up_hi = zface4(aw + 8, mza, kb, kd + 1, true, s0, sp1, sp2);    // scpb(kd+1)
      else up_hi = zface4(aw + 4, mza, kb, kd, false, sm1, s0, sp1);                      // scpt(kd)
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
  A.ntiles = d.ntiles; A.T = d.tile_T; A.nu_max = d.tile_nu_max; A.nr1_max = d.tile_nr1_max;
  A.mwa = d.mwa; A.mva = d.mva;
  A.dtr = dtr;
  A.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  A.ulist = d.tile_u.p; A.r1 = d.tile_r1.p; A.tc = d.tile_tc.p;
  A.a_w = d.a_w.p; A.volti = d.volti.p; A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p;
  A.rhos = rhos; A.ff = tp.ff.p;
  A.S = S; A.S0 = S0; A.SCT = SCT; A.OUT = OUT;
  A.err = status;
  const int order = d.tile_order;
  const size_t smem = tile_smem_bytes(order, d.tile_T, d.tile_nu_max, d.tile_nr1_max);
  const unsigned ngrp = (unsigned)((ntp + 63) / 64);
  const unsigned nblk = (unsigned)d.ntiles * ngrp;
  if (order == 2) {
    OG_CUDA(cudaFuncSetAttribute(k_tile<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile<2><<<nblk, TILE_THREADS, smem, s>>>(A);
  } else {
    OG_CUDA(cudaFuncSetAttribute(k_tile<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile<3><<<nblk, TILE_THREADS, smem, s>>>(A);
  }
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

}  // namespace olamgpu
