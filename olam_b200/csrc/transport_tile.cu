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
  float2* U = reinterpret_cast<float2*>(p);  p += al((size_t)A.nu_max * 256);
  float2* G = reinterpret_cast<float2*>(p);  p += al((size_t)A.nr1_max * NPL * 256);
  float2* Q0 = reinterpret_cast<float2*>(p); p += al((size_t)A.T * 2 * 256);   // scp0, sct rows of the tile
  int* R1 = reinterpret_cast<int*>(p);       p += al((size_t)A.nr1_max * R1W * 4);
  int* TC = reinterpret_cast<int*>(p);       p += al((size_t)A.T * TCW * 4);
  float* LV = reinterpret_cast<float*>(p);   p += al((size_t)A.T * TILE_LV * 4);
  int* UIW = reinterpret_cast<int*>(p);      p += al((size_t)A.nu_max * 4);
  float* AW = reinterpret_cast<float*>(p);   // a_w at levels kd-1, kd, kd+1 (4 each)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

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
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }

  const int mza = A.mza, ntp = A.ntp, kb = A.kb;
  const int t0 = grp * 64;
  const int seg = min(64, ntp - t0);  // tracers of this group (a multiple of 4)
  const int nch = seg >> 2;           // 16-byte chunks per row
  const bool act = 2 * lane < seg;

  auto stage = [&](int kd) {
    for (int i = tid; i < nU * 16; i += TILE_THREADS) {
      const int row = i >> 4, ch = i & 15;
      if (ch < nch)
        cp_async16(reinterpret_cast<char*>(U) + row * 256 + ch * 16,
                   A.S + ((size_t)UIW[row] * mza + kd) * ntp + t0 + ch * 4);
    }
    for (int i = tid; i < nT * 32; i += TILE_THREADS) {
      const int row = i >> 4, ch = i & 15;   // row = 2 * cell + (0: scp0, 1: sct)
      if (ch < nch)
        cp_async16(reinterpret_cast<char*>(Q0) + row * 256 + ch * 16,
                   ((row & 1) ? A.SCT : A.S0) + ((size_t)UIW[row >> 1] * mza + kd) * ntp + t0 + ch * 4);
    }
    cp_async_commit();
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

  stage(kb);
  for (int kd = kb; kd < mza; ++kd) {
    cp_async_wait_all();
    __syncthreads();
    // ---- phase A: gradient planes of the ring-1 cells (grad_t2d order:
    // differences to the cell, summed over the neighbours in table order)
    for (int r = warp; r < nR1; r += TILE_NW) {
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
      const char* Ul = reinterpret_cast<const char*>(U + lane);
      const float2 nsc = neg2(U[r * 32 + lane]);
      float2 g[NPL];
#pragma unroll
      for (int m = 0; m < NPL; ++m) g[m] = make_float2(0.f, 0.f);
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        const float2 d = add2(*reinterpret_cast<const float2*>(Ul + nbo[n]), nsc);
#pragma unroll
        for (int m = 0; m < NPL; ++m) g[m] = fma2s(cf[m * 6 + n], d, g[m]);
      }
#pragma unroll
      for (int m = 0; m < NPL; ++m) G[(r * NPL + m) * 32 + lane] = g[m];
    }
    __syncthreads();
    // ---- phase B: faces, vertical fluxes and the update of the tile columns
    const float* aw = AW;
    for (int c = warp; c < nT; c += TILE_NW) {
      const int* w = TC + c * TCW;
      const int4 h4 = reinterpret_cast<const int4*>(w)[0];
      const int iw = h4.x, side = h4.y;
      const int4 q1 = reinterpret_cast<const int4*>(w)[1];      // U offsets 0..3
      const int4 q2 = reinterpret_cast<const int4*>(w)[2];      // U offsets 4, 5, G offsets 0, 1
      const int4 q3 = reinterpret_cast<const int4*>(w)[3];      // G offsets 2..5
      const float4 dva = reinterpret_cast<const float4*>(w)[5];  // ev 4, 5, dv 0, 1
      const float4 dvb = reinterpret_cast<const float4*>(w)[6];  // dv 2..5
      const int nbu[6] = {q1.x, q1.y, q1.z, q1.w, q2.x, q2.y};
      const int nbg[6] = {q2.z, q2.w, q3.x, q3.y, q3.z, q3.w};
      const float dvv[6] = {dva.z, dva.w, dvb.x, dvb.y, dvb.z, dvb.w};
      const float4 l0 = reinterpret_cast<const float4*>(LV + c * TILE_LV)[0];
      const float4 l1 = reinterpret_cast<const float4*>(LV + c * TILE_LV)[1];
      const float4 l2 = reinterpret_cast<const float4*>(LV + c * TILE_LV)[2];
      const float vmv[6] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y};
      const float wkm1 = l1.z, wk0 = l1.w, vt = l2.x, rinv = l2.y, fexpl = l2.z;
      const size_t row = ((size_t)iw * mza + kd) * ntp + t0 + 2 * lane;
      const size_t lvl = (size_t)ntp;
      const float2 s0 = U[c * 32 + lane];
      const float2 s00 = Q0[(2 * c) * 32 + lane], st = Q0[(2 * c + 1) * 32 + lane];
      float2 sm1 = s0, sp1 = s0;
      const bool need_m2 = kd != kb && !(wkm1 < 0.f);
      const bool need_p2 = kd != mza - 1 && wk0 < 0.f;
      if (act) {
        if (kd - 1 >= kb) sm1 = __ldg(reinterpret_cast<const float2*>(A.S + row - lvl));
        if (kd + 1 < mza) sp1 = __ldg(reinterpret_cast<const float2*>(A.S + row + lvl));
      }
      float2 sm2 = sm1, sp2 = sp1;
      if (act && need_m2 && kd - 2 >= kb) sm2 = __ldg(reinterpret_cast<const float2*>(A.S + row - 2 * lvl));
      if (act && need_p2 && kd + 2 < mza) sp2 = __ldg(reinterpret_cast<const float2*>(A.S + row + 2 * lvl));
      const float2 ns00 = neg2(s00);
      float2 fd = make_float2(0.f, 0.f);
      const char* Ul = reinterpret_cast<const char*>(U + lane);
      const char* Gl = reinterpret_cast<const char*>(G + lane);
      const int cu = c * 256, cg = c * NPL * 256;
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        // upwind side of face n: the neighbour (inflow) or the cell itself
        const bool inflow = (vmv[n] < 0.f ? 1 : 0) != ((side >> n) & 1);
        const int su = inflow ? nbu[n] : cu, sg = inflow ? nbg[n] : cg;
        const float* off = reinterpret_cast<const float*>(w + TILE_TC_OFF + ((inflow ? 6 : 0) + n) * NPL);
        float2 val = *reinterpret_cast<const float2*>(Ul + su);
        if (NPL == 2) {
          const float2 o2 = *reinterpret_cast<const float2*>(off);
          val = fma2s(o2.x, *reinterpret_cast<const float2*>(Gl + sg), val);
          val = fma2s(o2.y, *reinterpret_cast<const float2*>(Gl + sg + 256), val);
        } else {
#pragma unroll
          for (int m = 0; m < NPL; ++m) val = fma2s(off[m], *reinterpret_cast<const float2*>(Gl + sg + m * 256), val);
        }
        fd = fma2s(dvv[n] * vmv[n], add2(val, ns00), fd);
      }
      // vertical upwind faces kd-1 and kd (grad_z_quadratic, bounded)
      float2 up_lo, up_hi;
      if (kd == kb) up_lo = s0;                                                    // scp_upw(kb-1) = scp(kb)
      else if (wkm1 < 0.f) up_lo = zface_t(aw + 4, mza, kb, kd, true, sm1, s0, sp1);      // scpb(kd)
      else up_lo = zface_t(aw, mza, kb, kd - 1, false, sm2, sm1, s0);                     // scpt(kd-1)
      if (kd == mza - 1) up_hi = s0;                                               // scp_upw(mza) = scp(mza)
      else if (wk0 < 0.f) up_hi = zface_t(aw + 8, mza, kb, kd + 1, true, s0, sp1, sp2);   // scpb(kd+1)
      else up_hi = zface_t(aw + 4, mza, kb, kd, false, sm1, s0, sp1);                     // scpt(kd)
      float2 o;
      {
        float v = fexpl * (wkm1 * (up_lo.x - s00.x) - wk0 * (up_hi.x - s00.x));
        o.x = s00.x + (st.x + vt * (fd.x + v)) * rinv;
        v = fexpl * (wkm1 * (up_lo.y - s00.y) - wk0 * (up_hi.y - s00.y));
        o.y = s00.y + (st.y + vt * (fd.y + v)) * rinv;
      }
      if (act) {
        *reinterpret_cast<float2*>(A.OUT + row) = o;
        if (kd == kb)
          for (int k2 = 0; k2 < kb; ++k2)
            *reinterpret_cast<float2*>(A.OUT + ((size_t)iw * mza + k2) * ntp + t0 + 2 * lane) = o;
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
