// transport_adjoint.cu -- adjoint of one unlimited scalar_transport_rk step
// (omodel/scalar_transport_rk.F90:30-615 with iscal_monot = 0 and no
// horizontal diffusion) for every registered tracer, on the batched layout.
//
// With the winds and densities fixed the step maps (scp, sct) linearly to
// the new scp; the adjoint applies the transpose, stage by stage in reverse:
//   k_weights       (transport_tile.cu) the per-(column, level) records of
//                   the forward's slot weights W, SW, volti / rhos, 1 / rhos
//                   and SW - sum W, once per step
//   k_adj_fold0     the forward copies level kb to the levels below it
//   k_adj_implicit  transpose of the implicit columns' tridif_fini solve
//   k_tile_adj      transpose of update_scalar per tile: for each column x,
//                   the slot weights of the columns that have x as a slot
//                   (the transposed slot table), the vertical quadratic
//                   faces transposed per face, and the scp0 / sct terms
// lam0 collects the adjoint of scp0 (the stage input of every stage's s00
// terms and the columns outside jtw_prog), lams the adjoint of sct.
#include "transport_kernels.cuh"

namespace olamgpu {

// columns outside jtw_prog keep their values through the step: their
// adjoint passes straight to lam0; lam0 and lams start at zero elsewhere
__global__ void k_adj_nonprog(const int* __restrict__ cols, int ncol, size_t colsize, float* __restrict__ lam,
                              float* __restrict__ lam0) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)ncol * colsize) return;
  const size_t x = (size_t)cols[i / colsize] * colsize + i % colsize;
  lam0[x] = lam[x];
  lam[x] = 0.f;
}

// the forward stage copies level kb to the levels below: their adjoint folds into kb
__global__ void k_adj_fold0(const int* __restrict__ prog, int nprog, const int* __restrict__ lpw, int mza, int ntp,
                            float* __restrict__ lam) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * ntp) return;
  const int iw = prog[i / ntp], t = (int)(i % ntp);
  const int kb = lpw[iw];
  float* c = lam + (size_t)iw * mza * ntp + t;
  float a = c[(size_t)kb * ntp];
  for (int k = 0; k < kb; ++k) { a += c[(size_t)k * ntp]; c[(size_t)k * ntp] = 0.f; }
  c[(size_t)kb * ntp] = a;
}

// transpose of the implicit vertical step (scalar_transport_rk.F90:347-375,
// tridif_fini): out' = s0 + T^-1 (out - s0 - G s0) with T = L U,
// L(k,k) = 1/cji(k), L(k,k-1) = b1(k), U(k,k+1) = scr1(k+1).  For lam' the
// adjoint of out': nu = T^-T lam', lam(out) = nu, lam0 += lam' - nu - G^T nu.
// One thread per (implicit column, tracer), sequential in k.
__global__ void k_adj_implicit(GridK g, const int* __restrict__ list, const int* __restrict__ count,
                               const float* __restrict__ b, const float* __restrict__ ff,
                               const float* __restrict__ wmasc, const float* __restrict__ rhos_st, int nrk,
                               int istage, float dtr, int ntp, float* __restrict__ lam, float* __restrict__ lam0) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *count;
  if (i >= (size_t)n * ntp) return;
  const int slot = (int)(i / ntp), t = (int)(i % ntp);
  const int mza = g.mza;
  const int iw = list[slot];
  const int kb = g.lpw[iw];
  const float* b1 = b + (size_t)slot * 3 * mza;
  const float* scr1 = b1 + mza;
  const float* cji = b1 + 2 * mza;
  const float* wm = wmasc + (size_t)iw * mza;
  const float ffv = ff[(size_t)iw * nrk + istage - 1];
  float* L = lam + (size_t)iw * mza * ntp + t;
  float* L0 = lam0 + (size_t)iw * mza * ntp + t;
  auto at = [&](float* p, int kd) -> float& { return p[(size_t)kd * ntp]; };
  for (int kd = 1; kd < kb; ++kd) { at(L, kb) += at(L, kd); at(L, kd) = 0.f; }
  // U^T z = lam' (forward sweep), kept in lam
  float prev = 0.f;
  for (int kd = kb; kd < mza; ++kd) {
    const float z = at(L, kd) - (kd > kb ? scr1[kd] * prev : 0.f);
    at(L0, kd) += at(L, kd);   // lam' part of lam0 += lam' - nu
    at(L, kd) = z;
    prev = z;
  }
  // L^T nu = z (backward sweep), then lam0 -= nu + G^T nu
  float nxt = 0.f;
  for (int kd = mza - 1; kd >= kb; --kd) {
    const float nu = cji[kd] * (at(L, kd) - (kd < mza - 1 ? b1[kd + 1] * nxt : 0.f));
    at(L, kd) = nu;
    nxt = nu;
    at(L0, kd) -= nu;
    const float c1 = ffv * dtr * g.volti[(size_t)iw * mza + kd] / rhos_st[(size_t)iw * mza + kd];
    const float gk = -c1 * nu;
    if (kd <= mza - 2) {   // min(wmasc(k),0) * (s0(k+1) - s0(k))
      const float a = fminf(wm[kd], 0.f) * gk;
      at(L0, kd + 1) += a;
      at(L0, kd) -= a;
    }
    if (kd - 1 >= kb) {    // max(wmasc(k-1),0) * (s0(k) - s0(k-1))
      const float a = fmaxf(wm[kd - 1], 0.f) * gk;
      at(L0, kd) += a;
      at(L0, kd - 1) -= a;
    }
  }
}

// ---- transpose of update_scalar over a tile -----------------------------------
struct TileAdjArgs {
  int mza, ntp, nrk, istage, kb, ntiles, T, nu_max, mwa;
  float dtr;
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const int* __restrict__ tc;
  const int* __restrict__ rev;
  const float* __restrict__ a_w;
  const float* __restrict__ wmasc;
  const float* __restrict__ ff;
  const float* __restrict__ wrec;   // (mwa, mza, TILE_WR)
  const float* __restrict__ L;      // adjoint of the stage output (batched layout)
  float* __restrict__ LIN;          // adjoint of the stage input
  float* __restrict__ L0;           // adjoint of scp0, accumulated
  float* __restrict__ LS;           // adjoint of sct, accumulated
  int* err;
};

#define TADJ_THREADS 256
#define TADJ_NW (TADJ_THREADS / 32)
#define TADJ_CF 28   // per column and level: TILE_NS slot coefficients, 5 vertical, lam0 and sct factors

__device__ __forceinline__ void cpa16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

struct G4 { float2 a, b; };
__device__ __forceinline__ G4 lds_g4(const char* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return G4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ G4 ldg_g4(const float* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return G4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ G4 fma_g4(float w, G4 x, G4 acc) {
  const float2 w2 = make_float2(w, w);
  return G4{__ffma2_rn(w2, x.a, acc.a), __ffma2_rn(w2, x.b, acc.b)};
}
__device__ __forceinline__ void st_g4(float* p, G4 v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}

__global__ void __launch_bounds__(TADJ_THREADS, 2) k_tile_adj(TileAdjArgs A) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int tile = blockIdx.x % A.ntiles, grp = blockIdx.x / A.ntiles;
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nT = h.w;
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  unsigned char* p = smraw;
  char* U = reinterpret_cast<char*>(p);   p += al((size_t)A.nu_max * 256);              // lam rows
  float* WS = reinterpret_cast<float*>(p); p += al((size_t)A.nu_max * TILE_WR * 4 + 16); // weight records (+ zeros)
  float* CF = reinterpret_cast<float*>(p); p += al((size_t)A.T * TADJ_CF * 4);
  int* REV = reinterpret_cast<int*>(p);    p += al((size_t)A.T * TILE_NS * 4);
  int* IWT = reinterpret_cast<int*>(p);    p += al((size_t)A.T * 4);
  int* UIW = reinterpret_cast<int*>(p);    p += al((size_t)A.nu_max * 4);
  float* AW = reinterpret_cast<float*>(p);  // a_w at levels kd-2 .. kd+2 (4 each)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  int bad = (nU > A.nu_max || nT > A.T || nT > nU) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nT * TILE_NS; i += TADJ_THREADS) {
      const int v = __ldg(A.rev + (size_t)tile * A.T * TILE_NS + i);
      if ((unsigned)(v >> 8) >= (unsigned)nU || (v & 255) > TILE_NS) bad = 11;
      REV[i] = v;
    }
    for (int i = tid; i < nT; i += TADJ_THREADS) {
      const int v = __ldg(A.tc + ((size_t)tile * A.T + i) * TILE_TCW + TILE_TC_IW);
      if (v < 1 || v >= A.mwa) bad = 12;
      IWT[i] = v;
    }
    for (int i = tid; i < nU; i += TADJ_THREADS) {
      const int v = __ldg(A.ulist + u_off + i);
      if (v < 1 || v >= A.mwa) bad = 13;
      UIW[i] = v;
    }
    if (tid < 4) WS[(size_t)nU * TILE_WR + tid] = 0.f;
  }
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }

  const int mza = A.mza, ntp = A.ntp, kb = A.kb;
  const int t0 = grp * 64;
  const int seg = min(64, ntp - t0);
  const int nch = seg >> 2;
  const int half = lane >> 4, hl = lane & 15;
  const bool act = 4 * hl < seg;
  const float dtr = A.dtr;

  auto stage = [&](int kd) {
    for (int i = tid; i < nU * 16; i += TADJ_THREADS) {
      const int r = i >> 4, ch = i & 15;
      if (ch < nch) cpa16(U + r * 256 + ch * 16, A.L + ((size_t)UIW[r] * mza + kd) * ntp + t0 + ch * 4);
    }
    for (int i = tid; i < nU * (TILE_WR / 4); i += TADJ_THREADS) {
      const int r = i / (TILE_WR / 4), ch = i - r * (TILE_WR / 4);
      cpa16(WS + r * TILE_WR + ch * 4, A.wrec + ((size_t)UIW[r] * mza + kd) * TILE_WR + ch * 4);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (tid < 20) {
      const int lev = kd - 2 + tid / 4, m = tid & 3;
      AW[tid] = (lev >= 0 && lev < mza) ? __ldg(A.a_w + lev + m * mza) : 0.f;
    }
  };

  stage(kb);
  for (int kd = kb; kd < mza; ++kd) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    // ---- phase C: coefficients of this level, a thread per (column, entry)
    for (int i = tid; i < nT * (TILE_NS + 1); i += TADJ_THREADS) {
      const int c = i / (TILE_NS + 1), e = i - c * (TILE_NS + 1);
      float* cf = CF + c * TADJ_CF;
      if (e < TILE_NS) {
        // the column across this transposed slot: its weight of our column, times
        // dtr * volti / rhos of that column
        const int v = REV[c * TILE_NS + e];
        const int uu = v >> 8, j = v & 255;
        cf[e] = j < TILE_NS ? dtr * WS[uu * TILE_WR + j] * WS[uu * TILE_WR + TILE_NS + 1] : 0.f;
        continue;
      }
      // the vertical faces kd-2 .. kd+1 transposed, and the own-column terms
      const int iw = IWT[c];
      const float* wm = A.wmasc + (size_t)iw * mza;
      const float fexpl = 1.0f - __ldg(A.ff + (size_t)iw * A.nrk + A.istage - 1);
      float cm[5] = {0.f, 0.f, 0.f, 0.f, 0.f};   // coefficients of mu(kd-2 .. kd+2)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int f = kd - 2 + q;
        if (f < kb || f > mza - 2) continue;
        const float w = __ldg(wm + f);
        const bool neg = w < 0.f;                 // upwind level f+1 (its bottom face), else f (top)
        const int lev = neg ? f + 1 : f;
        const int pos = kd - (neg ? f : f - 1);   // kd's place in the stencil (lev-1, lev, lev+1)
        const float* a = AW + (lev - (kd - 2)) * 4;
        const float c1 = a[neg ? 0 : 2], c2 = a[neg ? 1 : 3];
        const float it = lev <= mza - 2 ? 1.f : 0.f, ib = lev >= kb + 1 ? 1.f : 0.f;
        const float dF = pos == 0 ? -c2 * ib : (pos == 1 ? 1.f - c1 * it + c2 * ib : (pos == 2 ? c1 * it : 0.f));
        const float a2 = fexpl * w * dF;   // lam_F(f) = fexpl wm(f) (mu(f+1) - mu(f))
        cm[q + 1] += a2;
        cm[q] -= a2;
      }
      if (kd == kb) cm[2] += fexpl * __ldg(wm + kb - 1);
      if (kd == mza - 1) cm[2] -= fexpl * __ldg(wm + mza - 1);
      const float* ws = WS + c * TILE_WR;   // the tile columns are the first U rows
      cm[2] += ws[TILE_NS + 3];              // mu(x) (SW - sum W)
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const int k2 = kd - 2 + q;
        const float rv = (k2 >= kb && k2 < mza)
                             ? (q == 2 ? ws[TILE_NS + 1] : __ldg(A.wrec + ((size_t)iw * mza + k2) * TILE_WR + TILE_NS + 1))
                             : 0.f;
        cf[TILE_NS + q] = dtr * rv * cm[q];
      }
      cf[TILE_NS + 5] = 1.0f - dtr * ws[TILE_NS + 1] * (ws[TILE_NS] + fexpl * (__ldg(wm + kd - 1) - __ldg(wm + kd)));
      cf[TILE_NS + 6] = dtr * ws[TILE_NS + 2];
    }
    __syncthreads();
    // ---- phase B: the adjoint of the stage input, lam0 and lams, a half warp per column
    for (int c = 2 * warp + half; c < nT; c += 2 * TADJ_NW) {
      const int iw = IWT[c];
      const float* cf = CF + c * TADJ_CF;
      const size_t row = ((size_t)iw * mza + kd) * ntp + t0 + 4 * hl;
      const size_t lvl = (size_t)ntp;
      const char* Ul = U + hl * 16;
      const G4 lx = lds_g4(Ul + c * 256);
      G4 acc = G4{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      acc = fma_g4(cf[TILE_NS + 2], lx, acc);
#pragma unroll
      for (int q = 0; q < TILE_NS / 4; ++q) {
        const int4 r4 = reinterpret_cast<const int4*>(REV + c * TILE_NS)[q];
        const float4 c4 = reinterpret_cast<const float4*>(cf)[q];
        acc = fma_g4(c4.x, lds_g4(Ul + (r4.x & ~255)), acc);
        acc = fma_g4(c4.y, lds_g4(Ul + (r4.y & ~255)), acc);
        acc = fma_g4(c4.z, lds_g4(Ul + (r4.z & ~255)), acc);
        acc = fma_g4(c4.w, lds_g4(Ul + (r4.w & ~255)), acc);
      }
      if (act) {
        if (kd - 2 >= kb) acc = fma_g4(cf[TILE_NS + 0], ldg_g4(A.L + row - 2 * lvl), acc);
        if (kd - 1 >= kb) acc = fma_g4(cf[TILE_NS + 1], ldg_g4(A.L + row - lvl), acc);
        if (kd + 1 < mza) acc = fma_g4(cf[TILE_NS + 3], ldg_g4(A.L + row + lvl), acc);
        if (kd + 2 < mza) acc = fma_g4(cf[TILE_NS + 4], ldg_g4(A.L + row + 2 * lvl), acc);
        st_g4(A.LIN + row, acc);
        G4 l0 = ldg_g4(A.L0 + row), ls = ldg_g4(A.LS + row);
        l0 = fma_g4(cf[TILE_NS + 5], lx, l0);
        ls = fma_g4(cf[TILE_NS + 6], lx, ls);
        st_g4(A.L0 + row, l0);
        st_g4(A.LS + row, ls);
        if (kd == kb)
          for (int k2 = 0; k2 < kb; ++k2)
            st_g4(A.LIN + ((size_t)iw * mza + k2) * ntp + t0 + 4 * hl, G4{make_float2(0.f, 0.f), make_float2(0.f, 0.f)});
      }
    }
    __syncthreads();
    if (kd + 1 < mza) stage(kd + 1);
  }
}


static size_t tile_adj_smem_bytes(int T, int nu) {
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  return al((size_t)nu * 256) + al((size_t)nu * TILE_WR * 4 + 16) + al((size_t)T * TADJ_CF * 4) +
         al((size_t)T * TILE_NS * 4) + al((size_t)T * 4) + al((size_t)nu * 4) + 20 * 4;
}

static int launch_tile_adj(const DevGrid& d, const Transport& tp, const float* L, float* LIN, float* L0,
                           float* LS, int ntp, int istage, int nrk, float dtr, int* status, cudaStream_t s) {
  TileAdjArgs A;
  A.mza = d.mza; A.ntp = ntp; A.nrk = nrk; A.istage = istage; A.kb = 1;
  A.ntiles = d.ntiles; A.T = d.tile_T; A.nu_max = d.tile_nu_max; A.mwa = d.mwa;
  A.dtr = dtr;
  A.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  A.ulist = d.tile_u.p; A.tc = d.tile_tc.p; A.rev = d.tile_rev.p;
  A.a_w = d.a_w.p; A.wmasc = tp.wmasc.p; A.ff = tp.ff.p; A.wrec = tp.wrec.p;
  A.L = L; A.LIN = LIN; A.L0 = L0; A.LS = LS;
  A.err = status;
  const size_t smem = tile_adj_smem_bytes(d.tile_T, d.tile_nu_max);
  if (smem > 227 * 1024) { set_error("adjoint tile neighbourhood exceeds shared memory"); return OLAMGPU_E_UNSUPPORTED; }
  const unsigned ngrp = (unsigned)((ntp + 63) / 64);
  OG_CUDA(cudaFuncSetAttribute(k_tile_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_tile_adj<<<(unsigned)d.ntiles * ngrp, TADJ_THREADS, smem, s>>>(A);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

__global__ void k_adj_finish(size_t n, float* __restrict__ lam, const float* __restrict__ lam0) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lam[i] += lam0[i];
}

// per-tracer planes of the caller's arrays <-> the batched layout
static int planes_table(Transport& tp, int n, size_t plane, cudaStream_t s) {
  std::vector<float*> h(n);
  for (int i = 0; i < n; ++i) h[i] = tp.adj_planes.p + (size_t)i * plane;
  OG_CHECK(tp.adj_ptab.alloc(n));
  OG_CUDA(cudaMemcpyAsync(tp.adj_ptab.p, h.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
  OG_CUDA(cudaStreamSynchronize(s));   // h dies here
  return OLAMGPU_OK;
}

int transport_adjoint_run(const float* rho_old_host, float* const* lam, float* const* lam_sct) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!C.have_state || !C.hstate.vmasc || !C.hstate.wmasc || !C.hstate.rho) {
    set_error("state arrays vmasc/wmasc/rho were not registered at init");
    return OLAMGPU_E_STATE;
  }
  const int n = C.tr.n;
  if (n <= 0) return OLAMGPU_OK;
  if (!lam || !lam_sct) { set_error("lam and lam_sct must be arrays of num_scalar pointers"); return OLAMGPU_E_ARG; }
  for (int i = 0; i < n; ++i)
    if (!lam[i] || !lam_sct[i]) { set_error("a lam or lam_sct entry is NULL"); return OLAMGPU_E_ARG; }
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  cudaStream_t s = C.stream;
  const int mza = d.mza, mwa = d.mwa;
  const int nrk = C.opts.nrk_scal;
  const int order = C.opts.scal_horiz_adv_order;
  if (nrk != 2 && nrk != 3) { set_error("scalar_timestep_level must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (order != 2 && order != 3) { set_error("scal_horiz_adv_order must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (C.opts.iscal_monot != 0) {
    set_error("the adjoint covers the unlimited transport (iscal_monot = 0) only");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (tp.have_turb) {
    set_error("the adjoint does not cover horizontal diffusion of the tracers");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (!tile_stage_available(d, tp, order)) {
    set_error("the adjoint needs the tiled transport tables (grids without terrain, lpw = lpv = 2)");
    return OLAMGPU_E_UNSUPPORTED;
  }
  const int ntp = C.tr.ntp;
  const size_t plane = (size_t)mza * mwa, qn = plane * ntp;

  OG_CHECK(tp.adj_l[0].alloc(qn));
  OG_CHECK(tp.adj_l[1].alloc(qn));
  OG_CHECK(tp.adj_l0.alloc(qn));
  OG_CHECK(tp.adj_ls.alloc(qn));
  OG_CHECK(tp.adj_planes.alloc(plane * n));
  OG_CHECK(planes_table(tp, n, plane, s));
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(tp.adj_planes.p + (size_t)i * plane, lam[i], plane * sizeof(float),
                            cudaMemcpyHostToDevice, s));

  {
    // device work of the step (in RESIDENT mode the preparation uploads nothing)
    OG_PROF("adjoint", s);
    OG_CUDA(cudaMemsetAsync(tp.adj_l[1].p, 0, qn * sizeof(float), s));
    OG_CUDA(cudaMemsetAsync(tp.adj_l0.p, 0, qn * sizeof(float), s));
    OG_CUDA(cudaMemsetAsync(tp.adj_ls.p, 0, qn * sizeof(float), s));
    float dtlr[3];
    OG_CHECK(transport_prepare(C, rho_old_host, false, dtlr));
    const float* rhos_nrk = tp.rhos.p + (size_t)(nrk - 1) * plane;
    { OG_PROF("adj_gather", s); launch_gather_q(tp.adj_l[0].p, (const float* const*)tp.adj_ptab.p, n, ntp, plane, s); }
    { OG_PROF("adj_weights", s); OG_CHECK(launch_tile_weights(d, tp, rhos_nrk, s)); }
    float* L = tp.adj_l[0].p;
    float* LIN = tp.adj_l[1].p;
    const size_t colsize = (size_t)mza * ntp;
    if (d.n_nonprog > 0) {
      k_adj_nonprog<<<cdiv((size_t)d.n_nonprog * colsize, 256), 256, 0, s>>>(d.w_nonprog.p, d.n_nonprog, colsize,
                                                                            L, tp.adj_l0.p);
      OG_LAUNCHED();
    }
    for (int istage = nrk; istage >= 1; --istage) {
      const float dtr = dtlr[istage - 1];
      {
        OG_PROF("adj_implicit", s);
        k_adj_implicit<<<cdiv((size_t)d.nw_prog * ntp, 128), 128, 0, s>>>(
            gridk(d), tp.imp_list.p + (size_t)(istage - 1) * mwa, tp.imp_count.p + (istage - 1),
            tp.imp_b.p + (size_t)(istage - 1) * mwa * 3 * mza, tp.ff.p, tp.wmasc.p,
            tp.rhos.p + (size_t)(istage - 1) * plane, nrk, istage, dtr, ntp, L, tp.adj_l0.p);
        OG_LAUNCHED();
        k_adj_fold0<<<cdiv((size_t)d.nw_prog * ntp, 256), 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, mza, ntp, L);
        OG_LAUNCHED();
      }
      {
        OG_PROF("adj_stage", s);
        OG_CHECK(launch_tile_adj(d, tp, L, LIN, tp.adj_l0.p, tp.adj_ls.p, ntp, istage, nrk, dtr, C.status.p, s));
      }
      std::swap(L, LIN);
    }
    k_adj_finish<<<cdiv(qn, 256), 256, 0, s>>>(qn, L, tp.adj_l0.p);
    OG_LAUNCHED();
    launch_scatter_q(L, tp.adj_ptab.p, n, ntp, plane, s);
  }
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam[i], tp.adj_planes.p + (size_t)i * plane, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  launch_scatter_q(tp.adj_ls.p, tp.adj_ptab.p, n, ntp, plane, s);
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam_sct[i], tp.adj_planes.p + (size_t)i * plane, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

}  // namespace olamgpu
