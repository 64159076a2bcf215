// transport_adjoint.cu -- adjoint of one unlimited scalar_transport_rk step
// (omodel/scalar_transport_rk.F90:30-615 with iscal_monot = 0 and no
// horizontal diffusion) for every registered tracer, on the batched layout.
//
// With the winds and densities fixed the step maps (scp, sct) linearly to
// the new scp; the adjoint applies the transpose, stage by stage in reverse:
//   k_weights       (transport_tile.cu) the forward's per-(column, level)
//                   records: slot weights W, SW, volti / rhos, 1 / rhos,
//                   SW - sum W, once per step
//   k_adj_records   their transpose per (column x, level): for every column
//                   c that has x as its slot j (the transposed slot table),
//                   W_{c,j} volti_c / rhos_c; the vertical quadratic faces
//                   transposed into coefficients on lam(kd-2 .. kd+2); the
//                   own-column factors of lam(scp0) and lam(sct)
//   k_adj_implicit  transpose of the implicit columns' tridif_fini solve
//   k_adj_fold0     the forward copies level kb to the levels below it
//   k_tile_adj      transpose of update_scalar per tile: a gather over the
//                   transposed slots and the column's own levels
// lam0 collects the adjoint of scp0 (the s00 terms of every stage and the
// columns outside jtw_prog), lams the adjoint of sct.  Neither is cleared
// first: the first reverse stage writes them, later stages accumulate.
#include <algorithm>

#include "transport_kernels.cuh"
#include "tile_common.cuh"

namespace olamgpu {

// Columns outside jtw_prog keep their values through the step, so their
// adjoint passes through: the buffer the last reverse stage writes holds lam
// there, the other lam buffer and lams hold zero.
__global__ void k_adj_nonprog(const int* __restrict__ cols, int ncol, size_t colsize, float* __restrict__ lam,
                              float* __restrict__ other, float* __restrict__ lams, int final_is_other) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)ncol * colsize) return;
  const size_t x = (size_t)cols[i / colsize] * colsize + i % colsize;
  const float v = lam[x];
  if (lams) lams[x] = 0.f;   // (a window's sum keeps its zero there)
  if (final_is_other) { other[x] = v; lam[x] = 0.f; }
  else other[x] = 0.f;
}

// the forward stage copies level kb to the levels below: their adjoint folds
// into kb.  Blocks stride over the prognostic columns, threads over the tracers.
// thread per (column, four tracers); ntp is a multiple of 4
__global__ void k_adj_fold0(const int* __restrict__ prog, int nprog, const int* __restrict__ lpw, int mza, int ntp,
                            float* __restrict__ lam) {
  const int nq = ntp >> 2;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * nq) return;
  const int j = (int)(i / nq), t = (int)(i - (size_t)j * nq) * 4;
  const int iw = prog[j];
  const int kb = lpw[iw];
  float* c = lam + (size_t)iw * mza * ntp + t;
  float4 a = *reinterpret_cast<const float4*>(c + (size_t)kb * ntp);
  for (int k = 0; k < kb; ++k) {
    float4* p = reinterpret_cast<float4*>(c + (size_t)k * ntp);
    const float4 v = *p;
    a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
    *p = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  *reinterpret_cast<float4*>(c + (size_t)kb * ntp) = a;
}

// transpose of the implicit vertical step (scalar_transport_rk.F90:347-375,
// tridif_fini): out' = s0 + T^-1 (out - s0 - G s0) with T = L U,
// L(k,k) = 1/cji(k), L(k,k-1) = b1(k), U(k,k+1) = scr1(k+1).  For lam' the
// adjoint of out': nu = T^-T lam', lam(out) = nu, lam0 += lam' - nu - G^T nu.
// One thread per (implicit column, tracer), sequential in k.  On the first
// reverse stage (first != 0) lam0 of the column starts from zero.
__global__ void k_adj_implicit(GridK g, const int* __restrict__ list, const int* __restrict__ count,
                               const float* __restrict__ b, const float* __restrict__ ff,
                               const float* __restrict__ wmasc, const float* __restrict__ rhos_st, int nrk,
                               int istage, float dtr, int ntp, int first, float* __restrict__ lam,
                               float* __restrict__ lam0) {
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
  if (first)
    for (int kd = kb; kd < mza; ++kd) at(L0, kd) = 0.f;
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

// ---- transposed records, once per step -----------------------------------------
// Per (tile column x, level kd), TADJ_RW floats:
//   [0, TILE_NS)   W_{c,j} volti_c / rhos_c for the e-th (c, j) with x in
//                  c's slot j (0 for unused entries)
//   [20, 25)       the vertical faces transposed: coefficient of
//                  lam(kd-2+q) is dtr (fexpl a_q + (q == 2) d)
//   25 d           volti / rhos (SW - sum W), the diagonal of the horizontal part
//   26, 27         volti / rhos SW and volti / rhos (wmasc(kd-1) - wmasc(kd)):
//                  lam(scp0) gains lam (1 - dtr (b26 + fexpl b27))
//   28             1 / rhos: lam(sct) gains lam dtr / rhos
#define TADJ_RW 32

struct AdjRecArgs {
  int mza, T, kb, mwa;
  const int* __restrict__ lpw;      // each W column's floor (device level)
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const int* __restrict__ tc;
  const int* __restrict__ rev;
  const float* __restrict__ wrec;   // (mwa, mza, TILE_WR)
  const float* __restrict__ wmasc;
  const float* __restrict__ a_w;    // Fortran (mza, 2, 2)
  float* __restrict__ trec;         // (mwa, mza, TADJ_RW)
  int* err;
};

// one block per tile column, a thread per level
__global__ void k_adj_records(AdjRecArgs A) {
  __shared__ int cols[TILE_NS], js[TILE_NS], kbs[TILE_NS];
  __shared__ int xs;
  const int t = blockIdx.x / A.T, i = blockIdx.x - t * A.T;
  const int4 h = A.hdr[t];
  if (i >= h.w) return;   // padding of the last tile (uniform per block)
  if (threadIdx.x < TILE_NS) {
    const int v = __ldg(A.rev + (size_t)blockIdx.x * TILE_NS + threadIdx.x);
    int uu = v >> 8, j = v & 255;
    if ((unsigned)uu >= (unsigned)h.y || j > TILE_NS) {   // inconsistent table: record, contribute nothing
      if (atomicCAS(A.err, 0, 121) == 0) { A.err[1] = t; A.err[2] = blockIdx.x; A.err[3] = threadIdx.x; }
      uu = 0; j = TILE_NS;
    }
    int c = __ldg(A.ulist + h.x + uu);
    if (c < 1 || c >= A.mwa) { c = 1; j = TILE_NS; }
    cols[threadIdx.x] = c;
    js[threadIdx.x] = j;
    kbs[threadIdx.x] = max(A.kb, __ldg(A.lpw + c));   // c is prognosed from this level up
  }
  if (threadIdx.x == 0) {
    int x = __ldg(A.tc + (size_t)blockIdx.x * TILE_TCW + TILE_TC_IW);
    xs = (x >= 1 && x < A.mwa) ? x : 0;
  }
  __syncthreads();
  const int x = xs, mza = A.mza;
  if (x == 0) return;
  const int kb = max(A.kb, __ldg(A.lpw + x));   // x's own floor
  const float* wm = A.wmasc + (size_t)x * mza;
  auto rec = [&](int col, int k) { return A.wrec + ((size_t)col * mza + k) * TILE_WR; };
  for (int kd = kb + threadIdx.x; kd < mza; kd += blockDim.x) {
    float* o = A.trec + ((size_t)x * mza + kd) * TADJ_RW;
    float v4[4];
#pragma unroll
    for (int e = 0; e < TILE_NS; ++e) {
      const int j = js[e];
      const float* rc = rec(cols[e], kd);
      v4[e & 3] = (j < TILE_NS && kd >= kbs[e]) ? __ldg(rc + j) * __ldg(rc + TILE_NS + 1) : 0.f;
      if ((e & 3) == 3) reinterpret_cast<float4*>(o)[e >> 2] = make_float4(v4[0], v4[1], v4[2], v4[3]);
    }
    // faces f = kd-2 .. kd+1 (the ones whose upwind stencil can hold level
    // kd): lam_F(f) = fexpl wm(f) (mu(f+1) - mu(f)) times dF/dS(kd)
    float V[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int f = kd - 2 + q;
      if (f < kb || f > mza - 2) continue;
      const float w = __ldg(wm + f);
      const bool neg = w < 0.f;                 // upwind level f+1 (its bottom face), else f (top)
      const int lev = neg ? f + 1 : f;
      const int pos = kd - (neg ? f : f - 1);   // kd's place in the stencil (lev-1, lev, lev+1)
      const float c1 = __ldg(A.a_w + lev + (neg ? 0 : 2) * mza), c2 = __ldg(A.a_w + lev + (neg ? 1 : 3) * mza);
      const float it = lev <= mza - 2 ? 1.f : 0.f, ib = lev >= kb + 1 ? 1.f : 0.f;
      const float dF = pos == 0 ? -c2 * ib : (pos == 1 ? 1.f - c1 * it + c2 * ib : (pos == 2 ? c1 * it : 0.f));
      V[q + 1] += w * dF;
      V[q] -= w * dF;
    }
    if (kd == kb) V[2] += __ldg(wm + kb - 1);
    if (kd == mza - 1) V[2] -= __ldg(wm + mza - 1);
    const float* rx = rec(x, kd);
    const float rv = __ldg(rx + TILE_NS + 1);
    float a[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int k2 = kd - 2 + q;
      a[q] = (k2 >= kb && k2 < mza) ? (q == 2 ? rv : __ldg(rec(x, k2) + TILE_NS + 1)) * V[q] : 0.f;
    }
    reinterpret_cast<float4*>(o)[5] = make_float4(a[0], a[1], a[2], a[3]);
    reinterpret_cast<float4*>(o)[6] = make_float4(a[4], rv * __ldg(rx + TILE_NS + 3), rv * __ldg(rx + TILE_NS),
                                                  rv * (__ldg(wm + kd - 1) - __ldg(wm + kd)));
    reinterpret_cast<float4*>(o)[7] = make_float4(__ldg(rx + TILE_NS + 2), 0.f, 0.f, 0.f);
  }
}

// ---- transpose of update_scalar over a tile -----------------------------------
struct TileAdjArgs {
  int mza, ntp, nrk, istage, kb, ntiles, T, nu_max, mwa;
  const int* __restrict__ lpw;      // each W column's floor (device level)
  float dtr;
  int first, last;                  // first / last reverse stage of the step
  int ls_first;                     // LS is written, not accumulated (the first stage, unless a window sums it)
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const int* __restrict__ tc;
  const int* __restrict__ rev;
  const float* __restrict__ ff;     // (mwa, nrk)
  const float* __restrict__ trec;   // (mwa, mza, TADJ_RW)
  const float* __restrict__ L;      // adjoint of the stage output (batched layout)
  float* __restrict__ LIN;          // adjoint of the stage input (last stage: of the old scp)
  float* __restrict__ L0;           // adjoint of scp0
  float* __restrict__ LS;           // adjoint of sct
  const int* skip;                  // (ntr) or NULL: tracers whose results this launch leaves alone
  int ntr;                          // registered tracers (skip's length)
  int* err;
};

#define TADJ_THREADS 256

// a row of four tracers, leaving the ones flagged in mask (bit j: tracer j) alone
__device__ __forceinline__ void stg4m(float* p, F4 v, int mask) {
  if (mask == 0) { stg4(p, v); return; }
  if (mask == 15) return;
  if (!(mask & 1)) p[0] = v.a.x;
  if (!(mask & 2)) p[1] = v.a.y;
  if (!(mask & 4)) p[2] = v.b.x;
  if (!(mask & 8)) p[3] = v.b.y;
}

// G tracers per block: a U row of the tile's neighbourhood is 4 G bytes
size_t tile_adj_smem_bytes(int T, int nu, int G = 64) {
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  return 2 * al((size_t)nu * 4 * G) + 2 * al((size_t)T * TADJ_RW * 4) + al((size_t)nu * 8) +
         al((size_t)T * TILE_NS * 4) + 2 * al((size_t)T * 4);
}

// The same sweep as k_tile: level kd+1 is copied into one buffer while kd is
// computed from the other; G / 4 lanes own NC columns (four tracers a lane,
// G tracers a block: 64, or 32 so that 32 tracers leave no lane idle) with
// lam of the column's levels kd-2 .. kd+3 and its lam0 / lams rows in
// registers.
//   lam_in(x) = dtr (sum_e T_e lam(c_e) + sum_q (fexpl a_q + [q == 2] d) lam(kd-2+q))
//   lam0 += lam (1 - dtr (b26 + fexpl b27)),  lams += lam dtr / rhos
// On the first reverse stage lam0 is read only in implicit columns (the
// implicit transpose wrote it there) and lams is not read; on the last the
// result lam_in + lam0 is the adjoint of the old scp, written to LIN.
template <int NC, int G>
__global__ void __launch_bounds__(TADJ_THREADS, 2) k_tile_adj(TileAdjArgs A) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int LPC = G / 4;                        // lanes per column
  constexpr int CPW = 32 / LPC;                     // columns per warp
  constexpr int NG = CPW * (TADJ_THREADS / 32);     // column groups of a block
  constexpr int T = NG * NC;
  constexpr int RB = 4 * G;                         // bytes of a staged U row
  static_assert(G == 32 || G == 64, "32 or 64 tracers per block");
  const int ngrp = (A.ntp + G - 1) / G;   // the tracer groups of a tile side by side
  const int tile = blockIdx.x / ngrp, grp = blockIdx.x - tile * ngrp;
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nT = h.w;
  const int mza = A.mza, ntp = A.ntp, kb = A.kb;
  auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t ubuf = al((size_t)A.nu_max * RB), rbuf = al((size_t)T * TADJ_RW * 4);
  unsigned char* p = smraw;
  char* UB = reinterpret_cast<char*>(p);              p += 2 * ubuf;
  unsigned char* RBB = p;                             p += 2 * rbuf;
  long long* ROW = reinterpret_cast<long long*>(p);   p += al((size_t)A.nu_max * 8);
  int* REVO = reinterpret_cast<int*>(p);              p += al((size_t)T * TILE_NS * 4);
  int* IWT = reinterpret_cast<int*>(p);               p += al((size_t)T * 4);
  float* FEX = reinterpret_cast<float*>(p);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t0 = grp * G;

  int bad = (nU > A.nu_max || nT > T || nT > nU || A.T != T) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nT * TILE_NS; i += TADJ_THREADS) {
      const int v = __ldg(A.rev + (size_t)tile * T * TILE_NS + i);
      if ((unsigned)(v >> 8) >= (unsigned)nU || (v & 255) > TILE_NS) bad = 11;
      REVO[i] = (v >> 8) * RB;
    }
    for (int i = tid; i < nT; i += TADJ_THREADS) {
      const int v = __ldg(A.tc + ((size_t)tile * T + i) * TILE_TCW + TILE_TC_IW);
      if (v < 1 || v >= A.mwa) bad = 12;
      IWT[i] = v;
    }
    for (int i = tid; i < nU; i += TADJ_THREADS) {
      const int v = __ldg(A.ulist + u_off + i);
      if (v < 1 || v >= A.mwa) bad = 13;
      ROW[i] = (long long)v * mza * ntp + t0;
    }
  }
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }
  for (int i = tid; i < nT; i += TADJ_THREADS) FEX[i] = 1.0f - __ldg(A.ff + (size_t)IWT[i] * A.nrk + A.istage - 1);

  const int seg = min(G, ntp - t0);
  const int nch = seg >> 2;
  const int ch = tid & (LPC - 1);
  auto stage = [&](int k, int b) {
    char* Ub = UB + b * ubuf;
    float* Rb = reinterpret_cast<float*>(RBB + b * rbuf);
    const long long koff = (long long)k * ntp + ch * 4;
    if (ch < nch)
      for (int r = tid / LPC; r < nU; r += TADJ_THREADS / LPC) cp_async16(Ub + r * RB + ch * 16, A.L + ROW[r] + koff);
    for (int i = tid; i < nT * (TADJ_RW / 4); i += TADJ_THREADS) {
      const int c = i / (TADJ_RW / 4), q = i - c * (TADJ_RW / 4);
      cp_async16(Rb + c * TADJ_RW + q * 4, A.trec + ((size_t)IWT[c] * mza + k) * TADJ_RW + q * 4);
    }
    cp_async_commit();
  };

  const int sub = lane / LPC, hl = lane % LPC;
  const bool act = 4 * hl < seg;
  const int cb = CPW * warp + sub;
  const bool first = A.first != 0, last = A.last != 0, lsfirst = A.ls_first != 0;
  int skm = 0;   // this lane's tracers whose results are written elsewhere
  if (A.skip)
    for (int j = 0; j < 4; ++j) {
      const int tr = t0 + 4 * hl + j;
      if (tr < A.ntr && A.skip[tr]) skm |= 1 << j;
    }
  const float dtr = A.dtr;
  F4 m2[NC], m1[NC], p1[NC], p2[NC], p3[NC], l0[NC], ls[NC];
  long long cbase[NC];
  bool need0[NC];
  int kbc[NC];   // each column's own floor: levels below it are not prognosed
  stage(kb, 0);
  __syncthreads();   // FEX
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int c = cb + NG * n;
    m2[n] = m1[n] = p1[n] = p2[n] = p3[n] = l0[n] = ls[n] = zero4();
    cbase[n] = 0;
    need0[n] = false;
    kbc[n] = c < nT ? max(kb, __ldg(A.lpw + IWT[c])) : mza;
    if (c < nT && act) {
      need0[n] = !first || FEX[c] < 1.0f;
      cbase[n] = (long long)IWT[c] * mza * ntp + t0 + 4 * hl;
      const float* q = A.L + cbase[n];
      if (kb + 1 < mza) p1[n] = ldg4(q + (long long)(kb + 1) * ntp);
      if (kb + 2 < mza) p2[n] = ldg4(q + (long long)(kb + 2) * ntp);
      if (kb + 3 < mza) p3[n] = ldg4(q + (long long)(kb + 3) * ntp);
      if (need0[n]) l0[n] = ldg4(A.L0 + cbase[n] + (long long)kb * ntp);
      if (!lsfirst) ls[n] = ldg4(A.LS + cbase[n] + (long long)kb * ntp);
    }
  }
  cp_async_wait_all();
  __syncthreads();

  for (int kd = kb; kd < mza; ++kd) {
    const int cur = (kd - kb) & 1;
    if (kd + 1 < mza) stage(kd + 1, cur ^ 1);
    const char* Ul = UB + cur * ubuf + hl * 16;
    const float* Rc = reinterpret_cast<const float*>(RBB + cur * rbuf);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int c = cb + NG * n;
      if (c >= nT) continue;
      if (kd == kbc[n]) m2[n] = m1[n] = zero4();
      const float* rc = Rc + c * TADJ_RW;
      const F4 lx = lds4(Ul, c * RB);
      F4 acc = zero4();
      const int* ro = REVO + c * TILE_NS;
#pragma unroll
      for (int q = 0; q < TILE_NS / 4; ++q) {
        const int4 so = reinterpret_cast<const int4*>(ro)[q];
        const float4 w4 = reinterpret_cast<const float4*>(rc)[q];
        // zero transposed weights (no upwind path between the two columns
        // at this level) are not read
        if (w4.x != 0.f) acc = fma4s(w4.x, lds4(Ul, so.x), acc);
        if (w4.y != 0.f) acc = fma4s(w4.y, lds4(Ul, so.y), acc);
        if (w4.z != 0.f) acc = fma4s(w4.z, lds4(Ul, so.z), acc);
        if (w4.w != 0.f) acc = fma4s(w4.w, lds4(Ul, so.w), acc);
      }
      const float fx = FEX[c];
      const float4 r5 = reinterpret_cast<const float4*>(rc)[5];   // a0 .. a3
      const float4 r6 = reinterpret_cast<const float4*>(rc)[6];   // a4, d, b26, b27
      const float ri = rc[TILE_NS + 8];
      acc = fma4s(fx * r5.x, m2[n], acc);
      acc = fma4s(fx * r5.y, m1[n], acc);
      acc = fma4s(fmaf(fx, r5.z, r6.y), lx, acc);
      acc = fma4s(fx * r5.w, p1[n], acc);
      acc = fma4s(fx * r6.x, p2[n], acc);
      const F4 lin = scale4(dtr, acc);
      const F4 l0n = fma4s(1.0f - dtr * fmaf(fx, r6.w, r6.z), lx, l0[n]);
      const F4 lsn = fma4s(dtr * ri, lx, ls[n]);
      if (act) {
        const long long row = cbase[n] + (long long)kd * ntp;
        if (kd >= kbc[n]) {
          if (last) {
            stg4m(A.LIN + row, add4(lin, l0n), skm);
          } else {
            stg4m(A.LIN + row, lin, skm);
            stg4m(A.L0 + row, l0n, skm);
          }
          stg4m(A.LS + row, lsn, skm);
        }
        // the stage reads no level below the column's floor
        if (kd == kbc[n])
          for (int k2 = 0; k2 < kd; ++k2) {
            const long long r2 = cbase[n] + (long long)k2 * ntp;
            stg4m(A.LIN + r2, zero4(), skm);
            if (first) stg4m(A.L0 + r2, zero4(), skm);
            if (lsfirst) stg4m(A.LS + r2, zero4(), skm);
          }
        // slide the column's window up one level and read ahead
        m2[n] = m1[n]; m1[n] = lx; p1[n] = p2[n]; p2[n] = p3[n];
        if (kd + 4 < mza) p3[n] = ldg4(A.L + cbase[n] + (long long)(kd + 4) * ntp);
        if (kd + 1 < mza) {
          if (need0[n]) l0[n] = ldg4(A.L0 + cbase[n] + (long long)(kd + 1) * ntp);
          if (!lsfirst) ls[n] = ldg4(A.LS + cbase[n] + (long long)(kd + 1) * ntp);
        }
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
}

// the tiles the reverse stage runs: the adjoint's own 32-column tiles when
// they are built and fit in shared memory, else the stage kernel's
struct AdjTiles {
  const int4* hdr;
  const int *u, *tc, *rev;
  int T, ntiles, nu_max;
};

static AdjTiles adj_tiles_of(const DevGrid& d) {
  const auto& a = d.adj_tiles;
  if (a.T == 32 && a.order == d.tile_order && tile_adj_smem_bytes(a.T, a.nu_max) <= 227 * 1024)
    return {reinterpret_cast<const int4*>(a.hdr.p), a.u.p, a.tc.p, a.rev.p, a.T, a.ntiles, a.nu_max};
  return {reinterpret_cast<const int4*>(d.tile_hdr.p), d.tile_u.p, d.tile_tc.p, d.tile_rev.p,
          d.tile_T, d.ntiles, d.tile_nu_max};
}

static int launch_tile_adj(const DevGrid& d, const Transport& tp, const float* L, float* LIN, float* L0, float* LS,
                           int ntp, int istage, int nrk, float dtr, int first, int last, int ls_first,
                           int* status, cudaStream_t s, const int* skip = nullptr, int ntr = 0) {
  const AdjTiles t = adj_tiles_of(d);
  TileAdjArgs A;
  A.skip = skip; A.ntr = ntr;
  A.mza = d.mza; A.ntp = ntp; A.nrk = nrk; A.istage = istage; A.kb = 1; A.lpw = d.lpw.p;
  A.ntiles = t.ntiles; A.T = t.T; A.nu_max = t.nu_max; A.mwa = d.mwa;
  A.dtr = dtr; A.first = first; A.last = last; A.ls_first = ls_first;
  A.hdr = t.hdr;
  A.ulist = t.u; A.tc = t.tc; A.rev = t.rev;
  A.ff = tp.ff.p; A.trec = tp.adj_trec.p;
  A.L = L; A.LIN = LIN; A.L0 = L0; A.LS = LS;
  A.err = status;
  // 32 tracers or fewer on 32-column tiles: 8 lanes a column, 32 tracers a
  // block (a 64-tracer block would leave half its lanes idle)
  const int G = (t.T == 32 && ntp <= 32) ? 32 : 64;
  const size_t smem = tile_adj_smem_bytes(t.T, t.nu_max, G);
  const unsigned nblk = (unsigned)t.ntiles * (unsigned)((ntp + G - 1) / G);
  if (G == 32) {
    OG_CUDA(cudaFuncSetAttribute(k_tile_adj<1, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile_adj<1, 32><<<nblk, TADJ_THREADS, smem, s>>>(A);
  } else if (t.T == 32) {
    OG_CUDA(cudaFuncSetAttribute(k_tile_adj<2, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile_adj<2, 64><<<nblk, TADJ_THREADS, smem, s>>>(A);
  } else {
    OG_CUDA(cudaFuncSetAttribute(k_tile_adj<1, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile_adj<1, 64><<<nblk, TADJ_THREADS, smem, s>>>(A);
  }
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

static int launch_adj_records(const DevGrid& d, Transport& tp, int* status, cudaStream_t s) {
  const size_t n = (size_t)d.mza * d.mwa * TADJ_RW;
  if (tp.adj_trec.n != n) {
    OG_CHECK(tp.adj_trec.alloc(n));
    OG_CUDA(cudaMemsetAsync(tp.adj_trec.p, 0, tp.adj_trec.bytes(), s));
  }
  const AdjTiles t = adj_tiles_of(d);
  AdjRecArgs R;
  R.mza = d.mza; R.T = t.T; R.kb = 1; R.mwa = d.mwa; R.lpw = d.lpw.p;
  R.hdr = t.hdr;
  R.ulist = t.u; R.tc = t.tc; R.rev = t.rev;
  R.wrec = tp.wrec.p; R.wmasc = tp.wmasc.p; R.a_w = d.a_w.p; R.trec = tp.adj_trec.p;
  R.err = status;
  k_adj_records<<<(unsigned)t.ntiles * t.T, 64, 0, s>>>(R);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

// device pointer table of n planes of `plane` floats starting at base
static int planes_table(DevBuf<float*>& tab, float* base, int n, size_t plane, cudaStream_t s) {
  std::vector<float*> h(n);
  for (int i = 0; i < n; ++i) h[i] = base + (size_t)i * plane;
  OG_CHECK(tab.alloc(n));
  OG_CUDA(cudaMemcpyAsync(tab.p, h.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
  OG_CUDA(cudaStreamSynchronize(s));   // h dies here
  return OLAMGPU_OK;
}

// the options and tables the adjoint needs
static int adjoint_checks(Context& C) {
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!C.have_state || !C.hstate.vmasc || !C.hstate.wmasc || !C.hstate.rho) {
    set_error("state arrays vmasc/wmasc/rho were not registered at init");
    return OLAMGPU_E_STATE;
  }
  const DevGrid& d = C.g;
  const int nrk = C.opts.nrk_scal;
  const int order = C.opts.scal_horiz_adv_order;
  if (nrk != 2 && nrk != 3) { set_error("scalar_timestep_level must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (order != 2 && order != 3) { set_error("scal_horiz_adv_order must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (C.opts.iscal_monot == 1) {
    set_error("the adjoint covers the unlimited and the positive-definite transport (iscal_monot = 0 or 2)");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (C.tp.have_turb) {
    set_error("the adjoint does not cover horizontal diffusion of the tracers");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (!tile_stage_available(d, C.tp, order)) {
    set_error("the adjoint needs the tiled transport tables");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (!d.tile_closed) {
    set_error("the adjoint needs every neighbour of a prognosed column to be prognosed (a global domain)");
    return OLAMGPU_E_UNSUPPORTED;
  }
  return OLAMGPU_OK;
}

int adjoint_core(Context& C, const float* rho_old_host, bool ls_acc) {
  Transport& tp = C.tp;
  cudaStream_t s = C.stream;
  // the adjoint's 32-column tiles, once per grid, when the stage kernel runs narrower ones
  if (C.g.tile_T != 32 && (C.g.adj_tiles.T == 0 || C.g.adj_tiles.order != C.g.tile_order))
    OG_CHECK(build_adj_tiles(&C.hgrid, C.g, C.g.tile_order, s));
  const DevGrid& d = C.g;
  {
    const int at = adj_tiles_of(d).T;
    if (at != 16 && at != 32) {
      set_error("the adjoint runs on 16- or 32-column tiles; none could be built for this grid");
      return OLAMGPU_E_UNSUPPORTED;
    }
  }
  const int mza = d.mza, mwa = d.mwa;
  const int nrk = C.opts.nrk_scal;
  const int ntp = C.tr.ntp;
  const size_t plane = (size_t)mza * mwa, qn = plane * ntp;
  OG_CHECK(tp.adj_l[0].alloc(qn));
  OG_CHECK(tp.adj_l[1].alloc(qn));
  if (tp.adj_l0.n < qn) OG_CHECK(tp.adj_l0.alloc(qn));
  OG_CHECK(tp.adj_ls.alloc(qn));
  float dtlr[3];
  OG_CHECK(transport_prepare(C, rho_old_host, false, dtlr));
  const float* rhos_nrk = tp.rhos.p + (size_t)(nrk - 1) * plane;
  std::vector<int> modes, pdm;
  bool anylim = false, any_pdm = false;
  OG_CHECK(tracer_modes(C, modes, pdm, anylim, any_pdm));
  const bool pd = C.opts.iscal_monot == 2 && anylim;
  {
    OG_PROF("adj_records", s);
    OG_CHECK(launch_tile_weights(d, tp, rhos_nrk, s));
    OG_CHECK(launch_adj_records(d, tp, C.status.p, s));
  }
  // the positive-definite last stage is taken at the forward state: the
  // step again from its input tracers (Q[qcur]) and tendencies (qt) to the
  // last stage's input, and scp0' = scp0 + dtr sct / rho_old
  const float* S_in = nullptr;
  float* S0p = nullptr;
  if (pd) {
    OG_PROF("adj_pd_recompute", s);
    Tracers& tr = C.tr;
    const float* F = tr.q[tr.qcur].p;
    float* B1 = tr.q[(tr.qcur + 1) % 3].p;
    float* B2 = tr.q[(tr.qcur + 2) % 3].p;
    const float* in = F;
    float* outs[2] = {B1, B2};
    for (int istage = 1; istage < nrk; ++istage) {
      float* out = outs[(istage - 1) & 1];
      OG_CHECK(launch_tile_stage(d, tp, in, F, tr.qt.p, out, ntp, istage, nrk, dtlr[istage - 1], C.status.p, s));
      launch_implicit_solve(d, tp, nrk, istage, dtlr[istage - 1], CTView{F, ntp, 0}, TView{out, ntp, 0}, ntp, s);
      in = out;
    }
    S_in = in;
    S0p = in == B1 ? B2 : B1;
    OG_CUDA(cudaMemcpyAsync(S0p, F, qn * sizeof(float), cudaMemcpyDeviceToDevice, s));
    launch_scp0_pd_update(d, tp, TView{S0p, ntp, 0}, CTView{tr.qt.p, ntp, 0}, tp.d_mode.p + tr.n, tr.n,
                          dtlr[nrk - 1], s);
  }
  // the reverse stages alternate between the two lam buffers; the last
  // one writes into adj_l[fin]
  const int fin = nrk & 1;
  float* L = tp.adj_l[0].p;
  float* LIN = tp.adj_l[1].p;
  const size_t colsize = (size_t)mza * ntp;
  if (d.n_nonprog > 0) {
    k_adj_nonprog<<<cdiv((size_t)d.n_nonprog * colsize, 256), 256, 0, s>>>(d.w_nonprog.p, d.n_nonprog, colsize, L,
                                                                          LIN, ls_acc ? nullptr : tp.adj_ls.p, fin);
    OG_LAUNCHED();
  }
  for (int istage = nrk; istage >= 1; --istage) {
    const float dtr = dtlr[istage - 1];
    const int first = istage == nrk, last = istage == 1;
    {
      OG_PROF("adj_implicit", s);
      k_adj_implicit<<<cdiv((size_t)d.nw_prog * ntp, 128), 128, 0, s>>>(
          gridk(d), tp.imp_list.p + (size_t)(istage - 1) * mwa, tp.imp_count.p + (istage - 1),
          tp.imp_b.p + (size_t)(istage - 1) * mwa * 3 * mza, tp.ff.p, tp.wmasc.p,
          tp.rhos.p + (size_t)(istage - 1) * plane, nrk, istage, dtr, ntp, first, L, tp.adj_l0.p);
      OG_LAUNCHED();
      if (d.nw_prog > 0)
        k_adj_fold0<<<cdiv((size_t)d.nw_prog * (ntp / 4), 256), 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p,
                                                                             mza, ntp, L);
      OG_LAUNCHED();
    }
    const bool pd_stage = pd && first;
    if (pd_stage) {
      // the limited tracers' transpose; the batched kernel below leaves them alone
      OG_CHECK(pd_adjoint_stage(C, S_in, S0p, L, LIN, tp.adj_l0.p, tp.adj_ls.p, dtr, 0, C.tr.n, s));
    }
    {
      OG_PROF("adj_stage", s);
      OG_CHECK(launch_tile_adj(d, tp, L, LIN, tp.adj_l0.p, tp.adj_ls.p, ntp, istage, nrk, dtr, first, last,
                               first && !ls_acc, C.status.p, s, pd_stage ? tp.d_mode.p + C.tr.n : nullptr, C.tr.n));
    }
    std::swap(L, LIN);
  }
  return OLAMGPU_OK;
}

int transport_adjoint_run(const float* rho_old_host, float* const* lam, float* const* lam_sct) {
  Context& C = ctx();
  OG_CHECK(adjoint_checks(C));
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
  const int ntp = C.tr.ntp;
  const size_t plane = (size_t)mza * mwa, qn = plane * ntp;
  // per-tracer planes on the device start on 16-byte boundaries (the layout
  // transposes move them in 16-byte pieces)
  const size_t pstride = (plane + 3) & ~(size_t)3;

  OG_CHECK(tp.adj_l[0].alloc(qn));
  OG_CHECK(tp.adj_l0.alloc(std::max(qn, pstride * n)));
  OG_CHECK(tp.adj_planes.alloc(pstride * n));
  if (C.opts.iscal_monot == 2) {
    // the limited stage's adjoint is taken at the forward state: the
    // registered tracers and tendencies are the step's inputs
    if (C.coherence == OLAMGPU_SYNC_EACH_CALL) OG_CHECK(tracers_to_device(s));
    OG_CHECK(ensure_q(s));
  }
  OG_CHECK(planes_table(tp.adj_ptab, tp.adj_planes.p, n, pstride, s));
  // lams leaves through lam0's memory, which is free after the last stage
  OG_CHECK(planes_table(tp.adj_ptab2, tp.adj_l0.p, n, pstride, s));
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(tp.adj_planes.p + (size_t)i * pstride, lam[i], plane * sizeof(float),
                            cudaMemcpyHostToDevice, s));
  {
    // device work of the step (in RESIDENT mode the preparation uploads nothing)
    OG_PROF("adjoint", s);
    { OG_PROF("adj_gather", s); launch_gather_q(tp.adj_l[0].p, (const float* const*)tp.adj_ptab.p, n, ntp, plane, s); }
    OG_CHECK(adjoint_core(C, rho_old_host));
    {
      OG_PROF("adj_scatter", s);
      launch_scatter_q(tp.adj_l[nrk & 1].p, tp.adj_ptab.p, n, ntp, plane, s);
      launch_scatter_q(tp.adj_ls.p, tp.adj_ptab2.p, n, ntp, plane, s);
    }
  }
  for (int i = 0; i < n; ++i) {
    OG_CUDA(cudaMemcpyAsync(lam[i], tp.adj_planes.p + (size_t)i * pstride, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaMemcpyAsync(lam_sct[i], tp.adj_l0.p + (size_t)i * pstride, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  }
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

int adjoint_ready(Context& C) { return adjoint_checks(C); }

}  // namespace olamgpu
