// transport_tile.cu -- the fused RK stage of update_scalar in tiles.
//
// Restates, fused into one pass over the batched layout Q[iw][kd][ntp],
// omodel/scalar_transport_rk.F90:
//   grad_t2d / grad_t2d_quadratic (grad_lib.f90:236-341)  gradient planes
//   scalar_v_column (474-534)                             upwind V-face value
//   grad_z_quadratic (grad_lib.f90:166-229),
//   scalar_w_column (537-612)                             vertical faces, flux
//                                                         divergence, update
//
// The horizontal flux divergence of update_scalar,
//   sum_f dirv * vmasc * (upwind face value - S0),
// is linear in the tracer with weights that depend only on (column, level):
// with the reconstruction (gradient coefficients times face offsets) folded
// at set-up into a per-column table A[face][upwind side][slot], it is
//   fd = SW * (S - S0) + sum_j W_j * (S(slot j) - S)
//      = D * S - SW * S0 + sum_j W_j * S(slot j),   D = SW - sum_j W_j,
// over the column's <= TILE_NS neighbours and second neighbours, with
// W_j = sum_f dirv * vmasc * A[f][upwind][j].  The winds are fixed for the
// long step, so k_weights forms these per-(column, level) records once per
// step (both stages and the adjoint read them).  With terrain a column's
// faces, and the gradient terms across faces, below their lpv drop out (the
// reference's loops start at lpv): k_weights leaves out the faces and takes
// the slot weights of the level's terrain band; k_tile sweeps a tile from
// its lowest floor and stores each column from its own lpw up.
//
// k_tile: a block owns a tile of T = 16 NC consecutive prognostic columns
// and a group of 64 tracers and sweeps the levels bottom to top.  While it
// computes level kd from one shared-memory buffer it copies level kd+1 into
// the other (TMA four-row gathers, cp.async.bulk.tensor tile::gather4, on
// one mbarrier per buffer): the tracer rows of the tile's two-ring
// neighbourhood U and the tile columns' weight records.  A half warp owns NC
// columns, four tracers per lane (packed FFMA2); the column's own values at
// kd-2 .. kd+3 and its scp0 / sct rows stay in registers across levels (one
// row per level is read ahead from global memory), so the vertical quadratic
// faces -- linear in those rows with the records' coefficients -- need no
// staging.
#include <cudaTypedefs.h>

#include <algorithm>
#include <map>

#include "transport_kernels.cuh"
#include "tile_common.cuh"

namespace olamgpu {

struct WeightArgs {
  int mza, T, kb, ntiles;
  const int* __restrict__ lpw;      // lowest prognosed device level of each W column
  const int* __restrict__ lpv;      // and of each V face
  const float* __restrict__ band;   // terrain bands' slot weights (TILE_AW each)
  const int* __restrict__ band_lev; // the level at which each band ends
  const int4* __restrict__ hdr;
  const int* __restrict__ tc;
  const float* __restrict__ amat;
  const float* __restrict__ vmasc;
  const float* __restrict__ wmasc;
  const float* __restrict__ volti;
  const float* __restrict__ rhos;   // rhos(:,:,nrk)
  const float* __restrict__ a_w;    // Fortran (mza, 2, 2)
  float* __restrict__ wrec;         // (mwa, mza, TILE_WR)
};

struct TileArgs {
  int mza, ntp, nrk, istage, kb, ntiles, T, nu_max, mwa;
  int ks;                           // level chunks per tile (blocks per tile and group)
  const int* __restrict__ lpw;      // lowest prognosed device level of each W column
  int grp0, ngrp;                   // the tracer groups of 64 this launch runs
  float dtr;
  const int4* __restrict__ hdr;
  const int* __restrict__ ulist;
  const int* __restrict__ tc;
  const float* __restrict__ ff;     // (mwa, nrk)
  const float* __restrict__ wrec;   // (mwa, mza, TILE_WR)
  const float* __restrict__ S;
  const float* __restrict__ S0;
  const float* __restrict__ SCT;
  float* __restrict__ OUT;
  int* err;                         // device status record
};

#define TILE_THREADS 256
#define TILE_NW (TILE_THREADS / 32)
// polls of a level barrier before a block gives up (seconds at the slowest)
#define TILE_WAIT_POLLS (1u << 26)

// ---- per-(column, level) weight records, once per long step -------------------
// Record (TILE_WR floats):
//   [0, TILE_NS)  W_j, the slot weights
//   20 SW, 21 volti / rhos, 22 1 / rhos, 23 D = SW - sum W
//   24 .. 28      beta_q: the vertical flux wmasc(kd-1) upw(kd-1) - wmasc(kd) upw(kd)
//                 as sum_q beta_q S(kd-2+q), the upwind face values upw being
//                 grad_z_quadratic of the upwind level (bounded) or, at the
//                 bottom and top faces, S(kd) itself
//   29            omega = wmasc(kd) - wmasc(kd-1), the vertical flux's S0 term
//   30, 31        wmasc(kd-1), wmasc(kd)
// so that a stage is
//   scp = S0 + dtr / rhos sct + dtr volti / rhos (sum_j W_j S(slot j) + D S
//         - SW S0 + fexpl (sum_q beta_q S(kd-2+q) + omega S0)).
// Four tile columns per block of 256 threads, a thread per level.
__global__ void __launch_bounds__(256) k_weights(WeightArgs A) {
  __shared__ int wall[4][TILE_TCW];
  __shared__ __align__(16) float amall[4][TILE_AW];
  const int sub = threadIdx.x >> 6, lt = threadIdx.x & 63;
  const size_t r = (size_t)blockIdx.x * 4 + sub;   // tile-column record
  const int t = (int)(r / A.T), i = (int)(r - (size_t)t * A.T);
  const bool live = t < A.ntiles && i < A.hdr[t].w;   // not padding of the last tile
  int* w = wall[sub];
  float* am = amall[sub];
  if (live) {
    for (int q = lt; q < TILE_TCW; q += 64) w[q] = __ldg(A.tc + r * TILE_TCW + q);
    for (int q = lt; q < TILE_AW; q += 64) am[q] = __ldg(A.amat + r * TILE_AW + q);
  }
  __syncthreads();
  if (!live) return;
  const int iw = w[TILE_TC_IW], np = w[TILE_TC_NP], side = w[TILE_TC_SIDE];
  const int mza = A.mza, kb = max(A.kb, __ldg(A.lpw + iw));   // the column's own floor
  const int nband = w[TILE_TC_NB], boff = w[TILE_TC_BOFF];
  for (int kd = kb + lt; kd < mza; kd += 64) {
    float dvvm[6];
    int up[6];
    float sw = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int iv = w[TILE_TC_EV + f];
      const float vm = (f < np && kd >= __ldg(A.lpv + iv)) ? __ldg(A.vmasc + (size_t)iv * mza + kd) : 0.f;
      dvvm[f] = __int_as_float(w[TILE_TC_DV + f]) * vm;
      // 1: the neighbour across face f is upwind
      up[f] = ((vm < 0.f ? 1 : 0) != ((side >> f) & 1)) ? 1 : 0;
      sw = fmaf(__int_as_float(w[TILE_TC_DV + f]), vm, sw);
    }
    const size_t x = (size_t)iw * mza + kd;
    float* o = A.wrec + x * TILE_WR;
    float sumw = 0.f;
    // four slots at a time (16-byte reads of the face rows of A)
    auto slot_weights = [&](const float4* am4) {
#pragma unroll
      for (int q = 0; q < TILE_NS / 4; ++q) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          const float4 a = am4[(f * 2 + up[f]) * (TILE_NS / 4) + q];
          acc.x = fmaf(dvvm[f], a.x, acc.x);
          acc.y = fmaf(dvvm[f], a.y, acc.y);
          acc.z = fmaf(dvvm[f], a.z, acc.z);
          acc.w = fmaf(dvvm[f], a.w, acc.w);
        }
        sumw += acc.x;
        sumw += acc.y;
        sumw += acc.z;
        sumw += acc.w;
        reinterpret_cast<float4*>(o)[q] = acc;
      }
    };
    // the terrain band of level kd (bands end at increasing levels; past
    // the last one every term is above ground)
    int b = 0;
    while (b < nband && kd >= __ldg(A.band_lev + boff + b)) ++b;
    if (b < nband) slot_weights(reinterpret_cast<const float4*>(A.band + (size_t)(boff + b) * TILE_AW));
    else slot_weights(reinterpret_cast<const float4*>(am));
    // vertical faces: grad_z_quadratic at level lev from (lev-1, lev, lev+1),
    // S(lev) + c1' (S(lev+1) - S(lev)) + c2' (S(lev) - S(lev-1)), the primes
    // zeroing the differences across the column's ends
    float beta[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    auto face = [&](float wf, int lev, bool bot, int q0) {   // q0: beta index of S(lev-1)
      const float c1 = lev <= mza - 2 ? __ldg(A.a_w + lev + (bot ? 0 : 2) * mza) : 0.f;
      const float c2 = lev >= kb + 1 ? __ldg(A.a_w + lev + (bot ? 1 : 3) * mza) : 0.f;
      beta[q0] -= wf * c2;
      beta[q0 + 1] += wf * (1.f - c1 + c2);
      beta[q0 + 2] += wf * c1;
    };
    const float wkm1 = __ldg(A.wmasc + x - 1), wk0 = __ldg(A.wmasc + x);
    if (kd == kb) beta[2] += wkm1;                   // scp_upw(kb-1) = scp(kb)
    else if (wkm1 < 0.f) face(wkm1, kd, true, 1);    // scpb(kd) from (kd-1, kd, kd+1)
    else face(wkm1, kd - 1, false, 0);               // scpt(kd-1) from (kd-2, kd-1, kd)
    if (kd == mza - 1) beta[2] -= wk0;               // scp_upw(mza) = scp(mza)
    else if (wk0 < 0.f) face(-wk0, kd + 1, true, 2); // scpb(kd+1) from (kd, kd+1, kd+2)
    else face(-wk0, kd, false, 1);                   // scpt(kd) from (kd-1, kd, kd+1)
    const float rh = __ldg(A.rhos + x);
    reinterpret_cast<float4*>(o)[5] = make_float4(sw, __ldg(A.volti + x) / rh, 1.0f / rh, sw - sumw);
    reinterpret_cast<float4*>(o)[6] = make_float4(beta[0], beta[1], beta[2], beta[3]);
    reinterpret_cast<float4*>(o)[7] = make_float4(beta[4], wk0 - wkm1, wkm1, wk0);
  }
}

int launch_pair_records(const DevGrid& d, Transport& tp, cudaStream_t s);

int launch_tile_weights(const DevGrid& d, Transport& tp, const float* rhos, cudaStream_t s) {
  const size_t n = (size_t)d.mza * d.mwa * TILE_WR;
  if (tp.wrec.n != n) {
    OG_CHECK(tp.wrec.alloc(n));
    // records of columns outside the tiles (the dummy point) stay zero
    OG_CUDA(cudaMemsetAsync(tp.wrec.p, 0, tp.wrec.bytes(), s));
  }
  WeightArgs W;
  W.mza = d.mza; W.T = d.tile_T; W.kb = 1; W.ntiles = d.ntiles;
  W.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  W.tc = d.tile_tc.p; W.amat = d.tile_a.p;
  W.vmasc = tp.vmasc.p; W.wmasc = tp.wmasc.p; W.volti = d.volti.p; W.rhos = rhos; W.a_w = d.a_w.p;
  W.wrec = tp.wrec.p;
  W.lpw = d.lpw.p; W.lpv = d.lpv.p;
  W.band = d.tile_band.p; W.band_lev = d.tile_band_lev.p;
  k_weights<<<cdiv((size_t)d.ntiles * d.tile_T, 4), 256, 0, s>>>(W);
  OG_LAUNCHED();
  // the paired kernel reads the pairs' records, formed from these
  if (d.tile_pairk && d.tile_paired && d.tile_T == 16) OG_CHECK(launch_pair_records(d, tp, s));
  return OLAMGPU_OK;
}

// ---- the stage kernel -------------------------------------------------------------
// Shared memory (in this order; tile_smem_bytes in setup.cu sizes it the
// same way): two level buffers of U rows (4 G bytes each), two of the tile
// columns' records, the U rows' global row offsets, the slot byte offsets,
// the tile columns, their explicit fractions.
// Shape: LPC lanes per column, four tracers per lane, so a block's tracer
// group is G = 4 LPC tracers (32, 64 or 128) and a warp serves 32 / LPC
// columns at a time; NC columns per lane group, T = 8 warps x (32 / LPC) x
// NC columns per tile.  A launch may split the level sweep of a tile into
// KS chunks run by different blocks (A.ks).
// OFF: the type of element offsets into the batched arrays -- unsigned when
// they all fit in 32 bits (fewer address instructions), else long long.
template <int NC, int LPC, typename OFF, bool SPLIT, int NW = TILE_NW>
__global__ void __launch_bounds__(NW * 32, NW > TILE_NW ? 1 : (NC == 1 ? 3 : 2))
    k_tile(TileArgs A, const __grid_constant__ CUtensorMap tmS, const __grid_constant__ CUtensorMap tmR) {
  extern __shared__ __align__(16) unsigned char smraw[];
  // every four-row gather's shared-memory destination on a 128-byte boundary
  static_assert((4 * TILE_WR * 4) % 128 == 0 && (4 * 4 * 4 * LPC) % 128 == 0, "gather destinations");
  constexpr int NT = NW * 32;                // threads of the block
  constexpr int CPW = 32 / LPC;              // columns a warp serves at once
  constexpr int TW = NW * CPW;               // columns a block serves at once
  constexpr int T = TW * NC;
  constexpr int G = 4 * LPC;                 // tracers of the block's group
  constexpr int RB = 4 * G;                  // bytes of a staged row
  // block order: tile, then level chunk, then tracer group (the groups of a
  // tile run side by side, so its records are read once from HBM)
  const int ngrp = A.ngrp, nks = SPLIT ? A.ks : 1;
  const int tile = blockIdx.x / (ngrp * nks);
  const int rem = blockIdx.x - tile * ngrp * nks;
  const int ks = SPLIT ? rem / ngrp : 0, grp = A.grp0 + (rem - ks * ngrp);
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nT = h.w;
  const int mza = A.mza, ntp = A.ntp, kb = A.kb;   // kb: the lowest floor of any column
  // this block's levels [klo, khi) (the whole column without a split)
  const int chunk = SPLIT ? (mza - kb + nks - 1) / nks : mza - kb;
  const int klo = SPLIT ? kb + ks * chunk : kb, khi = SPLIT ? min(mza, klo + chunk) : mza;
  const int nu4 = (nU + 3) & ~3;      // rows gathered four at a time
  auto al = [](size_t b) { return (b + 127) & ~size_t(127); };
  const size_t ubuf = al((size_t)((A.nu_max + 3) & ~3) * RB), rbuf = al((size_t)T * TILE_WR * 4);
  // 128-byte aligned start (pointer arithmetic on the shared array keeps the
  // accesses shared-memory instructions)
  unsigned char* p = smraw + ((128u - (smem_addr(smraw) & 127u)) & 127u);
  unsigned long long* BAR = reinterpret_cast<unsigned long long*>(p); p += 128;   // a barrier per level buffer
  char* UB = reinterpret_cast<char*>(p);              p += 2 * ubuf;
  unsigned char* RBB = p;                             p += 2 * rbuf;
  int* RIDX = reinterpret_cast<int*>(p);              p += al((size_t)(A.nu_max + 3) * 4);
  int* SLOT = reinterpret_cast<int*>(p);              p += al((size_t)T * TILE_NS * 4);
  int* IWT = reinterpret_cast<int*>(p);               p += al((size_t)T * 4);
  float* FEX = reinterpret_cast<float*>(p);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t0 = grp * G;
  if (SPLIT && klo >= khi) return;   // an empty chunk (more chunks than levels): uniform per block

  // tables of this tile, checked once: every index must address the arrays
  // it is used on (a failure is recorded and the block does nothing)
  int bad = (nU > A.nu_max || nT > T || nT > nU || A.T != T) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nT * TILE_NS; i += NT) {
      const int c = i / TILE_NS, j = i - c * TILE_NS;
      const int v = __ldg(A.tc + ((size_t)tile * T + c) * TILE_TCW + TILE_TC_SLOT + j);
      if ((unsigned)v >= (unsigned)nU * 256u || (v & 255)) bad = 6;
      SLOT[i] = (v >> 8) * RB;
    }
    for (int i = tid; i < nT; i += NT) {
      const int v = __ldg(A.tc + ((size_t)tile * T + i) * TILE_TCW + TILE_TC_IW);
      if (v < 1 || v >= A.mwa) bad = 4;
      IWT[i] = v;
    }
    for (int i = tid; i < nu4; i += NT) {
      const int v = __ldg(A.ulist + u_off + (i < nU ? i : 0));   // padding rows repeat row 0
      if (v < 1 || v >= A.mwa) bad = 8;
      RIDX[i] = v * mza;
    }
  }
  if (tid == 0) {
    mbar_init(&BAR[0], NW);
    mbar_init(&BAR[1], NW);
    mbar_init_fence();
  }
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }
  for (int i = tid; i < nT; i += NT) FEX[i] = 1.0f - __ldg(A.ff + (size_t)IWT[i] * A.nrk + A.istage - 1);

  const int seg = min(G, ntp - t0);  // tracers of this group (a multiple of 4)
  // level k into buffer b, completing on barrier b: warp w's lane 0 gathers
  // the U-row quadruples w, w + 8, ... (TMA, RB bytes per row) and the
  // records of tile-column quadruples w, w + 8, ...
  auto stage = [&](int k, int b) {
    if (lane != 0) return;
    const int ng = nu4 >> 2, nr = (nT + 3) >> 2;
    const int myg = warp < ng ? (ng - warp + NW - 1) / NW : 0;
    const int myr = warp < nr ? (nr - warp + NW - 1) / NW : 0;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&BAR[b], (unsigned)(myg * 4 * RB + myr * 4 * TILE_WR * 4));
    char* Ub = UB + b * ubuf;
    for (int g = warp; g < ng; g += NW) {
      const int* r = RIDX + 4 * g;
      tma_gather4(Ub + 4 * g * RB, &tmS, t0, r[0] + k, r[1] + k, r[2] + k, r[3] + k, &BAR[b]);
    }
    for (int q = warp; q < nr; q += NW) {
      const int c0 = 4 * q;
      const int y0 = IWT[c0] * mza, y1 = IWT[min(c0 + 1, nT - 1)] * mza;
      const int y2 = IWT[min(c0 + 2, nT - 1)] * mza, y3 = IWT[min(c0 + 3, nT - 1)] * mza;
      tma_gather4(RBB + b * rbuf + c0 * TILE_WR * 4, &tmR, 0, y0 + k, y1 + k, y2 + k, y3 + k, &BAR[b]);
    }
  };

  // LPC lanes per column (columns cb, cb + TW, ...): lane hl of the group
  // holds tracers t0 + 4 hl .. + 3; the column's rows kd-2, kd-1, kd+1,
  // kd+2, kd+3 (read ahead) and its scp0 / sct rows at kd stay in registers
  const int sub = lane / LPC, hl = lane - sub * LPC;
  const bool act = 4 * hl < seg;
  const int cb = CPW * warp + sub;
  F4 m2[NC], m1[NC], p1[NC], p2[NC], p3[NC], s00[NC], st[NC];
  OFF cbase[NC];
  int kbc[NC];   // each column's own floor (lpw): levels below it are not prognosed
  stage(klo, 0);
#pragma unroll
  for (int n = 0; n < NC; ++n) {
    const int c = cb + TW * n;
    m2[n] = m1[n] = p1[n] = p2[n] = p3[n] = s00[n] = st[n] = zero4();
    cbase[n] = 0;
    kbc[n] = c < nT ? max(kb, __ldg(A.lpw + IWT[c])) : mza;
    if (c < nT && act) {
      cbase[n] = (OFF)IWT[c] * (OFF)mza * (OFF)ntp + (OFF)(t0 + 4 * hl);
      // a chunk above the column's floor starts with the rows below it
      if (SPLIT && klo - 2 >= kbc[n]) m2[n] = ldg4(A.S + (cbase[n] + (OFF)(klo - 2) * (OFF)ntp));
      if (SPLIT && klo - 1 >= kbc[n]) m1[n] = ldg4(A.S + (cbase[n] + (OFF)(klo - 1) * (OFF)ntp));
      if (klo + 1 < mza) p1[n] = ldg4(A.S + (cbase[n] + (OFF)(klo + 1) * (OFF)ntp));
      if (klo + 2 < mza) p2[n] = ldg4(A.S + (cbase[n] + (OFF)(klo + 2) * (OFF)ntp));
      if (klo + 3 < mza) p3[n] = ldg4(A.S + (cbase[n] + (OFF)(klo + 3) * (OFF)ntp));
      s00[n] = ldg4(A.S0 + (cbase[n] + (OFF)klo * (OFF)ntp));
      st[n] = ldg4(A.SCT + (cbase[n] + (OFF)klo * (OFF)ntp));
    }
  }
  __syncthreads();   // the explicit fractions
  // a level's copies are waited for at most TILE_WAIT_POLLS polls; a block
  // whose copies never complete records it and stops at the level's end
  int failed = 0;
  for (int kd = klo; kd < khi; ++kd) {
    const int lv = kd - klo, cur = lv & 1;
    if (!mbar_wait_bounded(&BAR[cur], (lv >> 1) & 1, TILE_WAIT_POLLS)) failed = 1;
    if (kd + 1 < khi) stage(kd + 1, cur ^ 1);
    const char* Ul = UB + cur * ubuf + hl * 16;
    const float* Rc = reinterpret_cast<const float*>(RBB + cur * rbuf);
#pragma unroll
    for (int n = 0; n < NC; ++n) {
      const int c = cb + TW * n;
      if (c >= nT) continue;
      // the column's window holds no level below its floor
      if (kd == kbc[n]) m2[n] = m1[n] = zero4();
      const float* rc = Rc + c * TILE_WR;
      const float4 r5 = reinterpret_cast<const float4*>(rc)[5];   // SW, volti/rhos, 1/rhos, D
      const float4 r6 = reinterpret_cast<const float4*>(rc)[6];   // beta0 .. beta3
      const float2 r7 = reinterpret_cast<const float2*>(rc)[14];  // beta4, omega
      const float fx = FEX[c];
      const F4 s0 = lds4(Ul, c * RB);
      // horizontal: sum_j W_j S(slot j) + D S - SW S0
      F4 fd = zero4();
      const int* sl = SLOT + c * TILE_NS;
#pragma unroll
      for (int q = 0; q < TILE_NS / 4; ++q) {
        const int4 so = reinterpret_cast<const int4*>(sl)[q];
        const float4 w4 = reinterpret_cast<const float4*>(rc)[q];
        // a slot whose weight is zero at this level (a face whose upwind
        // side does not reach it) is not read
        if (w4.x != 0.f) fd = fma4s(w4.x, lds4(Ul, so.x), fd);
        if (w4.y != 0.f) fd = fma4s(w4.y, lds4(Ul, so.y), fd);
        if (w4.z != 0.f) fd = fma4s(w4.z, lds4(Ul, so.z), fd);
        if (w4.w != 0.f) fd = fma4s(w4.w, lds4(Ul, so.w), fd);
      }
      // vertical quadratic upwind faces, fexpl times sum_q beta_q S(kd-2+q) + omega S0
      fd = fma4s(fx * r6.x, m2[n], fd);
      fd = fma4s(fx * r6.y, m1[n], fd);
      fd = fma4s(fmaf(fx, r6.z, r5.w), s0, fd);
      fd = fma4s(fx * r6.w, p1[n], fd);
      fd = fma4s(fx * r7.x, p2[n], fd);
      fd = fma4s(fmaf(fx, r7.y, -r5.x), s00[n], fd);
      // scp = scp0 + dtr * (sct + volti * (fluxdiv + fexpl * vflux)) / rhos
      const F4 o = fma4s(A.dtr * r5.y, fd, fma4s(A.dtr * r5.z, st[n], s00[n]));
      if (act) {
        if (kd >= kbc[n]) stg4(A.OUT + (cbase[n] + (OFF)kd * (OFF)ntp), o);
        // levels below the floor take the floor's value (scalar_w_column)
        if (kd == kbc[n])
          for (int k2 = 0; k2 < kd; ++k2) stg4(A.OUT + (cbase[n] + (OFF)k2 * (OFF)ntp), o);
        // slide the column's window up one level and read ahead
        m2[n] = m1[n]; m1[n] = s0; p1[n] = p2[n]; p2[n] = p3[n];
        if (kd + 4 < mza) p3[n] = ldg4(A.S + (cbase[n] + (OFF)(kd + 4) * (OFF)ntp));
        if (kd + 1 < mza) {
          s00[n] = ldg4(A.S0 + (cbase[n] + (OFF)(kd + 1) * (OFF)ntp));
          st[n] = ldg4(A.SCT + (cbase[n] + (OFF)(kd + 1) * (OFF)ntp));
        }
        // the rows these loads take two levels on, into L2 now (one level
        // of lead leaves the loads waiting on HBM)
        if (kd + 6 < mza) prefetch_l2(A.S + (cbase[n] + (OFF)(kd + 6) * (OFF)ntp));
        if (kd + 3 < mza) {
          prefetch_l2(A.S0 + (cbase[n] + (OFF)(kd + 3) * (OFF)ntp));
          prefetch_l2(A.SCT + (cbase[n] + (OFF)(kd + 3) * (OFF)ntp));
        }
      }
    }
    if (__syncthreads_or(failed)) {
      // the copies of this level and of the next one may still be in flight
      // into this block's shared memory: wait for them (bounded again) before
      // the block exits and its shared memory is handed to another block
      const bool cur_done = mbar_wait_bounded(&BAR[cur], (lv >> 1) & 1, TILE_WAIT_POLLS);
      const bool nxt_done = kd + 1 >= khi || mbar_wait_bounded(&BAR[cur ^ 1], ((lv + 1) >> 1) & 1, TILE_WAIT_POLLS);
      const int code = (cur_done && nxt_done) ? 130 : 131;
      if (tid == 0 && atomicCAS(A.err, 0, code) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = kd; }
      return;
    }
  }
}

// ---- the paired stage kernel ------------------------------------------------------
// 16-column tiles as 8 column pairs (2p, 2p+1), a warp per pair, 128
// tracers per block: each U row either column of a pair needs is read once
// and applied to both, with the pair's weights of the level gathered into
// one record per step (k_pair_records) -- the union rows with a non-zero
// weight for either column, their U indices and the two weights.
struct PairArgs {
  int mza, ntiles;
  const int4* __restrict__ hdr;
  const int* __restrict__ tc;
  const int* __restrict__ pair;     // (ntiles * 8, TILE_PT)
  const float* __restrict__ wrec;   // (mwa, mza, TILE_WR)
  float* __restrict__ prec;         // (ntiles * 8, mza, TILE_PR)
};

// a warp per (tile, pair), looping over the levels: the pair's table decoded
// once into registers (two union rows per lane); per level the two columns'
// records in two registers per lane (word = lane), the union rows' weights
// picked by shuffles, the non-zero ones compacted in order by a ballot, the
// record assembled in shared memory and stored whole (coalesced)
__global__ void __launch_bounds__(256) k_pair_records(PairArgs A) {
  __shared__ __align__(16) float rec[8][TILE_PR];
  const size_t tp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int mza = A.mza;
  if (tp >= (size_t)A.ntiles * 8) return;   // uniform per warp
  const int t = (int)(tp >> 3), pp = (int)(tp & 7);
  const int nT = A.hdr[t].w;
  float* r = rec[wl];
  const int ia = 2 * pp, ib = 2 * pp + 1;
  const bool hasa = ia < nT, hasb = ib < nT;
  const int iwa = hasa ? A.tc[((size_t)t * 16 + ia) * TILE_TCW + TILE_TC_IW] : 0;
  const int iwb = hasb ? A.tc[((size_t)t * 16 + ib) * TILE_TCW + TILE_TC_IW] : 0;
  const int* pt = A.pair + tp * TILE_PT;
  const int ne = hasa ? pt[0] : 0, jab = pt[1], jba = pt[2];
  // this lane's union rows e = lane and lane + 32: the row and its slots in A and B
  int code[2], ja[2], jb[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = lane + 32 * h;
    code[h] = (e < ne && e < TILE_PU) ? pt[4 + e] : 0;
    ja[h] = (e < ne) ? ((code[h] >> 8) & 255) - 1 : -1;
    jb[h] = (e < ne) ? ((code[h] >> 16) & 255) - 1 : -1;
  }
  const int src = lane < 10 ? 20 + lane : 0;
  const float* ra = A.wrec + (size_t)iwa * mza * TILE_WR + lane;
  const float* rb = A.wrec + (size_t)iwb * mza * TILE_WR + lane;
  float va = hasa ? ra[0] : 0.f, vb = hasb ? rb[0] : 0.f;
  for (int kd = 0; kd < mza; ++kd) {
    // the next level's words, loaded while this one is assembled
    const float na = (hasa && kd + 1 < mza) ? ra[(size_t)(kd + 1) * TILE_WR] : 0.f;
    const float nb = (hasb && kd + 1 < mza) ? rb[(size_t)(kd + 1) * TILE_WR] : 0.f;
    for (int i = lane; i < TILE_PR; i += 32) r[i] = 0.f;
    __syncwarp();
    unsigned char* rbt = reinterpret_cast<unsigned char*>(r + TILE_PR_IDX);
    float2* rw = reinterpret_cast<float2*>(r + TILE_PR_W);
    int cnt = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float xa = __shfl_sync(0xffffffffu, va, ja[h] < 0 ? 0 : ja[h]);
      const float xb = __shfl_sync(0xffffffffu, vb, jb[h] < 0 ? 0 : jb[h]);
      const float wa = ja[h] >= 0 ? xa : 0.f, wb = jb[h] >= 0 ? xb : 0.f;
      const bool nz = (wa != 0.f) || (wb != 0.f);
      const unsigned m = __ballot_sync(0xffffffffu, nz);
      const int pos = cnt + __popc(m & ((1u << lane) - 1u));
      if (nz) {
        rbt[pos] = (unsigned char)(code[h] & 255);
        rw[pos] = make_float2(wa, wb);
      }
      cnt += __popc(m);
    }
    // per column: SW, volti/rhos, 1/rhos, D, beta_0..4, omega (record words
    // 20..29), the other column's own-row weight, 0
    const float sa = __shfl_sync(0xffffffffu, va, lane == 10 ? (jab < 0 ? 0 : jab) : src);
    const float sb = __shfl_sync(0xffffffffu, vb, lane == 10 ? (jba < 0 ? 0 : jba) : src);
    if (lane < 11) {
      r[TILE_PR_A + lane] = lane < 10 ? sa : (jab >= 0 ? sa : 0.f);
      r[TILE_PR_B + lane] = lane < 10 ? sb : (jba >= 0 ? sb : 0.f);
    }
    if (lane == 0) r[0] = __int_as_float(cnt);
    __syncwarp();
    float4* o4 = reinterpret_cast<float4*>(A.prec + (tp * mza + kd) * TILE_PR);
    const float4* r4 = reinterpret_cast<const float4*>(r);
    if (lane < TILE_PR / 4) o4[lane] = r4[lane];
    __syncwarp();
    va = na;
    vb = nb;
  }
}

int launch_pair_records(const DevGrid& d, Transport& tp, cudaStream_t s) {
  if (!d.tile_paired || d.tile_T != 16) { set_error("pair records: no paired tiles"); return OLAMGPU_E_STATE; }
  const size_t n = (size_t)d.ntiles * 8 * d.mza * TILE_PR;
  if (tp.prec.n != n) OG_CHECK(tp.prec.alloc(n));
  PairArgs A;
  A.mza = d.mza; A.ntiles = d.ntiles;
  A.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  A.tc = d.tile_tc.p; A.pair = d.tile_pair.p; A.wrec = tp.wrec.p; A.prec = tp.prec.p;
  const size_t warps = (size_t)d.ntiles * 8;
  k_pair_records<<<(unsigned)cdiv(warps * 32, 256), 256, 0, s>>>(A);
  OG_LAUNCHED();
  tp.prec_gen = d.tile_gen;
  return OLAMGPU_OK;
}

// the stage over paired tiles: a warp per pair, 32 lanes over 128 tracers
static_assert((4 * TILE_PR * 4) % 128 == 0, "pair-record gather destinations on 128-byte boundaries");
template <typename OFF>
__global__ void __launch_bounds__(TILE_THREADS, 2)
    k_tile_pair(TileArgs A, const int* __restrict__ pair, const __grid_constant__ CUtensorMap tmS,
                const __grid_constant__ CUtensorMap tmP) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int T = 16, G = 128, RB = 4 * G;
  const int ngrp = A.ngrp;
  const int tile = blockIdx.x / ngrp;
  const int grp = A.grp0 + (blockIdx.x - tile * ngrp);
  const int4 h = A.hdr[tile];
  const int u_off = h.x, nU = h.y, nT = h.w;
  const int mza = A.mza, ntp = A.ntp, kb = A.kb;
  const int nu4 = (nU + 3) & ~3;
  auto al = [](size_t b) { return (b + 127) & ~size_t(127); };
  const size_t ubuf = al((size_t)((A.nu_max + 3) & ~3) * RB), rbuf = al((size_t)8 * TILE_PR * 4);
  unsigned char* p = smraw + ((128u - (smem_addr(smraw) & 127u)) & 127u);
  unsigned long long* BAR = reinterpret_cast<unsigned long long*>(p); p += 128;
  char* UB = reinterpret_cast<char*>(p);              p += 2 * ubuf;
  unsigned char* RBB = p;                             p += 2 * rbuf;
  int* RIDX = reinterpret_cast<int*>(p);              p += al((size_t)(A.nu_max + 3) * 4);
  int* IWT = reinterpret_cast<int*>(p);               p += al((size_t)T * 4);
  float* FEX = reinterpret_cast<float*>(p);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t0 = grp * G;

  int bad = (nU > A.nu_max || nT > T || nT > nU || A.T != T || nU > 256) ? 1 : 0;
  if (!bad) {
    for (int i = tid; i < nT; i += TILE_THREADS) {
      const int v = __ldg(A.tc + ((size_t)tile * T + i) * TILE_TCW + TILE_TC_IW);
      if (v < 1 || v >= A.mwa) bad = 4;
      IWT[i] = v;
    }
    for (int i = tid; i < nu4; i += TILE_THREADS) {
      const int v = __ldg(A.ulist + u_off + (i < nU ? i : 0));   // padding rows repeat row 0
      if (v < 1 || v >= A.mwa) bad = 8;
      RIDX[i] = v * mza;
    }
    // the pairs' union rows (the per-level records copy their indices)
    for (int i = tid; i < 8 * TILE_PU; i += TILE_THREADS) {
      const int* pt = pair + ((size_t)tile * 8 + i / TILE_PU) * TILE_PT;
      const int e = i % TILE_PU;
      if (e < pt[0] && (pt[4 + e] & 255) >= nU) bad = 10;
      if (e == 0 && pt[0] > TILE_PU) bad = 11;
    }
  }
  if (tid == 0) {
    mbar_init(&BAR[0], TILE_NW);
    mbar_init(&BAR[1], TILE_NW);
    mbar_init_fence();
  }
  if (__syncthreads_or(bad)) {
    if (bad && atomicCAS(A.err, 0, 100 + bad) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = tid; }
    return;
  }
  for (int i = tid; i < nT; i += TILE_THREADS) FEX[i] = 1.0f - __ldg(A.ff + (size_t)IWT[i] * A.nrk + A.istage - 1);

  const int seg = min(G, ntp - t0);
  // level k into buffer b: warp w's lane 0 gathers the U-row quadruples w,
  // w + 8, ...; warps 0 and 1 the records of pairs 0..3 and 4..7
  auto stage = [&](int k, int b) {
    if (lane != 0) return;
    const int ng = nu4 >> 2;
    const int myg = warp < ng ? (ng - warp + TILE_NW - 1) / TILE_NW : 0;
    const int myr = warp < 2 ? 1 : 0;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&BAR[b], (unsigned)(myg * 4 * RB + myr * 4 * TILE_PR * 4));
    char* Ub = UB + b * ubuf;
    for (int g = warp; g < ng; g += TILE_NW) {
      const int* r = RIDX + 4 * g;
      tma_gather4(Ub + 4 * g * RB, &tmS, t0, r[0] + k, r[1] + k, r[2] + k, r[3] + k, &BAR[b]);
    }
    if (myr) {
      const int y = (tile * 8 + 4 * warp) * mza + k;
      tma_gather4(RBB + b * rbuf + 4 * warp * TILE_PR * 4, &tmP, 0, y, y + mza, y + 2 * mza, y + 3 * mza, &BAR[b]);
    }
  };

  // the pair of this warp: columns 2 warp (A) and 2 warp + 1 (B); lane l
  // holds tracers t0 + 4 l .. + 3 of both
  const bool act = 4 * lane < seg;
  F4 m2[2], m1[2], p1[2], p2[2], p3[2], s00[2], st[2];
  OFF cbase[2];
  int kbc[2];
  stage(kb, 0);
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    const int c = 2 * warp + n;
    m2[n] = m1[n] = p1[n] = p2[n] = p3[n] = s00[n] = st[n] = zero4();
    cbase[n] = 0;
    kbc[n] = c < nT ? max(kb, __ldg(A.lpw + IWT[c])) : mza;
    if (c < nT && act) {
      cbase[n] = (OFF)IWT[c] * (OFF)mza * (OFF)ntp + (OFF)(t0 + 4 * lane);
      if (kb + 1 < mza) p1[n] = ldg4(A.S + (cbase[n] + (OFF)(kb + 1) * (OFF)ntp));
      if (kb + 2 < mza) p2[n] = ldg4(A.S + (cbase[n] + (OFF)(kb + 2) * (OFF)ntp));
      if (kb + 3 < mza) p3[n] = ldg4(A.S + (cbase[n] + (OFF)(kb + 3) * (OFF)ntp));
      s00[n] = ldg4(A.S0 + (cbase[n] + (OFF)kb * (OFF)ntp));
      st[n] = ldg4(A.SCT + (cbase[n] + (OFF)kb * (OFF)ntp));
    }
  }
  __syncthreads();   // the explicit fractions
  const bool hasa = 2 * warp < nT, hasb = 2 * warp + 1 < nT;
  const float fxa = hasa ? FEX[2 * warp] : 0.f, fxb = hasb ? FEX[2 * warp + 1] : 0.f;
  int failed = 0;
  for (int kd = kb; kd < mza; ++kd) {
    const int lv = kd - kb, cur = lv & 1;
    if (!mbar_wait_bounded(&BAR[cur], (lv >> 1) & 1, TILE_WAIT_POLLS)) failed = 1;
    if (kd + 1 < mza) stage(kd + 1, cur ^ 1);
    const char* Ul = UB + cur * ubuf + lane * 16;
    const float* rp = reinterpret_cast<const float*>(RBB + cur * rbuf) + warp * TILE_PR;
    if (hasa) {
      // the union rows: four per step, one word of byte indices and two
      // (wA, wB) pairs of weights per half
      const int cnt = min(__float_as_int(rp[0]), TILE_PU);
      const unsigned* ix4 = reinterpret_cast<const unsigned*>(rp + TILE_PR_IDX);
      const float4* w4 = reinterpret_cast<const float4*>(rp + TILE_PR_W);
      F4 fa = zero4(), fb = zero4();
      // eight rows per step (the entries past the count are row 0 with zero
      // weights), their loads issued together
      for (int e = 0; e < cnt; e += 8) {
        const uint2 ix2 = *reinterpret_cast<const uint2*>(ix4 + (e >> 2));
        const float4 w0 = w4[e >> 1], w1 = w4[(e >> 1) + 1], w2 = w4[(e >> 1) + 2], w3 = w4[(e >> 1) + 3];
        const F4 r0 = lds4(Ul, (int)(ix2.x & 255u) * RB);
        const F4 r1 = lds4(Ul, (int)((ix2.x >> 8) & 255u) * RB);
        const F4 r2 = lds4(Ul, (int)((ix2.x >> 16) & 255u) * RB);
        const F4 r3 = lds4(Ul, (int)(ix2.x >> 24) * RB);
        const F4 r4 = lds4(Ul, (int)(ix2.y & 255u) * RB);
        const F4 r5 = lds4(Ul, (int)((ix2.y >> 8) & 255u) * RB);
        const F4 r6 = lds4(Ul, (int)((ix2.y >> 16) & 255u) * RB);
        const F4 r7 = lds4(Ul, (int)(ix2.y >> 24) * RB);
        fa = fma4s(w0.x, r0, fa); fb = fma4s(w0.y, r0, fb);
        fa = fma4s(w0.z, r1, fa); fb = fma4s(w0.w, r1, fb);
        fa = fma4s(w1.x, r2, fa); fb = fma4s(w1.y, r2, fb);
        fa = fma4s(w1.z, r3, fa); fb = fma4s(w1.w, r3, fb);
        fa = fma4s(w2.x, r4, fa); fb = fma4s(w2.y, r4, fb);
        fa = fma4s(w2.z, r5, fa); fb = fma4s(w2.w, r5, fb);
        fa = fma4s(w3.x, r6, fa); fb = fma4s(w3.y, r6, fb);
        fa = fma4s(w3.z, r7, fa); fb = fma4s(w3.w, r7, fb);
      }
      // the two columns' own rows at kd
      const F4 sa = lds4(Ul, (2 * warp) * RB);
      const F4 sb = hasb ? lds4(Ul, (2 * warp + 1) * RB) : zero4();
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        if (n == 1 && !hasb) continue;
        if (kd == kbc[n]) m2[n] = m1[n] = zero4();
        const float* sc = rp + (n == 0 ? TILE_PR_A : TILE_PR_B);
        const float4 q0 = reinterpret_cast<const float4*>(sc)[0];   // SW, volti/rhos, 1/rhos, D
        const float4 q1 = reinterpret_cast<const float4*>(sc)[1];   // beta0 .. beta3
        const float4 q2 = reinterpret_cast<const float4*>(sc)[2];   // beta4, omega, other's own row, 0
        const float fx = n == 0 ? fxa : fxb;
        const F4 own = n == 0 ? sa : sb, other = n == 0 ? sb : sa;
        F4 fd = n == 0 ? fa : fb;
        fd = fma4s(q2.z, other, fd);
        fd = fma4s(fx * q1.x, m2[n], fd);
        fd = fma4s(fx * q1.y, m1[n], fd);
        fd = fma4s(fmaf(fx, q1.z, q0.w), own, fd);
        fd = fma4s(fx * q1.w, p1[n], fd);
        fd = fma4s(fx * q2.x, p2[n], fd);
        fd = fma4s(fmaf(fx, q2.y, -q0.x), s00[n], fd);
        const F4 o = fma4s(A.dtr * q0.y, fd, fma4s(A.dtr * q0.z, st[n], s00[n]));
        if (act) {
          if (kd >= kbc[n]) stg4(A.OUT + (cbase[n] + (OFF)kd * (OFF)ntp), o);
          if (kd == kbc[n])
            for (int k2 = 0; k2 < kd; ++k2) stg4(A.OUT + (cbase[n] + (OFF)k2 * (OFF)ntp), o);
          m2[n] = m1[n]; m1[n] = own; p1[n] = p2[n]; p2[n] = p3[n];
          if (kd + 4 < mza) p3[n] = ldg4(A.S + (cbase[n] + (OFF)(kd + 4) * (OFF)ntp));
          if (kd + 1 < mza) {
            s00[n] = ldg4(A.S0 + (cbase[n] + (OFF)(kd + 1) * (OFF)ntp));
            st[n] = ldg4(A.SCT + (cbase[n] + (OFF)(kd + 1) * (OFF)ntp));
          }
          if (kd + 6 < mza) prefetch_l2(A.S + (cbase[n] + (OFF)(kd + 6) * (OFF)ntp));
          if (kd + 3 < mza) {
            prefetch_l2(A.S0 + (cbase[n] + (OFF)(kd + 3) * (OFF)ntp));
            prefetch_l2(A.SCT + (cbase[n] + (OFF)(kd + 3) * (OFF)ntp));
          }
        }
      }
    }
    if (__syncthreads_or(failed)) {
      const bool cur_done = mbar_wait_bounded(&BAR[cur], (lv >> 1) & 1, TILE_WAIT_POLLS);
      const bool nxt_done = kd + 1 >= mza || mbar_wait_bounded(&BAR[cur ^ 1], ((lv + 1) >> 1) & 1, TILE_WAIT_POLLS);
      const int code = (cur_done && nxt_done) ? 130 : 131;
      if (tid == 0 && atomicCAS(A.err, 0, code) == 0) { A.err[1] = tile; A.err[2] = blockIdx.x; A.err[3] = kd; }
      return;
    }
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// a 2-D map over nrows rows of width floats with boxes of one row of box
// floats, for four-row gathers
static int row_map(CUtensorMap* m, const float* base, int width, size_t nrows, int box) {
  auto enc = tmap_encoder();
  if (!enc) { set_error("cuTensorMapEncodeTiled is not available"); return OLAMGPU_E_CUDA; }
  const cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)nrows};
  const cuuint64_t strides[1] = {(cuuint64_t)width * sizeof(float)};
  const cuuint32_t boxd[2] = {(cuuint32_t)box, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, boxd, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"); return OLAMGPU_E_CUDA; }
  return OLAMGPU_OK;
}

bool tile_stage_available(const DevGrid& d, const Transport& tp, int order) {
  (void)tp;
  return (d.tile_T == 8 || d.tile_T == 16 || d.tile_T == 32) && d.tile_order == order;
}

// the stage kernel of a tile shape (T columns, G tracers per block)
using TileKern = void (*)(TileArgs, const CUtensorMap, const CUtensorMap);
template <bool SPLIT>
static TileKern tile_kernel_s(int T, int G, bool off32) {
  // 32-column tiles of 128 tracers: a block of 16 warps, one per SM
  if (T == 32 && G == 128) return off32 ? k_tile<2, 32, unsigned, SPLIT, 16> : k_tile<2, 32, long long, SPLIT, 16>;
  if (T == 32 && G == 64) return off32 ? k_tile<2, 16, unsigned, SPLIT> : k_tile<2, 16, long long, SPLIT>;
  if (T == 32 && G == 32) return off32 ? k_tile<1, 8, unsigned, SPLIT> : k_tile<1, 8, long long, SPLIT>;
  if (T == 16 && G == 64) return off32 ? k_tile<1, 16, unsigned, SPLIT> : k_tile<1, 16, long long, SPLIT>;
  if (T == 16 && G == 128) return off32 ? k_tile<2, 32, unsigned, SPLIT> : k_tile<2, 32, long long, SPLIT>;
  // 8-column tiles of 128 tracers: a warp per column, three blocks per SM
  if (T == 8 && G == 128) return off32 ? k_tile<1, 32, unsigned, SPLIT> : k_tile<1, 32, long long, SPLIT>;
  return nullptr;
}
// threads of a shape's block
static unsigned tile_threads(int T, int G) { return (T == 32 && G == 128) ? 512u : (unsigned)TILE_THREADS; }
// the kernel of a shape; the level sweep is split (KS > 1) only in its own instance
static TileKern tile_kernel(int T, int G, bool off32, int KS = 1) {
  return KS > 1 ? tile_kernel_s<true>(T, G, off32) : tile_kernel_s<false>(T, G, off32);
}

// the largest dynamic shared memory a block may use
#define TILE_SMEM_LIMIT (227 * 1024)

// the paired kernel's layout: two level barriers, two level buffers of U
// rows of 128 tracers and of the 8 pairs' records, the U rows' global row
// indices, the tile columns, their explicit fractions
static size_t tile_pair_smem_bytes(int nu) {
  auto al = [](size_t b) { return (b + 127) & ~size_t(127); };
  const size_t nu4 = (size_t)((nu + 3) & ~3);
  return 127 + 128 + 2 * al(nu4 * 512) + 2 * al((size_t)8 * TILE_PR * 4) + al((size_t)(nu + 3) * 4) + al(16 * 4) +
         16 * 4;
}

bool tile_shape_fits(const DevGrid& d, int G) {
  return tile_kernel(d.tile_T, G, true) && tile_smem_bytes(d.tile_T, d.tile_nu_max, 4 * G) <= TILE_SMEM_LIMIT;
}

int launch_tile_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                      const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr, int* status,
                      cudaStream_t s, int grp0, int ngrp_run, int G_force) {
  if (tp.wrec.n != (size_t)d.mza * d.mwa * TILE_WR) {
    set_error("tile stage: the weight records of the step were not formed");
    return OLAMGPU_E_STATE;
  }
  const int G = G_force > 0 ? G_force : d.tile_G;
  const int KS = std::max(1, d.tile_KS);
  TileArgs A;
  A.mza = d.mza; A.ntp = ntp; A.nrk = nrk; A.istage = istage; A.kb = 1; A.ks = KS;
  A.ntiles = d.ntiles; A.T = d.tile_T; A.nu_max = d.tile_nu_max; A.mwa = d.mwa;
  A.dtr = dtr; A.lpw = d.lpw.p;
  A.hdr = reinterpret_cast<const int4*>(d.tile_hdr.p);
  A.ulist = d.tile_u.p; A.tc = d.tile_tc.p;
  A.ff = tp.ff.p; A.wrec = tp.wrec.p;
  A.S = S; A.S0 = S0; A.SCT = SCT; A.OUT = OUT;
  A.err = status;
  const size_t smem = tile_smem_bytes(d.tile_T, d.tile_nu_max, 4 * G);
  const int ngrp_all = (ntp + G - 1) / G;
  if (ngrp_run <= 0) { grp0 = 0; ngrp_run = ngrp_all; }
  if (grp0 < 0 || grp0 + ngrp_run > ngrp_all) { set_error("tile stage: tracer groups out of range"); return OLAMGPU_E_ARG; }
  A.grp0 = grp0; A.ngrp = ngrp_run;
  const unsigned nblk = (unsigned)d.ntiles * (unsigned)ngrp_run * (unsigned)KS;
  // element offsets in 32 bits when every array of the batched layout fits
  const bool off32 = (double)d.mwa * d.mza * ntp < 4294967296.0;
  if (d.tile_pairk && d.tile_T == 16 && G == 128 && KS == 1) {
    if (!d.tile_paired || !tp.prec.p || tp.prec_gen != d.tile_gen) {
      set_error("tile stage: the pair records of the step were not formed");
      return OLAMGPU_E_STATE;
    }
    const size_t psmem = tile_pair_smem_bytes(d.tile_nu_max);
    if (psmem > TILE_SMEM_LIMIT || d.tile_nu_max > 256) {
      set_error("tile stage: the paired tiles do not fit in shared memory");
      return OLAMGPU_E_UNSUPPORTED;
    }
    alignas(64) CUtensorMap tmS, tmP;
    OG_CHECK(row_map(&tmS, S, ntp, (size_t)d.mwa * d.mza, G));
    OG_CHECK(row_map(&tmP, tp.prec.p, TILE_PR, (size_t)d.ntiles * 8 * d.mza, TILE_PR));
    auto pk = off32 ? k_tile_pair<unsigned> : k_tile_pair<long long>;
    OG_CUDA(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem));
    A.ks = 1;
    pk<<<(unsigned)d.ntiles * (unsigned)ngrp_run, TILE_THREADS, psmem, s>>>(A, d.tile_pair.p, tmS, tmP);
    OG_LAUNCHED();
    return OLAMGPU_OK;
  }
  const TileKern kern = tile_kernel(d.tile_T, G, off32, KS);
  if (!kern || smem > TILE_SMEM_LIMIT) {
    set_error("tile stage: no kernel for " + std::to_string(d.tile_T) + "-column tiles of " + std::to_string(G) +
              " tracers within the shared memory");
    return OLAMGPU_E_UNSUPPORTED;
  }
  alignas(64) CUtensorMap tmS, tmR;
  OG_CHECK(row_map(&tmS, S, ntp, (size_t)d.mwa * d.mza, G));
  OG_CHECK(row_map(&tmR, tp.wrec.p, TILE_WR, (size_t)d.mwa * d.mza, TILE_WR));
  OG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<nblk, tile_threads(d.tile_T, G), smem, s>>>(A, tmS, tmR);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

// ---- tile-shape autotuner --------------------------------------------------------
// The stage kernel's shape -- columns per tile (T), tracers per block (G:
// LPC lanes per column) and level chunks per tile (KS, the levels a block's
// threads sweep) -- is chosen on the actual grid, tracer count and
// reconstruction order: each candidate the shared memory admits runs the
// stage on the step's own inputs a few times, and the fastest is kept.  The
// choice is cached per (grid, tracer count, order) for the process.
struct ShapeKey {
  unsigned long long h;
  bool operator<(const ShapeKey& o) const { return h < o.h; }
};
static std::map<ShapeKey, TileShape> g_shape_cache;

static unsigned long long shape_key(const olamgpu_grid* g, int ntp, int order) {
  unsigned long long h = 1469598103934665603ull;   // FNV-1a over the values that shape the tiles
  auto mix = [&](unsigned long long v) { h = (h ^ v) * 1099511628211ull; };
  mix((unsigned)g->mza); mix((unsigned)g->mwa); mix((unsigned)g->nw_prog); mix((unsigned)ntp); mix((unsigned)order);
  for (int j = 0; j < g->nw_prog; ++j) mix((unsigned)g->jtw_prog[j]);
  for (int i = 0; i < g->mwa; ++i) mix((unsigned)g->lpw[i]);
  return h;
}

int tile_autotune(Context& C, const float* S, const float* S0, const float* SCT, float* OUT, float dtr) {
  DevGrid& d = C.g;
  Transport& tp = C.tp;
  cudaStream_t s = C.stream;
  const int ntp = C.tr.ntp, nrk = C.opts.nrk_scal, order = C.opts.scal_horiz_adv_order;
  tp.tune_log.clear();
  const ShapeKey key{shape_key(&C.hgrid, ntp, order)};
  // ord: bit 0 the caller's order, bit 1 the paired kernel
  auto use = [&](const TileShape& sh) -> int {
    if (d.tile_T != sh.T || d.tile_ord != (sh.ord & 1)) OG_CHECK(build_tiles(&C.hgrid, d, order, s, sh.T, sh.ord & 1));
    d.tile_G = sh.G;
    d.tile_KS = sh.KS;
    d.tile_pairk = (sh.ord & 2) != 0 && d.tile_paired;
    if (d.tile_pairk) OG_CHECK(launch_pair_records(d, tp, s));
    return OLAMGPU_OK;
  };
  auto it = g_shape_cache.find(key);
  if (it != g_shape_cache.end()) {
    OG_CHECK(use(it->second));
    tp.tuned_ntp = ntp;
    return OLAMGPU_OK;
  }
  cudaEvent_t e0, e1;
  OG_CUDA(cudaEventCreate(&e0));
  OG_CUDA(cudaEventCreate(&e1));
  TileShape best{0, 0, 0, 0};
  float best_ms = 0.f;
  prof_suspend(true);
  int rc = OLAMGPU_OK;
  // split level sweeps only help where the tiles do not fill the GPU
  const int ks_max = (size_t)d.ntiles * (size_t)((ntp + 63) / 64) < 4 * 148 ? 2 : 1;
  const int Ts[3] = {32, 16, 8};
  d.tile_pairk = false;
  for (int ord = 0; ord <= 1 && rc == OLAMGPU_OK; ++ord)
  for (int T : Ts) {
    if (d.tile_T != T || d.tile_ord != ord) {
      rc = build_tiles(&C.hgrid, d, order, s, T, ord);
      if (rc != OLAMGPU_OK || d.tile_T != T) { rc = OLAMGPU_OK; continue; }   // no tables of this width
    }
    const int Gs[3] = {T == 8 ? 0 : 64, T == 32 ? 32 : 128, T == 32 ? 128 : 0};
    for (int G : Gs) {
      if (!G) continue;
      if (!tile_shape_fits(d, G)) continue;
      for (int KS = 1; KS <= ks_max; ++KS) {
        d.tile_G = G;
        d.tile_KS = KS;
        float ms = 1e30f;
        for (int r = 0; r < 4 && rc == OLAMGPU_OK; ++r) {
          cudaEventRecord(e0, s);
          rc = launch_tile_stage(d, tp, S, S0, SCT, OUT, ntp, nrk, nrk, dtr, C.status.p, s, 0, 0, 0);
          cudaEventRecord(e1, s);
          if (rc != OLAMGPU_OK) break;
          cudaEventSynchronize(e1);
          float t = 0.f;
          cudaEventElapsedTime(&t, e0, e1);
          if (r > 0) ms = std::min(ms, t);   // the first run warms up
        }
        if (rc != OLAMGPU_OK) break;
        tp.tune_log.push_back({T, G, KS, ord, 0, ms});
        if (!best.T || ms < best_ms) { best = TileShape{T, G, KS, ord}; best_ms = ms; }
        // the paired kernel on the same tiles, where its per-step pair
        // records fit in the free device memory
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t prec_b = (size_t)d.ntiles * 8 * d.mza * TILE_PR * sizeof(float);
        if (T == 16 && G == 128 && KS == 1 && d.tile_paired && d.tile_nu_max <= 256 &&
            tile_pair_smem_bytes(d.tile_nu_max) <= TILE_SMEM_LIMIT &&
            (tp.prec.n * sizeof(float) >= prec_b || free_b > prec_b + ((size_t)2 << 30))) {
          d.tile_pairk = true;
          // its per-step pair records count against it, shared by the nrk stages
          float rec_ms = 1e30f;
          for (int r = 0; r < 2 && rc == OLAMGPU_OK; ++r) {
            cudaEventRecord(e0, s);
            rc = launch_pair_records(d, tp, s);
            cudaEventRecord(e1, s);
            if (rc != OLAMGPU_OK) break;
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r > 0) rec_ms = t;
          }
          float pm = 1e30f;
          for (int r = 0; r < 4 && rc == OLAMGPU_OK; ++r) {
            cudaEventRecord(e0, s);
            rc = launch_tile_stage(d, tp, S, S0, SCT, OUT, ntp, nrk, nrk, dtr, C.status.p, s, 0, 0, 0);
            cudaEventRecord(e1, s);
            if (rc != OLAMGPU_OK) break;
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (r > 0) pm = std::min(pm, t);
          }
          d.tile_pairk = false;
          if (rc != OLAMGPU_OK) break;
          pm += rec_ms / (float)nrk;
          tp.tune_log.push_back({T, G, KS, ord | 2, 0, pm});
          if (pm < best_ms) { best = TileShape{T, G, KS, ord | 2}; best_ms = pm; }
        }
      }
      if (rc != OLAMGPU_OK) break;
    }
    if (rc != OLAMGPU_OK) break;
  }
  prof_suspend(false);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  OG_CHECK(rc);
  if (!best.T) { set_error("tile autotune: no shape runs on this grid"); return OLAMGPU_E_UNSUPPORTED; }
  for (auto& r : tp.tune_log)
    if (r.T == best.T && r.G == best.G && r.KS == best.KS && r.ord == best.ord) r.chosen = 1;
  if (!(best.ord & 2)) tp.prec.release();   // the pair records of the tuning runs
  OG_CHECK(use(best));
  g_shape_cache[key] = best;
  tp.tuned_ntp = ntp;
  return check_device_status();
}

}  // namespace olamgpu
