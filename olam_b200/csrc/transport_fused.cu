// transport_fused.cu -- one RK stage of update_scalar for every tracer in a
// single launch (batched layout Q[iw][kd][ntp], tracer index fastest).
//
// Restates, fused into one pass, omodel/scalar_transport_rk.F90:
//   grad_t2d / grad_t2d_quadratic (grad_lib.f90:236-341)   horizontal reconstruction
//   scalar_v_column (474-534)                              upwind V-face value
//   grad_z_quadratic (grad_lib.f90:166-229),
//   scalar_w_column (537-612)                              vertical reconstruction,
//                                                          flux divergence, update
// Work mapping.  A block owns one prognostic column and a chunk of KC levels;
// LPI lanes compute one (column, level) cell for every tracer, a lane
// holding 2 consecutive tracers (one float2) per pass.  Cells are independent, so
// there is no sequential chain over levels: latency is hidden by the many
// warps in flight.  The column's tables (neighbours, faces, directions, the
// folded reconstruction weights of both sides of each face and the
// neighbour lists of the upwind neighbours) are staged once per block in
// shared memory.
//
// The upwind side of a V face depends only on sign(vmasc(k,iv)), the same
// for every tracer, so a warp evaluates only the side it needs.  The value
// on side s of face iv is S(c) + sum_n ew[iv][s][n] * (S(nb_n(c)) - S(c)):
// the gradient (order 2) or quadratic (order 3) coefficients pre-multiplied
// by the face offsets at set-up, so the reference's gradient planes and
// face arrays never touch memory.
//
// HBM traffic per tracer and cell (ideal): read S, S0, SCT, write OUT = 16 B;
// neighbour and vertical rows are re-read from L1/L2.
#include "transport_kernels.cuh"

namespace olamgpu {

struct FusedArgs {
  int mza, nprog, nq, nrk, istage, nchunk;
  float dtr;
  const int* __restrict__ prog;
  const int* __restrict__ npoly;
  const int* __restrict__ w_nb;
  const int* __restrict__ w_ev;
  const float* __restrict__ w_dirv;
  const int* __restrict__ v_iw;
  const int* __restrict__ lpw;
  const int* __restrict__ lpv;
  const float* __restrict__ ew;     // (mva, 2, 8)
  const float* __restrict__ a_w;    // (mza, 2, 2)
  const float* __restrict__ volti;
  const float* __restrict__ vmasc;
  const float* __restrict__ wmasc;
  const float* __restrict__ rhos;   // rhos(:,:,nrk)
  const float* __restrict__ ff;     // (mwa, nrk)
  const int* __restrict__ colrec;   // (nprog, COLREC_WORDS)
  const float4* __restrict__ S;
  const float4* __restrict__ S0;
  const float4* __restrict__ SCT;
  float4* __restrict__ OUT;
};

__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a + w * b
__device__ __forceinline__ float2 axpy2(float2 a, float w, float2 b) {
  return make_float2(a.x + w * b.x, a.y + w * b.y);
}
__device__ __forceinline__ float2 ld2(const float2* p) { return __ldg(p); }

#define FUSED_NB 7
#define FUSED_KC 16
#define FUSED_THREADS 256
#ifndef FUSED_MINB
#define FUSED_MINB 2  // 2 blocks of 256 threads per SM: up to 128 registers
#endif


// grad_z_quadratic (bounded, zero-gradient BCs) at level lev from rows
// a = S(lev-1), b = S(lev), c = S(lev+1); returns the bottom (want_bot) or
// top face value of level lev.
__device__ __forceinline__ float2 zface(const float* __restrict__ a_w, int mza, int kb, int lev,
                                        bool want_bot, float2 a, float2 b, float2 c) {
  const bool top = (lev > mza - 2), bot = (lev < kb + 1);
  const float c1 = __ldg(a_w + lev + (want_bot ? 0 : 2 * mza));       // a_w(k,1,1|2)
  const float c2 = __ldg(a_w + lev + (want_bot ? mza : 3 * mza));     // a_w(k,2,1|2)
  float2 r;
  float dsk = top ? 0.f : (c.x - b.x), dskm1 = bot ? 0.f : (b.x - a.x);
  r.x = b.x + dsk * c1 + dskm1 * c2;
  dsk = top ? 0.f : (c.y - b.y); dskm1 = bot ? 0.f : (b.y - a.y);
  r.y = b.y + dsk * c1 + dskm1 * c2;
  return r;
}

// Per-block staging of a column record into the form the inner loop reads:
// 32-bit row bases of the cells it gathers, per-face weights as float4
// vectors (one broadcast LDS.128 per 4 weights) and a face-flag word.
struct FusedSmem {
  unsigned base[25];     // (point * mza) * nq2 for c, nb[0..5], new[6][3]
  float4 wown[6][2];     // own-side weights of face n over nb[0..5] (+2 pad)
  float4 wfar[6][2];     // far side: c, nb[n-1], nb[n+1], new0..2 (+1 pad)
  float dv[6];
  int own, nnew;         // bit n: this column is side 1 of face n; nnew(n) in 2 bits
  int rec[COLREC_WORDS]; // raw record (general path)
};

// LPI lanes cooperate on one (column, level) cell, each lane holding one
// float2 (2 tracers) per pass; a block covers KC levels of one column.
// Loads of a cell are issued in two rounds: everything whose address is
// known (own column, neighbours, scp0, tendency, winds), then the far-side
// rows of the inflow faces, whose choice depends on sign(vmasc).
template <int LPI>
__global__ void __launch_bounds__(FUSED_THREADS, FUSED_MINB) k_fused(FusedArgs A) {
  __shared__ FusedSmem T;
  const int j = blockIdx.x / A.nchunk;
  const int chunk = blockIdx.x - j * A.nchunk;
  const int mza = A.mza;
  const int nq2 = A.nq * 2;                  // float2 per (point, level) row
  int* R = T.rec;
  for (int i = threadIdx.x; i < COLREC_WORDS; i += FUSED_THREADS)
    R[i] = __ldg(A.colrec + (size_t)j * COLREC_WORDS + i);
  __syncthreads();
  const int iw = R[COLREC_IW], np = R[COLREC_NP], kb = R[COLREC_KB];
  const bool fast = R[COLREC_FAST] != 0;
  const unsigned colsz = (unsigned)mza * (unsigned)nq2;
  if (fast) {
    const int t = threadIdx.x;
    if (t < 25) {
      int p;
      if (t == 0) p = iw;
      else if (t < 7) p = R[COLREC_NB + t - 1];
      else {
        const int n = (t - 7) / 3, m = (t - 7) % 3;
        p = (m < R[COLREC_NNEW + n]) ? R[COLREC_NEW + n * 3 + m] : iw;
      }
      T.base[t] = (unsigned)p * colsz;
    } else if (t >= 32 && t < 32 + 48) {
      const int i = t - 32, n = i >> 3, m = i & 7;
      reinterpret_cast<float*>(&T.wown[n][0])[m] = (m < 6) ? __int_as_float(R[COLREC_WOWN + n * 7 + m]) : 0.f;
    } else if (t >= 96 && t < 96 + 48) {
      const int i = t - 96, n = i >> 3, m = i & 7;
      reinterpret_cast<float*>(&T.wfar[n][0])[m] = (m < 6) ? __int_as_float(R[COLREC_WU + n * 7 + m]) : 0.f;
    } else if (t >= 160 && t < 166) {
      T.dv[t - 160] = __int_as_float(R[COLREC_DV + t - 160]);
    } else if (t == 192) {
      int own = 0, nn = 0;
      for (int n = 0; n < 6; ++n) {
        own |= (R[COLREC_OWN + n] & 1) << n;
        nn |= (R[COLREC_NNEW + n] & 3) << (2 * n);
      }
      T.own = own;
      T.nnew = nn;
    }
    __syncthreads();
  }
  const float fexpl = 1.0f - __ldg(A.ff + (size_t)iw * A.nrk + A.istage - 1);
  const float* __restrict__ wm = A.wmasc + (size_t)iw * mza;
  const float2* __restrict__ S = reinterpret_cast<const float2*>(A.S);
  const float2* __restrict__ S0 = reinterpret_cast<const float2*>(A.S0);
  const float2* __restrict__ SCT = reinterpret_cast<const float2*>(A.SCT);
  float2* __restrict__ OUT = reinterpret_cast<float2*>(A.OUT);
  const size_t cbase = (size_t)iw * colsz;
  constexpr int IPP = FUSED_THREADS / LPI;   // cells per pass
  const int sub = threadIdx.x / LPI, lane = threadIdx.x % LPI;
  auto RF = [&](int i) { return __int_as_float(R[i]); };

  for (int kk = sub; kk < FUSED_KC; kk += IPP) {
    const int kd = chunk * FUSED_KC + kk;
    if (kd < kb || kd >= mza) continue;
    const float wkm1 = __ldg(wm + kd - 1), wk0 = __ldg(wm + kd);
    const float vt = __ldg(A.volti + (size_t)iw * mza + kd);
    const float rh = __ldg(A.rhos + (size_t)iw * mza + kd);
    const unsigned lvl = (unsigned)kd * (unsigned)nq2;
    if (fast) {
      // ---- flat hexagonal column
      float vm[6];
      unsigned inflow = 0;
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        vm[n] = __ldg(A.vmasc + (size_t)R[COLREC_EV + n] * mza + kd);
        const unsigned up1 = vm[n] < 0.f ? 1u : 0u;          // upwind side of face n
        inflow |= (up1 ^ ((T.own >> n) & 1u)) << n;
      }
      const int nnew = T.nnew;
      for (int q = lane; q < nq2; q += LPI) {
        const unsigned lq = lvl + (unsigned)q;
        const float2 s0 = ld2(S + cbase + lq);
        const float2 sm1 = (kd - 1 >= kb) ? ld2(S + cbase + lq - nq2) : s0;
        const float2 sp1 = (kd + 1 < mza) ? ld2(S + cbase + lq + nq2) : s0;
        const float2 sm2 = (kd - 2 >= kb) ? ld2(S + cbase + lq - 2 * nq2) : sm1;
        const float2 sp2 = (kd + 2 < mza) ? ld2(S + cbase + lq + 2 * nq2) : sp1;
        float2 sn[6];
#pragma unroll
        for (int n = 0; n < 6; ++n) sn[n] = ld2(S + (T.base[1 + n] + lq));
        const float2 s00 = ld2(S0 + cbase + lq);
        const float2 st = ld2(SCT + cbase + lq);
        float2 nw[6][3];
#pragma unroll
        for (int n = 0; n < 6; ++n)
#pragma unroll
          for (int m = 0; m < 3; ++m)
            if (((inflow >> n) & 1u) && m < ((nnew >> (2 * n)) & 3))
              nw[n][m] = ld2(S + (T.base[7 + n * 3 + m] + lq));
        float2 dn[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) dn[m] = sub2(sn[m], s0);
        float2 fd = make_float2(0.f, 0.f);
#pragma unroll
        for (int n = 0; n < 6; ++n) {
          float2 val;
          if (!((inflow >> n) & 1u)) {
            const float4 w0 = T.wown[n][0], w1 = T.wown[n][1];
            val = s0;
            val = axpy2(val, w0.x, dn[0]);
            val = axpy2(val, w0.y, dn[1]);
            val = axpy2(val, w0.z, dn[2]);
            val = axpy2(val, w0.w, dn[3]);
            val = axpy2(val, w1.x, dn[4]);
            val = axpy2(val, w1.y, dn[5]);
          } else {
            const float4 w0 = T.wfar[n][0], w1 = T.wfar[n][1];
            const float2 su = sn[n];
            const int nn = (nnew >> (2 * n)) & 3;
            val = su;
            val = axpy2(val, w0.x, sub2(s0, su));
            val = axpy2(val, w0.y, sub2(sn[(n + 5) % 6], su));
            val = axpy2(val, w0.z, sub2(sn[(n + 1) % 6], su));
            if (nn > 0) val = axpy2(val, w0.w, sub2(nw[n][0], su));
            if (nn > 1) val = axpy2(val, w1.x, sub2(nw[n][1], su));
            if (nn > 2) val = axpy2(val, w1.y, sub2(nw[n][2], su));
          }
          fd = axpy2(fd, T.dv[n] * vm[n], sub2(val, s00));
        }
        // ---- vertical upwind faces kd-1 and kd (grad_z_quadratic, bounded)
        float2 up_lo, up_hi;
        if (kd == kb) up_lo = s0;                                                   // scp_upw(kb-1) = scp(kb)
        else if (wkm1 < 0.f) up_lo = zface(A.a_w, mza, kb, kd, true, sm1, s0, sp1);        // scpb(kd)
        else up_lo = zface(A.a_w, mza, kb, kd - 1, false, sm2, sm1, s0);                   // scpt(kd-1)
        if (kd == mza - 1) up_hi = s0;                                              // scp_upw(mza) = scp(mza)
        else if (wk0 < 0.f) up_hi = zface(A.a_w, mza, kb, kd + 1, true, s0, sp1, sp2);     // scpb(kd+1)
        else up_hi = zface(A.a_w, mza, kb, kd, false, sm1, s0, sp1);                       // scpt(kd)
        float2 o;
        {
          float v = fexpl * (wkm1 * (up_lo.x - s00.x) - wk0 * (up_hi.x - s00.x));
          o.x = s00.x + A.dtr * (st.x + vt * (fd.x + v)) / rh;
          v = fexpl * (wkm1 * (up_lo.y - s00.y) - wk0 * (up_hi.y - s00.y));
          o.y = s00.y + A.dtr * (st.y + vt * (fd.y + v)) / rh;
        }
        OUT[cbase + lq] = o;
        if (kd == kb)
          for (int k2 = 0; k2 < kb; ++k2) OUT[cbase + (size_t)k2 * nq2 + q] = o;
      }
      continue;
    }
    // ---- general columns (the 12 pentagons, or terrain)
    float vm[FUSED_NB];
    bool inflow[FUSED_NB];
#pragma unroll
    for (int n = 0; n < FUSED_NB; ++n) {
      vm[n] = (n < np) ? __ldg(A.vmasc + (size_t)R[COLREC_EV + n] * mza + kd) : 0.f;
      inflow[n] = (n < np) && (kd >= R[COLREC_LPV + n]) && (((vm[n] < 0.f) ? 1 : 0) != R[COLREC_OWN + n]);
    }
    for (int q = lane; q < nq2; q += LPI) {
      const size_t lq = (size_t)lvl + q;
      const float2* Sc = S + cbase + lq;
      const float2 s0 = ld2(Sc);
      const float2 sm1 = (kd - 1 >= kb) ? ld2(Sc - nq2) : s0;
      const float2 sp1 = (kd + 1 < mza) ? ld2(Sc + nq2) : s0;
      const float2 sm2 = (kd - 2 >= kb) ? ld2(Sc - 2 * nq2) : sm1;
      const float2 sp2 = (kd + 2 < mza) ? ld2(Sc + 2 * nq2) : sp1;
      float2 sn[FUSED_NB];
#pragma unroll
      for (int n = 0; n < FUSED_NB; ++n)
        if (n < np) sn[n] = ld2(S + (size_t)R[COLREC_NB + n] * colsz + lq);
      const float2 s00 = ld2(S0 + cbase + lq);
      const float2 st = ld2(SCT + cbase + lq);
      float2 dn[FUSED_NB];
#pragma unroll
      for (int m = 0; m < FUSED_NB; ++m)
        if (m < np) dn[m] = sub2(sn[m], s0);
      float2 fd = make_float2(0.f, 0.f);
#pragma unroll
      for (int n = 0; n < FUSED_NB; ++n) {
        if (n >= np || kd < R[COLREC_LPV + n]) continue;
        float2 val;
        if (!inflow[n]) {
          val = s0;
#pragma unroll
          for (int m = 0; m < FUSED_NB; ++m)
            if (m < np) val = axpy2(val, RF(COLREC_WOWN + n * 7 + m), dn[m]);
        } else {
          const int u = R[COLREC_NB + n];
          const int iv = R[COLREC_EV + n];
          const float* w = A.ew + ((size_t)iv * 2 + (1 - R[COLREC_OWN + n])) * 8;
          const float2 su = sn[n];
          val = su;
          const int npu = __ldg(A.npoly + u);
          for (int m = 0; m < npu; ++m) {
            const int um = __ldg(A.w_nb + u * 8 + m);
            const float2 sx = (um == iw) ? s0 : ld2(S + (size_t)um * colsz + lq);
            val = axpy2(val, __ldg(w + m), sub2(sx, su));
          }
        }
        fd = axpy2(fd, RF(COLREC_DV + n) * vm[n], sub2(val, s00));
      }
      float2 up_lo, up_hi;
      if (kd == kb) up_lo = s0;
      else if (wkm1 < 0.f) up_lo = zface(A.a_w, mza, kb, kd, true, sm1, s0, sp1);
      else up_lo = zface(A.a_w, mza, kb, kd - 1, false, sm2, sm1, s0);
      if (kd == mza - 1) up_hi = s0;
      else if (wk0 < 0.f) up_hi = zface(A.a_w, mza, kb, kd + 1, true, s0, sp1, sp2);
      else up_hi = zface(A.a_w, mza, kb, kd, false, sm1, s0, sp1);
      float2 o;
      {
        float v = fexpl * (wkm1 * (up_lo.x - s00.x) - wk0 * (up_hi.x - s00.x));
        o.x = s00.x + A.dtr * (st.x + vt * (fd.x + v)) / rh;
        v = fexpl * (wkm1 * (up_lo.y - s00.y) - wk0 * (up_hi.y - s00.y));
        o.y = s00.y + A.dtr * (st.y + vt * (fd.y + v)) / rh;
      }
      OUT[cbase + lq] = o;
      if (kd == kb)
        for (int k2 = 0; k2 < kb; ++k2) OUT[cbase + (size_t)k2 * nq2 + q] = o;
    }
  }
}

void launch_fused_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                        const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr,
                        const float* rhos, cudaStream_t s) {
  FusedArgs A;
  A.mza = d.mza; A.nprog = d.nw_prog; A.nq = ntp / 4; A.nrk = nrk; A.istage = istage; A.dtr = dtr;
  A.nchunk = (d.mza + FUSED_KC - 1) / FUSED_KC;
  A.prog = d.jtw_prog.p; A.npoly = d.npoly.p; A.w_nb = d.w_nb.p; A.w_ev = d.w_ev.p;
  A.w_dirv = d.w_dirv.p; A.v_iw = d.v_iw.p; A.lpw = d.lpw.p; A.lpv = d.lpv.p;
  A.ew = d.ew_b.p; A.a_w = d.a_w.p; A.volti = d.volti.p;
  A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p; A.rhos = rhos; A.ff = tp.ff.p;
  A.colrec = d.colrec.p;
  A.S = reinterpret_cast<const float4*>(S);
  A.S0 = reinterpret_cast<const float4*>(S0);
  A.SCT = reinterpret_cast<const float4*>(SCT);
  A.OUT = reinterpret_cast<float4*>(OUT);
  const unsigned nblk = (unsigned)((size_t)d.nw_prog * A.nchunk);
  const int nq2 = ntp / 2;
  // lanes per cell: the power of two covering the tracer pairs, 4..256
  int lpi = 4;
  while (lpi < nq2 && lpi < FUSED_THREADS) lpi *= 2;
  switch (lpi) {
    case 4: k_fused<4><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    case 8: k_fused<8><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    case 16: k_fused<16><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    case 32: k_fused<32><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    case 64: k_fused<64><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    case 128: k_fused<128><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
    default: k_fused<256><<<nblk, FUSED_THREADS, 0, s>>>(A); break;
  }
  OG_LAUNCHED();
}

}  // namespace olamgpu
