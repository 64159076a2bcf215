// transport_fused.cu -- one RK stage of update_scalar for every tracer in a
// single launch (batched layout Q[iw][kd][ntp], tracer index fastest).
//
// Restates, fused into one pass, omodel/scalar_transport_rk.F90:
//   grad_t2d / grad_t2d_quadratic (grad_lib.f90:236-341)   horizontal reconstruction
//   scalar_v_column (474-534)                              upwind V-face value
//   scalar_w_column (537-612)                              vertical reconstruction,
//                                                          flux divergence, update
// Work mapping: one warp per prognostic column, lane = 4 consecutive tracers
// (one float4), loop over levels bottom to top.  The upwind side of a V face
// depends only on sign(vmasc(k,iv)), which is the same for every tracer, so
// a warp evaluates only the side it needs.  The reconstruction on side s of
// face iv is S(c) + sum_n ew[iv][s][n] * (S(nb_n(c)) - S(c)), the gradient
// (or quadratic) coefficients pre-multiplied by the face offsets at set-up;
// the intermediate gradient planes and face values of the reference never
// touch memory.  The column's own values k-1..k+2 stay in registers as a
// sliding window for the vertical quadratic reconstruction.  Winds, density,
// volumes and tables are loaded once per (column, level) and applied to all
// tracers held by the warp.
//
// HBM traffic per tracer and cell (ideal): read S, S0, SCT, write OUT = 16 B;
// neighbour rows are re-read from L1/L2.
#include "transport_kernels.cuh"

namespace olamgpu {

struct FusedArgs {
  int mza, nprog, nq, nrk, istage;
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
  const float4* __restrict__ S;
  const float4* __restrict__ S0;
  const float4* __restrict__ SCT;
  float4* __restrict__ OUT;
};

__device__ __forceinline__ float4 f4(float a) { return make_float4(a, a, a, a); }
__device__ __forceinline__ float4 operator-(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ float4 operator+(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 operator*(float a, float4 b) {
  return make_float4(a * b.x, a * b.y, a * b.z, a * b.w);
}
// a + w * b, evaluated as the Fortran writes it (the compiler may fuse)
__device__ __forceinline__ float4 axpy(float4 a, float w, float4 b) {
  return make_float4(a.x + w * b.x, a.y + w * b.y, a.z + w * b.z, a.w + w * b.w);
}

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

#define FUSED_MAXNB 7

template <int WPB>
__global__ void __launch_bounds__(WPB * 32) k_fused(FusedArgs A) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * WPB + warp;
  if (j >= A.nprog) return;
  const int mza = A.mza;
  const int iw = A.prog[j];
  const int np = A.npoly[iw];
  const int kb = A.lpw[iw];
  int nb[FUSED_MAXNB], ev[FUSED_MAXNB], own[FUSED_MAXNB];
  float dv[FUSED_MAXNB];
#pragma unroll
  for (int n = 0; n < FUSED_MAXNB; ++n) {
    nb[n] = A.w_nb[iw * 8 + n];
    ev[n] = A.w_ev[iw * 8 + n];
    dv[n] = A.w_dirv[iw * 8 + n];
    own[n] = (n < np) ? (A.v_iw[ev[n] * 2] == iw ? 0 : 1) : 0;
  }
  const float fexpl = 1.0f - A.ff[(size_t)iw * A.nrk + A.istage - 1];
  const float* wm = A.wmasc + (size_t)iw * mza;
  const int nq = A.nq;
  const size_t rowstride = (size_t)nq;  // float4 per (point, level) row

  for (int q0 = 0; q0 < nq; q0 += 32) {
    const int q = q0 + lane;
    if (q >= nq) break;
    auto row = [&](int p, int kd) { return ((size_t)p * mza + kd) * rowstride + q; };
    float4 sm1 = f4(0.f);
    float4 s0 = ld4(A.S + row(iw, kb));
    float4 sp1 = (kb + 1 < mza) ? ld4(A.S + row(iw, kb + 1)) : f4(0.f);
    float4 sp2 = (kb + 2 < mza) ? ld4(A.S + row(iw, kb + 2)) : f4(0.f);
    float4 up_prev = s0;  // scp_upw(kb-1) = scp(kb)
    float4 out_kb = f4(0.f);
    for (int kd = kb; kd < mza; ++kd) {
      // ---- vertical upwind face value at the top of level kd
      float4 up;
      if (kd <= mza - 2) {
        const float wk = __ldg(wm + kd);
        int lev;
        float4 a, b, c;
        if (wk < 0.f) { lev = kd + 1; a = s0; b = sp1; c = sp2; }   // scpb(k+1)
        else          { lev = kd;     a = sm1; b = s0; c = sp1; }   // scpt(k)
        float dsk, dskm1;
        const bool top = (lev > mza - 2), bot = (lev < kb + 1);
        const float a11 = __ldg(A.a_w + lev), a21 = __ldg(A.a_w + lev + mza);
        const float a12 = __ldg(A.a_w + lev + 2 * mza), a22 = __ldg(A.a_w + lev + 3 * mza);
        const float c1 = (wk < 0.f) ? a11 : a12;
        const float c2 = (wk < 0.f) ? a21 : a22;
        float4 r;
#define ZC(comp)                                              \
  dsk = top ? 0.f : (c.comp - b.comp);                        \
  dskm1 = bot ? 0.f : (b.comp - a.comp);                      \
  r.comp = b.comp + dsk * c1 + dskm1 * c2;
        ZC(x) ZC(y) ZC(z) ZC(w)
#undef ZC
        up = r;
      } else {
        up = s0;  // scp_upw(mza) = scp(mza)
      }
      // ---- horizontal flux divergence over the V faces of this column
      float4 sn[FUSED_MAXNB];
#pragma unroll
      for (int n = 0; n < FUSED_MAXNB; ++n)
        if (n < np) sn[n] = ld4(A.S + row(nb[n], kd));
      const float4 s00 = ld4(A.S0 + row(iw, kd));
      float4 fd = f4(0.f);
#pragma unroll
      for (int n = 0; n < FUSED_MAXNB; ++n) {
        if (n >= np) break;
        const int iv = ev[n];
        if (kd < __ldg(A.lpv + iv)) continue;
        const float vm = __ldg(A.vmasc + (size_t)iv * mza + kd);
        const int sd = (vm < 0.f) ? 1 : 0;
        const float* w = A.ew + ((size_t)iv * 2 + sd) * 8;
        float4 val;
        if (sd == own[n]) {
          val = s0;
#pragma unroll
          for (int m = 0; m < FUSED_MAXNB; ++m)
            if (m < np) val = axpy(val, __ldg(w + m), sn[m] - s0);
        } else {
          const int u = nb[n];
          const int npu = __ldg(A.npoly + u);
          const float4 su = sn[n];
          val = su;
          for (int m = 0; m < npu; ++m) {
            const int um = __ldg(A.w_nb + u * 8 + m);
            float4 sx = (um == iw) ? s0 : ld4(A.S + row(um, kd));
            val = axpy(val, __ldg(w + m), sx - su);
          }
        }
        const float f = dv[n] * vm;
        fd = axpy(fd, f, val - s00);
      }
      // ---- vertical flux divergence and update
      const float wkm1 = __ldg(wm + kd - 1), wk0 = __ldg(wm + kd);
      float4 vz;
      vz.x = fexpl * (wkm1 * (up_prev.x - s00.x) - wk0 * (up.x - s00.x));
      vz.y = fexpl * (wkm1 * (up_prev.y - s00.y) - wk0 * (up.y - s00.y));
      vz.z = fexpl * (wkm1 * (up_prev.z - s00.z) - wk0 * (up.z - s00.z));
      vz.w = fexpl * (wkm1 * (up_prev.w - s00.w) - wk0 * (up.w - s00.w));
      fd = fd + vz;
      const float4 st = ld4(A.SCT + row(iw, kd));
      const float vt = __ldg(A.volti + (size_t)iw * mza + kd);
      const float rh = __ldg(A.rhos + (size_t)iw * mza + kd);
      const float dtr = A.dtr;
      float4 o;
      o.x = s00.x + dtr * (st.x + vt * fd.x) / rh;
      o.y = s00.y + dtr * (st.y + vt * fd.y) / rh;
      o.z = s00.z + dtr * (st.z + vt * fd.z) / rh;
      o.w = s00.w + dtr * (st.w + vt * fd.w) / rh;
      A.OUT[row(iw, kd)] = o;
      if (kd == kb) out_kb = o;
      up_prev = up;
      sm1 = s0; s0 = sp1; sp1 = sp2;
      sp2 = (kd + 3 < mza) ? ld4(A.S + row(iw, kd + 3)) : f4(0.f);
    }
    for (int kd = 0; kd < kb; ++kd) A.OUT[row(iw, kd)] = out_kb;
  }
}

void launch_fused_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                        const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr,
                        const float* rhos, cudaStream_t s) {
  FusedArgs A;
  A.mza = d.mza; A.nprog = d.nw_prog; A.nq = ntp / 4; A.nrk = nrk; A.istage = istage; A.dtr = dtr;
  A.prog = d.jtw_prog.p; A.npoly = d.npoly.p; A.w_nb = d.w_nb.p; A.w_ev = d.w_ev.p;
  A.w_dirv = d.w_dirv.p; A.v_iw = d.v_iw.p; A.lpw = d.lpw.p; A.lpv = d.lpv.p;
  A.ew = d.ew_b.p; A.a_w = d.a_w.p; A.volti = d.volti.p;
  A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p; A.rhos = rhos; A.ff = tp.ff.p;
  A.S = reinterpret_cast<const float4*>(S);
  A.S0 = reinterpret_cast<const float4*>(S0);
  A.SCT = reinterpret_cast<const float4*>(SCT);
  A.OUT = reinterpret_cast<float4*>(OUT);
  constexpr int WPB = 8;
  k_fused<WPB><<<cdiv(d.nw_prog, WPB), WPB * 32, 0, s>>>(A);
  OG_LAUNCHED();
}

}  // namespace olamgpu
