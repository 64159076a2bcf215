// transport_adjoint_pd.cu -- adjoint of the positive-definite last RK stage of
// scalar_transport_rk (iscal_monot = 2: update_scalar_pd,
// omodel/scalar_transport_rk.F90:1085-1472, and the low-order pre-update of
// scp0 at :297-314) at the forward state, for the tracers with pdef.
//
// The limited stage is not linear in the tracers: its flux scale factors
//   scale = min(1, sc / max(fo, 0.01 sc)),  sc = max(onem rscp_low - eps0, 0),
//   fo = max(-onep dtr volti fluxdiv_out, eps0)
// depend on them.  The adjoint is the transpose of the stage's Jacobian at
// the forward state: every min / max / sign test takes the branch the
// forward took (the limiter's active masks), and where a scale is active its
// derivative with respect to the low-order density and the outflow is
// carried.  The forward's passes (transport_kernels.cu: k_grad, k_vflux,
// k_wcol in the positive-definite mode) are run again on the stage's input
// to record the face values, the flux corrections and the scale factors;
// five gather kernels then transpose the stage (no atomics, so the result
// repeats bit for bit):
//   k_pda_tend   scalar_tend_pd: mu = lam dtr volti / rhos per cell, the
//                adjoint of scp0' from the tendency, of the vertical faces
//   k_pda_scale  the renormalised faces' adjoint onto each cell's scale,
//                then through the scale to the outflow and the low-order
//                density (rscp_low)
//   k_pda_face   per V face: the adjoint of the low-order value and of the
//                high-order correction
//   k_pda_col    per column: the faces' adjoints gathered into the cell,
//                the vertical faces (grad_z_quadratic) and the low-order
//                vertical flux
//   k_pda_grad   the gradient planes (grad_t2d[_quadratic]) transposed
// and k_pda_merge writes the results of the pdef tracers into the batched
// adjoint arrays: the stage input's adjoint, scp0's (scp0' = scp0 + dtr
// sct / rho_old from lpw up) and sct's (dtr / rho_old times scp0's).
#include <algorithm>

#include "transport_kernels.cuh"

namespace olamgpu {

#define PDA_MAXZ 128

struct PdaArgs {
  GridK g;
  const int* prog; int nprog;
  const int* vlist; int nv;          // jtv_wadj
  int nt, ntp, t0, nrk, order;       // group of nt tracers from t0 of the batched layout
  float dtr;
  const int* mode;                   // (nt) MODE_PD where the tracer is limited
  const float* vmasc; const float* wmasc; const float* ff; const float* rhos; const float* rho_old;
  const float* S;                    // stage input (batched)
  const float* S0;                   // scp0' (batched)
  const float* L;                    // adjoint of the stage output (batched, below-ground folded)
  const float* L0imp;                // adjoint of scp0' from the implicit solve (batched; implicit columns)
  // forward records (compact, ld = nt): face values and corrections, scale factors
  const float* upv; const float* hiv; const float* sfv; const float* scale;
  // reverse scratch (compact)
  float* mu; float* lupw; float* lfl; float* lfout; float* l0p; float* lsin; float* lg; float* llo; float* lhi;
  const float* gxc; const float* gyc; const float* xy_h;   // gradient coefficients (bounded)
  const float* dxps; const float* dyps; const float* xx0; const float* xy0; const float* yy0;
};

__device__ __forceinline__ size_t cx(const PdaArgs& A, int p, int kd, int t) {
  return ((size_t)p * A.g.mza + kd) * A.nt + t;
}
__device__ __forceinline__ size_t bx(const PdaArgs& A, int p, int kd, int t) {
  return ((size_t)p * A.g.mza + kd) * A.ntp + A.t0 + t;
}

// scalar_tend_pd transposed: out = s0 + dtr volti fluxdiv / rhos
__global__ void k_pda_tend(PdaArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.nprog * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const GridK& g = A.g;
  const int mza = g.mza, iw = A.prog[i / A.nt], kb = g.lpw[iw], np = g.npoly[iw];
  const float fimpl = A.ff[(size_t)iw * A.nrk + A.nrk - 1];
  const float fe = fimpl > .001f ? 1.f - fimpl : 1.f;
  const float* wm = A.wmasc + (size_t)iw * mza;
  float face_acc = 0.f;   // the adjoint of the bottom face of the level, so far
  for (int kd = kb; kd < mza; ++kd) {
    const float lk = A.L[bx(A, iw, kd, t)];
    const size_t x = (size_t)iw * mza + kd;
    const float m = lk * A.dtr * g.volti[x] / A.rhos[x];
    A.mu[cx(A, iw, kd, t)] = m;
    float sdv = 0.f;
    for (int n = 0; n < np; ++n) {
      const int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      sdv += g.w_dirv[iw * 8 + n] * A.vmasc[(size_t)iv * mza + kd];
    }
    const float l0 = (fimpl > 0.f ? A.L0imp[bx(A, iw, kd, t)] : 0.f) + lk - m * sdv - m * fe * (wm[kd - 1] - wm[kd]);
    A.l0p[cx(A, iw, kd, t)] = l0;
    A.lupw[cx(A, iw, kd - 1, t)] = face_acc + m * fe * wm[kd - 1];
    face_acc = -m * fe * wm[kd];
  }
  A.lupw[cx(A, iw, mza - 1, t)] = face_acc;
}

// the forward's vertical face values of the limited stage (k_wcol, positive-definite mode)
struct PdCol {
  const PdaArgs& A;
  int iw, t, kb, mza;
  const float* wm;
  __device__ float S(int kd) const { return A.S[bx(A, iw, kd, t)]; }
  __device__ float S0(int kd) const { return A.S0[bx(A, iw, kd, t)]; }
  __device__ float lo_face(int kd) const {
    if (kd == kb - 1) return S(kb);
    if (kd == mza - 1) return S(mza - 1);
    return wm[kd] < 0.f ? S0(kd + 1) : S0(kd);
  }
  __device__ float hi_face(int kd) const {
    float sb, st;
    if (wm[kd] < 0.f) {
      const float a0 = S(kd), a1 = S(kd + 1), a2 = (kd + 2 < mza) ? S(kd + 2) : 0.f;
      zrec(A.g.a_w, mza, kd + 1, kb, a0, a1, a2, 0.f, false, false, sb, st);
      return sb - lo_face(kd);
    }
    const float am = (kd - 1 >= kb) ? S(kd - 1) : 0.f, a0 = S(kd), a1 = S(kd + 1);
    zrec(A.g.a_w, mza, kd, kb, am, a0, a1, 0.f, false, false, sb, st);
    return st - lo_face(kd);
  }
};

// the renormalised faces onto each cell's scale, then the scale transposed
__global__ void k_pda_scale(PdaArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.nprog * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const GridK& g = A.g;
  const int mza = g.mza, iw = A.prog[i / A.nt], kb = g.lpw[iw], np = g.npoly[iw];
  const float fimpl = A.ff[(size_t)iw * A.nrk + A.nrk - 1], fexpl = 1.f - fimpl;
  const float* wm = A.wmasc + (size_t)iw * mza;
  const PdCol col{A, iw, t, kb, mza, wm};
  const float eps0 = kEps0, onep = 1.0f + kEps1, onem = 1.0f - kEps1;
  const float mdtrp = -onep * A.dtr;
  float sfw_prev = 0.f, hiw_prev = 0.f;   // the bottom face of the level
  for (int kd = kb; kd < mza; ++kd) {
    const float hiw = kd <= mza - 2 ? col.hi_face(kd) : 0.f;
    const float sfw = kd <= mza - 2 ? fexpl * wm[kd] * hiw : 0.f;
    const float mu_c = A.mu[cx(A, iw, kd, t)];
    const float s00 = col.S0(kd);
    // the adjoint of this cell's scale: the V faces whose correction it scales,
    // the top face where it is the source (sfw >= 0), the bottom face where it
    // is the source (sfw < 0)
    float ls = 0.f, fl = 0.f, fout = 0.f;
    for (int n = 0; n < np; ++n) {
      const int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      const float dv = g.w_dirv[iw * 8 + n];
      const float vm = A.vmasc[(size_t)iv * mza + kd];
      const size_t o = cx(A, iv, kd, t);
      const float sf = A.sfv[o];
      const int sel = sf < 0.f ? g.v_iw[iv * 2 + 1] : g.v_iw[iv * 2];
      if (sel == iw) {
        const int nb = g.w_nb[iw * 8 + n];
        ls += vm * dv * (mu_c - A.mu[cx(A, nb, kd, t)]) * A.hiv[o];
      }
      fl = fl + dv * vm * (A.upv[o] - s00);
      fout = fout + fminf(dv * sf, 0.f);
    }
    if (kd <= mza - 2 && !(sfw < 0.f)) ls += A.lupw[cx(A, iw, kd, t)] * hiw;
    if (kd - 1 >= kb && sfw_prev < 0.f) ls += A.lupw[cx(A, iw, kd - 1, t)] * hiw_prev;
    // the forward's low-order flux and outflow of the cell (k_wcol)
    const float lo_m1 = col.lo_face(kd - 1), lo_k = col.lo_face(kd);
    const size_t x = (size_t)iw * mza + kd;
    const float rh = A.rhos[x], vt = g.volti[x];
    if (fimpl > .001f) {
      fl = fl + fexpl * (wm[kd - 1] * (lo_m1 - s00) - wm[kd] * (lo_k - s00)) + fimpl * s00 * (wm[kd] - wm[kd - 1]);
    } else {
      fl = fl + wm[kd - 1] * (lo_m1 - s00) - wm[kd] * (lo_k - s00);
    }
    fout = fout + fminf(sfw_prev, 0.f) - fmaxf(sfw, 0.f);
    const float rscp = s00 * rh + A.dtr * vt * fl;
    const float fo_raw = mdtrp * vt * fout;
    const float fo = fmaxf(fo_raw, eps0);
    const float sc_raw = onem * rscp - eps0;
    const float sc = fmaxf(sc_raw, 0.f);
    const float den = fmaxf(fo, 0.01f * sc);
    float lfo_out = 0.f, lfl_out = 0.f;
    // where the scale is active (below 1), carry its derivative
    if (ls != 0.f && A.scale[cx(A, iw, kd, t)] < 1.f) {
      float lsc = ls / den;
      const float lden = -ls * sc / (den * den);
      float lfo = 0.f;
      if (fo > 0.01f * sc) lfo = lden;
      else lsc += 0.01f * lden;
      if (fo_raw > eps0) lfo_out = lfo * mdtrp * vt;
      if (sc_raw > 0.f) {
        const float lr = onem * lsc;
        A.l0p[cx(A, iw, kd, t)] += lr * rh;
        lfl_out = lr * A.dtr * vt;
      }
    }
    A.lfout[cx(A, iw, kd, t)] = lfo_out;
    A.lfl[cx(A, iw, kd, t)] = lfl_out;
    sfw_prev = sfw;
    hiw_prev = hiw;
  }
}

// dirv of column iw on face iv
__device__ __forceinline__ float face_dirv(const GridK& g, int iw, int iv) {
  const int np = g.npoly[iw];
  for (int n = 0; n < np; ++n)
    if (g.w_ev[iw * 8 + n] == iv) return g.w_dirv[iw * 8 + n];
  return 0.f;
}

// per V face: the adjoint of the low-order value (llo, less the correction's)
// and of the high-order correction (lhi)
__global__ void k_pda_face(PdaArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const GridK& g = A.g;
  const int mza = g.mza;
  if (i >= (size_t)A.nv * mza * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const size_t r = i / A.nt;
  const int kd = (int)(r % mza), iv = A.vlist[r / mza];
  if (kd < g.lpv[iv]) return;
  const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  const float dv1 = face_dirv(g, iw1, iv), dv2 = face_dirv(g, iw2, iv);
  const float vm = A.vmasc[(size_t)iv * mza + kd];
  const size_t o = cx(A, iv, kd, t);
  const float sf = A.sfv[o];
  const float lupvf = vm * (dv1 * A.mu[cx(A, iw1, kd, t)] + dv2 * A.mu[cx(A, iw2, kd, t)]);
  const float sc = A.scale[cx(A, sf < 0.f ? iw2 : iw1, kd, t)];
  float lsf = 0.f;
  if (dv1 * sf < 0.f) lsf += dv1 * A.lfout[cx(A, iw1, kd, t)];
  if (dv2 * sf < 0.f) lsf += dv2 * A.lfout[cx(A, iw2, kd, t)];
  const float llow = lupvf + vm * (dv1 * A.lfl[cx(A, iw1, kd, t)] + dv2 * A.lfl[cx(A, iw2, kd, t)]);
  const float lh = lupvf * sc + vm * lsf;
  A.llo[o] = llow - lh;
  A.lhi[o] = lh;
}

// per column: the faces' adjoints gathered into its cells, the vertical faces
__global__ void k_pda_col(PdaArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.nprog * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const GridK& g = A.g;
  const int mza = g.mza, iw = A.prog[i / A.nt], kb = g.lpw[iw], np = g.npoly[iw];
  const float fimpl = A.ff[(size_t)iw * A.nrk + A.nrk - 1], fexpl = 1.f - fimpl;
  const bool imp = fimpl > .001f;
  const float fe2 = imp ? fexpl : 1.f;
  const float* wm = A.wmasc + (size_t)iw * mza;
  const PdCol col{A, iw, t, kb, mza, wm};
  const size_t wz = (size_t)g.mwa * mza * A.nt;
  float l0[PDA_MAXZ], ls[PDA_MAXZ];
  for (int kd = 0; kd < mza; ++kd) { l0[kd] = 0.f; ls[kd] = 0.f; }
  for (int kd = kb; kd < mza; ++kd) {
    const float lflc = A.lfl[cx(A, iw, kd, t)];
    float a0 = A.l0p[cx(A, iw, kd, t)], as = 0.f;
    float gm[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int n = 0; n < np; ++n) {
      const int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      const float dv = g.w_dirv[iw * 8 + n];
      const float vm = A.vmasc[(size_t)iv * mza + kd];
      a0 -= lflc * dv * vm;
      // this cell is the face's low-order source and its reconstructed side
      const int side = vm < 0.f ? 1 : 0;
      if (g.v_iw[iv * 2 + side] != iw) continue;
      const size_t o = cx(A, iv, kd, t);
      a0 += A.llo[o];
      const float lh = A.lhi[o];
      as += lh;
      const int e = iv * 2 + side;
      gm[0] += __ldg(A.dxps + e) * lh;
      gm[1] += __ldg(A.dyps + e) * lh;
      if (A.order == 3) {
        gm[2] += __ldg(A.xx0 + e) * lh;
        gm[3] += __ldg(A.xy0 + e) * lh;
        gm[4] += __ldg(A.yy0 + e) * lh;
      }
    }
    a0 -= lflc * fe2 * (wm[kd - 1] - wm[kd]);
    if (imp) a0 += lflc * fimpl * (wm[kd] - wm[kd - 1]);
    l0[kd] += a0;
    ls[kd] += as;
    const int i2d = A.order == 3 ? 5 : 2;
    for (int m = 0; m < i2d; ++m) A.lg[m * wz + cx(A, iw, kd, t)] = gm[m];
  }
  // vertical faces f = kb-1 .. mza-1 (the top face of device level f): the
  // low-order value's adjoint lul and, inside, the correction's lhw
  for (int f = kb - 1; f < mza; ++f) {
    float lul = A.lupw[cx(A, iw, f, t)];
    if (f + 1 <= mza - 1) lul += A.lfl[cx(A, iw, f + 1, t)] * fe2 * wm[f];
    if (f >= kb) lul -= A.lfl[cx(A, iw, f, t)] * fe2 * wm[f];
    if (f == kb - 1) { ls[kb] += lul; continue; }        // scp_upw(kb-1) = scp(kb)
    if (f == mza - 1) { ls[mza - 1] += lul; continue; }  // scp_upw(mza) = scp(mza)
    const float hiw = col.hi_face(f);
    const float sfw = fexpl * wm[f] * hiw;
    float lsw = 0.f;
    if (sfw < 0.f) lsw += A.lfout[cx(A, iw, f + 1, t)];
    if (sfw > 0.f) lsw -= A.lfout[cx(A, iw, f, t)];
    const float scl = A.scale[cx(A, iw, sfw < 0.f ? f + 1 : f, t)];
    const float lhw = A.lupw[cx(A, iw, f, t)] * scl + fexpl * wm[f] * lsw;
    lul -= lhw;
    if (wm[f] < 0.f) {
      // scpb(f+1) from (f, f+1, f+2)
      const int k = f + 1;
      const float a11 = k <= mza - 2 ? AW(g.a_w, mza, k, 1, 1) : 0.f;
      const float a21 = k >= kb + 1 ? AW(g.a_w, mza, k, 2, 1) : 0.f;
      if (k + 1 <= mza - 1) ls[k + 1] += lhw * a11;
      ls[k] += lhw * (1.f - a11 + a21);
      ls[k - 1] -= lhw * a21;
      l0[f + 1] += lul;
    } else {
      // scpt(f) from (f-1, f, f+1)
      const int k = f;
      const float a12 = AW(g.a_w, mza, k, 1, 2);
      const float a22 = k >= kb + 1 ? AW(g.a_w, mza, k, 2, 2) : 0.f;
      ls[k + 1] += lhw * a12;
      ls[k] += lhw * (1.f - a12 + a22);
      if (k - 1 >= kb) ls[k - 1] -= lhw * a22;
      l0[f] += lul;
    }
  }
  for (int kd = kb; kd < mza; ++kd) {
    A.l0p[cx(A, iw, kd, t)] = l0[kd];
    A.lsin[cx(A, iw, kd, t)] = ls[kd];
  }
}

// the gradient planes transposed (gather): g_m(iw) = sum_n c_m(n, iw) (S(iwn) - S(iw))
__global__ void k_pda_grad(PdaArgs A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const GridK& g = A.g;
  const int mza = g.mza;
  if (i >= (size_t)A.nprog * mza * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const size_t r = i / A.nt;
  const int kd = (int)(r % mza), c = A.prog[r / mza];
  if (kd < g.lpw[c]) return;
  const size_t wz = (size_t)g.mwa * mza * A.nt;
  const int i2d = A.order == 3 ? 5 : 2;
  auto coef = [&](int iw, int n, int m) -> float {
    if (A.order == 2) return m == 0 ? __ldg(A.gxc + iw * 7 + n) : __ldg(A.gyc + iw * 7 + n);
    return __ldg(A.xy_h + ((size_t)iw * 7 + n) * 5 + m);
  };
  float acc = 0.f;
  const int np = g.npoly[c];
  for (int n = 0; n < np; ++n) {
    const int iv = g.w_ev[c * 8 + n];
    if (kd < g.lpv[iv]) continue;
    // c's own gradient: -c_m(n, c) lam_g_m(c)
    for (int m = 0; m < i2d; ++m) acc -= coef(c, n, m) * A.lg[m * wz + cx(A, c, kd, t)];
    // the neighbour's gradient, in which c is its p-th neighbour across the same face
    const int nb = g.w_nb[c * 8 + n];
    const int npn = g.npoly[nb];
    for (int p = 0; p < npn; ++p) {
      if (g.w_ev[nb * 8 + p] != iv) continue;
      for (int m = 0; m < i2d; ++m) acc += coef(nb, p, m) * A.lg[m * wz + cx(A, nb, kd, t)];
      break;
    }
  }
  A.lsin[cx(A, c, kd, t)] += acc;
}

// the pdef tracers' results into the batched adjoint arrays (the first
// reverse stage writes them): the stage input's, scp0's and sct's adjoints
__global__ void k_pda_merge(PdaArgs A, float* __restrict__ LIN, float* __restrict__ L0, float* __restrict__ LS) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const GridK& g = A.g;
  const int mza = g.mza;
  if (i >= (size_t)A.nprog * mza * A.nt) return;
  const int t = (int)(i % A.nt);
  if (A.mode[t] != MODE_PD) return;
  const size_t r = i / A.nt;
  const int kd = (int)(r % mza), iw = A.prog[r / mza];
  const bool live = kd >= g.lpw[iw];
  const size_t b = bx(A, iw, kd, t);
  const float l0 = live ? A.l0p[cx(A, iw, kd, t)] : 0.f;
  LIN[b] = live ? A.lsin[cx(A, iw, kd, t)] : 0.f;
  L0[b] = l0;
  LS[b] = live ? l0 * A.dtr / A.rho_old[(size_t)iw * mza + kd] : 0.f;
}

// scratch of the reverse kernels for nt tracers (compact)
static int pda_scratch(Context& C, int nt, int order, DevBuf<float>& buf) {
  const size_t wz = (size_t)C.g.mwa * C.g.mza * nt, vz = (size_t)C.g.mva * C.g.mza * nt;
  const size_t need = wz * (6 + (order == 3 ? 5 : 2)) + vz * 2;
  if (buf.n < need) OG_CHECK(buf.alloc(need));
  return OLAMGPU_OK;
}

static DevBuf<float> g_pda;

void pd_adjoint_release() { g_pda.release(); }

int pd_adjoint_stage(Context& C, const float* S, const float* S0p, const float* L, float* LIN, float* L0,
                     float* LS, float dtr, int t0, int ntr, cudaStream_t s) {
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  const int mza = d.mza, order = C.opts.scal_horiz_adv_order, nrk = C.opts.nrk_scal;
  const int ntp = C.tr.ntp;
  if (mza > PDA_MAXZ) {
    set_error("the adjoint of the positive-definite limiter needs mza <= " + std::to_string(PDA_MAXZ));
    return OLAMGPU_E_UNSUPPORTED;
  }
  const size_t plane = (size_t)mza * d.mwa;
  const float* rhos_nrk = tp.rhos.p + (size_t)(nrk - 1) * plane;
  // tracer groups sized to a scratch budget (forward records and reverse scratch)
  const size_t per = (size_t)4 * mza * ((size_t)(8 + 3 * (order == 3 ? 5 : 2)) * d.mwa + (size_t)5 * d.mva) + 1;
  const int grp = (int)std::max<size_t>(1, std::min<size_t>((size_t)ntr, (size_t)(12ull << 30) / per));
  for (int g0 = t0; g0 < t0 + ntr; g0 += grp) {
    const int nt = std::min(grp, t0 + ntr - g0);
    // the forward's limited-stage passes on the stage input: face values,
    // corrections and scale factors of the group
    const size_t wz = (size_t)d.mwa * mza * nt, vz = (size_t)d.mva * mza * nt;
    const int i2d = order == 3 ? 5 : 2;
    auto grow = [](DevBuf<float>& b, size_t n) { return b.n >= n ? OLAMGPU_OK : b.alloc(n); };
    OG_CHECK(grow(tp.gx, wz * i2d));
    OG_CHECK(grow(tp.upv, vz));
    OG_CHECK(grow(tp.hiv, vz));
    OG_CHECK(grow(tp.sfv, vz));
    OG_CHECK(grow(tp.scale, wz * 2));
    OG_CHECK(grow(tp.upw, wz));
    OG_CHECK(pda_scratch(C, nt, order, g_pda));
    float* p = g_pda.p;
    PdaArgs A;
    A.g = gridk(d);
    A.prog = d.jtw_prog.p; A.nprog = d.nw_prog; A.vlist = d.jtv_wadj.p; A.nv = d.nv_wadj;
    A.nt = nt; A.ntp = ntp; A.t0 = g0; A.nrk = nrk; A.order = order; A.dtr = dtr;
    A.mode = tp.d_mode.p + g0;
    A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p; A.ff = tp.ff.p; A.rhos = rhos_nrk; A.rho_old = tp.rho_old.p;
    A.S = S; A.S0 = S0p; A.L = L; A.L0imp = L0;
    A.upv = tp.upv.p; A.hiv = tp.hiv.p; A.sfv = tp.sfv.p; A.scale = tp.scale.p;
    A.mu = p; p += wz;
    A.lupw = p; p += wz;
    A.lfl = p; p += wz;
    A.lfout = p; p += wz;
    A.l0p = p; p += wz;
    A.lsin = p; p += wz;
    A.lg = p; p += wz * i2d;
    A.llo = p; p += vz;
    A.lhi = p;
    A.gxc = d.gxc.p; A.gyc = d.gyc.p; A.xy_h = d.xy_h.p;
    A.dxps = d.dxps.p; A.dyps = d.dyps.p; A.xx0 = d.xx0_v.p; A.xy0 = d.xy0_v.p; A.yy0 = d.yy0_v.p;
    {
      OG_PROF("adj_pd_forward", s);
      launch_grad(d, CTView{S, ntp, g0}, tp.gx.p, nt, order, true, s);
      launch_vflux(d, tp, CTView{S, ntp, g0}, CTView{S0p, ntp, g0}, tp.gx.p, nt, order, false, A.mode, true, s);
      // the unlimited tracers of the group get an update the merge ignores
      launch_wcol(d, tp, CTView{S, ntp, g0}, CTView{S0p, ntp, g0}, CTView{S0p, ntp, g0}, rhos_nrk,
                  TView{A.lsin, nt, 0}, nt, nrk, nrk, dtr, A.mode, true, s);
    }
    {
      OG_PROF("adj_pd_stage", s);
      const size_t nc = (size_t)d.nw_prog * nt, nvk = (size_t)d.nv_wadj * mza * nt, nck = (size_t)d.nw_prog * mza * nt;
      k_pda_tend<<<cdiv(nc, 128), 128, 0, s>>>(A);
      k_pda_scale<<<cdiv(nc, 128), 128, 0, s>>>(A);
      k_pda_face<<<cdiv(nvk, 256), 256, 0, s>>>(A);
      k_pda_col<<<cdiv(nc, 128), 128, 0, s>>>(A);
      k_pda_grad<<<cdiv(nck, 256), 256, 0, s>>>(A);
      // the group's results into the batched arrays (the batched stage
      // kernel that follows leaves these tracers alone)
      k_pda_merge<<<cdiv(nck, 256), 256, 0, s>>>(A, LIN, L0, LS);
      OG_LAUNCHED(); OG_LAUNCHED(); OG_LAUNCHED(); OG_LAUNCHED(); OG_LAUNCHED(); OG_LAUNCHED();
    }
  }
  return OLAMGPU_OK;
}

}  // namespace olamgpu
