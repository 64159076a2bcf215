// dynamics_monot.cu -- fluxes_wrtv_monot (omodel/prog_wrtv_rk.f90:1133-1554):
// on the last RK stage of the acoustic step, the flux-corrected (FCT)
// upwinded face values of thil (ithil_monot > 0) and of vxe, vye, vze
// (iwind_monot > 0), replacing fluxes_wrtv's values for those fields.
//
// Per field, five passes over the same thread-per-(point, level) mapping as
// the other acoustic-step kernels:
//   k_mono_prep    scpt = scp0 + dtr volti sct / rho0 (1179-1186) and the
//                  bounded horizontal gradients of scp (grad_t2d, or
//                  grad_t2d_quadratic with xy_h)
//   k_mono_w       scalar_wflux_monot (1380-1446): the low-order W-face value
//                  from the upwind cell's scpt, the high-order one from
//                  grad_z_quadratic of scp with constant-gradient ends and
//                  a_wu, their difference and its flux arw wmc (high - low)
//   k_mono_v       scalar_vflux_monot (1293-1376): the same on V faces, the
//                  high-order value with the xx0_vu face terms, flux vmca (..)
//   k_mono_lim     scalar_monot_limiter (1450-1552): upwind-biased bounds,
//                  low-order flux divergence, incoming / outgoing high-order
//                  flux sums, and the cell's in / out scale factors
//   k_mono_apply_w / _v   face value = low + (high - low) * the smaller
//                  scale of the two cells the face's flux leaves and enters
// centered_monot = .false. and iorderv = 3, as the reference sets them.
#include "transport_kernels.cuh"

namespace olamgpu {

struct MonoArgs {
  int mza, mwa, mva, ord;
  float dtr;
  const int* __restrict__ npoly;
  const int* __restrict__ w_nb;
  const int* __restrict__ w_ev;
  const float* __restrict__ w_dirv;
  const int* __restrict__ v_iw;
  const int* __restrict__ lpw;
  const int* __restrict__ lpv;
  const float* __restrict__ volti;
  const float* __restrict__ arw;
  const float* __restrict__ a_wu;   // Fortran (mza, 2, 2)
  const float* __restrict__ gxc;    // (mwa, 7)
  const float* __restrict__ gyc;
  const float* __restrict__ xy_h;   // (mwa, 7, 5)
  const float* __restrict__ dxps;   // (mva, 2)
  const float* __restrict__ dyps;
  const float* __restrict__ xx0_vu;
  const float* __restrict__ xy0_vu;
  const float* __restrict__ yy0_vu;
  const float* __restrict__ scp;    // the field
  const float* __restrict__ scp0;   // its value at the start of the step
  const float* __restrict__ sct;    // its volume-weighted long-step tendency
  const double* __restrict__ rho;
  const double* __restrict__ rho0;
  const float* __restrict__ vmca;   // vmc arv of this stage
  const float* __restrict__ wmc;
  float* __restrict__ upw;          // this field's W-face values
  float* __restrict__ upv;          // this field's V-face values
  float* __restrict__ scpt;
  float* __restrict__ gx;           // gradient planes (5 x mwa x mza)
  float* __restrict__ hiw;          // high - low on W faces
  float* __restrict__ sfw;          // its flux
  float* __restrict__ hiv;          // high - low on V faces
  float* __restrict__ sfv;
  float* __restrict__ sin;          // scale_inout(:,:,1)
  float* __restrict__ sout;         // scale_inout(:,:,2)
};

#define MONO_PK(j, kd, n)                                          \
  const size_t i_ = (size_t)blockIdx.x * blockDim.x + threadIdx.x; \
  if (i_ >= (size_t)(n) * A.mza) return;                           \
  const int j = (int)(i_ / A.mza), kd = (int)(i_ % A.mza);

__global__ void k_mono_prep(const int* __restrict__ prog, int nprog, MonoArgs A) {
  MONO_PK(j, kd, nprog);
  const int iw = prog[j];
  if (kd < A.lpw[iw]) return;
  const size_t x = (size_t)iw * A.mza + kd;
  A.scpt[x] = A.scp0[x] + A.dtr * A.volti[x] * A.sct[x] / (float)A.rho0[x];
  if (A.ord < 2) return;
  const size_t plane = (size_t)A.mwa * A.mza;
  const float c0 = A.scp[x];
  float a[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  const int np = A.npoly[iw];
  for (int n = 0; n < np; ++n) {
    const int iv = A.w_ev[iw * 8 + n], iwn = A.w_nb[iw * 8 + n];
    if (kd < A.lpv[iv]) continue;
    const float d = A.scp[(size_t)iwn * A.mza + kd] - c0;
    if (A.ord == 2) {
      a[0] = a[0] + A.gxc[iw * 7 + n] * d;
      a[1] = a[1] + A.gyc[iw * 7 + n] * d;
    } else {
#pragma unroll
      for (int m = 0; m < 5; ++m) a[m] = a[m] + d * A.xy_h[((size_t)iw * 7 + n) * 5 + m];
    }
  }
  const int nplanes = A.ord == 2 ? 2 : 5;
  for (int m = 0; m < nplanes; ++m) A.gx[m * plane + x] = a[m];
}

// W face kd lies between levels kd and kd+1 (device indices); faces kb-1
// and mza-1 are the column's ends
__global__ void k_mono_w(const int* __restrict__ prog, int nprog, MonoArgs A) {
  MONO_PK(j, kd, nprog);
  const int iw = prog[j];
  const int kb = A.lpw[iw], mza = A.mza;
  if (kd < kb - 1) return;
  const size_t cb = (size_t)iw * mza, x = cb + kd;
  const float* S = A.scp + cb;
  if (kd == kb - 1 || kd == mza - 1) {
    A.upw[x] = kd == kb - 1 ? S[kb] : S[mza - 1];
    A.hiw[x] = 0.f;
    A.sfw[x] = 0.f;
    return;
  }
  const bool down = A.wmc[x] < 0.f;
  const float low = down ? A.scpt[x + 1] : A.scpt[x];
  // grad_z_quadratic(itopbc=1, ibotbc=1, bounded=.false.): the bottom face
  // of level kd+1 when the flux is downward, else the top face of level kd
  const int lev = down ? kd + 1 : kd;
  const float dsk = lev <= mza - 2 ? S[lev + 1] - S[lev] : S[mza - 1] - S[mza - 2];
  const float dskm1 = lev >= kb + 1 ? S[lev] - S[lev - 1] : S[kb + 1] - S[kb];
  const float c1 = A.a_wu[lev + (down ? 0 : 2) * mza], c2 = A.a_wu[lev + (down ? 1 : 3) * mza];
  const float high = S[lev] + dsk * c1 + dskm1 * c2;
  const float h = high - low;
  A.upw[x] = low;
  A.hiw[x] = h;
  A.sfw[x] = A.arw[x] * A.wmc[x] * h;
}

__global__ void k_mono_v(const int* __restrict__ vadj, int nv, MonoArgs A) {
  MONO_PK(j, kd, nv);
  const int iv = vadj[j];
  if (kd < A.lpv[iv]) return;
  const int mza = A.mza;
  const int iw1 = A.v_iw[iv * 2], iw2 = A.v_iw[iv * 2 + 1];
  const size_t plane = (size_t)A.mwa * mza;
  const size_t x1 = (size_t)iw1 * mza + kd, x2 = (size_t)iw2 * mza + kd, xv = (size_t)iv * mza + kd;
  const bool neg = A.vmca[xv] < 0.f;
  const float low = neg ? A.scpt[x2] : A.scpt[x1];
  float s1 = A.scp[x1], s2 = A.scp[x2];
  if (A.ord >= 2) {
    const float* G = A.gx;
    s1 = s1 + A.dxps[iv * 2] * G[x1] + A.dyps[iv * 2] * G[plane + x1];
    s2 = s2 + A.dxps[iv * 2 + 1] * G[x2] + A.dyps[iv * 2 + 1] * G[plane + x2];
    if (A.ord == 3) {
      s1 = s1 + A.xx0_vu[iv * 2] * G[2 * plane + x1] + A.xy0_vu[iv * 2] * G[3 * plane + x1] +
           A.yy0_vu[iv * 2] * G[4 * plane + x1];
      s2 = s2 + A.xx0_vu[iv * 2 + 1] * G[2 * plane + x2] + A.xy0_vu[iv * 2 + 1] * G[3 * plane + x2] +
           A.yy0_vu[iv * 2 + 1] * G[4 * plane + x2];
    }
  }
  const float h = (neg ? s2 : s1) - low;
  A.upv[xv] = low;
  A.hiv[xv] = h;
  A.sfv[xv] = A.vmca[xv] * h;
}

__global__ void k_mono_lim(const int* __restrict__ prog, int nprog, MonoArgs A) {
  MONO_PK(j, kd, nprog);
  const int iw = prog[j];
  const int kb = A.lpw[iw], mza = A.mza;
  if (kd < kb) return;
  const float eps0 = 1.e-32f, eps1 = 3.e-07f, onep = 1.0f + eps1;
  const size_t cb = (size_t)iw * mza, x = cb + kd;
  // vertical mass fluxes through the faces below and above the level
  const float wlo = kd >= kb + 1 ? A.wmc[x - 1] * A.arw[x - 1] : 0.f;
  const float whi = kd <= mza - 2 ? A.wmc[x] * A.arw[x] : 0.f;
  const float s = A.scpt[x];
  float smax = s, smin = s;
  if (kd >= kb + 1 && wlo > 0.f) { smax = fmaxf(smax, A.scpt[x - 1]); smin = fminf(smin, A.scpt[x - 1]); }
  if (kd <= mza - 2 && whi < 0.f) { smax = fmaxf(smax, A.scpt[x + 1]); smin = fminf(smin, A.scpt[x + 1]); }
  float fl = 0.f, fi = 0.f, fo = 0.f;
  const int np = A.npoly[iw];
  for (int n = 0; n < np; ++n) {
    const int iv = A.w_ev[iw * 8 + n], iwn = A.w_nb[iw * 8 + n];
    if (kd < A.lpv[iv]) continue;
    const float dv = A.w_dirv[iw * 8 + n];
    const size_t xv = (size_t)iv * mza + kd;
    const float vm = A.vmca[xv];
    fl = fl + dv * vm * (A.upv[xv] - s);
    fi = fi + fmaxf(dv * A.sfv[xv], 0.f);
    fo = fo + fminf(dv * A.sfv[xv], 0.f);
    if (dv * vm > 0.f) {
      const float sn = A.scpt[(size_t)iwn * mza + kd];
      smax = fmaxf(smax, sn);
      smin = fminf(smin, sn);
    }
  }
  fl = fl + wlo * (A.upw[x - 1] - s) - whi * (A.upw[x] - s);
  fi = fi + fmaxf(A.sfw[x - 1], 0.f) - fminf(A.sfw[x], 0.f);
  fo = fo + fminf(A.sfw[x - 1], 0.f) - fmaxf(A.sfw[x], 0.f);
  const float rhos = (float)A.rho[x];
  const float vt = A.volti[x];
  const float dtrp = onep * A.dtr;
  const float rscp_low = s * rhos + A.dtr * vt * fl;
  const float flux_in = fmaxf(dtrp * vt * fi, eps0);
  const float flux_out = fminf(dtrp * vt * fo, -eps0);
  const float epsr = eps1 * fabsf(rscp_low);
  const float sc_in = fmaxf(rhos * smax - (rscp_low + epsr) - eps0, 0.f);
  const float sc_out = fminf(rhos * smin - (rscp_low - epsr) + eps0, 0.f);
  A.sin[x] = fminf(1.f, sc_in / fmaxf(flux_in, 0.01f * sc_in));
  A.sout[x] = fminf(1.f, sc_out / fminf(flux_out, 0.01f * sc_out));
}

__global__ void k_mono_apply_w(const int* __restrict__ prog, int nprog, MonoArgs A) {
  MONO_PK(j, kd, nprog);
  const int iw = prog[j];
  if (kd < A.lpw[iw] || kd > A.mza - 2) return;
  const size_t x = (size_t)iw * A.mza + kd;
  float sc = fminf(A.sin[x + 1], A.sout[x]);
  if (A.sfw[x] < 0.f) sc = fminf(A.sin[x], A.sout[x + 1]);
  A.upw[x] = A.upw[x] + A.hiw[x] * sc;
}

__global__ void k_mono_apply_v(const int* __restrict__ vadj, int nv, MonoArgs A) {
  MONO_PK(j, kd, nv);
  const int iv = vadj[j];
  if (kd < A.lpv[iv]) return;
  const int mza = A.mza;
  const int iw1 = A.v_iw[iv * 2], iw2 = A.v_iw[iv * 2 + 1];
  const size_t x1 = (size_t)iw1 * mza + kd, x2 = (size_t)iw2 * mza + kd, xv = (size_t)iv * mza + kd;
  float sc = fminf(A.sin[x2], A.sout[x1]);
  if (A.sfv[xv] < 0.f) sc = fminf(A.sin[x1], A.sout[x2]);
  A.upv[xv] = A.upv[xv] + A.hiv[xv] * sc;
}

int dyn_monot_faces(Context& C, int field, const float* scp, const float* scp0, const float* sct, float dts,
                    int ord, cudaStream_t s) {
  const DevGrid& d = C.g;
  Dyn& y = C.dy;
  const size_t wz = (size_t)d.mza * d.mwa, vz = (size_t)d.mza * d.mva;
  auto grow = [&](DevBuf<float>& b, size_t n, bool zero) -> int {
    if (b.n >= n) return OLAMGPU_OK;
    OG_CHECK(b.alloc(n));
    // values of points outside jtw_prog are read (as neighbours), never
    // written: they start at zero
    if (zero) OG_CUDA(cudaMemsetAsync(b.p, 0, b.bytes(), s));
    return OLAMGPU_OK;
  };
  OG_CHECK(grow(y.m_scpt, wz, true));
  OG_CHECK(grow(y.m_gx, 5 * wz, true));
  OG_CHECK(grow(y.m_hiw, wz, false));
  OG_CHECK(grow(y.m_sfw, wz, false));
  OG_CHECK(grow(y.m_hiv, vz, false));
  OG_CHECK(grow(y.m_sfv, vz, false));
  OG_CHECK(grow(y.m_sin, wz, true));
  OG_CHECK(grow(y.m_sout, wz, true));
  MonoArgs A;
  A.mza = d.mza; A.mwa = d.mwa; A.mva = d.mva; A.ord = ord; A.dtr = dts;
  A.npoly = d.npoly.p; A.w_nb = d.w_nb.p; A.w_ev = d.w_ev.p; A.w_dirv = d.w_dirv.p; A.v_iw = d.v_iw.p;
  A.lpw = d.lpw.p; A.lpv = d.lpv.p; A.volti = d.volti.p; A.arw = y.arw.p; A.a_wu = d.a_wu.p;
  A.gxc = d.gxc.p; A.gyc = d.gyc.p; A.xy_h = d.xy_h.p; A.dxps = d.dxps.p; A.dyps = d.dyps.p;
  A.xx0_vu = d.xx0_vu.p; A.xy0_vu = d.xy0_vu.p; A.yy0_vu = d.yy0_vu.p;
  A.scp = scp; A.scp0 = scp0; A.sct = sct; A.rho = C.tp.rho.p; A.rho0 = y.rho0.p; A.vmca = y.vmca.p;
  A.wmc = y.wmc.p;
  A.upw = y.upw.p + (size_t)field * wz;
  A.upv = y.upv.p + (size_t)field * vz;
  A.scpt = y.m_scpt.p; A.gx = y.m_gx.p; A.hiw = y.m_hiw.p; A.sfw = y.m_sfw.p; A.hiv = y.m_hiv.p;
  A.sfv = y.m_sfv.p; A.sin = y.m_sin.p; A.sout = y.m_sout.p;
  const unsigned nbw = cdiv((size_t)d.nw_prog * d.mza, 256), nbva = cdiv((size_t)d.nv_wadj * d.mza, 256);
  if (nbw == 0) return OLAMGPU_OK;
  k_mono_prep<<<nbw, 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, A);
  k_mono_w<<<nbw, 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, A);
  OG_LAUNCHED(); OG_LAUNCHED();
  if (nbva) { k_mono_v<<<nbva, 256, 0, s>>>(d.jtv_wadj.p, d.nv_wadj, A); OG_LAUNCHED(); }
  k_mono_lim<<<nbw, 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, A);
  k_mono_apply_w<<<nbw, 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, A);
  OG_LAUNCHED(); OG_LAUNCHED();
  if (nbva) { k_mono_apply_v<<<nbva, 256, 0, s>>>(d.jtv_wadj.p, d.nv_wadj, A); OG_LAUNCHED(); }
  return OLAMGPU_OK;
}

}  // namespace olamgpu
