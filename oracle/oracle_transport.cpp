/*
 * oracle_transport.cpp -- TEST INFRASTRUCTURE ONLY (see oracle_common.h).
 * PARITY UNPINNED (no Fortran compiler, no reference golden vectors).
 *
 * CPU restatement of scalar_transport_rk and its callees:
 *   scalar_transport_rk    omodel/scalar_transport_rk.F90:30-385
 *   update_scalar          omodel/scalar_transport_rk.F90:389-615
 *   update_scalar_monot    omodel/scalar_transport_rk.F90:619-1081
 *   update_scalar_pd       omodel/scalar_transport_rk.F90:1085-1472
 *   check_cfls             omodel/scalar_transport_rk.F90:1476-1712
 *   grad_z_linear          omodel/grad_lib.f90:106-153
 *   grad_z_quadratic       omodel/grad_lib.f90:166-229
 *   grad_t2d               omodel/grad_lib.f90:236-269
 *   grad_t2d_quadratic     omodel/grad_lib.f90:278-341
 *   tridif_prep/fini       outils/tridiag_lib.f90:321-364
 * The column loops carry `#pragma omp parallel for` as the reference's
 * `!$omp parallel do`; results do not depend on the thread count.
 */
#include <cstdio>
#include <cstring>

#include "oracle_common.h"
#include "oracle_dual.h"

namespace oracle {

// scalar_transport_rk.F90:14-17 (real parameters: in precision T)
#define kEps0 1.e-32
#define kEps1 3.e-07

static const int kIorderv = 3;  // scalar_transport_rk.F90:20

/* grad_z_linear (grad_lib.f90:106-153) */
template <class T>
static void grad_z_linear(const GridT<T>& G, int iw, const T* scp /*col(1..mza) at [k-1]*/,
                          T* scp_bot, T* scp_top, int itop, int ibot) {
  const int mza = G.mza;
  const int kb = G.lpw(iw);
  std::vector<T> gwz(mza + 1);
  const float* dzim = G.g->dzim;
  const float* dzt_top = G.g->dzt_top;
  const float* dzt_bot = G.g->dzt_bot;
  for (int k = kb; k <= mza - 1; ++k) gwz[k] = (T)dzim[k - 1] * (scp[k] - scp[k - 1]);
  gwz[kb - 1] = 0;
  if (ibot != 0) gwz[kb - 1] = gwz[kb];
  gwz[mza] = 0;
  if (itop != 0) gwz[mza] = gwz[mza - 1];
  for (int k = kb; k <= mza; ++k) {
    T gzps = (T)0.5 * (gwz[k - 1] + gwz[k]);
    scp_bot[k - 1] = scp[k - 1] - gzps * (T)dzt_bot[k - 1];
    scp_top[k - 1] = scp[k - 1] + gzps * (T)dzt_top[k - 1];
  }
}

/* grad_z_quadratic (grad_lib.f90:166-229).  scp, scp_bot, scp_top are
 * columns indexed [k-1]; ds is indexed by k (0..mza). */
template <class T>
static void grad_z_quadratic(const GridT<T>& G, int iw, const T* scp, T* scp_bot, T* scp_top,
                             int itop, int ibot, bool constrained) {
  const int mza = G.mza;
  const int ka = G.lpw(iw);
  std::vector<T> ds(mza + 1);
  for (int k = ka; k <= mza - 1; ++k) ds[k] = scp[k] - scp[k - 1];
  ds[ka - 1] = 0;
  if (ibot != 0) ds[ka - 1] = ds[ka];
  ds[mza] = 0;
  if (itop != 0) ds[mza] = ds[mza - 1];
  const std::vector<T>& a = constrained ? G.a_w : G.a_wu;
  for (int k = ka; k <= mza; ++k) {
    scp_bot[k - 1] = scp[k - 1] + ds[k] * G.aw(a, k, 1, 1) + ds[k - 1] * G.aw(a, k, 2, 1);
    scp_top[k - 1] = scp[k - 1] + ds[k] * G.aw(a, k, 1, 2) + ds[k - 1] * G.aw(a, k, 2, 2);
  }
}

/* grad_t2d (grad_lib.f90:236-269): gxps, gyps columns [k-1] */
template <class T>
static void grad_t2d(const GridT<T>& G, int iw, const T* scp, T* gxps, T* gyps) {
  const int mza = G.mza;
  for (int k = 1; k <= mza; ++k) { gxps[k - 1] = 0; gyps[k - 1] = 0; }
  for (int n = 1; n <= G.npoly(iw); ++n) {
    int iwn = G.w_iw(iw, n);
    int ivn = G.w_iv(iw, n);
    T cx = G.gxps_coef(n, iw), cy = G.gyps_coef(n, iw);
    for (int k = G.lpv(ivn); k <= mza; ++k) {
      T dscp = F2(scp, k, iwn) - F2(scp, k, iw);
      gxps[k - 1] = gxps[k - 1] + cx * dscp;
      gyps[k - 1] = gyps[k - 1] + cy * dscp;
    }
  }
}

/* grad_t2d_quadratic (grad_lib.f90:278-341): g[m] are 5 columns [k-1] */
template <class T>
static void grad_t2d_quadratic(const GridT<T>& G, int iw, const T* scp, T* const g[5],
                               bool constrained) {
  const int mza = G.mza;
  for (int m = 0; m < 5; ++m)
    for (int k = 1; k <= mza; ++k) g[m][k - 1] = 0;
  const std::vector<T>& xy = constrained ? G.xy_h : G.xy_hu;
  for (int n = 1; n <= G.npoly(iw); ++n) {
    int iwn = G.w_iw(iw, n);
    int ivn = G.w_iv(iw, n);
    T c[5];
    for (int m = 0; m < 5; ++m) c[m] = G.xyh(xy, m + 1, n, iw);
    for (int k = G.lpv(ivn); k <= mza; ++k) {
      T sc = F2(scp, k, iwn) - F2(scp, k, iw);
      for (int m = 0; m < 5; ++m) g[m][k - 1] = g[m][k - 1] + sc * c[m];
    }
  }
}

/* gradient pass shared by update_scalar/_monot/_pd (iorderh 2 or 3) */
template <class T>
static void gradients(const GridT<T>& G, const T* scp, int iorderh, bool constrained,
                      std::vector<T>& gxyps) {
  const int mza = G.mza, mwa = G.mwa;
  const int nw = G.g->nw_prog;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T* base = gxyps.data();
    size_t plane = (size_t)mza * mwa;
    T* c0 = base + (size_t)(iw - 1) * mza;
    if (iorderh == 2) {
      grad_t2d(G, iw, scp, c0, c0 + plane);
    } else if (iorderh == 3) {
      T* g5[5] = {c0, c0 + plane, c0 + 2 * plane, c0 + 3 * plane, c0 + 4 * plane};
      grad_t2d_quadratic(G, iw, scp, g5, constrained);
    }
  }
}

/* scp1/scp2 of scalar_v_column (scalar_transport_rk.F90:490-527): the
 * reconstructed value on side s of V face iv at level k. */
template <class T>
static inline T side_value(const GridT<T>& G, const T* scp, const std::vector<T>& gxyps, int iorderh,
                           bool unbounded, int iv, int s, int k) {
  const int mza = G.mza, mwa = G.mwa;
  int iws = G.v_iw(iv, s);
  size_t plane = (size_t)mza * mwa;
  T v = F2(scp, k, iws);
  if (iorderh == 1) return v;
  const T* gx = gxyps.data();
  v = v + G.v2(G.dxps, s, iv) * gx[(size_t)(iws - 1) * mza + k - 1]
        + G.v2(G.dyps, s, iv) * gx[plane + (size_t)(iws - 1) * mza + k - 1];
  if (iorderh == 3) {
    const std::vector<T>& xx = unbounded ? G.xx0_vu : G.xx0_v;
    const std::vector<T>& xy = unbounded ? G.xy0_vu : G.xy0_v;
    const std::vector<T>& yy = unbounded ? G.yy0_vu : G.yy0_v;
    v = v + G.v2(xx, s, iv) * gx[2 * plane + (size_t)(iws - 1) * mza + k - 1]
          + G.v2(xy, s, iv) * gx[3 * plane + (size_t)(iws - 1) * mza + k - 1]
          + G.v2(yy, s, iv) * gx[4 * plane + (size_t)(iws - 1) * mza + k - 1];
  }
  return v;
}

/* The Fortran evaluates scp + dxps*g1 + dyps*g2 + ... left to right; the
 * helper above groups identically: ((scp + a) + b) + ... */

template <class T>
struct TransportCtx {
  const GridT<T>& G;
  int mza, mwa, mva;
  const std::vector<T>& vmasc;
  const std::vector<T>& wmasc;
  const std::vector<T>& ff_implic;  // (nrk, mwa)
  int nrk;
  T ff(int n, int iw) const { return ff_implic[(size_t)(iw - 1) * nrk + (n - 1)]; }
};

/* update_scalar (scalar_transport_rk.F90:389-615) */
template <class T>
static void update_scalar(const TransportCtx<T>& C, T* scp, const T* scp0, const T* sct,
                          const T* rhos, T dtr, int iorderh, int istage) {
  const GridT<T>& G = C.G;
  const int mza = G.mza, mwa = G.mwa, mva = G.mva;
  const int i2d = iorderh == 2 ? 2 : (iorderh == 3 ? 5 : 0);
  std::vector<T> gxyps((size_t)mza * mwa * (i2d > 0 ? i2d : 1));
  std::vector<T> scp_upv((size_t)mza * mva);
  const T* vmasc = C.vmasc.data();
  const T* wmasc = C.wmasc.data();
  if (iorderh > 1) gradients(G, scp, iorderh, true, gxyps);
  // scalar_v_column over jtv_wadj
  const int nv = G.g->nv_wadj;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nv; ++j) {
    int iv = G.g->jtv_wadj[j];
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T s1 = side_value(G, scp, gxyps, iorderh, false, iv, 1, k);
      T s2 = side_value(G, scp, gxyps, iorderh, false, iv, 2, k);
      T up = s1;
      if (F2(vmasc, k, iv) < (T)0) up = s2;
      F2(scp_upv.data(), k, iv) = up;
    }
  }
  // scalar_w_column over jtw_prog
  const int nw = G.g->nw_prog;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T fimpl = C.ff(istage, iw);
    int kb = G.lpw(iw);
    T fexpl = (T)1.0 - fimpl;
    std::vector<T> scpb(mza), scpt(mza), scp_upw(mza + 1), fluxdiv(mza + 1);
    const T* col = scp + (size_t)(iw - 1) * mza;
    scp_upw[kb - 1] = col[kb - 1];
    scp_upw[mza] = col[mza - 1];
    if (kIorderv == 1) {
      for (int k = kb; k <= mza - 1; ++k) { scpb[k - 1] = col[k - 1]; scpt[k - 1] = col[k - 1]; }
    } else if (kIorderv == 2) {
      grad_z_linear(G, iw, col, scpb.data(), scpt.data(), 0, 0);
    } else {
      grad_z_quadratic(G, iw, col, scpb.data(), scpt.data(), 0, 0, true);
    }
    for (int k = kb; k <= mza - 1; ++k) {
      scp_upw[k] = scpt[k - 1];
      if (F2(wmasc, k, iw) < (T)0) scp_upw[k] = scpb[k];
    }
    std::fill(fluxdiv.begin(), fluxdiv.end(), (T)0);
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      int iv = G.w_iv(iw, jv);
      T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k)
        fluxdiv[k] = fluxdiv[k] + d * F2(vmasc, k, iv) * (F2(scp_upv.data(), k, iv) - F2(scp0, k, iw));
    }
    for (int k = kb; k <= mza; ++k) {
      T s0 = F2(scp0, k, iw);
      fluxdiv[k] = fluxdiv[k] + fexpl * (F2(wmasc, k - 1, iw) * (scp_upw[k - 1] - s0)
                                         - F2(wmasc, k, iw) * (scp_upw[k] - s0));
      F2(scp, k, iw) = s0 + dtr * (F2(sct, k, iw) + G.volti_(k, iw) * fluxdiv[k]) / F2(rhos, k, iw);
    }
    for (int k = 1; k <= kb - 1; ++k) F2(scp, k, iw) = F2(scp, kb, iw);
  }
}

/* Shared by the monotonic and positive-definite variants: high-order and
 * low-order V-face values (scalar_vflux_monot 749-832, scalar_vflux_pd 1215-1285). */
template <class T>
static void vflux_hilo(const TransportCtx<T>& C, const T* scp, const T* scp0,
                       const std::vector<T>& gxyps, int iorderh, bool unbounded, bool pd,
                       std::vector<T>& scp_upv, std::vector<T>& scp_hiv, std::vector<T>& sfluxvh) {
  const GridT<T>& G = C.G;
  const int mza = G.mza;
  const T* vmasc = C.vmasc.data();
  const int nv = G.g->nv_wadj;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nv; ++j) {
    int iv = G.g->jtv_wadj[j];
    int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T s1, s2;
      if (iorderh == 1) {
        s1 = F2(scp, k, iw1);
        s2 = pd ? F2(scp, k, iw1) : F2(scp, k, iw2);  // scalar_transport_rk.F90:1237 (pd) vs 778
      } else {
        s1 = side_value(G, scp, gxyps, iorderh, unbounded, iv, 1, k);
        s2 = side_value(G, scp, gxyps, iorderh, unbounded, iv, 2, k);
      }
      T vm = F2(vmasc, k, iv);
      T lo = F2(scp0, k, iw1);
      if (vm < (T)0) lo = F2(scp0, k, iw2);
      T hi = s1;
      if (vm < (T)0) hi = s2;
      hi = hi - lo;
      F2(scp_upv.data(), k, iv) = lo;
      F2(scp_hiv.data(), k, iv) = hi;
      F2(sfluxvh.data(), k, iv) = vm * hi;
    }
  }
}

/* update_scalar_monot (scalar_transport_rk.F90:619-1081) */
template <class T>
static void update_scalar_monot(const TransportCtx<T>& C, T* scp, const T* scp0, const T* rhos,
                                T dtr, int iorderh, int istage) {
  const GridT<T>& G = C.G;
  const int mza = G.mza, mwa = G.mwa, mva = G.mva;
  const int i2d = iorderh == 2 ? 2 : (iorderh == 3 ? 5 : 0);
  std::vector<T> gxyps((size_t)mza * mwa * (i2d > 0 ? i2d : 1));
  std::vector<T> scp_upv((size_t)mza * mva), scp_hiv((size_t)mza * mva), sfluxvh((size_t)mza * mva);
  std::vector<T> scale_inout((size_t)mza * mwa * 2, (T)0), scp_upw((size_t)mza * mwa + 1);
  const T* vmasc = C.vmasc.data();
  const T* wmasc = C.wmasc.data();
  const T eps0 = (T)kEps0, eps1 = (T)kEps1, onep = (T)1.0 + eps1;
  if (iorderh > 1) gradients(G, scp, iorderh, false, gxyps);
  vflux_hilo(C, scp, scp0, gxyps, iorderh, true, false, scp_upv, scp_hiv, sfluxvh);
  const size_t plane = (size_t)mza * mwa;
  // scalar_wflux_and_scales_monot (835-1022); scp_upw(kb-1..mza) per column,
  // stored at scp_upw[(iw-1)*mza + k - 1] with k-1 = 0 for kb-1 = 1.
  const int nw = G.g->nw_prog;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T fimpl = C.ff(istage, iw);
    T dtrp = onep * dtr;
    int kb = G.lpw(iw);
    T fexpl = (T)1. - fimpl;
    T* upw = scp_upw.data() + (size_t)(iw - 1) * mza;  // upw[k-1] = scp_upw(k,iw)
    std::vector<T> scpb(mza), scpt(mza), hiw(mza + 1), sfw(mza + 1), smax(mza + 1), smin(mza + 1);
    std::vector<T> fl(mza + 1, (T)0), fin(mza + 1, (T)0), fout(mza + 1, (T)0);
    const T* s0c = scp0 + (size_t)(iw - 1) * mza;
    upw[kb - 2] = s0c[kb - 1];
    upw[mza - 1] = s0c[mza - 1];
    for (int k = kb; k <= mza - 1; ++k) {
      upw[k - 1] = s0c[k - 1];
      if (F2(wmasc, k, iw) < (T)0) upw[k - 1] = s0c[k];
    }
    const T* col = scp + (size_t)(iw - 1) * mza;
    if (kIorderv == 1) {
      for (int k = kb; k <= mza; ++k) { scpb[k - 1] = col[k - 1]; scpt[k - 1] = col[k - 1]; }
    } else if (kIorderv == 2) {
      grad_z_linear(G, iw, col, scpb.data(), scpt.data(), 1, 1);
    } else {
      grad_z_quadratic(G, iw, col, scpb.data(), scpt.data(), 1, 1, false);
    }
    sfw[kb - 1] = 0;
    sfw[mza] = 0;
    for (int k = kb; k <= mza - 1; ++k) {
      hiw[k] = scpt[k - 1];
      if (F2(wmasc, k, iw) < (T)0) hiw[k] = scpb[k];
      hiw[k] = hiw[k] - upw[k - 1];
      sfw[k] = fexpl * F2(wmasc, k, iw) * hiw[k];
    }
    for (int k = kb; k <= mza; ++k) { smax[k] = s0c[k - 1]; smin[k] = s0c[k - 1]; }
    for (int k = kb + 1; k <= mza; ++k)
      if (F2(wmasc, k - 1, iw) > (T)0) {
        smax[k] = fmax_(smax[k], s0c[k - 2]);
        smin[k] = fmin_(smin[k], s0c[k - 2]);
      }
    for (int k = kb; k <= mza - 1; ++k)
      if (F2(wmasc, k, iw) < (T)0) {
        smax[k] = fmax_(smax[k], s0c[k]);
        smin[k] = fmin_(smin[k], s0c[k]);
      }
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      int iv = G.w_iv(iw, jv), iwn = G.w_iw(iw, jv);
      T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k) {
        fl[k] = fl[k] + d * F2(vmasc, k, iv) * (F2(scp_upv.data(), k, iv) - s0c[k - 1]);
        fin[k] = fin[k] + fmax_(d * F2(sfluxvh.data(), k, iv), (T)0);
        fout[k] = fout[k] + fmin_(d * F2(sfluxvh.data(), k, iv), (T)0);
        if (d * F2(vmasc, k, iv) > (T)0) {
          smax[k] = fmax_(smax[k], F2(scp0, k, iwn));
          smin[k] = fmin_(smin[k], F2(scp0, k, iwn));
        }
      }
    }
    auto upwv = [&](int k) { return upw[k - 1]; };
    if (fimpl > (T)0.001) {
      for (int k = kb; k <= mza; ++k) {
        T dwi = fimpl * (F2(wmasc, k, iw) - F2(wmasc, k - 1, iw));
        fl[k] = fl[k] + fexpl * (F2(wmasc, k - 1, iw) * (upwv(k - 1) - s0c[k - 1])
                                 - F2(wmasc, k, iw) * (upwv(k) - s0c[k - 1]))
                + s0c[k - 1] * dwi;
        fin[k] = fin[k] + fmax_(sfw[k - 1], (T)0) - fmin_(sfw[k], (T)0);
        fout[k] = fout[k] + fmin_(sfw[k - 1], (T)0) - fmax_(sfw[k], (T)0);
        T imp = F2(rhos, k, iw) + dtr * G.volti_(k, iw) * dwi;
        smax[k] = imp * smax[k];
        smin[k] = imp * smin[k];
      }
    } else {
      for (int k = kb; k <= mza; ++k) {
        fl[k] = fl[k] + F2(wmasc, k - 1, iw) * (upwv(k - 1) - s0c[k - 1])
                - F2(wmasc, k, iw) * (upwv(k) - s0c[k - 1]);
        fin[k] = fin[k] + fmax_(sfw[k - 1], (T)0) - fmin_(sfw[k], (T)0);
        fout[k] = fout[k] + fmin_(sfw[k - 1], (T)0) - fmax_(sfw[k], (T)0);
        smax[k] = F2(rhos, k, iw) * smax[k];
        smin[k] = F2(rhos, k, iw) * smin[k];
      }
    }
    for (int k = kb; k <= mza; ++k) {
      T vt = G.volti_(k, iw);
      T rscp_low = s0c[k - 1] * F2(rhos, k, iw) + dtr * vt * fl[k];
      T flux_in = fmax_(dtrp * vt * fin[k], eps0);
      T flux_out = fmin_(dtrp * vt * fout[k], -eps0);
      T epsr = eps1 * abs_(rscp_low);
      T sc_in = fmax_(smax[k] - (rscp_low + epsr) - eps0, (T)0);
      T sc_out = fmin_(smin[k] - (rscp_low - epsr) + eps0, (T)0);
      scale_inout[(size_t)(iw - 1) * mza + k - 1] =
          fmin_((T)1., sc_in / fmax_(flux_in, (T)0.01 * sc_in));
      scale_inout[plane + (size_t)(iw - 1) * mza + k - 1] =
          fmin_((T)1., sc_out / fmin_(flux_out, (T)0.01 * sc_out));
    }
    const T* s1 = scale_inout.data() + (size_t)(iw - 1) * mza;
    const T* s2 = scale_inout.data() + plane + (size_t)(iw - 1) * mza;
    for (int k = kb; k <= mza - 1; ++k) {
      T scale = fmin_(s1[k], s2[k - 1]);
      if (sfw[k] < (T)0) scale = fmin_(s1[k - 1], s2[k]);
      upw[k - 1] = upw[k - 1] + hiw[k] * scale;
    }
  }
  // apply renormalisation to horizontal fluxes (711-724)
  const int nv = G.g->nv_wadj;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nv; ++j) {
    int iv = G.g->jtv_wadj[j];
    int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T a = scale_inout[(size_t)(iw2 - 1) * mza + k - 1];          // (k,iw2,1)
      T b = scale_inout[plane + (size_t)(iw1 - 1) * mza + k - 1];  // (k,iw1,2)
      T scale = fmin_(a, b);
      if (F2(sfluxvh.data(), k, iv) < (T)0)
        scale = fmin_(scale_inout[(size_t)(iw1 - 1) * mza + k - 1],
                      scale_inout[plane + (size_t)(iw2 - 1) * mza + k - 1]);
      F2(scp_upv.data(), k, iv) = F2(scp_upv.data(), k, iv) + F2(scp_hiv.data(), k, iv) * scale;
    }
  }
  // scalar_tend_monot (1025-1078)
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T fimpl = C.ff(istage, iw);
    int kb = G.lpw(iw);
    std::vector<T> fd(mza + 1, (T)0);
    const T* upw = scp_upw.data() + (size_t)(iw - 1) * mza;
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      int iv = G.w_iv(iw, jv);
      T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k)
        fd[k] = fd[k] + d * F2(vmasc, k, iv) * (F2(scp_upv.data(), k, iv) - F2(scp0, k, iw));
    }
    if (fimpl > (T).001) {
      T fexpl = (T)1. - fimpl;
      for (int k = kb; k <= mza; ++k) {
        T s0 = F2(scp0, k, iw);
        fd[k] = fd[k] + fexpl * (F2(wmasc, k - 1, iw) * (upw[k - 2] - s0) - F2(wmasc, k, iw) * (upw[k - 1] - s0));
        F2(scp, k, iw) = s0 + dtr * G.volti_(k, iw) * fd[k] / F2(rhos, k, iw);
      }
    } else {
      for (int k = kb; k <= mza; ++k) {
        T s0 = F2(scp0, k, iw);
        fd[k] = fd[k] + F2(wmasc, k - 1, iw) * (upw[k - 2] - s0) - F2(wmasc, k, iw) * (upw[k - 1] - s0);
        F2(scp, k, iw) = s0 + dtr * G.volti_(k, iw) * fd[k] / F2(rhos, k, iw);
      }
      for (int k = 2; k <= kb - 1; ++k) F2(scp, k, iw) = F2(scp, kb, iw);
    }
  }
}

/* update_scalar_pd (scalar_transport_rk.F90:1085-1472) */
template <class T>
static void update_scalar_pd(const TransportCtx<T>& C, T* scp, const T* scp0, const T* rhos,
                             T dtr, int iorderh, int istage) {
  const GridT<T>& G = C.G;
  const int mza = G.mza, mwa = G.mwa, mva = G.mva;
  const int i2d = iorderh == 2 ? 2 : (iorderh == 3 ? 5 : 0);
  std::vector<T> gxyps((size_t)mza * mwa * (i2d > 0 ? i2d : 1));
  std::vector<T> scp_upv((size_t)mza * mva), scp_hiv((size_t)mza * mva), sfluxvh((size_t)mza * mva);
  std::vector<T> scale_out((size_t)mza * mwa, (T)0), scp_upw((size_t)mza * mwa + 1);
  const T* vmasc = C.vmasc.data();
  const T* wmasc = C.wmasc.data();
  const T eps0 = (T)kEps0, onep = (T)1.0 + (T)kEps1, onem = (T)1.0 - (T)kEps1;
  if (iorderh > 1) gradients(G, scp, iorderh, true, gxyps);
  vflux_hilo(C, scp, scp0, gxyps, iorderh, false, true, scp_upv, scp_hiv, sfluxvh);
  const int nw = G.g->nw_prog;
  // scalar_wflux_and_scale_pd (1288-1414)
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T fimpl = C.ff(istage, iw);
    T mdtrp = -onep * dtr;
    int kb = G.lpw(iw);
    T fexpl = (T)1. - fimpl;
    T* upw = scp_upw.data() + (size_t)(iw - 1) * mza;
    std::vector<T> scpb(mza), scpt(mza), hiw(mza + 1), sfw(mza + 1);
    std::vector<T> fl(mza + 1, (T)0), fout(mza + 1, (T)0);
    const T* s0c = scp0 + (size_t)(iw - 1) * mza;
    const T* col = scp + (size_t)(iw - 1) * mza;
    upw[kb - 2] = col[kb - 1];   // scp_upw(kb-1) = scp(kb)   (1316)
    upw[mza - 1] = col[mza - 1]; // scp_upw(mza)  = scp(mza)  (1317)
    for (int k = kb; k <= mza - 1; ++k) {
      upw[k - 1] = s0c[k - 1];
      if (F2(wmasc, k, iw) < (T)0) upw[k - 1] = s0c[k];
    }
    if (kIorderv == 1) {
      for (int k = kb; k <= mza - 1; ++k) { scpb[k - 1] = col[k - 1]; scpt[k - 1] = col[k - 1]; }
    } else if (kIorderv == 2) {
      grad_z_linear(G, iw, col, scpb.data(), scpt.data(), 0, 0);
    } else {
      grad_z_quadratic(G, iw, col, scpb.data(), scpt.data(), 0, 0, true);
    }
    sfw[kb - 1] = 0;
    sfw[mza] = 0;
    for (int k = kb; k <= mza - 1; ++k) {
      hiw[k] = scpt[k - 1];
      if (F2(wmasc, k, iw) < (T)0) hiw[k] = scpb[k];
      hiw[k] = hiw[k] - upw[k - 1];
      sfw[k] = fexpl * F2(wmasc, k, iw) * hiw[k];
    }
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      int iv = G.w_iv(iw, jv);
      T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k) {
        fl[k] = fl[k] + d * F2(vmasc, k, iv) * (F2(scp_upv.data(), k, iv) - s0c[k - 1]);
        fout[k] = fout[k] + fmin_(d * F2(sfluxvh.data(), k, iv), (T)0);
      }
    }
    if (fimpl > (T).001) {
      for (int k = kb; k <= mza; ++k) {
        fl[k] = fl[k] + fexpl * (F2(wmasc, k - 1, iw) * (upw[k - 2] - s0c[k - 1])
                                 - F2(wmasc, k, iw) * (upw[k - 1] - s0c[k - 1]))
                + fimpl * s0c[k - 1] * (F2(wmasc, k, iw) - F2(wmasc, k - 1, iw));
        fout[k] = fout[k] + fmin_(sfw[k - 1], (T)0) - fmax_(sfw[k], (T)0);
      }
    } else {
      for (int k = kb; k <= mza; ++k) {
        fl[k] = fl[k] + F2(wmasc, k - 1, iw) * (upw[k - 2] - s0c[k - 1])
                - F2(wmasc, k, iw) * (upw[k - 1] - s0c[k - 1]);
        fout[k] = fout[k] + fmin_(sfw[k - 1], (T)0) - fmax_(sfw[k], (T)0);
      }
    }
    T* so = scale_out.data() + (size_t)(iw - 1) * mza;
    for (int k = kb; k <= mza; ++k) {
      T rscp_low = s0c[k - 1] * F2(rhos, k, iw) + dtr * G.volti_(k, iw) * fl[k];
      T flux_out = fmax_(mdtrp * G.volti_(k, iw) * fout[k], eps0);
      T sc_out = fmax_(onem * rscp_low - eps0, (T)0);
      so[k - 1] = fmin_((T)1., sc_out / fmax_(flux_out, (T)0.01 * sc_out));
    }
    for (int k = kb; k <= mza - 1; ++k) {
      T scale = so[k - 1];
      if (sfw[k] < (T)0) scale = so[k];
      upw[k - 1] = upw[k - 1] + hiw[k] * scale;
    }
  }
  const int nv = G.g->nv_wadj;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nv; ++j) {
    int iv = G.g->jtv_wadj[j];
    int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T scale = scale_out[(size_t)(iw1 - 1) * mza + k - 1];
      if (F2(sfluxvh.data(), k, iv) < (T)0) scale = scale_out[(size_t)(iw2 - 1) * mza + k - 1];
      F2(scp_upv.data(), k, iv) = F2(scp_upv.data(), k, iv) + F2(scp_hiv.data(), k, iv) * scale;
    }
  }
  // scalar_tend_pd (1417-1469)
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    T fimpl = C.ff(istage, iw);
    int kb = G.lpw(iw);
    std::vector<T> fd(mza + 1, (T)0);
    const T* upw = scp_upw.data() + (size_t)(iw - 1) * mza;
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      int iv = G.w_iv(iw, jv);
      T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k)
        fd[k] = fd[k] + d * F2(vmasc, k, iv) * (F2(scp_upv.data(), k, iv) - F2(scp0, k, iw));
    }
    if (fimpl > (T).001) {
      T fexpl = (T)1. - fimpl;
      for (int k = kb; k <= mza; ++k) {
        T s0 = F2(scp0, k, iw);
        fd[k] = fd[k] + fexpl * (F2(wmasc, k - 1, iw) * (upw[k - 2] - s0) - F2(wmasc, k, iw) * (upw[k - 1] - s0));
        F2(scp, k, iw) = s0 + dtr * G.volti_(k, iw) * fd[k] / F2(rhos, k, iw);
      }
    } else {
      for (int k = kb; k <= mza; ++k) {
        T s0 = F2(scp0, k, iw);
        fd[k] = fd[k] + F2(wmasc, k - 1, iw) * (upw[k - 2] - s0) - F2(wmasc, k, iw) * (upw[k - 1] - s0);
        F2(scp, k, iw) = s0 + dtr * G.volti_(k, iw) * fd[k] / F2(rhos, k, iw);
      }
      for (int k = 2; k <= kb - 1; ++k) F2(scp, k, iw) = F2(scp, kb, iw);
    }
  }
}

/* check_cfls (scalar_transport_rk.F90:1476-1712).  Serial reduction in
 * jtw_prog order, so the location of a tie is the first column reached. */
template <class T>
static void check_cfls(const GridT<T>& G, const std::vector<T>& vmasc, const std::vector<T>& wmasc,
                       const std::vector<T>& rho, const float* wc, int nrk, T dtl,
                       std::vector<T>& ff_implic, olamgpu_cfl_diag* diag) {
  const int mza = G.mza;
  const int nw = G.g->nw_prog;
  std::vector<T> cflv((size_t)nw * mza), cflhv((size_t)nw * mza);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    std::vector<T> cflh(mza + 1, (T)0), cfl(mza + 1, (T)0);
    T fimp[3] = {0, 0, 0};
    for (int n = 1; n <= G.npoly(iw); ++n) {
      int iv = G.w_iv(iw, n);
      T d = G.w_dirv(iw, n);
      for (int k = G.lpv(iv); k <= mza; ++k)
        cflh[k] = cflh[k] - fmin_(d * F2(vmasc.data(), k, iv), (T)0.0);
    }
    for (int k = G.lpw(iw); k <= mza; ++k) {
      T dovr = dtl * G.volti_(k, iw) / F2(rho.data(), k, iw);
      cflh[k] = cflh[k] * dovr;
      T cflw = (fmax_(F2(wmasc.data(), k, iw), (T)0.) - fmin_(F2(wmasc.data(), k - 1, iw), (T)0.)) * dovr;
      cfl[k] = cflh[k] + cflw;
      cflw = fmax_(cflw, (T).1);
      fimp[nrk - 1] = fmax_(fimp[nrk - 1], (cfl[k] - (T)0.98) / cflw);
      fimp[nrk - 2] = fmax_(fimp[nrk - 2], (cfl[k] - (T)1.98) / cflw);
      if (nrk == 3) fimp[0] = fmax_(fimp[0], (cfl[k] - (T)2.98) / cflw);
    }
    for (int n = 1; n <= nrk; ++n) {
      T f = fmin_((T)1.0, fimp[n - 1]);
      if (f < (T).02) f = 0;
      ff_implic[(size_t)(iw - 1) * nrk + (n - 1)] = f;
    }
    for (int k = 1; k <= mza; ++k) {
      cflv[(size_t)j * mza + k - 1] = cfl[k];
      cflhv[(size_t)j * mza + k - 1] = cflh[k];
    }
  }
  if (!diag) return;
  T ct = 0, ch = 0;
  float wm = 0;
  int itk = 1, itw = 1, ihk = 1, ihw = 1, iwk = 1, iww = 1;
  for (int j = 0; j < nw; ++j) {
    int iw = G.g->jtw_prog[j];
    int glob = G.g->iwglobe ? G.g->iwglobe[iw - 1] : iw;
    for (int k = G.lpw(iw); k <= mza; ++k) {
      T c = cflv[(size_t)j * mza + k - 1];
      if (c > ct || c != c) { ct = c; itk = k; itw = glob; }
      T h = cflhv[(size_t)j * mza + k - 1];
      if (h > ch || h != h) { ch = h; ihk = k; ihw = glob; }
      if (wc) {
        float w = F2(wc, k, iw);
        if (std::fabs(w) > std::fabs(wm) || w != w) { wm = w; iwk = k; iww = glob; }
      }
    }
  }
  diag->cfl_max = (float)ct; diag->cfl_k = itk; diag->cfl_iwglobe = itw;
  diag->cflh_max = (float)ch; diag->cflh_k = ihk; diag->cflh_iwglobe = ihw;
  diag->w_max = wm; diag->w_k = iwk; diag->w_iwglobe = iww;
}

/* tridif_prep / tridif_fini (tridiag_lib.f90:321-364), columns indexed by k */
template <class T>
static void tridif_prep(int ka, int kz, const T* cim1, const T* ci, const T* cip1, T* scr1, T* cji) {
  cji[ka] = (T)1.0 / ci[ka];
  for (int k = ka + 1; k <= kz; ++k) {
    scr1[k] = cji[k - 1] * cip1[k - 1];
    cji[k] = (T)1.0 / (ci[k] - cim1[k] * scr1[k]);
  }
}
template <class T>
static void tridif_fini(int ka, int kz, const T* cim1, const T* scr1, const T* cji, const T* rhs, T* soln) {
  soln[ka] = rhs[ka] * cji[ka];
  for (int k = ka + 1; k <= kz; ++k) soln[k] = cji[k] * (rhs[k] - cim1[k] * soln[k - 1]);
  for (int k = kz - 1; k >= ka; --k) soln[k] = soln[k] - scr1[k + 1] * soln[k + 1];
}

/* Per-long-step coefficients of scalar_transport_rk that depend only on the
 * winds and densities (scalar_transport_rk.F90:95-217): RK stage timesteps,
 * the implicit fractions from check_cfls, the stage densities rhos and the
 * implicit columns' tridiagonal factors.  Shared by the forward and adjoint. */
template <class T>
struct StepCoef {
  int nrk = 0;
  T dtlr[3] = {0, 0, 0};
  std::vector<T> vmasc, wmasc, rho_old, ff_implic, rhos;
  std::vector<int> kwtop;
  struct Imp { std::vector<int> iw; std::vector<T> b1, b2, b3; };
  std::vector<Imp> imp;
};

template <class T>
static int prepare_step(const GridT<T>& G, const olamgpu_grid* g, const olamgpu_opts* o, const float* vmasc_f,
                        const float* wmasc_f, const double* rho, const float* rho_old_f, const float* wc,
                        const int* khtopv, olamgpu_cfl_diag* diag, StepCoef<T>& S) {
  const int mza = g->mza, mwa = g->mwa, mva = g->mva;
  const int nrk = o->nrk_scal;
  if (nrk != 2 && nrk != 3) return OLAMGPU_E_UNSUPPORTED;
  S.nrk = nrk;
  const T dtl = (T)o->dtlm;  // real dtl = dtlm (r8 -> real)
  S.vmasc = cvt<T>(vmasc_f, (size_t)mza * mva);
  S.wmasc = cvt<T>(wmasc_f, (size_t)mza * mwa);
  S.rho_old = cvt<T>(rho_old_f, (size_t)mza * mwa);
  const T one3 = (T)1. / (T)3.;
  const T frk3[3] = {one3, (T)0.5, (T)1.0};
  const T frk2[2] = {(T)0.5, (T)1.0};
  for (int n = 0; n < nrk; ++n) S.dtlr[n] = dtl * (nrk == 3 ? frk3[n] : frk2[n]);

  S.ff_implic.assign((size_t)nrk * mwa, (T)0);
  check_cfls(G, S.vmasc, S.wmasc, S.rho_old, wc, nrk, dtl, S.ff_implic, diag);

  // rhos (117-162); nudging off
  S.rhos.assign((size_t)mza * mwa * nrk, (T)0);
  S.kwtop.assign(mwa + 1, 0);
  const size_t plane = (size_t)mza * mwa;
  for (int j = 0; j < g->nw_prog; ++j) {
    int iw = g->jtw_prog[j];
    int kb = G.lpw(iw);
    for (int k = kb; k <= mza; ++k) {
      T rhof = (T)F2(rho, k, iw);
      T ro = F2(S.rho_old.data(), k, iw);
      size_t ix = (size_t)(iw - 1) * mza + k - 1;
      if (nrk == 3) {
        S.rhos[ix] = (T)(2. / 3.) * ro + (T)(1. / 3.) * rhof;
        S.rhos[plane + ix] = (T)0.5 * (ro + rhof);
        S.rhos[2 * plane + ix] = rhof;
      } else {
        S.rhos[ix] = (T)0.5 * (ro + rhof);
        S.rhos[plane + ix] = rhof;
      }
    }
    if (khtopv) {
      int m = 0;
      for (int n = 1; n <= G.npoly(iw); ++n) m = std::max(m, khtopv[G.w_iv(iw, n) - 1]);
      S.kwtop[iw] = m;
    }
  }
  // implicit factorisation per stage (164-217); columns kept in jtw_prog order
  S.imp.assign(nrk, typename StepCoef<T>::Imp());
  for (int n = 1; n <= nrk; ++n) {
    auto& I = S.imp[n - 1];
    for (int j = 0; j < g->nw_prog; ++j) {
      int iw = g->jtw_prog[j];
      if (S.ff_implic[(size_t)(iw - 1) * nrk + n - 1] > (T)0.001) I.iw.push_back(iw);
    }
    size_t nn = I.iw.size();
    I.b1.assign(nn * (mza + 1), 0); I.b2.assign(nn * (mza + 1), 0); I.b3.assign(nn * (mza + 1), 0);
    for (size_t jj = 0; jj < nn; ++jj) {
      int iw = I.iw[jj];
      int kb = G.lpw(iw);
      std::vector<T> wup(mza + 1, 0), wdn(mza + 1, 0), b2a(mza + 1, 0), b3a(mza + 1, 0);
      for (int k = kb; k <= mza - 1; ++k) {
        wup[k] = fmax_(F2(S.wmasc.data(), k, iw), (T)0.);
        wdn[k] = fmin_(F2(S.wmasc.data(), k, iw), (T)0.);
      }
      T c1 = S.ff_implic[(size_t)(iw - 1) * nrk + n - 1] * S.dtlr[n - 1];
      T* b1 = &I.b1[jj * (mza + 1)];
      for (int k = kb; k <= mza; ++k) {
        T c2 = c1 * G.volti_(k, iw) / S.rhos[(size_t)(n - 1) * plane + (size_t)(iw - 1) * mza + k - 1];
        b1[k] = -c2 * wup[k - 1];
        b2a[k] = (T)1.0 + c2 * (wup[k] - wdn[k - 1]);
        b3a[k] = c2 * wdn[k];
      }
      tridif_prep(kb, mza, b1, b2a.data(), b3a.data(), &I.b2[jj * (mza + 1)], &I.b3[jj * (mza + 1)]);
    }
  }
  return OLAMGPU_OK;
}

/* implicit vertical transport of one stage (scalar_transport_rk.F90:347-375) */
template <class T>
static void implicit_step(const GridT<T>& G, const StepCoef<T>& SC, int istage, T dtr, T* scp, const T* scp0) {
  const int mza = G.mza, nrk = SC.nrk;
  const size_t plane = (size_t)mza * G.mwa;
  const auto& I = SC.imp[istage - 1];
  const int nn = (int)I.iw.size();
#pragma omp parallel for schedule(static)
  for (int jj = 0; jj < nn; ++jj) {
    int iw = I.iw[jj];
    int kb = G.lpw(iw);
    std::vector<T> dscp0(mza + 1, 0), delex(mza + 1, 0), del(mza + 1, 0);
    dscp0[mza] = 0;
    dscp0[kb - 1] = 0;
    for (int k = kb; k <= mza - 1; ++k) dscp0[k] = F2(scp0, k + 1, iw) - F2(scp0, k, iw);
    T ffv = SC.ff_implic[(size_t)(iw - 1) * nrk + istage - 1];
    for (int k = kb; k <= mza; ++k) {
      T c1 = ffv * dtr * G.volti_(k, iw) / SC.rhos[(size_t)(istage - 1) * plane + (size_t)(iw - 1) * mza + k - 1];
      delex[k] = F2(scp, k, iw) - F2(scp0, k, iw) -
                 c1 * (fmin_(F2(SC.wmasc.data(), k, iw), (T)0.) * dscp0[k] +
                       fmax_(F2(SC.wmasc.data(), k - 1, iw), (T)0.) * dscp0[k - 1]);
    }
    tridif_fini(kb, mza, &I.b1[(size_t)jj * (mza + 1)], &I.b2[(size_t)jj * (mza + 1)],
                &I.b3[(size_t)jj * (mza + 1)], delex.data(), del.data());
    for (int k = kb; k <= mza; ++k) F2(scp, k, iw) = F2(scp0, k, iw) + del[k];
    for (int k = 2; k <= kb - 1; ++k) F2(scp, k, iw) = F2(scp, kb, iw);
  }
}

/* scalar_transport_rk (scalar_transport_rk.F90:30-385) */
template <class T>
static int scalar_transport_rk(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                               T* const* scp_list, T* const* sct_list, const int* pdef,
                               const int* sgsmix, const float* vmasc_f, const float* wmasc_f,
                               const double* rho, const float* rho_old_f, const float* wc,
                               const float* akhodx, const int* khtopv, float* ff_out,
                               olamgpu_cfl_diag* diag) {
  GridT<T> G(g);
  const int mza = g->mza, mwa = g->mwa, mva = g->mva;
  const int iorder = o->scal_horiz_adv_order;
  const int imonot = o->iscal_monot;
  StepCoef<T> SC;
  int rc = prepare_step(G, g, o, vmasc_f, wmasc_f, rho, rho_old_f, wc, khtopv, diag, SC);
  if (rc != OLAMGPU_OK) return rc;
  const int nrk = SC.nrk;
  const T* dtlr = SC.dtlr;
  const std::vector<T>& vmasc = SC.vmasc;
  const std::vector<T>& wmasc = SC.wmasc;
  const std::vector<T>& rho_old = SC.rho_old;
  const std::vector<T>& ff_implic = SC.ff_implic;
  const std::vector<T>& rhos = SC.rhos;
  const std::vector<int>& kwtop = SC.kwtop;
  const size_t plane = (size_t)mza * mwa;
  if (ff_out)
    for (size_t i = 0; i < ff_implic.size(); ++i) ff_out[i] = (float)ff_implic[i];

  TransportCtx<T> C{G, mza, mwa, mva, vmasc, wmasc, ff_implic, nrk};
  std::vector<T> scp0(plane);
  const T* rhos_nrk = rhos.data() + (size_t)(nrk - 1) * plane;

  for (int n = 0; n < nscal; ++n) {
    T* scp = scp_list[n];
    T* sct = sct_list[n];
    for (int j = 0; j < g->nw_wadj; ++j) {
      int iw = g->jtw_wadj[j];
      for (int k = 1; k <= mza; ++k) F2(scp0.data(), k, iw) = F2(scp, k, iw);
    }
    // horizontal diffusion hook (244-274)
    if (sgsmix && sgsmix[n] && akhodx && khtopv) {
#pragma omp parallel for schedule(static)
      for (int j = 0; j < g->nw_prog; ++j) {
        int iw = g->jtw_prog[j];
        if (kwtop[iw] < G.lpw(iw)) continue;
        std::vector<T> fd(mza + 1, (T)0);
        for (int jv = 1; jv <= G.npoly(iw); ++jv) {
          int iv = G.w_iv(iw, jv), iwn = G.w_iw(iw, jv);
          for (int k = G.lpv(iv); k <= khtopv[iv - 1]; ++k)
            fd[k] = fd[k] + (T)F2(akhodx, k, iv) * (F2(scp, k, iwn) - F2(scp, k, iw));
        }
        for (int k = G.lpw(iw); k <= kwtop[iw]; ++k)
          F2(sct, k, iw) = F2(sct, k, iw) + fd[k] * G.volti_(k, iw);
      }
    }
    const bool pd = pdef ? (pdef[n] != 0) : false;
    for (int istage = 1; istage <= nrk; ++istage) {
      T dtr = dtlr[istage - 1];
      if (istage == nrk && imonot > 0 && pd) {
        for (int j = 0; j < g->nw_wadj; ++j) {
          int iw = g->jtw_wadj[j];
          int kb = G.lpw(iw);
          for (int k = kb; k <= mza; ++k)
            F2(scp0.data(), k, iw) = F2(scp0.data(), k, iw) + dtr * F2(sct, k, iw) / F2(rho_old.data(), k, iw);
          for (int k = 2; k <= kb - 1; ++k) F2(scp0.data(), k, iw) = F2(scp0.data(), kb, iw);
        }
      }
      if (istage == nrk && imonot == 1) {
        update_scalar_monot(C, scp, scp0.data(), rhos_nrk, dtr, iorder, istage);
      } else if (istage == nrk && imonot == 2 && pd) {
        update_scalar_pd(C, scp, scp0.data(), rhos_nrk, dtr, iorder, istage);
      } else {
        update_scalar(C, scp, scp0.data(), sct, rhos_nrk, dtr, iorder, istage);
      }
      implicit_step(G, SC, istage, dtr, scp, scp0.data());
    }
  }
  return OLAMGPU_OK;
}

/* The positive-definite last stage (update_scalar_pd,
 * scalar_transport_rk.F90:1085-1472) with every intermediate kept, for its
 * adjoint: the same arithmetic as update_scalar_pd above, in the same
 * order, on the stage input S and the pre-updated scp0' (S0). */
template <class T>
struct PdRecord {
  std::vector<T> gx, upv_low, hiv, sfv;             // faces: (mza, mva); gx: gradient planes
  std::vector<T> upw_low, hiw, sfw;                  // columns: (mza + 1) per W point, index k
  std::vector<T> rscp, fo_raw, fo, sc_raw, sc, den, scale;   // cells (mza, mwa)
};

template <class T>
static void pd_record(const TransportCtx<T>& C, const T* S, const T* S0, const T* rhos, T dtr, int iorderh,
                      int istage, PdRecord<T>& R) {
  const GridT<T>& G = C.G;
  const int mza = G.mza, mwa = G.mwa, mva = G.mva;
  const int i2d = iorderh == 2 ? 2 : (iorderh == 3 ? 5 : 0);
  const size_t plane = (size_t)mza * mwa, cols = (size_t)(mza + 1) * (mwa + 1);
  R.gx.assign(plane * (i2d > 0 ? i2d : 1), (T)0);
  R.upv_low.assign((size_t)mza * mva, (T)0); R.hiv = R.upv_low; R.sfv = R.upv_low;
  R.upw_low.assign(cols, (T)0); R.hiw = R.upw_low; R.sfw = R.upw_low;
  R.rscp.assign(plane, (T)0); R.fo_raw = R.rscp; R.fo = R.rscp; R.sc_raw = R.rscp; R.sc = R.rscp;
  R.den = R.rscp; R.scale = R.rscp;
  const T* vmasc = C.vmasc.data();
  const T* wmasc = C.wmasc.data();
  const T eps0 = (T)kEps0, onep = (T)1.0 + (T)kEps1, onem = (T)1.0 - (T)kEps1;
  if (iorderh > 1) gradients(G, S, iorderh, true, R.gx);
  vflux_hilo(C, S, S0, R.gx, iorderh, false, true, R.upv_low, R.hiv, R.sfv);
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j];
    const T fimpl = C.ff(istage, iw);
    const T mdtrp = -onep * dtr;
    const int kb = G.lpw(iw);
    const T fexpl = (T)1. - fimpl;
    T* upw = &R.upw_low[(size_t)iw * (mza + 1)];   // upw[k], k = kb-1 .. mza
    T* hiw = &R.hiw[(size_t)iw * (mza + 1)];
    T* sfw = &R.sfw[(size_t)iw * (mza + 1)];
    std::vector<T> scpb(mza), scpt(mza), fl(mza + 1, (T)0), fout(mza + 1, (T)0);
    const T* s0c = S0 + (size_t)(iw - 1) * mza;
    const T* col = S + (size_t)(iw - 1) * mza;
    upw[kb - 1] = col[kb - 1];
    upw[mza] = col[mza - 1];
    for (int k = kb; k <= mza - 1; ++k) {
      upw[k] = s0c[k - 1];
      if (F2(wmasc, k, iw) < (T)0) upw[k] = s0c[k];
    }
    grad_z_quadratic(G, iw, col, scpb.data(), scpt.data(), 0, 0, true);
    sfw[kb - 1] = 0;
    sfw[mza] = 0;
    for (int k = kb; k <= mza - 1; ++k) {
      hiw[k] = scpt[k - 1];
      if (F2(wmasc, k, iw) < (T)0) hiw[k] = scpb[k];
      hiw[k] = hiw[k] - upw[k];
      sfw[k] = fexpl * F2(wmasc, k, iw) * hiw[k];
    }
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      const int iv = G.w_iv(iw, jv);
      const T d = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k) {
        fl[k] = fl[k] + d * F2(vmasc, k, iv) * (F2(R.upv_low.data(), k, iv) - s0c[k - 1]);
        fout[k] = fout[k] + fmin_(d * F2(R.sfv.data(), k, iv), (T)0);
      }
    }
    for (int k = kb; k <= mza; ++k) {
      if (fimpl > (T).001)
        fl[k] = fl[k] + fexpl * (F2(wmasc, k - 1, iw) * (upw[k - 1] - s0c[k - 1])
                                 - F2(wmasc, k, iw) * (upw[k] - s0c[k - 1]))
                + fimpl * s0c[k - 1] * (F2(wmasc, k, iw) - F2(wmasc, k - 1, iw));
      else
        fl[k] = fl[k] + F2(wmasc, k - 1, iw) * (upw[k - 1] - s0c[k - 1])
                - F2(wmasc, k, iw) * (upw[k] - s0c[k - 1]);
      fout[k] = fout[k] + fmin_(sfw[k - 1], (T)0) - fmax_(sfw[k], (T)0);
      const size_t x = (size_t)(iw - 1) * mza + k - 1;
      R.rscp[x] = s0c[k - 1] * F2(rhos, k, iw) + dtr * G.volti_(k, iw) * fl[k];
      R.fo_raw[x] = mdtrp * G.volti_(k, iw) * fout[k];
      R.fo[x] = fmax_(R.fo_raw[x], eps0);
      R.sc_raw[x] = onem * R.rscp[x] - eps0;
      R.sc[x] = fmax_(R.sc_raw[x], (T)0);
      R.den[x] = fmax_(R.fo[x], (T)0.01 * R.sc[x]);
      R.scale[x] = fmin_((T)1., R.sc[x] / R.den[x]);
    }
  }
}

/* Transpose of the positive-definite last stage at the recorded forward
 * state, branch by branch: every min / max / sign test takes the side the
 * forward took (the limiter's active masks), so this is the transpose of
 * the stage's Jacobian there.  L: adjoint of the stage output (below-ground
 * levels already folded); adds the adjoint of the stage input S to Lin and
 * of S0 (scp0') to L0p. */
template <class T>
static void pd_stage_adjoint(const TransportCtx<T>& C, const PdRecord<T>& R, const T* S0, const T* rhos, T dtr,
                             int iorderh, int istage, const T* L, T* Lin, T* L0p) {
  const GridT<T>& G = C.G;
  const int mza = G.mza, mwa = G.mwa, mva = G.mva;
  const size_t plane = (size_t)mza * mwa;
  const int np2d = iorderh == 2 ? 2 : 5;
  const T* vm = C.vmasc.data();
  const T* wm = C.wmasc.data();
  const T onep = (T)1.0 + (T)kEps1, onem = (T)1.0 - (T)kEps1, eps0 = (T)kEps0;
  std::vector<T> Lupv((size_t)mza * mva, (T)0), Lupv_low((size_t)mza * mva, (T)0), Lhiv((size_t)mza * mva, (T)0),
      Lsfv((size_t)mza * mva, (T)0), Lscale(plane, (T)0), Lg(plane * np2d, (T)0);
  const size_t cw = (size_t)(mza + 1);
  std::vector<T> Lupw(cw * (mwa + 1), (T)0), Lupw_low(cw * (mwa + 1), (T)0), Lhiw(cw * (mwa + 1), (T)0),
      Lsfw(cw * (mwa + 1), (T)0);
  auto scale_at = [&](int k, int iw) { return R.scale[(size_t)(iw - 1) * mza + k - 1]; };
  // scalar_tend_pd: out = s0 + dtr volti fluxdiv / rhos
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j], kb = G.lpw(iw);
    const T fimpl = C.ff(istage, iw);
    const T fe = fimpl > (T).001 ? (T)1. - fimpl : (T)1.;
    T* lupw = &Lupw[(size_t)iw * cw];
    for (int k = kb; k <= mza; ++k) {
      const T lk = F2(L, k, iw);
      const T mu = lk * dtr * G.volti_(k, iw) / F2(rhos, k, iw);
      F2(L0p, k, iw) += lk;
      for (int jv = 1; jv <= G.npoly(iw); ++jv) {
        const int iv = G.w_iv(iw, jv);
        if (k < G.lpv(iv)) continue;
        const T a = mu * G.w_dirv(iw, jv) * F2(vm, k, iv);
        F2(Lupv.data(), k, iv) += a;
        F2(L0p, k, iw) -= a;
      }
      lupw[k - 1] += mu * fe * F2(wm, k - 1, iw);
      lupw[k] -= mu * fe * F2(wm, k, iw);
      F2(L0p, k, iw) -= mu * fe * (F2(wm, k - 1, iw) - F2(wm, k, iw));
    }
  }
  // vertical faces: upw = upw_low + hiw * scale(k or k+1)
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j], kb = G.lpw(iw);
    const T* lupw = &Lupw[(size_t)iw * cw];
    T* lul = &Lupw_low[(size_t)iw * cw];
    T* lhw = &Lhiw[(size_t)iw * cw];
    const T* hiw = &R.hiw[(size_t)iw * cw];
    const T* sfw = &R.sfw[(size_t)iw * cw];
    lul[kb - 1] += lupw[kb - 1];   // the boundary faces carry scp(kb), scp(mza) unscaled
    lul[mza] += lupw[mza];
    for (int k = kb; k <= mza - 1; ++k) {
      const int ks = sfw[k] < (T)0 ? k + 1 : k;
      lul[k] += lupw[k];
      lhw[k] += lupw[k] * scale_at(ks, iw);
      Lscale[(size_t)(iw - 1) * mza + ks - 1] += lupw[k] * hiw[k];
    }
  }
  // horizontal faces: upv = upv_low + hiv * scale(iw1, or iw2 where sfluxvh < 0)
  for (int j = 0; j < G.g->nv_wadj; ++j) {
    const int iv = G.g->jtv_wadj[j];
    const int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      const T a = F2(Lupv.data(), k, iv);
      const int ws = F2(R.sfv.data(), k, iv) < (T)0 ? iw2 : iw1;
      F2(Lupv_low.data(), k, iv) += a;
      F2(Lhiv.data(), k, iv) += a * scale_at(k, ws);
      Lscale[(size_t)(ws - 1) * mza + k - 1] += a * F2(R.hiv.data(), k, iv);
    }
  }
  // the scale factors: scale = min(1, sc / max(fo, 0.01 sc)), sc = max(onem rscp - eps0, 0),
  // fo = max(mdtrp volti fout, eps0), rscp = s0 rhos + dtr volti fl
  std::vector<T> Lfl(plane, (T)0), Lfout(plane, (T)0);
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j], kb = G.lpw(iw);
    for (int k = kb; k <= mza; ++k) {
      const size_t x = (size_t)(iw - 1) * mza + k - 1;
      const T ls = Lscale[x];
      const T ratio = R.sc[x] / R.den[x];
      if (ls == (T)0 || (T)1. < ratio) continue;   // min took 1: no dependence
      T lsc = ls / R.den[x];
      const T lden = -ls * R.sc[x] / (R.den[x] * R.den[x]);
      T lfo = 0;
      if (R.fo[x] > (T)0.01 * R.sc[x]) lfo = lden;
      else lsc += (T)0.01 * lden;
      if (R.fo_raw[x] > eps0) Lfout[x] += lfo * (-onep * dtr) * G.volti_(k, iw);
      if (R.sc_raw[x] > (T)0) {
        const T lr = onem * lsc;
        F2(L0p, k, iw) += lr * F2(rhos, k, iw);
        Lfl[x] += lr * dtr * G.volti_(k, iw);
      }
    }
  }
  // fout = sum_f min(dirv sfluxvh, 0) + min(sfw(k-1), 0) - max(sfw(k), 0);
  // fl = sum_f dirv vm (upv_low - s0) + the low-order vertical flux
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j], kb = G.lpw(iw);
    const T fimpl = C.ff(istage, iw);
    const T fexpl = (T)1. - fimpl;
    const bool imp = fimpl > (T).001;
    const T fe = imp ? fexpl : (T)1.;
    const T* sfw = &R.sfw[(size_t)iw * cw];
    T* lsw = &Lsfw[(size_t)iw * cw];
    T* lul = &Lupw_low[(size_t)iw * cw];
    for (int k = kb; k <= mza; ++k) {
      const size_t x = (size_t)(iw - 1) * mza + k - 1;
      const T lo = Lfout[x], lf = Lfl[x];
      for (int jv = 1; jv <= G.npoly(iw); ++jv) {
        const int iv = G.w_iv(iw, jv);
        if (k < G.lpv(iv)) continue;
        const T d = G.w_dirv(iw, jv);
        if (d * F2(R.sfv.data(), k, iv) < (T)0) F2(Lsfv.data(), k, iv) += d * lo;
        const T a = lf * d * F2(vm, k, iv);
        F2(Lupv_low.data(), k, iv) += a;
        F2(L0p, k, iw) -= a;
      }
      if (sfw[k - 1] < (T)0) lsw[k - 1] += lo;
      if (sfw[k] > (T)0) lsw[k] -= lo;
      lul[k - 1] += lf * fe * F2(wm, k - 1, iw);
      lul[k] -= lf * fe * F2(wm, k, iw);
      F2(L0p, k, iw) -= lf * fe * (F2(wm, k - 1, iw) - F2(wm, k, iw));
      if (imp) F2(L0p, k, iw) += lf * fimpl * (F2(wm, k, iw) - F2(wm, k - 1, iw));
    }
  }
  // sfw = fexpl wm hiw; hiw = (scpb(k+1) or scpt(k)) - upw_low; upw_low from s0
  // (interior faces) or S (the boundary faces); scpb / scpt of grad_z_quadratic(S)
  for (int j = 0; j < G.g->nw_prog; ++j) {
    const int iw = G.g->jtw_prog[j], kb = G.lpw(iw);
    const T fexpl = (T)1. - C.ff(istage, iw);
    T* lsw = &Lsfw[(size_t)iw * cw];
    T* lhw = &Lhiw[(size_t)iw * cw];
    T* lul = &Lupw_low[(size_t)iw * cw];
    std::vector<T> Lb(mza + 1, (T)0), Lt(mza + 1, (T)0), Lds(mza + 1, (T)0);
    for (int k = kb; k <= mza - 1; ++k) {
      lhw[k] += fexpl * F2(wm, k, iw) * lsw[k];
      if (F2(wm, k, iw) < (T)0) Lb[k + 1] += lhw[k];
      else Lt[k] += lhw[k];
      lul[k] -= lhw[k];
      if (F2(wm, k, iw) < (T)0) F2(L0p, k + 1, iw) += lul[k];
      else F2(L0p, k, iw) += lul[k];
    }
    F2(Lin, kb, iw) += lul[kb - 1];
    F2(Lin, mza, iw) += lul[mza];
    for (int k = kb; k <= mza; ++k) {
      F2(Lin, k, iw) += Lb[k] + Lt[k];
      Lds[k] += Lb[k] * G.aw(G.a_w, k, 1, 1) + Lt[k] * G.aw(G.a_w, k, 1, 2);
      Lds[k - 1] += Lb[k] * G.aw(G.a_w, k, 2, 1) + Lt[k] * G.aw(G.a_w, k, 2, 2);
    }
    for (int k = kb; k <= mza - 1; ++k) {
      F2(Lin, k + 1, iw) += Lds[k];
      F2(Lin, k, iw) -= Lds[k];
    }
  }
  // faces: sfluxvh = vm hiv; hiv = side value(upwind side) - s0(upwind cell); upv_low = s0(upwind cell)
  for (int j = 0; j < G.g->nv_wadj; ++j) {
    const int iv = G.g->jtv_wadj[j];
    for (int k = G.lpv(iv); k <= mza; ++k) {
      const T vmk = F2(vm, k, iv);
      const int s = vmk < (T)0 ? 2 : 1;
      const int iws = G.v_iw(iv, s);
      const T lh = F2(Lhiv.data(), k, iv) + vmk * F2(Lsfv.data(), k, iv);
      F2(L0p, k, iws) += F2(Lupv_low.data(), k, iv) - lh;
      if (lh == (T)0) continue;
      const size_t x = (size_t)(iws - 1) * mza + k - 1;
      Lin[x] += lh;
      if (iorderh == 1) continue;
      Lg[x] += G.v2(G.dxps, s, iv) * lh;
      Lg[plane + x] += G.v2(G.dyps, s, iv) * lh;
      if (iorderh == 3) {
        Lg[2 * plane + x] += G.v2(G.xx0_v, s, iv) * lh;
        Lg[3 * plane + x] += G.v2(G.xy0_v, s, iv) * lh;
        Lg[4 * plane + x] += G.v2(G.yy0_v, s, iv) * lh;
      }
    }
  }
  // grad_t2d[_quadratic] of S
  if (iorderh > 1)
    for (int j = 0; j < G.g->nw_prog; ++j) {
      const int iw = G.g->jtw_prog[j];
      for (int nn = 1; nn <= G.npoly(iw); ++nn) {
        const int iwn = G.w_iw(iw, nn), ivn = G.w_iv(iw, nn);
        T c[5];
        if (iorderh == 2) { c[0] = G.gxps_coef(nn, iw); c[1] = G.gyps_coef(nn, iw); }
        else for (int m = 0; m < 5; ++m) c[m] = G.xyh(G.xy_h, m + 1, nn, iw);
        for (int k = G.lpv(ivn); k <= mza; ++k) {
          const size_t x = (size_t)(iw - 1) * mza + k - 1;
          T t = 0;
          for (int m = 0; m < np2d; ++m) t += c[m] * Lg[m * plane + x];
          F2(Lin, k, iwn) += t;
          Lin[x] -= t;
        }
      }
    }
}

/* Adjoint of scalar_transport_rk for one long step with the winds and
 * densities fixed and no limiter (iscal_monot = 0, no horizontal diffusion):
 * the step maps (scp, sct) linearly to the new scp, and this applies the
 * transpose.  lam holds dJ/d(new scp) on entry and dJ/d(old scp) on exit;
 * lsct receives dJ/d(sct).  Each forward pass -- grad_t2d[_quadratic],
 * scalar_v_column, grad_z_quadratic, scalar_w_column, tridif_fini -- is
 * transposed in reverse order, stage by stage. */
template <class T>
static int scalar_transport_rk_adjoint(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                       T* const* lam_list, T* const* lsct_list, const float* vmasc_f,
                                       const float* wmasc_f, const double* rho, const float* rho_old_f,
                                       const float* wc, const T* const* scp_fwd = nullptr,
                                       const T* const* sct_fwd = nullptr, const int* pdef = nullptr) {
  if (o->iscal_monot == 1) return OLAMGPU_E_UNSUPPORTED;
  if (o->iscal_monot == 2 && pdef && (!scp_fwd || !sct_fwd))
    for (int n = 0; n < nscal; ++n)
      if (pdef[n]) return OLAMGPU_E_ARG;   // the limited stage needs the forward's inputs
  GridT<T> G(g);
  const int mza = g->mza, mwa = g->mwa, mva = g->mva;
  const int iorder = o->scal_horiz_adv_order;
  if (iorder != 2 && iorder != 3) return OLAMGPU_E_UNSUPPORTED;
  StepCoef<T> SC;
  int rc = prepare_step(G, g, o, vmasc_f, wmasc_f, rho, rho_old_f, wc, nullptr, nullptr, SC);
  if (rc != OLAMGPU_OK) return rc;
  const int nrk = SC.nrk;
  const size_t plane = (size_t)mza * mwa;
  const int np2d = iorder == 2 ? 2 : 5;
  const T* vm = SC.vmasc.data();
  const T* wm = SC.wmasc.data();
  const T* rhos_nrk = SC.rhos.data() + (size_t)(nrk - 1) * plane;
  std::vector<char> prog(mwa + 1, 0);
  for (int j = 0; j < g->nw_prog; ++j) prog[g->jtw_prog[j]] = 1;
  TransportCtx<T> C{G, mza, mwa, mva, SC.vmasc, SC.wmasc, SC.ff_implic, nrk};

  for (int n = 0; n < nscal; ++n) {
    T* lam = lam_list[n];
    T* ls = lsct_list[n];
    std::fill(ls, ls + plane, (T)0);
    // positive-definite last stage: recompute the forward to it and record
    // the stage's intermediates (its input, scp0' and the limiter's branches)
    const bool pdn = o->iscal_monot == 2 && pdef && pdef[n];
    PdRecord<T> R;
    std::vector<T> S0p, Lp;
    if (pdn) {
      std::vector<T> sf(scp_fwd[n], scp_fwd[n] + plane), s0(sf), st(sct_fwd[n], sct_fwd[n] + plane);
      for (int istage = 1; istage < nrk; ++istage) {
        update_scalar(C, sf.data(), s0.data(), st.data(), rhos_nrk, SC.dtlr[istage - 1], iorder, istage);
        implicit_step(G, SC, istage, SC.dtlr[istage - 1], sf.data(), s0.data());
      }
      S0p = s0;
      const T dtr = SC.dtlr[nrk - 1];
      for (int j = 0; j < g->nw_wadj; ++j) {
        const int iw = g->jtw_wadj[j], kb = G.lpw(iw);
        for (int k = kb; k <= mza; ++k)
          F2(S0p.data(), k, iw) = F2(S0p.data(), k, iw) + dtr * F2(st.data(), k, iw) / F2(SC.rho_old.data(), k, iw);
        for (int k = 2; k <= kb - 1; ++k) F2(S0p.data(), k, iw) = F2(S0p.data(), kb, iw);
      }
      pd_record(C, sf.data(), S0p.data(), rhos_nrk, dtr, iorder, nrk, R);
      Lp.assign(plane, (T)0);
    }
    std::vector<T> L(lam, lam + plane), L0(plane, (T)0), Lin(plane), Lupv((size_t)mza * mva),
        Lg(plane * np2d);
    // columns outside jtw_prog keep their values through the step
    for (int iw = 1; iw <= mwa; ++iw)
      if (!prog[iw])
        for (int k = 1; k <= mza; ++k) { F2(L0.data(), k, iw) += F2(L.data(), k, iw); F2(L.data(), k, iw) = 0; }

    for (int istage = nrk; istage >= 1; --istage) {
      const T dtr = SC.dtlr[istage - 1];
      const bool pd_stage = pdn && istage == nrk;
      // the stage's s0: scp0, or scp0' on the positive-definite stage
      T* L0s = pd_stage ? Lp.data() : L0.data();
      // ---- implicit columns: out' = s0 + T^-1 (out - s0 - G s0)
      auto& I = SC.imp[istage - 1];
      for (size_t jj = 0; jj < I.iw.size(); ++jj) {
        const int iw = I.iw[jj], kb = G.lpw(iw);
        const T* cim1 = &I.b1[jj * (mza + 1)];
        const T* scr1 = &I.b2[jj * (mza + 1)];
        const T* cji = &I.b3[jj * (mza + 1)];
        for (int k = 2; k <= kb - 1; ++k) { F2(L.data(), kb, iw) += F2(L.data(), k, iw); F2(L.data(), k, iw) = 0; }
        // T = L U with L(k,k) = 1/cji(k), L(k,k-1) = cim1(k), U(k,k+1) = scr1(k+1):
        // nu = T^-T lam: U^T z = lam (forward), then L^T nu = z (backward)
        std::vector<T> z(mza + 2, (T)0), nu(mza + 2, (T)0);
        for (int k = kb; k <= mza; ++k) z[k] = F2(L.data(), k, iw) - (k > kb ? scr1[k] * z[k - 1] : (T)0);
        for (int k = mza; k >= kb; --k) nu[k] = cji[k] * (z[k] - (k < mza ? cim1[k + 1] * nu[k + 1] : (T)0));
        const T ffv = SC.ff_implic[(size_t)(iw - 1) * nrk + istage - 1];
        for (int k = kb; k <= mza; ++k) {
          F2(L0s, k, iw) += F2(L.data(), k, iw) - nu[k];
          const T c1 = ffv * dtr * G.volti_(k, iw) / SC.rhos[(size_t)(istage - 1) * plane + (size_t)(iw - 1) * mza + k - 1];
          const T gk = -c1 * nu[k];
          if (k <= mza - 1) {   // min(wmasc(k),0) * (s0(k+1) - s0(k))
            const T a = fmin_(F2(wm, k, iw), (T)0.) * gk;
            F2(L0s, k + 1, iw) += a; F2(L0s, k, iw) -= a;
          }
          if (k - 1 >= kb) {    // max(wmasc(k-1),0) * (s0(k) - s0(k-1))
            const T a = fmax_(F2(wm, k - 1, iw), (T)0.) * gk;
            F2(L0s, k, iw) += a; F2(L0s, k - 1, iw) -= a;
          }
          F2(L.data(), k, iw) = nu[k];
        }
      }
      // ---- explicit update_scalar: out = s0 + dtr (sct + volti fluxdiv(s_in, s0)) / rhos
      std::fill(Lin.begin(), Lin.end(), (T)0);
      std::fill(Lupv.begin(), Lupv.end(), (T)0);
      std::fill(Lg.begin(), Lg.end(), (T)0);
      if (pd_stage) {
        for (int j = 0; j < g->nw_prog; ++j) {
          const int iw = g->jtw_prog[j], kb = G.lpw(iw);
          for (int k = 1; k <= kb - 1; ++k) { F2(L.data(), kb, iw) += F2(L.data(), k, iw); F2(L.data(), k, iw) = 0; }
        }
        pd_stage_adjoint(C, R, S0p.data(), rhos_nrk, dtr, iorder, nrk, L.data(), Lin.data(), Lp.data());
        // scp0' = scp0 + dtr sct / rho_old from lpw up
        for (int j = 0; j < g->nw_prog; ++j) {
          const int iw = g->jtw_prog[j], kb = G.lpw(iw);
          for (int k = kb; k <= mza; ++k) {
            F2(L0.data(), k, iw) += F2(Lp.data(), k, iw);
            F2(ls, k, iw) += F2(Lp.data(), k, iw) * dtr / F2(SC.rho_old.data(), k, iw);
          }
        }
        L.swap(Lin);
        continue;
      }
      for (int j = 0; j < g->nw_prog; ++j) {
        const int iw = g->jtw_prog[j], kb = G.lpw(iw);
        const T fexpl = (T)1.0 - SC.ff_implic[(size_t)(iw - 1) * nrk + istage - 1];
        for (int k = 1; k <= kb - 1; ++k) { F2(L.data(), kb, iw) += F2(L.data(), k, iw); F2(L.data(), k, iw) = 0; }
        std::vector<T> mu(mza + 1, (T)0), Lupw(mza + 1, (T)0), Lb(mza + 1, (T)0), Lt(mza + 1, (T)0), Lds(mza + 1, (T)0);
        for (int k = kb; k <= mza; ++k) {
          const T lk = F2(L.data(), k, iw);
          const T r = dtr / F2(rhos_nrk, k, iw);
          F2(ls, k, iw) += lk * r;
          F2(L0.data(), k, iw) += lk;
          mu[k] = lk * r * G.volti_(k, iw);
          // the vertical flux: fexpl (wm(k-1) (upw(k-1) - s0) - wm(k) (upw(k) - s0))
          F2(L0.data(), k, iw) -= mu[k] * fexpl * (F2(wm, k - 1, iw) - F2(wm, k, iw));
          Lupw[k - 1] += mu[k] * fexpl * F2(wm, k - 1, iw);
          Lupw[k] -= mu[k] * fexpl * F2(wm, k, iw);
        }
        // the horizontal flux: sum_v dirv vmasc (upv - s0)
        for (int jv = 1; jv <= G.npoly(iw); ++jv) {
          const int iv = G.w_iv(iw, jv);
          const T d = G.w_dirv(iw, jv);
          for (int k = G.lpv(iv); k <= mza; ++k) {
            const T a = mu[k] * d * F2(vm, k, iv);
            F2(Lupv.data(), k, iv) += a;
            F2(L0.data(), k, iw) -= a;
          }
        }
        // scp_upw: boundary faces take the column's end values, the others the
        // upwind level's quadratic face value (grad_z_quadratic, bounded)
        F2(Lin.data(), kb, iw) += Lupw[kb - 1];
        F2(Lin.data(), mza, iw) += Lupw[mza];
        for (int k = kb; k <= mza - 1; ++k) {
          if (F2(wm, k, iw) < (T)0) Lb[k + 1] += Lupw[k];
          else Lt[k] += Lupw[k];
        }
        for (int k = kb; k <= mza; ++k) {
          F2(Lin.data(), k, iw) += Lb[k] + Lt[k];
          Lds[k] += Lb[k] * G.aw(G.a_w, k, 1, 1) + Lt[k] * G.aw(G.a_w, k, 1, 2);
          Lds[k - 1] += Lb[k] * G.aw(G.a_w, k, 2, 1) + Lt[k] * G.aw(G.a_w, k, 2, 2);
        }
        for (int k = kb; k <= mza - 1; ++k) {   // ds(k) = s(k+1) - s(k)
          F2(Lin.data(), k + 1, iw) += Lds[k];
          F2(Lin.data(), k, iw) -= Lds[k];
        }
      }
      // scalar_v_column: upv = side value of the upwind side
      const std::vector<T>& xx = G.xx0_v;
      const std::vector<T>& xy = G.xy0_v;
      const std::vector<T>& yy = G.yy0_v;
      for (int j = 0; j < g->nv_wadj; ++j) {
        const int iv = g->jtv_wadj[j];
        for (int k = G.lpv(iv); k <= mza; ++k) {
          const T a = F2(Lupv.data(), k, iv);
          if (a == (T)0) continue;
          const int s = F2(vm, k, iv) < (T)0 ? 2 : 1;
          const int iws = G.v_iw(iv, s);
          const size_t x = (size_t)(iws - 1) * mza + k - 1;
          Lin[x] += a;
          Lg[x] += G.v2(G.dxps, s, iv) * a;
          Lg[plane + x] += G.v2(G.dyps, s, iv) * a;
          if (iorder == 3) {
            Lg[2 * plane + x] += G.v2(xx, s, iv) * a;
            Lg[3 * plane + x] += G.v2(xy, s, iv) * a;
            Lg[4 * plane + x] += G.v2(yy, s, iv) * a;
          }
        }
      }
      // grad_t2d[_quadratic]: g_m(iw) = sum_n c_m(n) (s(iwn) - s(iw))
      for (int j = 0; j < g->nw_prog; ++j) {
        const int iw = g->jtw_prog[j];
        for (int nn = 1; nn <= G.npoly(iw); ++nn) {
          const int iwn = G.w_iw(iw, nn), ivn = G.w_iv(iw, nn);
          T c[5];
          if (iorder == 2) { c[0] = G.gxps_coef(nn, iw); c[1] = G.gyps_coef(nn, iw); }
          else for (int m = 0; m < 5; ++m) c[m] = G.xyh(G.xy_h, m + 1, nn, iw);
          for (int k = G.lpv(ivn); k <= mza; ++k) {
            const size_t x = (size_t)(iw - 1) * mza + k - 1;
            T t = 0;
            for (int m = 0; m < np2d; ++m) t += c[m] * Lg[m * plane + x];
            F2(Lin.data(), k, iwn) += t;
            Lin[x] -= t;
          }
        }
      }
      L.swap(Lin);   // the adjoint of this stage's input, the previous stage's output
    }
    for (size_t i = 0; i < plane; ++i) lam[i] = L[i] + L0[i];
  }
  return OLAMGPU_OK;
}

}  // namespace oracle

extern "C" {

int oracle_scalar_transport_rk_f32(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                   float* const* scp, float* const* sct, const int* pdef,
                                   const int* sgsmix, const float* vmasc, const float* wmasc,
                                   const double* rho, const float* rho_old, const float* wc,
                                   const float* akhodx, const int* khtopv, float* ff_out,
                                   olamgpu_cfl_diag* diag) {
  return oracle::scalar_transport_rk<float>(g, o, nscal, scp, sct, pdef, sgsmix, vmasc, wmasc, rho,
                                            rho_old, wc, akhodx, khtopv, ff_out, diag);
}

int oracle_scalar_transport_rk_f64(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                   double* const* scp, double* const* sct, const int* pdef,
                                   const int* sgsmix, const float* vmasc, const float* wmasc,
                                   const double* rho, const float* rho_old, const float* wc,
                                   const float* akhodx, const int* khtopv, float* ff_out,
                                   olamgpu_cfl_diag* diag) {
  return oracle::scalar_transport_rk<double>(g, o, nscal, scp, sct, pdef, sgsmix, vmasc, wmasc, rho,
                                             rho_old, wc, akhodx, khtopv, ff_out, diag);
}

}

extern "C" {

int oracle_scalar_transport_rk_adjoint_f32(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                           float* const* lam, float* const* lsct, const float* vmasc,
                                           const float* wmasc, const double* rho, const float* rho_old,
                                           const float* wc) {
  return oracle::scalar_transport_rk_adjoint<float>(g, o, nscal, lam, lsct, vmasc, wmasc, rho, rho_old, wc);
}

int oracle_scalar_transport_rk_adjoint_f64(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                           double* const* lam, double* const* lsct, const float* vmasc,
                                           const float* wmasc, const double* rho, const float* rho_old,
                                           const float* wc) {
  return oracle::scalar_transport_rk_adjoint<double>(g, o, nscal, lam, lsct, vmasc, wmasc, rho, rho_old, wc);
}

/* The adjoint with the positive-definite limiter (iscal_monot = 2): the
 * forward step's inputs scp_fwd / sct_fwd and the pdef flags select and
 * reconstruct the limited last stage of every pdef tracer. */
int oracle_scalar_transport_rk_adjoint_pd_f32(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                              const float* const* scp_fwd, const float* const* sct_fwd,
                                              const int* pdef, float* const* lam, float* const* lsct,
                                              const float* vmasc, const float* wmasc, const double* rho,
                                              const float* rho_old, const float* wc) {
  return oracle::scalar_transport_rk_adjoint<float>(g, o, nscal, lam, lsct, vmasc, wmasc, rho, rho_old, wc, scp_fwd,
                                                    sct_fwd, pdef);
}

int oracle_scalar_transport_rk_adjoint_pd_f64(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                              const double* const* scp_fwd, const double* const* sct_fwd,
                                              const int* pdef, double* const* lam, double* const* lsct,
                                              const float* vmasc, const float* wmasc, const double* rho,
                                              const float* rho_old, const float* wc) {
  return oracle::scalar_transport_rk_adjoint<double>(g, o, nscal, lam, lsct, vmasc, wmasc, rho, rho_old, wc,
                                                     scp_fwd, sct_fwd, pdef);
}

}

extern "C" {

/* Tangent-linear of one scalar_transport_rk step in FP64: the step of
 * oracle_scalar_transport_rk_f64 on scp / sct (new scp returned in scp), and
 * in dscp its exact directional derivative along (dscp, dsct) -- the
 * Jacobian-vector product of the step, limiters included, with the winds
 * and densities fixed.  No horizontal diffusion. */
int oracle_scalar_transport_rk_tl_f64(const olamgpu_grid* g, const olamgpu_opts* o, int nscal,
                                      double* const* scp, double* const* dscp, double* const* sct,
                                      double* const* dsct, const int* pdef, const float* vmasc,
                                      const float* wmasc, const double* rho, const float* rho_old,
                                      const float* wc) {
  const size_t plane = (size_t)g->mza * g->mwa;
  std::vector<std::vector<oracle::Dual>> s(nscal), t(nscal);
  std::vector<oracle::Dual*> sp(nscal), tp(nscal);
  for (int n = 0; n < nscal; ++n) {
    s[n].resize(plane);
    t[n].resize(plane);
    for (size_t i = 0; i < plane; ++i) {
      s[n][i] = oracle::Dual(scp[n][i], dscp[n][i]);
      t[n][i] = oracle::Dual(sct[n][i], dsct[n][i]);
    }
    sp[n] = s[n].data();
    tp[n] = t[n].data();
  }
  const int rc = oracle::scalar_transport_rk<oracle::Dual>(g, o, nscal, sp.data(), tp.data(), pdef, nullptr, vmasc,
                                                          wmasc, rho, rho_old, wc, nullptr, nullptr, nullptr,
                                                          nullptr);
  for (int n = 0; n < nscal; ++n)
    for (size_t i = 0; i < plane; ++i) {
      scp[n][i] = s[n][i].v;
      dscp[n][i] = s[n][i].d;
    }
  return rc;
}

}
