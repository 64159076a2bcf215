/*
 * oracle_dynamics.cpp -- TEST INFRASTRUCTURE ONLY (see oracle_common.h).
 * PARITY UNPINNED (no Fortran compiler, no reference golden vectors).
 *
 * CPU restatement of the acoustic RK short step and its glue:
 *   init_wrtv_rk           omodel/prog_wrtv_rk.f90:36-54
 *   prog_wrtv_rk           omodel/prog_wrtv_rk.f90:58-488
 *   prog_wrt_begs          omodel/prog_wrtv_rk.f90:494-884
 *   prog_v_begs            omodel/prog_wrtv_rk.f90:888-946
 *   fluxes_wrtv            omodel/prog_wrtv_rk.f90:950-1129
 *   eddy diffusion         convect/pbl_driver.f90:136-238 (comp_horiz_k),
 *                          519-742 (solve_eddy_diff_heat / _vxe),
 *                          modules/mem_rayf.f90:177-220 (rayf_mix_top_vxe),
 *                          outils/tridiag_lib.f90:40-104 (tridv),
 *                          omodel/prog_wrtv_rk.f90:214-251 (their calls)
 *   fluxes_wrtv_monot      omodel/prog_wrtv_rk.f90:1133-1554 (with
 *                          scalar_wflux_monot, scalar_vflux_monot and
 *                          scalar_monot_limiter; centered_monot = .false.,
 *                          iorderv = 3)
 *   vel_t3d_hex            omodel/vel_t3d.f90:39-108
 *   update_vxe_undrgnd     omodel/prog_wrtv_rk.f90:1558-1595 (shaved cells,
 *                          with the start values of :202-211)
 *   divh_damp, vort_damp   omodel/vort_div_damp.f90:1-445
 *   laplacian2d/_m         omodel/grad_lib.f90:494-559
 *   tridiffo               outils/tridiag_lib.f90:10-36
 *   tend0, timeavg_momsc   omodel/timestep.f90:430-496, 563-612
 * Precision as declared: rho, press, rth0, rho0, hflx_rho, delex_rho,
 * delex_rhothil, rhothil, vflux_thil, press_ex, rho_ex, b5, b10 and the
 * implicit weights fr/fp2/fp3/pc2/pc3 are real(8); everything else is T.
 * Real literals that OLAM writes in default precision (e.g. fr = .70) keep
 * their single-precision value when promoted to real(8).
 * Not restated (off in every configuration this build runs): nudging,
 * the supercell test's thil_init offset, Lagrangian
 * particle sums, the shallow-water test cases.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>

#include "oracle_common.h"

namespace oracle {

typedef double R8;

template <class T>
struct DynState {
  R8 *rho, *press;
  T *thil, *wc, *wmc, *vxe, *vye, *vze, *vmc, *vc, *vmasc, *wmasc, *alpha_press, *pwfac, *pvfac;
  T *thilt, *vmxet, *vmyet, *vmzet, *vmt;
};

template <class T>
struct DynCtx {
  const olamgpu_grid* g;
  olamgpu_opts o;
  GridT<T> G;
  int mza, mwa, mva, mma;
  std::vector<T> arv, arw, volwi, volvi, wnx, wny, wnz, wnxo2, wnyo2, wnzo2, vnx, vny, vnz;
  std::vector<T> ecx, ecy, ecz, gdz_wgtm, gdz_wgtp, dniv, dniu, dnv, arw0, arm0, zfacit, dzit;
  std::vector<T> xx_yy, xx_yy_m, b20;
  // divh_damp saved state (vort_div_damp.f90:22-27)
  bool div_first = true;
  std::vector<T> div2d, fdivh;
  // vort_damp saved state (:263-268)
  bool vort_first = true;
  std::vector<T> vort2d, fvorth, fvortl, vfact;
  std::vector<int> lpmmin;
  // eddy diffusion (olamgpu_eddy host arrays; NULL: off) and comp_horiz_k's
  // outputs when the oracle computed them
  const olamgpu_eddy* eddy = nullptr;
  bool have_hk = false;
  std::vector<T> akmodx, akhodx;
  std::vector<int> kmtopv, khtopv;
  explicit DynCtx(const olamgpu_grid* gr, const olamgpu_opts* op) : g(gr), o(*op), G(gr) {
    mza = g->mza; mwa = g->mwa; mva = g->mva; mma = g->mma;
    arv = cvt<T>(g->arv, (size_t)mza * mva);
    arw = cvt<T>(g->arw, (size_t)mza * mwa);
    volwi = cvt<T>(g->volwi, (size_t)mza * mwa);
    volvi = cvt<T>(g->volvi, (size_t)mza * mva);
    wnx = cvt<T>(g->wnx, mwa); wny = cvt<T>(g->wny, mwa); wnz = cvt<T>(g->wnz, mwa);
    wnxo2 = cvt<T>(g->wnxo2, mwa); wnyo2 = cvt<T>(g->wnyo2, mwa); wnzo2 = cvt<T>(g->wnzo2, mwa);
    vnx = cvt<T>(g->vnx, mva); vny = cvt<T>(g->vny, mva); vnz = cvt<T>(g->vnz, mva);
    ecx = cvt<T>(g->ecvec_vx, (size_t)7 * mwa);
    ecy = cvt<T>(g->ecvec_vy, (size_t)7 * mwa);
    ecz = cvt<T>(g->ecvec_vz, (size_t)7 * mwa);
    gdz_wgtm = cvt<T>(g->gdz_wgtm, mza); gdz_wgtp = cvt<T>(g->gdz_wgtp, mza);
    dniv = cvt<T>(g->dniv, mva); dniu = cvt<T>(g->dniu, mva); dnv = cvt<T>(g->dnv, mva);
    arw0 = cvt<T>(g->arw0, mwa); arm0 = cvt<T>(g->arm0, mma);
    zfacit = cvt<T>(g->zfacit, mza); dzit = cvt<T>(g->dzit, mza);
    xx_yy = cvt<T>(g->xx_yy, (size_t)7 * mwa);
    xx_yy_m = cvt<T>(g->xx_yy_m, (size_t)3 * mma);
    // init_wrtv_rk (prog_wrtv_rk.f90:36-54)
    b20.assign(mza + 1, (T)1.0);
    if (o.rayf_cofw)
      for (int k = o.krayfw_bot; k <= mza - 1; ++k) b20[k] = (T)1.0 + (T)(float)o.dtsm * (T)o.rayf_cofw[k - 1];
  }
  int m_iv(int im, int j) const { return g->itab_m_iv[(size_t)(im - 1) * 3 + (j - 1)]; }
  int m_iw(int im, int j) const { return g->itab_m_iw[(size_t)(im - 1) * 3 + (j - 1)]; }
  int m_im(int im, int j) const { return g->itab_m_im[(size_t)(im - 1) * 3 + (j - 1)]; }
  int lpm(int im) const { return g->lpm[im - 1]; }
};

/* tridiffo (tridiag_lib.f90:10-36); arrays indexed by k */
template <class T>
static void tridiffo(int ka, int kz, const T* cim1, const T* ci, const T* cip1, const T* rhs, T* soln) {
  std::vector<T> scr1(kz + 2);
  T cji = (T)1.0 / ci[ka];
  soln[ka] = rhs[ka] * cji;
  for (int k = ka + 1; k <= kz; ++k) {
    scr1[k] = cji * cip1[k - 1];
    cji = (T)1.0 / (ci[k] - cim1[k] * scr1[k]);
    soln[k] = cji * (rhs[k] - cim1[k] * soln[k - 1]);
  }
  for (int k = kz - 1; k >= ka; --k) soln[k] = soln[k] - scr1[k + 1] * soln[k + 1];
}

/* laplacian2d (grad_lib.f90:494-524): delsq column [k-1] */
template <class T>
static void laplacian2d(const DynCtx<T>& X, int iw, const T* scp, T* delsq) {
  const int mza = X.mza;
  for (int k = 1; k <= mza; ++k) delsq[k - 1] = 0;
  for (int n = 1; n <= X.G.npoly(iw); ++n) {
    int iwn = X.G.w_iw(iw, n), ivn = X.G.w_iv(iw, n);
    T c = X.xx_yy[(size_t)(iw - 1) * 7 + n - 1];
    for (int k = X.G.lpv(ivn); k <= mza; ++k) {
      T sc = F2(scp, k, iwn) - F2(scp, k, iw);
      delsq[k - 1] = delsq[k - 1] + sc * c;
    }
  }
}

/* laplacian_m (grad_lib.f90:531-559) */
template <class T>
static void laplacian_m(const DynCtx<T>& X, int im, const T* scm, T* delsq) {
  const int mza = X.mza;
  for (int k = 1; k <= mza; ++k) delsq[k - 1] = 0;
  for (int j = 1; j <= 3; ++j) {
    int imn = X.m_im(im, j);
    T c = X.xx_yy_m[(size_t)(im - 1) * 3 + j - 1];
    for (int k = X.G.lpv(X.m_iv(im, j)); k <= mza; ++k) {
      T sc = F2(scm, k, imn) - F2(scm, k, im);
      delsq[k - 1] = delsq[k - 1] + sc * c;
    }
  }
}

/* divh_damp (vort_div_damp.f90:1-230) for divh_damp_level > 1 without
 * Rayleigh divergence damping.  The saved div2d is not cleared between
 * calls: plane 1 accumulates onto the value the previous call left there
 * (the last Laplacian output), exactly as the Fortran does. */
template <class T>
static void divh_damp(DynCtx<T>& X, const DynState<T>& s, T* vmt, R8 dtm) {
  const int mza = X.mza, mwa = X.mwa;
  const olamgpu_opts& o = X.o;
  bool dodiv = (o.divh_damp_fact > 1.e-7f) && (o.divh_damp_level > 0);
  if (!dodiv) return;
  const int level = o.divh_damp_level;
  const size_t plane = (size_t)mza * mwa;
  if (X.div_first) {
    X.div_first = false;
    int ilev = level > 1 ? 2 : 1;
    X.div2d.assign(plane * ilev, (T)0);
    if (level > 1) {
      // facth = -(-fact)**level / dtm: the power is in default real
      T p = (T)1;
      for (int i = 0; i < level; ++i) p = p * (T)(-o.divh_damp_fact);
      R8 facth = -((R8)p / dtm);
      X.fdivh.assign((size_t)mza * X.mva, (T)0);
      for (int j = 0; j < X.g->nv_prog; ++j) {
        int iv = X.g->jtv_prog[j];
        int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2);
        T amin = std::min(X.arw0[iw1 - 1], X.arw0[iw2 - 1]);
        T pw = (T)1;
        for (int i = 0; i < level - 1; ++i) pw = pw * amin;
        R8 factb = facth * (R8)pw;
        for (int k = X.G.lpv(iv); k <= mza; ++k) {
          R8 vmin = std::min(F2(X.g->volt, k, iw1), F2(X.g->volt, k, iw2));
          R8 v = factb * (R8)X.dniv[iv - 1] * (R8)X.zfacit[k - 1] * (R8)X.dzit[k - 1] * vmin *
                 (R8)((T)1. - (T)0.);
          X.fdivh[(size_t)(iv - 1) * mza + k - 1] = (T)v;
        }
      }
    } else {
      // level 1: fdivl = fact2 * dniv * zfacit * dzit * min(volt) with fact2 = fact/dtm
      X.fdivh.assign((size_t)mza * X.mva, (T)0);
      T fact2 = (T)o.divh_damp_fact / (T)dtm;
      for (int j = 0; j < X.g->nv_prog; ++j) {
        int iv = X.g->jtv_prog[j];
        int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2);
        for (int k = X.G.lpv(iv); k <= mza; ++k) {
          R8 vmin = std::min(F2(X.g->volt, k, iw1), F2(X.g->volt, k, iw2));
          R8 v = (R8)(fact2 * ((T)1. - (T)0.) + (T)0. * (T)0.) * (R8)X.dniv[iv - 1] *
                 (R8)X.zfacit[k - 1] * (R8)X.dzit[k - 1] * vmin;
          X.fdivh[(size_t)(iv - 1) * mza + k - 1] = (T)v;
        }
      }
    }
  }
  T* d1 = X.div2d.data();
  // horizontal divergence (:133-158)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    int iw = X.g->jtw_prog[j];
    for (int jv = 1; jv <= X.G.npoly(iw); ++jv) {
      int iv = X.G.w_iv(iw, jv);
      T dv = X.G.w_dirv(iw, jv);
      for (int k = X.G.lpv(iv); k <= mza; ++k)
        F2(d1, k, iw) = F2(d1, k, iw) - F2(X.arv.data(), k, iv) * dv * F2(s.vmc, k, iv);
    }
    for (int k = X.G.lpw(iw); k <= mza; ++k) F2(d1, k, iw) = F2(d1, k, iw) * X.G.volti_(k, iw);
  }
  if (level == 1) {
    for (int j = 0; j < X.g->nv_prog; ++j) {
      int iv = X.g->jtv_prog[j];
      int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2);
      for (int k = X.G.lpv(iv); k <= mza; ++k)
        F2(vmt, k, iv) = F2(vmt, k, iv) + F2(X.fdivh.data(), k, iv) * (F2(d1, k, iw2) - F2(d1, k, iw1));
    }
    return;
  }
  int il = 1, ih = 2;
  for (int nn = 1; nn <= level - 1; ++nn) {
    il = (nn - 1) % 2 + 1;
    ih = nn % 2 + 1;
    T* src = X.div2d.data() + (size_t)(il - 1) * plane;
    T* dst = X.div2d.data() + (size_t)(ih - 1) * plane;
    for (int j = 0; j < X.g->nw_prog; ++j) {
      int iw = X.g->jtw_prog[j];
      laplacian2d(X, iw, src, dst + (size_t)(iw - 1) * mza);
    }
  }
  T* dh = X.div2d.data() + (size_t)(ih - 1) * plane;
  for (int j = 0; j < X.g->nv_prog; ++j) {
    int iv = X.g->jtv_prog[j];
    int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2);
    for (int k = X.G.lpv(iv); k <= mza; ++k)
      F2(vmt, k, iv) = F2(vmt, k, iv) + F2(X.fdivh.data(), k, iv) * (F2(dh, k, iw2) - F2(dh, k, iw1));
  }
}

/* vort_damp (vort_div_damp.f90:234-445), flat terrain (lpmmin == lpm) */
template <class T>
static void vort_damp(DynCtx<T>& X, const DynState<T>& s, T* vmt, R8 dtm) {
  const int mza = X.mza, mma = X.mma;
  const olamgpu_opts& o = X.o;
  if (o.vort_damp_fact < 1.e-7f || o.vort_damp_level <= 0) return;
  const int level = o.vort_damp_level;
  const size_t plane = (size_t)mza * mma;
  if (X.vort_first) {
    X.vort_first = false;
    X.fvorth.assign(X.mva + 1, (T)0);
    X.fvortl.assign(X.mva + 1, (T)0);
    X.vfact.assign((size_t)3 * mma, (T)0);
    X.lpmmin.assign(mma + 1, 0);
    X.vort2d.assign(plane * (level == 1 ? 1 : 2), (T)0);
    for (int j = 0; j < X.g->nm_prog; ++j) {
      int im = X.g->jtm_prog[j];
      int lm = 1 << 30;
      for (int jv = 1; jv <= 3; ++jv) lm = std::min(lm, X.G.lpv(X.m_iv(im, jv)));
      X.lpmmin[im] = lm;
      for (int jv = 1; jv <= 3; ++jv) {
        int iv = X.m_iv(im, jv);
        T v = X.dnv[iv - 1] / X.arm0[im - 1];
        X.vfact[(size_t)(im - 1) * 3 + jv - 1] = (X.G.v_im(iv, 2) == im) ? v : -v;
      }
    }
    for (int j = 0; j < X.g->nv_prog; ++j) {
      int iv = X.g->jtv_prog[j];
      int im1 = X.G.v_im(iv, 1), im2 = X.G.v_im(iv, 2);
      T a = -(T)o.vort_damp_fact * std::min(X.arm0[im1 - 1], X.arm0[im2 - 1]);
      T ph = (T)1, pl = (T)1;
      for (int i = 0; i < level; ++i) ph = ph * a;
      for (int i = 0; i < level - 1; ++i) pl = pl * a;
      X.fvorth[iv] = (T)0.50 * X.dniu[iv - 1] / (T)dtm * ph;
      if (level > 2) X.fvortl[iv] = (T)0.50 * X.dniu[iv - 1] / (T)dtm * pl;
    }
  }
  T* v1 = X.vort2d.data();
  for (int j = 0; j < X.g->nm_prog; ++j) {
    int im = X.g->jtm_prog[j];
    for (int k = 1; k <= mza; ++k) F2(v1, k, im) = 0;
    for (int jv = 1; jv <= 3; ++jv) {
      int iv = X.m_iv(im, jv);
      T vf = X.vfact[(size_t)(im - 1) * 3 + jv - 1];
      for (int k = X.G.lpv(iv); k <= mza; ++k) F2(v1, k, im) = F2(v1, k, im) + F2(s.vc, k, iv) * vf;
    }
  }
  auto rr = [&](int k, int iw1, int iw2) { return (T)(F2(s.rho, k, iw1) + F2(s.rho, k, iw2)); };
  if (level == 1) {
    for (int j = 0; j < X.g->nv_prog; ++j) {
      int iv = X.g->jtv_prog[j];
      int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2), im1 = X.G.v_im(iv, 1), im2 = X.G.v_im(iv, 2);
      for (int k = X.G.lpv(iv); k <= mza; ++k)
        F2(vmt, k, iv) = F2(vmt, k, iv) + X.fvorth[iv] * (F2(v1, k, im2) - F2(v1, k, im1)) * rr(k, iw1, iw2);
    }
    return;
  }
  int il = 1, ih = 2;
  for (int nn = 1; nn <= level - 1; ++nn) {
    il = (nn - 1) % 2 + 1;
    ih = nn % 2 + 1;
    T* src = X.vort2d.data() + (size_t)(il - 1) * plane;
    T* dst = X.vort2d.data() + (size_t)(ih - 1) * plane;
    for (int j = 0; j < X.g->nm_prog; ++j) {
      int im = X.g->jtm_prog[j];
      laplacian_m(X, im, src, dst + (size_t)(im - 1) * mza);
    }
  }
  T* dl = X.vort2d.data() + (size_t)(il - 1) * plane;
  T* dh = X.vort2d.data() + (size_t)(ih - 1) * plane;
  for (int j = 0; j < X.g->nv_prog; ++j) {
    int iv = X.g->jtv_prog[j];
    int iw1 = X.G.v_iw(iv, 1), iw2 = X.G.v_iw(iv, 2), im1 = X.G.v_im(iv, 1), im2 = X.G.v_im(iv, 2);
    int ka = (level == 3) ? std::max(X.lpm(im1), X.lpm(im2)) : X.G.lpv(iv);
    for (int k = X.G.lpv(iv); k <= ka - 1; ++k)
      F2(vmt, k, iv) = F2(vmt, k, iv) + X.fvortl[iv] * (F2(dl, k, im2) - F2(dl, k, im1)) * rr(k, iw1, iw2);
    for (int k = ka; k <= mza; ++k)
      F2(vmt, k, iv) = F2(vmt, k, iv) + X.fvorth[iv] * (F2(dh, k, im2) - F2(dh, k, im1)) * rr(k, iw1, iw2);
  }
}

/* ---- eddy diffusion (convect/pbl_driver.f90, modules/mem_rayf.f90) ---------- */

static bool dcmip_mixing_case(int tc) {
  return tc == 110 || tc == 111 || tc == 112 || tc == 113 || tc == 114 || tc == 121 || tc == 122;
}

/* comp_horiz_k / comp_horiz_k_column (pbl_driver.f90:136-238) */
template <class T>
static void comp_horiz_k(DynCtx<T>& X, const DynState<T>& s) {
  const GridT<T>& G = X.G;
  const olamgpu_eddy& e = *X.eddy;
  const int mza = X.mza, mva = X.mva;
  X.akmodx.assign((size_t)mza * mva, (T)0);
  X.akhodx.assign((size_t)mza * mva, (T)0);
  // the arrays keep values the loops do not reach: start from OLAM's
  for (size_t i = 0; i < X.akmodx.size(); ++i) { X.akmodx[i] = (T)e.akmodx[i]; X.akhodx[i] = (T)e.akhodx[i]; }
  X.kmtopv.assign(e.kmtopv, e.kmtopv + mva);
  X.khtopv.assign(e.khtopv, e.khtopv + mva);
  const T dtl = (T)(float)X.o.dtlm;
  std::vector<T> hk0(mza + 1), akstab(mza + 1);
  for (int j = 0; j < X.g->nv_wadj; ++j) {
    const int iv = X.g->jtv_wadj[j];
    const int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    const int mrl = e.mrlv[iv - 1];
    const T fact1 = (T)0.95f / (dtl * (T)G.npoly(iw1));
    const T fact2 = (T)0.95f / (dtl * (T)G.npoly(iw2));
    const T akmin = (T)e.akmin[mrl - 1];
    const int lpv = G.lpv(iv);
    int& khv = X.khtopv[iv - 1];
    int& kmv = X.kmtopv[iv - 1];
    if (akmin > (T)1.e-7f) {
      const T bkmin = akmin * (T).075f * std::pow(std::min(X.arw0[iw1 - 1], X.arw0[iw2 - 1]), (T).66666666f);
      khv = mza;
      kmv = mza;
      for (int k = lpv; k <= mza; ++k) hk0[k] = (T)0.5f * (T)(F2(s.rho, k, iw1) + F2(s.rho, k, iw2)) * bkmin;
    } else {
      khv = std::max(e.khtop[iw1 - 1], e.khtop[iw2 - 1]);
      khv = khv >= lpv ? khv + 1 : 1;
      kmv = std::max(e.kmtop[iw1 - 1], e.kmtop[iw2 - 1]);
      kmv = kmv >= lpv ? kmv + 1 : 1;
    }
    for (int k = lpv; k <= std::min(mza, std::max(kmv, khv)); ++k) {
      const T stab1 = (T)(F2(s.rho, k, iw1) * (R8)(T)F2(X.g->volt, k, iw1) * (R8)fact1);
      const T stab2 = (T)(F2(s.rho, k, iw2) * (R8)(T)F2(X.g->volt, k, iw2) * (R8)fact2);
      akstab[k] = std::min(stab1, stab2);
    }
    auto vk = [&](const float* a, int k, int iw) { return (T)a[(size_t)(iw - 1) * mza + (k - 1)]; };
    for (int k = lpv; k <= std::min(mza, kmv); ++k) {
      T hkm = (T)0.25f * (vk(e.vkm, k, iw1) + vk(e.vkm, k, iw2) + vk(e.vkm, k - 1, iw1) + vk(e.vkm, k - 1, iw2));
      if (akmin > (T)1.e-7f) hkm = std::max(hkm, hk0[k]);
      F2(X.akmodx.data(), k, iv) = std::min(X.dniv[iv - 1] * F2(X.arv.data(), k, iv) * hkm, akstab[k]);
    }
    for (int k = lpv; k <= std::min(mza, khv); ++k) {
      T hkh = (T)0.25f * (vk(e.vkh, k, iw1) + vk(e.vkh, k, iw2) + vk(e.vkh, k - 1, iw1) + vk(e.vkh, k - 1, iw2));
      if (akmin > (T)1.e-7f) hkh = std::max(hkh, hk0[k]);
      F2(X.akhodx.data(), k, iv) = std::min(X.dniv[iv - 1] * F2(X.arv.data(), k, iv) * hkh, akstab[k]);
    }
  }
  X.have_hk = true;
}

/* tridv (tridiag_lib.f90:40-104) for nsp right-hand sides, arrays indexed by k */
template <class T>
static void tridv(const T* l, const T* d, const T* u, const std::vector<T>* b, std::vector<T>* x, int ka, int kz,
                  int nsp) {
  std::vector<T> gam(kz + 2);
  T bet = (T)1.0 / d[ka];
  for (int v = 0; v < nsp; ++v) x[v][ka] = bet * b[v][ka];
  for (int k = ka + 1; k <= kz; ++k) {
    gam[k] = bet * u[k - 1];
    bet = (T)1.0 / (d[k] - l[k] * gam[k]);
    for (int v = 0; v < nsp; ++v) x[v][k] = bet * (b[v][k] - l[k] * x[v][k - 1]);
  }
  for (int v = 0; v < nsp; ++v)
    for (int k = kz - 1; k >= ka; --k) x[v][k] = x[v][k] - gam[k + 1] * x[v][k + 1];
}

/* solve_eddy_diff_heat (pbl_driver.f90:519-624) on one column of thilt_short */
template <class T>
static void solve_eddy_diff_heat(const DynCtx<T>& X, const DynState<T>& s, int iw, T* thilt) {
  const olamgpu_eddy& e = *X.eddy;
  const GridT<T>& G = X.G;
  const int mza = X.mza;
  if (dcmip_mixing_case(e.test_case)) return;
  const int ka = G.lpw(iw), khtop = e.khtop[iw - 1];
  if (khtop < ka) return;
  const T dts = (T)(float)X.o.dtsm, forw_imp = (T)1.1f;
  const int kmax = khtop + 1;
  auto fld = [&](const float* a, int k) { return (T)a[(size_t)(iw - 1) * mza + (k - 1)]; };
  std::vector<T> dtomass(mza + 2), varp(mza + 2), v5(mza + 2), v6(mza + 2), v7(mza + 2), rhs(mza + 2), soln(mza + 2);
  for (int k = ka; k <= kmax; ++k) {
    const T dtom = dts * G.volti_(k, iw) / (T)F2(s.rho, k, iw);
    dtomass[k] = forw_imp * dtom;
    varp[k] = F2(s.thil, k, iw) + dtom * thilt[k - 1];
  }
  for (int k = ka; k <= khtop; ++k) {
    const T akodz = F2(X.arw.data(), k, iw) * fld(e.vkh, k) * (T)X.g->dzim[k - 1];
    rhs[k] = akodz * (varp[k] - varp[k + 1]);
    v5[k] = -akodz * dtomass[k];
    v7[k] = -akodz * dtomass[k + 1];
    v6[k] = (T)1. - v5[k] - v7[k];
  }
  // non-local PBL term
  const int mrl = e.mrlw[iw - 1];
  if (e.idiffk[mrl - 1] == 1 && fld(e.agamma, ka) > (T)1.e-7f * F2(X.arw.data(), ka, iw)) {
    const T wt0 = (T)e.sfluxt[iw - 1] * fld(e.theta, ka) / ((T)F2(s.rho, ka, iw) * (T)e.cp * fld(e.tair, ka));
    for (int k = ka; k <= e.kpblh[iw - 1]; ++k) rhs[k] = rhs[k] + wt0 * fld(e.agamma, k);
  }
  tridiffo(ka, khtop, v5.data(), v6.data(), v7.data(), rhs.data(), soln.data());
  std::vector<R8> flux(mza + 2, 0.0);
  for (int k = ka; k <= kmax - 1; ++k) flux[k] = (R8)soln[k];
  for (int k = ka; k <= kmax; ++k) thilt[k - 1] = thilt[k - 1] + (T)(flux[k - 1] - flux[k]);
}

/* solve_eddy_diff_vxe (pbl_driver.f90:628-742) on one column */
template <class T>
static void solve_eddy_diff_vxe(const DynCtx<T>& X, const DynState<T>& s, int iw, T* vmxet, T* vmyet, T* vmzet) {
  const olamgpu_eddy& e = *X.eddy;
  const GridT<T>& G = X.G;
  const int mza = X.mza;
  if (dcmip_mixing_case(e.test_case)) return;
  const int ka = G.lpw(iw), lsw = e.lsw[iw - 1], kmtop = e.kmtop[iw - 1];
  const T dts = (T)(float)X.o.dtsm, forw_imp = (T)1.1f;
  const int kmax = std::max(kmtop + 1, ka + lsw - 1);
  const int n = std::max(mza, kmax) + 2;
  std::vector<T> akodz(n, (T)0), dtomass(n), v3(n, (T)0), v5(n), v6(n), v7(n);
  std::vector<T> rhs[3] = {std::vector<T>(n), std::vector<T>(n), std::vector<T>(n)};
  std::vector<T> sol[3] = {std::vector<T>(n), std::vector<T>(n), std::vector<T>(n)};
  std::vector<T> v2[3] = {std::vector<T>(n, (T)0), std::vector<T>(n, (T)0), std::vector<T>(n, (T)0)};
  auto fld = [&](const float* a, int k) { return (T)a[(size_t)(iw - 1) * mza + (k - 1)]; };
  const T* ve[3] = {s.vxe, s.vye, s.vze};
  T* vt[3] = {vmxet, vmyet, vmzet};
  akodz[ka - 1] = 0;
  for (int k = kmtop + 1; k <= kmax; ++k) akodz[k] = 0;
  for (int k = ka; k <= kmtop; ++k) akodz[k] = F2(X.arw.data(), k, iw) * fld(e.vkm, k) * (T)X.g->dzim[k - 1];
  for (int k = ka; k <= kmax; ++k) {
    const T dtom = (T)((R8)(dts * G.volti_(k, iw)) / F2(s.rho, k, iw));
    dtomass[k] = forw_imp * dtom;
    v5[k] = -dtomass[k] * akodz[k - 1];
    v7[k] = -dtomass[k] * akodz[k];
    v6[k] = (T)1. - v5[k] - v7[k];
    for (int c = 0; c < 3; ++c) rhs[c][k] = F2(ve[c], k, iw);
  }
  // surface drag over the levels in contact with the surface
  for (int k = ka; k <= ka + lsw - 1; ++k) {
    const int ks = k - ka + 1;
    v3[k] = (T)e.akm_sfc[(size_t)(iw - 1) * e.nsw_max + (ks - 1)] * (T)(1.0f / X.g->dzt_bot[k - 1]);
    v6[k] = v6[k] + dtomass[k] * v3[k];
  }
  if (ka <= kmax) tridv(v5.data(), v6.data(), v7.data(), rhs, sol, ka, kmax, 3);
  for (int k = ka; k <= kmax - 1; ++k)
    for (int c = 0; c < 3; ++c) v2[c][k] = akodz[k] * (sol[c][k] - sol[c][k + 1]);
  for (int c = 0; c < 3; ++c) { v2[c][ka - 1] = 0; v2[c][kmax] = 0; }
  for (int k = ka; k <= ka + lsw - 1; ++k)
    for (int c = 0; c < 3; ++c) vt[c][k - 1] = vt[c][k - 1] + (v2[c][k - 1] - v2[c][k] - v3[k] * sol[c][k]);
  for (int k = ka + lsw; k <= kmax; ++k)
    for (int c = 0; c < 3; ++c) vt[c][k - 1] = vt[c][k - 1] + v2[c][k - 1] - v2[c][k];
}

/* rayf_mix_top_vxe (mem_rayf.f90:177-220) */
template <class T>
static void rayf_mix_top_vxe(const DynCtx<T>& X, const DynState<T>& s, int iw, T* vmxet, T* vmyet, T* vmzet) {
  const olamgpu_eddy& e = *X.eddy;
  const int mza = X.mza;
  if (!e.rayf_cofmix || e.krayfmix_bot >= mza) return;   // dorayfmix false
  const int ka = std::max(e.krayfmix_bot, X.G.lpw(iw));
  std::vector<T> fx(mza + 1, (T)0), fy(mza + 1, (T)0), fz(mza + 1, (T)0);
  for (int k = ka; k <= mza - 1; ++k) {
    const T fact = X.arw0[iw - 1] * (T)e.rayf_cofmix[k - 1] * (T)(F2(s.rho, k + 1, iw) + F2(s.rho, k, iw));
    fx[k] = fact * (F2(s.vxe, k, iw) - F2(s.vxe, k + 1, iw));
    fy[k] = fact * (F2(s.vye, k, iw) - F2(s.vye, k + 1, iw));
    fz[k] = fact * (F2(s.vze, k, iw) - F2(s.vze, k + 1, iw));
  }
  for (int k = ka; k <= mza; ++k) {
    vmxet[k - 1] = vmxet[k - 1] + fx[k - 1] - fx[k];
    vmyet[k - 1] = vmyet[k - 1] + fy[k - 1] - fy[k];
    vmzet[k - 1] = vmzet[k - 1] + fz[k - 1] - fz[k];
  }
}

/* fluxes_wrtv (prog_wrtv_rk.f90:950-1129): upwinded face values of one field */
template <class T>
static void fluxes_wrtv(const DynCtx<T>& X, const T* scp, T* scp_upw, T* scp_upv, const T* vmc,
                        const T* wmc, int iorderh) {
  const GridT<T>& G = X.G;
  const int mza = X.mza, mwa = X.mwa;
  const int i2d = iorderh == 2 ? 2 : (iorderh == 3 ? 5 : 0);
  std::vector<T> gxyps((size_t)mza * mwa * (i2d > 0 ? i2d : 1));
  const size_t plane = (size_t)mza * mwa;
  if (iorderh > 1) {
    for (int j = 0; j < X.g->nw_prog; ++j) {
      int iw = X.g->jtw_prog[j];
      T* c0 = gxyps.data() + (size_t)(iw - 1) * mza;
      if (iorderh == 2) {
        // grad_t2d
        for (int k = 1; k <= mza; ++k) { c0[k - 1] = 0; c0[plane + k - 1] = 0; }
        for (int n = 1; n <= G.npoly(iw); ++n) {
          int iwn = G.w_iw(iw, n), ivn = G.w_iv(iw, n);
          T cx = G.gxps_coef(n, iw), cy = G.gyps_coef(n, iw);
          for (int k = G.lpv(ivn); k <= mza; ++k) {
            T d = F2(scp, k, iwn) - F2(scp, k, iw);
            c0[k - 1] = c0[k - 1] + cx * d;
            c0[plane + k - 1] = c0[plane + k - 1] + cy * d;
          }
        }
      } else {
        // grad_t2d_quadratic(..., bounded=.false.)
        for (int m = 0; m < 5; ++m)
          for (int k = 1; k <= mza; ++k) c0[m * plane + k - 1] = 0;
        for (int n = 1; n <= G.npoly(iw); ++n) {
          int iwn = G.w_iw(iw, n), ivn = G.w_iv(iw, n);
          for (int k = G.lpv(ivn); k <= mza; ++k) {
            T sc = F2(scp, k, iwn) - F2(scp, k, iw);
            for (int m = 0; m < 5; ++m) c0[m * plane + k - 1] = c0[m * plane + k - 1] + sc * G.xyh(G.xy_hu, m + 1, n, iw);
          }
        }
      }
    }
  }
  // scalar_w_column (1085-1126)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    int iw = X.g->jtw_prog[j];
    int kb = G.lpw(iw);
    const T* col = scp + (size_t)(iw - 1) * mza;
    std::vector<T> ds(mza + 1), scpb(mza), scpt(mza);
    F2(scp_upw, kb - 1, iw) = col[kb - 1];
    F2(scp_upw, mza, iw) = col[mza - 1];
    for (int k = kb; k <= mza - 1; ++k) ds[k] = col[k] - col[k - 1];
    ds[kb - 1] = 0;
    ds[mza] = 0;
    for (int k = kb; k <= mza; ++k) {
      scpb[k - 1] = col[k - 1] + ds[k] * G.aw(G.a_w, k, 1, 1) + ds[k - 1] * G.aw(G.a_w, k, 2, 1);
      scpt[k - 1] = col[k - 1] + ds[k] * G.aw(G.a_w, k, 1, 2) + ds[k - 1] * G.aw(G.a_w, k, 2, 2);
    }
    for (int k = kb; k <= mza - 1; ++k) {
      T v = scpt[k - 1];
      if (F2(wmc, k, iw) < (T)0) v = scpb[k];
      F2(scp_upw, k, iw) = v;
    }
  }
  // scalar_v_column (1022-1082): quadratic terms use xx0_v (bounded) with
  // the unbounded gradients, as the reference does
  for (int j = 0; j < X.g->nv_wadj; ++j) {
    int iv = X.g->jtv_wadj[j];
    int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T s1 = F2(scp, k, iw1), s2 = F2(scp, k, iw2);
      if (iorderh >= 2) {
        const T* gx = gxyps.data();
        size_t o1 = (size_t)(iw1 - 1) * mza + k - 1, o2 = (size_t)(iw2 - 1) * mza + k - 1;
        s1 = s1 + G.v2(G.dxps, 1, iv) * gx[o1] + G.v2(G.dyps, 1, iv) * gx[plane + o1];
        s2 = s2 + G.v2(G.dxps, 2, iv) * gx[o2] + G.v2(G.dyps, 2, iv) * gx[plane + o2];
        if (iorderh == 3) {
          s1 = s1 + G.v2(G.xx0_v, 1, iv) * gx[2 * plane + o1] + G.v2(G.xy0_v, 1, iv) * gx[3 * plane + o1] +
               G.v2(G.yy0_v, 1, iv) * gx[4 * plane + o1];
          s2 = s2 + G.v2(G.xx0_v, 2, iv) * gx[2 * plane + o2] + G.v2(G.xy0_v, 2, iv) * gx[3 * plane + o2] +
               G.v2(G.yy0_v, 2, iv) * gx[4 * plane + o2];
        }
      }
      // the Fortran evaluates scp + a + b + c ... left to right
      T up = s1;
      if (F2(vmc, k, iv) < (T)0) up = s2;
      F2(scp_upv, k, iv) = up;
    }
  }
}

/* fluxes_wrtv_monot (prog_wrtv_rk.f90:1133-1554): on the last RK stage,
 * flux-corrected upwinded face values of one field.  Low-order faces take
 * the upwind cell of scpt = scp0 + dtr volti sct / rho0 (1179-1186);
 * high-order faces (scp with bounded horizontal gradients, grad_t2d or
 * grad_t2d_quadratic, the xx0_vu face terms, and grad_z_quadratic with
 * constant-gradient ends and a_wu) add their difference to the low-order
 * value scaled by the cell limiter of scalar_monot_limiter (1450-1552). */
template <class T>
static void fluxes_wrtv_monot(const DynCtx<T>& X, const T* scp, const T* scp0, const T* sct, T* scp_upw, T* scp_upv,
                              const R8* rho, const R8* rho0, const T* vmca, const T* wmc, T dtr, int iorderh) {
  const GridT<T>& G = X.G;
  const int mza = X.mza, mwa = X.mwa, mva = X.mva;
  const size_t plane = (size_t)mza * mwa, vplane = (size_t)mza * mva;
  const T eps0 = (T)1.e-32, eps1 = (T)3.e-07, onep = (T)1.0 + eps1;
  std::vector<T> scpt(plane, (T)0), sin_(plane, (T)0), sout(plane, (T)0);
  std::vector<T> sfluxvh(vplane, (T)0), scp_hiv(vplane, (T)0);
  std::vector<T> sfluxwh(plane + 1, (T)0), scp_hiw(plane + 1, (T)0);
  std::vector<T> gx(plane * 5, (T)0);
  // scpt (1179-1186)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    const int iw = X.g->jtw_prog[j];
    for (int k = G.lpw(iw); k <= mza; ++k)
      F2(scpt.data(), k, iw) = F2(scp0, k, iw) + dtr * G.volti_(k, iw) * F2(sct, k, iw) / (T)F2(rho0, k, iw);
  }
  // bounded horizontal gradients (1192-1206)
  if (iorderh > 1) {
    for (int j = 0; j < X.g->nw_prog; ++j) {
      const int iw = X.g->jtw_prog[j];
      T* c0 = gx.data() + (size_t)(iw - 1) * mza;
      for (int n = 1; n <= G.npoly(iw); ++n) {
        const int iwn = G.w_iw(iw, n), ivn = G.w_iv(iw, n);
        for (int k = G.lpv(ivn); k <= mza; ++k) {
          const T d = F2(scp, k, iwn) - F2(scp, k, iw);
          if (iorderh == 2) {
            c0[k - 1] = c0[k - 1] + G.gxps_coef(n, iw) * d;
            c0[plane + k - 1] = c0[plane + k - 1] + G.gyps_coef(n, iw) * d;
          } else {
            for (int m = 0; m < 5; ++m) c0[m * plane + k - 1] = c0[m * plane + k - 1] + d * G.xyh(G.xy_h, m + 1, n, iw);
          }
        }
      }
    }
  }
  // scalar_wflux_monot (1380-1446)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    const int iw = X.g->jtw_prog[j];
    const int kb = G.lpw(iw);
    const T* col = scp + (size_t)(iw - 1) * mza;
    F2(scp_upw, kb - 1, iw) = col[kb - 1];
    F2(scp_upw, mza, iw) = col[mza - 1];
    for (int k = kb; k <= mza - 1; ++k) {
      T v = F2(scpt.data(), k, iw);
      if (F2(wmc, k, iw) < (T)0) v = F2(scpt.data(), k + 1, iw);
      F2(scp_upw, k, iw) = v;
    }
    // grad_z_quadratic(itopbc=1, ibotbc=1, bounded=.false.)
    std::vector<T> ds(mza + 1), sb(mza + 1), st(mza + 1);
    for (int k = kb; k <= mza - 1; ++k) ds[k] = col[k] - col[k - 1];
    ds[kb - 1] = ds[kb];
    ds[mza] = ds[mza - 1];
    for (int k = kb; k <= mza; ++k) {
      sb[k] = col[k - 1] + ds[k] * G.aw(G.a_wu, k, 1, 1) + ds[k - 1] * G.aw(G.a_wu, k, 2, 1);
      st[k] = col[k - 1] + ds[k] * G.aw(G.a_wu, k, 1, 2) + ds[k - 1] * G.aw(G.a_wu, k, 2, 2);
    }
    F2(sfluxwh.data(), kb - 1, iw) = 0;
    F2(sfluxwh.data(), mza, iw) = 0;
    for (int k = kb; k <= mza - 1; ++k) {
      T h = st[k];
      if (F2(wmc, k, iw) < (T)0) h = sb[k + 1];
      h = h - F2(scp_upw, k, iw);
      F2(scp_hiw.data(), k, iw) = h;
      F2(sfluxwh.data(), k, iw) = F2(X.arw.data(), k, iw) * F2(wmc, k, iw) * h;
    }
  }
  // scalar_vflux_monot (1293-1376)
  for (int j = 0; j < X.g->nv_wadj; ++j) {
    const int iv = X.g->jtv_wadj[j];
    const int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      const bool neg = F2(vmca, k, iv) < (T)0;
      const T low = neg ? F2(scpt.data(), k, iw2) : F2(scpt.data(), k, iw1);
      F2(scp_upv, k, iv) = low;
      T s1 = F2(scp, k, iw1), s2 = F2(scp, k, iw2);
      if (iorderh >= 2) {
        const size_t o1 = (size_t)(iw1 - 1) * mza + k - 1, o2 = (size_t)(iw2 - 1) * mza + k - 1;
        s1 = s1 + G.v2(G.dxps, 1, iv) * gx[o1] + G.v2(G.dyps, 1, iv) * gx[plane + o1];
        s2 = s2 + G.v2(G.dxps, 2, iv) * gx[o2] + G.v2(G.dyps, 2, iv) * gx[plane + o2];
        if (iorderh == 3) {
          s1 = s1 + G.v2(G.xx0_vu, 1, iv) * gx[2 * plane + o1] + G.v2(G.xy0_vu, 1, iv) * gx[3 * plane + o1] +
               G.v2(G.yy0_vu, 1, iv) * gx[4 * plane + o1];
          s2 = s2 + G.v2(G.xx0_vu, 2, iv) * gx[2 * plane + o2] + G.v2(G.xy0_vu, 2, iv) * gx[3 * plane + o2] +
               G.v2(G.yy0_vu, 2, iv) * gx[4 * plane + o2];
        }
      }
      T h = neg ? s2 : s1;
      h = h - low;
      F2(scp_hiv.data(), k, iv) = h;
      F2(sfluxvh.data(), k, iv) = F2(vmca, k, iv) * h;
    }
  }
  // scalar_monot_limiter (1450-1552)
  const T dtrp = onep * dtr;
  for (int j = 0; j < X.g->nw_prog; ++j) {
    const int iw = X.g->jtw_prog[j];
    const int kb = G.lpw(iw);
    std::vector<T> wmca(mza + 1, (T)0), smax(mza + 1), smin(mza + 1), rhos(mza + 1), fl(mza + 1, (T)0),
        fi(mza + 1, (T)0), fo(mza + 1, (T)0);
    for (int k = kb; k <= mza - 1; ++k) wmca[k] = F2(wmc, k, iw) * F2(X.arw.data(), k, iw);
    for (int k = kb; k <= mza; ++k) {
      smax[k] = smin[k] = F2(scpt.data(), k, iw);
      rhos[k] = (T)F2(rho, k, iw);
    }
    for (int k = kb + 1; k <= mza; ++k)
      if (wmca[k - 1] > (T)0) {
        smax[k] = std::max(smax[k], F2(scpt.data(), k - 1, iw));
        smin[k] = std::min(smin[k], F2(scpt.data(), k - 1, iw));
      }
    for (int k = kb; k <= mza - 1; ++k)
      if (wmca[k] < (T)0) {
        smax[k] = std::max(smax[k], F2(scpt.data(), k + 1, iw));
        smin[k] = std::min(smin[k], F2(scpt.data(), k + 1, iw));
      }
    for (int jv = 1; jv <= G.npoly(iw); ++jv) {
      const int iv = G.w_iv(iw, jv), iwn = G.w_iw(iw, jv);
      const T dv = G.w_dirv(iw, jv);
      for (int k = G.lpv(iv); k <= mza; ++k) {
        fl[k] = fl[k] + dv * F2(vmca, k, iv) * (F2(scp_upv, k, iv) - F2(scpt.data(), k, iw));
        fi[k] = fi[k] + std::max(dv * F2(sfluxvh.data(), k, iv), (T)0);
        fo[k] = fo[k] + std::min(dv * F2(sfluxvh.data(), k, iv), (T)0);
        if (dv * F2(vmca, k, iv) > (T)0) {
          smax[k] = std::max(smax[k], F2(scpt.data(), k, iwn));
          smin[k] = std::min(smin[k], F2(scpt.data(), k, iwn));
        }
      }
    }
    for (int k = kb; k <= mza; ++k) {
      const T s = F2(scpt.data(), k, iw);
      fl[k] = fl[k] + wmca[k - 1] * (F2(scp_upw, k - 1, iw) - s) - wmca[k] * (F2(scp_upw, k, iw) - s);
      fi[k] = fi[k] + std::max(F2(sfluxwh.data(), k - 1, iw), (T)0) - std::min(F2(sfluxwh.data(), k, iw), (T)0);
      fo[k] = fo[k] + std::min(F2(sfluxwh.data(), k - 1, iw), (T)0) - std::max(F2(sfluxwh.data(), k, iw), (T)0);
      const T rscp_low = s * rhos[k] + dtr * G.volti_(k, iw) * fl[k];
      const T flux_in = std::max(dtrp * G.volti_(k, iw) * fi[k], eps0);
      const T flux_out = std::min(dtrp * G.volti_(k, iw) * fo[k], -eps0);
      const T epsr = eps1 * std::fabs(rscp_low);
      const T sc_in = std::max(rhos[k] * smax[k] - (rscp_low + epsr) - eps0, (T)0);
      const T sc_out = std::min(rhos[k] * smin[k] - (rscp_low - epsr) + eps0, (T)0);
      F2(sin_.data(), k, iw) = std::min((T)1, sc_in / std::max(flux_in, (T)0.01 * sc_in));
      F2(sout.data(), k, iw) = std::min((T)1, sc_out / std::min(flux_out, (T)0.01 * sc_out));
    }
  }
  // flux renormalisation (1250-1284)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    const int iw = X.g->jtw_prog[j];
    for (int k = G.lpw(iw); k <= mza - 1; ++k) {
      T sc = std::min(F2(sin_.data(), k + 1, iw), F2(sout.data(), k, iw));
      if (F2(sfluxwh.data(), k, iw) < (T)0) sc = std::min(F2(sin_.data(), k, iw), F2(sout.data(), k + 1, iw));
      F2(scp_upw, k, iw) = F2(scp_upw, k, iw) + F2(scp_hiw.data(), k, iw) * sc;
    }
  }
  for (int j = 0; j < X.g->nv_wadj; ++j) {
    const int iv = X.g->jtv_wadj[j];
    const int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
    for (int k = G.lpv(iv); k <= mza; ++k) {
      T sc = std::min(F2(sin_.data(), k, iw2), F2(sout.data(), k, iw1));
      if (F2(sfluxvh.data(), k, iv) < (T)0) sc = std::min(F2(sin_.data(), k, iw1), F2(sout.data(), k, iw2));
      F2(scp_upv, k, iv) = F2(scp_upv, k, iv) + F2(scp_hiv.data(), k, iv) * sc;
    }
  }
}

/* prog_wrtv_rk (prog_wrtv_rk.f90:58-488) */
template <class T>
static int prog_wrtv_rk(DynCtx<T>& X, const DynState<T>& s, int istp) {
  const GridT<T>& G = X.G;
  const olamgpu_opts& o = X.o;
  const int mza = X.mza, mwa = X.mwa, mva = X.mva;
  const R8 dtsm = o.dtsm, dtlm = o.dtlm;
  const size_t wz = (size_t)mza * mwa, vz = (size_t)mza * mva;
  if (!o.divh_damp_short && istp == 1) divh_damp(X, s, s.vmt, dtlm);
  if (!o.vort_damp_short && istp == 1) vort_damp(X, s, s.vmt, dtlm);
  std::vector<T> thil_upv(vz), vxe_upv(vz), vye_upv(vz), vze_upv(vz);
  std::vector<T> thil_upw(wz + 1), vxe_upw(wz + 1), vye_upw(wz + 1), vze_upw(wz + 1);
  std::vector<T> vmxet_rk(wz), vmyet_rk(wz), vmzet_rk(wz), thilt_rk(wz);
  std::vector<R8> rho0(wz), rth0(wz);
  std::vector<T> wmc0(wz), vmc0(vz), vmca(vz, (T)0);
  std::vector<T> thilt_short(wz), vmxet_short(wz), vmyet_short(wz), vmzet_short(wz), vmt_short(vz);
  const bool thil_monot = o.ithil_monot > 0, wind_monot = o.iwind_monot > 0;
  std::vector<T> thl0, vxe0, vye0, vze0;   // start values of the limited fields (186-198)
  if (thil_monot) thl0.assign(s.thil, s.thil + wz);
  if (wind_monot) { vxe0.assign(s.vxe, s.vxe + wz); vye0.assign(s.vye, s.vye + wz); vze0.assign(s.vze, s.vze + wz); }
  // prognostic shaved-cell method (202-211): the momentum of the levels of a
  // column with closed V faces (lve2 of them from lpw up) at the step's start
  const int* lve2 = X.g->lve2;
  int nve2 = 0;
  if (lve2)
    for (int iw = 2; iw <= mwa; ++iw) {
      nve2 = std::max(nve2, lve2[iw - 1]);
      for (int jv = 1; jv <= G.npoly(iw); ++jv)
        if (G.lpv(G.w_iv(iw, jv)) - G.lpw(iw) > lve2[iw - 1]) return OLAMGPU_E_ARG;   // a closed face not covered
    }
  const size_t nv2 = (size_t)std::max(nve2, 1);
  std::vector<T> vm0(3 * nv2 * (size_t)mwa);
  auto M0 = [&](int c, int ks, int iw) -> T& { return vm0[(((size_t)(iw - 1) * nv2) + ks - 1) * 3 + c]; };
  if (nve2)
    for (int j = 0; j < X.g->nw_prog; ++j) {
      const int iw = X.g->jtw_prog[j];
      for (int ks = 1; ks <= lve2[iw - 1]; ++ks) {
        const int k = ks + G.lpw(iw) - 1;
        const T rs = (T)F2(s.rho, k, iw);
        M0(0, ks, iw) = F2(s.vxe, k, iw) * rs;
        M0(1, ks, iw) = F2(s.vye, k, iw) * rs;
        M0(2, ks, iw) = F2(s.vze, k, iw) * rs;
      }
    }
  // column setup (166-253)
  for (int j = 0; j < X.g->nw_prog; ++j) {
    int iw = X.g->jtw_prog[j];
    F2(thil_upw.data(), mza, iw) = 0;
    F2(thil_upw.data(), G.lpw(iw) - 1, iw) = 0;
    for (int k = G.lpw(iw); k <= mza; ++k) {
      T v4 = (T)F2(X.g->volt, k, iw);
      F2(rth0.data(), k, iw) = (R8)F2(s.thil, k, iw) * F2(s.rho, k, iw);
      F2(rho0.data(), k, iw) = F2(s.rho, k, iw);
      F2(wmc0.data(), k, iw) = F2(s.wmc, k, iw);
      F2(thilt_short.data(), k, iw) = F2(s.thilt, k, iw) * v4;
      F2(vmxet_short.data(), k, iw) = F2(s.vmxet, k, iw) * v4;
      F2(vmyet_short.data(), k, iw) = F2(s.vmyet, k, iw) * v4;
      F2(vmzet_short.data(), k, iw) = F2(s.vmzet, k, iw) * v4;
    }
    // vertical eddy diffusion of heat and momentum, top-level wind mixing (214-225)
    T* sth = thilt_short.data() + (size_t)(iw - 1) * mza;
    T* svx = vmxet_short.data() + (size_t)(iw - 1) * mza;
    T* svy = vmyet_short.data() + (size_t)(iw - 1) * mza;
    T* svz = vmzet_short.data() + (size_t)(iw - 1) * mza;
    if (X.eddy) {
      solve_eddy_diff_heat(X, s, iw, sth);
      solve_eddy_diff_vxe(X, s, iw, svx, svy, svz);
      rayf_mix_top_vxe(X, s, iw, svx, svy, svz);
    }
    if (o.rayf_cof && o.initial == 1 && o.dn01d && o.th01d) {
      for (int k = o.krayf_bot; k <= mza; ++k) {
        T v4 = (T)F2(X.g->volt, k, iw);
        F2(thilt_short.data(), k, iw) = F2(thilt_short.data(), k, iw) +
            (T)o.rayf_cof[k - 1] * (T)o.dn01d[k - 1] * ((T)o.th01d[k - 1] - F2(s.thil, k, iw)) * v4;
      }
    }
    // horizontal diffusion (238-251)
    if (X.eddy) {
      const olamgpu_eddy& e = *X.eddy;
      for (int jv = 1; jv <= G.npoly(iw); ++jv) {
        const int iv = G.w_iv(iw, jv), iwn = G.w_iw(iw, jv);
        const int khv = X.have_hk ? X.khtopv[iv - 1] : e.khtopv[iv - 1];
        const int kmv = X.have_hk ? X.kmtopv[iv - 1] : e.kmtopv[iv - 1];
        auto akh = [&](int k) { return X.have_hk ? F2(X.akhodx.data(), k, iv) : (T)e.akhodx[(size_t)(iv - 1) * mza + k - 1]; };
        auto akm = [&](int k) { return X.have_hk ? F2(X.akmodx.data(), k, iv) : (T)e.akmodx[(size_t)(iv - 1) * mza + k - 1]; };
        for (int k = G.lpv(iv); k <= std::min(mza, khv); ++k)
          sth[k - 1] = sth[k - 1] + akh(k) * (F2(s.thil, k, iwn) - F2(s.thil, k, iw));
        for (int k = G.lpv(iv); k <= std::min(mza, kmv); ++k) {
          const T a = akm(k);
          svx[k - 1] = svx[k - 1] + a * (F2(s.vxe, k, iwn) - F2(s.vxe, k, iw));
          svy[k - 1] = svy[k - 1] + a * (F2(s.vye, k, iwn) - F2(s.vye, k, iw));
          svz[k - 1] = svz[k - 1] + a * (F2(s.vze, k, iwn) - F2(s.vze, k, iw));
        }
      }
    }
  }
  for (int j = 0; j < X.g->nv_prog; ++j) {
    int iv = X.g->jtv_prog[j];
    for (int k = 1; k <= mza; ++k) {
      F2(vmc0.data(), k, iv) = F2(s.vmc, k, iv);
      F2(vmt_short.data(), k, iv) = F2(s.vmt, k, iv);
    }
  }
  // Rayleigh friction on vmc (268-303), global domain
  if (o.rayf_cof && o.vc03d) {
    for (int j = 0; j < X.g->nv_prog; ++j) {
      int iv = X.g->jtv_prog[j];
      int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
      for (int k = o.krayf_bot; k <= mza; ++k) {
        R8 t = (R8)((T)o.rayf_cof[k - 1] * (T)0.5) * (F2(s.rho, k, iw1) + F2(s.rho, k, iw2)) *
               (R8)((T)F2(o.vc03d, k, iv) - F2(s.vc, k, iv));
        F2(vmt_short.data(), k, iv) = (T)((R8)F2(vmt_short.data(), k, iv) + t);
      }
    }
  }
  if (o.divh_damp_short) divh_damp(X, s, vmt_short.data(), dtsm);
  if (o.vort_damp_short) vort_damp(X, s, vmt_short.data(), dtsm);

  const R8 onethird = 1.0 / 3.0;
  const R8 xstg3[3] = {onethird, 0.5, 1.0};
  const R8 xstg2[2] = {0.5, 1.0};
  const int nrk = o.nrk_wrtv;
  // implicit weights: real(r8), parameter :: fr = .70 (a default-real literal)
  const R8 fr = (R8)0.70f, fp2 = (R8)0.70f, fp3 = (R8)0.70f;
  const float cpocv_f = 1004.f / 717.f;
  const float rocv_f = (1004.f - 717.f) / 717.f;
  const R8 pc2 = fp2 * (R8)cpocv_f, pc3 = fp3 * (R8)cpocv_f;
  const T rocv = (T)rocv_f;
  const T fcoriol = (T)o.fcoriol;

  for (int istage = 1; istage <= nrk; ++istage) {
    R8 dt8 = (nrk <= 2) ? xstg2[istage - 1] * dtsm : xstg3[istage - 1] * dtsm;
    T dts = (T)dt8;
    for (int j = 0; j < X.g->nw_prog; ++j) {
      int iw = X.g->jtw_prog[j];
      for (int k = G.lpw(iw); k <= mza; ++k) {
        F2(vmxet_rk.data(), k, iw) = F2(vmxet_short.data(), k, iw);
        F2(vmyet_rk.data(), k, iw) = F2(vmyet_short.data(), k, iw);
        F2(vmzet_rk.data(), k, iw) = F2(vmzet_short.data(), k, iw);
        F2(thilt_rk.data(), k, iw) = F2(thilt_short.data(), k, iw);
      }
    }
    for (int j = 0; j < X.g->nv_wadj; ++j) {
      int iv = X.g->jtv_wadj[j];
      for (int k = G.lpv(iv); k <= mza; ++k) F2(vmca.data(), k, iv) = F2(s.vmc, k, iv) * F2(X.arv.data(), k, iv);
      if (istage == nrk)
        for (int k = G.lpv(iv); k <= mza; ++k) F2(s.vmasc, k, iv) = F2(s.vmasc, k, iv) + F2(vmca.data(), k, iv);
    }
    // (370-399)
    if (istage == nrk && thil_monot)
      fluxes_wrtv_monot(X, s.thil, thl0.data(), thilt_short.data(), thil_upw.data(), thil_upv.data(), s.rho,
                        rho0.data(), vmca.data(), s.wmc, dts, o.thil_horiz_adv_order);
    else
      fluxes_wrtv(X, s.thil, thil_upw.data(), thil_upv.data(), s.vmc, s.wmc, o.thil_horiz_adv_order);
    if (istage == nrk && wind_monot) {
      fluxes_wrtv_monot(X, s.vxe, vxe0.data(), vmxet_short.data(), vxe_upw.data(), vxe_upv.data(), s.rho,
                        rho0.data(), vmca.data(), s.wmc, dts, o.wind_horiz_adv_order);
      fluxes_wrtv_monot(X, s.vye, vye0.data(), vmyet_short.data(), vye_upw.data(), vye_upv.data(), s.rho,
                        rho0.data(), vmca.data(), s.wmc, dts, o.wind_horiz_adv_order);
      fluxes_wrtv_monot(X, s.vze, vze0.data(), vmzet_short.data(), vze_upw.data(), vze_upv.data(), s.rho,
                        rho0.data(), vmca.data(), s.wmc, dts, o.wind_horiz_adv_order);
    } else {
      fluxes_wrtv(X, s.vxe, vxe_upw.data(), vxe_upv.data(), s.vmc, s.wmc, o.wind_horiz_adv_order);
      fluxes_wrtv(X, s.vye, vye_upw.data(), vye_upv.data(), s.vmc, s.wmc, o.wind_horiz_adv_order);
      fluxes_wrtv(X, s.vze, vze_upw.data(), vze_upv.data(), s.vmc, s.wmc, o.wind_horiz_adv_order);
    }

    // prog_wrt_begs (494-884) for every prognostic column
    for (int j = 0; j < X.g->nw_prog; ++j) {
      int iw = X.g->jtw_prog[j];
      const int ka = G.lpw(iw);
      std::vector<R8> hflx(mza + 1, 0), delex_rho(mza + 1, 0), delex_rt(mza + 1, 0), rhothil(mza + 1, 0);
      std::vector<R8> vflux_thil(mza + 1, 0), press_ex(mza + 2, 0), rho_ex(mza + 2, 0), b5(mza + 2, 0), b10(mza + 1, 0);
      std::vector<T> delex_wm(mza + 1, 0), wmf(mza + 1, 0), wma(mza + 1, 0), vfx(mza + 1, 0), vfy(mza + 1, 0),
          vfz(mza + 1, 0), b15(mza + 2, 0), b31(mza + 1, 0), b32(mza + 1, 0), b33(mza + 1, 0);
      vflux_thil[ka - 1] = 0; vflux_thil[mza] = 0;
      vfx[ka - 1] = vfx[mza] = 0; vfy[ka - 1] = vfy[mza] = 0; vfz[ka - 1] = vfz[mza] = 0;
      for (int k = ka; k <= mza; ++k) hflx[k] = 0;
      for (int jv = 1; jv <= G.npoly(iw); ++jv) {
        int iv = G.w_iv(iw, jv);
        int kbv = G.lpv(iv);
        if (G.w_dirv(iw, jv) > (T)0) {
          for (int k = kbv; k <= mza; ++k) {
            T vm = F2(vmca.data(), k, iv);
            hflx[k] = hflx[k] + (R8)vm;
            F2(thilt_rk.data(), k, iw) = F2(thilt_rk.data(), k, iw) + vm * F2(thil_upv.data(), k, iv);
            F2(vmxet_rk.data(), k, iw) = F2(vmxet_rk.data(), k, iw) + vm * F2(vxe_upv.data(), k, iv);
            F2(vmyet_rk.data(), k, iw) = F2(vmyet_rk.data(), k, iw) + vm * F2(vye_upv.data(), k, iv);
            F2(vmzet_rk.data(), k, iw) = F2(vmzet_rk.data(), k, iw) + vm * F2(vze_upv.data(), k, iv);
          }
        } else {
          for (int k = kbv; k <= mza; ++k) {
            T vm = F2(vmca.data(), k, iv);
            hflx[k] = hflx[k] - (R8)vm;
            F2(thilt_rk.data(), k, iw) = F2(thilt_rk.data(), k, iw) - vm * F2(thil_upv.data(), k, iv);
            F2(vmxet_rk.data(), k, iw) = F2(vmxet_rk.data(), k, iw) - vm * F2(vxe_upv.data(), k, iv);
            F2(vmyet_rk.data(), k, iw) = F2(vmyet_rk.data(), k, iw) - vm * F2(vye_upv.data(), k, iv);
            F2(vmzet_rk.data(), k, iw) = F2(vmzet_rk.data(), k, iw) - vm * F2(vze_upv.data(), k, iv);
          }
        }
      }
      // Coriolis, global domain (677-681)
      for (int k = ka; k <= mza; ++k) {
        T mass = (T)(F2(s.rho, k, iw) * F2(X.g->volt, k, iw));
        F2(vmxet_rk.data(), k, iw) = F2(vmxet_rk.data(), k, iw) + mass * fcoriol * F2(s.vye, k, iw);
        F2(vmyet_rk.data(), k, iw) = F2(vmyet_rk.data(), k, iw) - mass * fcoriol * F2(s.vxe, k, iw);
      }
      for (int k = ka; k <= mza; ++k) {
        rhothil[k] = F2(s.rho, k, iw) * (R8)F2(s.thil, k, iw);
        b10[k] = dt8 * (R8)G.volti_(k, iw);
        b5[k] = (R8)(F2(s.alpha_press, k, iw) * (T)std::pow((T)rhothil[k], rocv));
        b15[k] = (T)(b10[k] * b5[k]);
        delex_rho[k] = b10[k] * hflx[k];
        delex_rt[k] = b10[k] * (R8)F2(thilt_rk.data(), k, iw);
      }
      if (istage > 1)
        for (int k = ka; k <= mza; ++k) {
          delex_rho[k] = delex_rho[k] + F2(rho0.data(), k, iw) - F2(s.rho, k, iw);
          delex_rt[k] = delex_rt[k] + F2(rth0.data(), k, iw) - rhothil[k];
        }
      for (int k = ka; k <= mza; ++k) {
        press_ex[k] = b5[k] * (rhothil[k] + pc2 * delex_rt[k]);
        rho_ex[k] = F2(s.rho, k, iw) + fr * delex_rho[k];
      }
      const T wnx = X.wnx[iw - 1], wny = X.wny[iw - 1], wnz = X.wnz[iw - 1];
      for (int k = ka; k <= mza - 1; ++k) {
        T a = (T)(press_ex[k] - press_ex[k + 1]) * F2(s.pwfac, k, iw);
        T b = (T)(X.g->gdz_wgtm8[k - 1] * rho_ex[k] + X.g->gdz_wgtp8[k - 1] * rho_ex[k + 1]);
        T c = (wnx * (F2(vmxet_rk.data(), k, iw) + F2(vmxet_rk.data(), k + 1, iw)) +
               wny * (F2(vmyet_rk.data(), k, iw) + F2(vmyet_rk.data(), k + 1, iw)) +
               wnz * (F2(vmzet_rk.data(), k, iw) + F2(vmzet_rk.data(), k + 1, iw))) *
              F2(X.volwi.data(), k, iw);
        delex_wm[k] = F2(wmc0.data(), k, iw) + dts * (a - b + c);
      }
      T c8 = dts * (T)pc2;
      T c9 = -dts * dts * (T)fr;
      for (int k = ka; k <= mza - 1; ++k) {
        T b7 = dts * F2(X.volwi.data(), k, iw);
        T b8 = c8 * F2(s.pwfac, k, iw);
        T b21 = b7 * F2(s.wc, k - 1, iw);
        T b22 = b7 * F2(s.wc, k + 1, iw);
        T b23 = b8 * b15[k];
        T b24 = b8 * b15[k + 1];
        T b25 = c9 * G.volti_(k, iw) * X.gdz_wgtm[k - 1];
        T b26 = c9 * G.volti_(k + 1, iw) * X.gdz_wgtp[k - 1];
        b31[k] = -F2(X.arw.data(), k - 1, iw) * (b21 + b25 + b23 * F2(thil_upw.data(), k - 1, iw));
        b32[k] = X.b20[k] + F2(X.arw.data(), k, iw) * (b25 - b26 + (b23 + b24) * F2(thil_upw.data(), k, iw));
        b33[k] = F2(X.arw.data(), k + 1, iw) * (b22 + b26 - b24 * F2(thil_upw.data(), k + 1, iw));
      }
      if (ka <= mza - 1) tridiffo(ka, mza - 1, b31.data(), b32.data(), b33.data(), delex_wm.data(), wmf.data());
      wma[ka - 1] = 0;
      wma[mza] = 0;
      for (int k = ka; k <= mza - 1; ++k) wma[k] = wmf[k] * F2(X.arw.data(), k, iw);
      for (int k = ka; k <= mza - 1; ++k) {
        vflux_thil[k] = (R8)(wma[k] * F2(thil_upw.data(), k, iw));
        vfx[k] = wma[k] * F2(vxe_upw.data(), k, iw);
        vfy[k] = wma[k] * F2(vye_upw.data(), k, iw);
        vfz[k] = wma[k] * F2(vze_upw.data(), k, iw);
      }
      if (istage == nrk)
        for (int k = ka; k <= mza - 1; ++k) F2(s.wmasc, k, iw) = F2(s.wmasc, k, iw) + wma[k];
      for (int k = ka; k <= mza; ++k) {
        F2(s.rho, k, iw) = F2(rho0.data(), k, iw) +
                           dt8 * (R8)G.volti_(k, iw) * (hflx[k] + (R8)wma[k - 1] - (R8)wma[k]);
        delex_rt[k] = delex_rt[k] + b10[k] * (vflux_thil[k - 1] - vflux_thil[k]);
        F2(s.press, k, iw) = b5[k] * (rhothil[k] + pc3 * delex_rt[k]);
        F2(s.thil, k, iw) = (T)((rhothil[k] + delex_rt[k]) / F2(s.rho, k, iw));
        F2(vmxet_rk.data(), k, iw) = F2(vmxet_rk.data(), k, iw) + vfx[k - 1] - vfx[k];
        F2(vmyet_rk.data(), k, iw) = F2(vmyet_rk.data(), k, iw) + vfy[k - 1] - vfy[k];
        F2(vmzet_rk.data(), k, iw) = F2(vmzet_rk.data(), k, iw) + vfz[k - 1] - vfz[k];
      }
      for (int k = ka; k <= mza - 1; ++k) {
        F2(s.wmc, k, iw) = wmf[k];
        F2(s.wc, k, iw) = wmf[k] / (T)(X.g->zwgt_bot8[k - 1] * F2(s.rho, k, iw) +
                                      X.g->zwgt_top8[k - 1] * F2(s.rho, k + 1, iw));
      }
      F2(s.wc, ka - 1, iw) = F2(s.wc, ka, iw);
      for (int k = 1; k <= ka - 1; ++k) F2(s.thil, k, iw) = F2(s.thil, ka, iw);
    }
    // prog_v_begs (888-946)
    for (int j = 0; j < X.g->nv_prog; ++j) {
      int iv = X.g->jtv_prog[j];
      int iw1 = G.v_iw(iv, 1), iw2 = G.v_iw(iv, 2);
      T vx = X.vnx[iv - 1], vy = X.vny[iv - 1], vzz = X.vnz[iv - 1];
      for (int k = G.lpv(iv); k <= mza; ++k) {
        T pgf = (T)(F2(s.press, k, iw1) - F2(s.press, k, iw2)) * F2(s.pvfac, k, iv);
        T v = F2(vmc0.data(), k, iv) +
              dts * (F2(vmt_short.data(), k, iv) + pgf +
                     (vx * (F2(vmxet_rk.data(), k, iw1) + F2(vmxet_rk.data(), k, iw2)) +
                      vy * (F2(vmyet_rk.data(), k, iw1) + F2(vmyet_rk.data(), k, iw2)) +
                      vzz * (F2(vmzet_rk.data(), k, iw1) + F2(vmzet_rk.data(), k, iw2))) *
                         F2(X.volvi.data(), k, iv));
        F2(s.vmc, k, iv) = v;
        F2(s.vc, k, iv) = (T)2.0 * v / (T)(F2(s.rho, k, iw1) + F2(s.rho, k, iw2));
      }
    }
    // update_vxe_undrgnd (1558-1595): the prognosed velocities of the levels
    // with closed faces, then vel_t3d_hex (vel_t3d.f90:39-108), whose closed
    // faces take the normal component of those
    for (int j = 0; j < X.g->nw_prog; ++j) {
      int iw = X.g->jtw_prog[j];
      int ka = G.lpw(iw);
      const int nsh = lve2 ? lve2[iw - 1] : 0;
      std::vector<T> p1(3 * (size_t)std::max(nsh, 1));
      for (int ks = 1; ks <= nsh; ++ks) {
        const int k = ks + ka - 1;
        const T rsi = (T)1 / (T)F2(s.rho, k, iw);
        const T vt = (T)F2(X.g->volti, k, iw);
        p1[(ks - 1) * 3 + 0] = (M0(0, ks, iw) + dts * (F2(vmxet_rk.data(), k, iw) * vt)) * rsi;
        p1[(ks - 1) * 3 + 1] = (M0(1, ks, iw) + dts * (F2(vmyet_rk.data(), k, iw) * vt)) * rsi;
        p1[(ks - 1) * 3 + 2] = (M0(2, ks, iw) + dts * (F2(vmzet_rk.data(), k, iw) * vt)) * rsi;
      }
      for (int k = ka; k <= mza; ++k) {
        T wst = F2(s.wc, k - 1, iw) + F2(s.wc, k, iw);
        F2(s.vxe, k, iw) = wst * X.wnxo2[iw - 1];
        F2(s.vye, k, iw) = wst * X.wnyo2[iw - 1];
        F2(s.vze, k, iw) = wst * X.wnzo2[iw - 1];
      }
      for (int jv = 1; jv <= G.npoly(iw); ++jv) {
        int iv = G.w_iv(iw, jv);
        T ex = X.ecx[(size_t)(iw - 1) * 7 + jv - 1], ey = X.ecy[(size_t)(iw - 1) * 7 + jv - 1],
          ez = X.ecz[(size_t)(iw - 1) * 7 + jv - 1];
        for (int k = G.lpv(iv); k <= mza; ++k) {
          F2(s.vxe, k, iw) = F2(s.vxe, k, iw) + ex * F2(s.vc, k, iv);
          F2(s.vye, k, iw) = F2(s.vye, k, iw) + ey * F2(s.vc, k, iv);
          F2(s.vze, k, iw) = F2(s.vze, k, iw) + ez * F2(s.vc, k, iv);
        }
        for (int k = ka; k <= G.lpv(iv) - 1; ++k) {
          const int ksw = k - ka + 1;
          const T vcwall = X.vnx[iv - 1] * p1[(ksw - 1) * 3] + X.vny[iv - 1] * p1[(ksw - 1) * 3 + 1] +
                           X.vnz[iv - 1] * p1[(ksw - 1) * 3 + 2];
          F2(s.vxe, k, iw) = F2(s.vxe, k, iw) + ex * vcwall;
          F2(s.vye, k, iw) = F2(s.vye, k, iw) + ey * vcwall;
          F2(s.vze, k, iw) = F2(s.vze, k, iw) + ez * vcwall;
        }
      }
      for (int k = 1; k <= ka - 1; ++k) {
        F2(s.vxe, k, iw) = F2(s.vxe, ka, iw);
        F2(s.vye, k, iw) = F2(s.vye, ka, iw);
        F2(s.vze, k, iw) = F2(s.vze, ka, iw);
      }
    }
  }
  (void)wz; (void)vz; (void)mva;
  return OLAMGPU_OK;
}

/* tend0 (timestep.f90:430-496) for the hot-path arrays */
template <class T>
static void tend0(DynCtx<T>& X, const DynState<T>& s, T* rho_old) {
  const int mza = X.mza;
  for (int iw = 2; iw <= X.mwa; ++iw)
    for (int k = X.G.lpw(iw); k <= mza; ++k) {
      F2(s.vmxet, k, iw) = 0; F2(s.vmyet, k, iw) = 0; F2(s.vmzet, k, iw) = 0; F2(s.thilt, k, iw) = 0;
      F2(rho_old, k, iw) = (T)F2(s.rho, k, iw);
      F2(s.wmasc, k, iw) = 0;
    }
  for (int iv = 2; iv <= X.mva; ++iv)
    for (int k = X.G.lpv(iv); k <= mza; ++k) { F2(s.vmt, k, iv) = 0; F2(s.vmasc, k, iv) = 0; }
}

/* timeavg_momsc (timestep.f90:563-612) */
template <class T>
static void timeavg_momsc(DynCtx<T>& X, const DynState<T>& s) {
  const int mza = X.mza;
  if (X.o.nacoust <= 1) return;
  T a = (T)(float)X.o.nacoust;
  for (int j = 0; j < X.g->nv_wadj; ++j) {
    int iv = X.g->jtv_wadj[j];
    for (int k = X.G.lpv(iv); k <= mza; ++k) F2(s.vmasc, k, iv) = F2(s.vmasc, k, iv) / a;
  }
  for (int j = 0; j < X.g->nw_prog; ++j) {
    int iw = X.g->jtw_prog[j];
    for (int k = X.G.lpw(iw); k <= mza - 1; ++k) F2(s.wmasc, k, iw) = F2(s.wmasc, k, iw) / a;
  }
}

}  // namespace oracle

/* FP64 state: every field double (real promoted) */
typedef struct oracle_state64 {
  double *rho, *press, *thil, *wc, *wmc, *vxe, *vye, *vze, *vmc, *vc, *vmasc, *wmasc;
  double *alpha_press, *pwfac, *pvfac, *thilt, *vmxet, *vmyet, *vmzet, *vmt;
} oracle_state64;

extern "C" {

void* oracle_dyn_new_f32(const olamgpu_grid* g, const olamgpu_opts* o) { return new oracle::DynCtx<float>(g, o); }
void* oracle_dyn_new_f64(const olamgpu_grid* g, const olamgpu_opts* o) { return new oracle::DynCtx<double>(g, o); }
void oracle_dyn_free_f32(void* h) { delete (oracle::DynCtx<float>*)h; }
void oracle_dyn_free_f64(void* h) { delete (oracle::DynCtx<double>*)h; }

static oracle::DynState<float> st32(const olamgpu_state* s) {
  oracle::DynState<float> d;
  d.rho = s->rho; d.press = s->press; d.thil = s->thil; d.wc = s->wc; d.wmc = s->wmc;
  d.vxe = s->vxe; d.vye = s->vye; d.vze = s->vze; d.vmc = s->vmc; d.vc = s->vc;
  d.vmasc = s->vmasc; d.wmasc = s->wmasc; d.alpha_press = s->alpha_press; d.pwfac = s->pwfac;
  d.pvfac = s->pvfac; d.thilt = s->thilt; d.vmxet = s->vmxet; d.vmyet = s->vmyet;
  d.vmzet = s->vmzet; d.vmt = s->vmt;
  return d;
}
static oracle::DynState<double> st64(const oracle_state64* s) {
  oracle::DynState<double> d;
  d.rho = s->rho; d.press = s->press; d.thil = s->thil; d.wc = s->wc; d.wmc = s->wmc;
  d.vxe = s->vxe; d.vye = s->vye; d.vze = s->vze; d.vmc = s->vmc; d.vc = s->vc;
  d.vmasc = s->vmasc; d.wmasc = s->wmasc; d.alpha_press = s->alpha_press; d.pwfac = s->pwfac;
  d.pvfac = s->pvfac; d.thilt = s->thilt; d.vmxet = s->vmxet; d.vmyet = s->vmyet;
  d.vmzet = s->vmzet; d.vmt = s->vmt;
  return d;
}

void oracle_dyn_set_eddy_f32(void* h, const olamgpu_eddy* e) {
  auto* X = (oracle::DynCtx<float>*)h;
  X->eddy = e;
  X->have_hk = false;
}
void oracle_dyn_set_eddy_f64(void* h, const olamgpu_eddy* e) {
  auto* X = (oracle::DynCtx<double>*)h;
  X->eddy = e;
  X->have_hk = false;
}
/* comp_horiz_k into the oracle's own arrays; copies them out as float or
 * double (akmodx, akhodx (mza, mva)) and int (kmtopv, khtopv (mva)) */
int oracle_comp_horiz_k_f32(void* h, const olamgpu_state* s, float* akmodx, float* akhodx, int* kmtopv, int* khtopv) {
  auto* X = (oracle::DynCtx<float>*)h;
  if (!X->eddy) return OLAMGPU_E_STATE;
  oracle::comp_horiz_k(*X, st32(s));
  std::copy(X->akmodx.begin(), X->akmodx.end(), akmodx);
  std::copy(X->akhodx.begin(), X->akhodx.end(), akhodx);
  std::copy(X->kmtopv.begin(), X->kmtopv.end(), kmtopv);
  std::copy(X->khtopv.begin(), X->khtopv.end(), khtopv);
  return OLAMGPU_OK;
}
int oracle_comp_horiz_k_f64(void* h, const oracle_state64* s, double* akmodx, double* akhodx, int* kmtopv,
                            int* khtopv) {
  auto* X = (oracle::DynCtx<double>*)h;
  if (!X->eddy) return OLAMGPU_E_STATE;
  oracle::comp_horiz_k(*X, st64(s));
  std::copy(X->akmodx.begin(), X->akmodx.end(), akmodx);
  std::copy(X->akhodx.begin(), X->akhodx.end(), akhodx);
  std::copy(X->kmtopv.begin(), X->kmtopv.end(), kmtopv);
  std::copy(X->khtopv.begin(), X->khtopv.end(), khtopv);
  return OLAMGPU_OK;
}

int oracle_prog_wrtv_rk_f32(void* h, const olamgpu_state* s, int istp) {
  return oracle::prog_wrtv_rk(*(oracle::DynCtx<float>*)h, st32(s), istp);
}
int oracle_prog_wrtv_rk_f64(void* h, const oracle_state64* s, int istp) {
  return oracle::prog_wrtv_rk(*(oracle::DynCtx<double>*)h, st64(s), istp);
}
void oracle_tend0_f32(void* h, const olamgpu_state* s, float* rho_old) {
  oracle::tend0(*(oracle::DynCtx<float>*)h, st32(s), rho_old);
}
void oracle_tend0_f64(void* h, const oracle_state64* s, double* rho_old) {
  oracle::tend0(*(oracle::DynCtx<double>*)h, st64(s), rho_old);
}
void oracle_timeavg_momsc_f32(void* h, const olamgpu_state* s) {
  oracle::timeavg_momsc(*(oracle::DynCtx<float>*)h, st32(s));
}
void oracle_timeavg_momsc_f64(void* h, const oracle_state64* s) {
  oracle::timeavg_momsc(*(oracle::DynCtx<double>*)h, st64(s));
}

}
