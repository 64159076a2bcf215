/*
 * oracle_common.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The oracle is a CPU restatement of martinjotte/OLAM v7.0's hot path, used
 * by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker and the CPU baseline.  It is never linked into, loaded by or
 * called from the product library (olam_b200/libolamgpu.so).
 *
 * PARITY UNPINNED: the reference is Fortran and no Fortran compiler exists
 * where this project builds or runs, and the reference ships no golden
 * vectors, known-answer files or fixtures for this path.  The restatement
 * follows the reference line by line (file:line cited at each function),
 * keeps OLAM's operation order, and keeps real(4)/real(8) as declared; it is
 * cross-checked by property tests and an independent numpy restatement.
 *
 * Templated on T, the type of OLAM's `real`: float is the reference
 * precision, double is the FP64 run (every real promoted, real(8) unchanged).
 * Arrays use OLAM's Fortran layout and 1-based indices through the F2/F3
 * accessors below; neighbour tables hold OLAM's 1-based point indices.
 */
#ifndef OLAM_ORACLE_COMMON_H
#define OLAM_ORACLE_COMMON_H

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

#include "../include/olamgpu.h"

namespace oracle {

/* Fortran (mza, n) array, 1-based (k, i) */
#define F2(a, k, i) (a)[(size_t)((i) - 1) * (size_t)mza + (size_t)((k) - 1)]

template <class T>
static std::vector<T> cvt(const float* p, size_t n) {
  std::vector<T> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = (T)p[i];
  return v;
}

template <class T>
static inline T fmax_(T a, T b) { return a > b ? a : b; }
template <class T>
static inline T fmin_(T a, T b) { return a < b ? a : b; }

/* Grid views in precision T (converted once per call). */
template <class T>
struct GridT {
  const olamgpu_grid* g;
  int mza, mwa, mva, mma;
  std::vector<T> dirv, volti, gxc, gyc, a_w, a_wu, xy_h, xy_hu;
  std::vector<T> dxps, dyps, xx0_v, xy0_v, yy0_v, xx0_vu, xy0_vu, yy0_vu;
  explicit GridT(const olamgpu_grid* gr) : g(gr) {
    mza = g->mza; mwa = g->mwa; mva = g->mva; mma = g->mma;
    dirv = cvt<T>(g->itab_w_dirv, (size_t)7 * mwa);
    volti = cvt<T>(g->volti, (size_t)mza * mwa);
    gxc = cvt<T>(g->gxps_coef, (size_t)7 * mwa);
    gyc = cvt<T>(g->gyps_coef, (size_t)7 * mwa);
    a_w = cvt<T>(g->a_w, (size_t)mza * 4);
    a_wu = cvt<T>(g->a_wu, (size_t)mza * 4);
    xy_h = cvt<T>(g->xy_h, (size_t)35 * mwa);
    xy_hu = cvt<T>(g->xy_hu, (size_t)35 * mwa);
    dxps = cvt<T>(g->dxps, (size_t)2 * mva);
    dyps = cvt<T>(g->dyps, (size_t)2 * mva);
    xx0_v = cvt<T>(g->xx0_v, (size_t)2 * mva);
    xy0_v = cvt<T>(g->xy0_v, (size_t)2 * mva);
    yy0_v = cvt<T>(g->yy0_v, (size_t)2 * mva);
    xx0_vu = cvt<T>(g->xx0_vu, (size_t)2 * mva);
    xy0_vu = cvt<T>(g->xy0_vu, (size_t)2 * mva);
    yy0_vu = cvt<T>(g->yy0_vu, (size_t)2 * mva);
  }
  /* itab_w(iw)%x(j) */
  int npoly(int iw) const { return g->npoly[iw - 1]; }
  int w_iv(int iw, int j) const { return g->itab_w_iv[(size_t)(iw - 1) * 7 + (j - 1)]; }
  int w_iw(int iw, int j) const { return g->itab_w_iw[(size_t)(iw - 1) * 7 + (j - 1)]; }
  int w_im(int iw, int j) const { return g->itab_w_im[(size_t)(iw - 1) * 7 + (j - 1)]; }
  T w_dirv(int iw, int j) const { return dirv[(size_t)(iw - 1) * 7 + (j - 1)]; }
  /* itab_v(iv)%iw(s) */
  int v_iw(int iv, int s) const { return g->itab_v_iw[(size_t)(iv - 1) * 2 + (s - 1)]; }
  int v_im(int iv, int s) const { return g->itab_v_im[(size_t)(iv - 1) * 2 + (s - 1)]; }
  T v2(const std::vector<T>& a, int s, int iv) const { return a[(size_t)(iv - 1) * 2 + (s - 1)]; }
  int lpw(int iw) const { return g->lpw[iw - 1]; }
  int lpv(int iv) const { return g->lpv[iv - 1]; }
  /* a_w(k, i, j) of a Fortran (mza, 2, 2) array */
  T aw(const std::vector<T>& a, int k, int i, int j) const {
    return a[(size_t)(k - 1) + (size_t)mza * ((i - 1) + 2 * (j - 1))];
  }
  /* xy_h(m, n, iw) of a Fortran (5, 7, mwa) array */
  T xyh(const std::vector<T>& a, int m, int n, int iw) const {
    return a[(size_t)(m - 1) + 5 * ((size_t)(n - 1) + 7 * (size_t)(iw - 1))];
  }
  T gxps_coef(int n, int iw) const { return gxc[(size_t)(iw - 1) * 7 + (n - 1)]; }
  T gyps_coef(int n, int iw) const { return gyc[(size_t)(iw - 1) * 7 + (n - 1)]; }
  T volti_(int k, int iw) const { return volti[(size_t)(iw - 1) * mza + (k - 1)]; }
};

}  // namespace oracle

#endif
