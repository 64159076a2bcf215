// setup.cu -- grid upload and table packing (host side of init_wrtv_rk's
// replacement).  OLAM's tables (mem_ijtabs.f90:60-144) arrive 1-based with
// packed derived-type members; the device keeps 0-based, padded copies.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "internal.h"

namespace olamgpu {

static int check_index(const int* a, size_t n, int lo, int hi, const char* what) {
  for (size_t i = 0; i < n; ++i)
    if (a[i] < lo || a[i] > hi) {
      set_error(std::string("grid table ") + what + " holds an index outside [" +
                std::to_string(lo) + "," + std::to_string(hi) + "] at " + std::to_string(i));
      return OLAMGPU_E_ARG;
    }
  return OLAMGPU_OK;
}

static int upload_list(DevBuf<int>& b, const int* h, int n, int maxv, const char* what,
                       cudaStream_t s) {
  if (n < 0 || (n > 0 && !h)) {
    set_error(std::string("loop table ") + what + " missing");
    return OLAMGPU_E_ARG;
  }
  OG_CHECK(check_index(h, (size_t)n, 2, maxv, what));
  std::vector<int> v(n > 0 ? n : 1, 0);
  for (int i = 0; i < n; ++i) v[i] = h[i] - 1;
  OG_CHECK(b.alloc(v.size()));
  OG_CUDA(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

int upload_grid(const olamgpu_grid* g, DevGrid& d, cudaStream_t s) {
  const int mza = g->mza, mwa = g->mwa, mva = g->mva, mma = g->mma;
  if (mza < 3 || mwa < 2 || mva < 2 || mma < 2) {
    set_error("grid sizes mza/mwa/mva/mma out of range");
    return OLAMGPU_E_ARG;
  }
  const void* need[] = {g->npoly, g->itab_w_iv, g->itab_w_iw, g->itab_w_dirv, g->itab_v_iw,
                        g->lpw, g->lpv, g->volti, g->a_w, g->a_wu, g->dxps, g->dyps,
                        g->gxps_coef, g->gyps_coef, g->xy_h, g->xy_hu, g->xx0_v, g->xy0_v,
                        g->yy0_v, g->xx0_vu, g->xy0_vu, g->yy0_vu, g->dzt_top, g->dzt_bot,
                        g->dzim};
  for (const void* p : need)
    if (!p) {
      set_error("olamgpu_grid has a NULL array the transport path needs");
      return OLAMGPU_E_ARG;
    }
  d.mza = mza; d.mwa = mwa; d.mva = mva; d.mma = mma;
  d.nw_prog = g->nw_prog; d.nw_wadj = g->nw_wadj;
  d.nv_prog = g->nv_prog; d.nv_wadj = g->nv_wadj; d.nm_prog = g->nm_prog;
  OG_CHECK(upload_list(d.jtw_prog, g->jtw_prog, g->nw_prog, mwa, "jtw_prog", s));
  OG_CHECK(upload_list(d.jtw_wadj, g->jtw_wadj, g->nw_wadj, mwa, "jtw_wadj", s));
  OG_CHECK(upload_list(d.jtv_prog, g->jtv_prog, g->nv_prog, mva, "jtv_prog", s));
  OG_CHECK(upload_list(d.jtv_wadj, g->jtv_wadj, g->nv_wadj, mva, "jtv_wadj", s));
  // a table that is a contiguous ascending run needs no reads on the device
  auto run_start = [](const int* t, int n) -> int {
    if (n <= 0 || !t) return -1;
    for (int j = 1; j < n; ++j) if (t[j] != t[0] + j) return -1;
    return t[0] - 1;
  };
  d.off_wprog = run_start(g->jtw_prog, g->nw_prog);
  d.off_vwadj = run_start(g->jtv_wadj, g->nv_wadj);
  d.off_vprog = run_start(g->jtv_prog, g->nv_prog);
  d.off_wwadj = run_start(g->jtw_wadj, g->nw_wadj);
  if (g->jtm_prog && g->nm_prog > 0)
    OG_CHECK(upload_list(d.jtm_prog, g->jtm_prog, g->nm_prog, mma, "jtm_prog", s));

  std::vector<char> isprog(mwa, 0);
  for (int j = 0; j < g->nw_prog; ++j) isprog[g->jtw_prog[j] - 1] = 1;
  {
    std::vector<int> np_list;
    for (int i = 0; i < mwa; ++i) if (!isprog[i]) np_list.push_back(i);
    d.n_nonprog = (int)np_list.size();
    if (!np_list.empty()) OG_CHECK(upload(d.w_nonprog, np_list.data(), np_list.size(), s));
    OG_CUDA(cudaStreamSynchronize(s));
  }

  // itab_w: npoly in [3,7]; indices checked for the first npoly entries.  A
  // column that is not prognosed (the outer halo of a rank's part of a
  // decomposed domain) may name the dummy point 1 for a neighbour or edge
  // the rank does not hold; the stages never read past such a column.
  std::vector<int> npoly(mwa), nb((size_t)mwa * 8), ev((size_t)mwa * 8), im((size_t)mwa * 8, 0);
  std::vector<float> dirv((size_t)mwa * 8, 0.f);
  for (int iw = 0; iw < mwa; ++iw) {
    int np = g->npoly[iw];
    if (iw == 0) np = 0;  // dummy point
    if (np < 0 || np > 7 || (iw > 0 && np < 3)) {
      set_error("npoly out of range at W point " + std::to_string(iw + 1));
      return OLAMGPU_E_ARG;
    }
    npoly[iw] = np;
    for (int j = 0; j < 8; ++j) {
      nb[(size_t)iw * 8 + j] = iw;
      ev[(size_t)iw * 8 + j] = 0;
    }
    for (int j = 0; j < np; ++j) {
      int wv = g->itab_w_iv[(size_t)iw * 7 + j], ww = g->itab_w_iw[(size_t)iw * 7 + j];
      const int lo = isprog[iw] ? 2 : 1;
      if (wv < lo || wv > mva || ww < lo || ww > mwa) {
        set_error("itab_w neighbour index out of range at W point " + std::to_string(iw + 1));
        return OLAMGPU_E_ARG;
      }
      ev[(size_t)iw * 8 + j] = wv - 1;
      nb[(size_t)iw * 8 + j] = ww - 1;
      dirv[(size_t)iw * 8 + j] = g->itab_w_dirv[(size_t)iw * 7 + j];
      if (g->itab_w_im) im[(size_t)iw * 8 + j] = g->itab_w_im[(size_t)iw * 7 + j] - 1;
    }
  }
  OG_CHECK(upload(d.npoly, npoly.data(), npoly.size(), s));
  OG_CHECK(upload(d.w_nb, nb.data(), nb.size(), s));
  OG_CHECK(upload(d.w_ev, ev.data(), ev.size(), s));
  OG_CHECK(upload(d.w_im, im.data(), im.size(), s));
  OG_CHECK(upload(d.w_dirv, dirv.data(), dirv.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));

  std::vector<int> viw((size_t)mva * 2), vim((size_t)mva * 2, 0);
  for (int iv = 0; iv < mva; ++iv)
    for (int k = 0; k < 2; ++k) {
      int w = g->itab_v_iw[(size_t)iv * 2 + k];
      if (iv > 0 && (w < 1 || w > mwa)) {
        set_error("itab_v%iw index out of range at V point " + std::to_string(iv + 1));
        return OLAMGPU_E_ARG;
      }
      viw[(size_t)iv * 2 + k] = iv > 0 ? w - 1 : 0;
      if (g->itab_v_im) vim[(size_t)iv * 2 + k] = iv > 0 ? g->itab_v_im[(size_t)iv * 2 + k] - 1 : 0;
    }
  OG_CHECK(upload(d.v_iw, viw.data(), viw.size(), s));
  OG_CHECK(upload(d.v_im, vim.data(), vim.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));

  if (g->itab_m_iv && g->itab_m_iw && g->itab_m_im) {
    std::vector<int> miv((size_t)mma * 3), miw((size_t)mma * 3), mim((size_t)mma * 3);
    for (size_t i = 0; i < (size_t)mma * 3; ++i) {
      miv[i] = std::max(g->itab_m_iv[i] - 1, 0);
      miw[i] = std::max(g->itab_m_iw[i] - 1, 0);
      mim[i] = std::max(g->itab_m_im[i] - 1, 0);
    }
    OG_CHECK(upload(d.m_iv, miv.data(), miv.size(), s));
    OG_CHECK(upload(d.m_iw, miw.data(), miw.size(), s));
    OG_CHECK(upload(d.m_im, mim.data(), mim.size(), s));
    OG_CUDA(cudaStreamSynchronize(s));
  }

  std::vector<int> lpw(mwa), lpv(mva);
  for (int i = 0; i < mwa; ++i) {
    int l = g->lpw[i];
    if (i > 0 && (l < 2 || l > mza)) {
      set_error("lpw out of range [2,mza] at W point " + std::to_string(i + 1));
      return OLAMGPU_E_ARG;
    }
    lpw[i] = (i > 0 ? l : 2) - 1;
  }
  for (int i = 0; i < mva; ++i) {
    int l = g->lpv[i];
    if (i > 0 && (l < 2 || l > mza)) {
      set_error("lpv out of range [2,mza] at V point " + std::to_string(i + 1));
      return OLAMGPU_E_ARG;
    }
    lpv[i] = (i > 0 ? l : 2) - 1;
  }
  d.h_lpw = lpw;
  OG_CHECK(upload(d.lpw, lpw.data(), lpw.size(), s));
  OG_CHECK(upload(d.lpv, lpv.data(), lpv.size(), s));
  if (g->lpm) {
    std::vector<int> lpm(mma);
    for (int i = 0; i < mma; ++i) lpm[i] = std::max(g->lpm[i] - 1, 1);
    OG_CHECK(upload(d.lpm, lpm.data(), lpm.size(), s));
  }
  if (g->iwglobe) OG_CHECK(upload(d.iwglobe, g->iwglobe, (size_t)mwa, s));
  OG_CUDA(cudaStreamSynchronize(s));

  OG_CHECK(upload(d.gxc, g->gxps_coef, (size_t)mwa * 7, s));
  OG_CHECK(upload(d.gyc, g->gyps_coef, (size_t)mwa * 7, s));
  OG_CHECK(upload(d.xy_h, g->xy_h, (size_t)mwa * 35, s));
  OG_CHECK(upload(d.xy_hu, g->xy_hu, (size_t)mwa * 35, s));
  OG_CHECK(upload(d.dxps, g->dxps, (size_t)mva * 2, s));
  OG_CHECK(upload(d.dyps, g->dyps, (size_t)mva * 2, s));
  OG_CHECK(upload(d.xx0_v, g->xx0_v, (size_t)mva * 2, s));
  OG_CHECK(upload(d.xy0_v, g->xy0_v, (size_t)mva * 2, s));
  OG_CHECK(upload(d.yy0_v, g->yy0_v, (size_t)mva * 2, s));
  OG_CHECK(upload(d.xx0_vu, g->xx0_vu, (size_t)mva * 2, s));
  OG_CHECK(upload(d.xy0_vu, g->xy0_vu, (size_t)mva * 2, s));
  OG_CHECK(upload(d.yy0_vu, g->yy0_vu, (size_t)mva * 2, s));
  OG_CHECK(upload(d.a_w, g->a_w, (size_t)mza * 4, s));
  OG_CHECK(upload(d.a_wu, g->a_wu, (size_t)mza * 4, s));
  OG_CHECK(upload(d.volti, g->volti, (size_t)mza * mwa, s));
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

// Per V face and side, the reconstruction folded into one weight per
// neighbour of the upwind cell: value = S(c) + sum_n w_n (S(nb_n) - S(c)).
// Restates scalar_v_column (scalar_transport_rk.F90:497-525) composed with
// grad_t2d (grad_lib.f90:236-269) / grad_t2d_quadratic (:278-341).
int build_fused_weights(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s) {
  const int mva = g->mva;
  std::vector<float> wb((size_t)mva * 16, 0.f), wu((size_t)mva * 16, 0.f);
  for (int iv = 1; iv < mva; ++iv) {
    for (int sd = 0; sd < 2; ++sd) {
      int c = g->itab_v_iw[(size_t)iv * 2 + sd] - 1;
      int np = g->npoly[c];
      double dx = g->dxps[(size_t)iv * 2 + sd], dy = g->dyps[(size_t)iv * 2 + sd];
      for (int n = 0; n < np; ++n) {
        double vb, vu;
        if (order == 2) {
          vb = dx * (double)g->gxps_coef[(size_t)c * 7 + n] + dy * (double)g->gyps_coef[(size_t)c * 7 + n];
          vu = vb;
        } else {
          const float* xb = g->xy_h + ((size_t)c * 7 + n) * 5;
          const float* xu = g->xy_hu + ((size_t)c * 7 + n) * 5;
          size_t e = (size_t)iv * 2 + sd;
          vb = dx * xb[0] + dy * xb[1] + (double)g->xx0_v[e] * xb[2] + (double)g->xy0_v[e] * xb[3] +
               (double)g->yy0_v[e] * xb[4];
          vu = dx * xu[0] + dy * xu[1] + (double)g->xx0_vu[e] * xu[2] + (double)g->xy0_vu[e] * xu[3] +
               (double)g->yy0_vu[e] * xu[4];
        }
        wb[((size_t)iv * 2 + sd) * 8 + n] = (float)vb;
        wu[((size_t)iv * 2 + sd) * 8 + n] = (float)vu;
      }
    }
  }
  OG_CHECK(upload(d.ew_b, wb.data(), wb.size(), s));
  OG_CHECK(upload(d.ew_u, wu.data(), wu.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));
  d.ew_order = order;

  // Per-column records of the fused kernel (layout in internal.h, COLREC_*).
  // For a hexagonal column c the cell u across face n shares c and the two
  // faces' neighbours nb[n-1], nb[n+1] with c's own list, so the upwind
  // reconstruction on u's side needs only npoly(u) - 3 further rows; their
  // indices and all folded weights are stored here.
  const int nprog = g->nw_prog;
  std::vector<int> rec((size_t)nprog * COLREC_WORDS, 0);
  auto fbits = [](float f) { int i; std::memcpy(&i, &f, 4); return i; };
  for (int j = 0; j < nprog; ++j) {
    int* r = &rec[(size_t)j * COLREC_WORDS];
    const int c = g->jtw_prog[j] - 1;
    const int np = g->npoly[c];
    r[COLREC_IW] = c;
    r[COLREC_NP] = np;
    r[COLREC_KB] = g->lpw[c] - 1;
    bool fast = (np == 6) && (g->lpw[c] == 2);
    int nbc[7], evc[7];
    for (int n = 0; n < np; ++n) {
      nbc[n] = g->itab_w_iw[(size_t)c * 7 + n] - 1;
      evc[n] = g->itab_w_iv[(size_t)c * 7 + n] - 1;
    }
    for (int n = 0; n < 7; ++n) {
      const bool v = n < np;
      const int iv = v ? evc[n] : 0;
      const int own = v ? ((g->itab_v_iw[(size_t)iv * 2] - 1 == c) ? 0 : 1) : 0;
      r[COLREC_NB + n] = v ? nbc[n] : c;
      r[COLREC_EV + n] = iv;
      r[COLREC_OWN + n] = own;
      r[COLREC_LPV + n] = v ? g->lpv[iv] - 1 : 0;
      if (v && g->lpv[iv] != 2) fast = false;
      r[COLREC_DV + n] = fbits(v ? g->itab_w_dirv[(size_t)c * 7 + n] : 0.f);
      for (int m = 0; m < 7; ++m)
        r[COLREC_WOWN + n * 7 + m] = fbits(v && m < np ? wb[((size_t)iv * 2 + own) * 8 + m] : 0.f);
    }
    for (int n = 0; n < 6 && fast; ++n) {
      const int u = nbc[n], iv = evc[n];
      const int own = r[COLREC_OWN + n];
      const int su = 1 - own;  // u's side of face n
      const int prev = nbc[(n + np - 1) % np], next = nbc[(n + 1) % np];
      float wc = 0.f, wp = 0.f, wn = 0.f, wnew[4] = {0.f, 0.f, 0.f, 0.f};
      int nidx[4] = {c, c, c, c}, nn = 0, hits = 0;
      const int npu = g->npoly[u];
      for (int m = 0; m < npu; ++m) {
        const int x = g->itab_w_iw[(size_t)u * 7 + m] - 1;
        const float w = wb[((size_t)iv * 2 + su) * 8 + m];
        if (x == c) { wc = w; ++hits; }
        else if (x == prev) { wp = w; ++hits; }
        else if (x == next) { wn = w; ++hits; }
        else if (nn < 3) { wnew[nn] = w; nidx[nn] = x; ++nn; }
        else { fast = false; }
      }
      if (hits != 3) fast = false;
      r[COLREC_WU + n * 7 + 0] = fbits(wc);
      r[COLREC_WU + n * 7 + 1] = fbits(wp);
      r[COLREC_WU + n * 7 + 2] = fbits(wn);
      for (int q = 0; q < 4; ++q) r[COLREC_WU + n * 7 + 3 + q] = fbits(q < 3 ? wnew[q] : 0.f);
      for (int q = 0; q < 3; ++q) r[COLREC_NEW + n * 3 + q] = nidx[q];
      r[COLREC_NNEW + n] = nn;
    }
    r[COLREC_FAST] = fast ? 1 : 0;
  }
  OG_CHECK(upload(d.colrec, rec.data(), rec.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}


// ---- tiles of the tiled fused kernel ------------------------------------------

size_t tile_smem_bytes(int T, int nu, int rb) {
  auto al = [](size_t b) { return (b + 127) & ~size_t(127); };
  // k_tile's layout (128-byte aligned parts after aligning the base): two
  // level barriers, two level buffers of U rows (rows in fours) and of the
  // tile columns' weight records, the U rows' global row indices, slot
  // offsets, tile columns, explicit fractions
  const size_t nu4 = (size_t)((nu + 3) & ~3);
  return 127 + 128 + 2 * al(nu4 * rb) + 2 * al((size_t)T * TILE_WR * 4) + al((size_t)(nu + 3) * 4) +
         al((size_t)T * TILE_NS * 4) + al((size_t)T * 4) + (size_t)T * 4;
}

// Two blocks per SM: 228 KB of shared memory less 1 KB reserved per block.
#define TILE_SMEM_MAX (113 * 1024)

// weight of the n-th neighbour of the cell on side sd of face iv in that
// side's reconstructed face value: S(cell) + sum_n w_n (S(nb_n) - S(cell))
// (grad_t2d: dxps*gxps_coef + dyps*gyps_coef; grad_t2d_quadratic folds the
// quadratic terms xx0_v.. with xy_h the same way; bounded coefficients)
static double face_weight(const olamgpu_grid* g, int order, int iv, int sd, int n) {
  const int c = g->itab_v_iw[(size_t)iv * 2 + sd] - 1;
  const size_t e = (size_t)iv * 2 + sd;
  const double dx = g->dxps[e], dy = g->dyps[e];
  if (order == 2) return dx * (double)g->gxps_coef[(size_t)c * 7 + n] + dy * (double)g->gyps_coef[(size_t)c * 7 + n];
  const float* x = g->xy_h + ((size_t)c * 7 + n) * 5;
  return dx * x[0] + dy * x[1] + (double)g->xx0_v[e] * x[2] + (double)g->xy0_v[e] * x[3] + (double)g->yy0_v[e] * x[4];
}

// Distance along a Hilbert curve filling a 2^b x 2^b grid (the published
// iterative construction: at each scale take the quadrant's index along the
// curve, then reflect and transpose the point into that quadrant's frame).
static unsigned long long hilbert_index(unsigned b, unsigned x, unsigned y) {
  unsigned long long d = 0;
  for (unsigned s = 1u << (b - 1); s > 0; s >>= 1) {
    const unsigned rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
    d += (unsigned long long)s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) { x = s - 1 - (x & (s - 1)); y = s - 1 - (y & (s - 1)); }
      std::swap(x, y);
    }
    x &= s - 1;
    y &= s - 1;
  }
  return d;
}

// The prognosed columns in an order of the library's own that keeps nearby
// columns together, whatever the caller's numbering: each column's unit
// normal (its position on the sphere) is projected onto the face of the
// circumscribing cube it points at, and the faces' points are ordered along
// a Hilbert curve.  Without the normals, jtw_prog's order.
std::vector<int> locality_order(const olamgpu_grid* g) {
  const int nprog = g->nw_prog;
  std::vector<int> cols(nprog);
  for (int j = 0; j < nprog; ++j) cols[j] = g->jtw_prog[j] - 1;
  if (!g->wnx || !g->wny || !g->wnz) return cols;
  const unsigned bits = 16;
  const double q = (double)(1u << bits);
  std::vector<std::pair<unsigned long long, int>> key(nprog);
  for (int j = 0; j < nprog; ++j) {
    const int c = cols[j];
    const double p[3] = {g->wnx[c], g->wny[c], g->wnz[c]};
    int ax = 0;
    for (int a = 1; a < 3; ++a) if (std::fabs(p[a]) > std::fabs(p[ax])) ax = a;
    const double m = std::fabs(p[ax]) > 0 ? std::fabs(p[ax]) : 1.0;
    const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
    auto cell = [&](double v) {
      const double t = (v / m + 1.0) * 0.5 * q;
      return (unsigned)std::min(std::max(t, 0.0), q - 1.0);
    };
    const unsigned face = (unsigned)(2 * ax + (p[ax] > 0 ? 1 : 0));
    key[j] = {((unsigned long long)face << 40) | hilbert_index(bits, cell(p[o1]), cell(p[o2])), c};
  }
  std::stable_sort(key.begin(), key.end(),
                   [](const std::pair<unsigned long long, int>& a, const std::pair<unsigned long long, int>& b) {
                     return a.first < b.first;
                   });
  for (int j = 0; j < nprog; ++j) cols[j] = key[j].second;
  return cols;
}

void make_tiles(const olamgpu_grid* g, int order, TileHost& th, int T_req, int nu_cap, int ord) {
  th = TileHost();
  if (order != 2 && order != 3) return;
  const int nprog = g->nw_prog, mwa = g->mwa;
  if (nprog <= 0) return;
  // tiles are runs of this order's columns: the library's curve (ord 0) or
  // the caller's jtw_prog (ord 1)
  std::vector<int> cols;
  if (ord == 1) {
    cols.resize(nprog);
    for (int j = 0; j < nprog; ++j) cols[j] = g->jtw_prog[j] - 1;
  } else {
    cols = locality_order(g);
  }
  for (int j = 0; j < nprog; ++j) {
    const int c = g->jtw_prog[j] - 1;
    if (g->npoly[c] < 3 || g->npoly[c] > 6) return;  // left to the column kernel
  }
  auto nbr = [&](int c, int n) { return g->itab_w_iw[(size_t)c * 7 + n] - 1; };
  // slot columns of cell c: its neighbours, then their other neighbours
  std::vector<int> slots;
  auto cell_slots = [&](int c) {
    slots.clear();
    auto add = [&](int x) {
      if (x == c) return;
      for (int y : slots) if (y == x) return;
      slots.push_back(x);
    };
    for (int n = 0; n < g->npoly[c]; ++n) add(nbr(c, n));
    const int n1 = (int)slots.size();
    for (int i = 0; i < n1; ++i)
      for (int n = 0; n < g->npoly[slots[i]]; ++n) add(nbr(slots[i], n));
  };
  for (int j = 0; j < nprog; ++j) {
    cell_slots(g->jtw_prog[j] - 1);
    if ((int)slots.size() > TILE_NS) return;   // left to the column kernel
  }
  std::vector<int> stamp(mwa, -1), loc(mwa, 0);
  std::vector<int> U;
  // Tiles are runs of at most T columns of the order above; a run closes
  // early where one more column would take its two-ring neighbourhood
  // beyond the cap (where the curve jumps between faces of the cube), so
  // that no outlier sets every block's shared memory.  tstart[t] is the
  // first column of tile t.
  std::vector<int> tstart;
  // the neighbourhood of columns [j0, j1) in U (local index of column x:
  // loc[x] while stamp[x] == t)
  auto gather_cols = [&](int t, int j0, int j1) {
    U.clear();
    auto add = [&](int x) {
      if (stamp[x] != t) { stamp[x] = t; loc[x] = (int)U.size(); U.push_back(x); }
    };
    for (int j = j0; j < j1; ++j) add(cols[j]);
    const int nt = (int)U.size();
    for (int i = 0; i < nt; ++i)
      for (int n = 0; n < g->npoly[U[i]]; ++n) add(nbr(U[i], n));
    const int nr1 = (int)U.size();
    for (int i = nt; i < nr1; ++i)
      for (int n = 0; n < g->npoly[U[i]]; ++n) add(nbr(U[i], n));
  };
  auto gather = [&](int t, int T) {
    gather_cols(t, tstart[t], std::min(nprog, std::min(tstart[t + 1], tstart[t] + T)));
  };
  // the runs for width Tc and cap (0: no cap); returns the largest neighbourhood
  std::vector<int> mark(mwa, 0), trial;
  auto form = [&](int Tc, int cap) -> int {
    tstart.clear();
    std::fill(mark.begin(), mark.end(), 0);
    int nu_max = 0, j = 0, epoch = 0;
    while (j < nprog) {
      tstart.push_back(j);
      ++epoch;   // mark[x] == epoch: x is in the run's neighbourhood
      int nu = 0, len = 0;
      while (j + len < nprog && len < Tc) {
        const int c = cols[j + len];
        // the cells of the candidate's two rings not yet in the neighbourhood
        trial.clear();
        auto count = [&](int x) {
          if (mark[x] != epoch) { mark[x] = epoch; trial.push_back(x); }
        };
        count(c);
        for (int n = 0; n < g->npoly[c]; ++n) count(nbr(c, n));
        for (int n = 0; n < g->npoly[c]; ++n) {
          const int x = nbr(c, n);
          for (int m = 0; m < g->npoly[x]; ++m) count(nbr(x, m));
        }
        if (cap > 0 && len > 0 && nu + (int)trial.size() > cap) {
          for (int x : trial) mark[x] = 0;   // the run ends before this column
          break;
        }
        nu += (int)trial.size();
        ++len;
      }
      nu_max = std::max(nu_max, nu);
      j += len;
    }
    tstart.push_back(nprog);
    return nu_max;
  };
  int T = 0, numax = 0;
  // one or two columns for each of the 16 half-warps of a block (64 tracers
  // per block: 256-byte rows), or the width asked for.  Neighbourhoods are
  // capped where the blocks of the widest rows the stage kernel runs on
  // tiles of this width fit an SM: two for 32 columns (64 tracers,
  // 256-byte rows) and 16 columns (128 tracers, 512-byte rows), three for
  // 8 columns (128 tracers: a warp per column, one column each), or at
  // nu_cap when given.  8-column tiles only when asked for.
  const int cand[] = {32, 16, 8};
  for (int Tc : cand) {
    if (T_req > 0 && Tc != T_req) continue;
    if (T_req <= 0 && Tc == 8) continue;
    int cap = nu_cap;
    if (cap <= 0) {
      const int rb = Tc == 32 ? 256 : 512;
      const size_t smax = Tc == 8 ? (size_t)(227 / 3 - 1) * 1024 : (size_t)TILE_SMEM_MAX;
      cap = 4;
      while (tile_smem_bytes(Tc, cap + 4, rb) <= smax) cap += 4;
    }
    const int nu = form(Tc, cap);
    std::fill(stamp.begin(), stamp.end(), -1);
    if (nu <= 65535 && (T_req > 0 || tile_smem_bytes(Tc, nu, 256) <= TILE_SMEM_MAX)) {
      T = Tc; numax = nu;
      break;
    }
  }
  if (!T) return;  // neighbourhoods too large: the column kernel runs
  const int ntiles = (int)tstart.size() - 1;
  std::vector<int>& hdr = th.hdr;
  std::vector<int>& ulist = th.ulist;
  std::vector<int>& tc = th.tc;
  std::vector<float>& am = th.a;
  hdr.assign((size_t)ntiles * 4, 0);
  tc.assign((size_t)ntiles * T * TILE_TCW, 0);
  am.assign((size_t)ntiles * T * TILE_AW, 0.f);
  std::vector<int>& rv = th.rev;
  rv.assign((size_t)ntiles * T * TILE_NS, 0);
  auto fbits = [](float f) { int i; std::memcpy(&i, &f, 4); return i; };
  std::fill(stamp.begin(), stamp.end(), -1);
  std::vector<double> acc(TILE_AW);
  // pair tables index U rows with bytes
  auto nU_fits_bytes = [](size_t n) { return n <= 256; };
  bool break_pairs = false;
  for (int t = 0; t < ntiles; ++t) {
    gather(t, T);
    const int u_off = (int)ulist.size();
    const int nT = tstart[t + 1] - tstart[t];
    hdr[(size_t)t * 4 + 0] = u_off;
    hdr[(size_t)t * 4 + 1] = (int)U.size();
    hdr[(size_t)t * 4 + 3] = nT;
    ulist.insert(ulist.end(), U.begin(), U.end());
    for (int i = 0; i < nT; ++i) {
      const int c = U[i];
      int* w = &tc[((size_t)t * T + i) * TILE_TCW];
      float* a = &am[((size_t)t * T + i) * TILE_AW];
      const int np = g->npoly[c];
      cell_slots(c);
      const int ns = (int)slots.size();
      auto slot_of = [&](int x) {
        for (int j = 0; j < ns; ++j) if (slots[j] == x) return j;
        return -1;
      };
      w[TILE_TC_IW] = c;
      w[TILE_TC_NP] = np;
      w[TILE_TC_NS] = ns;
      for (int j = 0; j < TILE_NS; ++j) w[TILE_TC_SLOT + j] = (j < ns ? loc[slots[j]] : i) * 256;
      int side = 0;
      for (int f = 0; f < 6; ++f) {
        const bool v = f < np;
        const int iv = v ? g->itab_w_iv[(size_t)c * 7 + f] - 1 : 0;
        const int sd = v ? ((g->itab_v_iw[(size_t)iv * 2] - 1 == c) ? 0 : 1) : 0;
        side |= sd << f;
        w[TILE_TC_EV + f] = iv;
        w[TILE_TC_DV + f] = fbits(v ? g->itab_w_dirv[(size_t)c * 7 + f] : 0.f);
      }
      w[TILE_TC_SIDE] = side;
      // device level of the lowest prognosed level of face iv
      auto lpv_of = [&](int iv) { return g->lpv[iv] - 1; };
      auto edge = [&](int x, int n) { return g->itab_w_iv[(size_t)x * 7 + n] - 1; };
      // the slot weights at level lev: a gradient term counts where its
      // face is above ground (grad_t2d skips k < lpv)
      auto fold = [&](int lev) {
        std::fill(acc.begin(), acc.end(), 0.0);
        for (int f = 0; f < np; ++f) {
          const int iv = w[TILE_TC_EV + f], sd = (side >> f) & 1;
          // the cell upwind: S(c) + sum_n w_n (S(nb_n(c)) - S(c))
          for (int n = 0; n < np; ++n)
            if (lpv_of(edge(c, n)) <= lev)
              acc[(f * 2 + 0) * TILE_NS + slot_of(nbr(c, n))] += face_weight(g, order, iv, sd, n);
          // the neighbour u upwind: (1 - sum_n w_n)(S(u) - S(c)) + sum_n w_n (S(nb_n(u)) - S(c))
          const int u = nbr(c, f), npu = g->npoly[u];
          double sw = 0.0;
          for (int n = 0; n < npu; ++n) {
            if (lpv_of(edge(u, n)) > lev) continue;
            const double wn = face_weight(g, order, iv, 1 - sd, n);
            sw += wn;
            const int x = nbr(u, n);
            if (x != c) acc[(f * 2 + 1) * TILE_NS + slot_of(x)] += wn;
          }
          acc[(f * 2 + 1) * TILE_NS + slot_of(u)] += 1.0 - sw;
        }
      };
      fold(std::numeric_limits<int>::max());
      for (int k = 0; k < TILE_AW; ++k) a[k] = (float)acc[k];
      // terrain bands: the levels above the column's floor at which a term
      // of its faces' reconstructions comes above ground
      std::vector<int> ls;
      const int kbc = g->lpw[c] - 1;
      for (int f = 0; f < np; ++f) {
        const int u = nbr(c, f);
        for (int n = 0; n < np; ++n) ls.push_back(lpv_of(edge(c, n)));
        for (int n = 0; n < g->npoly[u]; ++n) ls.push_back(lpv_of(edge(u, n)));
      }
      std::sort(ls.begin(), ls.end());
      ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
      ls.erase(std::remove_if(ls.begin(), ls.end(), [&](int l) { return l <= kbc || l >= g->mza; }), ls.end());
      w[TILE_TC_BOFF] = (int)(th.band_lev.size());
      w[TILE_TC_NB] = (int)ls.size();
      for (size_t b = 0; b < ls.size(); ++b) {
        fold(b == 0 ? kbc : ls[b - 1]);
        for (int k = 0; k < TILE_AW; ++k) th.band.push_back((float)acc[k]);
        th.band_lev.push_back(ls[b]);
      }
      // transposed slots: the cells that have c as a slot are c's own slot
      // cells (the relation "within two rings" is symmetric)
      int* r = &rv[((size_t)t * T + i) * TILE_NS];
      const std::vector<int> mine = slots;
      for (int e = 0; e < TILE_NS; ++e) r[e] = i * 256 + TILE_NS;
      for (int e = 0; e < (int)mine.size(); ++e) {
        const int x = mine[e];
        cell_slots(x);
        int jx = -1;
        for (int j = 0; j < (int)slots.size(); ++j) if (slots[j] == c) jx = j;
        if (jx < 0) { th = TileHost(); return; }   // not symmetric: leave the grid to the column kernel
        r[e] = loc[x] * 256 + jx;
      }
      slots = mine;
    }
    // 16-column tiles: the union tables of the column pairs (2p, 2p+1)
    if (T == 16 && th.pair.size() != (size_t)ntiles * 8 * TILE_PT) th.pair.assign((size_t)ntiles * 8 * TILE_PT, 0);
    if (T == 16 && nU_fits_bytes(U.size())) {
      for (int pp = 0; pp < 8; ++pp) {
        int* pt = &th.pair[((size_t)t * 8 + pp) * TILE_PT];
        const int ia = 2 * pp, ib = 2 * pp + 1;
        if (ia >= nT) { pt[1] = pt[2] = -1; continue; }
        const bool hasb = ib < nT;
        const int* wa = &tc[((size_t)t * T + ia) * TILE_TCW];
        const int* wb = hasb ? &tc[((size_t)t * T + ib) * TILE_TCW] : nullptr;
        const int nsa = wa[TILE_TC_NS], nsb = hasb ? wb[TILE_TC_NS] : 0;
        std::vector<int> rows;
        auto slot_row = [](const int* w, int j) { return w[TILE_TC_SLOT + j] / 256; };
        for (int j = 0; j < nsa; ++j) rows.push_back(slot_row(wa, j));
        for (int j = 0; j < nsb; ++j) rows.push_back(slot_row(wb, j));
        std::sort(rows.begin(), rows.end());
        rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
        rows.erase(std::remove_if(rows.begin(), rows.end(), [&](int r) { return r == ia || r == ib; }), rows.end());
        if ((int)rows.size() > TILE_PU) { th.pair.clear(); break; }
        auto find = [&](const int* w, int ns, int r) {
          for (int j = 0; j < ns; ++j) if (slot_row(w, j) == r) return j;
          return -1;
        };
        pt[0] = (int)rows.size();
        pt[1] = hasb ? find(wa, nsa, ib) : -1;
        pt[2] = hasb ? find(wb, nsb, ia) : -1;
        for (size_t e = 0; e < rows.size(); ++e) {
          const int ja = find(wa, nsa, rows[e]), jb = hasb ? find(wb, nsb, rows[e]) : -1;
          pt[4 + e] = rows[e] | ((ja + 1) << 8) | ((jb + 1) << 16);
        }
      }
    } else if (T == 16) {
      th.pair.clear();
    }
    if (T == 16 && th.pair.empty()) break_pairs = true;
  }
  if (break_pairs) th.pair.clear();
  th.T = T;
  th.ntiles = ntiles;
  th.nu_max = numax;
  th.order = order;
}

int build_tiles(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s, int T, int ord) {
  d.tile_T = d.ntiles = d.tile_nu_max = 0;
  d.tile_order = 0;
  d.tile_closed = false;
  d.tile_paired = false;
  ++d.tile_gen;
  d.tile_ord = ord;
  TileHost th;
  make_tiles(g, order, th, T, 0, ord);
  if (!th.T) return OLAMGPU_OK;
  OG_CHECK(upload(d.tile_hdr, th.hdr.data(), th.hdr.size(), s));
  OG_CHECK(upload(d.tile_u, th.ulist.data(), th.ulist.size(), s));
  OG_CHECK(upload(d.tile_a, th.a.data(), th.a.size(), s));
  OG_CHECK(upload(d.tile_rev, th.rev.data(), th.rev.size(), s));
  OG_CHECK(upload(d.tile_tc, th.tc.data(), th.tc.size(), s));
  d.tile_paired = false;
  d.tile_pair.release();
  if (!th.pair.empty()) {
    OG_CHECK(upload(d.tile_pair, th.pair.data(), th.pair.size(), s));
    d.tile_paired = true;
  }
  d.tile_band.release();
  d.tile_band_lev.release();
  if (!th.band_lev.empty()) {
    OG_CHECK(upload(d.tile_band, th.band.data(), th.band.size(), s));
    OG_CHECK(upload(d.tile_band_lev, th.band_lev.data(), th.band_lev.size(), s));
  }
  OG_CUDA(cudaStreamSynchronize(s));
  // closed: every column of every neighbourhood is prognosed (a global
  // domain), so the transposed slots cover every column a stage reads
  std::vector<char> isprog(g->mwa, 0);
  for (int j = 0; j < g->nw_prog; ++j) isprog[g->jtw_prog[j] - 1] = 1;
  d.tile_closed = std::all_of(th.ulist.begin(), th.ulist.end(), [&](int x) { return isprog[x] != 0; });
  d.tile_T = th.T;
  d.ntiles = th.ntiles;
  d.tile_nu_max = th.nu_max;
  d.tile_order = order;
  return OLAMGPU_OK;
}

// 32-column tiles along the library's curve for the adjoint's reverse stage
// (hdr, U list, tile-cell records, transposed slots); none if they do not
// fit in shared memory
int build_adj_tiles(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s) {
  auto& a = d.adj_tiles;
  a.T = a.ntiles = a.nu_max = 0;
  TileHost th;
  make_tiles(g, order, th, 32, 0, 0);
  if (th.T != 32) return OLAMGPU_OK;
  OG_CHECK(upload(a.hdr, th.hdr.data(), th.hdr.size(), s));
  OG_CHECK(upload(a.u, th.ulist.data(), th.ulist.size(), s));
  OG_CHECK(upload(a.tc, th.tc.data(), th.tc.size(), s));
  OG_CHECK(upload(a.rev, th.rev.data(), th.rev.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));
  a.T = th.T;
  a.ntiles = th.ntiles;
  a.nu_max = th.nu_max;
  a.order = order;
  return OLAMGPU_OK;
}

}  // namespace olamgpu
