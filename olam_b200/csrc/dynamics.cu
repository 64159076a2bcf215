// dynamics.cu -- the acoustic RK short step prog_wrtv_rk and its glue on the
// device (omodel/prog_wrtv_rk.f90:36-488, omodel/timestep.f90:430-612).
//
// Kernel per reference routine, each over the reference's loop table:
//   k_setup_w / k_setup_v   column set-up and Rayleigh terms   (prog_wrtv_rk.f90:166-303)
//   k_div_* / k_lap_w       divh_damp                          (vort_div_damp.f90:1-230)
//   k_vort_* / k_lap_m      vort_damp                          (vort_div_damp.f90:234-445)
//   k_vmca                  vmca and vmasc on the last stage   (prog_wrtv_rk.f90:320-368); the
//                           stage copies *_rk = *_short and vmca of the other stages are
//                           formed inside k_wrt_begs
//   k_upw4, k_grad_upv4     fluxes_wrtv for thil, vxe, vye, vze (:950-1129), the four
//                           fields of one stage in one launch each (the
//                           gradients and the V-face values in one pass over
//                           the W cells); on the last stage the fields with
//                           ithil_monot / iwind_monot > 0 take
//                           dynamics_monot.cu's values
//   k_wrt_begs              prog_wrt_begs (:494-884): one warp per column, lanes over
//                           levels for the explicit terms and for the
//                           tridiagonal solve (tridiffo, tridiag_lib.f90:10-36,
//                           by parallel cyclic reduction)
//   k_prog_v                prog_v_begs (:888-946)
//   k_vel_t3d               vel_t3d_hex (vel_t3d.f90:39-108)
// With eddy diffusion registered, dynamics_eddy.cu's k_eddy_w follows
// k_setup_w (the vertical and horizontal eddy terms of :214-251).
// Precision as declared by OLAM: rho, press and the implicit weights are
// double; every other field is float.  Device level kd = Fortran k - 1.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "transport_kernels.cuh"

namespace olamgpu {

struct DynK {
  int mza, mwa, mva, mma;
  const int* __restrict__ npoly;
  const int* __restrict__ w_nb;
  const int* __restrict__ w_ev;
  const float* __restrict__ w_dirv;
  const int* __restrict__ v_iw;
  const int* __restrict__ v_im;
  const int* __restrict__ m_iv;
  const int* __restrict__ m_im;
  const int* __restrict__ lpw;
  const int* __restrict__ lpv;
  const int* __restrict__ lpm;
  const float* __restrict__ volti;
  const float* __restrict__ a_w;
  // flat: lpw = lpv = 2 everywhere (device level 1), no table read needed;
  // off_*: the loop table is the contiguous run off, off + 1, ... (a
  // global domain), no table read needed; -1 otherwise
  int flat, off_w, off_vp, off_va;
};

// lowest device level of a W / V point; a loop table's j-th entry
#define LPW(i) (g.flat ? 1 : g.lpw[i])
#define LPV(i) (g.flat ? 1 : g.lpv[i])
#define WTAB(j) (g.off_w >= 0 ? g.off_w + (j) : prog[j])
#define VPTAB(j) (g.off_vp >= 0 ? g.off_vp + (j) : vprog[j])
#define VATAB(j) (g.off_va >= 0 ? g.off_va + (j) : vadj[j])

static DynK dynk(const DevGrid& d) {
  DynK k;
  k.mza = d.mza; k.mwa = d.mwa; k.mva = d.mva; k.mma = d.mma;
  k.npoly = d.npoly.p; k.w_nb = d.w_nb.p; k.w_ev = d.w_ev.p; k.w_dirv = d.w_dirv.p;
  k.v_iw = d.v_iw.p; k.v_im = d.v_im.p; k.m_iv = d.m_iv.p; k.m_im = d.m_im.p;
  k.lpw = d.lpw.p; k.lpv = d.lpv.p; k.lpm = d.lpm.p; k.volti = d.volti.p; k.a_w = d.a_w.p;
  k.flat = ctx().tp.flat ? 1 : 0;
  k.off_w = d.off_wprog; k.off_vp = d.off_vprog; k.off_va = d.off_vwadj;
  return k;
}

// thread per (table entry j, level kd); n * mza < 2^31 (dyn_setup checks)
#define PK(j, kd, n)                                               \
  const unsigned i_ = blockIdx.x * blockDim.x + threadIdx.x;       \
  if (i_ >= (unsigned)(n) * (unsigned)g.mza) return;               \
  const int j = (int)(i_ / (unsigned)g.mza), kd = (int)(i_ - (unsigned)j * (unsigned)g.mza);

// ---- column set-up (prog_wrtv_rk.f90:166-253) --------------------------------
struct SetupW {
  const double* rho; const float* thil; const float* wmc;
  const float* thilt; const float* vmxet; const float* vmyet; const float* vmzet;
  const double* volt;
  double* rho0; double* rth0; float* wmc0;
  float* sh_th; float* sh_vx; float* sh_vy; float* sh_vz;
  const float* rayf_cof; const float* dn01d; const float* th01d; int krayf_bot;
};

__global__ void k_setup_w(DynK g, const int* __restrict__ prog, int nprog, SetupW a) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  if (kd < LPW(iw)) return;
  const size_t x = (size_t)iw * g.mza + kd;
  const float v4 = (float)a.volt[x];
  a.rth0[x] = (double)a.thil[x] * a.rho[x];
  a.rho0[x] = a.rho[x];
  a.wmc0[x] = a.wmc[x];
  float th = a.thilt[x] * v4;
  if (a.rayf_cof && kd >= a.krayf_bot - 1)
    th = th + a.rayf_cof[kd] * a.dn01d[kd] * (a.th01d[kd] - a.thil[x]) * v4;
  a.sh_th[x] = th;
  a.sh_vx[x] = a.vmxet[x] * v4;
  a.sh_vy[x] = a.vmyet[x] * v4;
  a.sh_vz[x] = a.vmzet[x] * v4;
}

__global__ void k_setup_v(DynK g, const int* __restrict__ vprog, int nv, const float* __restrict__ vmc,
                          const float* __restrict__ vmt, float* __restrict__ vmc0, float* __restrict__ sh_vmt,
                          const float* __restrict__ rayf_cof, const float* __restrict__ vc03d,
                          const float* __restrict__ vc, const double* __restrict__ rho, int krayf_bot) {
  PK(j, kd, nv);
  const int iv = VPTAB(j);
  const size_t x = (size_t)iv * g.mza + kd;
  vmc0[x] = vmc[x];
  float v = vmt[x];
  if (rayf_cof && kd >= krayf_bot - 1) {
    const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
    const double t = (double)(rayf_cof[kd] * 0.5f) * (rho[(size_t)iw1 * g.mza + kd] + rho[(size_t)iw2 * g.mza + kd]) *
                     (double)(vc03d[x] - vc[x]);
    v = (float)((double)v + t);
  }
  sh_vmt[x] = v;
}

// ---- divh_damp ----------------------------------------------------------------
__global__ void k_div_fdivh(DynK g, const int* __restrict__ vprog, int nv, const float* __restrict__ arw0,
                            const float* __restrict__ dniv, const float* __restrict__ zfacit,
                            const float* __restrict__ dzit, const double* __restrict__ volt, double facth,
                            int level, float fact2, float* __restrict__ fdivh) {
  PK(j, kd, nv);
  const int iv = VPTAB(j);
  if (kd < LPV(iv)) return;
  const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  const double vmin = fmin(volt[(size_t)iw1 * g.mza + kd], volt[(size_t)iw2 * g.mza + kd]);
  double v;
  if (level > 1) {
    const float amin = fminf(arw0[iw1], arw0[iw2]);
    float pw = 1.f;
    for (int i = 0; i < level - 1; ++i) pw = pw * amin;
    const double factb = facth * (double)pw;
    v = factb * (double)dniv[iv] * (double)zfacit[kd] * (double)dzit[kd] * vmin * 1.0;
  } else {
    v = (double)fact2 * (double)dniv[iv] * (double)zfacit[kd] * (double)dzit[kd] * vmin;
  }
  fdivh[(size_t)iv * g.mza + kd] = (float)v;
}

// The saved div2d is not cleared: plane 1 accumulates onto what the previous
// call left there, as the Fortran does (vort_div_damp.f90:136-148).
__global__ void k_div_accum(DynK g, const int* __restrict__ prog, int nprog, const float* __restrict__ arv,
                            const float* __restrict__ vmc, float* __restrict__ div1) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  const size_t x = (size_t)iw * g.mza + kd;
  float d = div1[x];
  const int np = g.npoly[iw];
  for (int n = 0; n < np; ++n) {
    const int iv = g.w_ev[iw * 8 + n];
    if (kd >= LPV(iv))
      d = d - arv[(size_t)iv * g.mza + kd] * g.w_dirv[iw * 8 + n] * vmc[(size_t)iv * g.mza + kd];
  }
  if (kd >= LPW(iw)) d = d * g.volti[x];
  div1[x] = d;
}

// laplacian2d (grad_lib.f90:494-524)
__global__ void k_lap_w(DynK g, const int* __restrict__ prog, int nprog, const float* __restrict__ xx_yy,
                        const float* __restrict__ src, float* __restrict__ dst) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  const size_t x = (size_t)iw * g.mza + kd;
  float d = 0.f;
  const int np = g.npoly[iw];
  for (int n = 0; n < np; ++n) {
    const int iv = g.w_ev[iw * 8 + n], iwn = g.w_nb[iw * 8 + n];
    if (kd >= LPV(iv)) d = d + (src[(size_t)iwn * g.mza + kd] - src[x]) * xx_yy[iw * 7 + n];
  }
  dst[x] = d;
}

__global__ void k_div_apply(DynK g, const int* __restrict__ vprog, int nv, const float* __restrict__ fdivh,
                            const float* __restrict__ dh, float* __restrict__ vmt) {
  PK(j, kd, nv);
  const int iv = VPTAB(j);
  if (kd < LPV(iv)) return;
  const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  const size_t x = (size_t)iv * g.mza + kd;
  vmt[x] = vmt[x] + fdivh[x] * (dh[(size_t)iw2 * g.mza + kd] - dh[(size_t)iw1 * g.mza + kd]);
}

// ---- vort_damp ----------------------------------------------------------------
__global__ void k_vort_first_m(DynK g, const int* __restrict__ mprog, int nm, const float* __restrict__ dnv,
                               const float* __restrict__ arm0, float* __restrict__ vfact,
                               int* __restrict__ lpmmin) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nm) return;
  const int im = mprog[j];
  int lm = 1 << 30;
  for (int jv = 0; jv < 3; ++jv) lm = min(lm, LPV(g.m_iv[im * 3 + jv]));
  lpmmin[im] = lm;
  for (int jv = 0; jv < 3; ++jv) {
    const int iv = g.m_iv[im * 3 + jv];
    const float v = dnv[iv] / arm0[im];
    vfact[im * 3 + jv] = (g.v_im[iv * 2 + 1] == im) ? v : -v;
  }
}

__global__ void k_vort_first_v(DynK g, const int* __restrict__ vprog, int nv, const float* __restrict__ dniu,
                               const float* __restrict__ arm0, float dtm_f, float fact, int level,
                               float* __restrict__ fvorth, float* __restrict__ fvortl) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nv) return;
  const int iv = VPTAB(j);
  const int im1 = g.v_im[iv * 2], im2 = g.v_im[iv * 2 + 1];
  const float a = -fact * fminf(arm0[im1], arm0[im2]);
  float ph = 1.f, pl = 1.f;
  for (int i = 0; i < level; ++i) ph = ph * a;
  for (int i = 0; i < level - 1; ++i) pl = pl * a;
  fvorth[iv] = 0.50f * dniu[iv] / dtm_f * ph;
  fvortl[iv] = (level > 2) ? 0.50f * dniu[iv] / dtm_f * pl : 0.f;
}

__global__ void k_vort(DynK g, const int* __restrict__ mprog, int nm, const float* __restrict__ vfact,
                       const float* __restrict__ vc, float* __restrict__ v1) {
  PK(j, kd, nm);
  const int im = mprog[j];
  float v = 0.f;
  for (int jv = 0; jv < 3; ++jv) {
    const int iv = g.m_iv[im * 3 + jv];
    if (kd >= LPV(iv)) v = v + vc[(size_t)iv * g.mza + kd] * vfact[im * 3 + jv];
  }
  v1[(size_t)im * g.mza + kd] = v;
}

// laplacian_m (grad_lib.f90:531-559)
__global__ void k_lap_m(DynK g, const int* __restrict__ mprog, int nm, const float* __restrict__ xx_yy_m,
                        const float* __restrict__ src, float* __restrict__ dst) {
  PK(j, kd, nm);
  const int im = mprog[j];
  const size_t x = (size_t)im * g.mza + kd;
  float d = 0.f;
  for (int jj = 0; jj < 3; ++jj) {
    const int imn = g.m_im[im * 3 + jj];
    if (kd >= LPV(g.m_iv[im * 3 + jj])) d = d + (src[(size_t)imn * g.mza + kd] - src[x]) * xx_yy_m[im * 3 + jj];
  }
  dst[x] = d;
}

__global__ void k_vort_apply(DynK g, const int* __restrict__ vprog, int nv, int level,
                             const float* __restrict__ fvorth, const float* __restrict__ fvortl,
                             const float* __restrict__ dl, const float* __restrict__ dh,
                             const double* __restrict__ rho, float* __restrict__ vmt) {
  PK(j, kd, nv);
  const int iv = VPTAB(j);
  if (kd < LPV(iv)) return;
  const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  const int im1 = g.v_im[iv * 2], im2 = g.v_im[iv * 2 + 1];
  const float rr = (float)(rho[(size_t)iw1 * g.mza + kd] + rho[(size_t)iw2 * g.mza + kd]);
  const size_t x = (size_t)iv * g.mza + kd;
  if (level == 1) {
    vmt[x] = vmt[x] + fvorth[iv] * (dh[(size_t)im2 * g.mza + kd] - dh[(size_t)im1 * g.mza + kd]) * rr;
    return;
  }
  const int ka = (level == 3) ? max(g.lpm[im1], g.lpm[im2]) : LPV(iv);
  if (kd < ka)
    vmt[x] = vmt[x] + fvortl[iv] * (dl[(size_t)im2 * g.mza + kd] - dl[(size_t)im1 * g.mza + kd]) * rr;
  else
    vmt[x] = vmt[x] + fvorth[iv] * (dh[(size_t)im2 * g.mza + kd] - dh[(size_t)im1 * g.mza + kd]) * rr;
}

// ---- stage kernels ----------------------------------------------------------------
__global__ void k_vmca(DynK g, const int* __restrict__ vadj, int nv, const float* __restrict__ vmc,
                       const float* __restrict__ arv, float* __restrict__ vmca, float* __restrict__ vmasc,
                       int last) {
  PK(j, kd, nv);
  const int iv = VATAB(j);
  if (kd < LPV(iv)) return;
  const size_t x = (size_t)iv * g.mza + kd;
  const float v = vmc[x] * arv[x];
  vmca[x] = v;
  if (last) vmasc[x] = vmasc[x] + v;
}

struct Four { const float* f[4]; };

struct VSide { const float* dxps; const float* dyps; const float* xx0_v; const float* xy0_v; const float* yy0_v; };

// The horizontal face values of fluxes_wrtv (prog_wrtv_rk.f90:973-1075) in
// one pass over the W cells: grad_t2d (ORD 2) or grad_t2d_quadratic with
// bounded=.false. (ORD 3) of the fields in gmask, kept in registers, then
// scalar_v_column for the faces this cell is upwind of -- side 1 of the
// face unless vmc < 0 -- each face being written by exactly one of its two
// cells: S(k,iw) + dxps dS/dx + dyps dS/dy (+ the quadratic terms at ORD 3)
// for the fields in gmask, S(k,iw) alone for those in pmask.  No gradient
// planes go through memory.  Thread per (column, level); the neighbour loop
// is outside the field loop, so each neighbour's table entries and
// coefficients are read once for the four fields.
template <int ORD>
__global__ void __launch_bounds__(256, ORD == 2 ? 6 : 1)   // order 2: 40 registers, six blocks per SM
k_grad_upv4(DynK g, const int* __restrict__ prog, int nprog, Four s, unsigned gmask,
                            unsigned pmask, const float* __restrict__ cx, const float* __restrict__ cy,
                            const float* __restrict__ xy_hu, VSide c, const float* __restrict__ vmc,
                            float* __restrict__ upv) {
  PK(j, kd, nprog);
  constexpr int NPL = ORD == 2 ? 2 : 5;
  const int iw = WTAB(j);
  const unsigned mza = g.mza;
  const size_t vplane = (size_t)g.mva * mza;
  const unsigned x = (unsigned)iw * mza + kd;
  const int np = g.npoly[iw];
  float c0[4], a[4][NPL];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    c0[f] = (((gmask | pmask) >> f) & 1u) ? s.f[f][x] : 0.f;
#pragma unroll
    for (int m = 0; m < NPL; ++m) a[f][m] = 0.f;
  }
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    if (n >= np) break;
    const int iv = g.w_ev[iw * 8 + n], iwn = g.w_nb[iw * 8 + n];
    if (kd < LPV(iv)) continue;
    float w[NPL];
    if (ORD == 2) {
      w[0] = cx[iw * 7 + n];
      w[1] = cy[iw * 7 + n];
    } else {
#pragma unroll
      for (int m = 0; m < NPL; ++m) w[m] = xy_hu[((size_t)iw * 7 + n) * 5 + m];
    }
    const unsigned xn = (unsigned)iwn * mza + kd;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      if (!((gmask >> f) & 1u)) continue;
      const float d = s.f[f][xn] - c0[f];
#pragma unroll
      for (int m = 0; m < NPL; ++m) a[f][m] = a[f][m] + w[m] * d;
    }
  }
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    if (n >= np) break;
    const int iv = g.w_ev[iw * 8 + n];
    if (kd < LPV(iv)) continue;
    const unsigned xv = (unsigned)iv * mza + kd;
    const int side = g.v_iw[iv * 2] == iw ? 0 : 1;
    if ((vmc[xv] < 0.f) != (side == 1)) continue;   // the other cell is upwind
    const float dx = c.dxps[iv * 2 + side], dy = c.dyps[iv * 2 + side];
    float xx = 0.f, xy = 0.f, yy = 0.f;
    if (ORD == 3) { xx = c.xx0_v[iv * 2 + side]; xy = c.xy0_v[iv * 2 + side]; yy = c.yy0_v[iv * 2 + side]; }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      if (!(((gmask | pmask) >> f) & 1u)) continue;
      float v = c0[f];
      if ((gmask >> f) & 1u) {
        v = v + dx * a[f][0] + dy * a[f][1];
        if (ORD == 3) v = v + xx * a[f][2] + xy * a[f][3] + yy * a[f][4];
      }
      upv[(size_t)f * vplane + xv] = v;
    }
  }
}

// vertical upwind face values of the four fields (scalar_w_column of
// fluxes_wrtv, prog_wrtv_rk.f90:1085-1126): thread per (column, face kd)
__global__ void k_upw4(DynK g, const int* __restrict__ prog, int nprog, Four s, const float* __restrict__ wmc,
                       float* __restrict__ upw) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  const int kb = LPW(iw);
  const int mza = g.mza;
  if (kd < kb - 1) return;
  const size_t plane = (size_t)g.mwa * mza;
  const size_t cb = (size_t)iw * mza;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float* S = s.f[f] + cb;
    float v;
    if (kd == kb - 1) v = S[kb];
    else if (kd == mza - 1) v = S[mza - 1];
    else {
      const bool down = wmc[cb + kd] < 0.f;
      const int lev = down ? kd + 1 : kd;
      const float b = S[lev];
      const float dsk = (lev <= mza - 2) ? S[lev + 1] - b : 0.f;
      const float dskm1 = (lev >= kb + 1) ? b - S[lev - 1] : 0.f;
      const float c1 = g.a_w[lev + (down ? 0 : 2 * mza)];
      const float c2 = g.a_w[lev + (down ? mza : 3 * mza)];
      v = b + dsk * c1 + dskm1 * c2;
    }
    upw[(size_t)f * plane + cb + kd] = v;
  }
}

// ---- prog_wrt_begs: one warp per column ------------------------------------------
struct WrtArgs {
  int istage, nrk;
  double dt8;
  float dts, fcoriol, c8, c9, rocv;
  double pc2, pc3, fr;
  const int* prog; int nprog;
  const float* vmc; const float* arv;                       // vmca = vmc arv
  const float* upv; const float* upw;                       // 4-field arrays
  const float* sh_th; const float* sh_vx; const float* sh_vy; const float* sh_vz;   // *_rk at stage start
  float* rk_vx; float* rk_vy; float* rk_vz;
  double* rho; double* press; const double* rho0; const double* rth0;
  float* thil; float* wc; float* wmc; const float* wmc0; const float* vxe; const float* vye;
  float* wmasc;
  const float* alpha_press; const float* pwfac;
  const double* volt; const float* volwi; const float* arw; const float* wn;
  const double* gdz_wgtm8; const double* gdz_wgtp8; const float* gdz_wgtm; const float* gdz_wgtp;
  const double* zwgt_bot8; const double* zwgt_top8; const float* b20;
};

#define WRT_WARPS 4
// per-warp shared scratch, arrays of mza entries
struct WrtSmem {
  double *hflx, *rt, *b10, *b5, *drt, *pex, *rex, *rhon;
  float *b15, *rkx, *rky, *rkz, *b31, *b32, *b33, *dwm, *wmf;
};

// The W system of prog_wrt_begs, b31(k) x(k-1) + b32(k) x(k) + b33(k) x(k+1)
// = dwm(k) for k = k0 .. k1, which the reference solves with the Thomas
// algorithm (tridiffo, outils/tridiag_lib.f90:10-36), solved here by
// parallel cyclic reduction over a warp: row i = k - k0 is updated by lane
// i % 32 (R rows per lane, i = lane + 32 r); in a step of stride s every row
// eliminates its couplings to rows i - s and i + s with those rows' current
// equations (rows outside the system act as identity rows), so after
// ceil(log2(n)) steps each row holds x(k) = d / b.  A lane keeps its rows'
// equations in registers and publishes, per step, a, c, d and 1 / b of each
// in the column's shared memory for the rows that eliminate against it (one
// division per row and step).  The equations are FP64 (the inputs and the
// result are the reference's real(4)): w is a small residual of large
// terms, and FP64 keeps it nearer the exact solve than a real(4) sweep.  The
// four FP64 arrays reuse pex and rex (not read after phase 2) and the float
// coefficient arrays themselves (read into registers first).
template <int R>
__device__ __forceinline__ void warp_tridiag(WrtSmem& m, int k0, int k1, int lane) {
  const int n = k1 - k0 + 1;
  double* A = m.pex;
  double* RB = m.rex;                               // 1 / b
  double* Cc = reinterpret_cast<double*>(m.b31);   // b31 and b32: 2 mza floats
  double* D = reinterpret_cast<double*>(m.b33);    // b33 and dwm
  double ra[R], rb[R], rc[R], rd[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane + 32 * r;
    ra[r] = i < n && i > 0 ? (double)m.b31[k0 + i] : 0.0;
    rb[r] = i < n ? (double)m.b32[k0 + i] : 1.0;
    rc[r] = i < n - 1 ? (double)m.b33[k0 + i] : 0.0;
    rd[r] = i < n ? (double)m.dwm[k0 + i] : 0.0;
  }
  __syncwarp();
  for (int s = 1; s < n; s <<= 1) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + 32 * r;
      if (i < n) { A[i] = ra[r]; RB[i] = 1.0 / rb[r]; Cc[i] = rc[r]; D[i] = rd[r]; }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + 32 * r;
      if (i >= n) continue;
      const int im = i - s, ip = i + s;
      double al = 0.0, ga = 0.0, am = 0.0, cm = 0.0, dm = 0.0, ap = 0.0, cp = 0.0, dp = 0.0;
      if (im >= 0) { al = -ra[r] * RB[im]; am = A[im]; cm = Cc[im]; dm = D[im]; }
      if (ip < n) { ga = -rc[r] * RB[ip]; ap = A[ip]; cp = Cc[ip]; dp = D[ip]; }
      rb[r] = rb[r] + al * cm + ga * ap;
      rd[r] = rd[r] + al * dm + ga * dp;
      ra[r] = al * am;
      rc[r] = ga * cp;
    }
    __syncwarp();
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane + 32 * r;
    if (i < n) m.wmf[k0 + i] = (float)(rd[r] / rb[r]);
  }
}

__global__ void __launch_bounds__(WRT_WARPS * 32, 8) k_wrt_begs(DynK g, WrtArgs A) {
  extern __shared__ double wsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * WRT_WARPS + warp;
  if (j >= A.nprog) return;
  const int mza = g.mza;
  double* base = wsm + (size_t)warp * mza * 13;  // 8 double + 9 float arrays (9 floats <= 5 doubles)
  WrtSmem m;
  m.hflx = base; m.rt = base + mza; m.b10 = base + 2 * mza; m.b5 = base + 3 * mza; m.drt = base + 4 * mza;
  m.pex = base + 5 * mza; m.rex = base + 6 * mza; m.rhon = base + 7 * mza;
  float* fb = reinterpret_cast<float*>(base + 8 * mza);
  m.b15 = fb; m.rkx = fb + mza; m.rky = fb + 2 * mza; m.rkz = fb + 3 * mza; m.b31 = fb + 4 * mza;
  m.b32 = fb + 5 * mza; m.b33 = fb + 6 * mza; m.dwm = fb + 7 * mza; m.wmf = fb + 8 * mza;

  const int iw = A.prog[j];
  const int kb = LPW(iw);
  const int np = g.npoly[iw];
  const size_t cb = (size_t)iw * mza;
  const size_t wplane = (size_t)g.mwa * mza, vplane = (size_t)g.mva * mza;
  const float* thil_upw = A.upw;
  const float* vxe_upw = A.upw + wplane;
  const float* vye_upw = A.upw + 2 * wplane;
  const float* vze_upw = A.upw + 3 * wplane;
  const float wnx = A.wn[iw * 3], wny = A.wn[iw * 3 + 1], wnz = A.wn[iw * 3 + 2];
  // the column's edges, read once: V point, with the sign bit set where the
  // edge's dirv is not positive; -1 past npoly
  int ev[7];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    const int iv = n < np ? g.w_ev[iw * 8 + n] : -1;
    ev[n] = (iv >= 0 && !(g.w_dirv[iw * 8 + n] > 0.f)) ? (iv | (int)0x80000000) : iv;
  }

  // phase 1: horizontal sums, Coriolis and explicit density / rho*thil terms
  for (int kd = kb + lane; kd < mza; kd += 32) {
    double hf = 0.0;
    // *_rk start each stage as *_short (prog_wrtv_rk.f90:320-330)
    float th = A.sh_th[cb + kd], vx = A.sh_vx[cb + kd], vy = A.sh_vy[cb + kd], vz = A.sh_vz[cb + kd];
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      if (ev[n] == -1) break;
      const int iv = ev[n] & 0x7fffffff;
      if (kd < LPV(iv)) continue;
      const size_t xv = (size_t)iv * mza + kd;
      const float vm = A.vmc[xv] * A.arv[xv];
      const float u0 = A.upv[xv], u1 = A.upv[vplane + xv], u2 = A.upv[2 * vplane + xv],
                  u3 = A.upv[3 * vplane + xv];
      if (ev[n] >= 0) {
        hf = hf + (double)vm;
        th = th + vm * u0;
        vx = vx + vm * u1;
        vy = vy + vm * u2;
        vz = vz + vm * u3;
      } else {
        hf = hf - (double)vm;
        th = th - vm * u0;
        vx = vx - vm * u1;
        vy = vy - vm * u2;
        vz = vz - vm * u3;
      }
    }
    const double rho = A.rho[cb + kd];
    const float mass = (float)(rho * A.volt[cb + kd]);
    vx = vx + mass * A.fcoriol * A.vye[cb + kd];
    vy = vy - mass * A.fcoriol * A.vxe[cb + kd];
    const double rt = rho * (double)A.thil[cb + kd];
    const double b10 = A.dt8 * (double)g.volti[cb + kd];
    const double b5 = (double)(A.alpha_press[cb + kd] * powf((float)rt, A.rocv));
    double drho = b10 * hf;
    double drt = b10 * (double)th;
    if (A.istage > 1) {
      drho = drho + A.rho0[cb + kd] - rho;
      drt = drt + A.rth0[cb + kd] - rt;
    }
    m.hflx[kd] = hf; m.rt[kd] = rt; m.b10[kd] = b10; m.b5[kd] = b5; m.drt[kd] = drt;
    m.pex[kd] = b5 * (rt + A.pc2 * drt);
    m.rex[kd] = rho + A.fr * drho;
    m.b15[kd] = (float)(b10 * b5);
    m.rkx[kd] = vx; m.rky[kd] = vy; m.rkz[kd] = vz;
  }
  __syncwarp();
  // phase 2: explicit W momentum and the tridiagonal coefficients (faces kb..mza-2)
  for (int kd = kb + lane; kd <= mza - 2; kd += 32) {
    const size_t x = cb + kd;
    const float a = (float)(m.pex[kd] - m.pex[kd + 1]) * A.pwfac[x];
    const float b = (float)(A.gdz_wgtm8[kd] * m.rex[kd] + A.gdz_wgtp8[kd] * m.rex[kd + 1]);
    const float c = (wnx * (m.rkx[kd] + m.rkx[kd + 1]) + wny * (m.rky[kd] + m.rky[kd + 1]) +
                     wnz * (m.rkz[kd] + m.rkz[kd + 1])) * A.volwi[x];
    m.dwm[kd] = A.wmc0[x] + A.dts * (a - b + c);
    const float b7 = A.dts * A.volwi[x];
    const float b8 = A.c8 * A.pwfac[x];
    const float b21 = b7 * A.wc[x - 1];
    const float b22 = b7 * A.wc[x + 1];
    const float b23 = b8 * m.b15[kd];
    const float b24 = b8 * m.b15[kd + 1];
    const float b25 = A.c9 * g.volti[x] * A.gdz_wgtm[kd];
    const float b26 = A.c9 * g.volti[x + 1] * A.gdz_wgtp[kd];
    m.b31[kd] = -A.arw[x - 1] * (b21 + b25 + b23 * thil_upw[x - 1]);
    m.b32[kd] = A.b20[kd] + A.arw[x] * (b25 - b26 + (b23 + b24) * thil_upw[x]);
    m.b33[kd] = A.arw[x + 1] * (b22 + b26 - b24 * thil_upw[x + 1]);
  }
  __syncwarp();
  // phase 3: tridiffo's system (faces kb..mza-2) by cyclic reduction across
  // the warp's lanes
  if (kb <= mza - 2) {
    if (mza - 1 - kb <= 64) warp_tridiag<2>(m, kb, mza - 2, lane);
    else warp_tridiag<4>(m, kb, mza - 2, lane);   // mza <= 128
  }
  __syncwarp();
  // phase 4: implicit fluxes and the updates of rho, press, thil and vm*et_rk
  for (int kd = kb + lane; kd < mza; kd += 32) {
    const size_t x = cb + kd;
    const float wma = (kd <= mza - 2) ? m.wmf[kd] * A.arw[x] : 0.f;
    const float wmam = (kd - 1 >= kb) ? m.wmf[kd - 1] * A.arw[x - 1] : 0.f;
    const double vft = (kd <= mza - 2) ? (double)(wma * thil_upw[x]) : 0.0;
    const double vftm = (kd - 1 >= kb) ? (double)(wmam * thil_upw[x - 1]) : 0.0;
    const float vfx = (kd <= mza - 2) ? wma * vxe_upw[x] : 0.f;
    const float vfxm = (kd - 1 >= kb) ? wmam * vxe_upw[x - 1] : 0.f;
    const float vfy = (kd <= mza - 2) ? wma * vye_upw[x] : 0.f;
    const float vfym = (kd - 1 >= kb) ? wmam * vye_upw[x - 1] : 0.f;
    const float vfz = (kd <= mza - 2) ? wma * vze_upw[x] : 0.f;
    const float vfzm = (kd - 1 >= kb) ? wmam * vze_upw[x - 1] : 0.f;
    if (A.istage == A.nrk && kd <= mza - 2) A.wmasc[x] = A.wmasc[x] + wma;
    const double rhon = A.rho0[x] + A.dt8 * (double)g.volti[x] * (m.hflx[kd] + (double)wmam - (double)wma);
    A.rho[x] = rhon;
    m.rhon[kd] = rhon;
    const double drt = m.drt[kd] + m.b10[kd] * (vftm - vft);
    A.press[x] = m.b5[kd] * (m.rt[kd] + A.pc3 * drt);
    A.thil[x] = (float)((m.rt[kd] + drt) / rhon);
    A.rk_vx[x] = m.rkx[kd] + vfxm - vfx;
    A.rk_vy[x] = m.rky[kd] + vfym - vfy;
    A.rk_vz[x] = m.rkz[kd] + vfzm - vfz;
  }
  __syncwarp();
  // phase 5: W momentum and velocity, bottom values
  for (int kd = kb + lane; kd <= mza - 2; kd += 32) {
    const size_t x = cb + kd;
    const float wf = m.wmf[kd];
    A.wmc[x] = wf;
    A.wc[x] = wf / (float)(A.zwgt_bot8[kd] * m.rhon[kd] + A.zwgt_top8[kd] * m.rhon[kd + 1]);
  }
  __syncwarp();
  if (lane == 0) {
    A.wc[cb + kb - 1] = A.wc[cb + kb];
    const float t = A.thil[cb + kb];
    for (int kd = 0; kd < kb; ++kd) A.thil[cb + kd] = t;
  }
}

// prog_v_begs (prog_wrtv_rk.f90:888-946)
__global__ void k_prog_v(DynK g, const int* __restrict__ vprog, int nv, float dts, const float* __restrict__ vmc0,
                         const float* __restrict__ vmt_short, const double* __restrict__ press,
                         const float* __restrict__ pvfac, const float* __restrict__ vn,
                         const float* __restrict__ rkx, const float* __restrict__ rky,
                         const float* __restrict__ rkz, const float* __restrict__ volvi,
                         const double* __restrict__ rho, float* __restrict__ vmc, float* __restrict__ vc) {
  PK(j, kd, nv);
  const int iv = VPTAB(j);
  if (kd < LPV(iv)) return;
  const int mza = g.mza;
  const int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  const size_t x = (size_t)iv * mza + kd, x1 = (size_t)iw1 * mza + kd, x2 = (size_t)iw2 * mza + kd;
  const float pgf = (float)(press[x1] - press[x2]) * pvfac[x];
  const float v = vmc0[x] + dts * (vmt_short[x] + pgf +
                                   (vn[iv * 3] * (rkx[x1] + rkx[x2]) + vn[iv * 3 + 1] * (rky[x1] + rky[x2]) +
                                    vn[iv * 3 + 2] * (rkz[x1] + rkz[x2])) * volvi[x]);
  vmc[x] = v;
  vc[x] = 2.0f * v / (float)(rho[x1] + rho[x2]);
}

// Prognostic shaved-cell method (prog_wrtv_rk.f90:202-211): the momentum of
// the lve2 lowest levels of a column with closed V faces at the step's start.
// A thread per (column, shaved level).
__global__ void k_shaved_save(DynK g, const int* __restrict__ prog, int nprog, const int* __restrict__ lve2,
                              int nve2, const float* __restrict__ vxe, const float* __restrict__ vye,
                              const float* __restrict__ vze, const double* __restrict__ rho, float* __restrict__ vm0) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * nve2) return;
  const int j = (int)(i / nve2), ks = (int)(i % nve2);
  const int iw = prog[j];
  if (ks >= lve2[iw]) return;
  const size_t x = (size_t)iw * g.mza + LPW(iw) + ks;
  const float rs = (float)rho[x];
  float* o = vm0 + ((size_t)iw * nve2 + ks) * 3;
  o[0] = vxe[x] * rs; o[1] = vye[x] * rs; o[2] = vze[x] * rs;
}

// the shaved-cell inputs of k_vel_t3d: lve2 == nullptr on grids without
// closed faces; prog != 0 in a stage of prog_wrtv_rk (the velocities of the
// shaved levels are prognosed first, update_vxe_undrgnd), 0 in diagvel_t3d
// (the cell's current velocities)
struct Shaved {
  const int* lve2;
  const float* vm0;
  const float *rkx, *rky, *rkz;
  const double* rho;
  const float* vn;
  int nve2, prog;
  float dts;
};

static Shaved shaved_args(const Dyn& y, const Transport& tp, int prog, float dts) {
  Shaved a{};
  if (y.nve2_max > 0) { a.lve2 = y.lve2.p; a.vm0 = y.vm0.p; a.nve2 = y.nve2_max; }
  a.rkx = y.rk_vx.p; a.rky = y.rk_vy.p; a.rkz = y.rk_vz.p;
  a.rho = tp.rho.p; a.vn = y.vn.p; a.prog = prog; a.dts = dts;
  return a;
}

// update_vxe_undrgnd (prog_wrtv_rk.f90:1558-1595) and vel_t3d_hex
// (vel_t3d.f90:39-108): a closed face (below its lpv) contributes the normal
// component of the cell's prognosed velocity at that level
__global__ void k_vel_t3d(DynK g, const int* __restrict__ prog, int nprog, const float* __restrict__ wc,
                          const float* __restrict__ vc, const float* __restrict__ wno2,
                          const float* __restrict__ ecv, float* __restrict__ vxe, float* __restrict__ vye,
                          float* __restrict__ vze, Shaved sh) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  const int kb = LPW(iw);
  if (kd < kb) return;
  const int mza = g.mza;
  const size_t cb = (size_t)iw * mza;
  const int ks = kd - kb;
  const bool shaved = sh.lve2 && ks < sh.lve2[iw];
  float p1x = 0.f, p1y = 0.f, p1z = 0.f;
  if (shaved) {
    if (sh.prog) {
      const float rsi = 1.0f / (float)sh.rho[cb + kd];
      const float vt = g.volti[cb + kd];
      const float* m = sh.vm0 + ((size_t)iw * sh.nve2 + ks) * 3;
      p1x = (m[0] + sh.dts * (sh.rkx[cb + kd] * vt)) * rsi;
      p1y = (m[1] + sh.dts * (sh.rky[cb + kd] * vt)) * rsi;
      p1z = (m[2] + sh.dts * (sh.rkz[cb + kd] * vt)) * rsi;
    } else {
      p1x = vxe[cb + kd]; p1y = vye[cb + kd]; p1z = vze[cb + kd];
    }
  }
  const float wst = wc[cb + kd - 1] + wc[cb + kd];
  float x = wst * wno2[iw * 3], y = wst * wno2[iw * 3 + 1], z = wst * wno2[iw * 3 + 2];
  const int np = g.npoly[iw];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    if (n >= np) break;
    const int iv = g.w_ev[iw * 8 + n];
    float v;
    if (kd >= LPV(iv)) v = vc[(size_t)iv * mza + kd];
    else if (shaved) v = sh.vn[iv * 3] * p1x + sh.vn[iv * 3 + 1] * p1y + sh.vn[iv * 3 + 2] * p1z;
    else continue;
    x = x + ecv[(iw * 7 + n) * 3] * v;
    y = y + ecv[(iw * 7 + n) * 3 + 1] * v;
    z = z + ecv[(iw * 7 + n) * 3 + 2] * v;
  }
  vxe[cb + kd] = x; vye[cb + kd] = y; vze[cb + kd] = z;
  if (kd == kb)
    for (int k2 = 0; k2 < kb; ++k2) { vxe[cb + k2] = x; vye[cb + k2] = y; vze[cb + k2] = z; }
}

// tend0 (timestep.f90:430-496) for the hot-path arrays
__global__ void k_tend0_w(DynK g, float* thilt, float* vmxet, float* vmyet, float* vmzet,
                          const double* rho, float* rho_old, float* wmasc) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)(g.mwa - 1) * g.mza) return;
  const int iw = 1 + (int)(i / g.mza), kd = (int)(i % g.mza);
  if (kd < LPW(iw)) return;
  const size_t x = (size_t)iw * g.mza + kd;
  thilt[x] = 0.f; vmxet[x] = 0.f; vmyet[x] = 0.f; vmzet[x] = 0.f;
  rho_old[x] = (float)rho[x];
  wmasc[x] = 0.f;
}

__global__ void k_tend0_v(DynK g, float* vmt, float* vmasc) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)(g.mva - 1) * g.mza) return;
  const int iv = 1 + (int)(i / g.mza), kd = (int)(i % g.mza);
  if (kd < LPV(iv)) return;
  const size_t x = (size_t)iv * g.mza + kd;
  vmt[x] = 0.f;
  vmasc[x] = 0.f;
}

// timeavg_momsc (timestep.f90:563-612)
__global__ void k_timeavg_v(DynK g, const int* __restrict__ vadj, int nv, float a, float* vmasc) {
  PK(j, kd, nv);
  const int iv = VATAB(j);
  if (kd < LPV(iv)) return;
  vmasc[(size_t)iv * g.mza + kd] = vmasc[(size_t)iv * g.mza + kd] / a;
}

__global__ void k_timeavg_w(DynK g, const int* __restrict__ prog, int nprog, float a, float* wmasc) {
  PK(j, kd, nprog);
  const int iw = WTAB(j);
  if (kd < LPW(iw) || kd > g.mza - 2) return;
  wmasc[(size_t)iw * g.mza + kd] = wmasc[(size_t)iw * g.mza + kd] / a;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <class T>
static int up(DevBuf<T>& b, const T* h, size_t n, cudaStream_t s, const char* name) {
  if (!h) {
    set_error(std::string("olamgpu_grid/opts: ") + name + " is NULL (needed by prog_wrtv_rk)");
    return OLAMGPU_E_ARG;
  }
  return upload(b, h, n, s);
}

int dyn_setup(const olamgpu_grid* g, const olamgpu_opts* o, cudaStream_t s) {
  Context& C = ctx();
  Dyn& y = C.dy;
  const int mza = g->mza, mwa = g->mwa, mva = g->mva, mma = g->mma;
  if (!g->itab_m_iv || !g->jtm_prog || g->nm_prog <= 0 || !g->lpm) {
    set_error("prog_wrtv_rk needs the M-point tables (itab_m, jtm_prog, lpm)");
    return OLAMGPU_E_ARG;
  }
  for (int i = 1; i < mma; ++i)
    if (g->lpm[i] < 2 || g->lpm[i] > mza) { set_error("lpm out of range [2,mza] at M point " + std::to_string(i + 1)); return OLAMGPU_E_ARG; }
  // shaved cells: lve2(iw) levels from lpw up have closed V faces; every
  // closed face must lie within them (hex_grid.f90 sets lve2 to the largest
  // lpv - lpw of the column's faces)
  int nve2 = 0;
  std::vector<int> lve2(mwa, 0);
  for (int i = 1; i < mwa; ++i) {
    const int l = g->lve2 ? g->lve2[i] : 0;
    if (l < 0 || l > mza) { set_error("lve2 out of range [0,mza] at W point " + std::to_string(i + 1)); return OLAMGPU_E_ARG; }
    for (int n = 0; n < g->npoly[i]; ++n) {
      const int iv = g->itab_w_iv[(size_t)i * 7 + n] - 1;
      if (iv >= 1 && iv < mva && g->lpv[iv] - g->lpw[i] > l) {
        set_error("lve2 at W point " + std::to_string(i + 1) + " does not cover its closed V faces (lpv - lpw)");
        return OLAMGPU_E_ARG;
      }
    }
    lve2[i] = l;
    nve2 = std::max(nve2, l);
  }
  y.nve2_max = nve2;
  if (nve2 > 0) {
    OG_CHECK(upload(y.lve2, lve2.data(), lve2.size(), s));
    OG_CHECK(y.vm0.alloc((size_t)mwa * nve2 * 3));
    OG_CUDA(cudaMemsetAsync(y.vm0.p, 0, y.vm0.bytes(), s));
  }
  if (mza > 128) { set_error("prog_wrtv_rk supports mza <= 128"); return OLAMGPU_E_UNSUPPORTED; }
  if ((size_t)std::max(std::max(mwa, mva), mma) * mza >= (1ull << 31)) {
    set_error("prog_wrtv_rk supports grids with max(mwa, mva, mma) * mza < 2^31");
    return OLAMGPU_E_UNSUPPORTED;
  }
  OG_CHECK(up(y.arv, g->arv, (size_t)mza * mva, s, "arv"));
  OG_CHECK(up(y.arw, g->arw, (size_t)mza * mwa, s, "arw"));
  OG_CHECK(up(y.volwi, g->volwi, (size_t)mza * mwa, s, "volwi"));
  OG_CHECK(up(y.volvi, g->volvi, (size_t)mza * mva, s, "volvi"));
  OG_CHECK(up(y.volt, g->volt, (size_t)mza * mwa, s, "volt"));
  {
    if (!g->wnx || !g->wnxo2 || !g->vnx || !g->ecvec_vx) { set_error("normals/ecvec missing"); return OLAMGPU_E_ARG; }
    std::vector<float> wn((size_t)mwa * 3), wno2((size_t)mwa * 3), vn((size_t)mva * 3), ec((size_t)mwa * 21);
    for (int i = 0; i < mwa; ++i) {
      wn[i * 3] = g->wnx[i]; wn[i * 3 + 1] = g->wny[i]; wn[i * 3 + 2] = g->wnz[i];
      wno2[i * 3] = g->wnxo2[i]; wno2[i * 3 + 1] = g->wnyo2[i]; wno2[i * 3 + 2] = g->wnzo2[i];
      for (int n = 0; n < 7; ++n) {
        ec[(i * 7 + n) * 3] = g->ecvec_vx[i * 7 + n];
        ec[(i * 7 + n) * 3 + 1] = g->ecvec_vy[i * 7 + n];
        ec[(i * 7 + n) * 3 + 2] = g->ecvec_vz[i * 7 + n];
      }
    }
    for (int i = 0; i < mva; ++i) { vn[i * 3] = g->vnx[i]; vn[i * 3 + 1] = g->vny[i]; vn[i * 3 + 2] = g->vnz[i]; }
    OG_CHECK(upload(y.wn, wn.data(), wn.size(), s));
    OG_CHECK(upload(y.wno2, wno2.data(), wno2.size(), s));
    OG_CHECK(upload(y.vn, vn.data(), vn.size(), s));
    OG_CHECK(upload(y.ecv, ec.data(), ec.size(), s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  OG_CHECK(up(y.gdz_wgtm, g->gdz_wgtm, mza, s, "gdz_wgtm"));
  OG_CHECK(up(y.gdz_wgtp, g->gdz_wgtp, mza, s, "gdz_wgtp"));
  OG_CHECK(up(y.gdz_wgtm8, g->gdz_wgtm8, mza, s, "gdz_wgtm8"));
  OG_CHECK(up(y.gdz_wgtp8, g->gdz_wgtp8, mza, s, "gdz_wgtp8"));
  OG_CHECK(up(y.zwgt_top8, g->zwgt_top8, mza, s, "zwgt_top8"));
  OG_CHECK(up(y.zwgt_bot8, g->zwgt_bot8, mza, s, "zwgt_bot8"));
  OG_CHECK(up(y.dniv, g->dniv, mva, s, "dniv"));
  OG_CHECK(up(y.dniu, g->dniu, mva, s, "dniu"));
  OG_CHECK(up(y.dnv, g->dnv, mva, s, "dnv"));
  OG_CHECK(up(y.arw0, g->arw0, mwa, s, "arw0"));
  OG_CHECK(up(y.arm0, g->arm0, mma, s, "arm0"));
  OG_CHECK(up(y.zfacit, g->zfacit, mza, s, "zfacit"));
  OG_CHECK(up(y.dzit, g->dzit, mza, s, "dzit"));
  OG_CHECK(up(y.xx_yy, g->xx_yy, (size_t)mwa * 7, s, "xx_yy"));
  OG_CHECK(up(y.xx_yy_m, g->xx_yy_m, (size_t)mma * 3, s, "xx_yy_m"));
  // init_wrtv_rk (prog_wrtv_rk.f90:36-54): b20 = 1 + dtsm * rayf_cofw
  std::vector<float> b20(mza, 1.0f);
  if (o->rayf_cofw)
    for (int k = o->krayfw_bot; k <= mza - 1; ++k) b20[k - 1] = 1.0f + (float)o->dtsm * o->rayf_cofw[k - 1];
  OG_CHECK(upload(y.b20, b20.data(), b20.size(), s));
  if (o->rayf_cof) {
    OG_CHECK(up(y.rayf_cof, o->rayf_cof, mza, s, "rayf_cof"));
    if (o->initial == 1) {
      OG_CHECK(up(y.dn01d, o->dn01d, mza, s, "dn01d"));
      OG_CHECK(up(y.th01d, o->th01d, mza, s, "th01d"));
    }
    OG_CHECK(up(y.vc03d, o->vc03d, (size_t)mza * mva, s, "vc03d"));
  }
  OG_CUDA(cudaStreamSynchronize(s));
  y.div_first = y.vort_first = true;
  y.uploaded = false;
  y.ready = true;
  return OLAMGPU_OK;
}

static int ensure_dyn_buffers(Context& C) {
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva, mz = (size_t)C.g.mza * C.g.mma;
  auto A = [](auto& b, size_t n) { return b.p ? OLAMGPU_OK : b.alloc(n); };
  OG_CHECK(A(tp.rho, wz)); OG_CHECK(A(tp.vmasc, vz)); OG_CHECK(A(tp.wmasc, wz)); OG_CHECK(A(tp.wc, wz));
  OG_CHECK(A(tp.rho_old, wz));
  OG_CHECK(A(y.press, wz)); OG_CHECK(A(y.rho0, wz)); OG_CHECK(A(y.rth0, wz));
  DevBuf<float>* w[] = {&y.thil, &y.wmc, &y.vxe, &y.vye, &y.vze, &y.alpha_press, &y.pwfac, &y.thilt,
                        &y.vmxet, &y.vmyet, &y.vmzet, &y.wmc0, &y.sh_th, &y.sh_vx, &y.sh_vy, &y.sh_vz,
                        &y.rk_vx, &y.rk_vy, &y.rk_vz};
  for (auto* b : w) OG_CHECK(A(*b, wz));
  DevBuf<float>* v[] = {&y.vmc, &y.vc, &y.pvfac, &y.vmt, &y.vmc0, &y.vmca, &y.sh_vmt, &y.fdivh};
  for (auto* b : v) OG_CHECK(A(*b, vz));
  OG_CHECK(A(y.upw, 4 * wz));
  OG_CHECK(A(y.upv, 4 * vz));
  OG_CHECK(A(y.div2d, 2 * wz));
  OG_CHECK(A(y.vort2d, 2 * mz));
  OG_CHECK(A(y.fvorth, C.g.mva)); OG_CHECK(A(y.fvortl, C.g.mva));
  OG_CHECK(A(y.vfact, 3 * (size_t)C.g.mma)); OG_CHECK(A(y.lpmmin, C.g.mma));
  return OLAMGPU_OK;
}

// host <-> device copies of the registered mem_basic / mem_tend arrays
int dyn_state_to_device(unsigned mask, cudaStream_t s) {
  Context& C = ctx();
  if (!C.have_state) return OLAMGPU_OK;
  OG_CHECK(ensure_dyn_buffers(C));
  const olamgpu_state& h = C.hstate;
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  auto cp = [&](void* d, const void* hp, size_t bytes) -> int {
    if (!hp) return OLAMGPU_OK;
    OG_CUDA(cudaMemcpyAsync(d, hp, bytes, cudaMemcpyHostToDevice, s));
    return OLAMGPU_OK;
  };
  if (mask & OLAMGPU_F_RHO) OG_CHECK(cp(tp.rho.p, h.rho, wz * 8));
  if (mask & OLAMGPU_F_PRESS) OG_CHECK(cp(y.press.p, h.press, wz * 8));
  if (mask & OLAMGPU_F_THIL) OG_CHECK(cp(y.thil.p, h.thil, wz * 4));
  if (mask & OLAMGPU_F_WC) OG_CHECK(cp(tp.wc.p, h.wc, wz * 4));
  if (mask & OLAMGPU_F_WMC) OG_CHECK(cp(y.wmc.p, h.wmc, wz * 4));
  if (mask & OLAMGPU_F_VXE) {
    OG_CHECK(cp(y.vxe.p, h.vxe, wz * 4)); OG_CHECK(cp(y.vye.p, h.vye, wz * 4)); OG_CHECK(cp(y.vze.p, h.vze, wz * 4));
  }
  if (mask & OLAMGPU_F_VMC) OG_CHECK(cp(y.vmc.p, h.vmc, vz * 4));
  if (mask & OLAMGPU_F_VC) OG_CHECK(cp(y.vc.p, h.vc, vz * 4));
  if (mask & OLAMGPU_F_VMASC) OG_CHECK(cp(tp.vmasc.p, h.vmasc, vz * 4));
  if (mask & OLAMGPU_F_WMASC) OG_CHECK(cp(tp.wmasc.p, h.wmasc, wz * 4));
  if (mask & OLAMGPU_F_FACS) {
    OG_CHECK(cp(y.alpha_press.p, h.alpha_press, wz * 4)); OG_CHECK(cp(y.pwfac.p, h.pwfac, wz * 4));
    OG_CHECK(cp(y.pvfac.p, h.pvfac, vz * 4));
  }
  if (mask & OLAMGPU_F_TEND) {
    OG_CHECK(cp(y.thilt.p, h.thilt, wz * 4)); OG_CHECK(cp(y.vmxet.p, h.vmxet, wz * 4));
    OG_CHECK(cp(y.vmyet.p, h.vmyet, wz * 4)); OG_CHECK(cp(y.vmzet.p, h.vmzet, wz * 4));
    OG_CHECK(cp(y.vmt.p, h.vmt, vz * 4));
  }
  // the registered arrays are page-locked: the copies read them when they
  // run, so they must end before the caller may write them again
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

int dyn_state_to_host(unsigned mask, cudaStream_t s) {
  Context& C = ctx();
  if (!C.have_state || !C.dy.thil.p) return OLAMGPU_OK;
  const olamgpu_state& h = C.hstate;
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  auto cp = [&](void* hp, const void* d, size_t bytes) -> int {
    if (!hp || !d) return OLAMGPU_OK;
    OG_CUDA(cudaMemcpyAsync(hp, d, bytes, cudaMemcpyDeviceToHost, s));
    return OLAMGPU_OK;
  };
  if (mask & OLAMGPU_F_RHO) OG_CHECK(cp(h.rho, tp.rho.p, wz * 8));
  if (mask & OLAMGPU_F_PRESS) OG_CHECK(cp(h.press, y.press.p, wz * 8));
  if (mask & OLAMGPU_F_THIL) OG_CHECK(cp(h.thil, y.thil.p, wz * 4));
  if (mask & OLAMGPU_F_WC) OG_CHECK(cp(h.wc, tp.wc.p, wz * 4));
  if (mask & OLAMGPU_F_WMC) OG_CHECK(cp(h.wmc, y.wmc.p, wz * 4));
  if (mask & OLAMGPU_F_VXE) {
    OG_CHECK(cp(h.vxe, y.vxe.p, wz * 4)); OG_CHECK(cp(h.vye, y.vye.p, wz * 4)); OG_CHECK(cp(h.vze, y.vze.p, wz * 4));
  }
  if (mask & OLAMGPU_F_VMC) OG_CHECK(cp(h.vmc, y.vmc.p, vz * 4));
  if (mask & OLAMGPU_F_VC) OG_CHECK(cp(h.vc, y.vc.p, vz * 4));
  if (mask & OLAMGPU_F_VMASC) OG_CHECK(cp(h.vmasc, tp.vmasc.p, vz * 4));
  if (mask & OLAMGPU_F_WMASC) OG_CHECK(cp(h.wmasc, tp.wmasc.p, wz * 4));
  if (mask & OLAMGPU_F_TEND) {
    OG_CHECK(cp(h.thilt, y.thilt.p, wz * 4)); OG_CHECK(cp(h.vmxet, y.vmxet.p, wz * 4));
    OG_CHECK(cp(h.vmyet, y.vmyet.p, wz * 4)); OG_CHECK(cp(h.vmzet, y.vmzet.p, wz * 4));
    OG_CHECK(cp(h.vmt, y.vmt.p, vz * 4));
  }
  return OLAMGPU_OK;
}

#define DYN_IN_MASK (OLAMGPU_F_RHO | OLAMGPU_F_PRESS | OLAMGPU_F_THIL | OLAMGPU_F_WC | OLAMGPU_F_WMC | \
                     OLAMGPU_F_VXE | OLAMGPU_F_VMC | OLAMGPU_F_VC | OLAMGPU_F_VMASC | OLAMGPU_F_WMASC | \
                     OLAMGPU_F_FACS | OLAMGPU_F_TEND)
#define DYN_OUT_MASK (OLAMGPU_F_RHO | OLAMGPU_F_PRESS | OLAMGPU_F_THIL | OLAMGPU_F_WC | OLAMGPU_F_WMC | \
                      OLAMGPU_F_VXE | OLAMGPU_F_VMC | OLAMGPU_F_VC | OLAMGPU_F_VMASC | OLAMGPU_F_WMASC | \
                      OLAMGPU_F_TEND)

static int divh_damp(Context& C, float* vmt, double dtm, cudaStream_t s) {
  const olamgpu_opts& o = C.opts;
  const DevGrid& d = C.g;
  Dyn& y = C.dy;
  if (!(o.divh_damp_fact > 1.e-7f) || o.divh_damp_level <= 0) return OLAMGPU_OK;
  const int level = o.divh_damp_level;
  const DynK g = dynk(d);
  const size_t wz = (size_t)d.mza * d.mwa;
  const unsigned nbv = cdiv((size_t)d.nv_prog * d.mza, 256), nbw = cdiv((size_t)d.nw_prog * d.mza, 256);
  if (y.div_first) {
    y.div_first = false;
    cudaMemsetAsync(y.div2d.p, 0, 2 * wz * sizeof(float), s);
    float p = 1.f;
    for (int i = 0; i < level; ++i) p = p * (-o.divh_damp_fact);
    const double facth = -((double)p / dtm);
    const float fact2 = o.divh_damp_fact / (float)dtm;
    k_div_fdivh<<<nbv, 256, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, y.arw0.p, y.dniv.p, y.zfacit.p, y.dzit.p,
                                    y.volt.p, facth, level, fact2, y.fdivh.p);
    OG_LAUNCHED();
  }
  float* d1 = y.div2d.p;
  k_div_accum<<<nbw, 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, y.arv.p, y.vmc.p, d1);
  OG_LAUNCHED();
  // border divergence for the Laplacian and the apply (vort_div_damp.f90:150)
  { HField f[1] = {{d1, 4}}; OG_CHECK(halo_exchange_fields(C, HALO_W, f, 1, s)); }
  const float* dh = d1;
  if (level > 1) {
    int ih = 2;
    for (int nn = 1; nn <= level - 1; ++nn) {
      const int il = (nn - 1) % 2 + 1;
      ih = nn % 2 + 1;
      k_lap_w<<<nbw, 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, y.xx_yy.p, y.div2d.p + (il - 1) * wz,
                                  y.div2d.p + (ih - 1) * wz);
      OG_LAUNCHED();
      { HField f[1] = {{y.div2d.p + (ih - 1) * wz, 4}}; OG_CHECK(halo_exchange_fields(C, HALO_W, f, 1, s)); }
    }
    dh = y.div2d.p + (ih - 1) * wz;
  }
  k_div_apply<<<nbv, 256, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, y.fdivh.p, dh, vmt);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

static int vort_damp(Context& C, float* vmt, double dtm, cudaStream_t s) {
  const olamgpu_opts& o = C.opts;
  const DevGrid& d = C.g;
  Dyn& y = C.dy;
  if (o.vort_damp_fact < 1.e-7f || o.vort_damp_level <= 0) return OLAMGPU_OK;
  const int level = o.vort_damp_level;
  const DynK g = dynk(d);
  const size_t mz = (size_t)d.mza * d.mma;
  if (y.vort_first) {
    y.vort_first = false;
    k_vort_first_m<<<cdiv(d.nm_prog, 128), 128, 0, s>>>(g, d.jtm_prog.p, d.nm_prog, y.dnv.p, y.arm0.p, y.vfact.p,
                                                        y.lpmmin.p);
    k_vort_first_v<<<cdiv(d.nv_prog, 128), 128, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, y.dniu.p, y.arm0.p, (float)dtm,
                                                        o.vort_damp_fact, level, y.fvorth.p, y.fvortl.p);
    OG_LAUNCHED(); OG_LAUNCHED();
  }
  const unsigned nbm = cdiv((size_t)d.nm_prog * d.mza, 256), nbv = cdiv((size_t)d.nv_prog * d.mza, 256);
  k_vort<<<nbm, 256, 0, s>>>(g, d.jtm_prog.p, d.nm_prog, y.vfact.p, y.vc.p, y.vort2d.p);
  OG_LAUNCHED();
  { HField f[1] = {{y.vort2d.p, 4}}; OG_CHECK(halo_exchange_fields(C, HALO_M, f, 1, s)); }
  int il = 1, ih = 1;
  if (level > 1) {
    for (int nn = 1; nn <= level - 1; ++nn) {
      il = (nn - 1) % 2 + 1;
      ih = nn % 2 + 1;
      k_lap_m<<<nbm, 256, 0, s>>>(g, d.jtm_prog.p, d.nm_prog, y.xx_yy_m.p, y.vort2d.p + (il - 1) * mz,
                                  y.vort2d.p + (ih - 1) * mz);
      OG_LAUNCHED();
      { HField f[1] = {{y.vort2d.p + (ih - 1) * mz, 4}}; OG_CHECK(halo_exchange_fields(C, HALO_M, f, 1, s)); }
    }
  }
  k_vort_apply<<<nbv, 256, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, level, y.fvorth.p, y.fvortl.p,
                                   y.vort2d.p + (il - 1) * mz, y.vort2d.p + (ih - 1) * mz, C.tp.rho.p, vmt);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

int dyn_prog_wrtv_rk(int istp) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!C.dy.ready) { set_error("prog_wrtv_rk was not set up (see olamgpu_init's status)"); return OLAMGPU_E_STATE; }
  if (!C.have_state) { set_error("prog_wrtv_rk needs the state arrays registered at init"); return OLAMGPU_E_STATE; }
  const olamgpu_opts& o = C.opts;
  if (o.nrk_wrtv != 2 && o.nrk_wrtv != 3) { set_error("acoust_timestep_level must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (C.halo.on && (!C.halo.dyn || o.ithil_monot > 0 || o.iwind_monot > 0)) {
    set_error("prog_wrtv_rk on a rank with a halo needs the V and M plans and no flux-corrected faces");
    return OLAMGPU_E_UNSUPPORTED;
  }
  cudaStream_t s = C.stream;
  OG_CHECK(ensure_dyn_buffers(C));
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL || !C.dy.uploaded) {
    OG_CHECK(dyn_state_to_device(DYN_IN_MASK, s));
    OG_CHECK(dyn_eddy_to_device(s));
  }
  C.dy.uploaded = true;
  const DevGrid& d = C.g;
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  const DynK g = dynk(d);
  const int mza = d.mza;
  const unsigned nbw = cdiv((size_t)d.nw_prog * mza, 256), nbv = cdiv((size_t)d.nv_prog * mza, 256),
                 nbva = cdiv((size_t)d.nv_wadj * mza, 256);
  OG_PROF("prog_wrtv_rk", s);
  if (!o.divh_damp_short && istp == 1) { OG_PROF("divh_damp", s); OG_CHECK(divh_damp(C, y.vmt.p, o.dtlm, s)); }
  if (!o.vort_damp_short && istp == 1) { OG_PROF("vort_damp", s); OG_CHECK(vort_damp(C, y.vmt.p, o.dtlm, s)); }
  SetupW sw{tp.rho.p, y.thil.p, y.wmc.p, y.thilt.p, y.vmxet.p, y.vmyet.p, y.vmzet.p, y.volt.p, y.rho0.p,
            y.rth0.p, y.wmc0.p, y.sh_th.p, y.sh_vx.p, y.sh_vy.p, y.sh_vz.p, y.rayf_cof.p, y.dn01d.p, y.th01d.p,
            o.krayf_bot};
  const bool rayleigh_th = o.rayf_cof && o.initial == 1;
  // with eddy diffusion the Rayleigh term on thil follows the eddy terms
  if (!rayleigh_th || y.eddy_on) sw.rayf_cof = nullptr;
  if (y.nve2_max > 0 && d.nw_prog > 0) {
    k_shaved_save<<<cdiv((size_t)d.nw_prog * y.nve2_max, 256), 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, y.lve2.p,
                                                                             y.nve2_max, y.vxe.p, y.vye.p, y.vze.p,
                                                                             tp.rho.p, y.vm0.p);
    OG_LAUNCHED();
  }
  { OG_PROF("setup_w", s); k_setup_w<<<nbw, 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, sw); OG_LAUNCHED(); }
  {
    OG_PROF("setup_v", s);
    k_setup_v<<<nbv, 256, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, y.vmc.p, y.vmt.p, y.vmc0.p, y.sh_vmt.p,
                                  (o.rayf_cof && o.vc03d) ? y.rayf_cof.p : nullptr, y.vc03d.p, y.vc.p, tp.rho.p,
                                  o.krayf_bot);
    OG_LAUNCHED();
  }
  if (y.eddy_on) {
    OG_PROF("eddy_columns", s);
    OG_CHECK(dyn_eddy_columns(C, rayleigh_th, s));
  }
  if (o.divh_damp_short) { OG_PROF("divh_damp", s); OG_CHECK(divh_damp(C, y.sh_vmt.p, o.dtsm, s)); }
  if (o.vort_damp_short) { OG_PROF("vort_damp", s); OG_CHECK(vort_damp(C, y.sh_vmt.p, o.dtsm, s)); }
  // start values of the fields fluxes_wrtv_monot limits (prog_wrtv_rk.f90:186-198)
  const bool thil_monot = o.ithil_monot > 0, wind_monot = o.iwind_monot > 0;
  const size_t wzb = (size_t)mza * d.mwa * sizeof(float);
  if (thil_monot) {
    OG_CHECK(y.th0.alloc((size_t)mza * d.mwa));
    OG_CUDA(cudaMemcpyAsync(y.th0.p, y.thil.p, wzb, cudaMemcpyDeviceToDevice, s));
  }
  if (wind_monot) {
    DevBuf<float>* b0[3] = {&y.vx0, &y.vy0, &y.vz0};
    const float* src[3] = {y.vxe.p, y.vye.p, y.vze.p};
    for (int i = 0; i < 3; ++i) {
      OG_CHECK(b0[i]->alloc((size_t)mza * d.mwa));
      OG_CUDA(cudaMemcpyAsync(b0[i]->p, src[i], wzb, cudaMemcpyDeviceToDevice, s));
    }
  }

  const int nrk = o.nrk_wrtv;
  const double third = 1.0 / 3.0;
  const double xstg3[3] = {third, 0.5, 1.0}, xstg2[2] = {0.5, 1.0};
  const size_t wz = (size_t)mza * d.mwa;
  for (int istage = 1; istage <= nrk; ++istage) {
    const double dt8 = (nrk <= 2 ? xstg2[istage - 1] : xstg3[istage - 1]) * o.dtsm;
    const float dts = (float)dt8;
    const int last = istage == nrk;
    // vmca = vmc arv is formed where it is read; the last stage also keeps
    // it (the flux-corrected faces read it) and adds it to vmasc
    if (last) {
      OG_PROF("vmca", s);
      k_vmca<<<nbva, 256, 0, s>>>(g, d.jtv_wadj.p, d.nv_wadj, y.vmc.p, y.arv.p, y.vmca.p, tp.vmasc.p, 1);
      OG_LAUNCHED();
    }
    Four f{{y.thil.p, y.vxe.p, y.vye.p, y.vze.p}};
    // fields by reconstruction order: thil has thil_horiz_adv_order, the
    // winds wind_horiz_adv_order (order 1: no gradient)
    const int ordf[4] = {o.thil_horiz_adv_order, o.wind_horiz_adv_order, o.wind_horiz_adv_order,
                         o.wind_horiz_adv_order};
    unsigned m2 = 0, m3 = 0;
    for (int q = 0; q < 4; ++q) { if (ordf[q] == 2) m2 |= 1u << q; if (ordf[q] >= 3) m3 |= 1u << q; }
    {
      OG_PROF("upw4", s);
      k_upw4<<<nbw, 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, f, y.wmc.p, y.upw.p);
      OG_LAUNCHED();
    }
    {
      OG_PROF("grad_upv4", s);
      // every face of jtv_wadj is written by its upwind cell: the columns
      // (and on a rank with a halo, ring 1, whose gradients the reference
      // exchanges) hold the gradients of their own faces' upwind sides
      DynK gg = g;
      const int* gt = d.jtw_prog.p;
      int gn = d.nw_prog;
      unsigned nbg = nbw;
      if (C.halo.on) {
        gg.off_w = d.off_wwadj;
        gt = d.jtw_wadj.p;
        gn = d.nw_wadj;
        nbg = cdiv((size_t)gn * mza, 256);
      }
      VSide vs{d.dxps.p, d.dyps.p, d.xx0_v.p, d.xy0_v.p, d.yy0_v.p};
      const unsigned plain = 0xFu & ~(m2 | m3);
      if (m2 || plain) {
        k_grad_upv4<2><<<nbg, 256, 0, s>>>(gg, gt, gn, f, m2, plain, d.gxc.p, d.gyc.p, d.xy_hu.p, vs, y.vmc.p,
                                           y.upv.p);
        OG_LAUNCHED();
      }
      if (m3) {
        k_grad_upv4<3><<<nbg, 256, 0, s>>>(gg, gt, gn, f, m3, 0u, d.gxc.p, d.gyc.p, d.xy_hu.p, vs, y.vmc.p,
                                           y.upv.p);
        OG_LAUNCHED();
      }
    }
    // last stage: flux-corrected face values replace those of the limited fields (370-399)
    if (last && thil_monot) {
      OG_PROF("monot_faces", s);
      OG_CHECK(dyn_monot_faces(C, 0, y.thil.p, y.th0.p, y.sh_th.p, dts, o.thil_horiz_adv_order, s));
    }
    if (last && wind_monot) {
      OG_PROF("monot_faces", s);
      OG_CHECK(dyn_monot_faces(C, 1, y.vxe.p, y.vx0.p, y.sh_vx.p, dts, o.wind_horiz_adv_order, s));
      OG_CHECK(dyn_monot_faces(C, 2, y.vye.p, y.vy0.p, y.sh_vy.p, dts, o.wind_horiz_adv_order, s));
      OG_CHECK(dyn_monot_faces(C, 3, y.vze.p, y.vz0.p, y.sh_vz.p, dts, o.wind_horiz_adv_order, s));
    }
    WrtArgs A;
    A.istage = istage; A.nrk = nrk; A.dt8 = dt8; A.dts = dts; A.fcoriol = o.fcoriol;
    A.fr = (double)0.70f;
    const float cpocv = 1004.f / 717.f;
    A.pc2 = A.fr * (double)cpocv;
    A.pc3 = A.fr * (double)cpocv;
    A.rocv = (1004.f - 717.f) / 717.f;
    A.c8 = dts * (float)A.pc2;
    A.c9 = -dts * dts * (float)A.fr;
    A.prog = d.jtw_prog.p; A.nprog = d.nw_prog;
    A.vmc = y.vmc.p; A.arv = y.arv.p; A.upv = y.upv.p; A.upw = y.upw.p;
    A.sh_th = y.sh_th.p; A.sh_vx = y.sh_vx.p; A.sh_vy = y.sh_vy.p; A.sh_vz = y.sh_vz.p;
    A.rk_vx = y.rk_vx.p; A.rk_vy = y.rk_vy.p; A.rk_vz = y.rk_vz.p;
    A.rho = tp.rho.p; A.press = y.press.p; A.rho0 = y.rho0.p; A.rth0 = y.rth0.p;
    A.thil = y.thil.p; A.wc = tp.wc.p; A.wmc = y.wmc.p; A.wmc0 = y.wmc0.p; A.vxe = y.vxe.p; A.vye = y.vye.p;
    A.wmasc = tp.wmasc.p; A.alpha_press = y.alpha_press.p; A.pwfac = y.pwfac.p;
    A.volt = y.volt.p; A.volwi = y.volwi.p; A.arw = y.arw.p; A.wn = y.wn.p;
    A.gdz_wgtm8 = y.gdz_wgtm8.p; A.gdz_wgtp8 = y.gdz_wgtp8.p; A.gdz_wgtm = y.gdz_wgtm.p; A.gdz_wgtp = y.gdz_wgtp.p;
    A.zwgt_bot8 = y.zwgt_bot8.p; A.zwgt_top8 = y.zwgt_top8.p; A.b20 = y.b20.p;
    const size_t smem = (size_t)WRT_WARPS * mza * 13 * sizeof(double);
    // eight blocks of four column warps per SM: 64 registers a thread and
    // the whole shared-memory carveout (8 x 25 KB at 61 levels; above 118
    // levels a block needs more than the default 48 KB)
    OG_CUDA(cudaFuncSetAttribute(k_wrt_begs, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    OG_CUDA(cudaFuncSetAttribute(k_wrt_begs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    { OG_PROF("wrt_begs", s); k_wrt_begs<<<cdiv(d.nw_prog, WRT_WARPS), WRT_WARPS * 32, smem, s>>>(g, A); OG_LAUNCHED(); }
    if (C.halo.on) {
      // prog_wrtv_rk.f90:418-429: what prog_v_begs reads at border V points
      OG_PROF("halo_exchange", s);
      HField f5[5] = {{y.press.p, 8}, {tp.rho.p, 8}, {y.rk_vx.p, 4}, {y.rk_vy.p, 4}, {y.rk_vz.p, 4}};
      OG_CHECK(halo_exchange_fields(C, HALO_W, f5, 5, s));
    }
    {
      OG_PROF("prog_v", s);
      k_prog_v<<<nbv, 256, 0, s>>>(g, d.jtv_prog.p, d.nv_prog, dts, y.vmc0.p, y.sh_vmt.p, y.press.p, y.pvfac.p,
                                   y.vn.p, y.rk_vx.p, y.rk_vy.p, y.rk_vz.p, y.volvi.p, tp.rho.p, y.vmc.p, y.vc.p);
      OG_LAUNCHED();
    }
    if (C.halo.on) {   // prog_wrtv_rk.f90:442-447
      OG_PROF("halo_exchange", s);
      HField f2[2] = {{y.vmc.p, 4}, {y.vc.p, 4}};
      OG_CHECK(halo_exchange_fields(C, HALO_V, f2, 2, s));
    }
    {
      OG_PROF("vel_t3d", s);
      k_vel_t3d<<<nbw, 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, tp.wc.p, y.vc.p, y.wno2.p, y.ecv.p, y.vxe.p,
                                    y.vye.p, y.vze.p, shaved_args(y, tp, 1, dts));
      OG_LAUNCHED();
    }
    if (C.halo.on) {   // prog_wrtv_rk.f90:464-472
      OG_PROF("halo_exchange", s);
      HField f6[6] = {{y.vxe.p, 4}, {y.vye.p, 4}, {y.vze.p, 4}, {y.wmc.p, 4}, {tp.wc.p, 4}, {y.thil.p, 4}};
      OG_CHECK(halo_exchange_fields(C, HALO_W, f6, 6, s));
    }
  }
  (void)wz;
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_host(DYN_OUT_MASK, s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

int dyn_tend0(float* rho_old_host) {
  Context& C = ctx();
  if (!C.initialised || !C.dy.ready || !C.have_state) { set_error("tend0 before init"); return OLAMGPU_E_STATE; }
  cudaStream_t s = C.stream;
  OG_CHECK(ensure_dyn_buffers(C));
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    // the kernels write levels k >= lpw only: the rest of each array it
    // returns keeps the caller's values
    OG_CHECK(dyn_state_to_device(OLAMGPU_F_RHO | OLAMGPU_F_TEND | OLAMGPU_F_VMASC | OLAMGPU_F_WMASC, s));
    if (rho_old_host)
      OG_CUDA(cudaMemcpyAsync(C.tp.rho_old.p, rho_old_host, (size_t)C.g.mza * C.g.mwa * 4, cudaMemcpyHostToDevice, s));
  } else if (!C.dy.uploaded) { OG_CHECK(dyn_state_to_device(DYN_IN_MASK, s)); C.dy.uploaded = true; }
  const DynK g = dynk(C.g);
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  k_tend0_w<<<cdiv((size_t)(C.g.mwa - 1) * C.g.mza, 256), 256, 0, s>>>(g, y.thilt.p, y.vmxet.p, y.vmyet.p,
                                                                      y.vmzet.p, tp.rho.p, tp.rho_old.p,
                                                                      tp.wmasc.p);
  k_tend0_v<<<cdiv((size_t)(C.g.mva - 1) * C.g.mza, 256), 256, 0, s>>>(g, y.vmt.p, tp.vmasc.p);
  OG_LAUNCHED(); OG_LAUNCHED();
  // scalar tendencies var_t = 0 for k >= lpw (the device copies)
  // (a window's adjoint lends the per-tracer arrays' memory out while it
  // runs the dynamics again: there are none to clear then)
  for (int n = 0; n < C.tr.n; ++n)
    if (C.tr.t[n].p) OG_CUDA(cudaMemsetAsync(C.tr.t[n].p, 0, (size_t)C.g.mza * C.g.mwa * 4, s));
  if (C.tr.q_valid && C.tr.qt.p) OG_CUDA(cudaMemsetAsync(C.tr.qt.p, 0, C.tr.qt.bytes(), s));
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_host(OLAMGPU_F_TEND | OLAMGPU_F_VMASC | OLAMGPU_F_WMASC, s));
    if (rho_old_host)
      OG_CUDA(cudaMemcpyAsync(rho_old_host, tp.rho_old.p, (size_t)C.g.mza * C.g.mwa * 4, cudaMemcpyDeviceToHost, s));
    for (int n = 0; n < C.tr.n; ++n)
      OG_CUDA(cudaMemcpyAsync(C.tr.h_t[n], C.tr.t[n].p, (size_t)C.g.mza * C.g.mwa * 4, cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  return OLAMGPU_OK;
}

int dyn_timeavg_momsc() {
  Context& C = ctx();
  if (!C.initialised || !C.dy.ready) { set_error("timeavg_momsc before init"); return OLAMGPU_E_STATE; }
  if (C.opts.nacoust <= 1) return OLAMGPU_OK;
  cudaStream_t s = C.stream;
  OG_CHECK(ensure_dyn_buffers(C));
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) OG_CHECK(dyn_state_to_device(OLAMGPU_F_VMASC | OLAMGPU_F_WMASC, s));
  else if (!C.dy.uploaded) { OG_CHECK(dyn_state_to_device(DYN_IN_MASK, s)); C.dy.uploaded = true; }
  const DynK g = dynk(C.g);
  const float a = (float)C.opts.nacoust;
  k_timeavg_v<<<cdiv((size_t)C.g.nv_wadj * C.g.mza, 256), 256, 0, s>>>(g, C.g.jtv_wadj.p, C.g.nv_wadj, a, C.tp.vmasc.p);
  k_timeavg_w<<<cdiv((size_t)C.g.nw_prog * C.g.mza, 256), 256, 0, s>>>(g, C.g.jtw_prog.p, C.g.nw_prog, a, C.tp.wmasc.p);
  OG_LAUNCHED(); OG_LAUNCHED();
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_host(OLAMGPU_F_VMASC | OLAMGPU_F_WMASC, s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  return OLAMGPU_OK;
}

// diagvel_t3d (vel_t3d.f90:7-35): vel_t3d_hex over jtw_prog
int dyn_diagvel_t3d() {
  Context& C = ctx();
  if (!C.initialised || !C.dy.ready || !C.have_state) { set_error("diagvel_t3d before init"); return OLAMGPU_E_STATE; }
  cudaStream_t s = C.stream;
  OG_CHECK(ensure_dyn_buffers(C));
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) OG_CHECK(dyn_state_to_device(OLAMGPU_F_WC | OLAMGPU_F_VC | OLAMGPU_F_VXE, s));
  else if (!C.dy.uploaded) { OG_CHECK(dyn_state_to_device(DYN_IN_MASK, s)); C.dy.uploaded = true; }
  const DevGrid& d = C.g;
  Dyn& y = C.dy;
  if (d.nw_prog > 0) {
    k_vel_t3d<<<cdiv((size_t)d.nw_prog * d.mza, 256), 256, 0, s>>>(dynk(d), d.jtw_prog.p, d.nw_prog, C.tp.wc.p, y.vc.p,
                                                                    y.wno2.p, y.ecv.p, y.vxe.p, y.vye.p, y.vze.p,
                                                                    shaved_args(y, C.tp, 0, 0.f));
    OG_LAUNCHED();
  }
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_host(OLAMGPU_F_VXE, s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

void dyn_release() {
  Dyn& y = ctx().dy;
  DevBuf<double>* d8[] = {&y.press, &y.rho0, &y.rth0, &y.volt, &y.zwgt_top8, &y.zwgt_bot8, &y.gdz_wgtm8, &y.gdz_wgtp8};
  for (auto* b : d8) b->release();
  DevBuf<float>* f[] = {&y.thil, &y.wmc, &y.vxe, &y.vye, &y.vze, &y.vmc, &y.vc, &y.alpha_press, &y.pwfac,
                        &y.pvfac, &y.thilt, &y.vmxet, &y.vmyet, &y.vmzet, &y.vmt, &y.wmc0, &y.vmc0, &y.vmca,
                        &y.sh_th, &y.sh_vx, &y.sh_vy, &y.sh_vz, &y.sh_vmt, &y.rk_vx, &y.rk_vy,
                        &y.rk_vz, &y.upw, &y.upv, &y.div2d, &y.fdivh, &y.vort2d, &y.fvorth, &y.fvortl,
                        &y.vfact, &y.arv, &y.arw, &y.volwi, &y.volvi, &y.wn, &y.wno2, &y.vn, &y.ecv,
                        &y.gdz_wgtm, &y.gdz_wgtp, &y.dniv, &y.dniu, &y.dnv, &y.arw0, &y.arm0, &y.zfacit,
                        &y.dzit, &y.xx_yy, &y.xx_yy_m, &y.b20, &y.rayf_cof, &y.dn01d, &y.th01d, &y.vc03d,
                        &y.th0, &y.vx0, &y.vy0, &y.vz0, &y.m_scpt, &y.m_gx, &y.m_hiw, &y.m_sfw, &y.m_hiv,
                        &y.m_sfv, &y.m_sin, &y.m_sout};
  for (auto* b : f) b->release();
  y.lpmmin.release();
  y.lve2.release();
  y.vm0.release();
  dyn_eddy_release();
  y = Dyn();
}

}  // namespace olamgpu
