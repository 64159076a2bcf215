// transport_kernels.cu -- CFL diagnosis, RK densities, implicit vertical
// solve, and the reference-mirroring transport passes (gradient, V face,
// W column, flux renormalisation, tendency) for any tracer count.
//
// The passes follow omodel/scalar_transport_rk.F90 one routine per kernel:
//   launch_grad     grad_t2d / grad_t2d_quadratic (grad_lib.f90:236-341)
//   launch_vflux    scalar_v_column (474-534), scalar_vflux_monot (749-832),
//                   scalar_vflux_pd (1215-1285)
//   launch_wcol     scalar_w_column (537-612), scalar_wflux_and_scales_monot
//                   (835-1022), scalar_wflux_and_scale_pd (1288-1414)
//   launch_vapply   the horizontal renormalisation loops (711-724, 1177-1190)
//   launch_tend     scalar_tend_monot (1025-1078), scalar_tend_pd (1417-1469)
// With one tracer in OLAM's (mza, mwa) layout they are the plain
// one-kernel-per-pass form; with a tracer group of the batched layout they
// run the last RK stage of the monotonic / positive-definite options.
//
// Device level index kd = Fortran k - 1.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <mutex>
#include <string>

#include "transport_kernels.cuh"

namespace olamgpu {


GridK gridk(const DevGrid& d) {
  GridK g;
  g.mza = d.mza; g.mwa = d.mwa; g.mva = d.mva;
  g.npoly = d.npoly.p; g.w_nb = d.w_nb.p; g.w_ev = d.w_ev.p; g.w_dirv = d.w_dirv.p;
  g.v_iw = d.v_iw.p; g.lpw = d.lpw.p; g.lpv = d.lpv.p; g.volti = d.volti.p;
  g.a_w = d.a_w.p; g.a_wu = d.a_wu.p;
  return g;
}

// ---------------------------------------------------------------------------
// check_cfls (scalar_transport_rk.F90:1476-1712)
// red[0..5]: (cfl key, cfl nan), (cflh key, cflh nan), (|w| key, w nan)
// key = float bits << 32 | (0xffffffff - order) so atomicMax keeps the largest
// value and, on ties, the first point in loop order; nan = order + 1 of the
// last NaN in loop order (OLAM's serial loop keeps the last NaN it meets).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// one warp per prognostic column, lanes over levels (coalesced in k)
__global__ void k_check_cfls(GridK g, const int* __restrict__ prog, int nprog,
                             const float* __restrict__ vmasc, const float* __restrict__ wmasc,
                             const float* __restrict__ rho, const float* __restrict__ wc, int nrk,
                             float dt, float* __restrict__ ff, unsigned long long* red) {
  const int j = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= nprog) return;
  const int mza = g.mza;
  const int iw = prog[j];
  const int np = g.npoly[iw];
  int ev[7];
  float dv[7];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    ev[n] = g.w_ev[iw * 8 + n];
    dv[n] = g.w_dirv[iw * 8 + n];
  }
  float fimp[3] = {0.f, 0.f, 0.f};
  unsigned long long kc = 0, kh = 0, kw = 0, nc = 0, nh = 0, nwn = 0;
  for (int kd = g.lpw[iw] + lane; kd < mza; kd += 32) {
    float cflh = 0.f;
#pragma unroll
    for (int n = 0; n < 7; ++n)
      if (n < np && kd >= g.lpv[ev[n]])
        cflh = cflh - fminf(dv[n] * __ldg(vmasc + (size_t)ev[n] * mza + kd), 0.0f);
    const float dovr = dt * g.volti[(size_t)iw * mza + kd] / rho[(size_t)iw * mza + kd];
    cflh = cflh * dovr;
    float cflw = (fmaxf(wmasc[(size_t)iw * mza + kd], 0.f) - fminf(wmasc[(size_t)iw * mza + kd - 1], 0.f)) * dovr;
    const float cfl = cflh + cflw;
    cflw = fmaxf(cflw, .1f);
    fimp[nrk - 1] = fmaxf(fimp[nrk - 1], (cfl - 0.98f) / cflw);
    fimp[nrk - 2] = fmaxf(fimp[nrk - 2], (cfl - 1.98f) / cflw);
    if (nrk == 3) fimp[0] = fmaxf(fimp[0], (cfl - 2.98f) / cflw);
    const unsigned int order = (unsigned int)j * (unsigned int)mza + (unsigned int)kd;
    const unsigned long long low = 0xffffffffull - order;
    if (cfl != cfl) nc = max(nc, order + 1ull);
    else if (cfl > 0.f) kc = max(kc, ((unsigned long long)__float_as_uint(cfl) << 32) | low);
    if (cflh != cflh) nh = max(nh, order + 1ull);
    else if (cflh > 0.f) kh = max(kh, ((unsigned long long)__float_as_uint(cflh) << 32) | low);
    if (wc) {
      const float w = wc[(size_t)iw * mza + kd];
      if (w != w) nwn = max(nwn, order + 1ull);
      else if (fabsf(w) > 0.f) kw = max(kw, ((unsigned long long)__float_as_uint(fabsf(w)) << 32) | low);
    }
  }
#pragma unroll
  for (int n = 0; n < 3; ++n)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) fimp[n] = fmaxf(fimp[n], __shfl_xor_sync(0xffffffffu, fimp[n], o));
  kc = warp_max_u64(kc); nc = warp_max_u64(nc);
  kh = warp_max_u64(kh); nh = warp_max_u64(nh);
  kw = warp_max_u64(kw); nwn = warp_max_u64(nwn);
  if (lane == 0) {
    for (int n = 0; n < nrk; ++n) {
      float f = fminf(1.0f, fimp[n]);
      if (f < .02f) f = 0.f;
      ff[(size_t)iw * nrk + n] = f;
    }
    if (red) {
      if (kc) atomicMax(&red[0], kc);
      if (nc) atomicMax(&red[1], nc);
      if (kh) atomicMax(&red[2], kh);
      if (nh) atomicMax(&red[3], nh);
      if (kw) atomicMax(&red[4], kw);
      if (nwn) atomicMax(&red[5], nwn);
    }
  }
}

void launch_check_cfls(const DevGrid& d, const Transport& tp, int nrk, float dtl,
                       unsigned long long* red, cudaStream_t s) {
  if (red) cudaMemsetAsync(red, 0, 6 * sizeof(unsigned long long), s);
  const int nb = 256;  // 8 columns per block
  k_check_cfls<<<cdiv((size_t)d.nw_prog * 32, nb), nb, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog,
                                                              tp.vmasc.p, tp.wmasc.p, tp.rho_old.p,
                                                              tp.wc.p, nrk, dtl, tp.ff.p, red);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// rhos (scalar_transport_rk.F90:117-152), nudging off
// ---------------------------------------------------------------------------
__global__ void k_rhos(GridK g, const int* __restrict__ prog, int nprog, const double* __restrict__ rho,
                       const float* __restrict__ rho_old, float* __restrict__ rhos, int nrk) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mza = g.mza;
  if (i >= (size_t)nprog * mza) return;
  int j = (int)(i / mza), kd = (int)(i % mza);
  int iw = prog[j];
  if (kd < g.lpw[iw]) return;
  size_t ix = (size_t)iw * mza + kd;
  size_t plane = (size_t)g.mwa * mza;
  float rhof = (float)rho[ix];
  float ro = rho_old[ix];
  if (nrk == 3) {
    rhos[ix] = (2.f / 3.f) * ro + (1.f / 3.f) * rhof;
    rhos[plane + ix] = 0.5f * (ro + rhof);
    rhos[2 * plane + ix] = rhof;
  } else {
    rhos[ix] = 0.5f * (ro + rhof);
    rhos[plane + ix] = rhof;
  }
}

void launch_rhos(const DevGrid& d, Transport& tp, int nrk, cudaStream_t s) {
  size_t n = (size_t)d.nw_prog * d.mza;
  k_rhos<<<cdiv(n, 256), 256, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, tp.rho.p, tp.rho_old.p,
                                      tp.rhos.p, nrk);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// implicit-column factorisation (scalar_transport_rk.F90:164-217) with
// tridif_prep (tridiag_lib.f90:321-338).  Column slots are handed out by an
// atomic counter; each column's result does not depend on its slot.
// imp_b[(n*mwa + slot)*3*mza + {0,1,2}*mza + kd] = b1, scr1, cji.
// ---------------------------------------------------------------------------
struct Dtlr { float v[3]; };

__global__ void k_implicit_prep(GridK g, const int* __restrict__ prog, int nprog,
                                const float* __restrict__ ff, const float* __restrict__ wmasc,
                                const float* __restrict__ rhos, int nrk, Dtlr dtlr,
                                int* __restrict__ list, int* __restrict__ count, float* __restrict__ b) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nprog) return;
  const int mza = g.mza;
  int iw = prog[j];
  int kb = g.lpw[iw];
  size_t plane = (size_t)g.mwa * mza;
  for (int n = 0; n < nrk; ++n) {
    float f = ff[(size_t)iw * nrk + n];
    if (!(f > 0.001f)) continue;
    int slot = atomicAdd(&count[n], 1);
    list[(size_t)n * g.mwa + slot] = iw;
    float* b1 = b + ((size_t)n * g.mwa + slot) * 3 * mza;
    float* scr1 = b1 + mza;
    float* cji = b1 + 2 * mza;
    float c1 = f * dtlr.v[n];
    const float* wm = wmasc + (size_t)iw * mza;
    // wup(kd) = max(wmasc,0), wdn(kd) = min(wmasc,0) for kd in [kb, mza-2];
    // zero at kb-1 and mza-1
    float cji_prev = 0.f, cip1_prev = 0.f;
    for (int kd = kb; kd < mza; ++kd) {
      float wup_m1 = (kd - 1 >= kb) ? fmaxf(wm[kd - 1], 0.f) : 0.f;
      float wdn_m1 = (kd - 1 >= kb) ? fminf(wm[kd - 1], 0.f) : 0.f;
      float wup = (kd <= mza - 2) ? fmaxf(wm[kd], 0.f) : 0.f;
      float wdn = (kd <= mza - 2) ? fminf(wm[kd], 0.f) : 0.f;
      float c2 = c1 * g.volti[(size_t)iw * mza + kd] / rhos[(size_t)n * plane + (size_t)iw * mza + kd];
      float cim1 = -c2 * wup_m1;
      float ci = 1.0f + c2 * (wup - wdn_m1);
      float cip1 = c2 * wdn;
      b1[kd] = cim1;
      if (kd == kb) {
        cji_prev = 1.0f / ci;
        cji[kd] = cji_prev;
        scr1[kd] = 0.f;
      } else {
        float sc = cji_prev * cip1_prev;
        scr1[kd] = sc;
        cji_prev = 1.0f / (ci - cim1 * sc);
        cji[kd] = cji_prev;
      }
      cip1_prev = cip1;
    }
  }
}

void launch_implicit_prep(const DevGrid& d, Transport& tp, int nrk, const float* dtlr, cudaStream_t s) {
  cudaMemsetAsync(tp.imp_count.p, 0, sizeof(int) * 3, s);
  Dtlr v{{dtlr[0], dtlr[1], nrk > 2 ? dtlr[2] : 0.f}};
  k_implicit_prep<<<cdiv(d.nw_prog, 128), 128, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, tp.ff.p,
                                                       tp.wmasc.p, tp.rhos.p, nrk, v, tp.imp_list.p,
                                                       tp.imp_count.p, tp.imp_b.p);
  OG_LAUNCHED();
}

// implicit vertical transport (scalar_transport_rk.F90:347-375) with
// tridif_fini (tridiag_lib.f90:344-364); one thread per (column, tracer).
__global__ void k_implicit_solve(GridK g, const int* __restrict__ list, const int* __restrict__ count,
                                 const float* __restrict__ b, const float* __restrict__ ff,
                                 const float* __restrict__ wmasc, const float* __restrict__ rhos_st,
                                 int nrk, int istage, float dtr, CTView scp0, TView scp, int nt) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  int n = *count;
  if (i >= (size_t)n * nt) return;
  int slot = (int)(i / nt), t = (int)(i % nt);
  const int mza = g.mza;
  int iw = list[slot];
  int kb = g.lpw[iw];
  const float* b1 = b + (size_t)slot * 3 * mza;
  const float* scr1 = b1 + mza;
  const float* cji = b1 + 2 * mza;
  const float* wm = wmasc + (size_t)iw * mza;
  float ffv = ff[(size_t)iw * nrk + istage - 1];
  auto S0 = [&](int kd) { return scp0.base[((size_t)iw * mza + kd) * scp0.ld + scp0.t0 + t]; };
  float* sp = scp.base + (size_t)iw * mza * scp.ld + scp.t0 + t;
  // forward elimination into soln (kept in the output column), then back
  // substitution; delex is formed on the fly from scp and scp0
  float prev = 0.f;
  for (int kd = kb; kd < mza; ++kd) {
    float s0 = S0(kd);
    float dk = (kd <= mza - 2) ? S0(kd + 1) - s0 : 0.f;
    float dkm1 = (kd - 1 >= kb) ? s0 - S0(kd - 1) : 0.f;
    float c1 = ffv * dtr * g.volti[(size_t)iw * mza + kd] / rhos_st[(size_t)iw * mza + kd];
    float delex = sp[(size_t)kd * scp.ld] - s0 - c1 * (fminf(wm[kd], 0.f) * dk + fmaxf(wm[kd - 1], 0.f) * dkm1);
    float sol = (kd == kb) ? delex * cji[kd] : cji[kd] * (delex - b1[kd] * prev);
    sp[(size_t)kd * scp.ld] = sol;
    prev = sol;
  }
  for (int kd = mza - 2; kd >= kb; --kd) {
    float v = sp[(size_t)kd * scp.ld] - scr1[kd + 1] * sp[(size_t)(kd + 1) * scp.ld];
    sp[(size_t)kd * scp.ld] = v;
  }
  for (int kd = kb; kd < mza; ++kd) sp[(size_t)kd * scp.ld] = S0(kd) + sp[(size_t)kd * scp.ld];
  for (int kd = 1; kd < kb; ++kd) sp[(size_t)kd * scp.ld] = sp[(size_t)kb * scp.ld];
}

void launch_implicit_solve(const DevGrid& d, const Transport& tp, int nrk, int istage, float dtr,
                           CTView scp0, TView scp, int nt, cudaStream_t s) {
  // an upper bound on the launch size; threads past the device count exit
  size_t n = (size_t)d.nw_prog * nt;
  size_t plane = (size_t)d.mwa * d.mza;
  const float* b = tp.imp_b.p + (size_t)(istage - 1) * d.mwa * 3 * d.mza;
  k_implicit_solve<<<cdiv(n, 128), 128, 0, s>>>(gridk(d), tp.imp_list.p + (size_t)(istage - 1) * d.mwa,
                                                tp.imp_count.p + (istage - 1), b, tp.ff.p, tp.wmasc.p,
                                                tp.rhos.p + (size_t)(istage - 1) * plane, nrk, istage,
                                                dtr, scp0, scp, nt);
  OG_LAUNCHED();
}

// horizontal diffusion hook (scalar_transport_rk.F90:244-274)
__global__ void k_diffusion(GridK g, const int* __restrict__ prog, int nprog,
                            const float* __restrict__ akhodx, const int* __restrict__ khtopv,
                            CTView scp, TView sct, int nt) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * nt) return;
  int j = (int)(i / nt), t = (int)(i % nt);
  const int mza = g.mza;
  int iw = prog[j];
  int np = g.npoly[iw];
  int kwtop = 0;
  for (int n = 0; n < np; ++n) kwtop = max(kwtop, khtopv[g.w_ev[iw * 8 + n]]);
  int kb = g.lpw[iw];
  // khtopv holds OLAM's 1-based top level; device level = khtopv - 1
  if (kwtop - 1 < kb) return;
  for (int kd = kb; kd <= kwtop - 1; ++kd) {
    float fd = 0.f;
    for (int n = 0; n < np; ++n) {
      int iv = g.w_ev[iw * 8 + n], iwn = g.w_nb[iw * 8 + n];
      if (kd >= g.lpv[iv] && kd <= khtopv[iv] - 1)
        fd = fd + akhodx[(size_t)iv * mza + kd] *
                      (scp.base[((size_t)iwn * mza + kd) * scp.ld + scp.t0 + t] -
                       scp.base[((size_t)iw * mza + kd) * scp.ld + scp.t0 + t]);
    }
    float* p = sct.base + ((size_t)iw * mza + kd) * sct.ld + sct.t0 + t;
    *p = *p + fd * g.volti[(size_t)iw * mza + kd];
  }
}

void launch_diffusion(const DevGrid& d, const Transport& tp, CTView scp, TView sct, int nt,
                      cudaStream_t s) {
  size_t n = (size_t)d.nw_prog * nt;
  k_diffusion<<<cdiv(n, 128), 128, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, tp.akhodx.p,
                                           tp.khtopv.p, scp, sct, nt);
  OG_LAUNCHED();
}

// last-stage low-order pre-update of scp0 for monotonic / positive-definite
// tracers (scalar_transport_rk.F90:297-314)
__global__ void k_scp0_pd(GridK g, const int* __restrict__ wadj, int nwadj, TView scp0, CTView sct,
                          const float* __restrict__ rho_old, const int* __restrict__ mode, int nt,
                          float dtr) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nwadj * nt) return;
  int j = (int)(i / nt), t = (int)(i % nt);
  if (!mode[t]) return;
  const int mza = g.mza;
  int iw = wadj[j];
  int kb = g.lpw[iw];
  for (int kd = kb; kd < mza; ++kd) {
    float* p = scp0.base + ((size_t)iw * mza + kd) * scp0.ld + scp0.t0 + t;
    *p = *p + dtr * sct.base[((size_t)iw * mza + kd) * sct.ld + sct.t0 + t] /
                  rho_old[(size_t)iw * mza + kd];
  }
  float v = scp0.base[((size_t)iw * mza + kb) * scp0.ld + scp0.t0 + t];
  for (int kd = 1; kd < kb; ++kd) scp0.base[((size_t)iw * mza + kd) * scp0.ld + scp0.t0 + t] = v;
}

void launch_scp0_pd_update(const DevGrid& d, const Transport& tp, TView scp0, CTView sct,
                           const int* mode, int nt, float dtr, cudaStream_t s) {
  size_t n = (size_t)d.nw_wadj * nt;
  k_scp0_pd<<<cdiv(n, 128), 128, 0, s>>>(gridk(d), d.jtw_wadj.p, d.nw_wadj, scp0, sct, tp.rho_old.p,
                                         mode, nt, dtr);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// pass 1: horizontal gradient planes gx[m][iw][kd][t] (compact, ld = nt)
// ---------------------------------------------------------------------------
__global__ void k_grad(GridK g, const int* __restrict__ prog, int nprog, CTView scp,
                       float* __restrict__ gx, int nt, int order, const float* __restrict__ cx,
                       const float* __restrict__ cy, const float* __restrict__ xy) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mza = g.mza;
  size_t tot = (size_t)nprog * mza * nt;
  if (i >= tot) return;
  int t = (int)(i % nt);
  size_t r = i / nt;
  int kd = (int)(r % mza);
  int j = (int)(r / mza);
  int iw = prog[j];
  int np = g.npoly[iw];
  size_t plane = (size_t)g.mwa * mza * nt;
  size_t o = ((size_t)iw * mza + kd) * nt + t;
  float sc0 = scp.base[((size_t)iw * mza + kd) * scp.ld + scp.t0 + t];
  if (order == 2) {
    float gxv = 0.f, gyv = 0.f;
    for (int n = 0; n < np; ++n) {
      int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      int iwn = g.w_nb[iw * 8 + n];
      float d = scp.base[((size_t)iwn * mza + kd) * scp.ld + scp.t0 + t] - sc0;
      gxv = gxv + __ldg(cx + iw * 7 + n) * d;
      gyv = gyv + __ldg(cy + iw * 7 + n) * d;
    }
    gx[o] = gxv;
    gx[plane + o] = gyv;
  } else {
    float a[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    for (int n = 0; n < np; ++n) {
      int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      int iwn = g.w_nb[iw * 8 + n];
      float d = scp.base[((size_t)iwn * mza + kd) * scp.ld + scp.t0 + t] - sc0;
      const float* c = xy + ((size_t)iw * 7 + n) * 5;
#pragma unroll
      for (int m = 0; m < 5; ++m) a[m] = a[m] + d * __ldg(c + m);
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) gx[m * plane + o] = a[m];
  }
}

// The one-tracer passes of the plain form (OLAM's own layout) give PLC
// lanes to a column or face (32 / PLC of them per warp) and keep PLU levels
// per lane in flight: the levels of a column are PLC apart per lane, PLC *
// PLU per round.
#define PLC 8
#define PLU 4

// grad_t2d / grad_t2d_quadratic of one tracer: the column's neighbours, face
// floors and coefficients held in registers (read once per column instead
// of once per element)
template <int ORDER>
__global__ void __launch_bounds__(256)
    k_grad1(GridK g, const int* __restrict__ prog, int nprog, const float* __restrict__ S, float* __restrict__ gx,
            const float* __restrict__ cx, const float* __restrict__ cy, const float* __restrict__ xy) {
  constexpr int M = ORDER == 2 ? 2 : 5;   // gradient planes
  const int w = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / PLC), hl = threadIdx.x % PLC;
  if (w >= nprog) return;
  const int mza = g.mza, iw = prog[w], np = g.npoly[iw];
  const size_t plane = (size_t)g.mwa * mza;
  int nb[7], lp[7];
  float c[7][M];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    nb[n] = iw; lp[n] = mza;
#pragma unroll
    for (int m = 0; m < M; ++m) c[n][m] = 0.f;
    if (n < np) {
      nb[n] = __ldg(g.w_nb + iw * 8 + n);
      lp[n] = __ldg(g.lpv + __ldg(g.w_ev + iw * 8 + n));
      if (ORDER == 2) { c[n][0] = __ldg(cx + iw * 7 + n); c[n][M - 1] = __ldg(cy + iw * 7 + n); }
      else {
#pragma unroll
        for (int m = 0; m < M; ++m) c[n][m] = __ldg(xy + ((size_t)iw * 7 + n) * 5 + m);
      }
    }
  }
  for (int k0 = hl; k0 < mza; k0 += PLC * PLU) {
    float a[PLU][M], s0[PLU];
#pragma unroll
    for (int u = 0; u < PLU; ++u) {
      const int k = k0 + PLC * u;
      s0[u] = k < mza ? S[(size_t)iw * mza + k] : 0.f;
#pragma unroll
      for (int m = 0; m < M; ++m) a[u][m] = 0.f;
    }
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      if (n >= np) continue;
#pragma unroll
      for (int u = 0; u < PLU; ++u) {
        const int k = k0 + PLC * u;
        if (k < mza && k >= lp[n]) {
          const float d = S[(size_t)nb[n] * mza + k] - s0[u];
#pragma unroll
          for (int m = 0; m < M; ++m) a[u][m] = a[u][m] + c[n][m] * d;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < PLU; ++u) {
      const int k = k0 + PLC * u;
      if (k >= mza) continue;
      const size_t o = (size_t)iw * mza + k;
#pragma unroll
      for (int m = 0; m < M; ++m) gx[m * plane + o] = a[u][m];
    }
  }
}

void launch_grad(const DevGrid& d, CTView scp, float* gx, int nt, int order, bool bounded,
                 cudaStream_t s) {
  if (nt == 1 && scp.ld == 1 && scp.t0 == 0) {
    const unsigned nb = cdiv((size_t)d.nw_prog * PLC, 256);
    if (order == 2)
      k_grad1<2><<<nb, 256, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, scp.base, gx, d.gxc.p, d.gyc.p, nullptr);
    else
      k_grad1<3><<<nb, 256, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, scp.base, gx, nullptr, nullptr,
                                    bounded ? d.xy_h.p : d.xy_hu.p);
    OG_LAUNCHED();
    return;
  }
  size_t n = (size_t)d.nw_prog * d.mza * nt;
  k_grad<<<cdiv(n, 256), 256, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, scp, gx, nt, order, d.gxc.p,
                                      d.gyc.p, bounded ? d.xy_h.p : d.xy_hu.p);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// pass 2: V-face values.  mode[t] == PLAIN: upv = upwind reconstruction.
// MONOT/PD: upv = low-order value from scp0, hiv = high-order correction,
// sfv = vmasc*hiv.
// ---------------------------------------------------------------------------
struct VCoef {
  const float* dxps; const float* dyps;
  const float* xx; const float* xy; const float* yy;
};

__device__ __forceinline__ float side_val(const CTView& scp, const float* __restrict__ gx, size_t plane,
                                          int mza, int nt, int order, const VCoef& vc, int iv, int sd,
                                          int iws, int kd, int t) {
  size_t o = ((size_t)iws * mza + kd) * nt + t;
  float v = scp.base[((size_t)iws * mza + kd) * scp.ld + scp.t0 + t];
  int e = iv * 2 + sd;
  v = v + __ldg(vc.dxps + e) * gx[o] + __ldg(vc.dyps + e) * gx[plane + o];
  if (order == 3)
    v = v + __ldg(vc.xx + e) * gx[2 * plane + o] + __ldg(vc.xy + e) * gx[3 * plane + o] +
        __ldg(vc.yy + e) * gx[4 * plane + o];
  return v;
}

__global__ void k_vflux(GridK g, const int* __restrict__ vlist, int nv, CTView scp, CTView scp0,
                        const float* __restrict__ gx, const float* __restrict__ vmasc, int nt, int order,
                        VCoef vc, const int* __restrict__ mode, float* __restrict__ upv,
                        float* __restrict__ hiv, float* __restrict__ sfv) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mza = g.mza;
  if (i >= (size_t)nv * mza * nt) return;
  int t = (int)(i % nt);
  size_t r = i / nt;
  int kd = (int)(r % mza);
  int iv = vlist[r / mza];
  if (kd < g.lpv[iv]) return;
  int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  size_t plane = (size_t)g.mwa * mza * nt;
  float s1 = side_val(scp, gx, plane, mza, nt, order, vc, iv, 0, iw1, kd, t);
  float s2 = side_val(scp, gx, plane, mza, nt, order, vc, iv, 1, iw2, kd, t);
  float vm = vmasc[(size_t)iv * mza + kd];
  size_t o = ((size_t)iv * mza + kd) * nt + t;
  int md = mode ? mode[t] : MODE_PLAIN;
  if (md == MODE_PLAIN) {
    float up = s1;
    if (vm < 0.f) up = s2;
    upv[o] = up;
  } else {
    float lo = scp0.base[((size_t)iw1 * mza + kd) * scp0.ld + scp0.t0 + t];
    if (vm < 0.f) lo = scp0.base[((size_t)iw2 * mza + kd) * scp0.ld + scp0.t0 + t];
    float hi = s1;
    if (vm < 0.f) hi = s2;
    hi = hi - lo;
    upv[o] = lo;
    hiv[o] = hi;
    sfv[o] = vm * hi;
  }
}

// the upwind V-face values of one tracer (plain mode, OLAM's layout): PLC
// lanes per face, PLU levels per lane in flight, the face's cells and
// coefficients in registers; only the upwind side's reconstruction is read
__device__ __forceinline__ float vface1(const float* __restrict__ S, const float* __restrict__ gx, size_t plane,
                                        int order, size_t o, float dx, float dy, float xx, float xy, float yy) {
  float v = S[o];
  v = v + dx * gx[o] + dy * gx[plane + o];
  if (order == 3) v = v + xx * gx[2 * plane + o] + xy * gx[3 * plane + o] + yy * gx[4 * plane + o];
  return v;
}

__global__ void __launch_bounds__(256)
    k_vflux1(GridK g, const int* __restrict__ vlist, int nv, const float* __restrict__ S,
             const float* __restrict__ gx, const float* __restrict__ vmasc, int order, VCoef vc,
             float* __restrict__ upv) {
  const int w = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / PLC), hl = threadIdx.x % PLC;
  if (w >= nv) return;
  const int mza = g.mza, iv = vlist[w], kv = g.lpv[iv];
  const size_t plane = (size_t)g.mwa * mza;
  // side 1 (itab_v%iw(1)) and side 2 coefficients, selected per level by the
  // sign of the flux (no runtime-indexed arrays: they would live in local memory)
  const int w1 = g.v_iw[iv * 2], w2 = g.v_iw[iv * 2 + 1];
  const int e1 = iv * 2, e2 = iv * 2 + 1;
  const float dx1 = __ldg(vc.dxps + e1), dy1 = __ldg(vc.dyps + e1), dx2 = __ldg(vc.dxps + e2), dy2 = __ldg(vc.dyps + e2);
  float xx1 = 0.f, xy1 = 0.f, yy1 = 0.f, xx2 = 0.f, xy2 = 0.f, yy2 = 0.f;
  if (order == 3) {
    xx1 = __ldg(vc.xx + e1); xy1 = __ldg(vc.xy + e1); yy1 = __ldg(vc.yy + e1);
    xx2 = __ldg(vc.xx + e2); xy2 = __ldg(vc.xy + e2); yy2 = __ldg(vc.yy + e2);
  }
  for (int k0 = kv + hl; k0 < mza; k0 += PLC * PLU) {
    float u[PLU];
#pragma unroll
    for (int q = 0; q < PLU; ++q) {
      const int k = k0 + PLC * q;
      u[q] = 0.f;
      if (k < mza) {
        const bool two = vmasc[(size_t)iv * mza + k] < 0.f;
        u[q] = vface1(S, gx, plane, order, (size_t)(two ? w2 : w1) * mza + k, two ? dx2 : dx1, two ? dy2 : dy1,
                      two ? xx2 : xx1, two ? xy2 : xy1, two ? yy2 : yy1);
      }
    }
#pragma unroll
    for (int q = 0; q < PLU; ++q) {
      const int k = k0 + PLC * q;
      if (k < mza) upv[(size_t)iv * mza + k] = u[q];
    }
  }
}

void launch_vflux(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, const float* gx,
                  int nt, int order, bool unbounded, const int* mode, bool anylim, cudaStream_t s) {
  VCoef vc{d.dxps.p, d.dyps.p, unbounded ? d.xx0_vu.p : d.xx0_v.p, unbounded ? d.xy0_vu.p : d.xy0_v.p,
           unbounded ? d.yy0_vu.p : d.yy0_v.p};
  if (nt == 1 && scp.ld == 1 && scp.t0 == 0 && !anylim) {
    k_vflux1<<<cdiv((size_t)d.nv_wadj * PLC, 256), 256, 0, s>>>(gridk(d), d.jtv_wadj.p, d.nv_wadj, scp.base, gx,
                                                              tp.vmasc.p, order, vc, tp.upv.p);
    OG_LAUNCHED();
    return;
  }
  size_t n = (size_t)d.nv_wadj * d.mza * nt;
  k_vflux<<<cdiv(n, 256), 256, 0, s>>>(gridk(d), d.jtv_wadj.p, d.nv_wadj, scp, scp0, gx, tp.vmasc.p, nt,
                                       order, vc, anylim ? mode : nullptr, tp.upv.p, tp.hiv.p, tp.sfv.p);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// pass 3: one thread per (column, tracer), sequential in k.
// ---------------------------------------------------------------------------
struct WcolArgs {
  GridK g;
  const int* prog; int nprog;
  CTView scp, scp0, sct;
  const float* rhos;        // stage density rhos(:,:,nrk)
  const float* vmasc; const float* wmasc; const float* ff;
  const float* upv; const float* sfv;   // compact (mva, mza, nt)
  float* scale;             // compact (2, mwa, mza, nt)
  float* upw;               // compact (mwa, mza, nt)
  TView out;
  int nt, istage, nrk; float dtr;
  const int* mode;
};

__global__ void k_wcol(WcolArgs A) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.nprog * A.nt) return;
  const GridK& g = A.g;
  const int mza = g.mza;
  int t = (int)(i % A.nt);
  int iw = A.prog[i / A.nt];
  int kb = g.lpw[iw];
  int np = g.npoly[iw];
  int md = A.mode ? A.mode[t] : MODE_PLAIN;
  float fimpl = A.ff[(size_t)iw * A.nrk + A.istage - 1];
  float fexpl = 1.0f - fimpl;
  const float* wm = A.wmasc + (size_t)iw * mza;
  auto S = [&](int kd) { return A.scp.base[((size_t)iw * mza + kd) * A.scp.ld + A.scp.t0 + t]; };
  auto S0 = [&](int kd) { return A.scp0.base[((size_t)iw * mza + kd) * A.scp0.ld + A.scp0.t0 + t]; };
  auto OUTP = [&](int kd) { return A.out.base + ((size_t)iw * mza + kd) * A.out.ld + A.out.t0 + t; };
  const size_t ntz = (size_t)A.nt;

  if (md == MODE_PLAIN) {
    // scalar_w_column (scalar_transport_rk.F90:537-612)
    float up_prev = S(kb);  // scp_upw(kb-1) = scp(kb)
    float sm1 = 0.f, s0 = S(kb), sp1 = (kb + 1 < mza) ? S(kb + 1) : 0.f;
    float sp2 = (kb + 2 < mza) ? S(kb + 2) : 0.f;
    for (int kd = kb; kd < mza; ++kd) {
      float up;
      if (kd <= mza - 2) {
        if (wm[kd] < 0.f) {
          // scpb(kd+1): level kd+1 with neighbours kd, kd+2
          float sb, st;
          zrec(g.a_w, mza, kd + 1, kb, s0, sp1, sp2, 0.f, false, false, sb, st);
          up = sb;
        } else {
          float sb, st;
          zrec(g.a_w, mza, kd, kb, sm1, s0, sp1, 0.f, false, false, sb, st);
          up = st;
        }
      } else {
        up = s0;  // scp_upw(mza) = scp(mza)
      }
      float s00 = S0(kd);
      float fd = 0.f;
      for (int n = 0; n < np; ++n) {
        int iv = g.w_ev[iw * 8 + n];
        if (kd < g.lpv[iv]) continue;
        fd = fd + g.w_dirv[iw * 8 + n] * A.vmasc[(size_t)iv * mza + kd] *
                      (A.upv[((size_t)iv * mza + kd) * ntz + t] - s00);
      }
      fd = fd + fexpl * (wm[kd - 1] * (up_prev - s00) - wm[kd] * (up - s00));
      float sctv = A.sct.base[((size_t)iw * mza + kd) * A.sct.ld + A.sct.t0 + t];
      *OUTP(kd) = s00 + A.dtr * (sctv + g.volti[(size_t)iw * mza + kd] * fd) / A.rhos[(size_t)iw * mza + kd];
      up_prev = up;
      sm1 = s0; s0 = sp1; sp1 = sp2;
      sp2 = (kd + 3 < mza) ? S(kd + 3) : 0.f;
    }
    float v = *OUTP(kb);
    for (int kd = 0; kd < kb; ++kd) *OUTP(kd) = v;
    return;
  }

  // monotonic (md == 1) / positive-definite (md == 2) scale factors
  const bool monot = (md == MODE_MONOT);
  const float eps0 = kEps0, eps1 = kEps1, onep = 1.0f + kEps1, onem = 1.0f - kEps1;
  const float* awu = g.a_wu;
  float* upwp = A.upw + (size_t)iw * mza * ntz + t;
  float* sc1 = A.scale + (size_t)iw * mza * ntz + t;
  float* sc2 = A.scale + ((size_t)g.mwa + iw) * mza * ntz + t;
  // low-order vertical upwind value scp_upw(k) at device face kd (between kd, kd+1)
  auto lo_face = [&](int kd) -> float {
    if (kd == kb - 1) return monot ? S0(kb) : S(kb);
    if (kd == mza - 1) return monot ? S0(mza - 1) : S(mza - 1);
    float v = S0(kd);
    if (wm[kd] < 0.f) v = S0(kd + 1);
    return v;
  };
  // high-order face correction hiw(kd) for kd in [kb, mza-2]
  auto hi_face = [&](int kd) -> float {
    float sb, st;
    if (wm[kd] < 0.f) {
      float a0 = S(kd), a1 = S(kd + 1), a2 = (kd + 2 < mza) ? S(kd + 2) : 0.f;
      zrec(monot ? awu : g.a_w, mza, kd + 1, kb, a0, a1, a2, 0.f, monot, monot, sb, st);
      return sb - lo_face(kd);
    } else {
      float am = (kd - 1 >= kb) ? S(kd - 1) : 0.f, a0 = S(kd), a1 = S(kd + 1);
      zrec(monot ? awu : g.a_w, mza, kd, kb, am, a0, a1, 0.f, monot, monot, sb, st);
      return st - lo_face(kd);
    }
  };
  float dtrp = onep * A.dtr;
  float mdtrp = -onep * A.dtr;
  float sfw_prev = 0.f;  // sfluxwh(kb-1) = 0
  for (int kd = kb; kd < mza; ++kd) {
    float sfw = 0.f;
    if (kd <= mza - 2) sfw = fexpl * wm[kd] * hi_face(kd);
    float s00 = S0(kd);
    float fl = 0.f, fin = 0.f, fout = 0.f;
    float smax = s00, smin = s00;
    if (monot) {
      if (kd >= kb + 1 && wm[kd - 1] > 0.f) { smax = fmaxf(smax, S0(kd - 1)); smin = fminf(smin, S0(kd - 1)); }
      if (kd <= mza - 2 && wm[kd] < 0.f) { smax = fmaxf(smax, S0(kd + 1)); smin = fminf(smin, S0(kd + 1)); }
    }
    for (int n = 0; n < np; ++n) {
      int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      float dv = g.w_dirv[iw * 8 + n];
      float vm = A.vmasc[(size_t)iv * mza + kd];
      size_t o = ((size_t)iv * mza + kd) * ntz + t;
      fl = fl + dv * vm * (A.upv[o] - s00);
      if (monot) fin = fin + fmaxf(dv * A.sfv[o], 0.f);
      fout = fout + fminf(dv * A.sfv[o], 0.f);
      if (monot && dv * vm > 0.f) {
        int iwn = g.w_nb[iw * 8 + n];
        float sn = A.scp0.base[((size_t)iwn * mza + kd) * A.scp0.ld + A.scp0.t0 + t];
        smax = fmaxf(smax, sn);
        smin = fminf(smin, sn);
      }
    }
    float lo_m1 = lo_face(kd - 1), lo_k = lo_face(kd);
    float rh = A.rhos[(size_t)iw * mza + kd];
    float vt = g.volti[(size_t)iw * mza + kd];
    if (fimpl > .001f) {
      float dwi = fimpl * (wm[kd] - wm[kd - 1]);
      if (monot) {
        fl = fl + fexpl * (wm[kd - 1] * (lo_m1 - s00) - wm[kd] * (lo_k - s00)) + s00 * dwi;
        fin = fin + fmaxf(sfw_prev, 0.f) - fminf(sfw, 0.f);
        fout = fout + fminf(sfw_prev, 0.f) - fmaxf(sfw, 0.f);
        float imp = rh + A.dtr * vt * dwi;
        smax = imp * smax;
        smin = imp * smin;
      } else {
        fl = fl + fexpl * (wm[kd - 1] * (lo_m1 - s00) - wm[kd] * (lo_k - s00)) +
             fimpl * s00 * (wm[kd] - wm[kd - 1]);
        fout = fout + fminf(sfw_prev, 0.f) - fmaxf(sfw, 0.f);
      }
    } else {
      fl = fl + wm[kd - 1] * (lo_m1 - s00) - wm[kd] * (lo_k - s00);
      if (monot) {
        fin = fin + fmaxf(sfw_prev, 0.f) - fminf(sfw, 0.f);
        smax = rh * smax;
        smin = rh * smin;
      }
      fout = fout + fminf(sfw_prev, 0.f) - fmaxf(sfw, 0.f);
    }
    float rscp_low = s00 * rh + A.dtr * vt * fl;
    if (monot) {
      float flux_in = fmaxf(dtrp * vt * fin, eps0);
      float flux_out = fminf(dtrp * vt * fout, -eps0);
      float epsr = eps1 * fabsf(rscp_low);
      float sc_in = fmaxf(smax - (rscp_low + epsr) - eps0, 0.f);
      float sc_out = fminf(smin - (rscp_low - epsr) + eps0, 0.f);
      sc1[(size_t)kd * ntz] = fminf(1.f, sc_in / fmaxf(flux_in, 0.01f * sc_in));
      sc2[(size_t)kd * ntz] = fminf(1.f, sc_out / fminf(flux_out, 0.01f * sc_out));
    } else {
      float flux_out = fmaxf(mdtrp * vt * fout, eps0);
      float sc_out = fmaxf(onem * rscp_low - eps0, 0.f);
      sc1[(size_t)kd * ntz] = fminf(1.f, sc_out / fmaxf(flux_out, 0.01f * sc_out));
    }
    sfw_prev = sfw;
  }
  // renormalised vertical face values (scp_upw) for the tendency pass
  upwp[(size_t)(kb - 1) * ntz] = lo_face(kb - 1);
  upwp[(size_t)(mza - 1) * ntz] = lo_face(mza - 1);
  for (int kd = kb; kd <= mza - 2; ++kd) {
    float hi = hi_face(kd);
    float sfw = fexpl * wm[kd] * hi;
    float scale;
    if (monot) {
      scale = fminf(sc1[(size_t)(kd + 1) * ntz], sc2[(size_t)kd * ntz]);
      if (sfw < 0.f) scale = fminf(sc1[(size_t)kd * ntz], sc2[(size_t)(kd + 1) * ntz]);
    } else {
      scale = sc1[(size_t)kd * ntz];
      if (sfw < 0.f) scale = sc1[(size_t)(kd + 1) * ntz];
    }
    upwp[(size_t)kd * ntz] = lo_face(kd) + hi * scale;
  }
}

// pass 3 of an unlimited stage, one thread per (level, column, tracer) with
// the level fastest for one tracer (nt = 1: a column's levels are adjacent,
// so every load of a warp is coalesced).  scalar_w_column
// (scalar_transport_rk.F90:537-612) has no recurrence in k: the face values
// scp_upw(k-1), scp_upw(k) come from grad_z_quadratic of the upwind level,
// i.e. from scp(k-2 .. k+2), and each cell's update is independent.
__global__ void k_wcell(WcolArgs A) {
  const GridK& g = A.g;
  const int mza = g.mza;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)A.nprog * mza * A.nt) return;
  int t, kd, j;
  if (A.nt == 1) { t = 0; kd = (int)(i % mza); j = (int)(i / mza); }
  else { t = (int)(i % A.nt); const size_t r = i / A.nt; kd = (int)(r % mza); j = (int)(r / mza); }
  const int iw = A.prog[j];
  const int kb = g.lpw[iw];
  if (kd < kb) return;   // written by the thread of level kb
  const int np = g.npoly[iw];
  const float fimpl = A.ff[(size_t)iw * A.nrk + A.istage - 1];
  const float fexpl = 1.0f - fimpl;
  const float* wm = A.wmasc + (size_t)iw * mza;
  auto S = [&](int k) { return A.scp.base[((size_t)iw * mza + k) * A.scp.ld + A.scp.t0 + t]; };
  // scp_upw at the top face of level f (f = kb-1 .. mza-1)
  auto upw = [&](int f) -> float {
    if (f == kb - 1) return S(kb);        // scp_upw(kb-1) = scp(kb)
    if (f == mza - 1) return S(mza - 1);  // scp_upw(mza) = scp(mza)
    float sb, st;
    if (wm[f] < 0.f) {                    // scpb(f+1) from (f, f+1, f+2)
      zrec(g.a_w, mza, f + 1, kb, S(f), S(f + 1), (f + 2 < mza) ? S(f + 2) : 0.f, 0.f, false, false, sb, st);
      return sb;
    }
    zrec(g.a_w, mza, f, kb, (f - 1 >= kb) ? S(f - 1) : 0.f, S(f), S(f + 1), 0.f, false, false, sb, st);
    return st;
  };
  const size_t ntz = (size_t)A.nt;
  const float s00 = A.scp0.base[((size_t)iw * mza + kd) * A.scp0.ld + A.scp0.t0 + t];
  float fd = 0.f;
  for (int n = 0; n < np; ++n) {
    const int iv = g.w_ev[iw * 8 + n];
    if (kd < g.lpv[iv]) continue;
    fd = fd + g.w_dirv[iw * 8 + n] * A.vmasc[(size_t)iv * mza + kd] * (A.upv[((size_t)iv * mza + kd) * ntz + t] - s00);
  }
  fd = fd + fexpl * (wm[kd - 1] * (upw(kd - 1) - s00) - wm[kd] * (upw(kd) - s00));
  const float sctv = A.sct.base[((size_t)iw * mza + kd) * A.sct.ld + A.sct.t0 + t];
  const float o = s00 + A.dtr * (sctv + g.volti[(size_t)iw * mza + kd] * fd) / A.rhos[(size_t)iw * mza + kd];
  float* out = A.out.base + (size_t)iw * mza * A.out.ld + A.out.t0 + t;
  out[(size_t)kd * A.out.ld] = o;
  if (kd == kb)
    for (int k = 0; k < kb; ++k) out[(size_t)k * A.out.ld] = o;
}

// the same for one tracer in OLAM's layout: PLC lanes per column, PLU
// levels per lane in flight, the column's faces (V point, dirv, floor) in
// registers
__global__ void __launch_bounds__(256, 3) k_wcell1(WcolArgs A) {
  const GridK& g = A.g;
  const int mza = g.mza;
  const int w = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) / PLC), hl = threadIdx.x % PLC;
  if (w >= A.nprog) return;
  const int iw = A.prog[w], kb = g.lpw[iw], np = g.npoly[iw];
  int ev[7], lp[7];
  float dv[7];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    ev[n] = 0; lp[n] = mza; dv[n] = 0.f;
    if (n < np) { ev[n] = g.w_ev[iw * 8 + n]; lp[n] = g.lpv[ev[n]]; dv[n] = g.w_dirv[iw * 8 + n]; }
  }
  const float fimpl = A.ff[(size_t)iw * A.nrk + A.istage - 1];
  const float fexpl = 1.0f - fimpl;
  const float* __restrict__ wm = A.wmasc + (size_t)iw * mza;
  const float* __restrict__ Sc = A.scp.base + (size_t)iw * mza;
  auto S = [&](int k) { return Sc[k]; };
  auto upw = [&](int f) -> float {
    if (f == kb - 1) return S(kb);
    if (f == mza - 1) return S(mza - 1);
    float sb, st;
    if (wm[f] < 0.f) {
      zrec(g.a_w, mza, f + 1, kb, S(f), S(f + 1), (f + 2 < mza) ? S(f + 2) : 0.f, 0.f, false, false, sb, st);
      return sb;
    }
    zrec(g.a_w, mza, f, kb, (f - 1 >= kb) ? S(f - 1) : 0.f, S(f), S(f + 1), 0.f, false, false, sb, st);
    return st;
  };
  // the update of level kd, from loads only (no store in between)
  auto cell = [&](int kd) -> float {
    const size_t x = (size_t)iw * mza + kd;
    const float s00 = A.scp0.base[x];
    float fd = 0.f;
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      if (n >= np || kd < lp[n]) continue;
      const size_t xv = (size_t)ev[n] * mza + kd;
      fd = fd + dv[n] * A.vmasc[xv] * (A.upv[xv] - s00);
    }
    fd = fd + fexpl * (wm[kd - 1] * (upw(kd - 1) - s00) - wm[kd] * (upw(kd) - s00));
    return s00 + A.dtr * (A.sct.base[x] + g.volti[x] * fd) / A.rhos[x];
  };
  float* out = A.out.base + (size_t)iw * mza;
  for (int k0 = kb + hl; k0 < mza; k0 += PLC * PLU) {
    float o[PLU];
#pragma unroll
    for (int q = 0; q < PLU; ++q) o[q] = k0 + PLC * q < mza ? cell(k0 + PLC * q) : 0.f;
#pragma unroll
    for (int q = 0; q < PLU; ++q)
      if (k0 + PLC * q < mza) out[k0 + PLC * q] = o[q];
    if (k0 == kb)
      for (int k = 0; k < kb; ++k) out[k] = o[0];
  }
}

void launch_wcell(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, CTView sct, const float* rhos,
                  TView out, int nt, int istage, int nrk, float dtr, cudaStream_t s) {
  WcolArgs A;
  A.g = gridk(d);
  A.prog = d.jtw_prog.p; A.nprog = d.nw_prog;
  A.scp = scp; A.scp0 = scp0; A.sct = sct; A.rhos = rhos;
  A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p; A.ff = tp.ff.p;
  A.upv = tp.upv.p; A.sfv = nullptr; A.scale = nullptr; A.upw = nullptr;
  A.out = out; A.nt = nt; A.istage = istage; A.nrk = nrk; A.dtr = dtr;
  A.mode = nullptr;
  if (nt == 1 && scp.ld == 1 && scp.t0 == 0 && scp0.ld == 1 && scp0.t0 == 0 && sct.ld == 1 && sct.t0 == 0 &&
      out.ld == 1 && out.t0 == 0) {
    k_wcell1<<<cdiv((size_t)d.nw_prog * PLC, 256), 256, 0, s>>>(A);
    OG_LAUNCHED();
    return;
  }
  const size_t n = (size_t)d.nw_prog * d.mza * nt;
  k_wcell<<<cdiv(n, 256), 256, 0, s>>>(A);
  OG_LAUNCHED();
}

void launch_wcol(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, CTView sct,
                 const float* rhos, TView out, int nt, int istage, int nrk, float dtr,
                 const int* mode, bool anylim, cudaStream_t s) {
  WcolArgs A;
  A.g = gridk(d);
  A.prog = d.jtw_prog.p; A.nprog = d.nw_prog;
  A.scp = scp; A.scp0 = scp0; A.sct = sct; A.rhos = rhos;
  A.vmasc = tp.vmasc.p; A.wmasc = tp.wmasc.p; A.ff = tp.ff.p;
  A.upv = tp.upv.p; A.sfv = tp.sfv.p; A.scale = tp.scale.p; A.upw = tp.upw.p;
  A.out = out; A.nt = nt; A.istage = istage; A.nrk = nrk; A.dtr = dtr;
  A.mode = anylim ? mode : nullptr;
  size_t n = (size_t)d.nw_prog * nt;
  k_wcol<<<cdiv(n, 128), 128, 0, s>>>(A);
  OG_LAUNCHED();
}

// pass 4: horizontal flux renormalisation (711-724 monot, 1177-1190 pd)
__global__ void k_vapply(GridK g, const int* __restrict__ vlist, int nv, int nt,
                         const int* __restrict__ mode, float* __restrict__ upv,
                         const float* __restrict__ hiv, const float* __restrict__ sfv,
                         const float* __restrict__ scale) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int mza = g.mza;
  if (i >= (size_t)nv * mza * nt) return;
  int t = (int)(i % nt);
  size_t r = i / nt;
  int kd = (int)(r % mza);
  int iv = vlist[r / mza];
  int md = mode[t];
  if (md == MODE_PLAIN || kd < g.lpv[iv]) return;
  int iw1 = g.v_iw[iv * 2], iw2 = g.v_iw[iv * 2 + 1];
  size_t o = ((size_t)iv * mza + kd) * nt + t;
  const size_t s2 = (size_t)g.mwa * mza * nt;
  size_t a1 = ((size_t)iw1 * mza + kd) * nt + t, a2 = ((size_t)iw2 * mza + kd) * nt + t;
  float sc;
  if (md == MODE_MONOT) {
    sc = fminf(scale[a2], scale[s2 + a1]);
    if (sfv[o] < 0.f) sc = fminf(scale[a1], scale[s2 + a2]);
  } else {
    sc = scale[a1];
    if (sfv[o] < 0.f) sc = scale[a2];
  }
  upv[o] = upv[o] + hiv[o] * sc;
}

void launch_vapply(const DevGrid& d, const Transport& tp, int nt, const int* mode, cudaStream_t s) {
  size_t n = (size_t)d.nv_wadj * d.mza * nt;
  k_vapply<<<cdiv(n, 256), 256, 0, s>>>(gridk(d), d.jtv_wadj.p, d.nv_wadj, nt, mode, tp.upv.p, tp.hiv.p,
                                        tp.sfv.p, tp.scale.p);
  OG_LAUNCHED();
}

// pass 5: tendency and update for limited tracers (scalar_tend_monot/_pd)
__global__ void k_tend(GridK g, const int* __restrict__ prog, int nprog, CTView scp_in, CTView scp0,
                       const float* __restrict__ rhos, const float* __restrict__ vmasc,
                       const float* __restrict__ wmasc, const float* __restrict__ ff,
                       const float* __restrict__ upv, const float* __restrict__ upw, TView out, int nt,
                       int istage, int nrk, float dtr, const int* __restrict__ mode) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * nt) return;
  const int mza = g.mza;
  int t = (int)(i % nt);
  if (mode[t] == MODE_PLAIN) return;
  int iw = prog[i / nt];
  int kb = g.lpw[iw];
  int np = g.npoly[iw];
  float fimpl = ff[(size_t)iw * nrk + istage - 1];
  const float* wm = wmasc + (size_t)iw * mza;
  const float* up = upw + (size_t)iw * mza * nt + t;
  for (int kd = kb; kd < mza; ++kd) {
    float s0 = scp0.base[((size_t)iw * mza + kd) * scp0.ld + scp0.t0 + t];
    float fd = 0.f;
    for (int n = 0; n < np; ++n) {
      int iv = g.w_ev[iw * 8 + n];
      if (kd < g.lpv[iv]) continue;
      fd = fd + g.w_dirv[iw * 8 + n] * vmasc[(size_t)iv * mza + kd] *
                    (upv[((size_t)iv * mza + kd) * nt + t] - s0);
    }
    float a = up[(size_t)(kd - 1) * nt], b = up[(size_t)kd * nt];
    if (fimpl > .001f) {
      float fexpl = 1.f - fimpl;
      fd = fd + fexpl * (wm[kd - 1] * (a - s0) - wm[kd] * (b - s0));
    } else {
      fd = fd + wm[kd - 1] * (a - s0) - wm[kd] * (b - s0);
    }
    out.base[((size_t)iw * mza + kd) * out.ld + out.t0 + t] =
        s0 + dtr * g.volti[(size_t)iw * mza + kd] * fd / rhos[(size_t)iw * mza + kd];
  }
  // The reference updates scp in place: scp(2:kb-1) = scp(kb) only in the
  // explicit branch, and levels it does not write keep the stage input.
  const float vkb = out.base[((size_t)iw * mza + kb) * out.ld + out.t0 + t];
  for (int kd = 0; kd < kb; ++kd) {
    const bool copy_kb = !(fimpl > .001f) && kd >= 1;
    out.base[((size_t)iw * mza + kd) * out.ld + out.t0 + t] =
        copy_kb ? vkb : scp_in.base[((size_t)iw * mza + kd) * scp_in.ld + scp_in.t0 + t];
  }
}

void launch_tend(const DevGrid& d, const Transport& tp, CTView scp_in, CTView scp0, const float* rhos,
                 TView out, int nt, int istage, int nrk, float dtr, const int* mode, cudaStream_t s) {
  size_t n = (size_t)d.nw_prog * nt;
  k_tend<<<cdiv(n, 128), 128, 0, s>>>(gridk(d), d.jtw_prog.p, d.nw_prog, scp_in, scp0, rhos, tp.vmasc.p,
                                      tp.wmasc.p, tp.ff.p, tp.upv.p, tp.upw.p, out, nt, istage, nrk, dtr,
                                      mode);
  OG_LAUNCHED();
}

// Points outside jtw_prog (OLAM's dummy point 1, and lateral-boundary or
// halo columns in other domains) are never updated; the reference keeps
// their values in place.  Stage outputs live in rotating buffers, so those
// columns are copied from the input into the final buffer.
__global__ void k_copy_cols(const int* __restrict__ cols, int ncol, const float* __restrict__ src,
                            float* __restrict__ dst, size_t colsize) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)ncol * colsize) return;
  size_t c = i / colsize, r = i % colsize;
  size_t off = (size_t)cols[c] * colsize + r;
  dst[off] = src[off];
}

void launch_copy_cols(const int* cols, int ncol, const float* src, float* dst, size_t colsize,
                      cudaStream_t s) {
  if (ncol <= 0) return;
  size_t n = (size_t)ncol * colsize;
  k_copy_cols<<<cdiv(n, 256), 256, 0, s>>>(cols, ncol, src, dst, colsize);
  OG_LAUNCHED();
}

// ---------------------------------------------------------------------------
// layout transposes.  q[(pk) * ntp + n] <-> src[n][pk], pk = point*mza + k.
// 32x32 tiles through shared memory; both sides coalesced.
// ---------------------------------------------------------------------------
// Layout transposes between the per-tracer arrays (one (mza, mwa) plane per
// tracer, the reference layout) and the batched layout Q[cell][ntp].  A
// thread moves a block of 4 cells x 8 tracers: eight 16-byte accesses along
// the cells of one tracer each (a warp covers 512 contiguous bytes per
// tracer) and four 32-byte accesses along the tracers of one cell each; the
// warps of a block take consecutive tracer octets of the same cells, so
// together they write (or read) whole rows of Q.  Tracers n .. ntp-1 of Q are
// zero.  Unaligned planes or a partial last quad take the element-wise path.
// width: tracer slots of a Q row written (a multiple of 4), stride: Q's row
// length; n <= width of them come from src, the rest are zero
__global__ void k_gather_q(float* __restrict__ q, const float* const* __restrict__ src, int n, int width,
                           int stride, size_t npk) {
  const size_t pk = ((size_t)blockIdx.x * 32 + threadIdx.x) * 4;
  const int t0 = (blockIdx.y * blockDim.y + threadIdx.y) * 8;
  if (pk >= npk || t0 >= width) return;
  const int nt = min(8, width - t0);   // 4 or 8
  const bool full = pk + 4 <= npk;
  float v[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i][0] = v[i][1] = v[i][2] = v[i][3] = 0.f;
    if (i < nt && t0 + i < n) {
      const float* p = src[t0 + i] + pk;
      if (full && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
        const float4 x = __ldcs(reinterpret_cast<const float4*>(p));
        v[i][0] = x.x; v[i][1] = x.y; v[i][2] = x.z; v[i][3] = x.w;
      } else {
        for (int j = 0; j < 4; ++j) if (pk + j < npk) v[i][j] = p[j];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (pk + j >= npk) break;
    float4* d = reinterpret_cast<float4*>(q + (pk + j) * stride + t0);
    __stcs(d, make_float4(v[0][j], v[1][j], v[2][j], v[3][j]));
    if (nt == 8) __stcs(d + 1, make_float4(v[4][j], v[5][j], v[6][j], v[7][j]));
  }
}

__global__ void k_scatter_q(const float* __restrict__ q, float* const* __restrict__ dst, int n, int width,
                            int stride, size_t npk) {
  const size_t pk = ((size_t)blockIdx.x * 32 + threadIdx.x) * 4;
  const int t0 = (blockIdx.y * blockDim.y + threadIdx.y) * 8;
  if (pk >= npk || t0 >= n) return;
  const int nt = min(8, width - t0);
  const bool full = pk + 4 <= npk;
  float v[8][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
    if (pk + j < npk) {
      const float4* sp = reinterpret_cast<const float4*>(q + (pk + j) * stride + t0);
      a = __ldcs(sp);
      if (nt == 8) b = __ldcs(sp + 1);
    }
    v[0][j] = a.x; v[1][j] = a.y; v[2][j] = a.z; v[3][j] = a.w;
    v[4][j] = b.x; v[5][j] = b.y; v[6][j] = b.z; v[7][j] = b.w;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i >= nt || t0 + i >= n) break;
    float* p = dst[t0 + i] + pk;
    if (full && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
      __stcs(reinterpret_cast<float4*>(p), make_float4(v[i][0], v[i][1], v[i][2], v[i][3]));
    } else {
      for (int j = 0; j < 4; ++j) if (pk + j < npk) p[j] = v[i][j];
    }
  }
}

// blocks of 32 cell quads x up to 16 tracer octets (warps)
static dim3 transpose_block(int ntr) { return dim3(32, std::max(1, std::min(16, (ntr + 7) / 8))); }

void launch_gather_q_range(float* q, const float* const* src, int n, int width, int stride, size_t npk,
                           cudaStream_t s) {
  const dim3 b = transpose_block(width);
  const dim3 grid(cdiv(cdiv(npk, 4), 32), cdiv(cdiv(width, 8), b.y));
  k_gather_q<<<grid, b, 0, s>>>(q, src, n, width, stride, npk);
  OG_LAUNCHED();
}

void launch_scatter_q_range(const float* q, float* const* dst, int n, int width, int stride, size_t npk,
                            cudaStream_t s) {
  const dim3 b = transpose_block(n);
  const dim3 grid(cdiv(cdiv(npk, 4), 32), cdiv(cdiv(n, 8), b.y));
  k_scatter_q<<<grid, b, 0, s>>>(q, dst, n, width, stride, npk);
  OG_LAUNCHED();
}

void launch_gather_q(float* q, const float* const* src, int n, int ntp, size_t npk, cudaStream_t s) {
  launch_gather_q_range(q, src, n, ntp, ntp, npk, s);
}

void launch_scatter_q(const float* q, float* const* dst, int n, int ntp, size_t npk, cudaStream_t s) {
  launch_scatter_q_range(q, dst, n, ntp, ntp, npk, s);
}

// ---------------------------------------------------------------------------
// Stage without allocation (olamgpu_update_scalar_noalloc): one explicit,
// unlimited RK stage of update_scalar for one tracer on device arrays the
// caller owns, through the plain passes above.  Its scratch -- the gradient
// planes (2 or 5 per cell), the V-face values and a zero implicit fraction
// per column -- lives in a fixed device array, so the call itself never
// allocates device memory.
// ---------------------------------------------------------------------------
// Scratch need in floats: i2d * mwa * mza (gradient planes, i2d = 2 for
// order 2 and 5 for order 3) + mva * mza (V-face values) + mwa (implicit
// fraction).  On the icosahedral grid (mwa = 10 NXP^2 + 3, mva = 30 NXP^2 + 1)
// with mza = 61 that fits up to NXP = 74 at order 2 and NXP = 58 at order 3.
#define NOALLOC_SCRATCH_FLOATS (16u << 20)   // 64 MiB
static __device__ __align__(256) float g_noalloc_scratch[NOALLOC_SCRATCH_FLOATS];

// Address of g_noalloc_scratch per device, looked up by the first call made
// with that device current and kept until olamgpu_finalize (after which an
// application may reset the device).  Guarded by a mutex: calls may come
// from several host threads.
static std::mutex g_noalloc_mu;
static float* g_noalloc_ptr[64] = {};

void noalloc_forget() {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  for (float*& p : g_noalloc_ptr) p = nullptr;
}

static int noalloc_scratch(int dev, float** out) {
  if (dev < 0 || dev >= 64) { set_error("device ordinal above 63"); return OLAMGPU_E_UNSUPPORTED; }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    float* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return OLAMGPU_E_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return OLAMGPU_OK;
}

static int update_scalar_noalloc(const float* scp, const float* scp0, const float* sct, const float* rhos,
                                 const float* vmasc, const float* wmasc, float dtr, float* out, void* stream) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!scp || !scp0 || !sct || !rhos || !vmasc || !wmasc || !out) {
    set_error("update_scalar_noalloc: NULL array");
    return OLAMGPU_E_ARG;
  }
  const DevGrid& d = C.g;
  const int order = C.opts.scal_horiz_adv_order;
  if (order != 2 && order != 3) { set_error("scal_horiz_adv_order must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  const size_t i2d = order == 3 ? 5 : 2;
  const size_t n_gx = i2d * d.mwa * d.mza, n_upv = (size_t)d.mva * d.mza, n_ff = d.mwa;
  const size_t need = n_gx + n_upv + n_ff;
  if (need > NOALLOC_SCRATCH_FLOATS) {
    set_error("update_scalar_noalloc: this grid needs " + std::to_string(need) +
              " floats of scratch; the fixed scratch holds " + std::to_string(NOALLOC_SCRATCH_FLOATS));
    return OLAMGPU_E_ARG;
  }
  // the grid tables live on the device olamgpu_init ran on: the call must
  // be made with that device current
  int dev = -1;
  OG_CUDA(cudaGetDevice(&dev));
  if (dev != C.device) {
    set_error("update_scalar_noalloc: device " + std::to_string(dev) + " is current, the library was initialised on " +
              std::to_string(C.device));
    return OLAMGPU_E_STATE;
  }
  float* scr = nullptr;
  OG_CHECK(noalloc_scratch(dev, &scr));
  float* gx = scr;
  float* upv = scr + n_gx;
  float* ff = upv + n_upv;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : C.stream;
  // every column explicit: the implicit fraction must read zero
  OG_CUDA(cudaMemsetAsync(ff, 0, n_ff * sizeof(float), s));
  const CTView in{scp, 1, 0}, in0{scp0, 1, 0}, tend{sct, 1, 0};
  const GridK g = gridk(d);
  const size_t ng = (size_t)d.nw_prog * d.mza;
  k_grad<<<cdiv(ng, 256), 256, 0, s>>>(g, d.jtw_prog.p, d.nw_prog, in, gx, 1, order, d.gxc.p, d.gyc.p, d.xy_h.p);
  const VCoef vc{d.dxps.p, d.dyps.p, d.xx0_v.p, d.xy0_v.p, d.yy0_v.p};
  const size_t nv = (size_t)d.nv_wadj * d.mza;
  k_vflux<<<cdiv(nv, 256), 256, 0, s>>>(g, d.jtv_wadj.p, d.nv_wadj, in, in0, gx, vmasc, 1, order, vc, nullptr,
                                        upv, nullptr, nullptr);
  WcolArgs A;
  A.g = g;
  A.prog = d.jtw_prog.p; A.nprog = d.nw_prog;
  A.scp = in; A.scp0 = in0; A.sct = tend; A.rhos = rhos;
  A.vmasc = vmasc; A.wmasc = wmasc; A.ff = ff;
  A.upv = upv; A.sfv = nullptr; A.scale = nullptr; A.upw = nullptr;
  A.out = TView{out, 1, 0}; A.nt = 1; A.istage = 1; A.nrk = 1; A.dtr = dtr;
  A.mode = nullptr;
  k_wcol<<<cdiv((size_t)d.nw_prog, 128), 128, 0, s>>>(A);
  OG_LAUNCHED(); OG_LAUNCHED(); OG_LAUNCHED();
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

}  // namespace olamgpu

extern "C" int olamgpu_update_scalar_noalloc(const float* scp, const float* scp0, const float* sct,
                                             const float* rhos, const float* vmasc, const float* wmasc,
                                             float dtr, float* out, void* stream) {
  return olamgpu::update_scalar_noalloc(scp, scp0, sct, rhos, vmasc, wmasc, dtr, out, stream);
}
