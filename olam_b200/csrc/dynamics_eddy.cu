// dynamics_eddy.cu -- eddy diffusion of heat and momentum inside the acoustic
// step's column set-up (omodel/prog_wrtv_rk.f90:214-251) and comp_horiz_k.
//
//   k_horiz_k   comp_horiz_k_column (convect/pbl_driver.f90:136-238): one
//               thread per (V point of jtv_wadj, level); writes akmodx,
//               akhodx and, on level 0, kmtopv / khtopv
//   k_eddy_w    one warp per column of jtw_prog, on the column's *_short
//               tendencies held in shared memory, in the reference's order:
//                 solve_eddy_diff_heat (pbl_driver.f90:519-624)
//                 solve_eddy_diff_vxe  (pbl_driver.f90:628-742)
//                 rayf_mix_top_vxe     (modules/mem_rayf.f90:177-220)
//                 the Rayleigh term on thil (prog_wrtv_rk.f90:226-233)
//                 horizontal diffusion of thil and the winds (:235-251)
//               lanes over levels for the coefficients and updates, lane 0
//               for tridiffo (tridiag_lib.f90:10-36), lanes 0-2 for the
//               three right-hand sides of tridv (tridiag_lib.f90:40-104)
// Column arrays in shared memory are indexed by the reference's level k
// (1-based); the global arrays by device level kd = k - 1.
#include <algorithm>
#include <vector>

#include "transport_kernels.cuh"

namespace olamgpu {

#define EDDY_WARPS 4
#define EDDY_ARRAYS 19

struct EddyArgs {
  int mza, mwa, nprog, nsw_max, krayfmix_bot, krayf_bot;
  int dcmip;            // DCMIP mixing test: no column eddy solves
  float dts, cp;
  const int* __restrict__ prog;
  const int* __restrict__ npoly;
  const int* __restrict__ w_nb;
  const int* __restrict__ w_ev;
  const int* __restrict__ lpw;
  const int* __restrict__ lpv;
  const float* __restrict__ volti;
  const float* __restrict__ arw;
  const float* __restrict__ arw0;
  const float* __restrict__ dzim;
  const float* __restrict__ dztbi;      // 1 / dzt_bot
  const double* __restrict__ rho;
  const double* __restrict__ volt;
  const float* __restrict__ thil;
  const float* __restrict__ vxe;
  const float* __restrict__ vye;
  const float* __restrict__ vze;
  const float* __restrict__ vkm;
  const float* __restrict__ vkh;
  const float* __restrict__ agamma;
  const float* __restrict__ akm_sfc;
  const float* __restrict__ sfluxt;
  const float* __restrict__ theta;
  const float* __restrict__ tair;
  const int* __restrict__ kmtop;
  const int* __restrict__ khtop;
  const int* __restrict__ kpblh;
  const int* __restrict__ lsw;
  const int* __restrict__ mrlw;
  const int* __restrict__ idiffk;
  const float* __restrict__ akmodx;
  const float* __restrict__ akhodx;
  const int* __restrict__ kmtopv;
  const int* __restrict__ khtopv;
  const float* __restrict__ rayf_cofmix;   // NULL: no top-level wind mixing
  const float* __restrict__ rayf_cof;      // NULL: no Rayleigh term on thil
  const float* __restrict__ dn01d;
  const float* __restrict__ th01d;
  float* __restrict__ sh_th;
  float* __restrict__ sh_vx;
  float* __restrict__ sh_vy;
  float* __restrict__ sh_vz;
};

__global__ void __launch_bounds__(EDDY_WARPS * 32) k_eddy_w(EddyArgs a) {
  extern __shared__ float esm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * EDDY_WARPS + warp;
  if (j >= a.nprog) return;
  const int mza = a.mza, n = mza + 2;
  float* base = esm + (size_t)warp * EDDY_ARRAYS * n;
  float* th = base;            // thilt_short, vm*et_short of the column
  float* vt[3] = {base + n, base + 2 * n, base + 3 * n};
  float* dtomass = base + 4 * n;
  float* v5 = base + 5 * n;
  float* v6 = base + 6 * n;
  float* v7 = base + 7 * n;
  float* v3 = base + 8 * n;
  float* akodz = base + 9 * n;
  float* rhs[3] = {base + 10 * n, base + 11 * n, base + 12 * n};   // tridv: solutions in place
  float* gam[3] = {base + 13 * n, base + 14 * n, base + 15 * n};
  float* varp = base + 16 * n;
  float* soln = base + 17 * n;
  float* scr = base + 18 * n;

  const int iw = a.prog[j];
  const int ka = a.lpw[iw] + 1;                       // reference level of the lowest T level
  const size_t cb = (size_t)iw * mza - 1;             // cb + k: column entry of level k
  const float* ve[3] = {a.vxe, a.vye, a.vze};
  float* sh[3] = {a.sh_vx, a.sh_vy, a.sh_vz};
  for (int k = ka + lane; k <= mza; k += 32) {
    th[k] = a.sh_th[cb + k];
    for (int c = 0; c < 3; ++c) vt[c][k] = sh[c][cb + k];
  }
  __syncwarp();

  // solve_eddy_diff_heat: implicit vertical diffusion of thil, flux form
  const int khtop = min(a.khtop[iw], mza - 1);
  if (!a.dcmip && khtop >= ka) {
    const int kmax = khtop + 1;
    for (int k = ka + lane; k <= kmax; k += 32) {
      const float dtom = a.dts * a.volti[cb + k] / (float)a.rho[cb + k];
      dtomass[k] = 1.1f * dtom;
      varp[k] = a.thil[cb + k] + dtom * th[k];
    }
    __syncwarp();
    for (int k = ka + lane; k <= khtop; k += 32) {
      const float ak = a.arw[cb + k] * a.vkh[cb + k] * a.dzim[k - 1];
      rhs[0][k] = ak * (varp[k] - varp[k + 1]);
      v5[k] = -ak * dtomass[k];
      v7[k] = -ak * dtomass[k + 1];
      v6[k] = 1.f - v5[k] - v7[k];
    }
    __syncwarp();
    // non-local PBL heat flux (idiffk = 1)
    if (a.idiffk[a.mrlw[iw] - 1] == 1 && a.agamma[cb + ka] > 1.e-7f * a.arw[cb + ka]) {
      const float wt0 = a.sfluxt[iw] * a.theta[cb + ka] / ((float)a.rho[cb + ka] * a.cp * a.tair[cb + ka]);
      const int kp = min(a.kpblh[iw], khtop);         // levels above khtop do not reach the solve
      for (int k = ka + lane; k <= kp; k += 32) rhs[0][k] = rhs[0][k] + wt0 * a.agamma[cb + k];
    }
    __syncwarp();
    if (lane == 0) {
      float cji = 1.f / v6[ka];
      soln[ka] = rhs[0][ka] * cji;
      for (int k = ka + 1; k <= khtop; ++k) {
        scr[k] = cji * v7[k - 1];
        cji = 1.f / (v6[k] - v5[k] * scr[k]);
        soln[k] = cji * (rhs[0][k] - v5[k] * soln[k - 1]);
      }
      for (int k = khtop - 1; k >= ka; --k) soln[k] = soln[k] - scr[k + 1] * soln[k + 1];
    }
    __syncwarp();
    for (int k = ka + lane; k <= kmax; k += 32) {
      const double fm = k - 1 >= ka ? (double)soln[k - 1] : 0.0;
      const double f = k <= kmax - 1 ? (double)soln[k] : 0.0;
      th[k] = th[k] + (float)(fm - f);
    }
    __syncwarp();
  }

  // solve_eddy_diff_vxe: implicit vertical diffusion of the three winds with
  // surface drag on the levels in contact with the surface
  if (!a.dcmip) {
    const int lsw = max(1, min(a.lsw[iw], mza - ka + 1));
    const int kmtop = min(a.kmtop[iw], mza - 1);
    const int kmax = max(kmtop + 1, ka + lsw - 1);
    for (int k = ka + lane; k <= kmax; k += 32) {
      const float akm1 = (k - 1 >= ka && k - 1 <= kmtop) ? a.arw[cb + k - 1] * a.vkm[cb + k - 1] * a.dzim[k - 2] : 0.f;
      const float ak = k <= kmtop ? a.arw[cb + k] * a.vkm[cb + k] * a.dzim[k - 1] : 0.f;
      akodz[k] = ak;
      const float dtom = (float)((double)(a.dts * a.volti[cb + k]) / a.rho[cb + k]);
      const float dm = 1.1f * dtom;
      const float l5 = -dm * akm1, l7 = -dm * ak;
      float l6 = 1.f - l5 - l7;
      float s3 = 0.f;
      if (k <= ka + lsw - 1) {
        s3 = a.akm_sfc[(size_t)iw * a.nsw_max + (k - ka)] * a.dztbi[k - 1];
        l6 = l6 + dm * s3;
      }
      v5[k] = l5; v6[k] = l6; v7[k] = l7; v3[k] = s3;
      for (int c = 0; c < 3; ++c) rhs[c][k] = ve[c][cb + k];
    }
    __syncwarp();
    if (lane < 3) {
      float* x = rhs[lane];
      float* gm = gam[lane];
      float bet = 1.f / v6[ka];
      x[ka] = bet * x[ka];
      for (int k = ka + 1; k <= kmax; ++k) {
        gm[k] = bet * v7[k - 1];
        bet = 1.f / (v6[k] - v5[k] * gm[k]);
        x[k] = bet * (x[k] - v5[k] * x[k - 1]);
      }
      for (int k = kmax - 1; k >= ka; --k) x[k] = x[k] - gm[k + 1] * x[k + 1];
    }
    __syncwarp();
    for (int k = ka + lane; k <= kmax; k += 32) {
      for (int c = 0; c < 3; ++c) {
        const float* x = rhs[c];
        const float v2m = (k - 1 >= ka) ? akodz[k - 1] * (x[k - 1] - x[k]) : 0.f;
        const float v2 = (k <= kmax - 1) ? akodz[k] * (x[k] - x[k + 1]) : 0.f;
        if (k <= ka + lsw - 1)
          vt[c][k] = vt[c][k] + (v2m - v2 - v3[k] * x[k]);
        else
          vt[c][k] = vt[c][k] + v2m - v2;
      }
    }
    __syncwarp();
  }

  // rayf_mix_top_vxe: mixing of the winds between the top levels
  if (a.rayf_cofmix && a.krayfmix_bot < mza) {
    const int kr = max(a.krayfmix_bot, ka);
    const float aw0 = a.arw0[iw];
    for (int k = kr + lane; k <= mza; k += 32) {
      for (int c = 0; c < 3; ++c) {
        float fm = 0.f, f = 0.f;
        if (k - 1 >= kr)
          fm = aw0 * a.rayf_cofmix[k - 2] * (float)(a.rho[cb + k] + a.rho[cb + k - 1]) *
               (ve[c][cb + k - 1] - ve[c][cb + k]);
        if (k <= mza - 1)
          f = aw0 * a.rayf_cofmix[k - 1] * (float)(a.rho[cb + k + 1] + a.rho[cb + k]) *
              (ve[c][cb + k] - ve[c][cb + k + 1]);
        vt[c][k] = vt[c][k] + fm - f;
      }
    }
  }

  // Rayleigh friction on thil, then horizontal diffusion
  const int np = a.npoly[iw];
  for (int k = ka + lane; k <= mza; k += 32) {
    float t = th[k];
    if (a.rayf_cof && k >= a.krayf_bot) {
      const float v4 = (float)a.volt[cb + k];
      t = t + a.rayf_cof[k - 1] * a.dn01d[k - 1] * (a.th01d[k - 1] - a.thil[cb + k]) * v4;
    }
    float u[3] = {vt[0][k], vt[1][k], vt[2][k]};
    for (int jv = 0; jv < np; ++jv) {
      const int iv = a.w_ev[iw * 8 + jv], iwn = a.w_nb[iw * 8 + jv];
      if (k < a.lpv[iv] + 1) continue;
      const size_t xn = (size_t)iwn * mza - 1 + k, xv = (size_t)iv * mza - 1 + k;
      if (k <= a.khtopv[iv]) t = t + a.akhodx[xv] * (a.thil[xn] - a.thil[cb + k]);
      if (k <= a.kmtopv[iv]) {
        const float m = a.akmodx[xv];
        for (int c = 0; c < 3; ++c) u[c] = u[c] + m * (ve[c][xn] - ve[c][cb + k]);
      }
    }
    a.sh_th[cb + k] = t;
    for (int c = 0; c < 3; ++c) sh[c][cb + k] = u[c];
  }
}

struct HorizKArgs {
  int mza, nv;
  float dtl;
  const int* __restrict__ vadj;
  const int* __restrict__ v_iw;
  const int* __restrict__ npoly;
  const int* __restrict__ lpv;
  const int* __restrict__ mrlv;
  const float* __restrict__ akmin;
  const int* __restrict__ kmtop;
  const int* __restrict__ khtop;
  const float* __restrict__ vkm;
  const float* __restrict__ vkh;
  const double* __restrict__ rho;
  const double* __restrict__ volt;
  const float* __restrict__ arw0;
  const float* __restrict__ arv;
  const float* __restrict__ dniv;
  float* __restrict__ akmodx;
  float* __restrict__ akhodx;
  int* __restrict__ kmtopv;
  int* __restrict__ khtopv;
};

__global__ void k_horiz_k(HorizKArgs a) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)a.nv * a.mza) return;
  const int mza = a.mza;
  const int iv = a.vadj[i / mza], k = (int)(i % mza) + 1;
  const int iw1 = a.v_iw[iv * 2], iw2 = a.v_iw[iv * 2 + 1];
  const float akmin = a.akmin[a.mrlv[iv] - 1];
  const int lpv = a.lpv[iv] + 1;
  const bool floor = akmin > 1.e-7f;
  int khv, kmv;
  if (floor) {
    khv = mza;
    kmv = mza;
  } else {
    khv = max(a.khtop[iw1], a.khtop[iw2]);
    khv = khv >= lpv ? khv + 1 : 1;
    kmv = max(a.kmtop[iw1], a.kmtop[iw2]);
    kmv = kmv >= lpv ? kmv + 1 : 1;
  }
  if (k == 1) { a.khtopv[iv] = khv; a.kmtopv[iv] = kmv; }
  if (k < lpv || k > min(mza, max(kmv, khv))) return;
  const size_t x1 = (size_t)iw1 * mza + k - 1, x2 = (size_t)iw2 * mza + k - 1;
  const float fact1 = 0.95f / (a.dtl * (float)a.npoly[iw1]);
  const float fact2 = 0.95f / (a.dtl * (float)a.npoly[iw2]);
  const float stab1 = (float)(a.rho[x1] * (double)(float)a.volt[x1] * (double)fact1);
  const float stab2 = (float)(a.rho[x2] * (double)(float)a.volt[x2] * (double)fact2);
  const float akstab = fminf(stab1, stab2);
  float hk0 = 0.f;
  if (floor) {
    const float bkmin = akmin * .075f * powf(fminf(a.arw0[iw1], a.arw0[iw2]), .66666666f);
    hk0 = 0.5f * (float)(a.rho[x1] + a.rho[x2]) * bkmin;
  }
  const float da = a.dniv[iv] * a.arv[(size_t)iv * mza + k - 1];
  if (k <= min(mza, kmv)) {
    float hkm = 0.25f * (a.vkm[x1] + a.vkm[x2] + a.vkm[x1 - 1] + a.vkm[x2 - 1]);
    if (floor) hkm = fmaxf(hkm, hk0);
    a.akmodx[(size_t)iv * mza + k - 1] = fminf(da * hkm, akstab);
  }
  if (k <= min(mza, khv)) {
    float hkh = 0.25f * (a.vkh[x1] + a.vkh[x2] + a.vkh[x1 - 1] + a.vkh[x2 - 1]);
    if (floor) hkh = fmaxf(hkh, hk0);
    a.akhodx[(size_t)iv * mza + k - 1] = fminf(da * hkh, akstab);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static bool dcmip_mixing_case(int tc) {
  return tc == 110 || tc == 111 || tc == 112 || tc == 113 || tc == 114 || tc == 121 || tc == 122;
}

// host -> device copies of the registered eddy inputs (and of comp_horiz_k's
// outputs unless the device holds newer ones)
int dyn_eddy_to_device(cudaStream_t s) {
  Context& C = ctx();
  Dyn& y = C.dy;
  if (!y.eddy_on) return OLAMGPU_OK;
  const olamgpu_eddy& e = y.heddy;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva, mwa = C.g.mwa, mva = C.g.mva;
  OG_CHECK(upload(y.e_vkm, e.vkm, wz, s));
  OG_CHECK(upload(y.e_vkh, e.vkh, wz, s));
  OG_CHECK(upload(y.e_agamma, e.agamma, wz, s));
  OG_CHECK(upload(y.e_theta, e.theta, wz, s));
  OG_CHECK(upload(y.e_tair, e.tair, wz, s));
  OG_CHECK(upload(y.e_akm_sfc, e.akm_sfc, mwa * (size_t)e.nsw_max, s));
  OG_CHECK(upload(y.e_sfluxt, e.sfluxt, mwa, s));
  OG_CHECK(upload(y.e_kmtop, e.kmtop, mwa, s));
  OG_CHECK(upload(y.e_khtop, e.khtop, mwa, s));
  OG_CHECK(upload(y.e_kpblh, e.kpblh, mwa, s));
  if (!y.hk_on_device) {
    OG_CHECK(upload(y.e_akmodx, e.akmodx, vz, s));
    OG_CHECK(upload(y.e_akhodx, e.akhodx, vz, s));
    OG_CHECK(upload(y.e_kmtopv, e.kmtopv, mva, s));
    OG_CHECK(upload(y.e_khtopv, e.khtopv, mva, s));
  }
  return OLAMGPU_OK;
}

// device -> host copies of comp_horiz_k's outputs
int dyn_eddy_to_host(cudaStream_t s) {
  Context& C = ctx();
  Dyn& y = C.dy;
  if (!y.eddy_on || !y.hk_on_device) return OLAMGPU_OK;
  const olamgpu_eddy& e = y.heddy;
  const size_t vz = (size_t)C.g.mza * C.g.mva, mva = C.g.mva;
  OG_CUDA(cudaMemcpyAsync(e.akmodx, y.e_akmodx.p, vz * 4, cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaMemcpyAsync(e.akhodx, y.e_akhodx.p, vz * 4, cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaMemcpyAsync(e.kmtopv, y.e_kmtopv.p, mva * 4, cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaMemcpyAsync(e.khtopv, y.e_khtopv.p, mva * 4, cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));
  y.hk_on_device = false;
  return OLAMGPU_OK;
}

int dyn_eddy_set(const olamgpu_eddy* e) {
  Context& C = ctx();
  Dyn& y = C.dy;
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!e) { y.eddy_on = false; y.hk_on_device = false; return OLAMGPU_OK; }
  if (!y.ready) { set_error("eddy diffusion needs prog_wrtv_rk's set-up (see olamgpu_init's status)"); return OLAMGPU_E_STATE; }
  const int mza = C.g.mza;
  if (!e->vkm || !e->vkh || !e->agamma || !e->akm_sfc || !e->sfluxt || !e->kmtop || !e->khtop || !e->kpblh ||
      !e->theta || !e->tair || !e->akmodx || !e->akhodx || !e->kmtopv || !e->khtopv || !e->lsw || !e->mrlw ||
      !e->mrlv || !e->idiffk || !e->akmin) {
    set_error("olamgpu_eddy: an array is NULL");
    return OLAMGPU_E_ARG;
  }
  if (e->nsw_max < 1 || e->mrls < 1) { set_error("olamgpu_eddy: nsw_max and mrls must be >= 1"); return OLAMGPU_E_ARG; }
  const olamgpu_grid& g = C.hgrid;
  if (!g.dzim || !g.dzt_bot) { set_error("eddy diffusion needs dzim and dzt_bot in olamgpu_grid"); return OLAMGPU_E_ARG; }
  const int mwa = C.g.mwa, mva = C.g.mva;
  // the kernels index idiffk / akmin by the refinement level and akm_sfc by
  // lsw at the points of jtw_prog and jtv_wadj only; elsewhere (the dummy
  // point 0, points outside the tables) the uploaded copies hold 1
  std::vector<int> mrlw(mwa, 1), mrlv(mva, 1), lsw(mwa, 1);
  for (int j = 0; j < g.nw_prog; ++j) {
    const int iw = g.jtw_prog[j] - 1;
    if (e->mrlw[iw] < 1 || e->mrlw[iw] > e->mrls || e->lsw[iw] < 1 || e->lsw[iw] > e->nsw_max) {
      set_error("olamgpu_eddy: mrlw or lsw out of range at W point " + std::to_string(iw + 1));
      return OLAMGPU_E_ARG;
    }
    mrlw[iw] = e->mrlw[iw];
    lsw[iw] = e->lsw[iw];
  }
  for (int j = 0; j < g.nv_wadj; ++j) {
    const int iv = g.jtv_wadj[j] - 1;
    if (e->mrlv[iv] < 1 || e->mrlv[iv] > e->mrls) {
      set_error("olamgpu_eddy: mrlv out of range at V point " + std::to_string(iv + 1));
      return OLAMGPU_E_ARG;
    }
    mrlv[iv] = e->mrlv[iv];
  }
  cudaStream_t s = C.stream;
  OG_CHECK(upload(y.e_mrlw, mrlw.data(), mwa, s));
  OG_CHECK(upload(y.e_mrlv, mrlv.data(), mva, s));
  OG_CHECK(upload(y.e_lsw, lsw.data(), mwa, s));
  OG_CHECK(upload(y.e_idiffk, e->idiffk, e->mrls, s));
  OG_CHECK(upload(y.e_akmin, e->akmin, e->mrls, s));
  std::vector<float> dztbi(mza);
  for (int k = 0; k < mza; ++k) dztbi[k] = 1.0f / g.dzt_bot[k];
  OG_CHECK(upload(y.e_dzim, g.dzim, mza, s));
  OG_CHECK(upload(y.e_dztbi, dztbi.data(), mza, s));
  const bool mix = e->rayf_cofmix && e->krayfmix_bot < mza;
  if (mix) {
    if (e->krayfmix_bot < 1) { set_error("olamgpu_eddy: krayfmix_bot must be >= 1"); return OLAMGPU_E_ARG; }
    OG_CHECK(upload(y.e_rayf, e->rayf_cofmix, mza, s));
  }
  y.heddy = *e;
  if (!mix) y.heddy.rayf_cofmix = nullptr;
  y.eddy_on = true;
  y.hk_on_device = false;
  OG_CHECK(dyn_eddy_to_device(s));
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

int dyn_comp_horiz_k() {
  Context& C = ctx();
  Dyn& y = C.dy;
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!y.eddy_on) { set_error("comp_horiz_k needs the eddy inputs (olamgpu_set_eddy)"); return OLAMGPU_E_STATE; }
  if (!C.have_state) { set_error("comp_horiz_k needs the state arrays registered at init"); return OLAMGPU_E_STATE; }
  cudaStream_t s = C.stream;
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  const bool sync = C.coherence == OLAMGPU_SYNC_EACH_CALL;
  if (!tp.rho.p) OG_CHECK(tp.rho.alloc((size_t)d.mza * d.mwa));
  if (sync || !y.uploaded) {
    OG_CHECK(dyn_state_to_device(OLAMGPU_F_RHO, s));
    OG_CHECK(dyn_eddy_to_device(s));
  }
  HorizKArgs a;
  a.mza = d.mza; a.nv = d.nv_wadj; a.dtl = (float)C.opts.dtlm;
  a.vadj = d.jtv_wadj.p; a.v_iw = d.v_iw.p; a.npoly = d.npoly.p; a.lpv = d.lpv.p;
  a.mrlv = y.e_mrlv.p; a.akmin = y.e_akmin.p; a.kmtop = y.e_kmtop.p; a.khtop = y.e_khtop.p;
  a.vkm = y.e_vkm.p; a.vkh = y.e_vkh.p; a.rho = tp.rho.p; a.volt = y.volt.p; a.arw0 = y.arw0.p;
  a.arv = y.arv.p; a.dniv = y.dniv.p;
  a.akmodx = y.e_akmodx.p; a.akhodx = y.e_akhodx.p; a.kmtopv = y.e_kmtopv.p; a.khtopv = y.e_khtopv.p;
  if (d.nv_wadj > 0) {
    k_horiz_k<<<cdiv((size_t)d.nv_wadj * d.mza, 256), 256, 0, s>>>(a);
    OG_LAUNCHED();
  }
  y.hk_on_device = true;
  // scalar transport's horizontal diffusion reads the same akhodx / khtopv
  const size_t vz = (size_t)d.mza * d.mva;
  OG_CHECK(tp.akhodx.alloc(vz));
  OG_CHECK(tp.khtopv.alloc(d.mva));
  OG_CUDA(cudaMemcpyAsync(tp.akhodx.p, y.e_akhodx.p, vz * 4, cudaMemcpyDeviceToDevice, s));
  OG_CUDA(cudaMemcpyAsync(tp.khtopv.p, y.e_khtopv.p, (size_t)d.mva * 4, cudaMemcpyDeviceToDevice, s));
  tp.have_turb = true;
  if (sync) OG_CHECK(dyn_eddy_to_host(s));
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

int dyn_eddy_columns(Context& C, bool rayleigh, cudaStream_t s) {
  Dyn& y = C.dy;
  const DevGrid& d = C.g;
  const olamgpu_opts& o = C.opts;
  const olamgpu_eddy& e = y.heddy;
  EddyArgs a;
  a.mza = d.mza; a.mwa = d.mwa; a.nprog = d.nw_prog; a.nsw_max = e.nsw_max;
  a.krayfmix_bot = e.krayfmix_bot; a.krayf_bot = o.krayf_bot;
  a.dcmip = dcmip_mixing_case(e.test_case);
  a.dts = (float)o.dtsm; a.cp = e.cp;
  a.prog = d.jtw_prog.p; a.npoly = d.npoly.p; a.w_nb = d.w_nb.p; a.w_ev = d.w_ev.p; a.lpw = d.lpw.p;
  a.lpv = d.lpv.p; a.volti = d.volti.p; a.arw = y.arw.p; a.arw0 = y.arw0.p; a.dzim = y.e_dzim.p;
  a.dztbi = y.e_dztbi.p; a.rho = C.tp.rho.p; a.volt = y.volt.p; a.thil = y.thil.p; a.vxe = y.vxe.p;
  a.vye = y.vye.p; a.vze = y.vze.p; a.vkm = y.e_vkm.p; a.vkh = y.e_vkh.p; a.agamma = y.e_agamma.p;
  a.akm_sfc = y.e_akm_sfc.p; a.sfluxt = y.e_sfluxt.p; a.theta = y.e_theta.p; a.tair = y.e_tair.p;
  a.kmtop = y.e_kmtop.p; a.khtop = y.e_khtop.p; a.kpblh = y.e_kpblh.p; a.lsw = y.e_lsw.p;
  a.mrlw = y.e_mrlw.p; a.idiffk = y.e_idiffk.p; a.akmodx = y.e_akmodx.p; a.akhodx = y.e_akhodx.p;
  a.kmtopv = y.e_kmtopv.p; a.khtopv = y.e_khtopv.p;
  a.rayf_cofmix = e.rayf_cofmix ? y.e_rayf.p : nullptr;
  a.rayf_cof = rayleigh ? y.rayf_cof.p : nullptr;
  a.dn01d = y.dn01d.p; a.th01d = y.th01d.p;
  a.sh_th = y.sh_th.p; a.sh_vx = y.sh_vx.p; a.sh_vy = y.sh_vy.p; a.sh_vz = y.sh_vz.p;
  if (d.nw_prog <= 0) return OLAMGPU_OK;
  const size_t smem = (size_t)EDDY_WARPS * EDDY_ARRAYS * (d.mza + 2) * sizeof(float);
  k_eddy_w<<<cdiv(d.nw_prog, EDDY_WARPS), EDDY_WARPS * 32, smem, s>>>(a);
  OG_LAUNCHED();
  return OLAMGPU_OK;
}

void dyn_eddy_release() {
  Dyn& y = ctx().dy;
  DevBuf<float>* f[] = {&y.e_vkm, &y.e_vkh, &y.e_agamma, &y.e_theta, &y.e_tair, &y.e_akm_sfc, &y.e_sfluxt,
                        &y.e_akmodx, &y.e_akhodx, &y.e_dzim, &y.e_dztbi, &y.e_akmin, &y.e_rayf};
  for (auto* b : f) b->release();
  DevBuf<int>* i[] = {&y.e_kmtop, &y.e_khtop, &y.e_kpblh, &y.e_kmtopv, &y.e_khtopv, &y.e_lsw, &y.e_mrlw,
                      &y.e_mrlv, &y.e_idiffk};
  for (auto* b : i) b->release();
  y.eddy_on = false;
  y.hk_on_device = false;
}

}  // namespace olamgpu
