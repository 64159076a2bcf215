// transport.cu -- scalar_transport_rk driver (omodel/scalar_transport_rk.F90:30-385).
//
// Call sequence per long step, all on the library stream:
//   check_cfls -> ff_implic and the CFL maxima           (:113)
//   rhos(:,:,1..nrk)                                     (:117-152)
//   implicit-column factorisation per stage             (:164-217)
//   per RK stage: update of every tracer, then the implicit vertical solve
// The fused form updates all tracers of a stage in one launch on the batched
// layout; the plain form runs the reference's passes tracer by tracer.
// Stage outputs rotate through three buffers (scp0 stays intact), so no
// stage writes a field another thread of the same launch still reads.
#include <algorithm>
#include <cstring>
#include <utility>

#include "transport_kernels.cuh"

namespace olamgpu {

static int mode_for(const Context& C, int n) {
  int imonot = C.opts.iscal_monot;
  if (imonot == 1) return MODE_MONOT;
  if (imonot == 2 && C.tr.pdef[n]) return MODE_PD;
  return MODE_PLAIN;
}

// The last RK stage's mode of every tracer (d_mode[0, n)) and the flags of
// the tracers whose scp0 takes the low-order pre-update (d_mode[n, 2n)),
// uploaded when they change only (the upload reads pageable host memory,
// which a recorded step could not repeat).
int tracer_modes(Context& C, std::vector<int>& modes, std::vector<int>& pdm, bool& anylim, bool& any_pdm) {
  Tracers& tr = C.tr;
  Transport& tp = C.tp;
  modes.assign(tr.n, MODE_PLAIN);
  pdm.assign(tr.n, 0);
  anylim = any_pdm = false;
  for (int n = 0; n < tr.n; ++n) {
    modes[n] = mode_for(C, n);
    anylim |= modes[n] != MODE_PLAIN;
    pdm[n] = (C.opts.iscal_monot > 0 && tr.pdef[n]) ? 1 : 0;
    any_pdm |= pdm[n] != 0;
  }
  std::vector<int> hm(modes);
  hm.insert(hm.end(), pdm.begin(), pdm.end());
  if (hm != tp.h_mode || !tp.d_mode.p) {
    OG_CHECK(tp.d_mode.alloc((size_t)std::max(tr.n, 1) * 2));
    if (tr.n > 0) {
      OG_CUDA(cudaMemcpyAsync(tp.d_mode.p, hm.data(), hm.size() * sizeof(int), cudaMemcpyHostToDevice, C.stream));
      OG_CUDA(cudaStreamSynchronize(C.stream));
    }
    tp.h_mode = hm;
  }
  return OLAMGPU_OK;
}

int tracers_to_device(cudaStream_t s) {
  Context& C = ctx();
  Tracers& tr = C.tr;
  const size_t plane = (size_t)C.g.mza * C.g.mwa;
  for (int n = 0; n < tr.n; ++n) {
    OG_CUDA(cudaMemcpyAsync(tr.p[n].p, tr.h_p[n], plane * sizeof(float), cudaMemcpyHostToDevice, s));
    OG_CUDA(cudaMemcpyAsync(tr.t[n].p, tr.h_t[n], plane * sizeof(float), cudaMemcpyHostToDevice, s));
  }
  tr.q_valid = false;
  return OLAMGPU_OK;
}

static int pointer_table(std::vector<DevBuf<float>>& bufs, DevBuf<float*>& dst, cudaStream_t s) {
  std::vector<float*> h(bufs.size());
  for (size_t i = 0; i < bufs.size(); ++i) {
    h[i] = bufs[i].p;
    if (!h[i]) { set_error("a per-tracer device array is missing"); return OLAMGPU_E_STATE; }
  }
  OG_CHECK(dst.alloc(std::max<size_t>(h.size(), 1)));
  if (!h.empty())
    OG_CUDA(cudaMemcpyAsync(dst.p, h.data(), h.size() * sizeof(float*), cudaMemcpyHostToDevice, s));
  // the host vector dies here: make the copy complete first
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

static DevBuf<float*> g_ptab;

int ensure_q(cudaStream_t s) {
  Context& C = ctx();
  Tracers& tr = C.tr;
  if (tr.q_valid) return OLAMGPU_OK;
  const size_t npk = (size_t)C.g.mza * C.g.mwa;
  for (int b = 0; b < 3; ++b) OG_CHECK(tr.q[b].alloc(npk * tr.ntp));
  OG_CHECK(tr.qt.alloc(npk * tr.ntp));
  OG_CHECK(pointer_table(tr.p, g_ptab, s));
  launch_gather_q(tr.q[tr.qcur].p, (const float* const*)g_ptab.p, tr.n, tr.ntp, npk, s);
  OG_CHECK(pointer_table(tr.t, g_ptab, s));
  launch_gather_q(tr.qt.p, (const float* const*)g_ptab.p, tr.n, tr.ntp, npk, s);
  OG_CUDA(cudaStreamSynchronize(s));
  tr.q_valid = true;
  return OLAMGPU_OK;
}

int ensure_plain(cudaStream_t s) {
  Context& C = ctx();
  Tracers& tr = C.tr;
  if (!tr.q_valid) return OLAMGPU_OK;
  const size_t npk = (size_t)C.g.mza * C.g.mwa;
  OG_CHECK(pointer_table(tr.p, g_ptab, s));
  launch_scatter_q(tr.q[tr.qcur].p, (float* const*)g_ptab.p, tr.n, tr.ntp, npk, s);
  OG_CHECK(pointer_table(tr.t, g_ptab, s));
  launch_scatter_q(tr.qt.p, (float* const*)g_ptab.p, tr.n, tr.ntp, npk, s);
  OG_CUDA(cudaStreamSynchronize(s));
  tr.q_valid = false;
  return OLAMGPU_OK;
}

int tracers_to_host(cudaStream_t s) {
  Context& C = ctx();
  Tracers& tr = C.tr;
  OG_CHECK(ensure_plain(s));
  const size_t plane = (size_t)C.g.mza * C.g.mwa;
  for (int n = 0; n < tr.n; ++n) {
    OG_CUDA(cudaMemcpyAsync(tr.h_p[n], tr.p[n].p, plane * sizeof(float), cudaMemcpyDeviceToHost, s));
    // tendencies change on the device only through the diffusion hook
    if (C.tp.have_turb && tr.sgsmix[n])
      OG_CUDA(cudaMemcpyAsync(tr.h_t[n], tr.t[n].p, plane * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  return OLAMGPU_OK;
}

// scratch of the reference-mirroring passes for a group of nt tracers
static int ensure_pass_scratch(Context& C, int nt, int order) {
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  const size_t wz = (size_t)d.mwa * d.mza * nt, vz = (size_t)d.mva * d.mza * nt;
  const int i2d = order == 3 ? 5 : 2;
  auto grow = [](DevBuf<float>& b, size_t n) { return b.n >= n ? OLAMGPU_OK : b.alloc(n); };
  OG_CHECK(grow(tp.gx, wz * i2d));
  OG_CHECK(grow(tp.upv, vz));
  OG_CHECK(grow(tp.hiv, vz));
  OG_CHECK(grow(tp.sfv, vz));
  OG_CHECK(grow(tp.scale, wz * 2));
  OG_CHECK(grow(tp.upw, wz));
  return OLAMGPU_OK;
}

// one RK stage through the reference's passes for tracers [t0, t0+nt) of a view
static void passes_stage(Context& C, CTView in, CTView scp0, CTView sct, TView out, int nt,
                         int istage, int nrk, float dtr, const float* rhos, const int* mode,
                         bool limited_stage, cudaStream_t s) {
  const DevGrid& d = C.g;
  const int order = C.opts.scal_horiz_adv_order;
  const bool monot = limited_stage && C.opts.iscal_monot == 1;
  { OG_PROF("pass_grad", s); launch_grad(d, in, C.tp.gx.p, nt, order, !monot, s); }
  { OG_PROF("pass_vflux", s); launch_vflux(d, C.tp, in, scp0, C.tp.gx.p, nt, order, monot, mode, limited_stage, s); }
  if (limited_stage) {
    // the limiters' scale factors run down each column (a thread per column)
    OG_PROF("pass_wcol", s);
    launch_wcol(d, C.tp, in, scp0, sct, rhos, out, nt, istage, nrk, dtr, mode, limited_stage, s);
  } else {
    OG_PROF("pass_wcol", s);
    launch_wcell(d, C.tp, in, scp0, sct, rhos, out, nt, istage, nrk, dtr, s);
  }
  if (limited_stage) {
    { OG_PROF("pass_vapply", s); launch_vapply(d, C.tp, nt, mode, s); }
    { OG_PROF("pass_tend", s); launch_tend(d, C.tp, in, scp0, rhos, out, nt, istage, nrk, dtr, mode, s); }
  }
}

// Inputs and per-step coefficients shared by the transport and its adjoint:
// winds and densities on the device (uploaded in SYNC_EACH_CALL mode, or on
// first use in RESIDENT mode), then check_cfls (ff_implic and the CFL
// maxima), the stage densities rhos and the implicit columns' factors.
int transport_prepare(Context& C, const float* rho_old_host, bool upload_tracers, float dtlr[3]) {
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  cudaStream_t s = C.stream;
  const int mza = d.mza, mwa = d.mwa, mva = d.mva;
  const int nrk = C.opts.nrk_scal;
  const size_t wz = (size_t)mza * mwa, vz = (size_t)mza * mva;
  // ---- inputs
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    if (!rho_old_host) { set_error("rho_old is NULL"); return OLAMGPU_E_ARG; }
    OG_CHECK(upload(tp.vmasc, C.hstate.vmasc, vz, s));
    OG_CHECK(upload(tp.wmasc, C.hstate.wmasc, wz, s));
    OG_CHECK(upload(tp.rho, C.hstate.rho, wz, s));
    if (C.hstate.wc) OG_CHECK(upload(tp.wc, C.hstate.wc, wz, s));
    OG_CHECK(upload(tp.rho_old, rho_old_host, wz, s));
    if (upload_tracers) OG_CHECK(tracers_to_device(s));
  } else {
    // RESIDENT: device copies persist; a field never uploaded is taken from
    // the registered host array on first use (the dynamics keeps them when
    // it runs on the device)
    if (C.dy.ready && !C.dy.uploaded) {
      OG_CHECK(dyn_state_to_device(OLAMGPU_F_ALL, s));
      C.dy.uploaded = true;
    }
    bool copied = false;
    if (!tp.vmasc.p) { OG_CHECK(upload(tp.vmasc, C.hstate.vmasc, vz, s)); copied = true; }
    if (!tp.wmasc.p) { OG_CHECK(upload(tp.wmasc, C.hstate.wmasc, wz, s)); copied = true; }
    if (!tp.rho.p) { OG_CHECK(upload(tp.rho, C.hstate.rho, wz, s)); copied = true; }
    if (!tp.wc.p && C.hstate.wc) { OG_CHECK(upload(tp.wc, C.hstate.wc, wz, s)); copied = true; }
    if (rho_old_host) { OG_CHECK(upload(tp.rho_old, rho_old_host, wz, s)); copied = true; }
    // page-locked sources are read when the copies run
    if (copied) OG_CUDA(cudaStreamSynchronize(s));
    if (!tp.rho_old.p) {
      set_error("rho_old is NULL and no device copy exists (pass it once or call olamgpu_tend0)");
      return OLAMGPU_E_STATE;
    }
  }
  if (!tp.vmasc.p || !tp.wmasc.p || !tp.rho.p || !tp.rho_old.p) {
    set_error("transport inputs missing on the device");
    return OLAMGPU_E_STATE;
  }
  OG_CHECK(tp.rhos.alloc((size_t)nrk * wz));
  OG_CHECK(tp.ff.alloc((size_t)nrk * mwa));
  OG_CHECK(tp.imp_list.alloc((size_t)nrk * mwa));
  OG_CHECK(tp.imp_count.alloc(3));
  OG_CHECK(tp.imp_b.alloc((size_t)nrk * mwa * 3 * mza));
  OG_CHECK(tp.cfl_loc.alloc(6));

  const float dtl = (float)C.opts.dtlm;
  const float one3 = 1.f / 3.f;
  for (int n = 0; n < nrk; ++n) dtlr[n] = dtl * (nrk == 3 ? (n == 0 ? one3 : (n == 1 ? 0.5f : 1.0f))
                                                          : (n == 0 ? 0.5f : 1.0f));
  { OG_PROF("check_cfls", s); launch_check_cfls(d, tp, nrk, dtl, tp.cfl_loc.p, s); }
  { OG_PROF("rhos", s); launch_rhos(d, tp, nrk, s); }
  { OG_PROF("implicit_prep", s); launch_implicit_prep(d, tp, nrk, dtlr, s); }
  return OLAMGPU_OK;
}

void transport_release_pipeline() {
  Transport& tp = ctx().tp;
  for (cudaEvent_t e : tp.ev) cudaEventDestroy(e);
  tp.ev.clear();
  if (tp.s_up) cudaStreamDestroy(tp.s_up);
  if (tp.s_dn) cudaStreamDestroy(tp.s_dn);
  tp.s_up = tp.s_dn = nullptr;
  tp.ptab_p.release();
  tp.ptab_t.release();
}

// The per-call step in tracer groups of 64 (one tile group each): the
// host->device copies of a group's scp and sct (stream s_up), its gather
// into the batched layout, its RK stages and its scatter back (the library
// stream), and the device->host copies of its result (stream s_dn) are
// ordered by events, so group g's step overlaps group g+1's copies in and
// group g-1's copies out on the two copy engines.  The state and the
// step's records are on the device already (transport_prepare, k_weights).
static int pipelined_step(Context& C, const float* dtlr, const float* rhos_nrk) {
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  Tracers& tr = C.tr;
  cudaStream_t s = C.stream;
  const int nrk = C.opts.nrk_scal, ntp = tr.ntp, n = tr.n;
  const size_t npk = (size_t)d.mza * d.mwa, plane = npk * sizeof(float);
  const int ngrp = (ntp + 63) / 64;
  if (!tp.s_up) OG_CUDA(cudaStreamCreateWithFlags(&tp.s_up, cudaStreamNonBlocking));
  if (!tp.s_dn) OG_CUDA(cudaStreamCreateWithFlags(&tp.s_dn, cudaStreamNonBlocking));
  while ((int)tp.ev.size() < 2 * ngrp + 1) {
    cudaEvent_t e;
    OG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    tp.ev.push_back(e);
  }
  for (int b = 0; b < 3; ++b) OG_CHECK(tr.q[b].alloc(npk * ntp));
  OG_CHECK(tr.qt.alloc(npk * ntp));
  {
    std::vector<float*> hp(n), ht(n);
    for (int i = 0; i < n; ++i) { hp[i] = tr.p[i].p; ht[i] = tr.t[i].p; }
    OG_CHECK(tp.ptab_p.alloc(n));
    OG_CHECK(tp.ptab_t.alloc(n));
    OG_CUDA(cudaMemcpyAsync(tp.ptab_p.p, hp.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
    OG_CUDA(cudaMemcpyAsync(tp.ptab_t.p, ht.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
    OG_CUDA(cudaStreamSynchronize(s));   // the host vectors die here
  }
  { OG_PROF("tile_weights", s); OG_CHECK(launch_tile_weights(d, tp, rhos_nrk, s)); }
  if (tp.autotune && tp.tuned_ntp != ntp) {
    // the shape on this step's inputs: the tracers' device copies and the
    // step's records (a rotation buffer as the scratch output)
    OG_CHECK(ensure_q(s));
    OG_CHECK(tile_autotune(C, tr.q[tr.qcur].p, tr.q[tr.qcur].p, tr.qt.p, tr.q[(tr.qcur + 1) % 3].p, dtlr[nrk - 1]));
    tr.q_valid = false;   // the per-tracer arrays are what the pipelined step reads
  }
  // the RK buffer sequence of the batched step
  const int a = tr.qcur;
  int bin[3], bout[3];
  {
    int in_b = a, out_b = (a + 1) % 3;
    for (int k = 0; k < nrk; ++k) {
      bin[k] = in_b;
      bout[k] = out_b;
      in_b = out_b;
      out_b = (out_b + 1) % 3;
      if (out_b == a) out_b = (out_b + 1) % 3;
    }
  }
  const int fin = bout[nrk - 1];
  // copies in may start at once: the previous call has ended
  for (int g = 0; g < ngrp; ++g) {
    const int tb = 64 * g, tc = std::min(64, n - tb), width = std::min(64, ntp - tb);
    if (tc <= 0) break;
    for (int i = tb; i < tb + tc; ++i) {
      OG_CUDA(cudaMemcpyAsync(tr.p[i].p, tr.h_p[i], plane, cudaMemcpyHostToDevice, tp.s_up));
      OG_CUDA(cudaMemcpyAsync(tr.t[i].p, tr.h_t[i], plane, cudaMemcpyHostToDevice, tp.s_up));
    }
    OG_CUDA(cudaEventRecord(tp.ev[2 * g], tp.s_up));
    OG_CUDA(cudaStreamWaitEvent(s, tp.ev[2 * g], 0));
    float* A = tr.q[a].p;
    launch_gather_q_range(A + tb, (const float* const*)tp.ptab_p.p + tb, tc, width, ntp, npk, s);
    launch_gather_q_range(tr.qt.p + tb, (const float* const*)tp.ptab_t.p + tb, tc, width, ntp, npk, s);
    for (int istage = 1; istage <= nrk; ++istage) {
      const float dtr = dtlr[istage - 1];
      float* IN = tr.q[bin[istage - 1]].p;
      float* OUT = tr.q[bout[istage - 1]].p;
      {
        OG_PROF(istage == 1 ? "tile_stage1" : "tile_stage", s);
        OG_CHECK(launch_tile_stage(d, tp, IN, A, tr.qt.p, OUT, ntp, istage, nrk, dtr, C.status.p, s, g, 1, 64));
      }
      {
        OG_PROF("implicit_solve", s);
        launch_implicit_solve(d, tp, nrk, istage, dtr, CTView{A, ntp, tb}, TView{OUT, ntp, tb}, width, s);
      }
    }
    launch_scatter_q_range(tr.q[fin].p + tb, tp.ptab_p.p + tb, tc, width, ntp, npk, s);
    OG_CUDA(cudaEventRecord(tp.ev[2 * g + 1], s));
    OG_CUDA(cudaStreamWaitEvent(tp.s_dn, tp.ev[2 * g + 1], 0));
    for (int i = tb; i < tb + tc; ++i)
      OG_CUDA(cudaMemcpyAsync(tr.h_p[i], tr.p[i].p, plane, cudaMemcpyDeviceToHost, tp.s_dn));
  }
  // the library stream ends after the last copy out
  OG_CUDA(cudaEventRecord(tp.ev[2 * ngrp], tp.s_dn));
  OG_CUDA(cudaStreamWaitEvent(s, tp.ev[2 * ngrp], 0));
  tr.qcur = fin;
  tr.q_valid = false;   // the per-tracer arrays hold the result too
  return OLAMGPU_OK;
}

int transport_run(const float* rho_old_host, olamgpu_cfl_diag* diag) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!C.have_state || !C.hstate.vmasc || !C.hstate.wmasc || !C.hstate.rho) {
    set_error("state arrays vmasc/wmasc/rho were not registered at init");
    return OLAMGPU_E_STATE;
  }
  if (C.tr.n <= 0) return OLAMGPU_OK;  // num_scalar = 0: the loop body never runs
  const DevGrid& d = C.g;
  Transport& tp = C.tp;
  Tracers& tr = C.tr;
  cudaStream_t s = C.stream;
  const int mza = d.mza, mwa = d.mwa, mva = d.mva;
  const int nrk = C.opts.nrk_scal;
  const int order = C.opts.scal_horiz_adv_order;
  const size_t wz = (size_t)mza * mwa;
  if (nrk != 2 && nrk != 3) { set_error("scalar_timestep_level must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (order != 2 && order != 3) { set_error("scal_horiz_adv_order must be 2 or 3"); return OLAMGPU_E_UNSUPPORTED; }
  if (C.opts.iscal_monot < 0 || C.opts.iscal_monot > 2) { set_error("iscal_monot must be 0, 1 or 2"); return OLAMGPU_E_UNSUPPORTED; }
  const bool batched = C.form != OLAMGPU_TRANSPORT_PLAIN;
  const bool tiled = C.form == OLAMGPU_TRANSPORT_FUSED && tile_stage_available(d, tp, order);
  if (C.halo.on && (!batched || C.opts.iscal_monot != 0)) {
    set_error("a halo exchange needs the unlimited step (iscal_monot = 0) in a batched transport form");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (batched && !tiled && !tp.flat) {
    set_error("the per-column fused transport form needs lpw = lpv = 2 (no terrain); use the tiled or plain form");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (batched && !tiled && (double)mwa * mza * (double)((tr.ntp + 3) / 4 * 2) >= 4294967296.0) {
    set_error("the fused transport form needs mwa * mza * ntp / 2 < 2^32; use the plain form");
    return OLAMGPU_E_UNSUPPORTED;
  }
  if (batched && !tiled && d.ew_order != order)
    OG_CHECK(build_fused_weights(&C.hgrid, C.g, order, s));

  // per-call step (SYNC_EACH_CALL) of the tiled, unlimited step on a global
  // domain: the tracers go through in groups of 64 so that the copies in,
  // the step and the copies out of different groups overlap
  const bool pipelined = C.coherence == OLAMGPU_SYNC_EACH_CALL && tiled && C.opts.iscal_monot == 0 &&
                         !tp.have_turb && !C.halo.on && d.n_nonprog == 0 && tr.n > 64 &&
                         tile_shape_fits(d, 64);   // its groups are 64 tracers wide
  float dtlr[3];
  OG_CHECK(transport_prepare(C, rho_old_host, !pipelined, dtlr));
  const float* rhos_nrk = tp.rhos.p + (size_t)(nrk - 1) * wz;

  // last-stage mode per tracer
  std::vector<int> modes, pdm;
  bool anylim = false, any_pdm = false;
  OG_CHECK(tracer_modes(C, modes, pdm, anylim, any_pdm));

  if (pipelined) {
    OG_CHECK(pipelined_step(C, dtlr, rhos_nrk));
  } else if (batched) {
    OG_CHECK(ensure_q(s));
    const int ntp = tr.ntp;
    const int a = tr.qcur;
    float* A = tr.q[a].p;
    float* T = tr.qt.p;
    // horizontal diffusion into the tendencies, per flagged tracer
    if (tp.have_turb)
      for (int n = 0; n < tr.n; ++n)
        if (tr.sgsmix[n]) launch_diffusion(d, tp, CTView{A, ntp, n}, TView{T, ntp, n}, 1, s);
    if (tiled) {
      OG_PROF("tile_weights", s);
      OG_CHECK(launch_tile_weights(d, tp, rhos_nrk, s));
      // the stage kernel's shape for this grid and tracer count, chosen on
      // this step's inputs (the next rotation buffer is scratch)
      if (tp.autotune && tp.tuned_ntp != ntp)
        OG_CHECK(tile_autotune(C, A, A, T, tr.q[(a + 1) % 3].p, dtlr[nrk - 1]));
    }
    int in_b = a, out_b = (a + 1) % 3;
    for (int istage = 1; istage <= nrk; ++istage) {
      const float dtr = dtlr[istage - 1];
      float* IN = tr.q[in_b].p;
      float* OUT = tr.q[out_b].p;
      const bool last = istage == nrk;
      if (last && any_pdm)
        launch_scp0_pd_update(d, tp, TView{A, ntp, 0}, CTView{T, ntp, 0}, tp.d_mode.p + tr.n, tr.n, dtr, s);
      if (last && anylim) {
        // limited last stage: the reference's passes over tracer groups sized
        // to a scratch budget
        const size_t per = (size_t)4 * mza * ((size_t)7 * mwa + (size_t)3 * mva) + 1;
        int grp = (int)std::max<size_t>(1, std::min<size_t>((size_t)tr.n, (size_t)(8ull << 30) / per));
        OG_CHECK(ensure_pass_scratch(C, grp, order));
        for (int g0 = 0; g0 < tr.n; g0 += grp) {
          int nt = std::min(grp, tr.n - g0);
          passes_stage(C, CTView{IN, ntp, g0}, CTView{A, ntp, g0}, CTView{T, ntp, g0},
                       TView{OUT, ntp, g0}, nt, istage, nrk, dtr, rhos_nrk, tp.d_mode.p + g0, true, s);
        }
      } else {
        OG_PROF(tiled ? (istage == 1 ? "tile_stage1" : "tile_stage") : (istage == 1 ? "fused_stage1" : "fused_stage"), s);
        if (tiled) OG_CHECK(launch_tile_stage(d, tp, IN, A, T, OUT, ntp, istage, nrk, dtr, C.status.p, s));
        else launch_fused_stage(d, tp, IN, A, T, OUT, ntp, istage, nrk, dtr, rhos_nrk, s);
      }
      { OG_PROF("implicit_solve", s); launch_implicit_solve(d, tp, nrk, istage, dtr, CTView{A, ntp, 0}, TView{OUT, ntp, 0}, ntp, s); }
      // border columns for the next stage (scalar_transport_rk.F90:343, 379)
      if (istage < nrk && C.halo.on) { OG_PROF("halo_exchange", s); OG_CHECK(halo_exchange(C, OUT, ntp, s)); }
      in_b = out_b;
      out_b = (out_b + 1) % 3;
      if (out_b == a) out_b = (out_b + 1) % 3;
    }
    launch_copy_cols(d.w_nonprog.p, d.n_nonprog, A, tr.q[in_b].p, (size_t)mza * ntp, s);
    tr.qcur = in_b;
    tr.q_valid = true;
  } else {
    OG_CHECK(ensure_plain(s));
    OG_CHECK(tp.plain_out[0].alloc(wz));
    OG_CHECK(tp.plain_out[1].alloc(wz));
    OG_CHECK(ensure_pass_scratch(C, 1, order));
    for (int n = 0; n < tr.n; ++n) {
      float* A = tr.p[n].p;
      float* T = tr.t[n].p;
      if (tp.have_turb && tr.sgsmix[n]) launch_diffusion(d, tp, CTView{A, 1, 0}, TView{T, 1, 0}, 1, s);
      float* bufs[2] = {tp.plain_out[0].p, tp.plain_out[1].p};
      const float* IN = A;
      int ob = 0;
      for (int istage = 1; istage <= nrk; ++istage) {
        const float dtr = dtlr[istage - 1];
        const bool last = istage == nrk;
        float* OUT = bufs[ob];
        if (last && pdm[n])
          launch_scp0_pd_update(d, tp, TView{A, 1, 0}, CTView{T, 1, 0}, tp.d_mode.p + tr.n + n, 1, dtr, s);
        const bool lim = last && modes[n] != MODE_PLAIN;
        passes_stage(C, CTView{IN, 1, 0}, CTView{A, 1, 0}, CTView{T, 1, 0}, TView{OUT, 1, 0}, 1, istage,
                     nrk, dtr, rhos_nrk, tp.d_mode.p + n, lim, s);
        { OG_PROF("implicit_solve", s); launch_implicit_solve(d, tp, nrk, istage, dtr, CTView{A, 1, 0}, TView{OUT, 1, 0}, 1, s); }
        IN = OUT;
        ob ^= 1;
      }
      // the final stage output becomes the tracer's device array
      launch_copy_cols(d.w_nonprog.p, d.n_nonprog, A, tp.plain_out[ob ^ 1].p, (size_t)mza, s);
      std::swap(tr.p[n], tp.plain_out[ob ^ 1]);
    }
  }

  if (diag) {
    unsigned long long red[6];
    OG_CUDA(cudaMemcpyAsync(red, tp.cfl_loc.p, sizeof(red), cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaStreamSynchronize(s));
    std::vector<int> prog(1);
    auto decode = [&](unsigned long long key, unsigned long long nan, float& v, int& k, int& iwg,
                      bool is_w) -> int {
      unsigned int order;
      v = 0.f; k = 1; iwg = 1;
      if (nan) { order = (unsigned int)(nan - 1); v = __builtin_nanf(""); }
      else if (key) {
        order = 0xffffffffu - (unsigned int)(key & 0xffffffffull);
        unsigned int bits = (unsigned int)(key >> 32);
        std::memcpy(&v, &bits, 4);
      } else return OLAMGPU_OK;
      int j = (int)(order / mza), kd = (int)(order % mza);
      int iw1 = C.hgrid.jtw_prog[j];  // 1-based
      k = kd + 1;
      iwg = C.hgrid.iwglobe ? C.hgrid.iwglobe[iw1 - 1] : iw1;
      if (is_w && C.hstate.wc && !nan) {
        float w;
        OG_CUDA(cudaMemcpy(&w, tp.wc.p + (size_t)(iw1 - 1) * mza + kd, 4, cudaMemcpyDeviceToHost));
        v = w;
      }
      return OLAMGPU_OK;
    };
    OG_CHECK(decode(red[0], red[1], diag->cfl_max, diag->cfl_k, diag->cfl_iwglobe, false));
    OG_CHECK(decode(red[2], red[3], diag->cflh_max, diag->cflh_k, diag->cflh_iwglobe, false));
    OG_CHECK(decode(red[4], red[5], diag->w_max, diag->w_k, diag->w_iwglobe, true));
  }
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL && !pipelined) OG_CHECK(tracers_to_host(s));
  OG_CUDA(cudaGetLastError());
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CUDA(cudaStreamSynchronize(s));
    OG_CHECK(check_device_status());
  }
  return OLAMGPU_OK;
}

}  // namespace olamgpu
