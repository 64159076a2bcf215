// window.cu -- a window of long steps with checkpoints, and the adjoint of its
// tracer transport with recomputation between the checkpoints.
//
// No counterpart in OLAM (the model has no adjoint).  The forward runs
// olamgpu_timestep's device sequence (omodel/timestep.f90:66-319: tend0, the
// acoustic steps, timeavg_momsc, scalar_transport_rk, set_scalars_bottom)
// nsteps times and keeps, at the start of every segment of nchk steps, the
// prognostic state the steps carry from one to the next: rho, press, thil,
// wc, wmc, the earth-Cartesian winds, vmc, vc and the damping's saved planes
// (and, when the limiter's adjoint needs them, the tracers).  The adjoint
// goes back segment by segment: it restores the segment's checkpoint, runs
// the segment's steps again -- only their dynamics when the transport is
// unlimited, whose adjoint does not depend on the tracers -- keeping each
// step's transport inputs (vmasc, wmasc, rho, rho_old: the winds and
// densities scalar_transport_rk reads), then applies the one-step adjoint
// (transport_adjoint.cu) to those steps in reverse order on the device.
// The adjoint of the tendencies is summed over the steps (the tendencies of
// the window are one field: the registered tendencies, or the surface
// emission, held for every step).  Afterwards the state after the window is
// put back, so the model continues from where the forward ended.
#include <algorithm>

#include "transport_kernels.cuh"

namespace olamgpu {

// the device buffers one long step hands to the next
static std::vector<std::pair<void*, size_t>> carried_state(Context& C, bool tracers) {
  Dyn& y = C.dy;
  Transport& tp = C.tp;
  std::vector<std::pair<void*, size_t>> v;
  auto add = [&](void* p, size_t b) { if (p && b) v.push_back({p, b}); };
  add(tp.rho.p, tp.rho.bytes());
  add(y.press.p, y.press.bytes());
  add(y.thil.p, y.thil.bytes());
  add(tp.wc.p, tp.wc.bytes());
  add(y.wmc.p, y.wmc.bytes());
  add(y.vxe.p, y.vxe.bytes());
  add(y.vye.p, y.vye.bytes());
  add(y.vze.p, y.vze.bytes());
  add(y.vmc.p, y.vmc.bytes());
  add(y.vc.p, y.vc.bytes());
  add(y.div2d.p, y.div2d.bytes());
  add(y.vort2d.p, y.vort2d.bytes());
  if (tracers) add(C.tr.q[C.tr.qcur].p, C.tr.q[C.tr.qcur].bytes());
  return v;
}

static size_t state_bytes(Context& C, bool tracers) {
  size_t b = 0;
  for (auto& f : carried_state(C, tracers)) b += (f.second + 255) & ~(size_t)255;
  return b;
}

static int copy_state(Context& C, DevBuf<char>& blob, bool tracers, bool save) {
  const size_t need = state_bytes(C, tracers);
  if (save && blob.n != need) OG_CHECK(blob.alloc(need));
  if (blob.n != need) { set_error("window: a checkpoint does not match the state"); return OLAMGPU_E_STATE; }
  size_t off = 0;
  for (auto& f : carried_state(C, tracers)) {
    char* b = blob.p + off;
    OG_CUDA(cudaMemcpyAsync(save ? b : f.first, save ? f.first : b, f.second, cudaMemcpyDeviceToDevice, C.stream));
    off += (f.second + 255) & ~(size_t)255;
  }
  return OLAMGPU_OK;
}

// the inputs scalar_transport_rk reads, per step: vmasc, wmasc, rho (r8), rho_old
static size_t step_bytes(const Context& C) {
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  return al(vz * 4) + al(wz * 4) + al(wz * 8) + al(wz * 4);
}

static int copy_step(Context& C, char* slot, bool save) {
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  Transport& tp = C.tp;
  const std::pair<void*, size_t> f[4] = {{tp.vmasc.p, vz * 4}, {tp.wmasc.p, wz * 4}, {tp.rho.p, wz * 8},
                                         {tp.rho_old.p, wz * 4}};
  size_t off = 0;
  for (const auto& x : f) {
    OG_CUDA(cudaMemcpyAsync(save ? slot + off : x.first, save ? x.first : slot + off, x.second,
                            cudaMemcpyDeviceToDevice, C.stream));
    off += (x.second + 255) & ~(size_t)255;
  }
  return OLAMGPU_OK;
}

__global__ void k_accumulate(float* __restrict__ acc, const float* __restrict__ x, size_t n, int first) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] = first ? x[i] : acc[i] + x[i];
}

void window_release() {
  Window& W = ctx().win;
  for (auto& b : W.chk) b.release();
  W.fin.release();
  W.seg.release();
  W.lsacc.release();
  W.ptab.release();
  W.planes.release();
  W = Window();
}

int window_forward(int nsteps, int nchk, unsigned flags) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (nsteps < 1 || nchk < 1) { set_error("window: nsteps and nchk must be at least 1"); return OLAMGPU_E_ARG; }
  if (C.coherence != OLAMGPU_RESIDENT) { set_error("window: set OLAMGPU_RESIDENT first"); return OLAMGPU_E_STATE; }
  if (!C.dy.ready || !C.have_state) { set_error("window: needs prog_wrtv_rk's set-up and the state arrays"); return OLAMGPU_E_STATE; }
  if (C.tr.n <= 0) { set_error("window: no scalars registered"); return OLAMGPU_E_STATE; }
  if (C.halo.on) { set_error("window: one domain only (no halo exchange)"); return OLAMGPU_E_UNSUPPORTED; }
  if (C.form != OLAMGPU_TRANSPORT_FUSED) { set_error("window: needs the tiled transport form"); return OLAMGPU_E_UNSUPPORTED; }
  OG_CHECK(adjoint_ready(C));
  Window& W = C.win;
  window_release();
  cudaStream_t s = C.stream;
  OG_CHECK(ensure_q(s));
  W.nsteps = nsteps;
  W.nchk = nchk;
  W.flags = flags & ~(unsigned)(OLAMGPU_TS_MAXMIN | OLAMGPU_TS_MASS);
  // the limiter's adjoint is taken at the forward state: checkpoints and
  // the recomputed segments keep the tracers too
  W.tracers = C.opts.iscal_monot == 2;
  const int nseg = (nsteps + nchk - 1) / nchk;
  W.chk.resize(nseg);
  W.chk_qcur.assign(nseg, 0);
  W.chk_div_first.assign(nseg, 0);
  W.chk_vort_first.assign(nseg, 0);
  for (int step = 0; step < nsteps; ++step) {
    if (step % nchk == 0) {
      const int g = step / nchk;
      // the first step allocates the dynamics' buffers: checkpoint 0 is
      // taken once they exist (tend0 does not read what it overwrites)
      if (step == 0 && (!C.dy.press.p || !C.dy.div2d.p)) OG_CHECK(dyn_tend0(nullptr));
      OG_CHECK(ensure_q(s));
      OG_CHECK(copy_state(C, W.chk[g], W.tracers, true));
      W.chk_qcur[g] = C.tr.qcur;
      W.chk_div_first[g] = C.dy.div_first;
      W.chk_vort_first[g] = C.dy.vort_first;
    }
    OG_CHECK(glue_timestep(W.flags, 0, nullptr));
  }
  OG_CHECK(ensure_q(s));
  OG_CHECK(copy_state(C, W.fin, true, true));
  W.fin_qcur = C.tr.qcur;
  W.fin_div_first = C.dy.div_first;
  W.fin_vort_first = C.dy.vort_first;
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  W.valid = true;
  return check_device_status();
}

int window_adjoint(float* const* lam, float* const* lam_sct) {
  Context& C = ctx();
  Window& W = C.win;
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!W.valid) { set_error("window adjoint: run olamgpu_window_forward first"); return OLAMGPU_E_STATE; }
  OG_CHECK(adjoint_ready(C));
  const int n = C.tr.n;
  if (!lam || !lam_sct) { set_error("lam and lam_sct must be arrays of num_scalar pointers"); return OLAMGPU_E_ARG; }
  for (int i = 0; i < n; ++i)
    if (!lam[i] || !lam_sct[i]) { set_error("a lam or lam_sct entry is NULL"); return OLAMGPU_E_ARG; }
  cudaStream_t s = C.stream;
  Transport& tp = C.tp;
  const DevGrid& d = C.g;
  const int ntp = C.tr.ntp, nrk = C.opts.nrk_scal;
  const size_t plane = (size_t)d.mza * d.mwa, qn = plane * ntp;
  const size_t pstride = (plane + 3) & ~(size_t)3;
  // per step: the transport inputs, and with the limiter the tracers at the step's start
  const size_t qbytes = (qn * sizeof(float) + 255) & ~(size_t)255;
  const size_t sb = step_bytes(C) + (W.tracers ? qbytes : 0);
  OG_CHECK(W.seg.alloc(sb * (size_t)W.nchk));
  OG_CHECK(W.lsacc.alloc(qn));
  OG_CHECK(W.planes.alloc(pstride * n));
  {
    std::vector<float*> h(n);
    for (int i = 0; i < n; ++i) h[i] = W.planes.p + (size_t)i * pstride;
    OG_CHECK(W.ptab.alloc(n));
    OG_CUDA(cudaMemcpyAsync(W.ptab.p, h.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
    OG_CUDA(cudaStreamSynchronize(s));   // h dies here
  }
  OG_CHECK(tp.adj_l[0].alloc(qn));
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(W.planes.p + (size_t)i * pstride, lam[i], plane * sizeof(float), cudaMemcpyHostToDevice, s));
  {
    OG_PROF("window_adjoint", s);
    launch_gather_q(tp.adj_l[0].p, (const float* const*)W.ptab.p, n, ntp, plane, s);
    const int nseg = (int)W.chk.size();
    bool first = true;
    for (int g = nseg - 1; g >= 0; --g) {
      const int s0 = g * W.nchk, s1 = std::min(W.nsteps, s0 + W.nchk);
      {
        // the segment's steps again from its checkpoint, keeping their transport inputs
        OG_PROF("window_recompute", s);
        C.tr.qcur = W.chk_qcur[g];
        C.tr.q_valid = true;
        OG_CHECK(copy_state(C, W.chk[g], W.tracers, false));
        C.dy.div_first = W.chk_div_first[g];
        C.dy.vort_first = W.chk_vort_first[g];
        for (int step = s0; step < s1; ++step) {
          char* slot = W.seg.p + sb * (size_t)(step - s0);
          if (W.tracers)
            OG_CUDA(cudaMemcpyAsync(slot + step_bytes(C), C.tr.q[C.tr.qcur].p, qn * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s));
          OG_CHECK(glue_run_sequence(C, W.flags, W.tracers));
          OG_CHECK(copy_step(C, slot, true));
        }
      }
      for (int step = s1 - 1; step >= s0; --step) {
        char* slot = W.seg.p + sb * (size_t)(step - s0);
        OG_CHECK(copy_step(C, slot, false));
        if (W.tracers)
          OG_CUDA(cudaMemcpyAsync(C.tr.q[C.tr.qcur].p, slot + step_bytes(C), qn * sizeof(float),
                                  cudaMemcpyDeviceToDevice, s));
        OG_CHECK(adjoint_core(C, nullptr));
        if (nrk & 1) std::swap(tp.adj_l[0], tp.adj_l[1]);   // the step's result back into adj_l[0]
        k_accumulate<<<cdiv(qn, 256), 256, 0, s>>>(W.lsacc.p, tp.adj_ls.p, qn, first ? 1 : 0);
        OG_LAUNCHED();
        first = false;
      }
    }
    // the model continues from the state after the window
    C.tr.qcur = W.fin_qcur;
    C.tr.q_valid = true;
    OG_CHECK(copy_state(C, W.fin, true, false));
    C.dy.div_first = W.fin_div_first;
    C.dy.vort_first = W.fin_vort_first;
    launch_scatter_q(tp.adj_l[0].p, W.ptab.p, n, ntp, plane, s);
  }
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam[i], W.planes.p + (size_t)i * pstride, plane * sizeof(float), cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));   // the planes are reused for the tendencies' adjoint
  launch_scatter_q(W.lsacc.p, W.ptab.p, n, ntp, plane, s);
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam_sct[i], W.planes.p + (size_t)i * pstride, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

}  // namespace olamgpu
