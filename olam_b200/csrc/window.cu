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
// A segment is reversed in parts of at most seg_steps steps when fewer
// steps' inputs fit (each part runs the segment again from its checkpoint).
// The adjoint of the tendencies is summed over the steps (the tendencies of
// the window are one field: the registered tendencies, or the surface
// emission, held for every step).  Afterwards the state after the window is
// put back, so the model continues from where the forward ended.
//
// Memory.  The checkpoints and the state after the window live on the
// device, or in page-locked host memory (olamgpu_window_memory).  With
// unlimited transport, when the device has no room for the adjoint's own
// buffers (or when asked), the adjoint is lean: the tracers are in the
// state after the window, so it borrows the three tracer rotation buffers
// and the tendencies' buffer for its four lam buffers, and frees the
// per-tracer device arrays (not read while the batched layout holds the
// tracers) for its records and the steps' inputs, allocating them again at
// the end.
#include <algorithm>

#include "transport_kernels.cuh"

namespace olamgpu {

// the device buffers one long step hands to the next
static std::vector<std::pair<void*, size_t>> carried_state(Context& C, bool tracers, bool qt = false) {
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
  // the lean adjoint lends the tendencies' buffer out: the state after the
  // window keeps it (it holds the last step's emission and diffusion)
  if (qt) add(C.tr.qt.p, C.tr.qt.bytes());
  return v;
}

static size_t state_bytes(Context& C, bool tracers, bool qt = false) {
  size_t b = 0;
  for (auto& f : carried_state(C, tracers, qt)) b += (f.second + 255) & ~(size_t)255;
  return b;
}

static char* blob_ptr(Context& C, const StateBlob& b) {
  return b.slot >= 0 ? C.winmem.pool[b.slot].p : b.dev.p;
}
static size_t blob_size(Context& C, const StateBlob& b) {
  return b.slot >= 0 ? C.winmem.pool[b.slot].n : b.dev.n;
}

// MemAvailable of /proc/meminfo in bytes (0 when it cannot be read)
static size_t host_available() {
  FILE* f = fopen("/proc/meminfo", "r");
  if (!f) return 0;
  char line[256];
  size_t kb = 0;
  while (fgets(line, sizeof line, f))
    if (sscanf(line, "MemAvailable: %zu kB", &kb) == 1) break;
  fclose(f);
  return kb * 1024;
}

// page-lock `add` more bytes of host memory only while they stay well inside
// what the host has free
static int host_guard(size_t add) {
  const size_t avail = host_available();
  if (avail && add > avail / 10 * 7) {
    set_error("window: " + std::to_string(add >> 20) + " MiB of page-locked host memory asked for, " +
              std::to_string(avail >> 20) + " MiB available");
    return OLAMGPU_E_NOMEM;
  }
  return OLAMGPU_OK;
}

// the storage of one saved state: pool entry `slot` on the host, else the device
static int blob_take(Context& C, StateBlob& b, int slot, size_t need) {
  WindowMem& M = C.winmem;
  if (!M.host) {
    b.slot = -1;
    return b.dev.alloc(need);
  }
  b.dev.release();
  if ((int)M.pool.size() <= slot) M.pool.resize(slot + 1);
  if (M.pool[slot].n != need) {
    const size_t had = M.pool[slot].n;
    M.pool[slot].release();
    OG_CHECK(host_guard(need > had ? need - had : 0));
    OG_CHECK(M.pool[slot].alloc(need));
  }
  b.slot = slot;
  return OLAMGPU_OK;
}

static int copy_state(Context& C, const StateBlob& blob, bool tracers, bool qt, bool save) {
  const size_t need = state_bytes(C, tracers, qt);
  char* base = blob_ptr(C, blob);
  if (!base || blob_size(C, blob) != need) {
    set_error("window: a checkpoint does not match the state");
    return OLAMGPU_E_STATE;
  }
  size_t off = 0;
  for (auto& f : carried_state(C, tracers, qt)) {
    char* b = base + off;
    OG_CUDA(cudaMemcpyAsync(save ? b : f.first, save ? f.first : b, f.second, cudaMemcpyDefault, C.stream));
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
  for (auto& b : W.chk) b.dev.release();
  W.fin.dev.release();
  W.seg.release();
  W.lsacc.release();
  W.ptab.release();
  W.planes.release();
  W = Window();
}

void window_memory_release() {
  WindowMem& M = ctx().winmem;
  for (auto& h : M.pool) h.release();
  M = WindowMem();
}

int window_memory(int flags, int segment_steps, int nsteps, int nchk) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (segment_steps < 0 || nsteps < 0 || nchk < 0) {
    set_error("window memory: segment_steps, nsteps and nchk must not be negative");
    return OLAMGPU_E_ARG;
  }
  // a window taken before keeps its states where they were: it is dropped
  window_release();
  WindowMem& M = C.winmem;
  if (!(flags & OLAMGPU_WIN_HOST)) {
    for (auto& h : M.pool) h.release();
    M.pool.clear();
  }
  M.host = (flags & OLAMGPU_WIN_HOST) != 0;
  M.lean_always = (flags & OLAMGPU_WIN_LEAN) != 0;
  M.seg_steps = segment_steps;
  if (!M.host || nsteps == 0 || nchk == 0) return OLAMGPU_OK;
  // page-lock now the states a window of nsteps with a checkpoint every nchk will keep
  if (!C.dy.press.p || !C.dy.div2d.p || C.tr.n <= 0) {
    set_error("window memory: the state's device buffers exist after the first long step; reserve after it");
    return OLAMGPU_E_STATE;
  }
  OG_CHECK(ensure_q(C.stream));
  const bool tracers = C.opts.iscal_monot == 2;
  const int nseg = (nsteps + nchk - 1) / nchk;
  std::vector<size_t> need(nseg + 1, state_bytes(C, tracers));
  need[0] = state_bytes(C, true, !tracers);
  size_t add = 0, had = 0;
  for (int i = 0; i <= nseg; ++i) add += need[i];
  for (size_t i = 0; i < M.pool.size(); ++i) had += M.pool[i].n;
  for (size_t i = nseg + 1; i < M.pool.size(); ++i) M.pool[i].release();
  M.pool.resize(nseg + 1);
  for (int i = 0; i <= nseg; ++i)
    if (M.pool[i].n != need[i]) M.pool[i].release();
  OG_CHECK(host_guard(add > had ? add - had : 0));
  for (int i = 0; i <= nseg; ++i) OG_CHECK(M.pool[i].alloc(need[i]));
  return OLAMGPU_OK;
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
  W.lean_ok = !W.tracers;
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
      OG_CHECK(blob_take(C, W.chk[g], g + 1, state_bytes(C, W.tracers)));
      OG_CHECK(copy_state(C, W.chk[g], W.tracers, false, true));
      W.chk_qcur[g] = C.tr.qcur;
      W.chk_div_first[g] = C.dy.div_first;
      W.chk_vort_first[g] = C.dy.vort_first;
    }
    OG_CHECK(glue_timestep(W.flags, 0, nullptr));
  }
  OG_CHECK(ensure_q(s));
  OG_CHECK(blob_take(C, W.fin, 0, state_bytes(C, true, W.lean_ok)));
  OG_CHECK(copy_state(C, W.fin, true, W.lean_ok, true));
  W.fin_qcur = C.tr.qcur;
  W.fin_div_first = C.dy.div_first;
  W.fin_vort_first = C.dy.vort_first;
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  W.valid = true;
  return check_device_status();
}

int window_rewind() {
  Context& C = ctx();
  Window& W = C.win;
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!W.valid || W.chk.empty()) { set_error("window rewind: no window has run"); return OLAMGPU_E_STATE; }
  // an unlimited window's checkpoints hold no tracers: those on the device
  // stay until the caller sends the new ones
  if (W.tracers) {
    C.tr.qcur = W.chk_qcur[0];
    C.tr.q_valid = true;
  }
  OG_CHECK(copy_state(C, W.chk[0], W.tracers, false, false));
  C.dy.div_first = W.chk_div_first[0];
  C.dy.vort_first = W.chk_vort_first[0];
  OG_CUDA(cudaStreamSynchronize(C.stream));
  return check_device_status();
}

// the steps [a, b) of checkpoint g's segment again from the checkpoint,
// keeping the transport inputs (and with the limiter the tracers at the
// start) of each into its slot of the segment buffer
static int recompute(Context& C, int g, int a, int b, size_t sb) {
  Window& W = C.win;
  cudaStream_t s = C.stream;
  OG_PROF("window_recompute", s);
  const size_t qn = (size_t)C.g.mza * C.g.mwa * C.tr.ntp;
  C.tr.qcur = W.chk_qcur[g];
  // in the lean form the tracer buffers hold the adjoint: tend0 must not
  // clear the tendencies' buffer, which holds the tendencies' adjoint
  C.tr.q_valid = !W.lean;
  OG_CHECK(copy_state(C, W.chk[g], W.tracers, false, false));
  C.dy.div_first = W.chk_div_first[g];
  C.dy.vort_first = W.chk_vort_first[g];
  for (int step = g * W.nchk; step < b; ++step) {
    char* slot = step >= a ? W.seg.p + sb * (size_t)(step - a) : nullptr;
    if (slot && W.tracers)
      OG_CUDA(cudaMemcpyAsync(slot + step_bytes(C), C.tr.q[C.tr.qcur].p, qn * sizeof(float),
                              cudaMemcpyDeviceToDevice, s));
    OG_CHECK(glue_run_sequence(C, W.flags, W.tracers));
    if (slot) OG_CHECK(copy_step(C, slot, true));
  }
  return OLAMGPU_OK;
}

// the one-step adjoint of the steps b-1 down to a, from their saved inputs
static int reverse(Context& C, int a, int b, size_t sb, bool& first) {
  Window& W = C.win;
  Transport& tp = C.tp;
  cudaStream_t s = C.stream;
  const size_t qn = (size_t)C.g.mza * C.g.mwa * C.tr.ntp;
  for (int step = b - 1; step >= a; --step) {
    char* slot = W.seg.p + sb * (size_t)(step - a);
    OG_CHECK(copy_step(C, slot, false));
    if (W.tracers)
      OG_CUDA(cudaMemcpyAsync(C.tr.q[C.tr.qcur].p, slot + step_bytes(C), qn * sizeof(float),
                              cudaMemcpyDeviceToDevice, s));
    // the lean form sums the tendencies' adjoint in adj_ls itself
    OG_CHECK(adjoint_core(C, nullptr, W.lean && !first));
    if (C.opts.nrk_scal & 1) std::swap(tp.adj_l[0], tp.adj_l[1]);   // the step's result back into adj_l[0]
    if (!W.lean) {
      k_accumulate<<<cdiv(qn, 256), 256, 0, s>>>(W.lsacc.p, tp.adj_ls.p, qn, first ? 1 : 0);
      OG_LAUNCHED();
    }
    first = false;
  }
  return OLAMGPU_OK;
}

static int planes_table(Window& W, int n, size_t pstride, cudaStream_t s) {
  std::vector<float*> h(n);
  for (int i = 0; i < n; ++i) h[i] = W.planes.p + (size_t)i * pstride;
  OG_CHECK(W.ptab.alloc(n));
  OG_CUDA(cudaMemcpyAsync(W.ptab.p, h.data(), n * sizeof(float*), cudaMemcpyHostToDevice, s));
  OG_CUDA(cudaStreamSynchronize(s));   // h dies here
  return OLAMGPU_OK;
}

// The lean adjoint's borrowed and freed memory, given back however the call
// ends: the buffers it allocated are freed, the state after the window is
// put back (on an error too, so the model state stays that of the window's
// end), the borrowed views are dropped and the per-tracer device arrays are
// allocated again (zero: the batched layout holds the tracers, and the
// tendencies were cleared by the last step's tend0).  Recorded long steps
// cleared the old per-tracer arrays: they are recorded again.
struct LeanScope {
  Context& C;
  bool on = false;
  bool fin_restored = false;
  explicit LeanScope(Context& c) : C(c) {}
  int finish() {
    if (!on) return OLAMGPU_OK;
    on = false;
    Window& W = C.win;
    Transport& tp = C.tp;
    Tracers& tr = C.tr;
    cudaStream_t s = C.stream;
    W.seg.release();
    W.planes.release();
    tp.adj_trec.release();
    int rc = OLAMGPU_OK;
    if (!fin_restored) {
      tr.qcur = W.fin_qcur;
      rc = copy_state(C, W.fin, true, true, false);
      C.dy.div_first = W.fin_div_first;
      C.dy.vort_first = W.fin_vort_first;
    }
    tr.q_valid = true;
    for (int b = 0; b < 2; ++b) tp.adj_l[b].release();
    tp.adj_l0.release();
    tp.adj_ls.release();
    const size_t plane = (size_t)C.g.mza * C.g.mwa;
    for (int n = 0; n < tr.n; ++n) {
      int r = tr.p[n].alloc(plane);
      if (r == OLAMGPU_OK) r = tr.t[n].alloc(plane);
      if (r == OLAMGPU_OK && cudaMemsetAsync(tr.p[n].p, 0, plane * sizeof(float), s) != cudaSuccess) r = OLAMGPU_E_CUDA;
      if (r == OLAMGPU_OK && cudaMemsetAsync(tr.t[n].p, 0, plane * sizeof(float), s) != cudaSuccess) r = OLAMGPU_E_CUDA;
      if (r != OLAMGPU_OK && rc == OLAMGPU_OK) rc = r;
    }
    const int re = emission_repoint(C, s);
    if (rc == OLAMGPU_OK) rc = re;
    glue_drop_graphs();
    return rc;
  }
  ~LeanScope() { finish(); }
};

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
  Tracers& tr = C.tr;
  const DevGrid& d = C.g;
  const int ntp = tr.ntp;
  const size_t plane = (size_t)d.mza * d.mwa, qn = plane * ntp;
  const size_t pstride = (plane + 3) & ~(size_t)3;
  // per step: the transport inputs, and with the limiter the tracers at the step's start
  const size_t qbytes = (qn * sizeof(float) + 255) & ~(size_t)255;
  const size_t sb = step_bytes(C) + (W.tracers ? qbytes : 0);
  const int part = C.winmem.seg_steps > 0 ? std::min(C.winmem.seg_steps, W.nchk) : W.nchk;
  // lean when the device has no room for the adjoint's own buffers: four
  // lam arrays, the tendencies' sum, the transposed records, the host
  // transfer planes and the steps' inputs (with 2 GiB to spare)
  W.lean = W.lean_ok && C.winmem.lean_always;
  if (W.lean_ok && !W.lean) {
    size_t fr = 0, tot = 0;
    OG_CUDA(cudaMemGetInfo(&fr, &tot));
    auto missing = [](const DevBuf<float>& b, size_t n) { return b.n == n ? (size_t)0 : n * sizeof(float); };
    const size_t need = missing(tp.adj_l[0], qn) + missing(tp.adj_l[1], qn) + missing(tp.adj_ls, qn) +
                        (tp.adj_l0.n >= qn ? 0 : qn * sizeof(float)) + qn * sizeof(float) +
                        missing(tp.adj_trec, plane * 32 /* floats a cell */) + pstride * n * sizeof(float) + sb * (size_t)part +
                        ((size_t)2 << 30);
    W.lean = need > fr;
  }
  LeanScope lean(C);
  if (W.lean) {
    // the tracers are in the state after the window: their buffers hold the
    // four lam arrays; the per-tracer arrays' memory goes to the records and
    // the steps' inputs (a one-step adjoint's own buffers are freed first)
    for (int b = 0; b < 3; ++b)
      if (tr.q[b].n != qn || tr.qt.n != qn) { set_error("window adjoint: the tracer buffers are missing"); return OLAMGPU_E_STATE; }
    for (int b = 0; b < 2; ++b) tp.adj_l[b].release();
    tp.adj_l0.release();
    tp.adj_ls.release();
    tp.adj_planes.release();
    tp.adj_trec.release();
    OG_CUDA(cudaStreamSynchronize(s));
    lean.on = true;
    for (int i = 0; i < n; ++i) { tr.p[i].release(); tr.t[i].release(); }
    tp.adj_l[0].borrow(tr.q[0].p, qn);
    tp.adj_l[1].borrow(tr.q[1].p, qn);
    tp.adj_l0.borrow(tr.q[2].p, qn);
    tp.adj_ls.borrow(tr.qt.p, qn);
  } else {
    OG_CHECK(W.lsacc.alloc(qn));
    OG_CHECK(tp.adj_l[0].alloc(qn));
  }
  OG_CHECK(W.planes.alloc(pstride * n));
  OG_CHECK(planes_table(W, n, pstride, s));
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(W.planes.p + (size_t)i * pstride, lam[i], plane * sizeof(float), cudaMemcpyHostToDevice, s));
  {
    OG_PROF("window_adjoint", s);
    launch_gather_q(tp.adj_l[0].p, (const float* const*)W.ptab.p, n, ntp, plane, s);
    if (W.lean) {
      OG_CUDA(cudaStreamSynchronize(s));   // the planes' memory goes to the steps' inputs
      W.planes.release();
    }
    OG_CHECK(W.seg.alloc(sb * (size_t)part));
    const int nseg = (int)W.chk.size();
    bool first = true;
    for (int g = nseg - 1; g >= 0; --g) {
      const int s0 = g * W.nchk, s1 = std::min(W.nsteps, s0 + W.nchk);
      // the segment's parts from the last: [a, b) with a = s0 + a multiple of part
      for (int b = s1; b > s0;) {
        const int a = s0 + (b - 1 - s0) / part * part;
        OG_CHECK(recompute(C, g, a, b, sb));
        OG_CHECK(reverse(C, a, b, sb, first));
        b = a;
      }
    }
    if (!W.lean) {
      // the model continues from the state after the window (with the
      // tendencies, which the dynamics run again cleared in tend0)
      tr.qcur = W.fin_qcur;
      tr.q_valid = true;
      OG_CHECK(copy_state(C, W.fin, true, W.lean_ok, false));
      C.dy.div_first = W.fin_div_first;
      C.dy.vort_first = W.fin_vort_first;
    } else {
      W.seg.release();
      tp.adj_trec.release();
      OG_CHECK(W.planes.alloc(pstride * n));
      OG_CHECK(planes_table(W, n, pstride, s));
    }
    launch_scatter_q(tp.adj_l[0].p, W.ptab.p, n, ntp, plane, s);
  }
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam[i], W.planes.p + (size_t)i * pstride, plane * sizeof(float), cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));   // the planes are reused for the tendencies' adjoint
  launch_scatter_q(W.lean ? tp.adj_ls.p : W.lsacc.p, W.ptab.p, n, ntp, plane, s);
  for (int i = 0; i < n; ++i)
    OG_CUDA(cudaMemcpyAsync(lam_sct[i], W.planes.p + (size_t)i * pstride, plane * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaGetLastError());
  OG_CUDA(cudaStreamSynchronize(s));
  OG_CHECK(lean.finish());
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

}  // namespace olamgpu
