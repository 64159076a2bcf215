// api.cu -- the extern "C" entry points declared in include/olamgpu.h.
//
// One library context per process (OLAM calls from its master thread,
// outside OpenMP regions, omodel/timestep.f90:205,254); every call returns a
// status code and never falls back to the CPU.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "transport_kernels.cuh"

namespace olamgpu {

unsigned long long g_launches = 0;

int check_device_status() {
  Context& C = ctx();
  if (!C.status.p) return OLAMGPU_OK;
  int h[4];
  OG_CUDA(cudaMemcpyAsync(h, C.status.p, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
  OG_CUDA(cudaStreamSynchronize(C.stream));
  if (h[0] == 130 || h[0] == 131) {
    // the tiled stage kernel's level copies did not complete within its poll limit
    set_error(std::string("a level copy of the tiled transport kernel timed out (tile ") + std::to_string(h[1]) +
              ", block " + std::to_string(h[2]) + ", level " + std::to_string(h[3]) +
              (h[0] == 131 ? "; copies were still in flight at exit)" : ")"));
    return OLAMGPU_E_NUMERIC;
  }
  if (h[0]) {
    set_error("a device bounds check failed (code " + std::to_string(h[0]) + ", value " + std::to_string(h[1]) +
              ", block " + std::to_string(h[2]) + ", thread " + std::to_string(h[3]) + ")");
    return OLAMGPU_E_NUMERIC;
  }
  return OLAMGPU_OK;
}

#ifdef OLAMGPU_DEBUG_SYNC
void debug_sync(const char* file, int line) {
  ++g_launches;
  static bool reported = false;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess && !reported) {
    reported = true;
    std::fprintf(stderr, "olamgpu: launch at %s:%d failed: %s\n", file, line, cudaGetErrorString(e));
  }
}
#endif

// ---- per-kernel event timing ----------------------------------------------
struct ProfRec { std::string name; cudaEvent_t a, b; };
static bool g_prof_on = false;
static std::vector<ProfRec> g_prof_pending;
static std::vector<cudaEvent_t> g_prof_pool;
static std::vector<std::string> g_prof_names;
static std::vector<double> g_prof_ms;
static std::vector<unsigned long long> g_prof_cnt;
// open scopes, innermost last (scopes nest: a step's scope holds its kernels')
static std::vector<std::pair<std::string, cudaEvent_t>> g_prof_open;

static cudaEvent_t prof_event() {
  if (!g_prof_pool.empty()) { cudaEvent_t e = g_prof_pool.back(); g_prof_pool.pop_back(); return e; }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

static bool g_prof_suspended = false;
void prof_suspend(bool on) { g_prof_suspended = on; }

void prof_begin(const char* name, cudaStream_t s) {
  if (!g_prof_on || g_prof_suspended) return;
  cudaEvent_t a = prof_event();
  cudaEventRecord(a, s);
  g_prof_open.push_back({name, a});
}

void prof_end(cudaStream_t s) {
  if (!g_prof_on || g_prof_suspended || g_prof_open.empty()) return;
  cudaEvent_t b = prof_event();
  cudaEventRecord(b, s);
  g_prof_pending.push_back({g_prof_open.back().first, g_prof_open.back().second, b});
  g_prof_open.pop_back();
}

static void prof_resolve() {
  for (auto& r : g_prof_pending) {
    float ms = 0.f;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    size_t i = 0;
    while (i < g_prof_names.size() && g_prof_names[i] != r.name) ++i;
    if (i == g_prof_names.size()) { g_prof_names.push_back(r.name); g_prof_ms.push_back(0); g_prof_cnt.push_back(0); }
    g_prof_ms[i] += ms;
    g_prof_cnt[i] += 1;
    g_prof_pool.push_back(r.a);
    g_prof_pool.push_back(r.b);
  }
  g_prof_pending.clear();
}

static std::string g_err;
void set_error(const std::string& m) { g_err = m; }
const std::string& last_error() { return g_err; }

Context& ctx() {
  static Context c;
  return c;
}

static int require_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count 0"));
    return OLAMGPU_E_NODEVICE;
  }
  int dev = 0;
  OG_CUDA(cudaGetDevice(&dev));
  cudaDeviceProp p;
  OG_CUDA(cudaGetDeviceProperties(&p, dev));
  if (p.major < 10) {
    set_error(std::string("device ") + p.name + " is not sm_100 class; this library is built for sm_100a");
    return OLAMGPU_E_NODEVICE;
  }
  ctx().device = dev;
  return OLAMGPU_OK;
}

// page-lock OLAM's state arrays in place so that the per-call copies run at
// full speed and asynchronously; a failure only costs transfer speed
static std::vector<void*> g_pinned_state;

static void register_state_arrays(Context& C) {
  if (!C.have_state) return;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  const olamgpu_state& h = C.hstate;
  const std::pair<void*, size_t> arr[] = {
      {h.rho, wz * 8}, {h.press, wz * 8}, {h.thil, wz * 4}, {h.wc, wz * 4}, {h.wmc, wz * 4}, {h.vxe, wz * 4},
      {h.vye, wz * 4}, {h.vze, wz * 4}, {h.vmc, vz * 4}, {h.vc, vz * 4}, {h.vmasc, vz * 4}, {h.wmasc, wz * 4},
      {h.alpha_press, wz * 4}, {h.pwfac, wz * 4}, {h.pvfac, vz * 4}, {h.thilt, wz * 4}, {h.vmxet, wz * 4},
      {h.vmyet, wz * 4}, {h.vmzet, wz * 4}, {h.vmt, vz * 4}};
  for (const auto& a : arr) {
    if (!a.first) continue;
    if (cudaHostRegister(a.first, a.second, cudaHostRegisterDefault) == cudaSuccess) g_pinned_state.push_back(a.first);
    cudaGetLastError();
  }
}

static void unregister_state_arrays() {
  for (void* p : g_pinned_state) cudaHostUnregister(p);
  g_pinned_state.clear();
  cudaGetLastError();
}

static void release_all() {
  unregister_state_arrays();
  window_release();
  window_memory_release();
  pd_adjoint_release();
  Context& C = ctx();
  DevGrid& d = C.g;
  DevBuf<int>* ib[] = {&d.jtw_prog, &d.jtv_wadj, &d.jtv_prog, &d.jtw_wadj, &d.jtm_prog, &d.npoly,
                       &d.w_nb, &d.w_ev, &d.w_im, &d.v_iw, &d.v_im, &d.m_iv, &d.m_iw, &d.m_im,
                       &d.lpw, &d.lpv, &d.lpm, &d.iwglobe, &d.w_nonprog, &d.colrec,
                       &d.tile_hdr, &d.tile_u, &d.tile_tc, &d.tile_rev, &d.tile_band_lev, &d.tile_pair};
  for (auto* b : ib) b->release();
  DevBuf<float>* fb[] = {&d.w_dirv, &d.gxc, &d.gyc, &d.xy_h, &d.xy_hu, &d.dxps, &d.dyps, &d.xx0_v,
                         &d.xy0_v, &d.yy0_v, &d.xx0_vu, &d.xy0_vu, &d.yy0_vu, &d.a_w, &d.a_wu,
                         &d.volti, &d.ew_b, &d.ew_u, &d.tile_a, &d.tile_band};
  for (auto* b : fb) b->release();
  d.ew_order = 0;
  {
    auto& a = d.adj_tiles;
    a.hdr.release(); a.u.release(); a.tc.release(); a.rev.release();
    a.T = a.ntiles = a.nu_max = a.order = 0;
  }
  d.tile_T = d.ntiles = d.tile_nu_max = d.tile_order = 0;
  d.tile_paired = false;
  d.tile_pairk = false;
  d.tile_G = 64;
  d.tile_KS = 1;
  d.tile_ord = 0;
  Tracers& tr = C.tr;
  for (size_t i = 0; i < tr.p.size(); ++i) {
    tr.p[i].release();
    tr.t[i].release();
    if (i < tr.pinned.size() && tr.pinned[i]) {
      cudaHostUnregister(tr.h_p[i]);
      cudaHostUnregister(tr.h_t[i]);
    }
  }
  for (auto& b : tr.q) b.release();
  tr.qt.release();
  tr.d_pdef.release();
  tr = Tracers();
  Transport& tp = C.tp;
  DevBuf<float>* tb[] = {&tp.vmasc, &tp.wmasc, &tp.rho_old, &tp.wc, &tp.rhos, &tp.ff, &tp.imp_b,
                         &tp.cfl_red, &tp.gx, &tp.upv, &tp.hiv, &tp.sfv, &tp.scale, &tp.upw,
                         &tp.plain_out[0], &tp.plain_out[1], &tp.akhodx, &tp.emis,
                         &tp.adj_l[0], &tp.adj_l[1], &tp.adj_l0, &tp.adj_ls, &tp.wrec, &tp.adj_trec, &tp.prec,
                         &tp.adj_planes};
  for (auto* b : tb) b->release();
  tp.rho.release();
  tp.imp_list.release();
  tp.imp_count.release();
  tp.cfl_loc.release();
  tp.d_mode.release();
  tp.h_mode.clear();
  tp.khtopv.release();
  tp.adj_ptab.release();
  tp.adj_ptab2.release();
  tp.have_turb = false;
  tp.have_emis = false;
  tp.autotune = true;
  tp.tuned_ntp = -1;
  tp.tune_log.clear();
  transport_release_pipeline();
  halo_release();
  glue_release();
  dyn_release();
  C.status.release();
}

}  // namespace olamgpu

using namespace olamgpu;

extern "C" {

const char* olamgpu_strerror(int status) {
  static std::string msg;
  const char* base = "unknown status";
  switch (status) {
    case OLAMGPU_OK: return "ok";
    case OLAMGPU_E_ARG: base = "invalid argument"; break;
    case OLAMGPU_E_STATE: base = "call out of order"; break;
    case OLAMGPU_E_UNSUPPORTED: base = "unsupported option"; break;
    case OLAMGPU_E_CUDA: base = "CUDA error"; break;
    case OLAMGPU_E_NOMEM: base = "device out of memory"; break;
    case OLAMGPU_E_NODEVICE: base = "no usable GPU"; break;
    case OLAMGPU_E_NUMERIC: base = "device status reported a failure"; break;
  }
  msg = std::string(base) + (last_error().empty() ? "" : ": " + last_error());
  return msg.c_str();
}

int olamgpu_init(const olamgpu_grid* grid, const olamgpu_opts* opts, const olamgpu_state* state) {
  if (!grid || !opts) { set_error("grid or opts is NULL"); return OLAMGPU_E_ARG; }
  Context& C = ctx();
  if (C.initialised) { set_error("olamgpu_init called twice without olamgpu_finalize"); return OLAMGPU_E_STATE; }
  if (opts->mdomain != 0) { set_error("only the global domain (mdomain = 0) is supported"); return OLAMGPU_E_UNSUPPORTED; }
  if (grid->mza > 512) { set_error("mza > 512 is not supported"); return OLAMGPU_E_UNSUPPORTED; }
  OG_CHECK(require_device());
  if (!C.stream) OG_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
  int rc = upload_grid(grid, C.g, C.stream);
  if (rc != OLAMGPU_OK) { release_all(); return rc; }
  C.hgrid = *grid;
  C.opts = *opts;
  C.coherence = OLAMGPU_SYNC_EACH_CALL;
  C.form = OLAMGPU_TRANSPORT_FUSED;
  C.tp.flat = true;
  for (int i = 1; i < grid->mwa; ++i) if (grid->lpw[i] != 2) C.tp.flat = false;
  for (int i = 1; i < grid->mva; ++i) if (grid->lpv[i] != 2) C.tp.flat = false;
  int order = opts->scal_horiz_adv_order;
  if (order == 2 || order == 3) {
    rc = build_fused_weights(grid, C.g, order, C.stream);
    if (rc != OLAMGPU_OK) { release_all(); return rc; }
    rc = build_tiles(grid, C.g, order, C.stream);
    if (rc != OLAMGPU_OK) { release_all(); return rc; }
  }
  if (state) { C.hstate = *state; C.have_state = true; } else C.have_state = false;
  register_state_arrays(C);
  // prog_wrtv_rk needs the dynamics state and the M-point tables; without
  // them only scalar_transport_rk is available
  if (state && state->thil && state->vmc && state->press && grid->itab_m_iv && grid->jtm_prog) {
    rc = dyn_setup(grid, opts, C.stream);
    if (rc != OLAMGPU_OK) { release_all(); return rc; }
  }
  rc = C.status.alloc(16);
  if (rc != OLAMGPU_OK) { release_all(); return rc; }
  cudaMemsetAsync(C.status.p, 0, 16 * sizeof(int), C.stream);
  OG_CUDA(cudaStreamSynchronize(C.stream));
  C.initialised = true;
  return OLAMGPU_OK;
}

int olamgpu_register_scalars(int num_scalar, float* const* var_p, float* const* var_t, const int* pdef,
                             const int* do_sgsmix) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (num_scalar < 0 || (num_scalar > 0 && (!var_p || !var_t))) { set_error("bad scalar table"); return OLAMGPU_E_ARG; }
  for (int n = 0; n < num_scalar; ++n)
    if (!var_p[n] || !var_t[n]) { set_error("NULL var_p/var_t for scalar " + std::to_string(n + 1)); return OLAMGPU_E_ARG; }
  glue_drop_graphs();
  window_release();
  C.tp.have_emis = false;   // the emission table is per registered scalar
  Tracers& tr = C.tr;
  // drop a previous registration
  for (size_t i = 0; i < tr.p.size(); ++i) {
    tr.p[i].release(); tr.t[i].release();
    if (i < tr.pinned.size() && tr.pinned[i]) { cudaHostUnregister(tr.h_p[i]); cudaHostUnregister(tr.h_t[i]); }
  }
  for (auto& b : tr.q) b.release();
  tr.qt.release();
  tr = Tracers();
  tr.n = num_scalar;
  tr.ntp = ((num_scalar + 3) / 4) * 4;
  const size_t plane = (size_t)C.g.mza * C.g.mwa;
  tr.h_p.assign(var_p, var_p + num_scalar);
  tr.h_t.assign(var_t, var_t + num_scalar);
  tr.pdef.resize(num_scalar);
  tr.sgsmix.resize(num_scalar);
  tr.pinned.assign(num_scalar, 0);
  tr.p.resize(num_scalar);
  tr.t.resize(num_scalar);
  for (int n = 0; n < num_scalar; ++n) {
    tr.pdef[n] = pdef ? (pdef[n] != 0) : 0;
    tr.sgsmix[n] = do_sgsmix ? (do_sgsmix[n] != 0) : 0;
    OG_CHECK(tr.p[n].alloc(plane));
    OG_CHECK(tr.t[n].alloc(plane));
    // page-lock OLAM's arrays in place; failure only costs transfer speed
    if (cudaHostRegister(tr.h_p[n], plane * sizeof(float), cudaHostRegisterDefault) == cudaSuccess) {
      if (cudaHostRegister(tr.h_t[n], plane * sizeof(float), cudaHostRegisterDefault) == cudaSuccess)
        tr.pinned[n] = 1;
      else
        cudaHostUnregister(tr.h_p[n]);
    }
    cudaGetLastError();
  }
  // initial device copy
  OG_CHECK(tracers_to_device(C.stream));
  OG_CUDA(cudaStreamSynchronize(C.stream));
  return OLAMGPU_OK;
}

int olamgpu_set_turb(const float* akhodx, const int* khtopv) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  glue_drop_graphs();
  if (!akhodx || !khtopv) { C.tp.have_turb = false; return OLAMGPU_OK; }
  OG_CHECK(upload(C.tp.akhodx, akhodx, (size_t)C.g.mza * C.g.mva, C.stream));
  OG_CHECK(upload(C.tp.khtopv, khtopv, (size_t)C.g.mva, C.stream));
  OG_CUDA(cudaStreamSynchronize(C.stream));
  C.tp.have_turb = true;
  return OLAMGPU_OK;
}

int olamgpu_set_eddy(const olamgpu_eddy* eddy) {
  glue_drop_graphs();
  return dyn_eddy_set(eddy);
}

int olamgpu_comp_horiz_k(void) { return dyn_comp_horiz_k(); }

int olamgpu_finalize(void) {
  Context& C = ctx();
  if (C.stream) cudaStreamSynchronize(C.stream);
  release_all();
  noalloc_forget();
  C.initialised = false;
  C.have_state = false;
  if (C.stream) { cudaStreamDestroy(C.stream); C.stream = nullptr; }
  return OLAMGPU_OK;
}

int olamgpu_set_coherence(int mode) {
  if (mode != OLAMGPU_SYNC_EACH_CALL && mode != OLAMGPU_RESIDENT) { set_error("unknown coherence mode"); return OLAMGPU_E_ARG; }
  if (ctx().coherence != mode) glue_drop_graphs();
  ctx().coherence = mode;
  return OLAMGPU_OK;
}

int olamgpu_set_transport_form(int form) {
  if (form != OLAMGPU_TRANSPORT_FUSED && form != OLAMGPU_TRANSPORT_PLAIN && form != OLAMGPU_TRANSPORT_FUSED_COLUMN) {
    set_error("unknown transport form");
    return OLAMGPU_E_ARG;
  }
  Context& C = ctx();
  if (C.initialised && (C.form == OLAMGPU_TRANSPORT_PLAIN) != (form == OLAMGPU_TRANSPORT_PLAIN)) {
    // keep the newest tracer values in the per-tracer mirrors across a switch
    OG_CHECK(ensure_plain(C.stream));
  }
  if (C.form != form) glue_drop_graphs();
  C.form = form;
  return OLAMGPU_OK;
}

int olamgpu_sync_to_device(unsigned fieldmask) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  cudaStream_t s = C.stream;
  const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
  if (fieldmask & (OLAMGPU_F_SCALARS | OLAMGPU_F_SCALAR_TEND)) {
    OG_CHECK(ensure_plain(s));
    for (int n = 0; n < C.tr.n; ++n) {
      if (fieldmask & OLAMGPU_F_SCALARS)
        OG_CUDA(cudaMemcpyAsync(C.tr.p[n].p, C.tr.h_p[n], wz * 4, cudaMemcpyHostToDevice, s));
      if (fieldmask & OLAMGPU_F_SCALAR_TEND)
        OG_CUDA(cudaMemcpyAsync(C.tr.t[n].p, C.tr.h_t[n], wz * 4, cudaMemcpyHostToDevice, s));
    }
  }
  if (C.have_state) {
    if (C.dy.ready) {
      OG_CHECK(dyn_state_to_device(fieldmask, s));
      if (fieldmask & OLAMGPU_F_EDDY) OG_CHECK(dyn_eddy_to_device(s));
    } else {
      if ((fieldmask & OLAMGPU_F_VMASC) && C.hstate.vmasc) OG_CHECK(upload(C.tp.vmasc, C.hstate.vmasc, vz, s));
      if ((fieldmask & OLAMGPU_F_WMASC) && C.hstate.wmasc) OG_CHECK(upload(C.tp.wmasc, C.hstate.wmasc, wz, s));
      if ((fieldmask & OLAMGPU_F_RHO) && C.hstate.rho) OG_CHECK(upload(C.tp.rho, C.hstate.rho, wz, s));
      if ((fieldmask & OLAMGPU_F_WC) && C.hstate.wc) OG_CHECK(upload(C.tp.wc, C.hstate.wc, wz, s));
    }
  }
  OG_CUDA(cudaStreamSynchronize(s));
  return OLAMGPU_OK;
}

int olamgpu_sync_to_host(unsigned fieldmask) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  cudaStream_t s = C.stream;
  if (fieldmask & (OLAMGPU_F_SCALARS | OLAMGPU_F_SCALAR_TEND)) {
    OG_CHECK(ensure_plain(s));
    const size_t wz = (size_t)C.g.mza * C.g.mwa;
    for (int n = 0; n < C.tr.n; ++n) {
      if (fieldmask & OLAMGPU_F_SCALARS)
        OG_CUDA(cudaMemcpyAsync(C.tr.h_p[n], C.tr.p[n].p, wz * 4, cudaMemcpyDeviceToHost, s));
      if (fieldmask & OLAMGPU_F_SCALAR_TEND)
        OG_CUDA(cudaMemcpyAsync(C.tr.h_t[n], C.tr.t[n].p, wz * 4, cudaMemcpyDeviceToHost, s));
    }
  }
  if (C.have_state) {
    if (C.dy.ready) {
      OG_CHECK(dyn_state_to_host(fieldmask, s));
      if (fieldmask & OLAMGPU_F_EDDY) OG_CHECK(dyn_eddy_to_host(s));
    } else {
      const size_t wz = (size_t)C.g.mza * C.g.mwa, vz = (size_t)C.g.mza * C.g.mva;
      auto cp = [&](void* h, const void* dv, size_t b) -> int {
        if (h && dv) OG_CUDA(cudaMemcpyAsync(h, dv, b, cudaMemcpyDeviceToHost, s));
        return OLAMGPU_OK;
      };
      if (fieldmask & OLAMGPU_F_VMASC) OG_CHECK(cp(C.hstate.vmasc, C.tp.vmasc.p, vz * 4));
      if (fieldmask & OLAMGPU_F_WMASC) OG_CHECK(cp(C.hstate.wmasc, C.tp.wmasc.p, wz * 4));
      if (fieldmask & OLAMGPU_F_RHO) OG_CHECK(cp(C.hstate.rho, C.tp.rho.p, wz * 8));
    }
  }
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

int olamgpu_scalar_transport_rk(const float* rho_old, olamgpu_cfl_diag* diag) {
  int rc = transport_run(rho_old, diag);
  if (rc == OLAMGPU_OK) {
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) { set_error(std::string("kernel launch: ") + cudaGetErrorString(e)); return OLAMGPU_E_CUDA; }
  }
  return rc;
}

int olamgpu_scalar_transport_rk_adjoint(const float* rho_old, float* const* lam, float* const* lam_sct) {
  int rc = transport_adjoint_run(rho_old, lam, lam_sct);
  if (rc == OLAMGPU_OK) {
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) { set_error(std::string("kernel launch: ") + cudaGetErrorString(e)); return OLAMGPU_E_CUDA; }
  }
  return rc;
}

int olamgpu_prog_wrtv_rk(int istp) { return dyn_prog_wrtv_rk(istp); }

int olamgpu_tend0(float* rho_old) { return dyn_tend0(rho_old); }

int olamgpu_timeavg_momsc(void) { return dyn_timeavg_momsc(); }

int olamgpu_set_halo(const olamgpu_halo* halo) {
  glue_drop_graphs();
  return halo_set(halo);
}

int olamgpu_set_scalars_bottom(void) { return glue_set_scalars_bottom(); }

int olamgpu_diagvel_t3d(void) { return dyn_diagvel_t3d(); }

int olamgpu_tracer_maxmin(float* smax) { return glue_tracer_maxmin(smax); }

int olamgpu_mass_sums(int nsel, const int* ids, double* sums) { return glue_mass_sums(nsel, ids, sums); }

int olamgpu_timestep(unsigned flags, int nmass, const int* mass_ids) {
  return glue_timestep(flags, nmass, mass_ids);
}

int olamgpu_timestep_diag(float* smax, double* sums) { return glue_timestep_diag(smax, sums); }

int olamgpu_set_surface_emission(const float* const* emis) { return emission_set(emis); }

int olamgpu_set_tile_shape(int T, int G, int KS, int ord) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  glue_drop_graphs();
  Transport& tp = C.tp;
  if (T == 0 && G == 0 && KS == 0) {   // back to the autotuner
    tp.autotune = true;
    tp.tuned_ntp = -1;
    return OLAMGPU_OK;
  }
  if ((T != 8 && T != 16 && T != 32) || (G != 32 && G != 64 && G != 128) || KS < 1 || KS > 8 || ord < 0 ||
      ord > 3) {
    set_error("tile shape: T 8, 16 or 32, G 32, 64 or 128, 1 <= KS <= 8, order 0..3");
    return OLAMGPU_E_ARG;
  }
  const bool paired = (ord & 2) != 0;
  if (paired && (T != 16 || G != 128 || KS != 1)) {
    set_error("tile shape: the paired kernel runs 16-column tiles of 128 tracers, KS = 1");
    return OLAMGPU_E_ARG;
  }
  const int order = C.opts.scal_horiz_adv_order;
  if (C.g.tile_T != T || C.g.tile_ord != (ord & 1)) OG_CHECK(build_tiles(&C.hgrid, C.g, order, C.stream, T, ord & 1));
  if (C.g.tile_T != T || !tile_shape_fits(C.g, G) || (paired && !C.g.tile_paired)) {
    set_error("tile shape: this grid has no " + std::to_string(T) + "-column tiles of " + std::to_string(G) +
              " tracers within the shared memory" + (paired ? " with column pairs" : ""));
    return OLAMGPU_E_UNSUPPORTED;
  }
  C.g.tile_G = G;
  C.g.tile_KS = KS;
  C.g.tile_pairk = paired;
  if (!paired) tp.prec.release();   // no pair records without the paired kernel
  tp.autotune = false;
  return OLAMGPU_OK;
}

int olamgpu_tile_shape(int* shape, int max, int* cand, float* ms) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return -OLAMGPU_E_STATE; }
  if (shape) {
    shape[0] = C.g.tile_T; shape[1] = C.g.tile_G; shape[2] = C.g.tile_KS;
    shape[3] = C.g.tile_ord | (C.g.tile_pairk ? 2 : 0);
  }
  const auto& L = C.tp.tune_log;
  for (int i = 0; i < (int)L.size() && i < max; ++i) {
    if (cand) {
      int* c = cand + 5 * i;
      c[0] = L[i].T; c[1] = L[i].G; c[2] = L[i].KS; c[3] = L[i].ord; c[4] = L[i].chosen;
    }
    if (ms) ms[i] = L[i].ms;
  }
  return (int)L.size();
}

int olamgpu_window_forward(int nsteps, int nchk, unsigned flags) { return window_forward(nsteps, nchk, flags); }

int olamgpu_window_adjoint(float* const* lam, float* const* lam_sct) { return window_adjoint(lam, lam_sct); }

int olamgpu_window_memory(int flags, int segment_steps, int nsteps, int nchk) {
  return window_memory(flags, segment_steps, nsteps, nchk);
}

int olamgpu_window_rewind(void) { return window_rewind(); }

void* olamgpu_stream(void) { return (void*)ctx().stream; }

int olamgpu_profile(int enable, int reset) {
  prof_resolve();
  if (reset) { g_prof_names.clear(); g_prof_ms.clear(); g_prof_cnt.clear(); }
  g_prof_on = enable != 0;
  return OLAMGPU_OK;
}

int olamgpu_profile_read(int max, char* names, double* total_ms, unsigned long long* counts) {
  Context& C = ctx();
  if (C.stream) cudaStreamSynchronize(C.stream);
  prof_resolve();
  int n = (int)g_prof_names.size();
  for (int i = 0; i < n && i < max; ++i) {
    if (names) {
      std::memset(names + 32 * i, 0, 32);
      std::strncpy(names + 32 * i, g_prof_names[i].c_str(), 31);
    }
    if (total_ms) total_ms[i] = g_prof_ms[i];
    if (counts) counts[i] = g_prof_cnt[i];
  }
  return n;
}

unsigned long long olamgpu_launch_count(int reset) {
  unsigned long long v = g_launches;
  if (reset) g_launches = 0;
  return v;
}

}  // extern "C"
