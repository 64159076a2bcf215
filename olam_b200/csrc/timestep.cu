// timestep.cu -- the device part of one long timestep (omodel/timestep.f90:
// 66-319) and the glue around the hot path that keeps it on the device:
//   k_bottom_fill   set_scalars_bottom (omodel/obnd.f90:7-36)
//   k_maxmin        tracer_maxmin (outils/check_nans.F90:164-203)
//   k_mass_part / k_mass_final   compute_mass_sums and mass_sum_from_*
//                   (outils/check_nans.F90:207-550), a fixed-order reduction
//   diagvel_t3d     (omodel/vel_t3d.f90:7-35) is dynamics.cu's k_vel_t3d
// olamgpu_timestep runs the long step's device sequence; in RESIDENT mode it
// records the sequence as a CUDA graph (one per tracer-buffer rotation) and
// replays it, so a long step costs one graph launch on the host.
#include <cfloat>
#include <cmath>
#include <cstring>

#include "transport_kernels.cuh"

namespace olamgpu {

#define MASS_BLOCKS 296   // 2 x 148 SMs
#define MASS_THREADS 256

// float -> unsigned key whose unsigned order is the float order
__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
static inline float key_to_float(unsigned k) {
  const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// element (cell x, tracer n) of a tracer view is base[x * stride + n]
__global__ void k_bottom_fill(const int* __restrict__ prog, int nprog, const int* __restrict__ lpw, int mza,
                              float* __restrict__ base, int stride, int nt) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * nt) return;
  const int j = (int)(i / nt), n = (int)(i % nt);
  const int iw = prog[j], kb = lpw[iw];
  const size_t c = (size_t)iw * mza;
  const float v = base[(c + kb) * stride + n];
  for (int kd = 0; kd < kb; ++kd) base[(c + kd) * stride + n] = v;
}

__global__ void k_key_init(unsigned* keys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = fkey(-FLT_MAX);
}

// blockDim (32, 8): x over tracers, y over cells
__global__ void k_maxmin(const int* __restrict__ prog, int nprog, const int* __restrict__ lpw, int mza,
                         const float* __restrict__ base, int stride, int nt, unsigned* __restrict__ keys) {
  __shared__ float shi[8][32], slo[8][32];
  const int n = blockIdx.y * 32 + threadIdx.x;
  float hi = -FLT_MAX, lo = FLT_MAX;
  if (n < nt) {
    const size_t ncell = (size_t)nprog * mza;
    for (size_t c = (size_t)blockIdx.x * 8 + threadIdx.y; c < ncell; c += (size_t)gridDim.x * 8) {
      const int iw = prog[c / mza], kd = (int)(c % mza);
      if (kd < lpw[iw]) continue;
      const float v = base[((size_t)iw * mza + kd) * stride + n];
      if (v != v) continue;
      hi = fmaxf(hi, v);
      lo = fminf(lo, v);
    }
  }
  shi[threadIdx.y][threadIdx.x] = hi;
  slo[threadIdx.y][threadIdx.x] = lo;
  __syncthreads();
  if (threadIdx.y == 0 && n < nt) {
    for (int r = 1; r < 8; ++r) { hi = fmaxf(hi, shi[r][threadIdx.x]); lo = fminf(lo, slo[r][threadIdx.x]); }
    atomicMax(&keys[2 * n], fkey(hi));
    atomicMax(&keys[2 * n + 1], fkey(-lo));
  }
}

struct MassArgs {
  const int* prog; int nprog; const int* lpw; int mza;
  const double* rho; const double* volt;
  int nsel;
  const float* sp[8]; int sstride[8];
  double* part;   // (MASS_BLOCKS, 1 + nsel)
};

// each block adds a fixed subset of the cells in a fixed order, then a fixed
// tree: the sums repeat bit for bit
__global__ void __launch_bounds__(MASS_THREADS) k_mass_part(MassArgs a) {
  __shared__ double red[MASS_THREADS];
  double acc[9];
  for (int m = 0; m <= a.nsel; ++m) acc[m] = 0.0;
  const size_t ncell = (size_t)a.nprog * a.mza;
  for (size_t c = (size_t)blockIdx.x * MASS_THREADS + threadIdx.x; c < ncell; c += (size_t)MASS_BLOCKS * MASS_THREADS) {
    const int iw = a.prog[c / a.mza], kd = (int)(c % a.mza);
    if (kd < a.lpw[iw]) continue;
    const size_t x = (size_t)iw * a.mza + kd;
    const double rv = a.rho[x] * a.volt[x];
    acc[0] += rv;
    for (int m = 0; m < a.nsel; ++m) acc[1 + m] += rv * (double)a.sp[m][x * a.sstride[m]];
  }
  for (int m = 0; m <= a.nsel; ++m) {
    red[threadIdx.x] = acc[m];
    __syncthreads();
    for (int h = MASS_THREADS / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) a.part[(size_t)blockIdx.x * (a.nsel + 1) + m] = red[0];
    __syncthreads();
  }
}

__global__ void k_mass_final(const double* __restrict__ part, int nm, double* __restrict__ out) {
  const int m = threadIdx.x;
  if (m >= nm) return;
  double s = 0.0;
  for (int b = 0; b < MASS_BLOCKS; ++b) s += part[(size_t)b * nm + m];
  out[m] = s;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

void glue_drop_graphs() {
  Glue& G = ctx().glue;
  for (auto& g : G.g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g = StepGraph();
  }
  G.eager_done = false;
}

void glue_release() {
  glue_drop_graphs();
  Glue& G = ctx().glue;
  G.keys.release();
  G.part.release();
  G.sums.release();
  G = Glue();
}

// the view (pointer, stride) of registered scalar n
static void scalar_view(Context& C, int n, float*& p, int& stride) {
  if (C.tr.q_valid) { p = C.tr.q[C.tr.qcur].p + n; stride = C.tr.ntp; }
  else { p = C.tr.p[n].p; stride = 1; }
}

static void launch_bottom_fill(Context& C, cudaStream_t s) {
  const DevGrid& d = C.g;
  Tracers& tr = C.tr;
  if (d.nw_prog <= 0) return;
  if (tr.n > 0) {
    if (tr.q_valid) {
      k_bottom_fill<<<cdiv((size_t)d.nw_prog * tr.ntp, 256), 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, d.mza,
                                                                         tr.q[tr.qcur].p, tr.ntp, tr.n);
      OG_LAUNCHED();
    } else {
      for (int n = 0; n < tr.n; ++n) {
        k_bottom_fill<<<cdiv(d.nw_prog, 256), 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, d.mza, tr.p[n].p, 1, 1);
        OG_LAUNCHED();
      }
    }
  }
  if (C.dy.thil.p) {
    k_bottom_fill<<<cdiv(d.nw_prog, 256), 256, 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, d.mza, C.dy.thil.p, 1, 1);
    OG_LAUNCHED();
  }
}

static int launch_maxmin(Context& C, cudaStream_t s) {
  const DevGrid& d = C.g;
  Tracers& tr = C.tr;
  Glue& G = C.glue;
  const int nk = std::max(2 * tr.n, 1);
  OG_CHECK(G.keys.alloc(nk));
  k_key_init<<<cdiv(nk, 256), 256, 0, s>>>(G.keys.p, 2 * tr.n);
  OG_LAUNCHED();
  if (tr.n == 0 || d.nw_prog <= 0) return OLAMGPU_OK;
  const unsigned gx = 4 * 148;
  if (tr.q_valid) {
    dim3 grid(gx, (tr.n + 31) / 32);
    k_maxmin<<<grid, dim3(32, 8), 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, d.mza, tr.q[tr.qcur].p, tr.ntp, tr.n,
                                          G.keys.p);
    OG_LAUNCHED();
  } else {
    for (int n = 0; n < tr.n; ++n) {
      k_maxmin<<<dim3(gx, 1), dim3(32, 8), 0, s>>>(d.jtw_prog.p, d.nw_prog, d.lpw.p, d.mza, tr.p[n].p, 1, 1,
                                                   G.keys.p + 2 * n);
      OG_LAUNCHED();
    }
  }
  return OLAMGPU_OK;
}

static int check_ids(Context& C, int nsel, const int* ids) {
  if (nsel < 0 || nsel > 8 || (nsel > 0 && !ids)) { set_error("mass sums: 0 <= nsel <= 8 scalar indices"); return OLAMGPU_E_ARG; }
  for (int i = 0; i < nsel; ++i)
    if (ids[i] < 1 || ids[i] > C.tr.n) {
      set_error("mass sums: scalar index " + std::to_string(ids[i]) + " is not registered");
      return OLAMGPU_E_ARG;
    }
  return OLAMGPU_OK;
}

static int launch_mass(Context& C, int nsel, const int* ids, cudaStream_t s) {
  const DevGrid& d = C.g;
  Glue& G = C.glue;
  OG_CHECK(G.part.alloc((size_t)MASS_BLOCKS * 9));
  OG_CHECK(G.sums.alloc(9));
  MassArgs a;
  a.prog = d.jtw_prog.p; a.nprog = d.nw_prog; a.lpw = d.lpw.p; a.mza = d.mza;
  a.rho = C.tp.rho.p; a.volt = C.dy.volt.p; a.nsel = nsel; a.part = G.part.p;
  for (int i = 0; i < 8; ++i) { a.sp[i] = nullptr; a.sstride[i] = 1; }
  for (int i = 0; i < nsel; ++i) {
    float* p; int st;
    scalar_view(C, ids[i] - 1, p, st);
    a.sp[i] = p;
    a.sstride[i] = st;
  }
  k_mass_part<<<MASS_BLOCKS, MASS_THREADS, 0, s>>>(a);
  k_mass_final<<<1, 32, 0, s>>>(G.part.p, nsel + 1, G.sums.p);
  OG_LAUNCHED(); OG_LAUNCHED();
  return OLAMGPU_OK;
}

static int require_ready(Context& C, const char* what) {
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  if (!C.dy.ready || !C.have_state) {
    set_error(std::string(what) + " needs prog_wrtv_rk's set-up and the state arrays registered at init");
    return OLAMGPU_E_STATE;
  }
  return OLAMGPU_OK;
}

// device copies of the inputs before a stand-alone glue call
static int glue_inputs(Context& C, unsigned mask, bool tracers, cudaStream_t s) {
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_device(mask, s));
    if (tracers && C.tr.n > 0) OG_CHECK(tracers_to_device(s));
  } else if (!C.dy.uploaded) {
    OG_CHECK(dyn_state_to_device(OLAMGPU_F_ALL, s));
    C.dy.uploaded = true;
  }
  return OLAMGPU_OK;
}

int glue_set_scalars_bottom() {
  Context& C = ctx();
  OG_CHECK(require_ready(C, "set_scalars_bottom"));
  cudaStream_t s = C.stream;
  OG_CHECK(glue_inputs(C, OLAMGPU_F_THIL, true, s));
  launch_bottom_fill(C, s);
  if (C.coherence == OLAMGPU_SYNC_EACH_CALL) {
    OG_CHECK(dyn_state_to_host(OLAMGPU_F_THIL, s));
    OG_CHECK(tracers_to_host(s));
    OG_CUDA(cudaStreamSynchronize(s));
  }
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

int glue_tracer_maxmin(float* smax) {
  Context& C = ctx();
  OG_CHECK(require_ready(C, "tracer_maxmin"));
  if (C.tr.n > 0 && !smax) { set_error("tracer_maxmin: smax is NULL"); return OLAMGPU_E_ARG; }
  cudaStream_t s = C.stream;
  OG_CHECK(glue_inputs(C, 0, true, s));
  OG_CHECK(launch_maxmin(C, s));
  std::vector<unsigned> k(std::max(2 * C.tr.n, 1));
  OG_CUDA(cudaMemcpyAsync(k.data(), C.glue.keys.p, 2 * C.tr.n * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < 2 * C.tr.n; ++i) smax[i] = key_to_float(k[i]);
  return check_device_status();
}

int glue_mass_sums(int nsel, const int* ids, double* sums) {
  Context& C = ctx();
  OG_CHECK(require_ready(C, "mass sums"));
  OG_CHECK(check_ids(C, nsel, ids));
  if (!sums) { set_error("mass sums: sums is NULL"); return OLAMGPU_E_ARG; }
  cudaStream_t s = C.stream;
  OG_CHECK(glue_inputs(C, OLAMGPU_F_RHO, nsel > 0, s));
  OG_CHECK(launch_mass(C, nsel, ids, s));
  OG_CUDA(cudaMemcpyAsync(sums, C.glue.sums.p, (size_t)(nsel + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

// ---- surface emission ----------------------------------------------------------
// OLAM's physics adds surface sources to the tracer tendencies between tend0
// and scalar_transport_rk; the long step on the device has no host physics in
// between, so a registered emission field E(iw) per tracer is added to
// var_t(lpw, iw) right after tend0.
__global__ void k_emission(const int* __restrict__ prog, int nprog, const int* __restrict__ lpw, int mza,
                           const float* __restrict__ emis, int ntp, int n, float* __restrict__ q,
                           float* const* __restrict__ planes) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)nprog * n) return;
  const int j = (int)(i / n), t = (int)(i % n);
  const int iw = prog[j];
  const size_t cell = (size_t)iw * mza + lpw[iw];
  const float e = emis[(size_t)iw * ntp + t];
  if (q) q[cell * ntp + t] += e;
  else planes[t][cell] += e;
}

static DevBuf<float*> g_emis_ptab;

void launch_emission(Context& C, cudaStream_t s) {
  Tracers& tr = C.tr;
  if (!C.tp.have_emis || tr.n <= 0 || C.g.nw_prog <= 0) return;
  float* q = nullptr;
  float* const* planes = nullptr;
  if (tr.q_valid && tr.qt.p) q = tr.qt.p;
  else planes = g_emis_ptab.p;
  k_emission<<<cdiv((size_t)C.g.nw_prog * tr.n, 256), 256, 0, s>>>(C.g.jtw_prog.p, C.g.nw_prog, C.g.lpw.p, C.g.mza,
                                                                  C.tp.emis.p, tr.ntp, tr.n, q, planes);
  OG_LAUNCHED();
}

int emission_set(const float* const* emis) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  glue_drop_graphs();
  Tracers& tr = C.tr;
  if (!emis) { C.tp.have_emis = false; return OLAMGPU_OK; }
  if (tr.n <= 0) { set_error("surface emission: register the scalars first"); return OLAMGPU_E_STATE; }
  const int mwa = C.g.mwa, ntp = tr.ntp;
  std::vector<float> h((size_t)mwa * ntp, 0.f);
  for (int n = 0; n < tr.n; ++n)
    if (emis[n])
      for (int iw = 0; iw < mwa; ++iw) h[(size_t)iw * ntp + n] = emis[n][iw];
  cudaStream_t s = C.stream;
  OG_CHECK(upload(C.tp.emis, h.data(), h.size(), s));
  std::vector<float*> pt(tr.n);
  for (int n = 0; n < tr.n; ++n) pt[n] = tr.t[n].p;
  OG_CHECK(upload(g_emis_ptab, pt.data(), pt.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));   // the host vectors die here
  C.tp.have_emis = true;
  return OLAMGPU_OK;
}

int emission_repoint(Context& C, cudaStream_t s) {
  Tracers& tr = C.tr;
  if (!C.tp.have_emis || tr.n <= 0) return OLAMGPU_OK;
  std::vector<float*> pt(tr.n);
  for (int n = 0; n < tr.n; ++n) pt[n] = tr.t[n].p;
  OG_CHECK(upload(g_emis_ptab, pt.data(), pt.size(), s));
  OG_CUDA(cudaStreamSynchronize(s));   // the host vector dies here
  return OLAMGPU_OK;
}

// the long step's device sequence (timestep.f90:66-319); without the
// transport (with_transport false) the dynamics and the glue of thil only
static int run_sequence(Context& C, unsigned flags, int nmass, const int* ids, bool with_transport = true) {
  cudaStream_t s = C.stream;
  OG_CHECK(dyn_tend0(nullptr));
  if (with_transport) launch_emission(C, s);
  if (flags & OLAMGPU_TS_HORIZ_K) OG_CHECK(dyn_comp_horiz_k());
  for (int j = 1; j <= C.opts.nacoust; ++j) OG_CHECK(dyn_prog_wrtv_rk(j));
  OG_CHECK(dyn_timeavg_momsc());
  if (!with_transport) {
    if (C.dy.thil.p && C.g.nw_prog > 0) {
      k_bottom_fill<<<cdiv(C.g.nw_prog, 256), 256, 0, s>>>(C.g.jtw_prog.p, C.g.nw_prog, C.g.lpw.p, C.g.mza,
                                                           C.dy.thil.p, 1, 1);
      OG_LAUNCHED();
    }
    OG_CUDA(cudaGetLastError());
    return OLAMGPU_OK;
  }
  OG_CHECK(transport_run(nullptr, nullptr));
  if (flags & OLAMGPU_TS_MAXMIN) OG_CHECK(launch_maxmin(C, s));
  launch_bottom_fill(C, s);
  if (C.halo.on) {
    // the border columns of the tracers and thil for the next step
    // (timestep.f90:310-314)
    if (C.tr.n > 0 && C.tr.q_valid) OG_CHECK(halo_exchange(C, C.tr.q[C.tr.qcur].p, C.tr.ntp, s));
    HField f[1] = {{C.dy.thil.p, 4}};
    OG_CHECK(halo_exchange_fields(C, HALO_W, f, 1, s));
  }
  if (flags & OLAMGPU_TS_MASS) OG_CHECK(launch_mass(C, nmass, ids, s));
  OG_CUDA(cudaGetLastError());
  return OLAMGPU_OK;
}

int glue_run_sequence(Context& C, unsigned flags, bool with_transport) {
  return run_sequence(C, flags & ~(unsigned)(OLAMGPU_TS_MAXMIN | OLAMGPU_TS_MASS), 0, nullptr, with_transport);
}

static bool same_step(const StepGraph& g, unsigned flags, int nmass, const int* ids) {
  if (!g.exec || g.flags != flags || g.nmass != nmass) return false;
  for (int i = 0; i < nmass; ++i)
    if (g.ids[i] != ids[i]) return false;
  return true;
}

int glue_timestep(unsigned flags, int nmass, const int* ids) {
  Context& C = ctx();
  OG_CHECK(require_ready(C, "timestep"));
  if (C.coherence != OLAMGPU_RESIDENT) {
    set_error("olamgpu_timestep keeps the state on the device: set OLAMGPU_RESIDENT first");
    return OLAMGPU_E_STATE;
  }
  if ((flags & OLAMGPU_TS_HORIZ_K) && !C.dy.eddy_on) {
    set_error("OLAMGPU_TS_HORIZ_K needs the eddy inputs (olamgpu_set_eddy)");
    return OLAMGPU_E_STATE;
  }
  if (!(flags & OLAMGPU_TS_MASS)) nmass = 0;
  OG_CHECK(check_ids(C, nmass, ids));
  Glue& G = C.glue;
  cudaStream_t s = C.stream;
  G.last_flags = flags;
  G.last_nmass = nmass;
  G.last_ntr = C.tr.n;
  // a halo exchange calls back into the host between stages: no graph
  const bool graph = (flags & OLAMGPU_TS_GRAPH) && C.form != OLAMGPU_TRANSPORT_PLAIN && C.tr.n > 0 && !C.halo.on;
  if (!graph) return run_sequence(C, flags, nmass, ids);
  // the graph reads the tracers from Q[qcur]; a sync to the device may have
  // refreshed the per-tracer arrays instead
  OG_CHECK(ensure_q(s));
  StepGraph& sg = G.g[C.tr.qcur];
  if (same_step(sg, flags, nmass, ids)) {
    OG_PROF("timestep_graph", s);
    OG_CUDA(cudaGraphLaunch(sg.exec, s));
    g_launches += sg.launches;
    C.tr.qcur = sg.qcur_after;
    C.tr.q_valid = true;
    if (flags & OLAMGPU_TS_HORIZ_K) C.dy.hk_on_device = true;
    return OLAMGPU_OK;
  }
  if (!G.eager_done) {
    // first run: buffers, first-call set-up (damping factors, tile records)
    OG_CHECK(run_sequence(C, flags, nmass, ids));
    G.eager_done = true;
    return OLAMGPU_OK;
  }
  // record this rotation's step; on failure put the host state back and run
  // the step as it is
  if (sg.exec) { cudaGraphExecDestroy(sg.exec); sg = StepGraph(); }
  const int qcur0 = C.tr.qcur;
  const bool qv0 = C.tr.q_valid, hk0 = C.dy.hk_on_device;
  const unsigned long long l0 = g_launches;
  prof_suspend(true);
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  int rc = e == cudaSuccess ? run_sequence(C, flags, nmass, ids) : OLAMGPU_E_CUDA;
  cudaGraph_t gr = nullptr;
  if (e == cudaSuccess) e = cudaStreamEndCapture(s, &gr);
  prof_suspend(false);
  cudaGraphExec_t ex = nullptr;
  if (rc == OLAMGPU_OK && e == cudaSuccess && gr) e = cudaGraphInstantiate(&ex, gr, 0);
  if (gr) cudaGraphDestroy(gr);
  if (rc != OLAMGPU_OK || e != cudaSuccess || !ex) {
    cudaGetLastError();
    C.tr.qcur = qcur0;
    C.tr.q_valid = qv0;
    C.dy.hk_on_device = hk0;
    g_launches = l0;
    if (ex) cudaGraphExecDestroy(ex);
    set_error(std::string("timestep graph capture failed: ") + cudaGetErrorString(e));
    return run_sequence(C, flags, nmass, ids);
  }
  sg.exec = ex;
  sg.flags = flags;
  sg.nmass = nmass;
  for (int i = 0; i < nmass; ++i) sg.ids[i] = ids[i];
  sg.qcur_after = C.tr.qcur;
  sg.launches = g_launches - l0;
  OG_PROF("timestep_graph", s);
  OG_CUDA(cudaGraphLaunch(ex, s));
  return OLAMGPU_OK;
}

int glue_timestep_diag(float* smax, double* sums) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  Glue& G = C.glue;
  cudaStream_t s = C.stream;
  if (smax && (G.last_flags & OLAMGPU_TS_MAXMIN) && G.keys.p && G.last_ntr > 0) {
    std::vector<unsigned> k(2 * G.last_ntr);
    OG_CUDA(cudaMemcpyAsync(k.data(), G.keys.p, k.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < k.size(); ++i) smax[i] = key_to_float(k[i]);
  }
  if (sums && (G.last_flags & OLAMGPU_TS_MASS) && G.sums.p)
    OG_CUDA(cudaMemcpyAsync(sums, G.sums.p, (size_t)(G.last_nmass + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
  OG_CUDA(cudaStreamSynchronize(s));
  return check_device_status();
}

}  // namespace olamgpu
