// transport_kernels.cuh -- kernel declarations and device helpers shared by
// the transport translation units.
#pragma once

#include "internal.h"

namespace olamgpu {

// A tracer field: element (point p, level k, tracer t) lives at
// base[((size_t)p * mza + k) * ld + t0 + t].  ld = 1, t0 = 0 is OLAM's own
// (mza, n) layout of one tracer; ld = ntp is the batched layout.
struct TView {
  float* base;
  int ld;
  int t0;
};

struct CTView {
  const float* base;
  int ld;
  int t0;
};

// Device-side grid pointers passed by value to kernels.
struct GridK {
  int mza, mwa, mva;
  const int* __restrict__ npoly;
  const int* __restrict__ w_nb;
  const int* __restrict__ w_ev;
  const float* __restrict__ w_dirv;
  const int* __restrict__ v_iw;
  const int* __restrict__ lpw;
  const int* __restrict__ lpv;
  const float* __restrict__ volti;
  const float* __restrict__ a_w;   // Fortran (mza,2,2)
  const float* __restrict__ a_wu;
};

GridK gridk(const DevGrid& d);

// the positive-definite / monotonic limiters' constants (scalar_transport_rk.F90:14-17)
static const float kEps0 = 1.e-32f;
static const float kEps1 = 3.e-07f;

// a_w(k, i, j) of a Fortran (mza, 2, 2) array at device level kd
__device__ __forceinline__ float AW(const float* a, int mza, int kd, int i, int j) {
  return __ldg(a + kd + mza * ((i - 1) + 2 * (j - 1)));
}

// grad_z_quadratic (grad_lib.f90:166-229) at device level kd, from the three
// column values around it.  Boundary flags as itopbc/ibotbc.
__device__ __forceinline__ void zrec(const float* a, int mza, int kd, int kb, float sm1, float s0,
                                     float sp1, float sp2_unused, bool ibot, bool itop,
                                     float& sb, float& st) {
  (void)sp2_unused;
  float ds_k, ds_km1;
  if (kd <= mza - 2) ds_k = sp1 - s0;
  else ds_k = itop ? (s0 - sm1) : 0.f;
  if (kd >= kb + 1) ds_km1 = s0 - sm1;
  else ds_km1 = ibot ? ((kb <= mza - 2) ? sp1 - s0 : 0.f) : 0.f;
  sb = s0 + ds_k * AW(a, mza, kd, 1, 1) + ds_km1 * AW(a, mza, kd, 2, 1);
  st = s0 + ds_k * AW(a, mza, kd, 1, 2) + ds_km1 * AW(a, mza, kd, 2, 2);
}


// Per-tracer update mode on the last RK stage.
enum { MODE_PLAIN = 0, MODE_MONOT = 1, MODE_PD = 2 };

// ---- launchers (transport_kernels.cu) ------------------------------------
void launch_check_cfls(const DevGrid& d, const Transport& tp, int nrk, float dtl,
                       unsigned long long* red, cudaStream_t s);
void launch_rhos(const DevGrid& d, Transport& tp, int nrk, cudaStream_t s);
void launch_implicit_prep(const DevGrid& d, Transport& tp, int nrk, const float* dtlr,
                          cudaStream_t s);
void launch_implicit_solve(const DevGrid& d, const Transport& tp, int nrk, int istage, float dtr,
                           CTView scp0, TView scp, int nt, cudaStream_t s);
void launch_diffusion(const DevGrid& d, const Transport& tp, CTView scp, TView sct, int nt,
                      cudaStream_t s);
void launch_scp0_pd_update(const DevGrid& d, const Transport& tp, TView scp0, CTView sct,
                           const int* mode, int nt, float dtr, cudaStream_t s);

// reference-mirroring passes, generic tracer count nt
void launch_grad(const DevGrid& d, CTView scp, float* gx, int nt, int order, bool bounded,
                 cudaStream_t s);
void launch_vflux(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, const float* gx,
                  int nt, int order, bool unbounded, const int* mode, bool anylim, cudaStream_t s);
void launch_wcol(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, CTView sct,
                 const float* rhos, TView out, int nt, int istage, int nrk, float dtr,
                 const int* mode, bool anylim, cudaStream_t s);
// pass 3 of an unlimited stage, a thread per cell (coalesced in k)
void launch_wcell(const DevGrid& d, const Transport& tp, CTView scp, CTView scp0, CTView sct, const float* rhos,
                  TView out, int nt, int istage, int nrk, float dtr, cudaStream_t s);
void launch_vapply(const DevGrid& d, const Transport& tp, int nt, const int* mode, cudaStream_t s);
void launch_tend(const DevGrid& d, const Transport& tp, CTView scp_in, CTView scp0, const float* rhos,
                 TView out, int nt, int istage, int nrk, float dtr, const int* mode, cudaStream_t s);

// fused batched update (plain mode), all tracers of the batched layout
void launch_fused_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                        const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr,
                        const float* rhos, cudaStream_t s);

// the same update in tiles of columns (grids without terrain; transport_tile.cu):
// the step's per-(column, level) weight records (into tp.wrec), then a stage
bool tile_stage_available(const DevGrid& d, const Transport& tp, int order);
int launch_tile_weights(const DevGrid& d, Transport& tp, const float* rhos, cudaStream_t s);
// grp0 / ngrp_run: the tracer groups of G tracers this launch runs (0, 0:
// all); G_force: tracers per block (0: the tuned shape's)
int launch_tile_stage(const DevGrid& d, const Transport& tp, const float* S, const float* S0,
                      const float* SCT, float* OUT, int ntp, int istage, int nrk, float dtr, int* status,
                      cudaStream_t s, int grp0 = 0, int ngrp_run = 0, int G_force = 0);
// does the current tile width have a stage kernel of G tracers per block
// within the shared memory
bool tile_shape_fits(const DevGrid& d, int G);
// choose the stage kernel's shape on the step's inputs (S, S0, SCT; OUT is
// scratch); rebuilds the tile tables when the width changes
int tile_autotune(Context& C, const float* S, const float* S0, const float* SCT, float* OUT, float dtr);

// copy the columns outside jtw_prog (colsize floats each) from src to dst
void launch_copy_cols(const int* cols, int ncol, const float* src, float* dst, size_t colsize,
                      cudaStream_t s);

// layout transposes: per-tracer arrays <-> batched layout
// tracers [0, n) of src / dst into slots [0, width) of Q rows of length
// stride (q and src / dst offset by the caller to a tracer range)
void launch_gather_q_range(float* q, const float* const* src, int n, int width, int stride, size_t npk,
                           cudaStream_t s);
void launch_scatter_q_range(const float* q, float* const* dst, int n, int width, int stride, size_t npk,
                            cudaStream_t s);
void launch_gather_q(float* q, const float* const* src, int n, int ntp, size_t npts_k,
                     cudaStream_t s);
void launch_scatter_q(const float* q, float* const* dst, int n, int ntp, size_t npts_k,
                      cudaStream_t s);

// the tracers' last-stage modes on the device (tp.d_mode: modes, then the
// flags of the low-order scp0 pre-update), uploaded when they change
int tracer_modes(Context& C, std::vector<int>& modes, std::vector<int>& pdm, bool& anylim, bool& any_pdm);

// adjoint of the positive-definite last stage (transport_adjoint_pd.cu) for
// the tracers [t0, t0 + nt) of the batched layout whose mode is MODE_PD: S
// the stage input, S0p scp0', L the adjoint of the stage output (below-ground
// levels folded), L0 the implicit solve's adjoint of scp0'; writes their
// LIN (adjoint of S), L0 (of scp0) and LS (of sct)
int pd_adjoint_stage(Context& C, const float* S, const float* S0p, const float* L, float* LIN, float* L0,
                     float* LS, float dtr, int t0, int nt, cudaStream_t s);
void pd_adjoint_release();

// inputs and per-step coefficients shared by the transport and its adjoint
// (transport.cu): uploads, check_cfls, rhos, implicit factors; dtlr per stage
int transport_prepare(Context& C, const float* rho_old_host, bool upload_tracers, float dtlr[3]);

}  // namespace olamgpu
