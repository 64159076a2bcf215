/*
 * olamgpu.h -- C-ABI of the B200 implementation of OLAM's dynamical-core hot
 * path: the acoustic RK short step (prog_wrtv_rk) and the flux-form tracer
 * transport (scalar_transport_rk).
 *
 * The caller is OLAM's Fortran model through ISO_C_BINDING, so every array is
 * passed exactly as OLAM holds it: Fortran column-major (mza, n) with the
 * vertical index fastest, neighbour tables with OLAM's 1-based indices, and
 * point 1 of every horizontal dimension as OLAM's dummy point.  No argument
 * is a C++ or PyTorch type.  Every function returns an int status
 * (OLAMGPU_OK = 0); olamgpu_strerror() turns it into text.  There is no CPU
 * fallback: a missing or unusable GPU is an error.
 *
 * Reference interfaces replaced (martinjotte/OLAM v7.0):
 *   olamgpu_init                 -> wrtv_rk::init_wrtv_rk  (omodel/prog_wrtv_rk.f90:36-54),
 *                                   called at omodel/olam_run.f90:566 after
 *                                   alloc_adv (:342) and the state initialisation
 *   olamgpu_prog_wrtv_rk         -> wrtv_rk::prog_wrtv_rk  (omodel/prog_wrtv_rk.f90:58-488),
 *                                   called at omodel/timestep.f90:205
 *   olamgpu_scalar_transport_rk  -> scalar_transport::scalar_transport_rk(rho_old)
 *                                   (omodel/scalar_transport_rk.F90:30-385),
 *                                   called at omodel/timestep.f90:254
 *   olamgpu_tend0                -> tend0 (omodel/timestep.f90:430-496)
 *   olamgpu_timeavg_momsc        -> timeavg_momsc (omodel/timestep.f90:563-612)
 */
#ifndef OLAMGPU_H
#define OLAMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  OLAMGPU_OK = 0,
  OLAMGPU_E_ARG = 1,          /* null pointer, bad size or inconsistent table  */
  OLAMGPU_E_STATE = 2,        /* call out of order (not initialised, ...)      */
  OLAMGPU_E_UNSUPPORTED = 3,  /* option combination this build does not run    */
  OLAMGPU_E_CUDA = 4,         /* CUDA runtime error (message via strerror)     */
  OLAMGPU_E_NOMEM = 5,        /* device allocation failed                      */
  OLAMGPU_E_NODEVICE = 6,     /* no usable sm_100 device                       */
  OLAMGPU_E_NUMERIC = 7       /* device status word reported a failure         */
};

/* ---- grid (modules mem_grid, mem_ijtabs, mem_adv) ----------------------- */
/* Sizes are OLAM's: mza levels, mwa/mva/mma points INCLUDING dummy point 1.
 * Per-point tables of OLAM derived types are passed packed, e.g. itab_w%iv
 * as an int array (7, mwa) (member index fastest). */
typedef struct olamgpu_grid {
  int mza, mwa, mva, mma;

  /* loop tables jtab_w(jtw_prog)%iw(1:jend) etc. (1-based point indices) */
  int nw_prog;  const int* jtw_prog;
  int nw_wadj;  const int* jtw_wadj;
  int nv_prog;  const int* jtv_prog;
  int nv_wadj;  const int* jtv_wadj;
  int nm_prog;  const int* jtm_prog;

  /* itab_w (mem_ijtabs.f90:74-110): (7, mwa) unless noted */
  const int*   npoly;        /* (mwa) */
  const int*   itab_w_iv;
  const int*   itab_w_iw;
  const int*   itab_w_im;
  const float* itab_w_dirv;
  const float* ecvec_vx;
  const float* ecvec_vy;
  const float* ecvec_vz;
  const int*   iwglobe;      /* (mwa) */

  /* itab_v (mem_ijtabs.f90:60-72): (2, mva) */
  const int*   itab_v_iw;
  const int*   itab_v_im;
  const float* dxps;
  const float* dyps;

  /* itab_m (mem_ijtabs.f90:46-58): (3, mma) */
  const int*   itab_m_iv;
  const int*   itab_m_iw;
  const int*   itab_m_im;

  /* lowest prognosed levels (mem_grid.f90:20-24); lve2(iw), the number of
   * levels from lpw(iw) up with closed V faces (the prognostic shaved-cell
   * method of prog_wrtv_rk), must be at least lpv - lpw of every face of
   * the column (OLAM's grid sets it to the largest); NULL reads as 0 */
  const int* lpw;  const int* lpv;  const int* lpm;  const int* lve2;

  /* 1-D vertical arrays (mza) */
  const float*  zm;  const float* zt;  const float* dzm;  const float* dzt;
  const float*  dzim; const float* dzit; const float* dzt_top; const float* dzt_bot;
  const float*  zfacit;
  const double* zwgt_top8; const double* zwgt_bot8;
  const double* gdz_wgtm8; const double* gdz_wgtp8;
  const float*  gdz_wgtm;  const float*  gdz_wgtp;

  /* horizontal metrics */
  const float* wnx;  const float* wny;  const float* wnz;     /* (mwa) */
  const float* wnxo2; const float* wnyo2; const float* wnzo2; /* (mwa) */
  const float* vnx;  const float* vny;  const float* vnz;     /* (mva) */
  const float* dnu;  const float* dniu; const float* dnv; const float* dniv; /* (mva) */
  const float* arw0; const float* arm0;                        /* (mwa), (mma) */

  /* 3-D control volumes */
  const float*  arv;    /* (mza, mva) */
  const float*  arw;    /* (mza, mwa) */
  const double* volt;   /* (mza, mwa) */
  const float*  volti;  /* (mza, mwa) */
  const float*  volwi;  /* (mza, mwa) */
  const float*  volvi;  /* (mza, mva) */

  /* reconstruction coefficients */
  const float* gxps_coef; const float* gyps_coef;   /* (7, mwa) */
  const float* a_w;  const float* a_wu;              /* (mza, 2, 2) */
  const float* xy_h; const float* xy_hu;             /* (5, 7, mwa) */
  const float* xx0_v;  const float* xy0_v;  const float* yy0_v;   /* (2, mva) */
  const float* xx0_vu; const float* xy0_vu; const float* yy0_vu;  /* (2, mva) */
  const float* xx_yy;   /* (7, mwa) */
  const float* xx_yy_m; /* (3, mma) */
} olamgpu_grid;

/* ---- namelist options (oname_coms.f90:189-236, misc_coms) ----------------- */
typedef struct olamgpu_opts {
  double dtlm, dtsm;            /* long and acoustic timesteps [s]            */
  int    nacoust;
  int    nrk_wrtv, nrk_scal;    /* acoust_ / scalar_timestep_level (2 or 3)    */
  int    thil_horiz_adv_order, wind_horiz_adv_order, scal_horiz_adv_order;
  int    ithil_monot, iwind_monot, iscal_monot;
  float  divh_damp_fact;  int divh_damp_level;  int divh_damp_short;
  float  vort_damp_fact;  int vort_damp_level;  int vort_damp_short;
  float  fcoriol;               /* 2*omega for a global domain                 */
  int    mdomain;               /* 0 = global (the only domain this build runs)*/
  /* Rayleigh friction (modules/mem_rayf.f90); all off when the pointers are NULL */
  int          krayf_bot;       /* first level of rayf_cof, > mza when off      */
  const float* rayf_cof;        /* (mza) or NULL                                */
  const float* dn01d;           /* (mza) reference density   (initial == 1)     */
  const float* th01d;           /* (mza) reference theta     (initial == 1)     */
  const float* vc03d;           /* (mza, mva) reference VC                      */
  int          krayfw_bot;
  const float* rayf_cofw;       /* (mza) or NULL: W damping via b20             */
  int          initial;
} olamgpu_opts;

/* ---- prognostic state (mem_basic, mem_tend) ------------------------------ */
/* Host arrays the library reads and writes at the sync points. */
typedef struct olamgpu_state {
  double* rho;   double* press;                          /* (mza, mwa) r8 */
  float*  thil;  float* wc; float* wmc;                  /* (mza, mwa)    */
  float*  vxe;   float* vye; float* vze;                 /* (mza, mwa)    */
  float*  vmc;   float* vc;                              /* (mza, mva)    */
  float*  vmasc;                                         /* (mza, mva)    */
  float*  wmasc;                                         /* (mza, mwa)    */
  float*  alpha_press; float* pwfac;                     /* (mza, mwa)    */
  float*  pvfac;                                         /* (mza, mva)    */
  float*  thilt; float* vmxet; float* vmyet; float* vmzet; /* (mza, mwa)  */
  float*  vmt;                                           /* (mza, mva)    */
} olamgpu_state;

/* field masks for olamgpu_sync_* */
enum {
  OLAMGPU_F_RHO = 1u << 0,   OLAMGPU_F_PRESS = 1u << 1, OLAMGPU_F_THIL = 1u << 2,
  OLAMGPU_F_WC = 1u << 3,    OLAMGPU_F_WMC = 1u << 4,   OLAMGPU_F_VXE = 1u << 5,
  OLAMGPU_F_VMC = 1u << 6,   OLAMGPU_F_VC = 1u << 7,    OLAMGPU_F_VMASC = 1u << 8,
  OLAMGPU_F_WMASC = 1u << 9, OLAMGPU_F_TEND = 1u << 10, OLAMGPU_F_FACS = 1u << 11,
  OLAMGPU_F_SCALARS = 1u << 12, OLAMGPU_F_SCALAR_TEND = 1u << 13,
  OLAMGPU_F_EDDY = 1u << 14,     /* the olamgpu_eddy arrays                     */
  OLAMGPU_F_ALL = 0xffffu
};

/* diagnostics written by check_cfls (scalar_transport_rk.F90:1476-1712) */
typedef struct olamgpu_cfl_diag {
  float cfl_max;  int cfl_k;  int cfl_iwglobe;     /* max total CFL  */
  float cflh_max; int cflh_k; int cflh_iwglobe;    /* max horiz CFL  */
  float w_max;    int w_k;    int w_iwglobe;       /* max |W| (signed) */
} olamgpu_cfl_diag;

/* ---- lifecycle ------------------------------------------------------------ */

/* Replaces init_wrtv_rk (prog_wrtv_rk.f90:36-54).  Uploads the grid, packs
 * the device neighbour tables (0-based), builds the transport tiles, and
 * allocates device mirrors.  Must be called once, after alloc_adv. */
int olamgpu_init(const olamgpu_grid* grid, const olamgpu_opts* opts,
                 const olamgpu_state* state);

/* Registers the tracer table (var_tables.f90:53-69): num_scalar arrays
 * var_p(mza,mwa) and tendencies var_t(mza,mwa), pdef and do_sgsmix flags.
 * The host arrays are page-locked in place for fast transfers. */
int olamgpu_register_scalars(int num_scalar, float* const* var_p,
                             float* const* var_t, const int* pdef,
                             const int* do_sgsmix);

/* Optional turbulence inputs of the horizontal-diffusion hook
 * (scalar_transport_rk.F90:244-274): akhodx (mza, mva), khtopv (mva).
 * Without them diffusion is inactive, as with OLAM's idiffk = 0. */
int olamgpu_set_turb(const float* akhodx, const int* khtopv);

/* ---- eddy diffusion inside the acoustic step ------------------------------
 * Inputs that OLAM's PBL scheme leaves in mem_turb each long step, the
 * comp_horiz_k outputs, and the grid / option values the column solves
 * read (convect/pbl_driver.f90:136-238, 519-742; modules/mem_rayf.f90:
 * 177-220; omodel/prog_wrtv_rk.f90:214-251).  Host arrays in OLAM layout,
 * read (and for comp_horiz_k written) at the sync points like the state. */
typedef struct olamgpu_eddy {
  float* vkm;    float* vkh;       /* (mza, mwa) eddy viscosity / heat diffusivity */
  float* agamma;                   /* (mza, mwa) non-local heat term (idiffk = 1)  */
  float* akm_sfc;                  /* (nsw_max, mwa) surface momentum exchange     */
  float* sfluxt;                   /* (mwa) surface sensible heat flux [W m^-2]    */
  int*   kmtop;  int* khtop; int* kpblh;      /* (mwa) 1-based levels             */
  float* theta;  float* tair;      /* (mza, mwa)                                   */
  float* akmodx; float* akhodx;    /* (mza, mva) comp_horiz_k outputs              */
  int*   kmtopv; int* khtopv;      /* (mva)     comp_horiz_k outputs               */
  const int* lsw; int nsw_max;     /* (mwa) levels in contact with the surface     */
  const int* mrlw; const int* mrlv;              /* (mwa), (mva) itab_w/v%mrl*     */
  int mrls; const int* idiffk; const float* akmin;   /* (mrls) namelist values    */
  int test_case;                   /* DCMIP cases 110-114, 121, 122 mix elsewhere  */
  float cp;                        /* consts_coms cp                               */
  int krayfmix_bot;                /* first level of rayf_cofmix                   */
  const float* rayf_cofmix;        /* (mza) or NULL: no top-level wind mixing      */
} olamgpu_eddy;

/* Registers the eddy-diffusion inputs (NULL: off, as with idiffk = 0).  From
 * then on prog_wrtv_rk adds, in each call's column set-up, the implicit
 * vertical heat and momentum diffusion (solve_eddy_diff_heat / _vxe), the
 * top-level wind mixing (rayf_mix_top_vxe) and the horizontal diffusion of
 * thil and the winds. */
int olamgpu_set_eddy(const olamgpu_eddy* eddy);

/* Replaces comp_horiz_k (pbl_driver.f90:136-238): akmodx, akhodx, kmtopv,
 * khtopv from vkm, vkh, kmtop, khtop and rho, for every V point of
 * jtv_wadj. */
int olamgpu_comp_horiz_k(void);

int olamgpu_finalize(void);
const char* olamgpu_strerror(int status);

/* ---- hot path ------------------------------------------------------------- */

/* Coherence of host and device copies.
 * OLAMGPU_SYNC_EACH_CALL (default): every hot-path call uploads its inputs
 *   from the registered host arrays and downloads its outputs, so the call
 *   is a drop-in for the Fortran routine.
 * OLAMGPU_RESIDENT: state stays on the device between calls; the caller
 *   moves fields with olamgpu_sync_to_device / olamgpu_sync_to_host where CPU
 *   physics reads or writes them.
 * olamgpu_init restores the defaults (SYNC_EACH_CALL, fused transport). */
enum { OLAMGPU_SYNC_EACH_CALL = 0, OLAMGPU_RESIDENT = 1 };
int olamgpu_set_coherence(int mode);
int olamgpu_sync_to_device(unsigned fieldmask);
int olamgpu_sync_to_host(unsigned fieldmask);

/* Transport form.
 * OLAMGPU_TRANSPORT_FUSED (default): all tracers of an RK stage in one
 *   launch over the batched layout, in tiles of neighbouring columns whose
 *   neighbourhood is staged in shared memory (one column per block where
 *   the tile tables do not fit).  Runs any lpw / lpv (terrain).
 * OLAMGPU_TRANSPORT_PLAIN: one set of kernels per tracer mirroring the
 *   reference's passes (kept for comparison).
 * OLAMGPU_TRANSPORT_FUSED_COLUMN: the batched form with one column per
 *   block (kept for comparison; grids without terrain only). */
enum { OLAMGPU_TRANSPORT_FUSED = 0, OLAMGPU_TRANSPORT_PLAIN = 1, OLAMGPU_TRANSPORT_FUSED_COLUMN = 2 };
int olamgpu_set_transport_form(int form);

/* Replaces scalar_transport_rk(rho_old) (scalar_transport_rk.F90:30-385).
 * rho_old(mza,mwa) is the host array OLAM passes; in RESIDENT mode it may
 * be NULL, and the device copy saved by olamgpu_tend0 is used.
 * diag (optional) receives the check_cfls maxima. */
int olamgpu_scalar_transport_rk(const float* rho_old, olamgpu_cfl_diag* diag);

/* Adjoint of one scalar_transport_rk step (scalar_transport_rk.F90:30-615)
 * for every registered tracer, with the winds, densities and implicit
 * fractions of the step fixed: the unlimited step (iscal_monot = 0, no
 * horizontal diffusion) maps (scp, sct) linearly to the new scp, and this
 * applies its transpose.  lam[n] (mza,mwa) holds dJ/d(new scp) of tracer n
 * on entry and dJ/d(old scp) on return; lam_sct[n] receives dJ/d(sct).
 * rho_old and the registered vmasc / wmasc / rho are those of the forward
 * step.  With the positive-definite limiter (iscal_monot = 2, tracers with
 * pdef set; update_scalar_pd, scalar_transport_rk.F90:1085-1472) the
 * registered var_p / var_t must hold the forward step's inputs: the step is
 * run forward again on the device, the limiter's branches (which faces are
 * scaled, which factor is the minimum) are recorded, and the transpose of
 * the step's Jacobian at that state is applied.  No counterpart in the
 * reference (OLAM has no adjoint); any lpw / lpv (terrain); iscal_monot = 1
 * and tracer diffusion get OLAMGPU_E_UNSUPPORTED. */
int olamgpu_scalar_transport_rk_adjoint(const float* rho_old, float* const* lam, float* const* lam_sct);

/* Replaces prog_wrtv_rk() (prog_wrtv_rk.f90:58-488); istp is mem_ijtabs%istp. */
int olamgpu_prog_wrtv_rk(int istp);

/* Glue of timestep (timestep.f90:430-496, 563-612). */
int olamgpu_tend0(float* rho_old);
int olamgpu_timeavg_momsc(void);

/* ---- halo exchange of the tracer step over ranks ---------------------------
 * When a rank's grid is one part of a decomposed domain (its own columns
 * prognosed, two rings of neighbours held as a halo), scalar_transport_rk
 * exchanges the tracers of the border columns after every RK stage but the
 * last, as omodel/scalar_transport_rk.F90:315-322, 343, 379 does with
 * mpi_post_direct_send/recv_w.  The halo is two rings deep, so the
 * reconstruction planes that OLAM also exchanges (:416-440) are recomputed
 * locally.  The library packs, per neighbour, the columns to send (all
 * levels, all tracers) and calls the exchange hook, which moves them (MPI,
 * NCCL) and fills the receive buffers; the library then writes them into
 * the halo columns.  The step must be the unlimited one (iscal_monot = 0)
 * in a batched transport form; otherwise OLAMGPU_E_UNSUPPORTED. */
typedef struct olamgpu_halo {
  int nnb;                         /* neighbour ranks                           */
  const int* rank;                 /* (nnb) their ranks                          */
  const int* nsend; const int* send_cols;   /* (nnb), concatenated 1-based W    */
  const int* nrecv; const int* recv_cols;   /* indices of this rank's grid      */
  int host_staged;                 /* 1: the hook gets host buffers (the library
                                      copies through pinned memory around it);
                                      0: device buffers, and the hook orders its
                                      transfers on the stream it is given      */
  /* moves sendbuf[i] (sendcount[i] floats) to rank[i] and receives recvbuf[i]
   * (recvcount[i] floats) from it; returns 0 on success */
  int (*exchange)(void* user, int nnb, const int* rank, float* const* sendbuf, const size_t* sendcount,
                  float* const* recvbuf, const size_t* recvcount, void* stream);
  void* user;
  /* the acoustic step's V- and M-point plans, (nnb) counts and concatenated
   * 1-based indices as for the columns; NULL counts: no V / M points move
   * (then prog_wrtv_rk on this rank returns OLAMGPU_E_UNSUPPORTED) */
  const int* nsend_v; const int* send_v; const int* nrecv_v; const int* recv_v;
  const int* nsend_m; const int* send_m; const int* nrecv_m; const int* recv_m;
} olamgpu_halo;

/* Registers the halo plan (NULL: one domain, no exchange).  With the V and
 * M plans, prog_wrtv_rk exchanges as omodel/prog_wrtv_rk.f90:418-472 does
 * after prog_wrt_begs (press, rho, vm*et_rk), prog_v_begs (vmc, vc) and
 * vel_t3d (vxe, vye, vze, wmc, wc, thil), and the damping exchanges its
 * divergence and vorticity planes (omodel/vort_div_damp.f90:150, 208 and
 * the M-point ones); the gradients of ring-1 columns are computed locally
 * instead of exchanged.  olamgpu_timestep also exchanges the tracers and
 * thil after set_scalars_bottom (omodel/timestep.f90:310-314). */
int olamgpu_set_halo(const olamgpu_halo* halo);

/* ---- long-step glue on the device ------------------------------------------
 * set_scalars_bottom (omodel/obnd.f90:7-36): below-ground levels 1..lpw-1
 * of every registered scalar and of thil take the value at lpw, over
 * jtw_prog.  diagvel_t3d (omodel/vel_t3d.f90:7-35): vxe, vye, vze from wc
 * and vc over jtw_prog. */
int olamgpu_set_scalars_bottom(void);
int olamgpu_diagvel_t3d(void);

/* tracer_maxmin (outils/check_nans.F90:164-203): smax[2n] = the largest
 * value and smax[2n+1] = minus the smallest value of scalar n over
 * jtw_prog, levels lpw..mza (-huge(1.) when no point is seen).  Values that
 * are NaN are skipped.  Synchronises the stream. */
int olamgpu_tracer_maxmin(float* smax);

/* compute_mass_sums (outils/check_nans.F90:207-332) and the
 * mass_sum_from_* helpers: sums[0] = sum of rho * volt and sums[1 + i] =
 * sum of rho * volt * scalar[ids[i] - 1] (e.g. rr_w, rr_co2, an added
 * scalar) over jtw_prog, levels lpw..mza, in real(8).  0 <= nsel <= 8.
 * The device adds in a fixed order, so a sum repeats bit for bit from run
 * to run; it differs from a serial CPU sum by round-off only.
 * Synchronises the stream. */
int olamgpu_mass_sums(int nsel, const int* ids, double* sums);

/* One long step of the dynamical core on the device, in timestep.f90's
 * order (:66-319) for the parts this library holds: tend0 (rho_old kept on
 * the device), [comp_horiz_k], nacoust x prog_wrtv_rk, timeavg_momsc,
 * scalar_transport_rk, [tracer_maxmin], set_scalars_bottom, [mass sums].
 * Physics that OLAM runs between them stays on the host and is not called.
 * With OLAMGPU_TS_GRAPH in RESIDENT mode, the first call runs the sequence
 * as it is, and the first call for each of the three tracer-buffer
 * rotations after it records the sequence as a CUDA graph; later calls
 * replay the graph (no host work per kernel, no host round-trip).
 * Registering scalars, eddy inputs, turbulence or a halo, or changing the
 * coherence or transport form, drops the recorded graphs.  The plain
 * transport form, and a rank with a halo exchange (its hook runs on the
 * host between stages), always run without a graph.  The diagnostics of the last
 * call are read with olamgpu_timestep_diag. */
enum {
  OLAMGPU_TS_GRAPH = 1u << 0,     /* record / replay the step as a CUDA graph      */
  OLAMGPU_TS_HORIZ_K = 1u << 1,   /* comp_horiz_k first (eddy inputs registered)   */
  OLAMGPU_TS_MAXMIN = 1u << 2,    /* tracer_maxmin after the tracer step           */
  OLAMGPU_TS_MASS = 1u << 3       /* mass sums of rho and mass_ids at the end      */
};
int olamgpu_timestep(unsigned flags, int nmass, const int* mass_ids);
/* smax as olamgpu_tracer_maxmin (2 x num_scalar), sums as olamgpu_mass_sums
 * (1 + nmass); either may be NULL.  Synchronises the stream and returns a
 * status the device recorded during the step, if any. */
int olamgpu_timestep_diag(float* smax, double* sums);

/* ---- shape of the tiled stage kernel -------------------------------------------
 * The tiled transport kernel runs tiles of up to T neighbouring columns (8,
 * 16 or 32) with G tracers per block (32, 64 or 128; 8-column tiles 128), the levels of a tile
 * swept by KS blocks, the tiles running along the library's own curve over
 * the columns' positions (ord bit 0 clear) or along the caller's jtw_prog
 * (bit 0 set); ord bit 1 selects the paired form (T = 16, G = 128, KS = 1:
 * a warp serves two neighbouring columns and reads each tracer row either
 * of them needs once).  By
 * default an autotuner picks the shape on the first step for a grid and
 * tracer count: every shape the shared memory admits runs the stage on that
 * step's inputs and the fastest is kept (cached per grid, tracer count and
 * order for the process).  olamgpu_set_tile_shape forces a shape (all zero:
 * back to the autotuner).  olamgpu_tile_shape returns the shape in use
 * (shape[4]: T, G, KS, ord) and, for up to max candidates of the last
 * tuning, cand[5 i ..] = T, G, KS, ord, chosen and ms[i] the stage time in
 * milliseconds; it returns the number of candidates (or minus a status).
 * The batching replaces the reference's serial loop over tracers
 * (omodel/scalar_transport_rk.F90:223). */
int olamgpu_set_tile_shape(int T, int G, int KS, int ord);
int olamgpu_tile_shape(int* shape, int max, int* cand, float* ms);

/* ---- surface emission and the checkpointed window adjoint -------------------
 * Surface emission: OLAM's physics adds surface sources to the tracer
 * tendencies between tend0 and scalar_transport_rk (omodel/timestep.f90:
 * 76-254); a long step on the device (olamgpu_timestep) has no host physics
 * in between, so emis[n] (mwa), per registered scalar n (NULL entries: none;
 * a NULL array: off), is added to var_t(lpw(iw), iw) of scalar n right
 * after tend0 of every device long step.  Registering scalars drops it. */
int olamgpu_set_surface_emission(const float* const* emis);

/* A window of nsteps device long steps (olamgpu_timestep's sequence, with
 * `flags` as there: OLAMGPU_TS_GRAPH replays the recorded step) that keeps a
 * checkpoint of the state carried from step to step (rho, press, thil, wc,
 * wmc, vxe/vye/vze, vmc, vc and the damping's saved planes) at the start of
 * every segment of nchk steps, and the state after the last step.  RESIDENT
 * mode, one domain, the tiled transport form, and the options the adjoint
 * runs (see olamgpu_scalar_transport_rk_adjoint).  No counterpart in OLAM:
 * the forward half of the window adjoint. */
int olamgpu_window_forward(int nsteps, int nchk, unsigned flags);

/* Adjoint of the window's tracer transport, with the winds and densities of
 * every step those of the forward: lam[n] (mza, mwa) holds dJ/d(scalar n
 * after the window) on entry and dJ/d(scalar n before it) on return;
 * lam_sct[n] receives dJ/d(var_t of scalar n), the tendency held for every
 * step of the window (so dJ/d(emis[n](iw)) is lam_sct[n](lpw(iw), iw)).
 * Segment by segment from the last, the segment's checkpoint is restored,
 * its steps' dynamics are run again to regenerate the winds and densities
 * each step's transport read (vmasc, wmasc, rho, rho_old), and the one-step
 * adjoint is applied to those steps in reverse order, all on the device.
 * The state after the window is restored at the end.  Device memory: one
 * checkpoint per segment (unless olamgpu_window_memory puts them in host
 * memory) plus the transport inputs of the steps reversed at once (nchk, or
 * olamgpu_window_memory's segment_steps) and the adjoint's buffers (or,
 * lean, none of its own: see olamgpu_window_memory).  No counterpart in
 * OLAM. */
int olamgpu_window_adjoint(float* const* lam, float* const* lam_sct);

/* Where the next window keeps its states, and how its adjoint uses the
 * device.  OLAMGPU_WIN_HOST in `flags`: the checkpoints and the state after
 * the window in page-locked host memory (device copies over PCIe when they
 * are taken and restored), so that the device holds only the model and the
 * adjoint's working set; with nsteps and nchk > 0 the host memory for such
 * a window is page-locked now (after the first long step, whose buffers fix
 * the sizes), else by olamgpu_window_forward.  A request above 70 % of the
 * host's available memory fails with OLAMGPU_E_NOMEM.  With unlimited
 * transport the adjoint is lean when the device has no room for its own
 * buffers: its four lam arrays occupy the tracer buffers (the tracers are in
 * the state after the window) and the per-tracer device arrays are freed
 * during the call and allocated again at its end, so a recorded long step is
 * recorded again on the next olamgpu_timestep; OLAMGPU_WIN_LEAN makes it
 * lean always.  segment_steps > 0: the adjoint holds the transport inputs of
 * at most that many steps at once, running a segment again from its
 * checkpoint for each part of it (more recomputation, less device memory);
 * 0: a whole segment.  Drops a window taken before.  No counterpart in
 * OLAM. */
enum {
  OLAMGPU_WIN_HOST = 1,           /* checkpoints in page-locked host memory          */
  OLAMGPU_WIN_LEAN = 2            /* the lean adjoint even when the device has room  */
};
int olamgpu_window_memory(int flags, int segment_steps, int nsteps, int nchk);

/* Put the state at the start of the last window back on the device (its
 * first checkpoint: the dynamics and the damping's saved planes, and with
 * the limiter the tracers), so that the same window can run again from the
 * same start -- the next iteration of an inversion with new initial
 * tracers or sources.  An unlimited window's checkpoints hold no tracers:
 * send the new ones after the rewind (olamgpu_sync_to_device with
 * OLAMGPU_F_SCALARS).  The window stays valid.  No counterpart in OLAM. */
int olamgpu_window_rewind(void);

/* One explicit RK stage of update_scalar (scalar_transport_rk.F90:389-615:
 * grad_t2d[_quadratic], scalar_v_column, scalar_w_column; every column
 * explicit, no limiter) for ONE tracer, on device arrays the caller owns, in
 * OLAM's (mza, mwa) / (mza, mva) layout: out = the stage's update of scp
 * from scp0, sct, rhos (the stage density, real(4)), vmasc, wmasc with
 * timestep dtr, using the grid and scal_horiz_adv_order given to
 * olamgpu_init.  Columns outside jtw_prog are not written.  No counterpart
 * in the reference: it serves callers that must not allocate device memory
 * during the call (a caller whose memory is fixed up front, or that records
 * its work into a CUDA graph).  The call allocates nothing: its scratch is
 * a fixed 64 MiB device array (gradient planes, V-face values, a zeroed
 * implicit fraction): i2d * mwa * mza + mva * mza + mwa floats must fit in
 * 16 Mi (i2d = 2 for order 2, 5 for order 3), i.e. up to NXP = 74 at order 2
 * and NXP = 58 at order 3 with mza = 61; larger grids get OLAMGPU_E_ARG.
 * The call must be made with the device of olamgpu_init current (else
 * OLAMGPU_E_STATE).  The first call on a device looks the scratch up (make
 * it before any stream capture; olamgpu_finalize forgets it); calls that
 * overlap in time share the scratch and race, so serialise them.  stream: a
 * cudaStream_t, or NULL for the library's stream. */
int olamgpu_update_scalar_noalloc(const float* scp, const float* scp0, const float* sct,
                                  const float* rhos, const float* vmasc, const float* wmasc,
                                  float dtr, float* out, void* stream);

/* Device-side CUDA stream the library launches on (cudaStream_t as void*),
 * so a caller can order its own work against the library's. */
void* olamgpu_stream(void);

/* Number of library kernel launches issued since the last reset. */
unsigned long long olamgpu_launch_count(int reset);

/* Per-kernel device timing (the tracing facility; OLAM itself only prints
 * per-step wall time, omodel/olam_run.f90:990-1032).  While enabled, every
 * library launch is bracketed by CUDA events on the library stream.
 * olamgpu_profile_read synchronises the stream, then fills up to max entries:
 * names (32 bytes each, NUL-terminated), accumulated milliseconds and launch
 * counts; it returns the number of kernels seen, or a negative status. */
int olamgpu_profile(int enable, int reset);
int olamgpu_profile_read(int max, char* names, double* total_ms,
                         unsigned long long* counts);

#ifdef __cplusplus
}
#endif
#endif /* OLAMGPU_H */
