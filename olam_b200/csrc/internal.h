// internal.h -- device data structures and helpers of libolamgpu.so.
//
// Device layout.  Grid and state arrays keep OLAM's Fortran layout
// (mza, n) with k contiguous and OLAM's dummy point 1 at index 0, so a host
// array is uploaded with one copy.  Neighbour tables are converted once to
// 0-based indices and padded to 8 entries per W point.  Tracers have two
// device layouts:
//   * per-tracer (mza, mwa) arrays, the reference layout, used by the plain
//     one-kernel-per-pass form and as the staging mirror of host arrays;
//   * the batched layout Q[mwa][mza][ntp] (tracer index fastest, ntp = number
//     of tracers padded to a multiple of 4), used by the fused kernels: the
//     tracers of one (k, iw) cell form one contiguous row, so a warp gathers
//     a neighbour cell for every tracer with one coalesced 16-byte-per-lane
//     load, and every wind, density and table value loaded for that cell is
//     reused across all tracers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/olamgpu.h"

#define OLAMGPU_MAXNB 8  // padded neighbour count per W point (OLAM allows 7)

// Column record of the fused transport kernel (32-bit words; floats stored
// by bit pattern).  Built once at set-up for every prognostic column.
#define COLREC_IW 0     // 0-based W index
#define COLREC_NP 1     // npoly
#define COLREC_KB 2     // lowest prognosed level (0-based)
#define COLREC_FAST 3   // 1: hexagon whose neighbours share the usual 3 cells
#define COLREC_NB 4     // [7] neighbour W points
#define COLREC_EV 11    // [7] faces
#define COLREC_OWN 18   // [7] side index (0/1) of this column on each face
#define COLREC_LPV 25   // [7] lowest level of each face (0-based)
#define COLREC_DV 32    // [7] dirv (float)
#define COLREC_WOWN 39  // [7][7] own-side folded weights over nb (float)
#define COLREC_WU 88    // [6][7] far-side weights: c, nb[n-1], nb[n+1], new0..3 (float)
#define COLREC_NEW 130  // [6][3] far-side further neighbours
#define COLREC_NNEW 148 // [6] count of further neighbours
#define COLREC_WORDS 160

namespace olamgpu {

// ---- error handling ---------------------------------------------------------

void set_error(const std::string& msg);
const std::string& last_error();

#define OG_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      ::olamgpu::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return (e_ == cudaErrorMemoryAllocation) ? OLAMGPU_E_NOMEM : OLAMGPU_E_CUDA; \
    }                                                                        \
  } while (0)

#define OG_CHECK(rc_expr)             \
  do {                                \
    int rc_ = (rc_expr);              \
    if (rc_ != OLAMGPU_OK) return rc_; \
  } while (0)

// counts kernel launches issued by the library (olamgpu_launch_count)
extern unsigned long long g_launches;
#ifdef OLAMGPU_DEBUG_SYNC
// diagnostic builds: wait for every launch and name the first one that failed
void debug_sync(const char* file, int line);
#define OG_LAUNCHED() ::olamgpu::debug_sync(__FILE__, __LINE__)
#else
#define OG_LAUNCHED() (++::olamgpu::g_launches)
#endif

// per-kernel event timing (olamgpu_profile); no-ops while disabled
void prof_begin(const char* name, cudaStream_t s);
void prof_end(cudaStream_t s);
struct ProfScope {
  cudaStream_t s;
  ProfScope(const char* name, cudaStream_t st) : s(st) { prof_begin(name, st); }
  ~ProfScope() { prof_end(s); }
};
#define OG_PROF(name, s) ::olamgpu::ProfScope og_prof_scope_(name, s)

// a device array; a borrowed one is a view of memory another buffer owns
// (release forgets it without freeing)
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool owned = true;
  int alloc(size_t count) {
    if (p && n == count) return OLAMGPU_OK;
    release();
    if (count == 0) return OLAMGPU_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return OLAMGPU_E_NOMEM;
    }
    n = count;
    return OLAMGPU_OK;
  }
  void borrow(T* q, size_t count) {
    release();
    p = q;
    n = count;
    owned = false;
  }
  void release() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    n = 0;
    owned = true;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// page-locked host memory (device copies to and from it run asynchronously)
struct HostBuf {
  char* p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    if (p && n == count) return OLAMGPU_OK;
    release();
    if (count == 0) return OLAMGPU_OK;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), count, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
      return OLAMGPU_E_NOMEM;
    }
    n = count;
    return OLAMGPU_OK;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
};

// ---- device grid ------------------------------------------------------------

struct DevGrid {
  int mza = 0, mwa = 0, mva = 0, mma = 0;
  int nw_prog = 0, nv_wadj = 0, nv_prog = 0, nw_wadj = 0, nm_prog = 0;
  DevBuf<int> jtw_prog, jtv_wadj, jtv_prog, jtw_wadj, jtm_prog;  // 0-based
  int off_wprog = -1, off_vwadj = -1, off_vprog = -1, off_wwadj = -1;   // contiguous tables: first entry (0-based), else -1
  DevBuf<int> npoly;     // (mwa)
  DevBuf<int> w_nb;      // (mwa, 8) 0-based W neighbours, padded with self
  DevBuf<int> w_ev;      // (mwa, 8) 0-based V neighbours, padded with 0
  DevBuf<int> w_im;      // (mwa, 8) 0-based M neighbours
  DevBuf<float> w_dirv;  // (mwa, 8)
  DevBuf<int> v_iw;      // (mva, 2) 0-based
  DevBuf<int> v_im;      // (mva, 2) 0-based
  DevBuf<int> m_iv, m_iw, m_im;  // (mma, 3) 0-based
  DevBuf<int> lpw, lpv, lpm;     // 0-based lowest prognosed level
  DevBuf<int> iwglobe;
  DevBuf<int> w_nonprog;         // W points outside jtw_prog (0-based)
  int n_nonprog = 0;
  // reconstruction coefficients (float, OLAM layouts)
  DevBuf<float> gxc, gyc;        // (mwa, 7)
  DevBuf<float> xy_h, xy_hu;     // (mwa, 7, 5)
  DevBuf<float> dxps, dyps;      // (mva, 2)
  DevBuf<float> xx0_v, xy0_v, yy0_v, xx0_vu, xy0_vu, yy0_vu;  // (mva, 2)
  DevBuf<float> a_w, a_wu;       // Fortran (mza, 2, 2)
  DevBuf<float> volti;           // (mwa, mza)
  // fused-kernel stencil weights: for V face iv and side s the value
  // reconstructed from cell c = iw(s) is
  //   S(c) + sum_n ew[iv][s][n] * (S(w_nb[c][n]) - S(c))
  // (order 2: dxps*gxps_coef + dyps*gyps_coef; order 3 folds the quadratic
  //  terms xx0_v.. with xy_h the same way).  Bounded and unbounded sets.
  DevBuf<float> ew_b, ew_u;      // (mva, 2, 8)
  int ew_order = 0;
  DevBuf<int> colrec;            // (nw_prog, COLREC_WORDS) fused-kernel column records
  // Tile tables of the tiled fused kernel.  Tile t owns tile_T
  // consecutive prognostic columns; its neighbourhood U lists those columns,
  // then the rest of their neighbours, then the rest of those cells'
  // neighbours.  hdr[t] = {u_off, nU, 0, nT}.
  DevBuf<int> tile_hdr;          // (ntiles, 4)
  DevBuf<int> tile_u;            // (sum nU) column of each U entry
  DevBuf<int> tile_tc;           // (ntiles * tile_T, TILE_TCW) tile-cell records
  DevBuf<float> tile_a;          // (ntiles * tile_T, TILE_AW) slot weights
  DevBuf<int> tile_rev;          // (ntiles * tile_T, TILE_NS) transposed slots
  // terrain: slot weights of the level bands of a column below which some
  // term of its faces' reconstructions is under ground (TILE_AW floats per
  // band) and the level at which each band ends
  DevBuf<float> tile_band;
  DevBuf<int> tile_band_lev;
  int tile_T = 0, ntiles = 0, tile_nu_max = 0, tile_order = 0;
  int tile_G = 64, tile_KS = 1;  // the stage kernel's tracers per block and level chunks
  int tile_ord = 0;              // the order the tiles run along (make_tiles)
  bool tile_closed = false;      // every neighbourhood column is prognosed
  DevBuf<int> tile_pair;         // (ntiles * 8, TILE_PT): 16-column tiles as 8 column pairs
  bool tile_paired = false;      // tile_pair holds the tables of the current tiles
  bool tile_pairk = false;       // the stage runs the paired kernel (16 columns, 128 tracers)
  int tile_gen = 0;              // counts the tile builds (records of other tiles are stale)
  // The adjoint's own tiles when the stage kernel runs another width: the
  // reverse stage moves half as many bytes again per row as the forward and
  // is fastest on 32-column tiles (fewer halo rows per column); the same
  // tables as above, built on first use (T = 0: not built).
  struct {
    DevBuf<int> hdr, u, tc, rev;
    int T = 0, ntiles = 0, nu_max = 0, order = 0;
  } adj_tiles;
  std::vector<int> h_lpw;        // host copies used at set-up
};

// Tile-cell record (TILE_TCW words, in 16-byte groups): column, side bits
// (bit n: the cell is side 2, itab_v%iw(2), of face n), np, number of
// slots; the U-row byte offsets (U index * 256) of the TILE_NS slot columns
// -- the cell's neighbours, then their other neighbours; unused slots point
// at the cell itself; V index of each face; dirv of each face (pentagons:
// the sixth face has dirv 0); the cell's first terrain band and its number
// of bands (0 where every term is above ground at every level); pad.
#define TILE_NS 20
#define TILE_TC_IW 0
#define TILE_TC_SIDE 1
#define TILE_TC_NP 2
#define TILE_TC_NS 3
#define TILE_TC_SLOT 4
#define TILE_TC_EV 24
#define TILE_TC_DV 30
#define TILE_TC_BOFF 36
#define TILE_TC_NB 37
#define TILE_TCW 40
// Slot weights (TILE_AW floats per tile cell): A[f][k][j] for face f < 6,
// k = 0 when the cell is the upwind side of face f and 1 when the
// neighbour across it is, slot j < TILE_NS: the weight of S(slot j) - S(cell)
// in (upwind face value) - S(cell).  The order-2 or order-3 reconstruction
// (gradient coefficients times face offsets) is folded into A at set-up.
// With terrain the gradient of a cell leaves out, at level k, the
// neighbours across its faces under ground (k < lpv of the face); a cell's
// levels then fall into bands [lo, hi) with one A each, the last band (all
// terms present) being the table above.
#define TILE_AW (6 * 2 * TILE_NS)
// Transposed slots (TILE_NS ints per tile cell), for the adjoint: for each
// column c that has this cell as its slot j, c's U-row byte offset | j;
// unused entries hold the cell's own offset | TILE_NS.
// Per-(column, level) weight record of a long step (TILE_WR floats, read by
// the stage kernel and the adjoint; layout at k_weights): the slot weights
// W[0..TILE_NS), SW, volti / rhos, 1 / rhos, SW - sum W, the vertical flux's
// coefficients on S(kd-2 .. kd+2) and on S0, wmasc(kd-1), wmasc(kd).
#define TILE_WR 32
// Column pairs of a 16-column tile (the paired stage kernel): columns 2p and
// 2p+1 of tile order form pair p, and a warp serves both from one read of
// each U row either of them needs.  Pair table (TILE_PT words): the number
// of union rows ne (the rows of either column's slots other than the two
// columns' own rows), the slot of column B in column A's slots (-1: none),
// the slot of A in B's, 0, then per union row r | (ja + 1) << 8 | (jb + 1)
// << 16 with ja, jb the row's slot in A's and B's slots (-1: not a slot).
#define TILE_PU 40
#define TILE_PT (4 + TILE_PU)
// Pair record of a level (TILE_PR words, written per step from the two
// columns' weight records): [0] the number of union rows with a non-zero
// weight at this level; per column (A at 4, B at 16, 12 words each): SW,
// volti/rhos, 1/rhos, D, beta_0..4, omega, the weight of the other column's
// own row, 0; from word 28 the rows' U indices as bytes (TILE_PU of them),
// from word 40 their weights (wA, wB) in the same order.
#define TILE_PR 120
#define TILE_PR_A 4
#define TILE_PR_B 16
#define TILE_PR_IDX 28
#define TILE_PR_W 40

// a shape of the tiled stage kernel: columns per tile, tracers per block,
// level chunks per tile
struct TileShape { int T, G, KS, ord; };
// one candidate the autotuner timed (ms per stage launch)
struct TuneRec { int T, G, KS, ord, chosen; float ms; };

struct Tracers {
  int n = 0, ntp = 0;            // count and padded count (multiple of 4)
  std::vector<float*> h_p, h_t;  // registered host arrays
  std::vector<int> pdef, sgsmix;
  std::vector<int> pinned;       // 1 where cudaHostRegister succeeded
  // per-tracer device mirrors (reference layout)
  std::vector<DevBuf<float>> p, t, p_alt;
  // batched layout and rotation buffers
  DevBuf<float> q[3];            // Q layouts: q[cur] holds the tracers
  DevBuf<float> qt;              // tendencies in Q layout
  int qcur = 0;
  bool q_valid = false;          // Q holds the newest values (else per-tracer p)
  DevBuf<int> d_pdef;
};

struct Transport {
  DevBuf<float> vmasc, wmasc, rho_old, wc;  // (mva|mwa, mza)
  DevBuf<double> rho;
  DevBuf<float> rhos;        // (nrk, mwa, mza)
  DevBuf<float> ff;          // (mwa, nrk)
  DevBuf<int> imp_list;      // (nrk, mwa): implicit columns per stage
  DevBuf<int> imp_count;     // (nrk)
  DevBuf<float> imp_b;       // (nrk, mwa, 3, mza): b1, scr1, cji per column slot
  DevBuf<float> cfl_red;     // reduction scratch
  DevBuf<unsigned long long> cfl_loc;
  // scratch for the reference-mirroring passes
  DevBuf<float> gx;          // gradient planes
  DevBuf<float> upv, hiv, sfv;   // V-face arrays
  DevBuf<float> scale, upw;      // W arrays for monot/pd
  DevBuf<float> plain_out[2];    // per-tracer stage outputs of the plain form
  // the pipelined per-call step (transport.cu): copy streams, events of
  // its tracer groups, device tables of the per-tracer arrays
  cudaStream_t s_up = nullptr, s_dn = nullptr;
  std::vector<cudaEvent_t> ev;
  DevBuf<float*> ptab_p, ptab_t;
  DevBuf<int> d_mode;            // per-tracer last-stage mode
  std::vector<int> h_mode;       // what d_mode holds (uploaded when it changes)
  DevBuf<float> wrec;            // (mwa, mza, TILE_WR) weight records of the step
  DevBuf<float> prec;            // (ntiles * 8, mza, TILE_PR) pair records of the step (paired kernel)
  int prec_gen = -1;             // the tile build prec was formed for
  // adjoint (transport_adjoint.cu): lam rotation, lam0, lams in the batched
  // layout, per-tracer planes
  DevBuf<float> adj_l[2], adj_l0, adj_ls, adj_planes;
  DevBuf<float> adj_trec;        // (mwa, mza, 32) transposed records of the step
  DevBuf<float*> adj_ptab, adj_ptab2;
  bool flat = true;              // lpw == lpv == 2 everywhere (fused form requirement)
  DevBuf<float> akhodx;
  DevBuf<int> khtopv;
  bool have_turb = false;
  // surface emission (olamgpu_set_surface_emission): (mwa, ntp), added to
  // the tendencies at lpw after tend0 of each long step
  DevBuf<float> emis;
  bool have_emis = false;
  // tile-shape autotuner (transport_tile.cu): on while no shape is forced;
  // tuned_ntp is the tracer count the current shape was chosen for
  bool autotune = true;
  int tuned_ntp = -1;
  std::vector<TuneRec> tune_log;
};

// Device state and scratch of prog_wrtv_rk (omodel/prog_wrtv_rk.f90).  The
// fields it shares with scalar_transport_rk (rho, vmasc, wmasc, wc, rho_old)
// live in Transport so one device copy serves both.
struct Dyn {
  bool ready = false;            // grid metrics uploaded
  bool uploaded = false;         // RESIDENT mode: host state copied once
  DevBuf<double> press, rho0, rth0;
  DevBuf<float> thil, wmc, vxe, vye, vze, vmc, vc, alpha_press, pwfac, pvfac;
  DevBuf<float> thilt, vmxet, vmyet, vmzet, vmt;       // long-step tendencies
  DevBuf<float> wmc0, vmc0, vmca;
  DevBuf<float> sh_th, sh_vx, sh_vy, sh_vz, sh_vmt;    // *_short
  DevBuf<float> rk_vx, rk_vy, rk_vz;                   // *_rk (thilt_rk stays in registers)
  DevBuf<float> upw, upv;        // 4 fields: thil, vxe, vye, vze
  DevBuf<float> div2d, fdivh, vort2d, fvorth, fvortl, vfact;
  DevBuf<int> lpmmin;
  // prognostic shaved-cell method: lve2 of every W column and the start
  // momentum of its lve2 lowest levels, (mwa, nve2_max, 3); none on grids
  // where no column has a closed face (nve2_max = 0)
  DevBuf<int> lve2;
  DevBuf<float> vm0;
  int nve2_max = 0;
  bool div_first = true, vort_first = true;
  // grid metrics of the dynamics
  DevBuf<float> arv, arw, volwi, volvi, wn, wno2, vn, ecv, gdz_wgtm, gdz_wgtp;
  DevBuf<float> dniv, dniu, dnv, arw0, arm0, zfacit, dzit, xx_yy, xx_yy_m, b20;
  DevBuf<double> volt, zwgt_top8, zwgt_bot8, gdz_wgtm8, gdz_wgtp8;
  DevBuf<float> rayf_cof, dn01d, th01d, vc03d;
  // fluxes_wrtv_monot (dynamics_monot.cu): start values of the limited
  // fields, and scratch shared by the fields in turn
  DevBuf<float> th0, vx0, vy0, vz0;
  DevBuf<float> m_scpt, m_gx, m_hiw, m_sfw, m_hiv, m_sfv, m_sin, m_sout;
  // eddy diffusion (dynamics_eddy.cu): the registered host arrays and their
  // device copies; hk_on_device: comp_horiz_k's outputs were last written
  // on the device (host copies stale until a sync to the host)
  bool eddy_on = false, hk_on_device = false;
  olamgpu_eddy heddy{};
  DevBuf<float> e_vkm, e_vkh, e_agamma, e_theta, e_tair, e_akm_sfc, e_sfluxt, e_akmodx, e_akhodx;
  DevBuf<float> e_dzim, e_dztbi, e_akmin, e_rayf;
  DevBuf<int> e_kmtop, e_khtop, e_kpblh, e_kmtopv, e_khtopv, e_lsw, e_mrlw, e_mrlv, e_idiffk;
};

// one recorded long step (timestep.cu): the graph of the sequence for the
// tracer buffer rotation it started from
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  unsigned flags = 0;
  int nmass = 0;
  int ids[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int qcur_after = 0;
  unsigned long long launches = 0;   // library kernels in the graph
};

struct Glue {
  DevBuf<unsigned> keys;     // tracer_maxmin: (2, num_scalar) ordered keys
  DevBuf<double> part;       // mass sums: per-block partial sums
  DevBuf<double> sums;       // mass sums: (1 + nsel)
  StepGraph g[3];            // indexed by the tracer rotation at the step's start
  bool eager_done = false;   // a step ran without a graph since the last drop
  unsigned last_flags = 0;
  int last_nmass = 0, last_ntr = 0;
};

// halo exchange of the tracer step (halo.cu)
// a point kind's exchange lists (W columns, V or M points)
struct HaloList {
  std::vector<int> nsend, nrecv;     // per neighbour
  size_t ns = 0, nr = 0;
  DevBuf<int> send, recv;            // 0-based indices, neighbour after neighbour
};

struct Halo {
  bool on = false, host_staged = false, dyn = false;
  std::vector<int> rank, nsend, nrecv;
  size_t ns = 0, nr = 0;             // columns sent / received in all
  DevBuf<int> send_cols, recv_cols;  // 0-based W indices, neighbour after neighbour
  HaloList lv, lm;                   // V and M points (the acoustic step)
  DevBuf<int> wsend, wrecv;          // copies of the column lists for field exchanges
  DevBuf<float> sendbuf, recvbuf;    // packed columns (all levels and tracers)
  float* hsend = nullptr;            // pinned host copies (host-staged hook)
  float* hrecv = nullptr;
  size_t hcap = 0;
  int (*fn)(void*, int, const int*, float* const*, const size_t*, float* const*, const size_t*, void*) = nullptr;
  void* user = nullptr;
};

// checkpointed window of long steps (window.cu): the state at the start of
// every segment of nchk steps, the state after the window, and the step
// inputs of the part of a segment being reversed
struct StateBlob {                   // one saved state, on the device or in page-locked host memory
  DevBuf<char> dev;
  int slot = -1;                     // its entry of WindowMem::pool when on the host
};

struct Window {
  bool valid = false;
  bool tracers = false;              // checkpoints hold the tracers (limited transport)
  bool lean_ok = false;              // unlimited transport: the adjoint may borrow the tracer buffers
  bool lean = false;                 // this adjoint call does
  int nsteps = 0, nchk = 0;
  unsigned flags = 0;
  std::vector<StateBlob> chk;
  std::vector<int> chk_qcur;
  std::vector<char> chk_div_first, chk_vort_first;
  StateBlob fin;
  int fin_qcur = 0;
  bool fin_div_first = false, fin_vort_first = false;
  DevBuf<char> seg;                  // (steps held at once) x the inputs of one step
  DevBuf<float> lsacc;               // adjoint of the tendencies, summed over the steps
  DevBuf<float*> ptab;
  DevBuf<float> planes;
};

// where the next window keeps its states (olamgpu_window_memory); kept
// across windows so that the host memory is page-locked once
struct WindowMem {
  bool host = false;                 // checkpoints and the final state in page-locked host memory
  bool lean_always = false;          // the lean adjoint even when the device has room for its own buffers
  int seg_steps = 0;                 // steps whose transport inputs the adjoint holds at once (0: nchk)
  std::vector<HostBuf> pool;         // the final state, then checkpoints 0 .. nseg-1
};

struct Context {
  bool initialised = false;
  int device = -1;
  cudaStream_t stream = nullptr;
  olamgpu_opts opts{};
  olamgpu_grid hgrid{};      // host pointers as given (valid while OLAM runs)
  olamgpu_state hstate{};
  bool have_state = false;
  int coherence = OLAMGPU_SYNC_EACH_CALL;
  int form = OLAMGPU_TRANSPORT_FUSED;
  DevGrid g;
  Tracers tr;
  Transport tp;
  Dyn dy;
  Glue glue;
  Halo halo;
  Window win;
  WindowMem winmem;
  DevBuf<int> status;        // device status word (bounds/NaN flags)
};

Context& ctx();

// set-up helpers (setup.cu)
int upload_grid(const olamgpu_grid* g, DevGrid& d, cudaStream_t s);
int build_fused_weights(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s);
// host tile tables (layouts above); T == 0 when the grid is left to the column kernel
struct TileHost {
  int T = 0, ntiles = 0, nu_max = 0, order = 0;
  std::vector<int> hdr, ulist, tc, rev;
  std::vector<float> a;
  std::vector<float> band;       // terrain bands (TILE_AW floats each)
  std::vector<int> band_lev;     // the device level at which each band ends
  std::vector<int> pair;         // 16-column tiles: the column pairs' union tables (TILE_PT words each)
};
// T: tile width (0: the widest whose neighbourhoods fit two blocks per SM)
// nu_cap: the largest neighbourhood of a tile (0: where two blocks of 64
// tracers fit an SM)
// ord: the order tiles run along -- 0 the library's own curve over the
// columns' positions, 1 the caller's jtw_prog
void make_tiles(const olamgpu_grid* g, int order, TileHost& th, int T = 0, int nu_cap = 0, int ord = 0);
int build_tiles(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s, int T = 0, int ord = 0);
int build_adj_tiles(const olamgpu_grid* g, DevGrid& d, int order, cudaStream_t s);
// dynamic shared memory of the stage kernel: T columns, nu_max rows of rb bytes
size_t tile_smem_bytes(int T, int nu_max, int rb);

// dynamics entry points (dynamics.cu)
int dyn_setup(const olamgpu_grid* g, const olamgpu_opts* o, cudaStream_t s);
int dyn_prog_wrtv_rk(int istp);
int dyn_tend0(float* rho_old_host);
int dyn_timeavg_momsc();
int dyn_state_to_device(unsigned mask, cudaStream_t s);
int dyn_state_to_host(unsigned mask, cudaStream_t s);
void dyn_release();
// the flux-corrected face values of field 0 (thil) .. 3 (vze) on the last
// RK stage (dynamics_monot.cu): scp, its start value, its *_short tendency
int dyn_eddy_set(const olamgpu_eddy* e);
int dyn_eddy_to_device(cudaStream_t s);
int dyn_eddy_to_host(cudaStream_t s);
int dyn_comp_horiz_k();
// the eddy-diffusion column terms on sh_th / sh_vx / sh_vy / sh_vz after
// k_setup_w; with rayleigh, also the Rayleigh term on thil (which k_setup_w
// then leaves out, so that the terms add in the reference's order)
int dyn_eddy_columns(Context& C, bool rayleigh, cudaStream_t s);
void dyn_eddy_release();
int dyn_monot_faces(Context& C, int field, const float* scp, const float* scp0, const float* sct, float dts,
                    int ord, cudaStream_t s);

// reads the device status record (call with the library stream idle); a
// kernel that found an inconsistent table reports it here
int check_device_status();

// transport entry points (transport.cu)
int transport_run(const float* rho_old_host, olamgpu_cfl_diag* diag);
void transport_release_pipeline();
// halo exchange (halo.cu)
int halo_set(const olamgpu_halo* h);
int halo_exchange(Context& C, float* Q, int ntp, cudaStream_t s);
// fields of mza elements per point (4 or 8 bytes each) of one point kind
enum { HALO_W = 0, HALO_V = 1, HALO_M = 2 };
struct HField { void* p; int esize; };
int halo_exchange_fields(Context& C, int kind, const HField* f, int nf, cudaStream_t s);
void halo_release();
// long-step glue and the recorded step (timestep.cu)
int glue_set_scalars_bottom();
int glue_tracer_maxmin(float* smax);
int glue_mass_sums(int nsel, const int* ids, double* sums);
int glue_timestep(unsigned flags, int nmass, const int* ids);
int glue_timestep_diag(float* smax, double* sums);
void glue_drop_graphs();
void glue_release();
int dyn_diagvel_t3d();
// profiling off while a stream is being recorded into a graph
void prof_suspend(bool on);
// adjoint of one unlimited step (transport_adjoint.cu)
int transport_adjoint_run(const float* rho_old_host, float* const* lam, float* const* lam_sct);
// the options and tables the adjoint needs (OLAMGPU_OK when it can run)
int adjoint_ready(Context& C);
// the reverse step on the device, at the step inputs held in tp (winds,
// densities, rho_old): tp.adj_l[0] holds the adjoint of the step's output
// in the batched layout; on return tp.adj_l[nrk & 1] holds the adjoint of
// its input and tp.adj_ls that of the tendencies
// ls_acc: the adjoint of the tendencies accumulates into adj_ls (a window
// sums it over its steps) instead of starting from zero
int adjoint_core(Context& C, const float* rho_old_host, bool ls_acc = false);
// the long step's device sequence (timestep.cu); without the transport:
// the dynamics and the glue of thil only
int glue_run_sequence(Context& C, unsigned flags, bool with_transport);
// checkpointed window of long steps (window.cu)
int window_forward(int nsteps, int nchk, unsigned flags);
int window_adjoint(float* const* lam, float* const* lam_sct);
void window_release();
int window_memory(int flags, int segment_steps, int nsteps, int nchk);
int window_rewind();
void window_memory_release();
// surface emission of the registered tracers (timestep.cu)
int emission_set(const float* const* emis);
void launch_emission(Context& C, cudaStream_t s);
// the emission's table of per-tracer tendency arrays, after those moved
int emission_repoint(Context& C, cudaStream_t s);
// forgets the scratch address of olamgpu_update_scalar_noalloc (finalize)
void noalloc_forget();
int tracers_to_device(cudaStream_t s);   // host -> per-tracer mirrors (-> Q)
int tracers_to_host(cudaStream_t s);     // (Q ->) per-tracer mirrors -> host
int ensure_q(cudaStream_t s);            // per-tracer mirrors -> Q if needed
int ensure_plain(cudaStream_t s);        // Q -> per-tracer mirrors if needed

template <class T>
int upload(DevBuf<T>& b, const T* h, size_t n, cudaStream_t s) {
  OG_CHECK(b.alloc(n));
  if (n) OG_CUDA(cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return OLAMGPU_OK;
}

inline unsigned int cdiv(size_t a, size_t b) { return (unsigned int)((a + b - 1) / b); }

}  // namespace olamgpu
