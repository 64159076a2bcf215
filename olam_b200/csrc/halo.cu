// halo.cu -- halo exchange of the tracer step between ranks of a decomposed
// domain (omodel/scalar_transport_rk.F90:315-322, 343, 379: the border
// columns of every tracer move after each RK stage but the last).
//   k_halo_pack    the columns to send, all levels and tracers of the batched
//                  layout, one contiguous block per column, neighbour after
//                  neighbour
//   k_halo_unpack  the received blocks into the halo columns
// The transfer itself is the caller's exchange hook (MPI or NCCL), on host
// buffers through pinned memory or on device buffers in stream order.
#include <algorithm>
#include <vector>

#include "transport_kernels.cuh"

namespace olamgpu {

__global__ void k_halo_pack(const float4* __restrict__ q, const int* __restrict__ cols, size_t ncols, size_t per4,
                            float4* __restrict__ buf) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncols * per4) return;
  const size_t c = i / per4, o = i - c * per4;
  buf[i] = q[(size_t)cols[c] * per4 + o];
}

__global__ void k_halo_unpack(float4* __restrict__ q, const int* __restrict__ cols, size_t ncols, size_t per4,
                              const float4* __restrict__ buf) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncols * per4) return;
  const size_t c = i / per4, o = i - c * per4;
  q[(size_t)cols[c] * per4 + o] = buf[i];
}

// fields of one point kind: word w of point i of the packed buffer is word
// (w - off[k]) of field k's column at point idx[i]; off[k] prefix sums of the
// fields' words per point (mza or 2 mza)
struct FieldPack {
  const unsigned* src[8];
  unsigned* dst[8];
  int off[9];
  int nf;
};

__global__ void k_field_pack(FieldPack F, const int* __restrict__ idx, size_t npts, unsigned* __restrict__ buf) {
  const size_t per = (size_t)F.off[F.nf];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts * per) return;
  const size_t pt = i / per;
  const int w = (int)(i - pt * per);
  int k = 0;
  while (k + 1 < F.nf && w >= F.off[k + 1]) ++k;
  const int len = F.off[k + 1] - F.off[k];
  buf[i] = F.src[k][(size_t)idx[pt] * len + (w - F.off[k])];
}

__global__ void k_field_unpack(FieldPack F, const int* __restrict__ idx, size_t npts,
                               const unsigned* __restrict__ buf) {
  const size_t per = (size_t)F.off[F.nf];
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts * per) return;
  const size_t pt = i / per;
  const int w = (int)(i - pt * per);
  int k = 0;
  while (k + 1 < F.nf && w >= F.off[k + 1]) ++k;
  const int len = F.off[k + 1] - F.off[k];
  F.dst[k][(size_t)idx[pt] * len + (w - F.off[k])] = buf[i];
}

static void list_release(HaloList& L) {
  L.send.release();
  L.recv.release();
  L = HaloList();
}

void halo_release() {
  Halo& H = ctx().halo;
  list_release(H.lv);
  list_release(H.lm);
  H.wsend.release();
  H.wrecv.release();
  H.send_cols.release();
  H.recv_cols.release();
  H.sendbuf.release();
  H.recvbuf.release();
  if (H.hsend) cudaFreeHost(H.hsend);
  if (H.hrecv) cudaFreeHost(H.hrecv);
  H = Halo();
}

int halo_set(const olamgpu_halo* h) {
  Context& C = ctx();
  if (!C.initialised) { set_error("olamgpu_init has not been called"); return OLAMGPU_E_STATE; }
  halo_release();
  if (!h) return OLAMGPU_OK;
  if (h->nnb < 0 || (h->nnb > 0 && (!h->rank || !h->nsend || !h->nrecv || !h->exchange))) {
    set_error("olamgpu_halo: nnb, rank, nsend, nrecv and exchange must be given");
    return OLAMGPU_E_ARG;
  }
  Halo& H = C.halo;
  const int mwa = C.g.mwa;
  std::vector<int> sc, rc;
  for (int i = 0; i < h->nnb; ++i) {
    if (h->nsend[i] < 0 || h->nrecv[i] < 0) { set_error("olamgpu_halo: negative count"); return OLAMGPU_E_ARG; }
    H.rank.push_back(h->rank[i]);
    H.nsend.push_back(h->nsend[i]);
    H.nrecv.push_back(h->nrecv[i]);
  }
  size_t ns = 0, nr = 0;
  for (int i = 0; i < h->nnb; ++i) { ns += h->nsend[i]; nr += h->nrecv[i]; }
  if ((ns && !h->send_cols) || (nr && !h->recv_cols)) { set_error("olamgpu_halo: column lists missing"); return OLAMGPU_E_ARG; }
  // 1-based W indices of this rank's grid -> 0-based, checked
  std::vector<char> isprog(mwa, 0);
  for (int j = 0; j < C.hgrid.nw_prog; ++j) isprog[C.hgrid.jtw_prog[j] - 1] = 1;
  for (size_t i = 0; i < ns; ++i) {
    const int c = h->send_cols[i] - 1;
    if (c < 1 || c >= mwa || !isprog[c]) {
      set_error("olamgpu_halo: send column " + std::to_string(c + 1) + " is not a prognosed column of this rank");
      return OLAMGPU_E_ARG;
    }
    sc.push_back(c);
  }
  for (size_t i = 0; i < nr; ++i) {
    const int c = h->recv_cols[i] - 1;
    if (c < 1 || c >= mwa || isprog[c]) {
      set_error("olamgpu_halo: receive column " + std::to_string(c + 1) + " is not a halo column of this rank");
      return OLAMGPU_E_ARG;
    }
    rc.push_back(c);
  }
  OG_CHECK(upload(H.send_cols, sc.data(), sc.size(), C.stream));
  OG_CHECK(upload(H.recv_cols, rc.data(), rc.size(), C.stream));
  OG_CHECK(upload(H.wsend, sc.data(), sc.size(), C.stream));
  OG_CHECK(upload(H.wrecv, rc.data(), rc.size(), C.stream));
  // V and M plans of the acoustic step
  auto take = [&](HaloList& L, const int* ns_, const int* sidx, const int* nr_, const int* ridx, int maxv,
                  const char* what) -> int {
    std::vector<int> a, b;
    size_t ts = 0, trr = 0;
    for (int i = 0; i < h->nnb; ++i) {
      if (ns_[i] < 0 || nr_[i] < 0) { set_error(std::string("olamgpu_halo: negative ") + what + " count"); return OLAMGPU_E_ARG; }
      L.nsend.push_back(ns_[i]);
      L.nrecv.push_back(nr_[i]);
      ts += ns_[i];
      trr += nr_[i];
    }
    if ((ts && !sidx) || (trr && !ridx)) { set_error(std::string("olamgpu_halo: ") + what + " lists missing"); return OLAMGPU_E_ARG; }
    for (size_t i = 0; i < ts; ++i) {
      if (sidx[i] < 2 || sidx[i] > maxv) { set_error(std::string("olamgpu_halo: ") + what + " index out of range"); return OLAMGPU_E_ARG; }
      a.push_back(sidx[i] - 1);
    }
    for (size_t i = 0; i < trr; ++i) {
      if (ridx[i] < 2 || ridx[i] > maxv) { set_error(std::string("olamgpu_halo: ") + what + " index out of range"); return OLAMGPU_E_ARG; }
      b.push_back(ridx[i] - 1);
    }
    L.ns = ts;
    L.nr = trr;
    OG_CHECK(upload(L.send, a.data(), a.size(), C.stream));
    OG_CHECK(upload(L.recv, b.data(), b.size(), C.stream));
    return OLAMGPU_OK;
  };
  H.dyn = h->nsend_v && h->nrecv_v && h->nsend_m && h->nrecv_m;
  if (H.dyn) {
    OG_CHECK(take(H.lv, h->nsend_v, h->send_v, h->nrecv_v, h->recv_v, C.g.mva, "V"));
    OG_CHECK(take(H.lm, h->nsend_m, h->send_m, h->nrecv_m, h->recv_m, C.g.mma, "M"));
  }
  OG_CUDA(cudaStreamSynchronize(C.stream));
  H.ns = ns;
  H.nr = nr;
  H.host_staged = h->host_staged != 0;
  H.fn = h->exchange;
  H.user = h->user;
  H.on = h->nnb > 0;
  return OLAMGPU_OK;
}

// the border columns of Q (the batched layout, ntp tracers) after a stage
int halo_exchange(Context& C, float* Q, int ntp, cudaStream_t s) {
  Halo& H = C.halo;
  if (!H.on) return OLAMGPU_OK;
  const size_t per = (size_t)C.g.mza * ntp, per4 = per / 4;   // ntp is a multiple of 4
  OG_CHECK(H.sendbuf.n >= H.ns * per ? OLAMGPU_OK : H.sendbuf.alloc(std::max<size_t>(H.ns * per, 4)));
  OG_CHECK(H.recvbuf.n >= H.nr * per ? OLAMGPU_OK : H.recvbuf.alloc(std::max<size_t>(H.nr * per, 4)));
  if (H.ns) {
    k_halo_pack<<<cdiv(H.ns * per4, 256), 256, 0, s>>>(reinterpret_cast<const float4*>(Q), H.send_cols.p, H.ns, per4,
                                                       reinterpret_cast<float4*>(H.sendbuf.p));
    OG_LAUNCHED();
  }
  const int nnb = (int)H.rank.size();
  std::vector<float*> sb(nnb), rb(nnb);
  std::vector<size_t> scount(nnb), rcount(nnb);
  float* sbase = H.sendbuf.p;
  float* rbase = H.recvbuf.p;
  if (H.host_staged) {
    if (H.hcap < std::max(H.ns, H.nr) * per) {
      if (H.hsend) cudaFreeHost(H.hsend);
      if (H.hrecv) cudaFreeHost(H.hrecv);
      H.hsend = H.hrecv = nullptr;
      H.hcap = 0;
      const size_t cap = std::max<size_t>(std::max(H.ns, H.nr) * per, 4);
      OG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&H.hsend), cap * sizeof(float), cudaHostAllocDefault));
      OG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&H.hrecv), cap * sizeof(float), cudaHostAllocDefault));
      H.hcap = cap;
    }
    if (H.ns) OG_CUDA(cudaMemcpyAsync(H.hsend, H.sendbuf.p, H.ns * per * sizeof(float), cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaStreamSynchronize(s));
    sbase = H.hsend;
    rbase = H.hrecv;
  }
  size_t so = 0, ro = 0;
  for (int i = 0; i < nnb; ++i) {
    scount[i] = (size_t)H.nsend[i] * per;
    rcount[i] = (size_t)H.nrecv[i] * per;
    sb[i] = sbase + so;
    rb[i] = rbase + ro;
    so += scount[i];
    ro += rcount[i];
  }
  const int rc = H.fn(H.user, nnb, H.rank.data(), sb.data(), scount.data(), rb.data(), rcount.data(), (void*)s);
  if (rc != 0) {
    set_error("the halo exchange hook returned " + std::to_string(rc));
    return OLAMGPU_E_CUDA;
  }
  if (H.host_staged && H.nr)
    OG_CUDA(cudaMemcpyAsync(H.recvbuf.p, H.hrecv, H.nr * per * sizeof(float), cudaMemcpyHostToDevice, s));
  if (H.nr) {
    k_halo_unpack<<<cdiv(H.nr * per4, 256), 256, 0, s>>>(reinterpret_cast<float4*>(Q), H.recv_cols.p, H.nr, per4,
                                                         reinterpret_cast<const float4*>(H.recvbuf.p));
    OG_LAUNCHED();
  }
  if (H.host_staged) OG_CUDA(cudaStreamSynchronize(s));   // the pinned buffers are reused next stage
  return OLAMGPU_OK;
}

// the host side of one exchange: packed send buffers (device) -> hook ->
// packed receive buffers (device), through pinned memory when host-staged
static int run_hook(Halo& H, const std::vector<int>& nsend, const std::vector<int>& nrecv, size_t per,
                    float* dsend, float* drecv, size_t ns, size_t nr, cudaStream_t s) {
  const int nnb = (int)H.rank.size();
  std::vector<float*> sb(nnb), rb(nnb);
  std::vector<size_t> scount(nnb), rcount(nnb);
  float* sbase = dsend;
  float* rbase = drecv;
  if (H.host_staged) {
    const size_t need = std::max(ns, nr) * per;
    if (H.hcap < need) {
      if (H.hsend) cudaFreeHost(H.hsend);
      if (H.hrecv) cudaFreeHost(H.hrecv);
      H.hsend = H.hrecv = nullptr;
      H.hcap = 0;
      const size_t cap = std::max<size_t>(need, 4);
      OG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&H.hsend), cap * sizeof(float), cudaHostAllocDefault));
      OG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&H.hrecv), cap * sizeof(float), cudaHostAllocDefault));
      H.hcap = cap;
    }
    if (ns) OG_CUDA(cudaMemcpyAsync(H.hsend, dsend, ns * per * sizeof(float), cudaMemcpyDeviceToHost, s));
    OG_CUDA(cudaStreamSynchronize(s));
    sbase = H.hsend;
    rbase = H.hrecv;
  }
  size_t so = 0, ro = 0;
  for (int i = 0; i < nnb; ++i) {
    scount[i] = (size_t)nsend[i] * per;
    rcount[i] = (size_t)nrecv[i] * per;
    sb[i] = sbase + so;
    rb[i] = rbase + ro;
    so += scount[i];
    ro += rcount[i];
  }
  const int rc = H.fn(H.user, nnb, H.rank.data(), sb.data(), scount.data(), rb.data(), rcount.data(), (void*)s);
  if (rc != 0) {
    set_error("the halo exchange hook returned " + std::to_string(rc));
    return OLAMGPU_E_CUDA;
  }
  if (H.host_staged && nr) OG_CUDA(cudaMemcpyAsync(drecv, H.hrecv, nr * per * sizeof(float), cudaMemcpyHostToDevice, s));
  return OLAMGPU_OK;
}

int halo_exchange_fields(Context& C, int kind, const HField* f, int nf, cudaStream_t s) {
  Halo& H = C.halo;
  if (!H.on || !H.dyn) return OLAMGPU_OK;
  if (nf < 1 || nf > 8) { set_error("halo field exchange: 1..8 fields"); return OLAMGPU_E_ARG; }
  const std::vector<int>& nsend = kind == HALO_W ? H.nsend : (kind == HALO_V ? H.lv.nsend : H.lm.nsend);
  const std::vector<int>& nrecv = kind == HALO_W ? H.nrecv : (kind == HALO_V ? H.lv.nrecv : H.lm.nrecv);
  const size_t ns = kind == HALO_W ? H.ns : (kind == HALO_V ? H.lv.ns : H.lm.ns);
  const size_t nr = kind == HALO_W ? H.nr : (kind == HALO_V ? H.lv.nr : H.lm.nr);
  const int* sidx = kind == HALO_W ? H.wsend.p : (kind == HALO_V ? H.lv.send.p : H.lm.send.p);
  const int* ridx = kind == HALO_W ? H.wrecv.p : (kind == HALO_V ? H.lv.recv.p : H.lm.recv.p);
  FieldPack F{};
  F.nf = nf;
  F.off[0] = 0;
  for (int k = 0; k < nf; ++k) {
    F.src[k] = static_cast<const unsigned*>(f[k].p);
    F.dst[k] = static_cast<unsigned*>(f[k].p);
    F.off[k + 1] = F.off[k] + C.g.mza * (f[k].esize / 4);
  }
  const size_t per = (size_t)F.off[nf];
  OG_CHECK(H.sendbuf.n >= ns * per ? OLAMGPU_OK : H.sendbuf.alloc(std::max<size_t>(ns * per, 4)));
  OG_CHECK(H.recvbuf.n >= nr * per ? OLAMGPU_OK : H.recvbuf.alloc(std::max<size_t>(nr * per, 4)));
  if (ns) {
    k_field_pack<<<cdiv(ns * per, 256), 256, 0, s>>>(F, sidx, ns, reinterpret_cast<unsigned*>(H.sendbuf.p));
    OG_LAUNCHED();
  }
  OG_CHECK(run_hook(H, nsend, nrecv, per, H.sendbuf.p, H.recvbuf.p, ns, nr, s));
  if (nr) {
    k_field_unpack<<<cdiv(nr * per, 256), 256, 0, s>>>(F, ridx, nr, reinterpret_cast<const unsigned*>(H.recvbuf.p));
    OG_LAUNCHED();
  }
  if (H.host_staged) OG_CUDA(cudaStreamSynchronize(s));   // the pinned buffers are reused
  return OLAMGPU_OK;
}

}  // namespace olamgpu
