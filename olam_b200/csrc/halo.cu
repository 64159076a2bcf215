// halo.cu -- halo exchange of the tracer step between ranks of a decomposed
// domain (omodel/scalar_transport_rk.F90:315-322, 343, 379: the border
// columns of every tracer move after each RK stage but the last).
//   k_halo_pack    the columns to send, all levels and tracers of the batched
//                  layout, one contiguous block per column, neighbour after
//                  neighbour
//   k_halo_unpack  the received blocks into the halo columns
// The transfer itself is the caller's exchange hook (MPI or NCCL), on host
// buffers through pinned memory or on device buffers in stream order.
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

void halo_release() {
  Halo& H = ctx().halo;
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

}  // namespace olamgpu
