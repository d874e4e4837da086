// Batched RGF: hundreds of independent block-tridiagonal matrices (the energy
// loop A(E_k) = E_k I - H - Sigma(E_k) of a transport calculation) in one
// persistent launch.
//
// The reference inverts one matrix per call (src/sinv/algorithms/rgf/rgf.py:17);
// a single RGF chain is a sequence of dependent block operations and leaves
// most of a B200 idle.  Here every SM runs one CTA that takes whole instances
// from a device work queue (largest cost b^3 n first, so the long instances
// start early) and walks their sweeps with CTA-local barriers only.  The
// chains of different instances overlap across the 148 SMs, which turns the
// latency-bound recursion into a throughput-bound batch.
//
// Each CTA owns a scratch slot in the workspace (the T / side buffers of the
// sweep, sized for the largest instance), reused instance after instance.
#include <algorithm>
#include <vector>

#include "host_util.h"
#include "rgf_sweep.cuh"

namespace sinvb {

template <class T>
struct BatchEntry {
  const T* diag;
  const T* upper;
  const T* lower;
  T* Gd;
  T* Gu;
  T* Gl;
  int n, b;
  int orig;  // index in the caller's descriptor array
  int pad;
};
static_assert(sizeof(BatchEntry<cplx>) == 64, "64-byte entries");

template <class T>
__global__ void __launch_bounds__(kThreads, 1) rgf_batched_kernel(unsigned char* ws) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
  const BatchEntry<T>* entries = reinterpret_cast<const BatchEntry<T>*>(ws + hdr->desc_offset);
  if (blockIdx.x >= hdr->nslots) return;
  unsigned char* slot = ws + hdr->slots_offset + (size_t)blockIdx.x * hdr->slot_bytes;
  const int count = hdr->count;
  const unsigned flags = hdr->flags;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  __shared__ int next;
  __shared__ int inst_status;
  TeamCta team;
  while (true) {
    if (threadIdx.x == 0) {
      next = (int)atomicAdd(&hdr->queue_head, 1u);
      inst_status = 0;
    }
    __syncthreads();
    const int k = next;
    if (k >= count) return;
    const BatchEntry<T> e = entries[k];
    const size_t bb = (size_t)e.b * e.b;
    RgfParams<T> p;
    p.diag = e.diag;
    p.upper = e.upper;
    p.lower = e.lower;
    p.Gd = e.Gd;
    p.Gu = e.Gu;
    p.Gl = e.Gl;
    T* s = reinterpret_cast<T*>(slot);
    p.T0 = s;
    p.T1 = s + bb;
    p.Winv = s + 2 * bb;
    T* xp = p.Winv + invert_side_elems(e.b);
    p.X = save ? e.Gl : xp;
    p.P = save ? e.Gu : xp + (size_t)(e.n - 1) * bb;
    p.hdr = hdr;
    p.status = &inst_status;
    p.n = e.n;
    p.b = e.b;
    p.flags = flags;
    if (e.b <= 32)
      rgf_sweep<T, 32, 32>(team, p, smem);
    else
      rgf_sweep<T, 64, 64>(team, p, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (hdr->inst_status) hdr->inst_status[e.orig] = inst_status;
      if (inst_status) report(&hdr->status, inst_status);
    }
    __syncthreads();  // `next` / `inst_status` are rewritten by the next dequeue
  }
}

constexpr size_t kBatchedSmem = sizeof(GjShared<cplx>) > (size_t)gemm_smem_elems<cplx, 64, 64>() * 16
                                    ? sizeof(GjShared<cplx>)
                                    : (size_t)gemm_smem_elems<cplx, 64, 64>() * 16;

static size_t elem_bytes(int dtype) { return (dtype == SINVB_C128 || dtype == SINVB_C64) ? 16 : 8; }

struct BatchLayout {
  size_t desc_offset, slots_offset, slot_bytes, total;
  unsigned nslots;
};

static unsigned batch_slots() {
  // one CTA per SM: the sweep kernels use up to 232 registers per thread
  return (unsigned)device_sm_count();
}

static BatchLayout batch_layout(const sinvb_batch_desc* d, int count, int dtype, unsigned flags) {
  BatchLayout L{};
  const size_t es = elem_bytes(dtype);
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  size_t slot = 0;
  for (int k = 0; k < count; k++) {
    size_t bb = (size_t)d[k].b * d[k].b;
    size_t s = 2 * bb + invert_side_elems(d[k].b);
    if (!save) s += 2 * (size_t)(d[k].n - 1) * bb;
    slot = std::max(slot, s * es);
  }
  L.nslots = batch_slots();
  L.desc_offset = sizeof(WsHeader);
  L.slots_offset = align_up(L.desc_offset + (size_t)count * sizeof(BatchEntry<cplx>), 256);
  L.slot_bytes = align_up(std::max<size_t>(slot, 256), 256);
  L.total = L.slots_offset + (size_t)L.nslots * L.slot_bytes;
  return L;
}

static int check_batch(const sinvb_batch_desc* d, int count, unsigned flags, const void* ws, size_t ws_bytes,
                       int dtype) {
  if (!d || count < 1 || !ws) return SINVB_EINVAL;
  if ((uintptr_t)ws % 256) return SINVB_EWORKSPACE;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  const size_t align = elem_bytes(dtype);
  for (int k = 0; k < count; k++) {
    const sinvb_batch_desc& e = d[k];
    if (e.n < 1 || e.b < 1 || !e.diag || !e.G_diag) return SINVB_EINVAL;
    if (e.n > 1 && (!e.upper || !e.lower)) return SINVB_EINVAL;
    if (save && e.n > 1 && (!e.G_upper || !e.G_lower)) return SINVB_EINVAL;
    for (const void* q : {e.diag, e.upper, e.lower, (const void*)e.G_diag, (const void*)e.G_upper, (const void*)e.G_lower})
      if (q && (uintptr_t)q % align) return SINVB_EINVAL;
  }
  if (ws_bytes < batch_layout(d, count, dtype, flags).total) return SINVB_EWORKSPACE;
  return check_device();
}

template <class T>
static int launch_batched(void* ws, cudaStream_t stream) {
  auto k = rgf_batched_kernel<T>;
  SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchedSmem));
  // reset status, barrier and queue; the kernel clears per-instance status itself
  SINVB_CUDA(cudaMemsetAsync(ws, 0, 16, stream));
  k<<<batch_slots(), kThreads, kBatchedSmem, stream>>>((unsigned char*)ws);
  SINVB_CUDA(cudaGetLastError());
  return SINVB_OK;
}

template <class T>
static int upload_and_run(const sinvb_batch_desc* d, int count, unsigned flags, void* ws, size_t ws_bytes,
                          int* status, cudaStream_t stream, int dtype) {
  int rc = check_batch(d, count, flags, ws, ws_bytes, dtype);
  if (rc) return rc;
  const BatchLayout L = batch_layout(d, count, dtype, flags);
  std::vector<BatchEntry<T>> entries(count);
  for (int k = 0; k < count; k++) {
    BatchEntry<T>& e = entries[k];
    e.diag = (const T*)d[k].diag;
    e.upper = (const T*)d[k].upper;
    e.lower = (const T*)d[k].lower;
    e.Gd = (T*)d[k].G_diag;
    e.Gu = (T*)d[k].G_upper;
    e.Gl = (T*)d[k].G_lower;
    e.n = d[k].n;
    e.b = d[k].b;
    e.orig = k;
    e.pad = 0;
  }
  // largest first (cost ~ b^3 n): long chains start while short ones fill in
  std::stable_sort(entries.begin(), entries.end(), [](const BatchEntry<T>& x, const BatchEntry<T>& y) {
    return (double)x.b * x.b * x.b * x.n > (double)y.b * y.b * y.b * y.n;
  });
  WsHeader h{};
  h.count = count;
  h.flags = flags;
  h.nslots = L.nslots;
  h.slot_bytes = L.slot_bytes;
  h.desc_offset = L.desc_offset;
  h.slots_offset = L.slots_offset;
  h.inst_status = status;
  unsigned char* w = (unsigned char*)ws;
  SINVB_CUDA(cudaMemcpyAsync(w, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(w + L.desc_offset, entries.data(), count * sizeof(BatchEntry<T>),
                             cudaMemcpyHostToDevice, stream));
  // the pageable copies above are staged before they return; the host arrays may go
  return launch_batched<T>(ws, stream);
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_rgf_batched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype, unsigned flags) {
  if (!descs || count < 1 || dtype < 0 || dtype > 1) return 0;
  return batch_layout(descs, count, dtype, flags).total;
}

int sinvb_rgf_batched_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128);
}

int sinvb_rgf_batched_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64);
}

int sinvb_rgf_batched_rerun_z(void* workspace, sinvb_stream_t stream) {
  if (!workspace || (uintptr_t)workspace % 256) return SINVB_EINVAL;
  int rc = check_device();
  return rc ? rc : launch_batched<cplx>(workspace, (cudaStream_t)stream);
}

int sinvb_rgf_batched_rerun_d(void* workspace, sinvb_stream_t stream) {
  if (!workspace || (uintptr_t)workspace % 256) return SINVB_EINVAL;
  int rc = check_device();
  return rc ? rc : launch_batched<double>(workspace, (cudaStream_t)stream);
}

}  // extern "C"
