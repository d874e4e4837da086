// Adjoint of the RGF selected inversion: kernels and C-ABI entry points.
// The device code (adjoint.cuh) reverses both sweeps of
// src/sinv/algorithms/rgf/rgf.py:44-62 with sqrt(n) checkpoints.
#include <algorithm>
#include <cmath>
#include <vector>

#include "adjoint.cuh"
#include "batch_queue.cuh"
#include "host_util.h"

namespace sinvb {

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) adjoint_cta_kernel(AdjParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamCta team;
  rgf_adjoint<T, BM, BN>(team, p, reinterpret_cast<T*>(smem_raw));
}

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) adjoint_grid_kernel(AdjParams<T> p, WsHeader* hdr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamDyn team{&hdr->barrier_count, &hdr->status, (int)blockIdx.x, (int)gridDim.x, 0u};
  rgf_adjoint<T, BM, BN>(team, p, reinterpret_cast<T*>(smem_raw));
}

// Checkpoint spacing c = ceil(sqrt(n)) and the number of checkpoints.
static int ckpt_every(int n) {
  int c = (int)std::ceil(std::sqrt((double)n));
  return c < 1 ? 1 : c;
}

struct AdjLayout {
  size_t seg_g, seg_P, tmp, side, total;
};

static AdjLayout adj_layout(int n, int b, int dtype) {
  const size_t es = dtype == SINVB_C128 ? 16 : 8;
  const size_t bb = (size_t)b * b;
  const int c = ckpt_every(n);
  AdjLayout L{};
  size_t off = sizeof(WsHeader);
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  L.seg_g = take(c * bb * es);
  L.seg_P = take(c * bb * es);
  L.tmp = take(9 * bb * es);
  L.side = take(invert_side_elems(b) * es);
  L.total = off;
  return L;
}

template <class T, int BM, int BN>
static int launch_adj(const AdjParams<T>& p, bool grid, WsHeader* hdr, cudaStream_t stream) {
  constexpr size_t g = (size_t)gemm_smem_elems<T, BM, BN>() * sizeof(T);
  constexpr size_t smem = g > sizeof(GjShared<T>) ? g : sizeof(GjShared<T>);
  if (!grid) {
    auto k = adjoint_cta_kernel<T, BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<1, kThreads, smem, stream>>>(p);
    SINVB_CUDA(cudaGetLastError());
  } else {
    auto k = adjoint_grid_kernel<T, BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void* args[] = {(void*)&p, (void*)&hdr};
    SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(device_sm_count()), dim3(kThreads), args, smem,
                                           stream));
  }
  return SINVB_OK;
}

template <class T>
static int run_adjoint(const void* diag, const void* upper, const void* lower, const void* Gd, const void* Gu,
                       const void* Gl, const void* bGd, const void* bGu, const void* bGl, const void* ckpt, int every,
                       int n, int b, unsigned flags, void* aD, void* aU, void* aL, void* ws, size_t ws_bytes,
                       cudaStream_t stream, int dtype) {
  if (n < 1 || b < 1 || !diag || !Gd || !bGd || !aD || !ws) return SINVB_EINVAL;
  if (n > 1 && (!upper || !lower || !Gu || !Gl || !aU || !aL)) return SINVB_EINVAL;
  if (every != ckpt_every(n)) return SINVB_EINVAL;
  if ((n - 1) / every >= 1 && !ckpt) return SINVB_EINVAL;
  if ((uintptr_t)ws % 256) return SINVB_EWORKSPACE;
  const AdjLayout L = adj_layout(n, b, dtype);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* w = (unsigned char*)ws;
  AdjParams<T> p;
  p.diag = (const T*)diag;
  p.upper = (const T*)upper;
  p.lower = (const T*)lower;
  p.Gd = (const T*)Gd;
  p.Gu = (const T*)Gu;
  p.Gl = (const T*)Gl;
  p.bGd = (const T*)bGd;
  p.bGu = (const T*)bGu;
  p.bGl = (const T*)bGl;
  p.aD = (T*)aD;
  p.aU = (T*)aU;
  p.aL = (T*)aL;
  p.ckpt = (const T*)ckpt;
  p.seg_g = (T*)(w + L.seg_g);
  p.seg_P = (T*)(w + L.seg_P);
  p.tmp = (T*)(w + L.tmp);
  p.side = (T*)(w + L.side);
  WsHeader* hdr = (WsHeader*)w;
  p.status = &hdr->status;
  p.n = n;
  p.b = b;
  p.c = every;
  p.flags = flags;
  SINVB_CUDA(cudaMemsetAsync(w, 0, sizeof(WsHeader), stream));
  const bool grid = (flags & SINVB_FORCE_GRID) || (!(flags & SINVB_FORCE_CTA) && b > 48);
  if (b <= 32 || grid) return launch_adj<T, 32, 32>(p, grid, hdr, stream);
  return launch_adj<T, 64, 64>(p, grid, hdr, stream);
}

// ---- batched adjoint: many instances (the energy loop) in one persistent launch

// One instance in the workspace (queue order).
template <class T>
struct AdjEntry {
  const T* diag;
  const T* upper;
  const T* lower;
  const T* Gd;
  const T* Gu;
  const T* Gl;
  const T* bGd;
  const T* bGu;
  const T* bGl;
  const T* ckpt;
  T* aD;
  T* aU;
  T* aL;
  int n, b, c;
  int orig;        // index in the caller's descriptor array
  int team;        // CTAs of this instance's team
  int slot_start;  // first queue slot of this instance
};

// Scratch of one team: the segment's g and P blocks, the 9 temporaries and
// the inversion side buffer, 256-byte aligned parts.
static size_t adj_slot_bytes(int n, int b, size_t es) {
  const size_t bb = (size_t)b * b;
  const size_t c = (size_t)ckpt_every(n);
  return align_up(c * bb * es, 256) * 2 + align_up(9 * bb * es, 256) + align_up(invert_side_elems(b) * es, 256);
}

// The reverse sweeps of every instance, instances taken from a device queue
// (largest b^3 n first) by teams of CTAs, as the batched RGF kernel takes its
// forward sweeps; every wait bounded by wait_ns.
template <class T>
__global__ void __launch_bounds__(kThreads, 1) adjoint_batched_kernel(unsigned char* ws, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
  const AdjEntry<T>* entries = reinterpret_cast<const AdjEntry<T>*>(ws + hdr->desc_offset);
  ItemArea* items = reinterpret_cast<ItemArea*>(ws + hdr->items_offset);
  const int count = hdr->count;
  __shared__ int sh_slot;
  while (true) {
    if (threadIdx.x == 0) sh_slot = (int)atomicAdd(&hdr->queue_head, 1u);
    __syncthreads();
    const int s = sh_slot;
    __syncthreads();
    if (s >= hdr->total_slots) break;
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (entries[mid].slot_start <= s) lo = mid; else hi = mid - 1;
    }
    const AdjEntry<T> e = entries[lo];
    ItemArea* item = items + lo;
    const int rank = s - e.slot_start;
    if (rank == 0 && threadIdx.x == 0) {
      const int id = acquire_scratch(hdr, &item->status, wait_ns);
      item->slot_id = id;
      item->scratch = id < 0 ? nullptr : ws + hdr->slots_offset + (size_t)id * hdr->slot_bytes;
      __threadfence();
    }
    TeamDyn team{&item->counter, &item->status, rank, e.team, 0u, wait_ns};
    unsigned char* slot = team.sync() ? *((unsigned char* volatile*)&item->scratch) : nullptr;
    if (slot) {
      const size_t es = sizeof(T), bb = (size_t)e.b * e.b;
      AdjParams<T> p;
      p.diag = e.diag;
      p.upper = e.upper;
      p.lower = e.lower;
      p.Gd = e.Gd;
      p.Gu = e.Gu;
      p.Gl = e.Gl;
      p.bGd = e.bGd;
      p.bGu = e.bGu;
      p.bGl = e.bGl;
      p.aD = e.aD;
      p.aU = e.aU;
      p.aL = e.aL;
      p.ckpt = e.ckpt;
      unsigned char* q = slot;
      p.seg_g = reinterpret_cast<T*>(q);
      q += align_up(e.c * bb * es, 256);
      p.seg_P = reinterpret_cast<T*>(q);
      q += align_up(e.c * bb * es, 256);
      p.tmp = reinterpret_cast<T*>(q);
      q += align_up(9 * bb * es, 256);
      p.side = reinterpret_cast<T*>(q);
      p.status = &item->status;
      p.n = e.n;
      p.b = e.b;
      p.c = e.c;
      p.flags = hdr->flags;
      if (e.b <= 32)
        rgf_adjoint<T, 32, 32>(team, p, smem);
      else
        rgf_adjoint<T, 64, 64>(team, p, smem);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (rank == 0) finish_item(hdr, item, e.orig);
      leave_item(hdr, item, e.team);
    }
  }
}

static int adj_team(int b, int count, int grid, unsigned flags) {
  if (flags & SINVB_FORCE_CTA) return 1;
  int t = b >= 1024 ? 8 : b >= 512 ? 4 : b >= 256 ? 2 : 1;
  if ((long)t * count < grid && b >= 128) t = std::max(t, std::min({grid / count, std::max(1, b / 64), 16}));
  return t;
}

struct AdjBatchLayout {
  size_t desc_offset, items_offset, slots_offset, slot_bytes, total;
  unsigned nslots;
};

static AdjBatchLayout adj_batch_layout(const sinvb_adjoint_desc* d, int count, int dtype, unsigned flags) {
  const size_t es = dtype == SINVB_C128 ? 16 : 8;
  const int grid = device_sm_count();
  AdjBatchLayout L{};
  size_t slot = 256;
  int min_team = grid;
  for (int k = 0; k < count; k++) {
    slot = std::max(slot, adj_slot_bytes(d[k].n, d[k].b, es));
    min_team = std::min(min_team, adj_team(d[k].b, count, grid, flags));
  }
  L.nslots = std::min<unsigned>(grid / min_team, 256u);
  L.desc_offset = sizeof(WsHeader);
  L.items_offset = align_up(L.desc_offset + (size_t)count * sizeof(AdjEntry<cplx>), 256);
  L.slots_offset = align_up(L.items_offset + (size_t)count * sizeof(ItemArea), 256);
  L.slot_bytes = align_up(slot, 256);
  L.total = L.slots_offset + (size_t)L.nslots * L.slot_bytes;
  return L;
}

template <class T>
static int run_adjoint_batched(const sinvb_adjoint_desc* d, int count, unsigned flags, void* ws, size_t ws_bytes,
                               int* status, cudaStream_t stream, int dtype) {
  if (!d || count < 1 || !ws) return SINVB_EINVAL;
  if ((uintptr_t)ws % 256) return SINVB_EWORKSPACE;
  if (flags & ~(SINVB_SYM | SINVB_SAVE_OFFDIAG | SINVB_FORCE_CTA)) return SINVB_EINVAL;
  const size_t align = dtype == SINVB_C128 ? 16 : 8;
  for (int k = 0; k < count; k++) {
    const sinvb_adjoint_desc& e = d[k];
    if (e.n < 1 || e.b < 1 || !e.diag || !e.G_diag || !e.bG_diag || !e.aD) return SINVB_EINVAL;
    if (e.n > 1 && (!e.upper || !e.lower || !e.G_upper || !e.G_lower || !e.aU || !e.aL)) return SINVB_EINVAL;
    if ((e.n - 1) / ckpt_every(e.n) >= 1 && !e.checkpoints) return SINVB_EINVAL;
    for (const void* q : {e.diag, e.upper, e.lower, e.G_diag, e.G_upper, e.G_lower, e.bG_diag, e.bG_upper,
                          e.bG_lower, e.checkpoints, (const void*)e.aD, (const void*)e.aU, (const void*)e.aL})
      if (q && (uintptr_t)q % align) return SINVB_EINVAL;
  }
  const AdjBatchLayout L = adj_batch_layout(d, count, dtype, flags);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  const int grid = device_sm_count();
  std::vector<AdjEntry<T>> entries(count);
  for (int k = 0; k < count; k++) {
    AdjEntry<T>& e = entries[k];
    e.diag = (const T*)d[k].diag;
    e.upper = (const T*)d[k].upper;
    e.lower = (const T*)d[k].lower;
    e.Gd = (const T*)d[k].G_diag;
    e.Gu = (const T*)d[k].G_upper;
    e.Gl = (const T*)d[k].G_lower;
    e.bGd = (const T*)d[k].bG_diag;
    e.bGu = (const T*)d[k].bG_upper;
    e.bGl = (const T*)d[k].bG_lower;
    e.ckpt = (const T*)d[k].checkpoints;
    e.aD = (T*)d[k].aD;
    e.aU = (T*)d[k].aU;
    e.aL = (T*)d[k].aL;
    e.n = d[k].n;
    e.b = d[k].b;
    e.c = ckpt_every(d[k].n);
    e.orig = k;
    e.team = adj_team(d[k].b, count, grid, flags);
  }
  std::stable_sort(entries.begin(), entries.end(), [](const AdjEntry<T>& x, const AdjEntry<T>& y) {
    return (double)x.b * x.b * x.b * x.n > (double)y.b * y.b * y.b * y.n;
  });
  int total_slots = 0;
  for (auto& e : entries) {
    e.slot_start = total_slots;
    total_slots += e.team;
  }
  WsHeader h{};
  h.count = count;
  h.flags = flags;
  h.nslots = L.nslots;
  h.slot_bytes = L.slot_bytes;
  h.desc_offset = L.desc_offset;
  h.slots_offset = L.slots_offset;
  h.inst_status = status;
  h.items_offset = L.items_offset;
  h.total_slots = total_slots;
  unsigned char* w = (unsigned char*)ws;
  SINVB_CUDA(cudaMemcpyAsync(w, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(w + L.desc_offset, entries.data(), count * sizeof(AdjEntry<T>), cudaMemcpyHostToDevice,
                             stream));
  SINVB_CUDA(cudaMemsetAsync(w + L.items_offset, 0, (size_t)count * sizeof(ItemArea), stream));
  auto k = adjoint_batched_kernel<T>;
  constexpr size_t g = (size_t)gemm_smem_elems<T, 64, 64>() * sizeof(T);
  constexpr size_t smem = g > sizeof(GjShared<T>) ? g : sizeof(GjShared<T>);
  SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  unsigned long long wait_ns = kTeamWaitNs;
  void* args[] = {(void*)&w, (void*)&wait_ns};
  SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(kThreads), args, smem, stream));
  return SINVB_OK;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

int sinvb_rgf_checkpoints(int n, int* every, int* count) {
  if (n < 1 || !every || !count) return SINVB_EINVAL;
  *every = ckpt_every(n);
  *count = (n - 1) / *every;
  return SINVB_OK;
}

size_t sinvb_rgf_adjoint_workspace_size(int n, int b, int dtype, unsigned flags) {
  (void)flags;
  if (n < 1 || b < 1 || (dtype != SINVB_C128 && dtype != SINVB_F64)) return 0;
  return adj_layout(n, b, dtype).total;
}

size_t sinvb_rgf_adjoint_batched_workspace_size(const sinvb_adjoint_desc* descs, int count, int dtype,
                                                unsigned flags) {
  if (!descs || count < 1 || (dtype != SINVB_C128 && dtype != SINVB_F64)) return 0;
  return adj_batch_layout(descs, count, dtype, flags).total;
}

int sinvb_rgf_adjoint_batched_z(const sinvb_adjoint_desc* descs, int count, unsigned flags, void* workspace,
                                size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  return run_adjoint_batched<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                   SINVB_C128);
}

int sinvb_rgf_adjoint_batched_d(const sinvb_adjoint_desc* descs, int count, unsigned flags, void* workspace,
                                size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  return run_adjoint_batched<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                     SINVB_F64);
}

int sinvb_rgf_adjoint_z(const void* diag, const void* upper, const void* lower, const void* G_diag,
                        const void* G_upper, const void* G_lower, const void* bG_diag, const void* bG_upper,
                        const void* bG_lower, const void* checkpoints, int every, int n, int b, unsigned flags,
                        void* aD, void* aU, void* aL, void* workspace, size_t workspace_bytes,
                        sinvb_stream_t stream) {
  return run_adjoint<cplx>(diag, upper, lower, G_diag, G_upper, G_lower, bG_diag, bG_upper, bG_lower, checkpoints,
                           every, n, b, flags, aD, aU, aL, workspace, workspace_bytes, (cudaStream_t)stream,
                           SINVB_C128);
}

int sinvb_rgf_adjoint_d(const void* diag, const void* upper, const void* lower, const void* G_diag,
                        const void* G_upper, const void* G_lower, const void* bG_diag, const void* bG_upper,
                        const void* bG_lower, const void* checkpoints, int every, int n, int b, unsigned flags,
                        void* aD, void* aU, void* aL, void* workspace, size_t workspace_bytes,
                        sinvb_stream_t stream) {
  return run_adjoint<double>(diag, upper, lower, G_diag, G_upper, G_lower, bG_diag, bG_upper, bG_lower, checkpoints,
                             every, n, b, flags, aD, aU, aL, workspace, workspace_bytes, (cudaStream_t)stream,
                             SINVB_F64);
}

}  // extern "C"
