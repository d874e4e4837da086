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
#include <cmath>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "batch_queue.cuh"
#include "host_util.h"
#include "rgf_sweep.cuh"

namespace sinvb {

// The instance count and flags of the last upload into a workspace, kept
// host-side so a re-run needs no device read (the kernel reads everything else
// from the workspace header).
static std::mutex g_count_mutex;
static std::unordered_map<const void*, std::pair<int, unsigned>>& count_table() {
  static std::unordered_map<const void*, std::pair<int, unsigned>> t;
  return t;
}
// Device wait bound of the launches that use a workspace (set by
// sinvb_rgf_batched_set_wait_limit; absent: kTeamWaitNs).
static std::unordered_map<const void*, unsigned long long>& wait_table() {
  static std::unordered_map<const void*, unsigned long long> t;
  return t;
}
static unsigned long long wait_limit_of(const void* ws) {
  std::lock_guard<std::mutex> lock(g_count_mutex);
  auto it = wait_table().find(ws);
  return it == wait_table().end() ? kTeamWaitNs : it->second;
}

template <class T>
struct BatchEntry {
  const T* diag;
  const T* upper;
  const T* lower;
  T* Gd;
  T* Gu;
  T* Gl;
  int n, b;
  int orig;        // index in the caller's descriptor array
  int team;        // CTAs working on this instance
  int slot_start;  // first queue slot of this instance (entries are in queue order)
  int int8;        // mixed batches: this instance's products run on the int8 tensor cores
  T* ckpt;         // optional: checkpoints g_{s c - 1} of the forward sweep for the adjoint
};
static_assert(sizeof(BatchEntry<cplx>) == 80, "80-byte entries");

// Smallest block size whose products a mixed-precision batch runs on the int8
// tensor cores (measured on B200: at b = 256 both paths take the same time).
constexpr int kMixedMinB = 256;

// Digits of the mixed-precision products (flags bits 12-15; 0 means 7).
__host__ __device__ inline int mixed_digits(unsigned flags) {
  const int d = (int)((flags >> 12) & 15u);
  return d == 0 ? 7 : d;
}

// Bytes of the FP64 part of a team's scratch slot (T / side buffers and, when
// off-diagonal blocks are not saved, the X / P blocks); the digit planes of the
// mixed-precision products follow.
__host__ __device__ inline size_t fp64_slot_bytes(int n, int b, size_t es, bool save) {
  const size_t bb = (size_t)b * b;
  size_t s = 4 * bb + invert_side_elems(b);
  if (!save) s += 2 * (size_t)(n - 1) * bb;
  return (s * es + 255) / 256 * 256;
}

// Persistent: every CTA repeatedly takes one queue slot.  Slot s belongs to the
// instance k with slot_start[k] <= s < slot_start[k] + team[k], with rank
// s - slot_start[k] in that instance's team.  Slots are handed out in order,
// so a team completes as soon as its last member frees up; with teams sized
// by block size (large blocks first) members mostly arrive together.  Every
// CTA of the launch is resident (cooperative launch), so each team wait ends.
// wait_ns bounds every wait of the launch (team barriers, scratch slots,
// streamed ready words).
template <class T, bool Mixed>
__global__ void __launch_bounds__(kThreads, 1) rgf_batched_kernel(unsigned char* ws, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
  const BatchEntry<T>* entries = reinterpret_cast<const BatchEntry<T>*>(ws + hdr->desc_offset);
  ItemArea* items = reinterpret_cast<ItemArea*>(ws + hdr->items_offset);
  const int count = hdr->count;
  const int total_slots = hdr->total_slots;
  const unsigned flags = hdr->flags;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  const bool inplace = flags & SINVB_INPLACE;
  // mixed precision: block products on the int8 tensor cores; this CTA holds
  // its TMEM for the whole persistent loop
  const int oz_digits = Mixed ? mixed_digits(flags) : 0;
  __shared__ OzState oz_state;
  if (Mixed) oz_setup(&oz_state);
  __shared__ int sh_slot;
  while (true) {
    if (threadIdx.x == 0) sh_slot = (int)atomicAdd(&hdr->queue_head, 1u);
    __syncthreads();
    const int s = sh_slot;
    __syncthreads();  // sh_slot is rewritten by the next dequeue
    if (s >= total_slots) break;
    int lo = 0, hi = count - 1;  // last entry with slot_start <= s
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (entries[mid].slot_start <= s) lo = mid; else hi = mid - 1;
    }
    const int k = lo;
    const BatchEntry<T> e = entries[k];
    ItemArea* item = items + k;
    const int rank = s - e.slot_start;
    if (rank == 0 && threadIdx.x == 0) {
      // an instance whose streamed inputs never arrived is skipped
      const bool ready = !hdr->ready || wait_ready(hdr, e.orig, &item->status, wait_ns);
      const int id = ready ? acquire_scratch(hdr, &item->status, wait_ns) : -1;
      item->slot_id = id;
      item->scratch = id < 0 ? nullptr : ws + hdr->slots_offset + (size_t)id * hdr->slot_bytes;
      __threadfence();
    }
    TeamDyn team{&item->counter, &item->status, rank, e.team, 0u, wait_ns};
    // formation: the rank-0 scratch pointer is visible after this; without a
    // slot (inputs never arrived, or none came free; reported) the team skips
    unsigned char* slot = team.sync() ? *((unsigned char* volatile*)&item->scratch) : nullptr;
    if (!slot) {
      if (threadIdx.x == 0) {
        if (rank == 0) finish_item(hdr, item, e.orig);
        leave_item(hdr, item, e.team);
      }
      continue;
    }
    const size_t bb = (size_t)e.b * e.b;
    RgfParams<T> p;
    p.diag = e.diag;
    p.upper = e.upper;
    p.lower = e.lower;
    p.Gd = inplace ? const_cast<T*>(e.diag) : e.Gd;
    p.Gu = inplace ? const_cast<T*>(e.upper) : e.Gu;
    p.Gl = inplace ? const_cast<T*>(e.lower) : e.Gl;
    T* sp = reinterpret_cast<T*>(slot);
    p.T0 = sp;
    p.T1 = sp + bb;
    p.T2 = sp + 2 * bb;
    p.T3 = sp + 3 * bb;
    p.Winv = sp + 4 * bb;
    T* xp = p.Winv + invert_side_elems(e.b);
    p.X = save ? p.Gl : xp;
    p.P = save ? p.Gu : xp + (size_t)(e.n - 1) * bb;
    p.hdr = hdr;
    p.status = &item->status;
    p.n = e.n;
    p.b = e.b;
    p.flags = flags;
    p.ckpt = e.ckpt;  // c = ceil(sqrt(n)), as the adjoint's segments (sinvb_rgf_checkpoints)
    p.ckpt_every = e.ckpt ? max(1, (int)ceil(sqrt((double)e.n))) : 1;
    // small blocks keep FP64 DMMA products: the int8 path's fixed costs
    // (digit slicing, pipeline fill) outweigh its faster products there
    p.oz_digits = e.int8 ? oz_digits : 0;
    p.oz_scratch = slot + fp64_slot_bytes(e.n, e.b, sizeof(T), save);
    p.oz = &oz_state;
    if (e.b <= 32)
      rgf_sweep<T, 32, 32, Mixed>(team, p, smem);
    else
      rgf_sweep<T, 64, 64, Mixed>(team, p, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (rank == 0) finish_item(hdr, item, e.orig);
      leave_item(hdr, item, e.team);
    }
  }
  if (Mixed) oz_teardown(&oz_state);
}

constexpr size_t kBatchedSmem = sizeof(GjShared<cplx>) > (size_t)gemm_smem_elems<cplx, 64, 64>() * 16
                                    ? sizeof(GjShared<cplx>)
                                    : (size_t)gemm_smem_elems<cplx, 64, 64>() * 16;

static size_t elem_bytes(int dtype) { return (dtype == SINVB_C128 || dtype == SINVB_C64) ? 16 : 8; }

struct BatchLayout {
  size_t desc_offset, items_offset, slots_offset, slot_bytes, total;
  unsigned nslots;
};

static unsigned batch_slots() {
  // one CTA per SM: the sweep kernels use up to 232 registers per thread
  return (unsigned)device_sm_count();
}

static int team_size(int b, unsigned flags) {
  if (flags & SINVB_FORCE_CTA) return 1;
  if (b >= 1024) return 8;
  if (b >= 512) return 4;
  if (b >= 256) return 2;
  return 1;
}

// Team of every instance: team_size(b), and when the default teams leave CTAs
// of the grid idle (few instances), teams of b >= 256 grow to grid / count
// CTAs, at most b / 64 (one 64-wide tile column each) and 16.
//
// A caller's schedule (sinvb_batch_schedule, e.g. from the autotuner) sets
// the team of any instance it names instead.
static std::vector<int> batch_teams(const sinvb_batch_desc* d, int count, unsigned flags, int grid,
                                    const sinvb_batch_schedule* sched = nullptr) {
  std::vector<int> t(count);
  long total = 0;
  for (int k = 0; k < count; k++) total += t[k] = team_size(d[k].b, flags);
  if (!(flags & SINVB_FORCE_CTA) && total < grid) {
    const int share = grid / count;
    for (int k = 0; k < count; k++)
      if (d[k].b >= 256) t[k] = std::max(t[k], std::min({share, d[k].b / 64, 16}));
  }
  if (sched && sched->team)
    for (int k = 0; k < count; k++)
      if (sched->team[k] > 0) t[k] = std::min(sched->team[k], grid);
  return t;
}

// Smallest block size whose products a mixed batch runs on the int8 tensor cores.
static int mixed_min_b(const sinvb_batch_schedule* sched) {
  return sched && sched->mixed_min_b > 0 ? sched->mixed_min_b : kMixedMinB;
}

static BatchLayout batch_layout(const sinvb_batch_desc* d, int count, int dtype, unsigned flags,
                                const sinvb_batch_schedule* sched = nullptr) {
  BatchLayout L{};
  const size_t es = elem_bytes(dtype);
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  const bool mixed = flags & SINVB_PREC_MIXED;
  const int min_b = mixed_min_b(sched);
  size_t slot = 0;
  for (int k = 0; k < count; k++) {
    size_t s = fp64_slot_bytes(d[k].n, d[k].b, es, save);
    if (mixed && d[k].b >= min_b) s += 2 * oz_op_scratch(d[k].b, d[k].b, d[k].b, mixed_digits(flags));
    slot = std::max(slot, s);
  }
  // scratch slots: as many as teams can run at once (grid / smallest team)
  const std::vector<int> teams = batch_teams(d, count, flags, (int)batch_slots(), sched);
  const int min_team = *std::min_element(teams.begin(), teams.end());
  L.nslots = std::min<unsigned>(batch_slots() / min_team, 256u);
  L.desc_offset = sizeof(WsHeader);
  L.items_offset = align_up(L.desc_offset + (size_t)count * sizeof(BatchEntry<cplx>), 256);
  L.slots_offset = align_up(L.items_offset + (size_t)count * sizeof(ItemArea), 256);
  L.slot_bytes = align_up(std::max<size_t>(slot, 256), 256);
  L.total = L.slots_offset + (size_t)L.nslots * L.slot_bytes;
  return L;
}

static int check_batch(const sinvb_batch_desc* d, int count, unsigned flags, const void* ws, size_t ws_bytes,
                       int dtype, const sinvb_batch_schedule* sched = nullptr) {
  if (!d || count < 1 || !ws) return SINVB_EINVAL;
  if (sched) {
    if (sched->mixed_min_b < 0) return SINVB_EINVAL;
    if (sched->team)
      for (int k = 0; k < count; k++)
        if (sched->team[k] < 0 || sched->team[k] > (int)batch_slots()) return SINVB_EINVAL;
  }
  if ((uintptr_t)ws % 256) return SINVB_EWORKSPACE;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  const size_t align = elem_bytes(dtype);
  for (int k = 0; k < count; k++) {
    const sinvb_batch_desc& e = d[k];
    const bool inplace = flags & SINVB_INPLACE;
    if (e.n < 1 || e.b < 1 || !e.diag || (!inplace && !e.G_diag)) return SINVB_EINVAL;
    if (e.n > 1 && (!e.upper || !e.lower)) return SINVB_EINVAL;
    if (!inplace && save && e.n > 1 && (!e.G_upper || !e.G_lower)) return SINVB_EINVAL;
    if (inplace && !save) return SINVB_EINVAL;
    for (const void* q : {e.diag, e.upper, e.lower, (const void*)e.G_diag, (const void*)e.G_upper, (const void*)e.G_lower})
      if (q && (uintptr_t)q % align) return SINVB_EINVAL;
  }
  if (ws_bytes < batch_layout(d, count, dtype, flags, sched).total) return SINVB_EWORKSPACE;
  return check_device();
}

// CTAs per instance: enough tiles per CTA to stay busy, few enough barriers.


template <class T>
static int launch_batched(void* ws, int count, unsigned flags, cudaStream_t stream) {
  const bool mixed = std::is_same<T, cplx>::value && (flags & SINVB_PREC_MIXED);
  auto k = mixed ? rgf_batched_kernel<T, std::is_same<T, cplx>::value> : rgf_batched_kernel<T, false>;
  size_t smem = kBatchedSmem;
  if (flags & SINVB_PREC_MIXED)
    smem = std::max(smem, std::max(oz_smem_bytes(mixed_digits(flags)), oz_slice_smem(mixed_digits(flags))));
  SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // reset status, barrier and queue, the scratch bitmap, and every instance's team area
  SINVB_CUDA(cudaMemsetAsync(ws, 0, 16, stream));
  SINVB_CUDA(cudaMemsetAsync((unsigned char*)ws + offsetof(WsHeader, slot_bits), 0, sizeof(WsHeader::slot_bits),
                             stream));
  const size_t items_offset = align_up(sizeof(WsHeader) + (size_t)count * sizeof(BatchEntry<cplx>), 256);
  SINVB_CUDA(cudaMemsetAsync((unsigned char*)ws + items_offset, 0, (size_t)count * sizeof(ItemArea), stream));
  unsigned char* w = (unsigned char*)ws;
  unsigned long long wait_ns = wait_limit_of(ws);
  void* args[] = {(void*)&w, (void*)&wait_ns};
  // cooperative: every CTA resident, so a team member waiting for the others always gets them
  SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(batch_slots()), dim3(kThreads), args, smem,
                                         stream));
  return SINVB_OK;
}

template <class T>
static int upload_and_run(const sinvb_batch_desc* d, int count, unsigned flags, void* ws, size_t ws_bytes,
                          int* status, cudaStream_t stream, int dtype, const unsigned* ready = nullptr,
                          unsigned* done = nullptr, unsigned gen = 0, const sinvb_batch_schedule* sched = nullptr,
                          void* const* ckpts = nullptr) {
  int rc = check_batch(d, count, flags, ws, ws_bytes, dtype, sched);
  if (rc) return rc;
  const BatchLayout L = batch_layout(d, count, dtype, flags, sched);
  const std::vector<int> teams = batch_teams(d, count, flags, (int)batch_slots(), sched);
  const bool mixed = flags & SINVB_PREC_MIXED;
  const int min_b = mixed_min_b(sched);
  std::vector<double> prio(count);
  for (int k = 0; k < count; k++)
    prio[k] = sched && sched->priority ? (double)sched->priority[k] : (double)d[k].b * d[k].b * d[k].b * d[k].n;
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
    e.team = teams[k];
    e.slot_start = 0;
    e.int8 = mixed && d[k].b >= min_b;
    e.ckpt = ckpts ? (T*)ckpts[k] : nullptr;
  }
  // longest first (by default cost ~ b^3 n; a schedule may give its own
  // estimates): long chains start while short ones fill in
  std::stable_sort(entries.begin(), entries.end(), [&](const BatchEntry<T>& x, const BatchEntry<T>& y) {
    return prio[x.orig] > prio[y.orig];
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
  h.ready = ready;
  h.done = done;
  h.gen = gen;
  unsigned char* w = (unsigned char*)ws;
  SINVB_CUDA(cudaMemcpyAsync(w, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(w + L.desc_offset, entries.data(), count * sizeof(BatchEntry<T>),
                             cudaMemcpyHostToDevice, stream));
  // the pageable copies above are staged before they return; the host arrays may go
  {
    std::lock_guard<std::mutex> lock(g_count_mutex);
    count_table()[ws] = {count, flags};
  }
  return launch_batched<T>(ws, count, flags, stream);
}

template <class T>
static int rerun(void* ws, cudaStream_t stream) {
  int count = -1;
  unsigned flags = 0;
  {
    std::lock_guard<std::mutex> lock(g_count_mutex);
    auto it = count_table().find(ws);
    if (it != count_table().end()) {
      count = it->second.first;
      flags = it->second.second;
    }
  }
  if (count < 1) return SINVB_EINVAL;  // nothing uploaded into this workspace
  return launch_batched<T>(ws, count, flags, stream);
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
  if ((flags & SINVB_PREC_MIXED) && mixed_digits(flags) > kOzMaxDigits) return SINVB_EINVAL;
  if (flags & SINVB_PREC_MIXED)
    for (int k = 0; k < count; k++)
      if (descs && 2 * descs[k].b > (1 << 14)) return SINVB_EINVAL;
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128);
}

int sinvb_rgf_batched_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64);
}

int sinvb_rgf_batched_stream_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, const unsigned* ready, unsigned* done,
                               unsigned gen, sinvb_stream_t stream) {
  if (!ready || !done || gen == 0) return SINVB_EINVAL;
  if ((flags & SINVB_PREC_MIXED) && mixed_digits(flags) > kOzMaxDigits) return SINVB_EINVAL;
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128, ready, done, gen);
}

int sinvb_rgf_batched_stream_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, const unsigned* ready, unsigned* done,
                               unsigned gen, sinvb_stream_t stream) {
  if (!ready || !done || gen == 0) return SINVB_EINVAL;
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64, ready, done, gen);
}

size_t sinvb_rgf_batched_sched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype, unsigned flags,
                                              const sinvb_batch_schedule* sched) {
  if (!descs || count < 1 || dtype < 0 || dtype > 1) return 0;
  return batch_layout(descs, count, dtype, flags, sched).total;
}

int sinvb_rgf_batched_sched_z(const sinvb_batch_desc* descs, int count, unsigned flags,
                              const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes, int* status,
                              sinvb_stream_t stream) {
  if ((flags & SINVB_PREC_MIXED) && mixed_digits(flags) > kOzMaxDigits) return SINVB_EINVAL;
  if (flags & SINVB_PREC_MIXED)
    for (int k = 0; k < count; k++)
      if (descs && descs[k].b >= mixed_min_b(sched) && 2 * descs[k].b > (1 << 14)) return SINVB_EINVAL;
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128, nullptr, nullptr, 0, sched);
}

int sinvb_rgf_batched_sched_d(const sinvb_batch_desc* descs, int count, unsigned flags,
                              const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes, int* status,
                              sinvb_stream_t stream) {
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64, nullptr, nullptr, 0, sched);
}

int sinvb_rgf_batched_stream_sched_z(const sinvb_batch_desc* descs, int count, unsigned flags,
                                     const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                                     int* status, const unsigned* ready, unsigned* done, unsigned gen,
                                     sinvb_stream_t stream) {
  if (!ready || !done || gen == 0) return SINVB_EINVAL;
  if ((flags & SINVB_PREC_MIXED) && mixed_digits(flags) > kOzMaxDigits) return SINVB_EINVAL;
  if (flags & SINVB_PREC_MIXED)
    for (int k = 0; k < count; k++)
      if (descs && descs[k].b >= mixed_min_b(sched) && 2 * descs[k].b > (1 << 14)) return SINVB_EINVAL;
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128, ready, done, gen, sched);
}

int sinvb_rgf_batched_stream_sched_d(const sinvb_batch_desc* descs, int count, unsigned flags,
                                     const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                                     int* status, const unsigned* ready, unsigned* done, unsigned gen,
                                     sinvb_stream_t stream) {
  if (!ready || !done || gen == 0) return SINVB_EINVAL;
  if (flags & SINVB_PREC_MIXED) return SINVB_EUNSUPPORTED;
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64, ready, done, gen, sched);
}

int sinvb_rgf_batched_ckpt_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* const* checkpoints,
                             void* workspace, size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  if (!checkpoints || (flags & (SINVB_PREC_MIXED | SINVB_INPLACE))) return SINVB_EINVAL;
  for (int k = 0; k < count; k++) {
    if (!descs) return SINVB_EINVAL;
    const int c = std::max(1, (int)std::ceil(std::sqrt((double)descs[k].n)));
    if ((descs[k].n - 1) / c > 0 && (!checkpoints[k] || (uintptr_t)checkpoints[k] % 16)) return SINVB_EINVAL;
  }
  return upload_and_run<cplx>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                              SINVB_C128, nullptr, nullptr, 0, nullptr, checkpoints);
}

int sinvb_rgf_batched_ckpt_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* const* checkpoints,
                             void* workspace, size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  if (!checkpoints || (flags & (SINVB_PREC_MIXED | SINVB_INPLACE))) return SINVB_EINVAL;
  for (int k = 0; k < count; k++) {
    if (!descs) return SINVB_EINVAL;
    const int c = std::max(1, (int)std::ceil(std::sqrt((double)descs[k].n)));
    if ((descs[k].n - 1) / c > 0 && (!checkpoints[k] || (uintptr_t)checkpoints[k] % 8)) return SINVB_EINVAL;
  }
  return upload_and_run<double>(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream,
                                SINVB_F64, nullptr, nullptr, 0, nullptr, checkpoints);
}

int sinvb_rgf_batched_set_wait_limit(const void* workspace, double seconds) {
  if (!workspace || !(seconds > 0.0) || seconds > 3600.0) return SINVB_EINVAL;
  std::lock_guard<std::mutex> lock(g_count_mutex);
  wait_table()[workspace] = (unsigned long long)(seconds * 1e9);
  return SINVB_OK;
}

int sinvb_rgf_batched_rerun_z(void* workspace, sinvb_stream_t stream) {
  if (!workspace || (uintptr_t)workspace % 256) return SINVB_EINVAL;
  int rc = check_device();
  return rc ? rc : rerun<cplx>(workspace, (cudaStream_t)stream);
}

int sinvb_rgf_batched_rerun_d(void* workspace, sinvb_stream_t stream) {
  if (!workspace || (uintptr_t)workspace % 256) return SINVB_EINVAL;
  int rc = check_device();
  return rc ? rc : rerun<double>(workspace, (cudaStream_t)stream);
}

}  // extern "C"
