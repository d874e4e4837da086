// Batched lesser Green's function: the retarded and lesser blocks of many
// energies (A(E_k), Sigma<(E_k)) in one persistent launch.
//
// A transport code runs rgf (src/sinv/algorithms/rgf/rgf.py:17-64) and then
// G< = G Sigma< G^H at every energy of its loop; each instance is one chain of
// dependent block operations.  As in the batched RGF kernel, every SM runs one
// CTA that takes queue slots; the slots of an instance form its team (one CTA
// below b = 256, more for larger blocks), which walks the lesser sweep pair
// (lesser_sweep.cuh) with team barriers only, in a scratch slot taken from the
// workspace bitmap.  Every wait is bounded (SINVB_STATUS_TIMEOUT).
#include <algorithm>
#include <vector>

#include "batch_queue.cuh"
#include "host_util.h"
#include "lesser_sweep.cuh"

namespace sinvb {

struct LesserEntry {
  const cplx* diag;
  const cplx* upper;
  const cplx* lower;
  const cplx* sig;
  cplx* Gd;
  cplx* Gu;
  cplx* Gl;
  cplx* GLd;
  cplx* GLu;
  int n, b;
  int orig;        // index in the caller's descriptor array
  int team;        // CTAs working on this instance
  int slot_start;  // first queue slot of this instance (entries are in queue order)
  int pad;
};

// Scratch of one instance: the five b x b temporaries of the sweep and the
// side buffer of the blocked inversion.
__host__ __device__ inline size_t lesser_tmp_bytes(int b) { return align_up((size_t)b * b * sizeof(cplx), 256); }
__host__ __device__ inline size_t lesser_slot_bytes(int b) {
  return 5 * lesser_tmp_bytes(b) + align_up(invert_side_elems(b) * sizeof(cplx), 256);
}

__global__ void __launch_bounds__(kThreads, 1) lesser_batched_kernel(unsigned char* ws, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
  const LesserEntry* entries = reinterpret_cast<const LesserEntry*>(ws + hdr->desc_offset);
  ItemArea* items = reinterpret_cast<ItemArea*>(ws + hdr->items_offset);
  const int count = hdr->count;
  __shared__ int sh_slot;
  while (true) {
    if (threadIdx.x == 0) sh_slot = (int)atomicAdd(&hdr->queue_head, 1u);
    __syncthreads();
    const int s = sh_slot;
    __syncthreads();  // sh_slot is rewritten by the next dequeue
    if (s >= hdr->total_slots) break;
    int lo = 0, hi = count - 1;  // last entry with slot_start <= s
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (entries[mid].slot_start <= s) lo = mid; else hi = mid - 1;
    }
    const LesserEntry e = entries[lo];
    ItemArea* item = items + lo;
    const int rank = s - e.slot_start;
    if (rank == 0 && threadIdx.x == 0) {
      const int id = acquire_scratch(hdr, &item->status, wait_ns);
      item->slot_id = id;
      item->scratch = id < 0 ? nullptr : ws + hdr->slots_offset + (size_t)id * hdr->slot_bytes;
      __threadfence();
    }
    TeamDyn team{&item->counter, &item->status, rank, e.team, 0u, wait_ns};
    // formation: the rank-0 scratch pointer is visible after this; without a
    // slot (none came free within the bound; reported) the team skips
    unsigned char* slot = team.sync() ? *((unsigned char* volatile*)&item->scratch) : nullptr;
    if (slot) {
      LesserParams p;
      p.diag = e.diag;
      p.upper = e.upper;
      p.lower = e.lower;
      p.sig = e.sig;
      p.Gd = e.Gd;
      p.Gu = e.Gu;
      p.Gl = e.Gl;
      p.GLd = e.GLd;
      p.GLu = e.GLu;
      for (int t = 0; t < 5; t++) p.tmp[t] = reinterpret_cast<cplx*>(slot + t * lesser_tmp_bytes(e.b));
      p.side = reinterpret_cast<cplx*>(slot + 5 * lesser_tmp_bytes(e.b));
      p.hdr = hdr;
      p.status = &item->status;
      p.n = e.n;
      p.b = e.b;
      if (e.b <= 32)
        lesser_sweep<32, 32>(team, p, smem);
      else
        lesser_sweep<64, 64>(team, p, smem);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (rank == 0) finish_item(hdr, item, e.orig);
      leave_item(hdr, item, e.team);
    }
  }
}

// CTAs per instance: one below b = 256, then one per 128 columns up to 8; when
// the instances leave CTAs of the grid idle, teams of b >= 128 grow to
// grid / count CTAs (at most b / 64 and 16).
static int lesser_team(int b, int count, int grid, unsigned flags) {
  if (flags & SINVB_FORCE_CTA) return 1;
  int t = b >= 1024 ? 8 : b >= 512 ? 4 : b >= 256 ? 2 : 1;
  if ((long)t * count < grid && b >= 128) t = std::max(t, std::min({grid / count, std::max(1, b / 64), 16}));
  return std::min(t, grid);
}

struct LesserBatchLayout {
  size_t desc_offset, items_offset, slots_offset, slot_bytes, total;
  unsigned nslots;
};

static LesserBatchLayout lesser_batch_layout(const sinvb_lesser_desc* d, int count, unsigned flags) {
  const int grid = device_sm_count();
  LesserBatchLayout L{};
  size_t slot = 256;
  int min_team = grid;
  for (int k = 0; k < count; k++) {
    slot = std::max(slot, lesser_slot_bytes(d[k].b));
    min_team = std::min(min_team, lesser_team(d[k].b, count, grid, flags));
  }
  // scratch slots: as many as teams can run at once (grid / smallest team)
  L.nslots = std::min<unsigned>(grid / std::max(1, min_team), 256u);
  L.desc_offset = sizeof(WsHeader);
  L.items_offset = align_up(L.desc_offset + (size_t)count * sizeof(LesserEntry), 256);
  L.slots_offset = align_up(L.items_offset + (size_t)count * sizeof(ItemArea), 256);
  L.slot_bytes = align_up(slot, 256);
  L.total = L.slots_offset + (size_t)L.nslots * L.slot_bytes;
  return L;
}

static bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  if (!a || !b || !na || !nb) return false;
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

static int check_lesser_batch(const sinvb_lesser_desc* d, int count, unsigned flags, const void* ws) {
  if (!d || count < 1 || !ws) return SINVB_EINVAL;
  if (flags & ~SINVB_FORCE_CTA) return SINVB_EINVAL;
  if ((uintptr_t)ws % 256) return SINVB_EWORKSPACE;
  for (int k = 0; k < count; k++) {
    const sinvb_lesser_desc& e = d[k];
    if (e.n < 1 || e.b < 1 || !e.diag || !e.sigma_lesser || !e.G_diag || !e.GL_diag) return SINVB_EINVAL;
    if (e.n > 1 && (!e.upper || !e.lower || !e.G_upper || !e.G_lower || !e.GL_upper)) return SINVB_EINVAL;
    for (const void* q : {e.diag, e.upper, e.lower, e.sigma_lesser, (const void*)e.G_diag, (const void*)e.G_upper,
                          (const void*)e.G_lower, (const void*)e.GL_diag, (const void*)e.GL_upper})
      if (q && (uintptr_t)q % 16) return SINVB_EINVAL;
    // the sweep writes its outputs while it still reads the inputs
    const size_t bb = (size_t)e.b * e.b * sizeof(cplx), nd = (size_t)e.n * bb, no = (size_t)(e.n - 1) * bb;
    const void* in[4] = {e.diag, e.upper, e.lower, e.sigma_lesser};
    const size_t nin[4] = {nd, no, no, nd};
    const void* out[5] = {e.G_diag, e.G_upper, e.G_lower, e.GL_diag, e.GL_upper};
    const size_t nout[5] = {nd, no, no, nd, no};
    for (int i = 0; i < 5; i++) {
      for (int j = 0; j < 4; j++)
        if (overlaps(out[i], nout[i], in[j], nin[j])) return SINVB_EINVAL;
      for (int j = i + 1; j < 5; j++)
        if (overlaps(out[i], nout[i], out[j], nout[j])) return SINVB_EINVAL;
    }
  }
  return SINVB_OK;
}

static int run_lesser_batched(const sinvb_lesser_desc* d, int count, unsigned flags, void* ws, size_t ws_bytes,
                              int* status, cudaStream_t stream) {
  int rc = check_lesser_batch(d, count, flags, ws);
  if (rc) return rc;
  rc = check_device();
  if (rc) return rc;
  const LesserBatchLayout L = lesser_batch_layout(d, count, flags);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  const int grid = device_sm_count();
  std::vector<LesserEntry> entries(count);
  for (int k = 0; k < count; k++) {
    LesserEntry& e = entries[k];
    e.diag = (const cplx*)d[k].diag;
    e.upper = (const cplx*)d[k].upper;
    e.lower = (const cplx*)d[k].lower;
    e.sig = (const cplx*)d[k].sigma_lesser;
    e.Gd = (cplx*)d[k].G_diag;
    e.Gu = (cplx*)d[k].G_upper;
    e.Gl = (cplx*)d[k].G_lower;
    e.GLd = (cplx*)d[k].GL_diag;
    e.GLu = (cplx*)d[k].GL_upper;
    e.n = d[k].n;
    e.b = d[k].b;
    e.orig = k;
    e.team = lesser_team(d[k].b, count, grid, flags);
    e.pad = 0;
  }
  // longest chains first (cost ~ b^3 n): they start while short ones fill in
  std::stable_sort(entries.begin(), entries.end(), [](const LesserEntry& x, const LesserEntry& y) {
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
  // the pageable copies are staged before they return; the host arrays may go
  SINVB_CUDA(cudaMemcpyAsync(w, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(w + L.desc_offset, entries.data(), count * sizeof(LesserEntry), cudaMemcpyHostToDevice,
                             stream));
  SINVB_CUDA(cudaMemsetAsync(w + L.items_offset, 0, (size_t)count * sizeof(ItemArea), stream));
  auto k = lesser_batched_kernel;
  constexpr size_t g = (size_t)gemm_smem_elems<cplx, 64, 64>() * sizeof(cplx);
  constexpr size_t smem = g > sizeof(GjShared<cplx>) ? g : sizeof(GjShared<cplx>);
  SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  unsigned long long wait_ns = kTeamWaitNs;
  void* args[] = {(void*)&w, (void*)&wait_ns};
  // cooperative: every CTA resident, so a team member waiting for the others always gets them
  SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(grid), dim3(kThreads), args, smem, stream));
  return SINVB_OK;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_rgf_lesser_batched_workspace_size(const sinvb_lesser_desc* descs, int count, unsigned flags) {
  if (!descs || count < 1 || check_device()) return 0;
  return lesser_batch_layout(descs, count, flags).total;
}

int sinvb_rgf_lesser_batched_z(const sinvb_lesser_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  return run_lesser_batched(descs, count, flags, workspace, workspace_bytes, status, (cudaStream_t)stream);
}

}  // extern "C"
