// Allocation-free RGF entry point.
//
// Some callers cannot allocate device memory at the point where they need a
// selected inversion.  Examples: a host callback or an allocator hook that
// must not re-enter the allocator; a sandboxed plugin whose host application
// owns every device allocation and hands it only inputs and outputs.  For
// them this file provides
// sinvb_rgf_z_noalloc: the single-matrix RGF sweep (one CTA walks the whole
// sweep) with its scratch memory in a file-scope device array that belongs to
// the library, so the caller passes only the inputs and the outputs.
//
// Limits and rules:
//  * block size b <= kNoAllocMaxB (64) and SINVB_SAVE_OFFDIAG set when n > 1
//    (the sweep keeps its per-block-row products in G_upper / G_lower);
//  * the array is kNoAllocScratchBytes (131,328 bytes); every GPU that loads
//    the library holds it until the process exits;
//  * the first call on a device does the set-up with that device current: it
//    looks up the array's device address (cudaGetSymbolAddress) and sets the
//    shared-memory attribute of both kernel instances;
//  * the output arrays must not overlap the inputs or each other (the sweep
//    keeps per-row products in G_upper / G_lower while it still reads A);
//    overlapping ranges are rejected with SINVB_EINVAL;
//  * every call uses the same array: calls that overlap on the GPU (two
//    streams, or two threads) race on it and must be serialised by the caller;
//  * the array keeps the contents of the last call; each call clears the
//    parts that must start at zero (status word, barrier counter) itself.
#include <mutex>

#include "host_util.h"
#include "rgf_sweep.cuh"

namespace sinvb {

constexpr int kNoAllocMaxB = 64;
// 256-byte header + the two b x b complex blocks of the sweep's T ping-pong.
constexpr size_t kNoAllocScratchBytes = sizeof(WsHeader) + 2 * (size_t)kNoAllocMaxB * kNoAllocMaxB * sizeof(cplx);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocDevices = 64;
static void* g_noalloc_addr[kNoAllocDevices];
static std::mutex g_noalloc_mutex;

template <int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) rgf_noalloc_kernel(RgfParams<cplx> p, int* status_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamCta team;
  rgf_sweep<cplx, BM, BN>(team, p, reinterpret_cast<cplx*>(smem_raw));
  __syncthreads();
  if (threadIdx.x == 0 && status_out) *status_out = *p.status;
}

template <int BM, int BN>
constexpr size_t noalloc_smem() {
  constexpr size_t g = (size_t)gemm_smem_elems<cplx, BM, BN>() * sizeof(cplx);
  return g > sizeof(GjShared<cplx>) ? g : sizeof(GjShared<cplx>);
}

template <int BM, int BN>
static int launch_noalloc(const RgfParams<cplx>& p, int* status_out, cudaStream_t stream) {
  rgf_noalloc_kernel<BM, BN><<<1, kThreads, noalloc_smem<BM, BN>(), stream>>>(p, status_out);
  SINVB_CUDA(cudaGetLastError());
  return SINVB_OK;
}

// True when the byte ranges [a, a + na) and [b, b + nb) share a byte.
static bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  if (!a || !b || !na || !nb) return false;
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

// Device address of g_noalloc_scratch on the current device (looked up once per device).
static int noalloc_scratch(void** out) {
  int dev = 0;
  SINVB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocDevices) return SINVB_EUNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    SINVB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return SINVB_ECUDA;
    // both kernel instances get their shared-memory size now, so that no
    // later call (whatever its b) performs device set-up
    SINVB_CUDA(cudaFuncSetAttribute(rgf_noalloc_kernel<32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)noalloc_smem<32, 32>()));
    SINVB_CUDA(cudaFuncSetAttribute(rgf_noalloc_kernel<64, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)noalloc_smem<64, 64>()));
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return SINVB_OK;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" int sinvb_rgf_z_noalloc(const void* diag, const void* upper, const void* lower, int n, int b,
                                   unsigned flags, void* G_diag, void* G_upper, void* G_lower, int* status,
                                   sinvb_stream_t stream) {
  if (n < 1 || b < 1 || !diag || !G_diag) return SINVB_EINVAL;
  if (b > kNoAllocMaxB) return SINVB_EINVAL;  // scratch holds two b x b blocks of at most 64 x 64
  if (n > 1 && (!upper || !lower)) return SINVB_EINVAL;
  if (n > 1 && !(flags & SINVB_SAVE_OFFDIAG)) return SINVB_EINVAL;
  if (n > 1 && (!G_upper || !G_lower)) return SINVB_EINVAL;
  if (flags & ~(SINVB_SYM | SINVB_SAVE_OFFDIAG)) return SINVB_EINVAL;
  for (const void* q : {diag, upper, lower, (const void*)G_diag, (const void*)G_upper, (const void*)G_lower})
    if (q && (uintptr_t)q % 16) return SINVB_EINVAL;
  {  // outputs may overlap neither the inputs nor each other
    const size_t bb = (size_t)b * b * sizeof(cplx);
    const size_t nd = (size_t)n * bb, no = n > 1 ? (size_t)(n - 1) * bb : 0;
    const void* in[3] = {diag, upper, lower};
    const size_t in_n[3] = {nd, no, no};
    const void* out[3] = {G_diag, G_upper, G_lower};
    const size_t out_n[3] = {nd, no, no};
    for (int o = 0; o < 3; o++) {
      for (int i = 0; i < 3; i++)
        if (overlaps(out[o], out_n[o], in[i], in_n[i])) return SINVB_EINVAL;
      for (int o2 = o + 1; o2 < 3; o2++)
        if (overlaps(out[o], out_n[o], out[o2], out_n[o2])) return SINVB_EINVAL;
    }
  }
  int rc = check_device();
  if (rc) return rc;
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  unsigned char* s = (unsigned char*)scratch;
  cudaStream_t st = (cudaStream_t)stream;
  // status word and barrier counter must start at zero; the blocks need no clearing
  SINVB_CUDA(cudaMemsetAsync(s, 0, sizeof(WsHeader), st));
  RgfParams<cplx> p;
  p.diag = (const cplx*)diag;
  p.upper = (const cplx*)upper;
  p.lower = (const cplx*)lower;
  p.Gd = (cplx*)G_diag;
  p.Gu = (cplx*)G_upper;
  p.Gl = (cplx*)G_lower;
  p.X = p.Gl;
  p.P = p.Gu;
  p.T0 = reinterpret_cast<cplx*>(s + sizeof(WsHeader));
  p.T1 = p.T0 + (size_t)b * b;
  p.T2 = p.T3 = nullptr;  // in-place mode only
  p.Winv = nullptr;  // blocks of at most 64 x 64 invert without the side buffer
  p.hdr = reinterpret_cast<WsHeader*>(s);
  p.status = &p.hdr->status;
  p.n = n;
  p.b = b;
  p.flags = flags;
  p.ckpt = nullptr;
  p.ckpt_every = 1;
  p.oz_digits = 0;
  p.oz_scratch = nullptr;
  p.oz = nullptr;
  if (b <= 32) return launch_noalloc<32, 32>(p, status, st);
  return launch_noalloc<64, 64>(p, status, st);
}
