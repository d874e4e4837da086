// Adjoint of the RGF selected inversion: kernels and C-ABI entry points.
// The device code (adjoint.cuh) reverses both sweeps of
// src/sinv/algorithms/rgf/rgf.py:44-62 with sqrt(n) checkpoints.
#include <cmath>

#include "adjoint.cuh"
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
