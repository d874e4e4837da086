// Serial RGF selected inversion: kernels and C-ABI entry points.
//
// Entry points replace src/sinv/algorithms/rgf/rgf.py:17-64 (rgf) in the
// block-array form of src/sinv/algorithms/rgf/rgf2sided.py:18-24.
//
// Teams: one CTA walks the whole sweep for small blocks (everything stays on
// one SM, barriers are __syncthreads); larger blocks use the whole GPU as one
// team (cooperative launch, one or two CTAs per SM, bounded grid barriers).
#include <cstdio>
#include <mutex>

#include "rgf_sweep.cuh"
#include "host_util.h"

namespace sinvb {

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) rgf_cta_kernel(RgfParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamCta team;
  rgf_sweep<T, BM, BN>(team, p, reinterpret_cast<T*>(smem_raw));
}

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) rgf_grid_kernel(RgfParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamDyn team{&p.hdr->barrier_count, p.status, (int)blockIdx.x, (int)gridDim.x, 0u};
  rgf_sweep<T, BM, BN>(team, p, reinterpret_cast<T*>(smem_raw));
}

// Elementwise precision conversion (float <-> double, complex handled as 2x floats).
__global__ void widen_kernel(const float* __restrict__ src, double* __restrict__ dst, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
__global__ void narrow_kernel(const double* __restrict__ src, float* __restrict__ dst, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

template <class T, int BM, int BN>
constexpr size_t sweep_smem_bytes() {
  size_t g = (size_t)gemm_smem_elems<T, BM, BN>() * sizeof(T);
  size_t j = sizeof(GjShared<T>);
  return g > j ? g : j;
}

struct RgfLayout {
  size_t X, P, T0, T1, T2, T3, Winv, wide_in, wide_out, total;
};

// Workspace layout (bytes, 256-aligned pieces after the 256-byte header).
static RgfLayout rgf_layout(int n, int b, int dtype, unsigned flags) {
  const size_t es = (dtype == SINVB_C128 || dtype == SINVB_C64) ? 16 : 8;
  const size_t bb = (size_t)b * b;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  RgfLayout L{};
  size_t off = sizeof(WsHeader);
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  if (!save) {
    L.X = take((size_t)(n - 1) * bb * es);
    L.P = take((size_t)(n - 1) * bb * es);
  }
  L.T0 = take(bb * es);
  L.T1 = take(bb * es);
  if (flags & SINVB_INPLACE) {
    L.T2 = take(bb * es);
    L.T3 = take(bb * es);
  }
  L.Winv = take(invert_side_elems(b) * es);
  if (dtype == SINVB_C64 || dtype == SINVB_F32) {
    L.wide_in = take((size_t)(3 * n - 2) * bb * es);
    L.wide_out = take((size_t)(save ? 3 * n - 2 : n) * bb * es);
  }
  L.total = off;
  return L;
}

template <class T, int BM, int BN>
static int launch_sweep(const RgfParams<T>& p, bool grid, cudaStream_t stream) {
  constexpr size_t smem = sweep_smem_bytes<T, BM, BN>();
  void* args[] = {(void*)&p};
  if (!grid) {
    auto k = rgf_cta_kernel<T, BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SINVB_CUDA(cudaLaunchKernel((const void*)k, dim3(1), dim3(kThreads), args, smem, stream));
  } else {
    auto k = rgf_grid_kernel<T, BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SINVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem));
    if (per_sm < 1) return SINVB_EUNSUPPORTED;
    int grid_ctas = device_sm_count() * (per_sm > 2 ? 2 : per_sm);
    SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(grid_ctas), dim3(kThreads), args, smem, stream));
  }
  return SINVB_OK;
}

// Team and tile choice for one matrix.
static bool use_grid_team(int b, unsigned flags) {
  if (flags & SINVB_FORCE_GRID) return true;
  if (flags & SINVB_FORCE_CTA) return false;
  return b > 48;
}

template <class T>
static int run_rgf(const T* diag, const T* upper, const T* lower, int n, int b, unsigned flags, T* Gd, T* Gu,
                   T* Gl, unsigned char* ws, const RgfLayout& L, cudaStream_t stream, T* ckpt = nullptr,
                   int ckpt_every = 1) {
  RgfParams<T> p;
  p.ckpt = ckpt;
  p.ckpt_every = ckpt_every;
  p.oz_digits = 0;
  p.oz_scratch = nullptr;
  p.oz = nullptr;
  p.diag = diag;
  p.upper = upper;
  p.lower = lower;
  const bool inplace = flags & SINVB_INPLACE;
  p.Gd = inplace ? const_cast<T*>(diag) : Gd;
  p.Gu = inplace ? const_cast<T*>(upper) : Gu;
  p.Gl = inplace ? const_cast<T*>(lower) : Gl;
  Gu = p.Gu;
  Gl = p.Gl;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  p.X = save ? Gl : reinterpret_cast<T*>(ws + L.X);
  p.P = save ? Gu : reinterpret_cast<T*>(ws + L.P);
  p.T0 = reinterpret_cast<T*>(ws + L.T0);
  p.T1 = reinterpret_cast<T*>(ws + L.T1);
  p.T2 = inplace ? reinterpret_cast<T*>(ws + L.T2) : nullptr;
  p.T3 = inplace ? reinterpret_cast<T*>(ws + L.T3) : nullptr;
  p.Winv = reinterpret_cast<T*>(ws + L.Winv);
  p.hdr = reinterpret_cast<WsHeader*>(ws);
  p.status = &p.hdr->status;
  p.n = n;
  p.b = b;
  p.flags = flags;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), stream));
  const bool grid = use_grid_team(b, flags);
  if (b <= 32 || grid) return launch_sweep<T, 32, 32>(p, grid, stream);
  return launch_sweep<T, 64, 64>(p, grid, stream);
}

static int check_args(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                      const void* Gd, const void* Gu, const void* Gl, const void* ws, size_t ws_bytes, int dtype) {
  const bool inplace = flags & SINVB_INPLACE;
  if (n < 1 || b < 1 || !diag || !ws) return SINVB_EINVAL;
  if (!inplace && !Gd) return SINVB_EINVAL;
  if (n > 1 && (!upper || !lower)) return SINVB_EINVAL;
  if (!inplace && (flags & SINVB_SAVE_OFFDIAG) && n > 1 && (!Gu || !Gl)) return SINVB_EINVAL;
  if (inplace && (!(flags & SINVB_SAVE_OFFDIAG) || dtype == SINVB_C64 || dtype == SINVB_F32)) return SINVB_EINVAL;
  if ((flags & SINVB_FORCE_GRID) && (flags & SINVB_FORCE_CTA)) return SINVB_EINVAL;
  if ((uintptr_t)ws % 256 != 0) return SINVB_EWORKSPACE;
  if (ws_bytes < rgf_layout(n, b, dtype, flags).total) return SINVB_EWORKSPACE;
  const size_t align = (dtype == SINVB_C128) ? 16 : (dtype == SINVB_F32 ? 4 : 8);
  for (const void* q : {diag, upper, lower, Gd, Gu, Gl})
    if (q && (uintptr_t)q % align != 0) return SINVB_EINVAL;
  return check_device();
}

// Single precision: widen into the workspace, run the FP64 sweep, round back.
template <class T>
int rgf_single(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                      void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                      cudaStream_t stream, int dtype) {
  int rc = check_args(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes, dtype);
  if (rc) return rc;
  const RgfLayout L = rgf_layout(n, b, dtype, flags);
  unsigned char* ws = (unsigned char*)workspace;
  const size_t per = (Elem<T>::kComplex ? 2 : 1);  // floats per element
  const size_t bb = (size_t)b * b;
  const bool save = flags & SINVB_SAVE_OFFDIAG;
  T* win = reinterpret_cast<T*>(ws + L.wide_in);
  T* wout = reinterpret_cast<T*>(ws + L.wide_out);
  const int cgrid = 4 * device_sm_count();
  widen_kernel<<<cgrid, 256, 0, stream>>>((const float*)diag, (double*)win, n * bb * per);
  if (n > 1) {
    widen_kernel<<<cgrid, 256, 0, stream>>>((const float*)upper, (double*)(win + n * bb), (n - 1) * bb * per);
    widen_kernel<<<cgrid, 256, 0, stream>>>((const float*)lower, (double*)(win + (2 * n - 1) * bb),
                                            (n - 1) * bb * per);
  }
  SINVB_CUDA(cudaGetLastError());
  T* gd = wout;
  T* gu = save ? wout + n * bb : nullptr;
  T* gl = save ? wout + (2 * n - 1) * bb : nullptr;
  rc = run_rgf<T>(win, win + n * bb, win + (2 * n - 1) * bb, n, b, flags, gd, gu, gl, ws, L, stream);
  if (rc) return rc;
  narrow_kernel<<<cgrid, 256, 0, stream>>>((const double*)gd, (float*)G_diag, n * bb * per);
  if (save && n > 1) {
    narrow_kernel<<<cgrid, 256, 0, stream>>>((const double*)gu, (float*)G_upper, (n - 1) * bb * per);
    narrow_kernel<<<cgrid, 256, 0, stream>>>((const double*)gl, (float*)G_lower, (n - 1) * bb * per);
  }
  SINVB_CUDA(cudaGetLastError());
  return SINVB_OK;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_rgf_workspace_size(int n, int b, int dtype, unsigned flags) {
  if (n < 1 || b < 1 || dtype < 0 || dtype > 3) return 0;
  return rgf_layout(n, b, dtype, flags).total;
}

int sinvb_rgf_z(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  int rc = check_args(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                      SINVB_C128);
  if (rc) return rc;
  return run_rgf<cplx>((const cplx*)diag, (const cplx*)upper, (const cplx*)lower, n, b, flags, (cplx*)G_diag,
                       (cplx*)G_upper, (cplx*)G_lower, (unsigned char*)workspace,
                       rgf_layout(n, b, SINVB_C128, flags), (cudaStream_t)stream);
}

int sinvb_rgf_d(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  int rc = check_args(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                      SINVB_F64);
  if (rc) return rc;
  return run_rgf<double>((const double*)diag, (const double*)upper, (const double*)lower, n, b, flags,
                         (double*)G_diag, (double*)G_upper, (double*)G_lower, (unsigned char*)workspace,
                         rgf_layout(n, b, SINVB_F64, flags), (cudaStream_t)stream);
}

int sinvb_rgf_c(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  return rgf_single<cplx>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                          (cudaStream_t)stream, SINVB_C64);
}

int sinvb_rgf_s(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  return rgf_single<double>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                            (cudaStream_t)stream, SINVB_F32);
}

}  // extern "C"

// Forward sweep that also saves the adjoint's checkpoints g_{s*c-1} -> ckpt[s-1].
template <class T>
static int rgf_ckpt(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                    void* G_diag, void* G_upper, void* G_lower, void* ckpt, int every, void* workspace,
                    size_t workspace_bytes, cudaStream_t stream, int dtype) {
  if (!(flags & SINVB_SAVE_OFFDIAG) || (flags & SINVB_INPLACE) || every < 1) return SINVB_EINVAL;
  if ((n - 1) / every >= 1 && !ckpt) return SINVB_EINVAL;
  int rc = check_args(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes, dtype);
  if (rc) return rc;
  return run_rgf<T>((const T*)diag, (const T*)upper, (const T*)lower, n, b, flags, (T*)G_diag, (T*)G_upper,
                    (T*)G_lower, (unsigned char*)workspace, rgf_layout(n, b, dtype, flags), stream, (T*)ckpt, every);
}

extern "C" {

int sinvb_rgf_forward_ckpt_z(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                             void* G_diag, void* G_upper, void* G_lower, void* checkpoints, int every,
                             void* workspace, size_t workspace_bytes, sinvb_stream_t stream) {
  return rgf_ckpt<cplx>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, checkpoints, every, workspace,
                        workspace_bytes, (cudaStream_t)stream, SINVB_C128);
}

int sinvb_rgf_forward_ckpt_d(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                             void* G_diag, void* G_upper, void* G_lower, void* checkpoints, int every,
                             void* workspace, size_t workspace_bytes, sinvb_stream_t stream) {
  return rgf_ckpt<double>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, checkpoints, every, workspace,
                          workspace_bytes, (cudaStream_t)stream, SINVB_F64);
}

}  // extern "C"
