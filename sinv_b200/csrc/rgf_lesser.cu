// Lesser Green's function in the RGF sweeps: G< = G Sigma< G^H on the
// tridiagonal blocks, for a block-diagonal Sigma< (the lesser self-energy of
// contacts or scattering).  No reference counterpart: this is the step a
// transport code takes after rgf (src/sinv/algorithms/rgf/rgf.py:17-64) in
// its energy loop.  The recursions (derived from the block elimination of
// rgf.py:44-62; every term checked against dense G Sigma< G^H):
//
//   forward   g<_i = g_i (Sigma<_i + L_i g<_{i-1} L_i^H) g_i^H
//   backward  W = G_{i+1} L_{i+1},  Y = X_i W g<_i,  X_i = g_i U_i
//             G<_ii      = g<_i + X_i G<_{i+1} X_i^H + Y - Y^H      (g< is anti-Hermitian)
//             G<_{i,i+1} = -g<_i W^H - X_i G<_{i+1}
//             G<_{i+1,i} = -(G<_{i,i+1})^H
//
// with L_i = A_{i,i-1}, U_i = A_{i,i+1}.  The retarded blocks come out of the
// same sweep as in rgf_sweep.cuh (X_i kept in G_lower, P_{i+1} = L_{i+1} g_i
// in G_upper until the backward step).
#include "host_util.h"
#include "lesser_sweep.cuh"

namespace sinvb {

template <int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) lesser_cta_kernel(LesserParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamCta team;
  lesser_sweep<BM, BN>(team, p, reinterpret_cast<cplx*>(smem_raw));
}

template <int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) lesser_grid_kernel(LesserParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TeamDyn team{&p.hdr->barrier_count, p.status, (int)blockIdx.x, (int)gridDim.x, 0u};
  lesser_sweep<BM, BN>(team, p, reinterpret_cast<cplx*>(smem_raw));
}

static size_t lesser_ws(int b) {
  size_t off = sizeof(WsHeader);
  off += 5 * align_up((size_t)b * b * sizeof(cplx), 256);
  off += align_up(invert_side_elems(b) * sizeof(cplx), 256);
  return off;
}

template <int BM, int BN>
static int lesser_launch(const LesserParams& p, bool grid, cudaStream_t stream) {
  static_assert(BM == 32 || BM == 64, "tile");
  size_t smem = (size_t)gemm_smem_elems<cplx, BM, BN>() * sizeof(cplx);
  if (smem < sizeof(GjShared<cplx>)) smem = sizeof(GjShared<cplx>);
  void* args[] = {(void*)&p};
  if (!grid) {
    auto k = lesser_cta_kernel<BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SINVB_CUDA(cudaLaunchKernel((const void*)k, dim3(1), dim3(kThreads), args, smem, stream));
  } else {
    auto k = lesser_grid_kernel<BM, BN>;
    SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SINVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem));
    if (per_sm < 1) return SINVB_EUNSUPPORTED;
    const int g = device_sm_count() * (per_sm > 2 ? 2 : per_sm);
    SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(g), dim3(kThreads), args, smem, stream));
  }
  return SINVB_OK;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_rgf_lesser_workspace_size(int n, int b) {
  (void)n;
  return b < 1 ? 0 : lesser_ws(b);
}

int sinvb_rgf_lesser_z(const void* diag, const void* upper, const void* lower, const void* sigma_lesser, int n,
                       int b, unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* GL_diag,
                       void* GL_upper, void* workspace, size_t workspace_bytes, sinvb_stream_t stream) {
  if (n < 1 || b < 1 || !diag || !sigma_lesser || !G_diag || !GL_diag || !workspace) return SINVB_EINVAL;
  if (n > 1 && (!upper || !lower || !G_upper || !G_lower || !GL_upper)) return SINVB_EINVAL;
  if (flags & ~(SINVB_FORCE_CTA | SINVB_FORCE_GRID)) return SINVB_EINVAL;
  if ((flags & SINVB_FORCE_CTA) && (flags & SINVB_FORCE_GRID)) return SINVB_EINVAL;
  for (const void* q : {diag, upper, lower, sigma_lesser, (const void*)G_diag, (const void*)G_upper,
                        (const void*)G_lower, (const void*)GL_diag, (const void*)GL_upper})
    if (q && (uintptr_t)q % 16) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  if (workspace_bytes < lesser_ws(b)) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  cudaStream_t st = (cudaStream_t)stream;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), st));
  LesserParams p;
  p.diag = (const cplx*)diag;
  p.upper = (const cplx*)upper;
  p.lower = (const cplx*)lower;
  p.sig = (const cplx*)sigma_lesser;
  p.Gd = (cplx*)G_diag;
  p.Gu = (cplx*)G_upper;
  p.Gl = (cplx*)G_lower;
  p.GLd = (cplx*)GL_diag;
  p.GLu = (cplx*)GL_upper;
  size_t off = sizeof(WsHeader);
  for (int k = 0; k < 5; k++) {
    p.tmp[k] = reinterpret_cast<cplx*>(ws + off);
    off += align_up((size_t)b * b * sizeof(cplx), 256);
  }
  p.side = reinterpret_cast<cplx*>(ws + off);
  p.hdr = reinterpret_cast<WsHeader*>(ws);
  p.status = &p.hdr->status;
  p.n = n;
  p.b = b;
  const bool grid = (flags & SINVB_FORCE_GRID) || (!(flags & SINVB_FORCE_CTA) && b > 48);
  if (grid) return lesser_launch<64, 64>(p, true, st);  // the whole GPU: 64 x 64 tiles at every b
  return b <= 32 ? lesser_launch<32, 32>(p, false, st) : lesser_launch<64, 64>(p, false, st);
}

}  // extern "C"
