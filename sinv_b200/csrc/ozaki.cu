// Standalone mixed-precision complex GEMM on the int8 tensor cores (Ozaki
// scheme, ozaki.cuh): C = beta D + alpha A B with FP64 complex operands and a
// chosen number of digits.  The selected-inversion sweeps use the same device
// routines for their block products in SINVB_PREC_MIXED mode.
#include "host_util.h"
#include "ozaki.cuh"

namespace sinvb {

struct OzLayout {
  size_t ea, fb, ap, bp, total;
};

static OzLayout oz_layout(const OzShape& s) {
  OzLayout L{};
  size_t off = sizeof(WsHeader);
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  L.ea = take((size_t)s.M * 4);
  L.fb = take((size_t)s.N * 4);
  L.ap = take((size_t)s.S * s.a_plane());
  L.bp = take((size_t)s.S * s.b_plane());
  L.total = off;
  return L;
}

__global__ void __launch_bounds__(256) oz_slice_a_kernel(const cplx* A, int lda, OzShape s, int8_t* planes, int* ea) {
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  oz_slice_a(A, lda, s, planes, ea, gwarp, nwarps);
}
__global__ void __launch_bounds__(256) oz_slice_bexp_kernel(const cplx* B, int ldb, OzShape s, int* fb) {
  oz_slice_b_exponents(B, ldb, s, fb, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
__global__ void __launch_bounds__(256) oz_slice_bdig_kernel(const cplx* B, int ldb, OzShape s, int8_t* planes,
                                                            const int* fb) {
  oz_slice_b_digits(B, ldb, s, planes, fb, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Persistent over output tiles: every CTA allocates TMEM once and walks tiles.
__global__ void __launch_bounds__(256, 1) oz_gemm_kernel(OzOp op, int* status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ OzState st;
  oz_setup(&st);
  const int tiles_m = oz_pad(op.s.M, kOzTileM) / kOzTileM, tiles_n = op.s.Np / kOzTileN;
  for (int t = blockIdx.x; t < tiles_m * tiles_n; t += gridDim.x) {
    if (!oz_tile(op, t / tiles_n, t % tiles_n, &st, smem, status)) break;
  }
  oz_teardown(&st);
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_zgemm_ozaki_workspace_size(int M, int N, int K, int digits) {
  if (M < 1 || N < 1 || K < 1 || digits < 1 || digits > kOzMaxDigits) return 0;
  return oz_layout(oz_shape(M, N, K, digits)).total;
}

int sinvb_zgemm_ozaki(int M, int N, int K, double alpha, const void* A, int lda, const void* B, int ldb,
                      double beta, const void* D, int ldd, void* C, int ldc, int digits, void* workspace,
                      size_t workspace_bytes, sinvb_stream_t stream) {
  if (M < 1 || N < 1 || K < 1 || !A || !B || !C || !workspace) return SINVB_EINVAL;
  if (digits < 1 || digits > kOzMaxDigits || 2 * K > (1 << 14)) return SINVB_EINVAL;
  if (lda < K || ldb < N || ldc < N || (D && ldd < N)) return SINVB_EINVAL;
  for (const void* q : {A, B, D, (const void*)C})
    if (q && (uintptr_t)q % 16) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  const OzShape s = oz_shape(M, N, K, digits);
  const OzLayout L = oz_layout(s);
  if (workspace_bytes < L.total) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  cudaStream_t st = (cudaStream_t)stream;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), st));
  const int sms = device_sm_count();
  oz_slice_a_kernel<<<sms * 4, 256, 0, st>>>((const cplx*)A, lda, s, (int8_t*)(ws + L.ap), (int*)(ws + L.ea));
  oz_slice_bexp_kernel<<<(N + 255) / 256, 256, 0, st>>>((const cplx*)B, ldb, s, (int*)(ws + L.fb));
  oz_slice_bdig_kernel<<<sms * 4, 256, 0, st>>>((const cplx*)B, ldb, s, (int8_t*)(ws + L.bp),
                                                (const int*)(ws + L.fb));
  SINVB_CUDA(cudaGetLastError());
  OzOp op;
  op.a_planes = (const int8_t*)(ws + L.ap);
  op.b_planes = (const int8_t*)(ws + L.bp);
  op.ea = (const int*)(ws + L.ea);
  op.fb = (const int*)(ws + L.fb);
  op.s = s;
  op.D = (const cplx*)D;
  op.C = (cplx*)C;
  op.ldd = ldd;
  op.ldc = ldc;
  op.alpha = alpha;
  op.beta = beta;
  const size_t smem = oz_smem_bytes(digits);
  SINVB_CUDA(cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = (oz_pad(M, kOzTileM) / kOzTileM) * (s.Np / kOzTileN);
  const int grid = tiles < sms ? tiles : sms;
  oz_gemm_kernel<<<grid, 256, smem, st>>>(op, &((WsHeader*)ws)->status);
  SINVB_CUDA(cudaGetLastError());
  return SINVB_OK;
}

}  // extern "C"
