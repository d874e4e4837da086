// Standalone mixed-precision complex GEMM on the int8 tensor cores (Ozaki
// scheme, ozaki.cuh): C = beta D + alpha A B with FP64 complex operands and a
// chosen number of digits.  The selected-inversion sweeps use the same device
// routines for their block products in SINVB_PREC_MIXED mode.
#include "host_util.h"
#include "ozaki.cuh"

namespace sinvb {

// Workspace: the status header, then the exponents and digit planes in the
// order oz_bind lays them out.
static size_t oz_workspace_bytes(int M, int N, int K, int S) { return sizeof(WsHeader) + oz_op_scratch(M, N, K, S); }

// Digits of both operands: CTAs [0, ctas_a) take groups of 8 A rows, the
// others 32-column blocks of B.
__global__ void __launch_bounds__(256) oz_slice_kernel(GemmOp<cplx> g, OzOp op, int ctas_a) {
  extern __shared__ __align__(16) unsigned char slice_smem[];
  if ((int)blockIdx.x < ctas_a)
    oz_slice_ops(op.s.S, &g, &op, 1, 1u, 0u, blockIdx.x, ctas_a, 0, 1, slice_smem);
  else
    oz_slice_ops(op.s.S, &g, &op, 1, 0u, 1u, 0, 1, blockIdx.x - ctas_a, gridDim.x - ctas_a, slice_smem);
}

// Persistent over output tiles: every CTA allocates TMEM once and walks tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(256, 1) oz_gemm_kernel(OzOp op, int* status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ OzState st;
  oz_setup(&st);
  oz_tiles(&op, 1, blockIdx.x, gridDim.x, &st, smem, status);
  oz_teardown(&st);
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_zgemm_ozaki_workspace_size(int M, int N, int K, int digits) {
  if (M < 1 || N < 1 || K < 1 || digits < 1 || digits > kOzMaxDigits) return 0;
  return oz_workspace_bytes(M, N, K, digits);
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
  if (workspace_bytes < oz_workspace_bytes(M, N, K, digits)) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  cudaStream_t st = (cudaStream_t)stream;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), st));
  const int sms = device_sm_count();
  OzOp op;
  oz_bind(op, M, N, K, digits, ws + sizeof(WsHeader), alpha, beta, (const cplx*)D, ldd, (cplx*)C, ldc);
  int ctas_a = (M + 7) / 8;  // one CTA per group of 8 rows
  if (ctas_a > sms) ctas_a = sms;
  int ctas_b = (N + 31) / 32;  // one CTA per 32-column block
  if (ctas_b > sms) ctas_b = sms;
  const GemmOp<cplx> g = make_op<cplx>(M, N, K, alpha, (const cplx*)A, lda, (const cplx*)B, ldb, (const cplx*)D, ldd,
                                       (cplx*)C, ldc);
  const size_t slice_smem = oz_slice_smem(digits);
  SINVB_CUDA(cudaFuncSetAttribute(oz_slice_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)slice_smem));
  oz_slice_kernel<<<ctas_a + ctas_b, 256, slice_smem, st>>>(g, op, ctas_a);
  SINVB_CUDA(cudaGetLastError());
  const size_t smem = oz_smem_bytes(digits);
  SINVB_CUDA(cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int tiles = op.tiles;
  const int grid = tiles < sms ? tiles : sms;
  oz_gemm_kernel<<<grid, 256, smem, st>>>(op, &((WsHeader*)ws)->status);
  SINVB_CUDA(cudaGetLastError());
  return SINVB_OK;
}

}  // extern "C"
