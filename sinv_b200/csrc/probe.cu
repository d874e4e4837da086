// FP64 tensor-core peak probe (a measurement aid for roofline figures; no
// counterpart in the reference).
//
// B200 has no FP64 kind of tcgen05.mma, so the FP64 tensor ceiling of the
// selected-inversion kernels is the warp-level DMMA rate.  The probe runs
// independent mma.sync.m8n8k4.f64 chains on every SM (8 warps per CTA, two CTAs
// per SM, register operands only, no memory traffic) and times them with CUDA
// events on the caller's stream.
#include "common.cuh"
#include "host_util.h"

namespace sinvb {

constexpr int kProbeChains = 8;

// Written only when the kernel argument `keep` is non-zero (never, in practice);
// the unknown-at-compile-time store keeps the MMA chains from being removed.
static __device__ double g_probe_sink;

__global__ void __launch_bounds__(256) dmma_probe_kernel(int iters, int keep) {
  double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4;
  double c[kProbeChains][2];
#pragma unroll
  for (int i = 0; i < kProbeChains; i++) c[i][0] = c[i][1] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < kProbeChains; i++) dmma884(c[i][0], c[i][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kProbeChains; i++) s += c[i][0] + c[i][1];
  if (keep) g_probe_sink = s;
}

}  // namespace sinvb

using namespace sinvb;

extern "C" int sinvb_fp64_mma_peak(int iters, double* tflops, sinvb_stream_t stream) {
  if (iters < 1 || !tflops) return SINVB_EINVAL;
  int rc = check_device();
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = 2 * device_sm_count(), block = 256;
  cudaEvent_t e0, e1;
  SINVB_CUDA(cudaEventCreate(&e0));
  SINVB_CUDA(cudaEventCreate(&e1));
  dmma_probe_kernel<<<grid, block, 0, s>>>(iters / 4 + 1, 0);  // warm-up
  SINVB_CUDA(cudaEventRecord(e0, s));
  dmma_probe_kernel<<<grid, block, 0, s>>>(iters, 0);
  SINVB_CUDA(cudaGetLastError());
  SINVB_CUDA(cudaEventRecord(e1, s));
  SINVB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SINVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double flops = 2.0 * 8 * 8 * 4 * kProbeChains * (double)iters * (grid * block / 32);
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SINVB_OK;
}
