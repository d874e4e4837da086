// Library-wide entry points of libsinvb: version, status strings, device
// checks, workspace status read-back.
#include <cstring>

#include "common.cuh"
#include "host_util.h"

namespace sinvb {

static thread_local cudaError_t g_last_cuda = cudaSuccess;
void set_last_cuda_error(cudaError_t e) { g_last_cuda = e; }

constexpr int kMaxDevices = 64;
static int g_sm_count[kMaxDevices];
static int g_dev_ok[kMaxDevices];  // 0 unknown, 1 ok, -1 unsupported

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  if (!g_sm_count[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_sm_count[dev] = n > 0 ? n : 148;
  }
  return g_sm_count[dev];
}

int check_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_cuda_error(e);
    return SINVB_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return SINVB_EUNSUPPORTED;
  if (!g_dev_ok[dev]) {
    int major = 0, coop = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    g_dev_ok[dev] = (major == 10 && coop) ? 1 : -1;
  }
  return g_dev_ok[dev] == 1 ? SINVB_OK : SINVB_EUNSUPPORTED;
}

}  // namespace sinvb

extern "C" {

int sinvb_version(void) { return 110; }

const char* sinvb_status_string(int code) {
  switch (code) {
    case SINVB_OK: return "ok";
    case SINVB_EINVAL: return "invalid argument";
    case SINVB_ECUDA: return cudaGetErrorString(sinvb::g_last_cuda);
    case SINVB_EWORKSPACE: return "workspace too small or not 256-byte aligned";
    case SINVB_EUNSUPPORTED: return "no sm_100 (B200) device with cooperative launch";
    case SINVB_STATUS_PIVOT: return "zero or non-finite pivot in a pivot-free block inversion";
    case SINVB_STATUS_TIMEOUT: return "a bounded device wait gave up";
    default: return "unknown status";
  }
}

int sinvb_workspace_status(const void* workspace, sinvb_stream_t stream, int* status) {
  if (!workspace || !status) return SINVB_EINVAL;
  sinvb::WsHeader h;
  SINVB_CUDA(cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  SINVB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  *status = h.status;
  return SINVB_OK;
}

}  // extern "C"
