// Host-built executor schedules (executor.cuh) and the kernel that runs one
// uploaded into a workspace: the BCR selected inversion (bcr.cu) and the PDIV
// selected inversion (pdiv.cu) are both such schedules.
#pragma once

#include <algorithm>
#include <vector>

#include "executor.cuh"
#include "host_util.h"

namespace sinvb {

// Host-side builder of an executor schedule.
struct Sched {
  std::vector<ExecOp> ops;
  std::vector<ExecPhase> phases;
  int bm, bn;
  int cur_units = 0;

  void begin() {
    ExecPhase p{};
    p.op_begin = p.op_end = (int)ops.size();
    phases.push_back(p);
    cur_units = 0;
  }
  void push(ExecOp o) {
    o.unit_start = cur_units;
    int u = exec_units(o, bm, bn);
    if (u == 0) return;
    cur_units += u;
    ops.push_back(o);
    phases.back().op_end = (int)ops.size();
    phases.back().units = cur_units;
  }
  // C = D + alpha (A B [+ A2 B2]); all blocks m x m with leading dimension ld.
  void gemm(int m, double alpha, const void* A, const void* B, const void* D, void* C, const void* A2 = nullptr,
            const void* B2 = nullptr, int ld = -1, int M = -1, int N = -1, int K = -1, int lda = -1, int ldb = -1,
            int ldc = -1, int ldd = -1) {
    ExecOp o{};
    o.kind = kExecGemm;
    o.M = M < 0 ? m : M;
    o.N = N < 0 ? m : N;
    o.K = K < 0 ? m : K;
    int l = ld < 0 ? m : ld;
    o.lda = lda < 0 ? l : lda;
    o.ldb = ldb < 0 ? l : ldb;
    o.ldc = ldc < 0 ? l : ldc;
    o.ldd = ldd < 0 ? l : ldd;
    o.alpha = alpha;
    o.A = A; o.B = B; o.D = D; o.C = C;
    if (A2) {
      o.A2 = A2; o.B2 = B2;
      o.K2 = o.K; o.lda2 = o.lda; o.ldb2 = o.ldb;
    }
    push(o);
  }
  void gj(int m, void* blk, int ld) {
    ExecOp o{};
    o.kind = kExecGj;
    o.M = m;
    o.ldc = ld;
    o.C = blk;
    push(o);
  }
  void copy(int rows, int cols, const void* src, int lds, void* dst, int ldd, bool transpose = false) {
    ExecOp o{};
    o.kind = kExecCopy;
    o.M = rows;
    o.N = cols;
    o.lda = lds;
    o.ldc = ldd;
    o.transpose = transpose;
    o.A = src;
    o.C = dst;
    push(o);
  }
};

// Phases of a blocked Gauss-Jordan inversion (the schedule form of
// team_invert) of every m x m block in blks; side[x] holds the W / R panels of
// block x (invert_side_elems(m) elements).
template <class T>
void invert_many(Sched& s, const std::vector<T*>& blks, const std::vector<T*>& side, int m) {
  if (blks.empty()) return;
  if (m <= kGjMax) {
    s.begin();
    for (T* a : blks) s.gj(m, a, m);
    return;
  }
  const int np = (m + kPanel - 1) / kPanel;
  int pK0 = -1, pkb = 0;
  auto W = [&](size_t x) { return side[x]; };
  auto R = [&](size_t x) { return side[x] + (size_t)m * kPanel; };
  auto write_back = [&](size_t x) {
    T* a = blks[x];
    const int r1 = pK0 + pkb;
    s.copy(pK0, pkb, W(x), kPanel, a + pK0, m);
    s.copy(m - r1, pkb, W(x) + (size_t)r1 * kPanel, kPanel, a + (size_t)r1 * m + pK0, m);
    s.copy(pkb, pK0, R(x), m, a + (size_t)pK0 * m, m);
    s.copy(pkb, m - r1, R(x) + r1, m, a + (size_t)pK0 * m + r1, m);
  };
  for (int p = 0; p < np; p++) {
    const int K0 = p * kPanel, kb = std::min(kPanel, m - K0), right = K0 + kb;
    s.begin();
    for (size_t x = 0; x < blks.size(); x++) {
      s.gj(kb, blks[x] + (size_t)K0 * m + K0, m);
      if (pK0 >= 0) write_back(x);
    }
    s.begin();
    for (size_t x = 0; x < blks.size(); x++) {
      T* a = blks[x];
      T* Dinv = a + (size_t)K0 * m + K0;
      T* row = a + (size_t)K0 * m;
      s.gemm(m, 1.0, Dinv, row, nullptr, R(x), nullptr, nullptr, m, kb, K0, kb);
      s.gemm(m, 1.0, Dinv, row + right, nullptr, R(x) + right, nullptr, nullptr, m, kb, m - right, kb);
    }
    s.begin();
    for (size_t x = 0; x < blks.size(); x++) {
      T* a = blks[x];
      T* Dinv = a + (size_t)K0 * m + K0;
      int rs[2] = {0, right}, rn[2] = {K0, m - right};
      for (int ri = 0; ri < 2; ri++) {
        T* colK = a + (size_t)rs[ri] * m + K0;
        for (int ci = 0; ci < 2; ci++) {
          T* C = a + (size_t)rs[ri] * m + rs[ci];
          s.gemm(m, -1.0, colK, R(x) + rs[ci], C, C, nullptr, nullptr, m, rn[ri], rn[ci], kb);
        }
        s.gemm(m, -1.0, colK, Dinv, nullptr, W(x) + (size_t)rs[ri] * kPanel, nullptr, nullptr, m, rn[ri], kb, kb,
               m, m, kPanel);
      }
    }
    pK0 = K0;
    pkb = kb;
  }
  s.begin();
  for (size_t x = 0; x < blks.size(); x++) write_back(x);
}


// Body of a schedule kernel.  The workspace holds a WsHeader whose
// desc_offset / items_offset locate the op table and the phases.  One matrix
// (hdr->count == 0): singular blocks are reported in the header's status word.
// A batch (hdr->count > 0): op.inst indexes one status word per matrix at
// hdr->slots_offset, copied to the caller's array at the end.  nphases < 0:
// the phase count stored in the header (a re-run).
template <class T, int BM, int BN>
__device__ __forceinline__ void run_uploaded_schedule(unsigned char* ws, int nphases) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WsHeader* hdr = reinterpret_cast<WsHeader*>(ws);
  if (nphases < 0) nphases = hdr->sched_phases;
  const ExecOp* ops = reinterpret_cast<const ExecOp*>(ws + hdr->desc_offset);
  const ExecPhase* phases = reinterpret_cast<const ExecPhase*>(ws + hdr->items_offset);
  const int count = hdr->count;
  int* op_status = count > 0 ? reinterpret_cast<int*>(ws + hdr->slots_offset) : &hdr->status;
  TeamDyn team{&hdr->barrier_count, &hdr->status, (int)blockIdx.x, (int)gridDim.x, 0u};
  const bool ok = run_schedule<T, BM, BN>(team, ops, phases, nphases, op_status, reinterpret_cast<T*>(smem_raw));
  if (count > 0 && blockIdx.x == 0) {
    for (int k = threadIdx.x; k < count; k += blockDim.x) {
      int st = *((volatile int*)&op_status[k]);
      if (!ok && st == 0) st = SINVB_STATUS_TIMEOUT;
      if (hdr->inst_status) hdr->inst_status[k] = st;
      if (st) report(&hdr->status, st);
    }
  }
}

// Cooperative launch of a schedule kernel on every SM.
template <class T, int BM, int BN>
int launch_schedule_kernel(void (*k)(unsigned char*, int), unsigned char* ws, int nphases, cudaStream_t stream) {
  constexpr size_t g = (size_t)gemm_smem_elems<T, BM, BN>() * sizeof(T);
  constexpr size_t smem = g > sizeof(GjShared<T>) ? g : sizeof(GjShared<T>);
  SINVB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  void* args[] = {(void*)&ws, (void*)&nphases};
  SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)k, dim3(device_sm_count()), dim3(kThreads), args, smem,
                                         stream));
  return SINVB_OK;
}

}  // namespace sinvb
