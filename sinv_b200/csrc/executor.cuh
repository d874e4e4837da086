// A schedule executor: a persistent cooperative kernel that runs a host-built
// list of phases.  Each phase is a set of independent work units (GEMM output
// tiles, small Gauss-Jordan inversions, block copies); phases are separated
// by a grid barrier.  The BCR selected inversion, whose reductions and
// productions are independent across the rows of a level
// (src/sinv/algorithms/bcr/bcr_serial.py:207-212, :437-466), runs as one such
// schedule on the whole GPU.
#pragma once

#include "block_inverse.cuh"

namespace sinvb {

enum ExecKind : int { kExecGemm = 0, kExecGj = 1, kExecCopy = 2 };

// One operation of a phase.  GEMM: C = D + alpha (A B [+ A2 B2]).  GJ: invert
// the M x M block at C (ldc) in place, M <= 64.  COPY: C[M x N] = A (lda),
// transposed when `transpose` is set.
struct ExecOp {
  int kind;
  int M, N, K, K2;
  int lda, ldb, ldd, ldc, lda2, ldb2;
  int transpose;
  int unit_start;  // first work unit of the op within its phase
  int inst;        // status word of the op (the matrix it belongs to in a batch)
  double alpha;
  const void* A;
  const void* B;
  const void* D;
  void* C;
  const void* A2;
  const void* B2;
};
static_assert(sizeof(ExecOp) == 112, "112-byte ops");

struct ExecPhase {
  int op_begin, op_end;  // ops [op_begin, op_end) of the op table
  int units;             // work units in the phase
  int pad;
};

constexpr int kCopyChunk = 4096;  // elements per copy work unit

__host__ __device__ inline int exec_tiles(int M, int N, int bm, int bn) {
  return (M <= 0 || N <= 0) ? 0 : ((M + bm - 1) / bm) * ((N + bn - 1) / bn);
}

__host__ __device__ inline int exec_units(const ExecOp& o, int bm, int bn) {
  if (o.kind == kExecGemm) return exec_tiles(o.M, o.N, bm, bn);
  if (o.kind == kExecGj) return 1;
  long long elems = (long long)o.M * o.N;
  return (int)((elems + kCopyChunk - 1) / kCopyChunk);
}

template <class T, int BM, int BN>
__device__ void exec_unit(const ExecOp& o, int u, int* status, T* smem) {
  if (o.kind == kExecGemm) {
    GemmOp<T> g = make_op<T>(o.M, o.N, o.K, o.alpha, (const T*)o.A, o.lda, (const T*)o.B, o.ldb, (const T*)o.D,
                             o.ldd, (T*)o.C, o.ldc);
    g.A2 = (const T*)o.A2;
    g.B2 = (const T*)o.B2;
    g.lda2 = o.lda2;
    g.ldb2 = o.ldb2;
    g.K2 = o.K2;
    const int tn = (o.N + BN - 1) / BN;
    cta_gemm_tile<T, BM, BN>(g, u / tn, u % tn, smem);
  } else if (o.kind == kExecGj) {
    cta_gj_invert<T>((T*)o.C, o.ldc, o.M, status + o.inst, smem);
  } else {
    const T* src = (const T*)o.A;
    T* dst = (T*)o.C;
    const long long total = (long long)o.M * o.N;
    const long long e0 = (long long)u * kCopyChunk;
    const long long e1 = e0 + kCopyChunk < total ? e0 + kCopyChunk : total;
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      int i = (int)(e / o.N), j = (int)(e % o.N);
      if (o.transpose)
        dst[(size_t)j * o.ldc + i] = src[(size_t)i * o.lda + j];
      else
        dst[(size_t)i * o.ldc + j] = src[(size_t)i * o.lda + j];
    }
  }
}

// Runs every phase with the whole team.  Units of a phase are dealt round-robin
// over the team's CTAs; the op of a unit is found by binary search on
// unit_start.  A singular block is reported in status[op.inst].  Returns false
// when a barrier gave up.
template <class T, int BM, int BN, class Team>
__device__ bool run_schedule(Team& team, const ExecOp* ops, const ExecPhase* phases, int nphases, int* status,
                             T* smem) {
  for (int ph = 0; ph < nphases; ph++) {
    const ExecPhase P = phases[ph];
    for (int u = team.rank(); u < P.units; u += team.size()) {
      int lo = P.op_begin, hi = P.op_end - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ops[mid].unit_start <= u) lo = mid; else hi = mid - 1;
      }
      const ExecOp o = ops[lo];
      exec_unit<T, BM, BN>(o, u - o.unit_start, status, smem);
    }
    if (!team.sync()) return false;
  }
  return true;
}

}  // namespace sinvb
