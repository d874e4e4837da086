// Parallel Schur reduction (PSR) selected inversion on one GPU.
//
// Reference: src/sinv/algorithms/psr/psr_seqsolve.py:20-943 with the
// partitioning of src/sinv/algorithms/psr/psr_utils.py:61-100.  The reference
// gives each of P MPI processes one partition of the block rows; here each
// partition is a team of CTAs of one cooperative launch:
//
//   1. every team reduces its partition (psr_seqsolve.py:127-310): the first
//      partition eliminates downwards, the last upwards, a central partition
//      downwards from its second row while keeping its top row t, which
//      gathers the fill-in couplings A[t,i] / A[i,t];
//   2. the whole grid gathers the reduced system (psr_seqsolve.py:313-467):
//      the boundary rows [bot_0, t_1, B_1, ..., t_{P-1}], which form a block
//      tridiagonal system of 2(P-1) blocks, and inverts it with an RGF sweep
//      (the reference inverts it densely, :470-493; only its tridiagonal
//      blocks are used afterwards);
//   3. every team produces its partition's blocks from the boundary blocks of
//      the inverse (psr_seqsolve.py:647-900).
//
// A single matrix then runs chains of about n/P steps per team plus 2(P-1)
// reduced steps instead of one chain of n.  Every block inverse is refined by
// one Newton step (refine_invert).  Inverse blocks are computed once
// in the reduction and kept (the production's inv(A_ii) is the same inversion
// of the same block, psr_seqsolve.py:737, :783, :860, :896).
//
// Storage (per block row i, b x b blocks in the workspace):
//   D[i]       reduced diagonal, inverted in place once eliminated
//   LA[i] UA[i]  first / central partitions: L[i,i-1], U[i-1,i];
//                last partition: L[i,i+1], U[i+1,i]
//   LT[j] UT[j]  central partitions: L[t,j], U[j,t]
//   FR[i] FC[i]  central partitions: fill-in A[t,i], A[i,t] (i >= t+2)
//   GR[i] GC[i]  central partitions: G[t,i], G[i,t] (i >= t+2)
#include <algorithm>
#include <cmath>

#include "block_inverse.cuh"
#include "host_util.h"

namespace sinvb {
namespace {

constexpr int kPsrMaxP = 32;

template <class T>
struct PsrParams {
  const T* diag;
  const T* upper;
  const T* lower;
  T* Gd;
  T* Gu;
  T* Gl;
  T* D;
  T* LA;
  T* UA;
  T* LT;
  T* UT;
  T* FR;
  T* FC;
  T* GR;
  T* GC;
  T* Rd;   // reduced system: R diagonal, R-1 upper, R-1 lower blocks
  T* Ru;
  T* Rl;
  T* RGd;  // its selected inverse
  T* RGu;
  T* RGl;
  T* T0;   // reduced sweep: T = -G_{i+1} P_{i+1}
  T* side;  // P + 1 inversion side buffers (one per team, one for the reduced sweep)
  size_t side_elems;
  T* work;  // P + 1 pairs of b x b blocks for the refined inversions
  unsigned* team_bar;  // P team barrier counters
  WsHeader* hdr;
  int* status;
  int n, b, P;
  int row0;  // global block row of element 0 of the row-indexed arrays (0 for a whole matrix)
};

// Partition k of n block rows over P (psr_utils.py:61-100): n / P rows each,
// the remainder in the first.
__host__ __device__ __forceinline__ int part_start(int n, int P, int k) {
  const int base = n / P;
  return k == 0 ? 0 : n - base * (P - k);
}
__host__ __device__ __forceinline__ int part_size(int n, int P, int k) {
  const int base = n / P;
  return k == 0 ? n - base * (P - 1) : base;
}

// Block of global row i in an array whose element 0 is global row row0.
template <class T>
struct Blk {
  T* base;
  size_t bb;
  int row0;
  __device__ __forceinline__ T* operator()(int i) const { return base + (size_t)(i - row0) * bb; }
};

// C = -(A B + A2 B2) (+ D when given)
template <class T>
__device__ __forceinline__ GemmOp<T> neg2(int b, const T* A, const T* B, const T* A2, const T* B2, const T* D, T* C) {
  GemmOp<T> o = make_op<T>(b, b, b, -1.0, A, b, B, b, D, b, C, b);
  return with_second<T>(o, A2, b, kOpN, B2, b, kOpN, 1);
}

// In-place inverse of the b x b block a, refined by one Newton step
// X1 = X0 + X0 (I - A X0) = 2 X0 - X0 (A X0).  The reference inverts with
// LAPACK (partial pivoting); team_invert is a pivot-free blocked Gauss-Jordan,
// whose error grows on the undamped indefinite blocks PSR inverts (a central
// partition's first eliminated block is E - H_ii as given), and the step
// squares its residual.  work: two b x b blocks.
template <class T, int BM, int BN, class Team>
__device__ bool refine_invert(Team& team, T* a, int b, T* work, T* side, int* status, GemmOp<T>* ops, T* smem) {
  T* X = work;
  T* AX = work + (size_t)b * b;
  team_copy<T>(team, b, b, a, b, X, b);
  if (!team.sync()) return false;
  if (!team_invert<T, BM, BN>(team, X, b, b, side, status, smem)) return false;
  ops[0] = make_op<T>(b, b, b, 1.0, a, b, X, b, nullptr, 0, AX, b);  // A X0
  team_gemm<T, BM, BN>(team, ops, 1, smem);
  if (!team.sync()) return false;
  ops[0] = make_op<T>(b, b, b, -1.0, X, b, AX, b, X, b, a, b);       // 2 X0 - X0 (A X0)
  ops[0].beta = 2.0;
  team_gemm<T, BM, BN>(team, ops, 1, smem);
  return team.sync();
}

// Partition reductions, psr_seqsolve.py:160-177 (first), :215-232 (last),
// :270-310 (central).  D[s .. s+m) starts as a copy of the diagonal.
template <class T, int BM, int BN, class Team>
__device__ bool psr_reduce(Team& team, const PsrParams<T>& p, int part, T* side, T* work, GemmOp<T>* ops,
                           T* smem) {
  const int b = p.b, P = p.P, s = part_start(p.n, P, part), m = part_size(p.n, P, part);
  const size_t bb = (size_t)b * b;
  const int r0 = p.row0;
  const Blk<T> D{p.D, bb, r0}, LA{p.LA, bb, r0}, UA{p.UA, bb, r0}, LT{p.LT, bb, r0}, UT{p.UT, bb, r0},
      FR{p.FR, bb, r0}, FC{p.FC, bb, r0};
  const Blk<const T> up{p.upper, bb, r0}, lo{p.lower, bb, r0};
  team_copy<T>(team, m * b, b, p.diag + (size_t)(s - r0) * bb, b, D(s), b);
  if (!team.sync()) return false;
  if (part == 0) {
    for (int i = s + 1; i < s + m; i++) {
      if (!refine_invert<T, BM, BN>(team, D(i - 1), b, work, side, p.status, ops, smem)) return false;
      ops[0] = make_op<T>(b, b, b, 1.0, lo(i - 1), b, D(i - 1), b, nullptr, 0, LA(i), b);  // L[i,i-1]
      ops[1] = make_op<T>(b, b, b, 1.0, D(i - 1), b, up(i - 1), b, nullptr, 0, UA(i), b);  // U[i-1,i]
      team_gemm<T, BM, BN>(team, ops, 2, smem);
      if (!team.sync()) return false;
      ops[0] = make_op<T>(b, b, b, -1.0, LA(i), b, up(i - 1), b, D(i), b, D(i), b);
      team_gemm<T, BM, BN>(team, ops, 1, smem);
      if (!team.sync()) return false;
    }
  } else if (part == P - 1) {
    for (int i = s + m - 2; i >= s; i--) {
      if (!refine_invert<T, BM, BN>(team, D(i + 1), b, work, side, p.status, ops, smem)) return false;
      ops[0] = make_op<T>(b, b, b, 1.0, up(i), b, D(i + 1), b, nullptr, 0, LA(i), b);  // L[i,i+1]
      ops[1] = make_op<T>(b, b, b, 1.0, D(i + 1), b, lo(i), b, nullptr, 0, UA(i), b);  // U[i+1,i]
      team_gemm<T, BM, BN>(team, ops, 2, smem);
      if (!team.sync()) return false;
      ops[0] = make_op<T>(b, b, b, -1.0, LA(i), b, lo(i), b, D(i), b, D(i), b);
      team_gemm<T, BM, BN>(team, ops, 1, smem);
      if (!team.sync()) return false;
    }
  } else {
    const int t = s;
    for (int i = t + 2; i < s + m; i++) {
      if (!refine_invert<T, BM, BN>(team, D(i - 1), b, work, side, p.status, ops, smem)) return false;
      const T* At = (i - 1 == t + 1) ? lo(t) : FC(i - 1);  // A[i-1,t]
      const T* Ta = (i - 1 == t + 1) ? up(t) : FR(i - 1);  // A[t,i-1]
      ops[0] = make_op<T>(b, b, b, 1.0, lo(i - 1), b, D(i - 1), b, nullptr, 0, LA(i), b);  // L[i,i-1]
      ops[1] = make_op<T>(b, b, b, 1.0, Ta, b, D(i - 1), b, nullptr, 0, LT(i - 1), b);      // L[t,i-1]
      ops[2] = make_op<T>(b, b, b, 1.0, D(i - 1), b, up(i - 1), b, nullptr, 0, UA(i), b);  // U[i-1,i]
      ops[3] = make_op<T>(b, b, b, 1.0, D(i - 1), b, At, b, nullptr, 0, UT(i - 1), b);      // U[i-1,t]
      team_gemm<T, BM, BN>(team, ops, 4, smem);
      if (!team.sync()) return false;
      ops[0] = make_op<T>(b, b, b, -1.0, LA(i), b, up(i - 1), b, D(i), b, D(i), b);       // A_ii
      ops[1] = make_op<T>(b, b, b, -1.0, LT(i - 1), b, At, b, D(t), b, D(t), b);          // A_tt
      ops[2] = make_op<T>(b, b, b, -1.0, LA(i), b, At, b, nullptr, 0, FC(i), b);          // A[i,t]
      ops[3] = make_op<T>(b, b, b, -1.0, LT(i - 1), b, up(i - 1), b, nullptr, 0, FR(i), b);  // A[t,i]
      team_gemm<T, BM, BN>(team, ops, 4, smem);
      if (!team.sync()) return false;
    }
  }
  return true;
}

// Partition productions, psr_seqsolve.py:694-737 (first), :740-783 (last),
// :786-900 (central).  The boundary blocks of G come from the reduced system.
template <class T, int BM, int BN, class Team>
__device__ bool psr_produce(Team& team, const PsrParams<T>& p, int part, GemmOp<T>* ops, T* smem) {
  const int b = p.b, P = p.P, s = part_start(p.n, P, part), m = part_size(p.n, P, part);
  const size_t bb = (size_t)b * b;
  const int r0 = p.row0;
  const Blk<T> D{p.D, bb, r0}, LA{p.LA, bb, r0}, UA{p.UA, bb, r0}, LT{p.LT, bb, r0}, UT{p.UT, bb, r0},
      GR{p.GR, bb, r0}, GC{p.GC, bb, r0};
  const Blk<T> Gd{p.Gd, bb, r0}, Gu{p.Gu, bb, r0}, Gl{p.Gl, bb, r0};
  if (part == 0) {
    for (int i = s + m - 1; i > s; i--) {
      ops[0] = make_op<T>(b, b, b, -1.0, Gd(i), b, LA(i), b, nullptr, 0, Gl(i - 1), b);  // G[i,i-1]
      ops[1] = make_op<T>(b, b, b, -1.0, UA(i), b, Gd(i), b, nullptr, 0, Gu(i - 1), b);  // G[i-1,i]
      team_gemm<T, BM, BN>(team, ops, 2, smem);
      if (!team.sync()) return false;
      ops[0] = make_op<T>(b, b, b, -1.0, UA(i), b, Gl(i - 1), b, D(i - 1), b, Gd(i - 1), b);
      team_gemm<T, BM, BN>(team, ops, 1, smem);
      if (!team.sync()) return false;
    }
  } else if (part == P - 1) {
    for (int i = s; i < s + m - 1; i++) {
      ops[0] = make_op<T>(b, b, b, -1.0, Gd(i), b, LA(i), b, nullptr, 0, Gu(i), b);  // G[i,i+1]
      ops[1] = make_op<T>(b, b, b, -1.0, UA(i), b, Gd(i), b, nullptr, 0, Gl(i), b);  // G[i+1,i]
      team_gemm<T, BM, BN>(team, ops, 2, smem);
      if (!team.sync()) return false;
      ops[0] = make_op<T>(b, b, b, -1.0, UA(i), b, Gu(i), b, D(i + 1), b, Gd(i + 1), b);
      team_gemm<T, BM, BN>(team, ops, 1, smem);
      if (!team.sync()) return false;
    }
  } else {
    const int t = s, B = s + m - 1;
    // G[t,j] / G[j,t] live in GR / GC, except G[t,t+1] / G[t+1,t], which are outputs
    auto Gtr = [&](int j) { return j == t + 1 ? Gu(t) : GR(j); };
    auto Gtc = [&](int j) { return j == t + 1 ? Gl(t) : GC(j); };
    {
      ops[0] = neg2<T>(b, GC(B), LT(B - 1), Gd(B), LA(B), nullptr, Gl(B - 1));       // G[B,B-1]
      ops[1] = neg2<T>(b, UA(B), Gd(B), UT(B - 1), GR(B), nullptr, Gu(B - 1));       // G[B-1,B]
      ops[2] = neg2<T>(b, Gd(t), LT(B - 1), GR(B), LA(B), nullptr, Gtr(B - 1));      // G[t,B-1]
      ops[3] = neg2<T>(b, UA(B), GC(B), UT(B - 1), Gd(t), nullptr, Gtc(B - 1));      // G[B-1,t]
      team_gemm<T, BM, BN>(team, ops, 4, smem);
      if (!team.sync()) return false;
    }
    for (int i = B - 1; i >= t + 2; i--) {
      {  // G_ii = inv(A_ii) - U[i,t] G[t,i] - U[i,i+1] G[i+1,i]
        ops[0] = neg2<T>(b, UT(i), GR(i), UA(i + 1), Gl(i), D(i), Gd(i));
        team_gemm<T, BM, BN>(team, ops, 1, smem);
        if (!team.sync()) return false;
      }
      ops[0] = neg2<T>(b, UT(i - 1), GR(i), UA(i), Gd(i), nullptr, Gu(i - 1));     // G[i-1,i]
      ops[1] = neg2<T>(b, GC(i), LT(i - 1), Gd(i), LA(i), nullptr, Gl(i - 1));     // G[i,i-1]
      ops[2] = neg2<T>(b, Gd(t), LT(i - 1), GR(i), LA(i), nullptr, Gtr(i - 1));    // G[t,i-1]
      ops[3] = neg2<T>(b, UA(i), GC(i), UT(i - 1), Gd(t), nullptr, Gtc(i - 1));    // G[i-1,t]
      team_gemm<T, BM, BN>(team, ops, 4, smem);
      if (!team.sync()) return false;
    }
    ops[0] = neg2<T>(b, UT(t + 1), Gu(t), UA(t + 2), Gl(t + 1), D(t + 1), Gd(t + 1));  // G[t+1,t+1]
    team_gemm<T, BM, BN>(team, ops, 1, smem);
    if (!team.sync()) return false;
  }
  return true;
}

// Selected inversion of the reduced system (R blocks in Rd / Ru / Rl) by the
// whole grid, the recursions of src/sinv/algorithms/rgf/rgf.py:44-62:
//   forward   X_{i-1} = g_{i-1} U_{i-1} (in RGl),  P_i = L_i g_{i-1} (in RGu),
//             g_i = (A_ii - P_i U_{i-1})^-1 (in RGd)
//   backward  T = -G_{i+1} P_{i+1};  G_{i,i+1} = -X_i G_{i+1};  G_ii = g_i - X_i T;
//             G_{i+1,i} = T
template <class T, int BM, int BN, class Team>
__device__ bool reduced_sweep(Team& all, const PsrParams<T>& p, int R, GemmOp<T>* ops, T* smem) {
  const int b = p.b;
  const size_t bb = (size_t)b * b;
  const Blk<T> A{p.Rd, bb, 0}, U{p.Ru, bb, 0}, L{p.Rl, bb, 0}, Gd{p.RGd, bb, 0}, Gu{p.RGu, bb, 0}, Gl{p.RGl, bb, 0};
  T* Winv = p.side + (size_t)p.P * p.side_elems;
  T* work = p.work + (size_t)p.P * 2 * bb;
  team_copy<T>(all, b, b, A(0), b, Gd(0), b);
  if (!all.sync()) return false;
  if (!refine_invert<T, BM, BN>(all, Gd(0), b, work, Winv, p.status, ops, smem)) return false;
  for (int i = 1; i < R; i++) {
    ops[0] = make_op<T>(b, b, b, 1.0, Gd(i - 1), b, U(i - 1), b, nullptr, 0, Gl(i - 1), b);
    ops[1] = make_op<T>(b, b, b, 1.0, L(i - 1), b, Gd(i - 1), b, nullptr, 0, Gu(i - 1), b);
    team_gemm<T, BM, BN>(all, ops, 2, smem);
    if (!all.sync()) return false;
    ops[0] = make_op<T>(b, b, b, -1.0, Gu(i - 1), b, U(i - 1), b, A(i), b, Gd(i), b);
    team_gemm<T, BM, BN>(all, ops, 1, smem);
    if (!all.sync()) return false;
    if (!refine_invert<T, BM, BN>(all, Gd(i), b, work, Winv, p.status, ops, smem)) return false;
  }
  for (int i = R - 2; i >= 0; i--) {
    ops[0] = make_op<T>(b, b, b, -1.0, Gd(i + 1), b, Gu(i), b, nullptr, 0, p.T0, b);
    team_gemm<T, BM, BN>(all, ops, 1, smem);
    if (!all.sync()) return false;
    ops[0] = make_op<T>(b, b, b, -1.0, Gl(i), b, Gd(i + 1), b, nullptr, 0, Gu(i), b);
    ops[1] = make_op<T>(b, b, b, -1.0, Gl(i), b, p.T0, b, Gd(i), b, Gd(i), b);
    team_gemm<T, BM, BN>(all, ops, 2, smem);
    if (!all.sync()) return false;
    team_copy<T>(all, b, b, p.T0, b, Gl(i), b);
    if (!all.sync()) return false;
  }
  return true;
}

// Block row of reduced row x: [bot_0, t_1, B_1, ..., t_{P-1}].
template <class T>
__device__ __forceinline__ int reduced_row(const PsrParams<T>& p, int x) {
  if (x == 0) return part_size(p.n, p.P, 0) - 1;
  const int part = (x + 1) / 2;
  const int s = part_start(p.n, p.P, part);
  return (x & 1) ? s : s + part_size(p.n, p.P, part) - 1;
}

// CTAs are split into P teams (CTA c belongs to team floor(c P / G)); every
// CTA passes every grid barrier, also after its team gave up on a wait, so the
// others' waits end.
template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) psr_kernel(PsrParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  const int G = gridDim.x, me = blockIdx.x, P = p.P, b = p.b;
  const size_t bb = (size_t)b * b;
  const int part = (int)(((long long)me * P) / G);
  const int first = (int)(((long long)part * G + P - 1) / P);
  const int last = (int)(((long long)(part + 1) * G + P - 1) / P);
  TeamDyn all{&p.hdr->barrier_count, p.status, me, G, 0u};
  TeamDyn team{&p.team_bar[part], p.status, me - first, last - first, 0u};
  T* side = p.side + (size_t)part * p.side_elems;
  const int R = 2 * (P - 1);

  GemmOp<T> ops[4];  // one scratch op table for every phase (keeps the stack frame small)
  psr_reduce<T, BM, BN>(team, p, part, side, p.work + (size_t)part * 2 * bb, ops, smem);
  if (!all.sync()) return;
  // gather the reduced system (psr_seqsolve.py:336-384, 410-467)
  for (int x = 0; x < R; x++) {
    const int r = reduced_row(p, x);
    team_copy<T>(all, b, b, p.D + (size_t)r * bb, b, p.Rd + (size_t)x * bb, b);
    if (x + 1 < R) {
      const bool link = (x & 1) == 0;  // bot_p -> t_{p+1}: the input couplings; t_p -> B_p: the fill-in
      const int B = reduced_row(p, x + 1);
      team_copy<T>(all, b, b, link ? p.upper + (size_t)r * bb : p.FR + (size_t)B * bb, b, p.Ru + (size_t)x * bb, b);
      team_copy<T>(all, b, b, link ? p.lower + (size_t)r * bb : p.FC + (size_t)B * bb, b, p.Rl + (size_t)x * bb, b);
    }
  }
  if (!all.sync()) return;
  if (!reduced_sweep<T, BM, BN>(all, p, R, ops, smem)) return;
  if (!all.sync()) return;
  // scatter the boundary blocks of the inverse (psr_seqsolve.py:520-645)
  for (int x = 0; x < R; x++) {
    const int r = reduced_row(p, x);
    team_copy<T>(all, b, b, p.RGd + (size_t)x * bb, b, p.Gd + (size_t)r * bb, b);
    if (x + 1 < R) {
      const bool link = (x & 1) == 0;
      const int B = reduced_row(p, x + 1);
      team_copy<T>(all, b, b, p.RGu + (size_t)x * bb, b, link ? p.Gu + (size_t)r * bb : p.GR + (size_t)B * bb, b);
      team_copy<T>(all, b, b, p.RGl + (size_t)x * bb, b, link ? p.Gl + (size_t)r * bb : p.GC + (size_t)B * bb, b);
    }
  }
  if (!all.sync()) return;
  psr_produce<T, BM, BN>(team, p, part, ops, smem);
}

// Partitions when the caller passes 0: about sqrt(n/2), which balances the
// 2n/P partition steps against the 4(P-1) steps of the reduced sweep.
int psr_auto_partitions(int n) {
  int P = (int)(std::sqrt(n / 2.0) + 0.5);
  P = std::min(P, std::min(kPsrMaxP, n / 3));
  return std::max(P, 3);
}

struct PsrLayout {
  size_t bar, blocks, reduced, T0, work, side, total, side_elems;
};

// rows: block rows the launch holds (n for a whole matrix, the partition's m
// for one partition); teams: P for a whole matrix (with the reduced system on
// the device), 1 for one partition.
PsrLayout psr_layout(int rows, int b, int P, int teams, size_t es) {
  PsrLayout L{};
  const size_t bb = (size_t)b * b * es;
  const int R = teams > 1 ? 2 * (P - 1) : 0;
  size_t off = sizeof(WsHeader);
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  L.bar = take((size_t)teams * sizeof(unsigned));
  L.blocks = take(9 * (size_t)rows * bb);
  L.reduced = take(R > 0 ? (size_t)(3 * R - 2) * 2 * bb : 0);
  L.T0 = take(bb);
  L.work = take((size_t)(teams + 1) * 2 * bb);
  L.side_elems = invert_side_elems(b);
  L.side = take((size_t)(teams + 1) * L.side_elems * es);
  L.total = off;
  return L;
}

int psr_partitions(int n, int partitions) {
  const int P = partitions > 0 ? partitions : psr_auto_partitions(n);
  if (P < 3 || P > kPsrMaxP || n < 3 * P) return -1;  // psr_utils.py:55-58, psr_seqsolve.py:43-44
  return P;
}

template <class T>
int psr_check(const void* diag, const void* Gd, const void* const* others, int nothers, const void* workspace,
              size_t workspace_bytes, size_t need) {
  if (!diag || !Gd || !workspace) return SINVB_EINVAL;
  if ((uintptr_t)diag % sizeof(T) || (uintptr_t)Gd % sizeof(T)) return SINVB_EINVAL;
  for (int k = 0; k < nothers; k++)
    if (others[k] && (uintptr_t)others[k] % sizeof(T)) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  if (workspace_bytes < need) return SINVB_EWORKSPACE;
  return check_device();
}

// rows / row0: the block rows the arrays hold and the global row of their
// first element; teams as in psr_layout.
template <class T>
PsrParams<T> psr_params(const void* diag, const void* upper, const void* lower, int n, int b, int P, int rows,
                        int row0, int teams, void* Gd, void* Gu, void* Gl, unsigned char* ws) {
  const PsrLayout L = psr_layout(rows, b, P, teams, sizeof(T));
  const size_t bb = (size_t)b * b;
  PsrParams<T> p{};
  p.diag = (const T*)diag;
  p.upper = (const T*)upper;
  p.lower = (const T*)lower;
  p.Gd = (T*)Gd;
  p.Gu = (T*)Gu;
  p.Gl = (T*)Gl;
  T* blk = reinterpret_cast<T*>(ws + L.blocks);
  T** arrays[9] = {&p.D, &p.LA, &p.UA, &p.LT, &p.UT, &p.FR, &p.FC, &p.GR, &p.GC};
  for (int k = 0; k < 9; k++) *arrays[k] = blk + (size_t)k * rows * bb;
  if (teams > 1) {
    const int R = 2 * (P - 1);
    T* red = reinterpret_cast<T*>(ws + L.reduced);
    p.Rd = red;
    p.Ru = p.Rd + (size_t)R * bb;
    p.Rl = p.Ru + (size_t)(R - 1) * bb;
    p.RGd = p.Rl + (size_t)(R - 1) * bb;
    p.RGu = p.RGd + (size_t)R * bb;
    p.RGl = p.RGu + (size_t)(R - 1) * bb;
  }
  p.T0 = reinterpret_cast<T*>(ws + L.T0);
  p.side = reinterpret_cast<T*>(ws + L.side);
  p.work = reinterpret_cast<T*>(ws + L.work);
  p.side_elems = L.side_elems;
  p.team_bar = reinterpret_cast<unsigned*>(ws + L.bar);
  p.hdr = reinterpret_cast<WsHeader*>(ws);
  p.status = &p.hdr->status;
  p.n = n;
  p.b = b;
  p.P = P;
  p.row0 = row0;
  return p;
}

// Cooperative launch on the whole GPU (up to two CTAs per SM).
template <class T, class Kern>
int psr_launch(Kern kern, void** args, int min_grid, cudaStream_t stream) {
  const size_t g = (size_t)gemm_smem_elems<T, 64, 64>() * sizeof(T);
  const size_t smem = g > sizeof(GjShared<T>) ? g : sizeof(GjShared<T>);
  SINVB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SINVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
  if (per_sm < 1) return SINVB_EUNSUPPORTED;
  const int grid = device_sm_count() * (per_sm > 2 ? 2 : per_sm);
  if (grid < min_grid) return SINVB_EUNSUPPORTED;
  SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kThreads), args, smem, stream));
  return SINVB_OK;
}

template <class T>
int psr_run(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, unsigned flags,
            void* Gd, void* Gu, void* Gl, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (flags || n < 1 || b < 1) return SINVB_EINVAL;
  const int P = psr_partitions(n, partitions);
  if (P < 0 || !upper || !lower || !Gu || !Gl) return SINVB_EINVAL;
  const void* others[4] = {upper, lower, Gu, Gl};
  const PsrLayout L = psr_layout(n, b, P, P, sizeof(T));
  int rc = psr_check<T>(diag, Gd, others, 4, workspace, workspace_bytes, L.total);
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  PsrParams<T> p = psr_params<T>(diag, upper, lower, n, b, P, n, 0, P, Gd, Gu, Gl, ws);
  SINVB_CUDA(cudaMemsetAsync(ws, 0, L.blocks, stream));  // header, team barriers
  void* args[] = {(void*)&p};
  if (b <= 32) return psr_launch<T>(psr_kernel<T, 32, 32>, args, P, stream);
  return psr_launch<T>(psr_kernel<T, 64, 64>, args, P, stream);
}

constexpr int kPsrSlots = 6;

// One partition on its own GPU, the form a rank of a multi-GPU PSR runs
// (psr_seqsolve.py:52-70 on process `part`), with the whole grid as the team
// and only the partition's rows t .. B in memory (local arrays, element 0 =
// row t).  stage 0 reduces the partition and writes its part of the reduced
// system to six boundary slots (psr_seqsolve.py:387-467): first partition
// D[B]; last D[t]; central D[t], D[B], A[t,B], A[B,t]; and in slots 4, 5 the
// couplings to the next partition A[B,B+1], A[B+1,B] (zero for the last).
// stage 1 reads the boundary blocks of the inverse from slots 0-3 (first
// G[B,B]; last G[t,t]; central G[t,t], G[B,B], G[t,B], G[B,t];
// psr_seqsolve.py:564-644) and produces the partition.  The workspace carries
// the reduction from stage 0 to stage 1.
template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) psr_part_kernel(PsrParams<T> p, int part, int stage, T* bnd) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  const int P = p.P, b = p.b;
  const size_t bb = (size_t)b * b;
  const int t = part_start(p.n, P, part), B = t + part_size(p.n, P, part) - 1;
  const size_t lt = (size_t)(t - p.row0) * bb, lB = (size_t)(B - p.row0) * bb;  // local offsets of rows t, B
  TeamDyn all{&p.hdr->barrier_count, p.status, (int)blockIdx.x, (int)gridDim.x, 0u};
  GemmOp<T> ops[4];
  if (stage == 0) {
    if (!psr_reduce<T, BM, BN>(all, p, part, p.side, p.work, ops, smem)) return;
    const bool central = part > 0 && part < P - 1;
    team_copy<T>(all, b, b, p.D + (part == 0 ? lB : lt), b, bnd, b);
    if (central) {
      team_copy<T>(all, b, b, p.D + lB, b, bnd + bb, b);
      team_copy<T>(all, b, b, p.FR + lB, b, bnd + 2 * bb, b);
      team_copy<T>(all, b, b, p.FC + lB, b, bnd + 3 * bb, b);
    }
    if (part < P - 1) {
      team_copy<T>(all, b, b, p.upper + lB, b, bnd + 4 * bb, b);
      team_copy<T>(all, b, b, p.lower + lB, b, bnd + 5 * bb, b);
    }
    all.sync();
  } else {
    const bool central = part > 0 && part < P - 1;
    team_copy<T>(all, b, b, bnd, b, p.Gd + (part == 0 ? lB : lt), b);
    if (central) {
      team_copy<T>(all, b, b, bnd + bb, b, p.Gd + lB, b);
      team_copy<T>(all, b, b, bnd + 2 * bb, b, p.GR + lB, b);
      team_copy<T>(all, b, b, bnd + 3 * bb, b, p.GC + lB, b);
    }
    if (!all.sync()) return;
    psr_produce<T, BM, BN>(all, p, part, ops, smem);
  }
}

// diag: the partition's m diagonal blocks; upper / lower: its couplings
// A[i,i+1] / A[i+1,i] for rows t .. B (m blocks; m - 1 for the last
// partition, which has no next); G_diag / G_upper / G_lower likewise.
template <class T>
int psr_part_run(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, int part,
                 int stage, void* boundary, void* Gd, void* Gu, void* Gl, void* workspace, size_t workspace_bytes,
                 cudaStream_t stream) {
  if (n < 1 || b < 1) return SINVB_EINVAL;
  const int P = psr_partitions(n, partitions);
  if (P < 0 || part < 0 || part >= P || (stage != 0 && stage != 1) || !boundary) return SINVB_EINVAL;
  if (!upper || !lower || !Gu || !Gl) return SINVB_EINVAL;
  const int m = part_size(n, P, part), t = part_start(n, P, part);
  const void* others[5] = {upper, lower, Gu, Gl, boundary};
  const PsrLayout L = psr_layout(m, b, P, 1, sizeof(T));
  int rc = psr_check<T>(diag, Gd, others, 5, workspace, workspace_bytes, L.total);
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  PsrParams<T> p = psr_params<T>(diag, upper, lower, n, b, P, m, t, 1, Gd, Gu, Gl, ws);
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), stream));  // status and barrier; the reduction stays
  if (stage == 0) SINVB_CUDA(cudaMemsetAsync(boundary, 0, kPsrSlots * (size_t)b * b * sizeof(T), stream));
  T* bnd = (T*)boundary;
  void* args[] = {(void*)&p, (void*)&part, (void*)&stage, (void*)&bnd};
  if (b <= 32) return psr_launch<T>(psr_part_kernel<T, 32, 32>, args, 1, stream);
  return psr_launch<T>(psr_part_kernel<T, 64, 64>, args, 1, stream);
}

}  // namespace
}  // namespace sinvb

using namespace sinvb;

extern "C" {

int sinvb_psr_partitions(int n, int partitions) { return psr_partitions(n, partitions); }

size_t sinvb_psr_workspace_size(int n, int b, int partitions, int dtype, unsigned flags) {
  if (flags || b < 1 || (dtype != SINVB_C128 && dtype != SINVB_F64)) return 0;
  const int P = psr_partitions(n, partitions);
  if (P < 0) return 0;
  return psr_layout(n, b, P, P, dtype == SINVB_C128 ? 16 : 8).total;
}

size_t sinvb_psr_part_workspace_size(int n, int b, int partitions, int part, int dtype) {
  if (b < 1 || (dtype != SINVB_C128 && dtype != SINVB_F64)) return 0;
  const int P = psr_partitions(n, partitions);
  if (P < 0 || part < 0 || part >= P) return 0;
  return psr_layout(part_size(n, P, part), b, P, 1, dtype == SINVB_C128 ? 16 : 8).total;
}

int sinvb_psr_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  return psr_run<cplx>(diag, upper, lower, n, b, partitions, flags, G_diag, G_upper, G_lower, workspace,
                       workspace_bytes, (cudaStream_t)stream);
}

int sinvb_psr_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream) {
  return psr_run<double>(diag, upper, lower, n, b, partitions, flags, G_diag, G_upper, G_lower, workspace,
                         workspace_bytes, (cudaStream_t)stream);
}

int sinvb_psr_part_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, int part,
                     int stage, void* boundary, void* G_diag, void* G_upper, void* G_lower, void* workspace,
                     size_t workspace_bytes, sinvb_stream_t stream) {
  return psr_part_run<cplx>(diag, upper, lower, n, b, partitions, part, stage, boundary, G_diag, G_upper, G_lower,
                            workspace, workspace_bytes, (cudaStream_t)stream);
}

int sinvb_psr_part_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, int part,
                     int stage, void* boundary, void* G_diag, void* G_upper, void* G_lower, void* workspace,
                     size_t workspace_bytes, sinvb_stream_t stream) {
  return psr_part_run<double>(diag, upper, lower, n, b, partitions, part, stage, boundary, G_diag, G_upper, G_lower,
                              workspace, workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
