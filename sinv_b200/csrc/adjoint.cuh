// Hand-written adjoint (reverse mode) of both RGF sweeps.
//
// Forward (src/sinv/algorithms/rgf/rgf.py:44-62), with L_{i+1} = A_{i+1,i},
// U_i = A_{i,i+1}:
//   g_0 = A_00^{-1};  S_i = A_ii - P_i U_{i-1},  P_i = L_i g_{i-1},  g_i = S_i^{-1}
//   G_{n-1} = g_{n-1};  Y_i = g_i U_i,  lf_i = G_{i+1} P_{i+1}
//   G_{i+1,i} = -lf_i,  G_{i,i+1} = -Y_i G_{i+1}  (or G_{i+1,i}^T),  G_i = g_i + Y_i lf_i
//
// Given the upstream adjoints Gb (dL/dG*, the convention of torch for complex
// tensors; plain dL/dG for real ones), the adjoint runs the two sweeps in
// reverse (x^H is the conjugate transpose, the plain transpose for reals):
//
// R1, reverse of the backward sweep, i = 0 .. n-2 ascending:
//   Gbar   = Gb_ii + carry_i                       (carry_0 = 0)
//   lfb    = Y^H Gbar - Gb_{i+1,i}
//   Yb     = Gbar lf^H - Gb_{i,i+1} G_{i+1}^H
//   carry_{i+1} = lfb P_{i+1}^H - Y^H Gb_{i,i+1}   (adjoint reaching G_{i+1})
//   Pb     = G_{i+1}^H lfb
//   gb_i   = Gbar + Yb U_i^H + L_{i+1}^H Pb
//   Ub_i   = g_i^H Yb,    Lb_{i+1} = Pb g_i^H
//   then gb_{n-1} = Gb_{n-1,n-1} + carry_{n-1}.
// R2, reverse of the forward sweep, i = n-1 .. 0 descending:
//   Sb_i = -g_i^H gb_i g_i^H  = Ab_ii
//   Pb_i = -Sb_i U_{i-1}^H,   Ub_{i-1} -= P_i^H Sb_i
//   Lb_i += Pb_i g_{i-1}^H,   gb_{i-1} += L_i^H Pb_i
//
// With sym_mat (G_{i,i+1} = G_{i+1,i}^T), Gb_{i,i+1} flows into Gb_{i+1,i} as its
// plain transpose and drops out of the Yb / carry terms.
//
// Memory: the left-connected blocks g_i are not kept.  The forward pass saves
// g_{s c - 1} (c ~ sqrt(n)) and each segment [s c, (s+1) c) is recomputed from
// its checkpoint once for R1 and once for R2: O(sqrt(n)) blocks of scratch.
// gb_i lives in the Ab_ii output slot until R2 turns it into Ab_ii.
#pragma once

#include "rgf_sweep.cuh"

namespace sinvb {

template <class T>
struct AdjParams {
  const T* diag;
  const T* upper;
  const T* lower;
  const T* Gd;
  const T* Gu;
  const T* Gl;
  const T* bGd;  // upstream adjoints; bGu / bGl may be null (zero)
  const T* bGu;
  const T* bGl;
  T* aD;  // outputs: adjoints of diag, upper, lower
  T* aU;
  T* aL;
  const T* ckpt;  // g_{s c - 1} for s = 1 .. nseg-1
  T* seg_g;       // c blocks: g of the current segment
  T* seg_P;       // c blocks: P_i of the current segment
  T* tmp;         // 9 b x b temporaries
  T* side;        // invert_side_elems(b)
  int* status;
  int n, b, c;
  unsigned flags;
};

// out = x + y (y optional, optionally transposed)
template <class T, class Team>
__device__ void team_add(Team& team, int b, const T* x, const T* y, bool y_transposed, T* out) {
  const size_t total = (size_t)b * b;
  const size_t stride = (size_t)team.size() * blockDim.x;
  for (size_t e = (size_t)team.rank() * blockDim.x + threadIdx.x; e < total; e += stride) {
    int i = (int)(e / b), j = (int)(e % b);
    T v = x ? x[e] : Elem<T>::zero();
    if (y) v = v + (y_transposed ? y[(size_t)j * b + i] : y[e]);
    out[e] = v;
  }
}

template <class T>
__device__ __forceinline__ GemmOp<T> gop(int b, double alpha, const T* A, int opA, const T* B, int opB, const T* D,
                                         double beta, T* C) {
  GemmOp<T> o = make_op<T>(b, b, b, alpha, A, b, B, b, D, b, C, b);
  o.opA = opA;
  o.opB = opB;
  o.beta = beta;
  return o;
}

// Recomputes g_i (and P_i) of segment s into seg_g / seg_P.  Returns the
// segment length, or -1 when a barrier gave up.
template <class T, int BM, int BN, class Team>
__device__ int recompute_segment(Team& team, const AdjParams<T>& p, int s, T* smem) {
  const int b = p.b, n = p.n, c = p.c;
  const size_t bb = (size_t)b * b;
  const int start = s * c, len = min(c, n - start);
  for (int j = 0; j < len; j++) {
    const int i = start + j;
    T* g = p.seg_g + (size_t)j * bb;
    if (i == 0) {
      team_copy<T>(team, b, b, p.diag, b, g, b);
    } else {
      const T* gprev = j > 0 ? p.seg_g + (size_t)(j - 1) * bb : p.ckpt + (size_t)(s - 1) * bb;
      T* P = p.seg_P + (size_t)j * bb;
      GemmOp<T> op = make_op<T>(b, b, b, 1.0, p.lower + (size_t)(i - 1) * bb, b, gprev, b, nullptr, 0, P, b);
      team_gemm<T, BM, BN>(team, &op, 1, smem);
      if (!team.sync()) return -1;
      op = make_op<T>(b, b, b, -1.0, P, b, p.upper + (size_t)(i - 1) * bb, b, p.diag + (size_t)i * bb, b, g, b);
      team_gemm<T, BM, BN>(team, &op, 1, smem);
    }
    if (!team.sync()) return -1;
    if (!team_invert<T, BM, BN>(team, g, b, b, p.side, p.status, smem)) return -1;
  }
  return len;
}

template <class T, int BM, int BN, class Team>
__device__ void rgf_adjoint(Team& team, const AdjParams<T>& p, T* smem) {
  const int n = p.n, b = p.b, c = p.c;
  const size_t bb = (size_t)b * b;
  const bool sym = p.flags & SINVB_SYM;
  const int nseg = (n + c - 1) / c;
  T* Gbar = p.tmp;
  T* carry = p.tmp + bb;
  T* Y = p.tmp + 2 * bb;
  T* lfb = p.tmp + 3 * bb;
  T* Yb = p.tmp + 4 * bb;
  T* Pb = p.tmp + 5 * bb;
  T* Pn = p.tmp + 6 * bb;
  T* bGlE = p.tmp + 7 * bb;
  T* T1 = p.tmp + 8 * bb;

  // ---- R1: reverse of the backward sweep, ascending
  for (int s = 0; s < nseg; s++) {
    const int len = recompute_segment<T, BM, BN>(team, p, s, smem);
    if (len < 0) return;
    for (int j = 0; j < len; j++) {
      const int i = s * c + j;
      if (i > n - 2) break;
      const T* g = p.seg_g + (size_t)j * bb;
      const T* U = p.upper + (size_t)i * bb;
      const T* L = p.lower + (size_t)i * bb;  // L_{i+1}
      const T* G1 = p.Gd + (size_t)(i + 1) * bb;
      const T* Gl = p.Gl + (size_t)i * bb;     // -lf
      const T* bGu = p.bGu ? p.bGu + (size_t)i * bb : nullptr;
      const T* bGl = p.bGl ? p.bGl + (size_t)i * bb : nullptr;
      const T* P = (j + 1 < len) ? p.seg_P + (size_t)(j + 1) * bb : Pn;
      {  // Y = g U;  Gbar = Gb_ii + carry;  P_{i+1} at a segment end;  effective Gb_{i+1,i}
        GemmOp<T> ops[2];
        int q = 0;
        ops[q++] = make_op<T>(b, b, b, 1.0, g, b, U, b, nullptr, 0, Y, b);
        if (j + 1 >= len) ops[q++] = make_op<T>(b, b, b, 1.0, L, b, g, b, nullptr, 0, Pn, b);
        team_gemm<T, BM, BN>(team, ops, q, smem);
        team_add<T>(team, b, p.bGd + (size_t)i * bb, i > 0 ? carry : nullptr, false, Gbar);
        if (sym) team_add<T>(team, b, bGl, bGu, true, bGlE);
      }
      if (!team.sync()) return;
      const T* bGlEff = sym ? bGlE : bGl;
      {  // lfb = Y^H Gbar - Gb_{i+1,i};  Yb = -(Gbar Gl^H + Gb_{i,i+1} G1^H)
        GemmOp<T> ops[2];
        ops[0] = gop<T>(b, 1.0, Y, kOpH, Gbar, kOpN, bGlEff, -1.0, lfb);
        ops[1] = gop<T>(b, -1.0, Gbar, kOpN, Gl, kOpH, nullptr, 0.0, Yb);
        if (bGu && !sym) ops[1] = with_second<T>(ops[1], bGu, b, kOpN, G1, b, kOpH, 1);
        team_gemm<T, BM, BN>(team, ops, 2, smem);
      }
      if (!team.sync()) return;
      {  // carry = lfb P^H - Y^H Gb_{i,i+1};  Pb = G1^H lfb;  Ub_i = g^H Yb
        GemmOp<T> ops[3];
        ops[0] = gop<T>(b, 1.0, lfb, kOpN, P, kOpH, nullptr, 0.0, carry);
        if (bGu && !sym) ops[0] = with_second<T>(ops[0], Y, b, kOpH, bGu, b, kOpN, -1);
        ops[1] = gop<T>(b, 1.0, G1, kOpH, lfb, kOpN, nullptr, 0.0, Pb);
        ops[2] = gop<T>(b, 1.0, g, kOpH, Yb, kOpN, nullptr, 0.0, p.aU + (size_t)i * bb);
        team_gemm<T, BM, BN>(team, ops, 3, smem);
      }
      if (!team.sync()) return;
      {  // gb_i = Gbar + Yb U^H + L^H Pb -> aD[i];  Lb_{i+1} = Pb g^H -> aL[i]
        GemmOp<T> ops[2];
        ops[0] = gop<T>(b, 1.0, Yb, kOpN, U, kOpH, Gbar, 1.0, p.aD + (size_t)i * bb);
        ops[0] = with_second<T>(ops[0], L, b, kOpH, Pb, b, kOpN, 1);
        ops[1] = gop<T>(b, 1.0, Pb, kOpN, g, kOpH, nullptr, 0.0, p.aL + (size_t)i * bb);
        team_gemm<T, BM, BN>(team, ops, 2, smem);
      }
      if (!team.sync()) return;
    }
  }
  team_add<T>(team, b, p.bGd + (size_t)(n - 1) * bb, n > 1 ? carry : nullptr, false, p.aD + (size_t)(n - 1) * bb);
  if (!team.sync()) return;

  // ---- R2: reverse of the forward sweep, descending
  for (int s = nseg - 1; s >= 0; s--) {
    const int len = recompute_segment<T, BM, BN>(team, p, s, smem);
    if (len < 0) return;
    for (int j = len - 1; j >= 0; j--) {
      const int i = s * c + j;
      const T* g = p.seg_g + (size_t)j * bb;
      T* gb = p.aD + (size_t)i * bb;
      {  // T1 = gb g^H
        GemmOp<T> op = gop<T>(b, 1.0, gb, kOpN, g, kOpH, nullptr, 0.0, T1);
        team_gemm<T, BM, BN>(team, &op, 1, smem);
      }
      if (!team.sync()) return;
      {  // Ab_ii = Sb = -g^H T1 (over gb, which is no longer needed)
        GemmOp<T> op = gop<T>(b, -1.0, g, kOpH, T1, kOpN, nullptr, 0.0, gb);
        team_gemm<T, BM, BN>(team, &op, 1, smem);
      }
      if (!team.sync()) return;
      if (i == 0) break;
      const T* Sb = gb;
      const T* U = p.upper + (size_t)(i - 1) * bb;
      const T* L = p.lower + (size_t)(i - 1) * bb;
      const T* P = p.seg_P + (size_t)j * bb;
      const T* gprev = j > 0 ? p.seg_g + (size_t)(j - 1) * bb : p.ckpt + (size_t)(s - 1) * bb;
      T* aU = p.aU + (size_t)(i - 1) * bb;
      T* aL = p.aL + (size_t)(i - 1) * bb;
      {  // Pb = -Sb U^H;  Ub_{i-1} -= P^H Sb
        GemmOp<T> ops[2];
        ops[0] = gop<T>(b, -1.0, Sb, kOpN, U, kOpH, nullptr, 0.0, Pb);
        ops[1] = gop<T>(b, -1.0, P, kOpH, Sb, kOpN, aU, 1.0, aU);
        team_gemm<T, BM, BN>(team, ops, 2, smem);
      }
      if (!team.sync()) return;
      {  // Lb_i += Pb g_{i-1}^H;  gb_{i-1} += L^H Pb
        GemmOp<T> ops[2];
        ops[0] = gop<T>(b, 1.0, Pb, kOpN, gprev, kOpH, aL, 1.0, aL);
        ops[1] = gop<T>(b, 1.0, L, kOpH, Pb, kOpN, p.aD + (size_t)(i - 1) * bb, 1.0, p.aD + (size_t)(i - 1) * bb);
        team_gemm<T, BM, BN>(team, ops, 2, smem);
      }
      if (!team.sync()) return;
    }
  }
}

}  // namespace sinvb
