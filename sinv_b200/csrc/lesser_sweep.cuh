// The lesser sweep pair (shared by the single-matrix and batched kernels).
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
#pragma once

#include "block_inverse.cuh"

namespace sinvb {

struct LesserParams {
  const cplx* diag;
  const cplx* upper;
  const cplx* lower;
  const cplx* sig;  // Sigma<_i, n blocks
  cplx* Gd;
  cplx* Gu;
  cplx* Gl;
  cplx* GLd;        // g<_i, then G<_ii
  cplx* GLu;        // G<_{i,i+1}
  cplx* tmp[5];     // b x b each
  cplx* side;       // invert_side_elems(b)
  WsHeader* hdr;
  int* status;
  int n, b;
};

// out += Y - Y^H on a b x b block, split over the team.
template <class Team>
__device__ void team_add_skew(Team& team, int b, const cplx* Y, cplx* out) {
  const size_t total = (size_t)b * b;
  const size_t stride = (size_t)team.size() * blockDim.x;
  for (size_t e = (size_t)team.rank() * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int i = (int)(e / b), j = (int)(e % b);
    const cplx y = Y[e], yt = Y[(size_t)j * b + i];
    out[e] = cplx{out[e].re + y.re - yt.re, out[e].im + y.im + yt.im};
  }
}

__host__ __device__ inline GemmOp<cplx> with_ops(GemmOp<cplx> o, int opA, int opB, double beta) {
  o.opA = opA;
  o.opB = opB;
  o.beta = beta;
  return o;
}

template <int BM, int BN, class Team>
__device__ void lesser_sweep(Team& team, const LesserParams& p, cplx* smem) {
  const int n = p.n, b = p.b;
  const size_t bb = (size_t)b * b;
  cplx* const* t = p.tmp;
  GemmOp<cplx> ops[4];  // one array for every phase (keeps the stack frame small)
  // g_0, g<_0
  team_copy<cplx>(team, b, b, p.diag, b, p.Gd, b);
  if (!team.sync()) return;
  if (!team_invert<cplx, BM, BN>(team, p.Gd, b, b, p.side, p.status, smem)) return;
  {
    ops[0] = make_op<cplx>(b, b, b, 1.0, p.Gd, b, p.sig, b, nullptr, 0, t[0], b);  // V = g Sigma<
    team_gemm<cplx, BM, BN>(team, ops, 1, smem);
  }
  if (!team.sync()) return;
  {
    ops[0] = with_ops(make_op<cplx>(b, b, b, 1.0, t[0], b, p.Gd, b, nullptr, 0, p.GLd, b), kOpN, kOpH, 1.0);
    team_gemm<cplx, BM, BN>(team, ops, 1, smem);  // g<_0 = V g_0^H
  }
  if (!team.sync()) return;
  for (int i = 1; i < n; i++) {
    const cplx* g = p.Gd + (i - 1) * bb;
    const cplx* gl = p.GLd + (i - 1) * bb;
    const cplx* U = p.upper + (i - 1) * bb;
    const cplx* L = p.lower + (i - 1) * bb;
    {  // X_{i-1} = g U,  P_i = L g,  Q = L g<
      ops[0] = make_op<cplx>(b, b, b, 1.0, g, b, U, b, nullptr, 0, p.Gl + (i - 1) * bb, b);
      ops[1] = make_op<cplx>(b, b, b, 1.0, L, b, g, b, nullptr, 0, p.Gu + (i - 1) * bb, b);
      ops[2] = make_op<cplx>(b, b, b, 1.0, L, b, gl, b, nullptr, 0, t[0], b);
      team_gemm<cplx, BM, BN>(team, ops, 3, smem);
    }
    if (!team.sync()) return;
    {  // S_i = A_ii - P_i U,  R = Sigma<_i + Q L^H
      ops[0] = make_op<cplx>(b, b, b, -1.0, p.Gu + (i - 1) * bb, b, U, b, p.diag + i * bb, b, p.Gd + i * bb, b);
      ops[1] = with_ops(make_op<cplx>(b, b, b, 1.0, t[0], b, L, b, p.sig + i * bb, b, t[1], b), kOpN, kOpH, 1.0);
      team_gemm<cplx, BM, BN>(team, ops, 2, smem);
    }
    if (!team.sync()) return;
    if (!team_invert<cplx, BM, BN>(team, p.Gd + i * bb, b, b, p.side, p.status, smem)) return;
    {  // V = g_i R
      ops[0] = make_op<cplx>(b, b, b, 1.0, p.Gd + i * bb, b, t[1], b, nullptr, 0, t[0], b);
      team_gemm<cplx, BM, BN>(team, ops, 1, smem);
    }
    if (!team.sync()) return;
    {  // g<_i = V g_i^H
      ops[0] = with_ops(make_op<cplx>(b, b, b, 1.0, t[0], b, p.Gd + i * bb, b, nullptr, 0, p.GLd + i * bb, b), kOpN,
                        kOpH, 1.0);
      team_gemm<cplx, BM, BN>(team, ops, 1, smem);
    }
    if (!team.sync()) return;
  }
  cplx* T = t[0];
  cplx* W = t[1];
  cplx* XG = t[2];
  cplx* Z = t[3];
  cplx* Y = t[4];
  for (int i = n - 2; i >= 0; i--) {
    cplx* Gn = p.Gd + (i + 1) * bb;    // G_{i+1}
    cplx* GLn = p.GLd + (i + 1) * bb;  // G<_{i+1}
    cplx* X = p.Gl + i * bb;           // X_i
    cplx* P = p.Gu + i * bb;           // P_{i+1}
    cplx* gl = p.GLd + i * bb;         // g<_i, becomes G<_ii
    const cplx* Ln = p.lower + i * bb;  // L_{i+1}
    {  // T = -G_{i+1} P_{i+1} (= G_{i+1,i}),  W = G_{i+1} L_{i+1},  XG = X_i G<_{i+1}
      ops[0] = make_op<cplx>(b, b, b, -1.0, Gn, b, P, b, nullptr, 0, T, b);
      ops[1] = make_op<cplx>(b, b, b, 1.0, Gn, b, Ln, b, nullptr, 0, W, b);
      ops[2] = make_op<cplx>(b, b, b, 1.0, X, b, GLn, b, nullptr, 0, XG, b);
      team_gemm<cplx, BM, BN>(team, ops, 3, smem);
    }
    if (!team.sync()) return;
    {  // G_{i,i+1} = -X G_{i+1};  G_ii = g_i - X T;  Z = W g<_i;  G<_{i,i+1} = -g<_i W^H - XG
      cplx* Gi = p.Gd + i * bb;
      ops[0] = make_op<cplx>(b, b, b, -1.0, X, b, Gn, b, nullptr, 0, P, b);
      ops[1] = make_op<cplx>(b, b, b, -1.0, X, b, T, b, Gi, b, Gi, b);
      ops[2] = make_op<cplx>(b, b, b, 1.0, W, b, gl, b, nullptr, 0, Z, b);
      ops[3] = with_ops(make_op<cplx>(b, b, b, -1.0, gl, b, W, b, XG, b, p.GLu + i * bb, b), kOpN, kOpH, -1.0);
      team_gemm<cplx, BM, BN>(team, ops, 4, smem);
    }
    if (!team.sync()) return;
    {  // Y = X Z;  G<_ii = g<_i + XG X^H
      ops[0] = make_op<cplx>(b, b, b, 1.0, X, b, Z, b, nullptr, 0, Y, b);
      ops[1] = with_ops(make_op<cplx>(b, b, b, 1.0, XG, b, X, b, gl, b, gl, b), kOpN, kOpH, 1.0);
      team_gemm<cplx, BM, BN>(team, ops, 2, smem);
    }
    if (!team.sync()) return;
    team_add_skew(team, b, Y, gl);          // G<_ii += Y - Y^H
    team_copy<cplx>(team, b, b, T, b, X, b);  // G_{i+1,i} over X_i (no longer read)
    if (!team.sync()) return;
  }
}

}  // namespace sinvb
