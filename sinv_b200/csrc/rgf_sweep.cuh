// The RGF selected-inversion sweep on one team of CTAs.
//
// Reference: src/sinv/algorithms/rgf/rgf.py:17-64.
//   forward  (rgf.py:44-48):  g_0 = A_00^{-1},
//                             g_i = (A_ii - A_{i,i-1} g_{i-1} A_{i-1,i})^{-1}
//   backward (rgf.py:51-62):  lf = G_{i+1} A_{i+1,i} g_i
//                             G_{i+1,i} = -lf
//                             G_{i,i+1} = -g_i A_{i,i+1} G_{i+1}   (or G_{i+1,i}^T if sym)
//                             G_ii      = g_i + g_i A_{i,i+1} lf
//
// Schedule (6 block products per block row instead of the reference's 8):
//   forward step i:  X_{i-1} = g_{i-1} U_{i-1},  P_i = L_i g_{i-1}     (phase F1)
//                    S_i = A_ii - P_i U_{i-1}                          (phase F2)
//                    g_i = S_i^{-1} in place                           (team_invert)
//   backward step i: T   = -G_{i+1} P_{i+1}           (= G_{i+1,i})    (phase B1)
//                    G_{i,i+1} = -X_i G_{i+1}                          (phase B2)
//                    G_ii = g_i - X_i T                                (phase B2)
// with U_i = A_{i,i+1}, L_{i+1} = A_{i+1,i}.  (A g) A and G (A g) replace the
// reference's (G A) g association; the difference is rounding only.
//
// Storage: g_i is built in G_diag[i].  With SAVE_OFFDIAG, X_i lives in
// G_lower[i] and P_{i+1} in G_upper[i] until the backward step overwrites
// them; otherwise both live in the workspace.  T alternates between two
// workspace blocks and is copied to G_lower[i] one phase later.
//
// In place (SINVB_INPLACE): G_diag, G_upper, G_lower are the input arrays.
// A_{i,i-1} is dead after F1 of step i and A_{i-1,i} after F2, so X_{i-1} and
// P_i are first written to a pair of workspace blocks (alternating between
// two pairs by step parity) and copied over the dead inputs one phase later.
#pragma once

#include <type_traits>

#include "block_inverse.cuh"
#include "ozaki.cuh"

namespace sinvb {

template <class T>
struct RgfParams {
  const T* diag;
  const T* upper;
  const T* lower;
  T* Gd;
  T* Gu;
  T* Gl;
  T* X;    // n-1 blocks (may alias Gl)
  T* P;    // n-1 blocks (may alias Gu)
  T* T0;   // b*b
  T* T1;   // b*b
  T* T2;   // b*b (in place only)
  T* T3;   // b*b (in place only)
  T* Winv; // invert_side_elems(b)
  WsHeader* hdr;   // grid-team barrier counter (unused by other teams)
  int* status;     // device status word of this matrix
  int n, b;
  unsigned flags;
  T* ckpt;         // optional: g_{s*c-1} saved to ckpt[s-1] (s = 1, 2, ...) for the adjoint
  int ckpt_every;  // c
  // mixed precision (complex only): block products on the int8 tensor cores
  int oz_digits;              // digits of the tensor-core products (Mixed sweeps; 0: FP64 products)
  unsigned char* oz_scratch;  // 2 x oz_op_scratch(b, b, b, digits) bytes
  OzState* oz;                // per-CTA pipeline state (TMEM allocated by the kernel)
};

// The block products of a sweep phase: FP64 DMMA, or (Mixed, complex only)
// the int8 tensor-core Ozaki products when p.oz_digits > 0.  The block
// inverses always stay in FP64.  Mixed is a template switch so that kernels
// without the tensor-core path do not carry its registers.  `slots` places
// the digit planes of the operands (two A and two B slots) so that an
// operand shared by consecutive products is sliced once per phase:
//   F1  g U (A0, B0), L g (A1, B1)     F2  P U (A1 sliced, B0 = U reused)
//   B1  G P (A0, B0)                   B2  X G (A1, B1), X T (A1 = X reused, B0)
template <class T, int BM, int BN, bool Mixed, class Team>
__device__ __forceinline__ bool sweep_gemm(Team& team, const RgfParams<T>& p, const GemmOp<T>* ops, int nops, T* smem,
                                           const OzSlots& slots) {
  if constexpr (Mixed && std::is_same<T, cplx>::value) {
    if (p.oz_digits > 0)
      return team_gemm_ozaki(team, ops, nops, p.oz_digits, p.oz_scratch, slots, p.oz,
                             reinterpret_cast<unsigned char*>(smem), p.status);
  }
  team_gemm<T, BM, BN>(team, ops, nops, smem);
  return true;
}

template <class T, int BM, int BN, bool Mixed = false, class Team>
__device__ void rgf_sweep(Team& team, const RgfParams<T>& p, T* smem) {
  const int n = p.n, b = p.b;
  const size_t bb = (size_t)b * b;
  const bool sym = p.flags & SINVB_SYM;
  const bool save = p.flags & SINVB_SAVE_OFFDIAG;

  const bool inplace = p.flags & SINVB_INPLACE;

  // g_0 = A_00^{-1}
  if (!inplace) {
    team_copy<T>(team, b, b, p.diag, b, p.Gd, b);
    if (!team.sync()) return;
  }
  if (!team_invert<T, BM, BN>(team, p.Gd, b, b, p.Winv, p.status, smem)) return;

  for (int i = 1; i < n; i++) {
    const T* g = p.Gd + (i - 1) * bb;
    const T* U = p.upper + (i - 1) * bb;
    const T* L = p.lower + (i - 1) * bb;
    // in place: X_{i-1} / P_i go to a temp pair, alternating by parity
    T* Xd = inplace ? ((i & 1) ? p.T2 : p.T0) : p.X + (i - 1) * bb;
    T* Pd = inplace ? ((i & 1) ? p.T3 : p.T1) : p.P + (i - 1) * bb;
    {  // F1
      GemmOp<T> ops[2];
      ops[0] = make_op<T>(b, b, b, 1.0, g, b, U, b, nullptr, 0, Xd, b);
      ops[1] = make_op<T>(b, b, b, 1.0, L, b, g, b, nullptr, 0, Pd, b);
      if (!sweep_gemm<T, BM, BN, Mixed>(team, p, ops, 2, smem, OzSlots{{0, 1}, {0, 1}, 3u, 3u})) return;
      if (inplace && i >= 2)  // P_{i-1} over A_{i-2,i-1}, dead since F2 of step i-1
        team_copy<T>(team, b, b, (i & 1) ? p.T1 : p.T3, b, p.Gu + (i - 2) * bb, b);
      if (p.ckpt && i % p.ckpt_every == 0)  // checkpoint g_{i-1} for the adjoint
        team_copy<T>(team, b, b, g, b, p.ckpt + (size_t)(i / p.ckpt_every - 1) * bb, b);
    }
    if (!team.sync()) return;
    {  // F2: S_i = A_ii - P_i U_{i-1}
      GemmOp<T> op = make_op<T>(b, b, b, -1.0, Pd, b, U, b, p.diag + i * bb, b, p.Gd + i * bb, b);
      if (!sweep_gemm<T, BM, BN, Mixed>(team, p, &op, 1, smem, OzSlots{{1, 0}, {0, 0}, 1u, 0u})) return;
      if (inplace)  // X_{i-1} over A_{i,i-1}, dead since F1
        team_copy<T>(team, b, b, Xd, b, p.Gl + (i - 1) * bb, b);
    }
    if (!team.sync()) return;
    if (!team_invert<T, BM, BN>(team, p.Gd + i * bb, b, b, p.Winv, p.status, smem)) return;
  }
  if (inplace && n >= 2) {
    team_copy<T>(team, b, b, ((n - 1) & 1) ? p.T3 : p.T1, b, p.Gu + (n - 2) * bb, b);
    if (!team.sync()) return;
  }

  T* prevT = nullptr;
  int prevI = -1;
  for (int i = n - 2; i >= 0; i--) {
    T* Tcur = (i & 1) ? p.T1 : p.T0;
    {  // B1: T = -G_{i+1} P_{i+1}; flush the previous T into G_lower / G_upper
      GemmOp<T> op = make_op<T>(b, b, b, -1.0, p.Gd + (i + 1) * bb, b, p.P + i * bb, b, nullptr, 0, Tcur, b);
      if (!sweep_gemm<T, BM, BN, Mixed>(team, p, &op, 1, smem, OzSlots{{0, 0}, {0, 0}, 1u, 1u})) return;
      if (prevT && save) {
        team_copy<T>(team, b, b, prevT, b, p.Gl + prevI * bb, b);
        if (sym) team_copy<T>(team, b, b, prevT, b, p.Gu + prevI * bb, b, true);
      }
    }
    if (!team.sync()) return;
    {  // B2
      GemmOp<T> ops[2];
      int q = 0;
      const T* X = p.X + i * bb;
      if (save && !sym)
        ops[q++] = make_op<T>(b, b, b, -1.0, X, b, p.Gd + (i + 1) * bb, b, nullptr, 0, p.Gu + i * bb, b);
      T* Gii = p.Gd + i * bb;
      ops[q++] = make_op<T>(b, b, b, -1.0, X, b, Tcur, b, Gii, b, Gii, b);
      // X is sliced once: by the first product, reused by the second
      const OzSlots sl = q == 2 ? OzSlots{{1, 1}, {1, 0}, 1u, 3u} : OzSlots{{1, 0}, {0, 0}, 1u, 1u};
      if (!sweep_gemm<T, BM, BN, Mixed>(team, p, ops, q, smem, sl)) return;
    }
    if (!team.sync()) return;
    prevT = Tcur;
    prevI = i;
  }
  if (prevT && save) {
    team_copy<T>(team, b, b, prevT, b, p.Gl + prevI * bb, b);
    if (sym) team_copy<T>(team, b, b, prevT, b, p.Gu + prevI * bb, b, true);
    team.sync();
  }
}

}  // namespace sinvb
