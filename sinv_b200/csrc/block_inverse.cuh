// Pivot-free in-place block inversion (Gauss-Jordan).
//
// The reference inverts every block with numpy.linalg.inv (LAPACK getrf/getri
// with partial pivoting, src/sinv/algorithms/rgf/rgf.py:44,48).  The RGF and
// BCR recursions have no pivoting across blocks; inside a block this library
// eliminates without pivoting as well and reports a zero or non-finite pivot
// through the workspace status word (SINVB_STATUS_PIVOT) instead of trapping.
//
// Gauss-Jordan on an m x m matrix, step k (p = a_kk):
//   a_kk <- 1/p,  a_kj <- a_kj/p,  a_ik <- -a_ik/p,  a_ij <- a_ij - a_ik a_kj/p
// After m steps the array holds the inverse; m^3 multiply-adds in total.
//
// * cta_gj_invert: one CTA, m <= 64.  The block lives in registers (thread
//   (ty, tx) of a 16 x 16 grid owns rows ty+16r and columns tx+16c); row k,
//   column k and 1/a_kk are published through double-buffered shared arrays,
//   so one barrier per step suffices.
// * team_invert: any m.  Blocked Gauss-Jordan over PW-wide panels:
//   (1) invert the diagonal panel block (cta_gj_invert for PW <= 64; for
//       PW = 128 by the whole team, recursively in 64-wide panels),
//   (2) scale the row panel by it (DMMA GEMM) into a side buffer,
//   (3) rank-PW update of every other block and the new column panel
//       (DMMA GEMMs), the column panel going to a side buffer; both panels
//       are copied back while the next pivot block is inverted.
#pragma once

#include "block_gemm.cuh"

namespace sinvb {

// Blocks of at most kGjMax rows are inverted unblocked by one CTA.  Larger
// blocks go in panels: the explicit inverse of each pivot block costs accuracy
// on blocks far from diagonal dominance.  RGF inverts the damped Schur
// complements S_i with 128-wide panels whose pivot blocks are themselves
// inverted in 64-wide panels (the same 64 x 64 pivot inverses as 64-wide
// panels; tight-binding: ~1e-12 vs 2e-13 unblocked); BCR inverts raw reduced
// diagonal blocks, where 64-wide panels lost three digits (1.8e-9 vs 3e-12)
// and 32-wide panels lose about one.
constexpr int kGjMax = 64;
constexpr int kPanelRgf = 64;
constexpr int kPanel = 32;      // BCR

template <class T>
struct GjShared {
  T rowbuf[2][kGjMax];
  T colbuf[2][kGjMax];
  T pinv[2];
};

// Inverts the m x m block at a (leading dimension lda), m <= kGjMax, in place.
// Returns false (and reports) on a zero / non-finite pivot; the block then
// holds non-finite values.
template <class T>
__device__ bool cta_gj_invert(T* a, int lda, int m, int* status, void* smem_raw) {
  GjShared<T>& sh = *reinterpret_cast<GjShared<T>*>(smem_raw);
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  T v[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int i = ty + 16 * r, j = tx + 16 * c;
      v[r][c] = (i < m && j < m) ? a[(size_t)i * lda + j] : Elem<T>::zero();
    }
  __syncthreads();  // smem may still be read by a previous user
  // publish column 0, row 0 and 1/a_00
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int i = ty + 16 * r, j = tx + 16 * c;
      if (j == 0 && i < m) sh.colbuf[0][i] = v[r][c];
      if (i == 0 && j < m) sh.rowbuf[0][j] = v[r][c];
      if (i == 0 && j == 0) sh.pinv[0] = recip(v[r][c]);
    }
  bool bad = false;
  for (int k = 0; k < m; k++) {
    __syncthreads();
    const int buf = k & 1, nbuf = buf ^ 1;
    const T ip = sh.pinv[buf];
    if (tid == 0 && !bad && !pivot_ok(sh.rowbuf[buf][k])) {
      bad = true;
      report(status, SINVB_STATUS_PIVOT);
    }
    T rk[4], ck[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int j = tx + 16 * c;
      rk[c] = j < m ? sh.rowbuf[buf][j] * ip : Elem<T>::zero();
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      int i = ty + 16 * r;
      ck[r] = i < m ? sh.colbuf[buf][i] : Elem<T>::zero();
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        int i = ty + 16 * r, j = tx + 16 * c;
        T x = v[r][c];
        if (i == k) {
          x = (j == k) ? ip : rk[c];
        } else if (j == k) {
          x = -(ck[r] * ip);
        } else {
          x = fms(x, ck[r], rk[c]);
        }
        v[r][c] = x;
        if (k + 1 < m) {
          if (j == k + 1 && i < m) sh.colbuf[nbuf][i] = x;
          if (i == k + 1 && j < m) sh.rowbuf[nbuf][j] = x;
          if (i == k + 1 && j == k + 1) sh.pinv[nbuf] = recip(x);
        }
      }
  }
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int i = ty + 16 * r, j = tx + 16 * c;
      if (i < m && j < m) a[(size_t)i * lda + j] = v[r][c];
    }
  __syncthreads();
  return !bad;
}

// Copies a rows x cols rectangle (optionally transposed: dst[j][i] = src[i][j]),
// split over the team's CTAs.  No synchronisation.
template <class T, class Team>
__device__ void team_copy(Team& team, int rows, int cols, const T* src, int lds, T* dst, int ldd,
                          bool transpose = false) {
  const size_t total = (size_t)rows * cols;
  const size_t stride = (size_t)team.size() * blockDim.x;
  for (size_t e = (size_t)team.rank() * blockDim.x + threadIdx.x; e < total; e += stride) {
    int i = (int)(e / cols), j = (int)(e % cols);
    if (transpose)
      dst[(size_t)j * ldd + i] = src[(size_t)i * lds + j];
    else
      dst[(size_t)i * ldd + j] = src[(size_t)i * lds + j];
  }
}

// Elements of side buffer team_invert needs for an m x m block with panels of
// PW: the new column panel W (m x PW, leading dimension PW), the scaled row
// panel R (PW x m, leading dimension m) and, when PW > kGjMax, the side
// buffer of the nested inversion of a PW x PW pivot block (panels of PW / 2).
__host__ __device__ constexpr size_t invert_side_elems_pw(int m, int PW) {
  return m <= kGjMax ? 0
                     : (m <= PW && PW > kGjMax) ? invert_side_elems_pw(m, PW / 2)
                                                : 2 * (size_t)m * PW + (PW > kGjMax ? invert_side_elems_pw(PW, PW / 2) : 0);
}
// ... for the widest panels used (RGF)
__host__ __device__ inline size_t invert_side_elems(int m) { return invert_side_elems_pw(m, kPanelRgf); }

// Inverts the m x m block at a (lda) in place with the whole team.  `side` holds
// invert_side_elems(m) elements.  Starts and ends with the block visible to the
// whole team (the caller synchronised before; this function synchronises
// after).  Returns false when a team barrier gave up.
//
// Per kPanel-wide panel K (rows/columns K0 .. K0+kb):
//   phase 1: D = A[K,K]^{-1} in place (one CTA); write back the previous
//            panel's W and R (they were read by the previous phase 3)
//   phase 2: R[K, J] = D A[K, J] for J outside K        (out of place: no tile
//            of the product reads what another tile writes)
//   phase 3: A[I, J] -= A[I, K] R[K, J],  W[I] = -A[I, K] D   for I, J outside K
template <class T, int BM, int BN, int PW = kPanelRgf, class Team>
__device__ bool team_invert(Team& team, T* a, int lda, int m, T* side, int* status, T* smem) {
  if (m <= kGjMax) {
    if (team.rank() == 0) cta_gj_invert<T>(a, lda, m, status, smem);
    return team.sync();
  }
  if constexpr (PW > kGjMax) {
    if (m <= PW) return team_invert<T, BM, BN, PW / 2>(team, a, lda, m, side, status, smem);
  }
  T* W = side;                       // m x PW
  T* R = side + (size_t)m * PW;      // PW x m, leading dimension m
  T* inner = R + (size_t)PW * m;     // nested pivot-block inversion (PW > kGjMax)
  const int np = (m + PW - 1) / PW;
  int pK0 = -1, pkb = 0;
  auto write_back = [&]() {
    const int r1 = pK0 + pkb;
    team_copy<T>(team, pK0, pkb, W, PW, a + pK0, lda);
    team_copy<T>(team, m - r1, pkb, W + (size_t)r1 * PW, PW, a + (size_t)r1 * lda + pK0, lda);
    team_copy<T>(team, pkb, pK0, R, m, a + (size_t)pK0 * lda, lda);
    team_copy<T>(team, pkb, m - r1, R + r1, m, a + (size_t)pK0 * lda + r1, lda);
  };
  for (int p = 0; p < np; p++) {
    const int K0 = p * PW, kb = min(PW, m - K0), right = K0 + kb;
    T* Dinv = a + (size_t)K0 * lda + K0;
    if constexpr (PW > kGjMax) {
      // the whole team inverts the pivot block (64-wide panels) after the
      // previous panel is written back
      if (pK0 >= 0) write_back();
      if (!team.sync()) return false;
      if (!team_invert<T, BM, BN, PW / 2>(team, Dinv, lda, kb, inner, status, smem)) return false;
    } else {
      if (team.rank() == 0) cta_gj_invert<T>(Dinv, lda, kb, status, smem);
      if (pK0 >= 0) write_back();
      if (!team.sync()) return false;
    }
    {
      GemmOp<T> ops[2];
      ops[0] = make_op<T>(kb, K0, kb, 1.0, Dinv, lda, a + (size_t)K0 * lda, lda, nullptr, 0, R, m);
      ops[1] = make_op<T>(kb, m - right, kb, 1.0, Dinv, lda, a + (size_t)K0 * lda + right, lda, nullptr, 0,
                          R + right, m);
      team_gemm<T, BM, BN>(team, ops, 2, smem);
    }
    if (!team.sync()) return false;
    {
      GemmOp<T> ops[6];
      int rs[2] = {0, right}, rn[2] = {K0, m - right};
      int q = 0;
      for (int ri = 0; ri < 2; ri++) {
        const T* colK = a + (size_t)rs[ri] * lda + K0;
        for (int ci = 0; ci < 2; ci++) {
          T* C = a + (size_t)rs[ri] * lda + rs[ci];
          ops[q++] = make_op<T>(rn[ri], rn[ci], kb, -1.0, colK, lda, R + rs[ci], m, C, lda, C, lda);
        }
        ops[q++] = make_op<T>(rn[ri], kb, kb, -1.0, colK, lda, Dinv, lda, nullptr, 0,
                              W + (size_t)rs[ri] * PW, PW);
      }
      team_gemm<T, BM, BN>(team, ops, q, smem);
    }
    if (!team.sync()) return false;
    pK0 = K0;
    pkb = kb;
  }
  write_back();
  return team.sync();
}

}  // namespace sinvb
