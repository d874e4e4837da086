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
//   (ty, tx) of a 16 x 16 grid owns rows ty+16r and columns tx+16c); row k
//   and column k are published through double-buffered shared arrays, so one
//   barrier per step suffices; every thread forms 1/a_kk itself.
// * team_invert: any m.  Blocked Gauss-Jordan over PW-wide panels:
//   (1) invert the diagonal panel block (cta_gj_invert for PW <= 64; for
//       PW = 128 by the whole team, recursively in 64-wide panels),
//   (2) scale the row panel by it (DMMA GEMM) into a side buffer,
//   (3) rank-PW update of every other block and the new column panel
//       (DMMA GEMMs), the column panel going to a side buffer; both panels
//       are copied back while the next pivot block is inverted.
//   Teams of at most one CTA per panel instead give each CTA whole column
//   blocks: each inverts the pivot block itself and scales / updates its own
//   columns, so a panel costs one team barrier instead of three and no CTA
//   waits while another inverts the pivot block.
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
};

// One 16-step block of the Gauss-Jordan sweep: pivots k = 16 KB + kk.  With
// KB a compile-time constant, pivot row k is row KB of the 16 threads with
// ty == kk and pivot column k is column KB of the threads with tx == kk, so
// the special cases of the pivot row and column are a handful of selects
// instead of a test per element.  Step k, p = a_kk, in one uniform update:
//   a_ij <- [i != k and j != k] a_ij - c_i r_j,
//   r_j = a_kj / p (r_k = 1 / p),   c_i = a_ik (c_k = -1),
// which gives a_kk <- 1/p, a_kj <- a_kj/p, a_ik <- -a_ik/p and
// a_ij <- a_ij - a_ik a_kj / p.  The next pivot row and column are published
// through double-buffered shared arrays, one barrier per step.
template <int KB, class T>
__device__ __forceinline__ void gj_block16(T (&v)[4][4], GjShared<T>& sh, int m, int* status, bool& bad) {
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  for (int kk = 0; kk < 16; kk++) {
    const int k = 16 * KB + kk;
    if (k >= m) break;
    __syncthreads();
    const int buf = k & 1, nbuf = buf ^ 1;
    const T p = sh.rowbuf[buf][k];
    const T ip = recip(p);
    if (tid == 0 && !bad && !pivot_ok(p)) {
      bad = true;
      report(status, SINVB_STATUS_PIVOT);
    }
    T rk[4], ck[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      rk[c] = sh.rowbuf[buf][tx + 16 * c] * ip;
      if (c == KB && tx == kk) rk[c] = ip;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      ck[r] = sh.colbuf[buf][ty + 16 * r];
      if (r == KB && ty == kk) ck[r] = -Elem<T>::one();
    }
    if (ty == kk) {
#pragma unroll
      for (int c = 0; c < 4; c++) v[KB][c] = Elem<T>::zero();
    }
    if (tx == kk) {
#pragma unroll
      for (int r = 0; r < 4; r++) v[r][KB] = Elem<T>::zero();
    }
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) v[r][c] = fms(v[r][c], ck[r], rk[c]);
    if (k + 1 < m) {  // publish row and column k + 1
      if (kk < 15) {
        if (ty == kk + 1) {
#pragma unroll
          for (int c = 0; c < 4; c++) sh.rowbuf[nbuf][tx + 16 * c] = v[KB][c];
        }
        if (tx == kk + 1) {
#pragma unroll
          for (int r = 0; r < 4; r++) sh.colbuf[nbuf][ty + 16 * r] = v[r][KB];
        }
      } else if constexpr (KB < 3) {
        if (ty == 0) {
#pragma unroll
          for (int c = 0; c < 4; c++) sh.rowbuf[nbuf][tx + 16 * c] = v[KB + 1][c];
        }
        if (tx == 0) {
#pragma unroll
          for (int r = 0; r < 4; r++) sh.colbuf[nbuf][ty + 16 * r] = v[r][KB + 1];
        }
      }
    }
  }
}

// Inverts the m x m block at src (leading dimension lds), m <= kGjMax, into
// dst (ldd); dst may be src.  Returns false (and reports) on a zero /
// non-finite pivot; the block then holds non-finite values.
template <class T>
__device__ bool cta_gj_invert_to(const T* src, int lds, T* dst, int ldd, int m, int* status, void* smem_raw) {
  GjShared<T>& sh = *reinterpret_cast<GjShared<T>*>(smem_raw);
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  T v[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int i = ty + 16 * r, j = tx + 16 * c;
      v[r][c] = (i < m && j < m) ? src[(size_t)i * lds + j] : Elem<T>::zero();
    }
  __syncthreads();  // smem may still be read by a previous user
  if (ty == 0) {    // publish row 0 and column 0
#pragma unroll
    for (int c = 0; c < 4; c++) sh.rowbuf[0][tx + 16 * c] = v[0][c];
  }
  if (tx == 0) {
#pragma unroll
    for (int r = 0; r < 4; r++) sh.colbuf[0][ty + 16 * r] = v[r][0];
  }
  bool bad = false;
  gj_block16<0>(v, sh, m, status, bad);
  gj_block16<1>(v, sh, m, status, bad);
  gj_block16<2>(v, sh, m, status, bad);
  gj_block16<3>(v, sh, m, status, bad);
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      int i = ty + 16 * r, j = tx + 16 * c;
      if (i < m && j < m) dst[(size_t)i * ldd + j] = v[r][c];
    }
  __syncthreads();
  return !bad;
}

// ... in place.
template <class T>
__device__ bool cta_gj_invert(T* a, int lda, int m, int* status, void* smem_raw) {
  return cta_gj_invert_to<T>(a, lda, a, lda, m, status, smem_raw);
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
// PW.  PW <= kGjMax: two m x PW column panels (leading dimension PW; the
// shared-row schedule's W and R, the column-owner schedule's double-buffered
// W) and one PW x PW pivot-block copy per panel (the column-owner schedule
// gives each of its CTAs, at most one per panel, a private copy).
// PW > kGjMax: W, R and the side buffer of the nested inversion of a PW x PW
// pivot block (panels of PW / 2).
__host__ __device__ constexpr size_t invert_side_elems_pw(int m, int PW) {
  return m <= kGjMax ? 0
         : (m <= PW && PW > kGjMax) ? invert_side_elems_pw(m, PW / 2)
         : 2 * (size_t)m * PW + (PW > kGjMax ? invert_side_elems_pw(PW, PW / 2)
                                             : (size_t)((m + PW - 1) / PW) * PW * PW);
}

// Every tile of one op, computed by this CTA alone.
template <class T, int BM, int BN>
__device__ __forceinline__ void cta_gemm_op(const GemmOp<T>& op, T* smem) {
  if (op.M <= 0 || op.N <= 0) return;
  const int tm_n = (op.M + BM - 1) / BM, tn_n = (op.N + BN - 1) / BN;
  for (int tm = 0; tm < tm_n; tm++)
    for (int tn = 0; tn < tn_n; tn++) cta_gemm_tile<T, BM, BN>(op, tm, tn, smem);
}

// Blocked Gauss-Jordan with the column blocks owned by the team's CTAs (block
// j, columns j PW ..., by CTA j mod size), for teams of at most one CTA per
// panel.  One team barrier per panel: after it, the pivot block A[K,K] and the
// pivot column panel A[:,K] are final, and per panel K every CTA
//   (1) inverts A[K,K] itself into a private copy D (no CTA waits for another
//       to do it),
//   (2) scales its own column blocks of the pivot row in place,
//       A[K,J] <- D A[K,J] (one CTA reads and writes that tile, and its whole
//       K extent is loaded before the tile is stored),
//   (3) updates its own column blocks, A[I,J] -= A[I,K] A[K,J] for I != K;
// and the owner of K writes the new column panel W = -A[:,K] D to a side
// buffer (the other CTAs still read A[:,K]); at the start of the next panel,
// after the barrier, it copies W and D into column block K, which from then
// on only it reads.  W alternates between two buffers by panel parity, so one
// owner's copy-in never meets the next owner's writes.  The arithmetic is
// that of the shared-row schedule below, tile for tile.
template <class T, int BM, int BN, int PW, class Team>
__device__ bool team_invert_owned(Team& team, T* a, int lda, int m, T* side, int* status, T* smem) {
  const int np = (m + PW - 1) / PW;
  const int me = team.rank(), nt = team.size();
  T* Wb[2] = {side, side + (size_t)m * PW};
  T* D = side + 2 * (size_t)m * PW + (size_t)me * PW * PW;
  TeamCta self;
  for (int p = 0; p <= np; p++) {
    if (p > 0 && (p - 1) % nt == me) {  // copy-in of the previous panel's column block
      const int P0 = (p - 1) * PW, pb = min(PW, m - P0), r1 = P0 + pb;
      const T* W = Wb[(p - 1) & 1];
      team_copy<T>(self, P0, pb, W, PW, a + P0, lda);
      team_copy<T>(self, m - r1, pb, W + (size_t)r1 * PW, PW, a + (size_t)r1 * lda + P0, lda);
      team_copy<T>(self, pb, pb, D, PW, a + (size_t)P0 * lda + P0, lda);
      __syncthreads();
    }
    if (p == np) break;
    const int K0 = p * PW, kb = min(PW, m - K0), r1 = K0 + kb;
    cta_gj_invert_to<T>(a + (size_t)K0 * lda + K0, lda, D, PW, kb, status, smem);
    for (int j = me; j < np; j += nt) {  // (2) pivot row, own column blocks
      if (j == p) continue;
      const int J0 = j * PW, wj = min(PW, m - J0);
      T* Rk = a + (size_t)K0 * lda + J0;
      cta_gemm_op<T, BM, BN>(make_op<T>(kb, wj, kb, 1.0, D, PW, Rk, lda, nullptr, 0, Rk, lda), smem);
    }
    for (int j = me; j < np; j += nt) {  // (3) rank-kb update, own column blocks
      if (j == p) continue;
      const int J0 = j * PW, wj = min(PW, m - J0);
      const T* Rk = a + (size_t)K0 * lda + J0;
      cta_gemm_op<T, BM, BN>(make_op<T>(K0, wj, kb, -1.0, a + K0, lda, Rk, lda, a + J0, lda, a + J0, lda), smem);
      T* below = a + (size_t)r1 * lda + J0;
      cta_gemm_op<T, BM, BN>(
          make_op<T>(m - r1, wj, kb, -1.0, a + (size_t)r1 * lda + K0, lda, Rk, lda, below, lda, below, lda), smem);
    }
    if (p % nt == me) {  // the new pivot column panel, into the side buffer
      T* W = Wb[p & 1];
      cta_gemm_op<T, BM, BN>(make_op<T>(K0, kb, kb, -1.0, a + K0, lda, D, PW, nullptr, 0, W, PW), smem);
      cta_gemm_op<T, BM, BN>(make_op<T>(m - r1, kb, kb, -1.0, a + (size_t)r1 * lda + K0, lda, D, PW, nullptr, 0,
                                        W + (size_t)r1 * PW, PW),
                             smem);
    }
    if (!team.sync()) return false;
  }
  return team.sync();
}
// ... for the widest panels used (RGF)
__host__ __device__ inline size_t invert_side_elems(int m) { return invert_side_elems_pw(m, kPanelRgf); }

// Inverts the m x m block at a (lda) in place with the whole team.  `side` holds
// invert_side_elems(m) elements.  Starts and ends with the block visible to the
// whole team (the caller synchronised before; this function synchronises
// after).  Returns false when a team barrier gave up.
//
// Teams of at most one CTA per panel take the column-owner schedule above
// (one barrier per panel).  Larger teams (a whole GPU on one matrix) take the
// shared-row schedule, three barriers per PW-wide panel K (rows/columns
// K0 .. K0+kb):
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
  if constexpr (PW <= kGjMax && BM >= PW) {
    // teams of at most one CTA per panel (the batched kernel's, single CTAs);
    // BM >= PW: a pivot-row tile is one GEMM tile (scaled in place)
    if (team.size() <= (m + PW - 1) / PW) return team_invert_owned<T, BM, BN, PW>(team, a, lda, m, side, status, smem);
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
