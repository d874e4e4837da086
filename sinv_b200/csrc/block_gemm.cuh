// Block GEMM on the FP64 tensor cores (DMMA, mma.sync m8n8k4.f64).
//
//   C[M x N] = beta D + alpha ( op(A) op(B) + sign2 op(A2) op(B2) )
//
// op(X) is X or X^H (conjugate transpose; plain transpose for real types),
// D may alias C (each tile reads its own D before writing), the second product
// is optional (BCR's productions are two-term sums,
// src/sinv/algorithms/bcr/bcr_serial.py:361-383; the adjoint sweeps need
// signed sums of conjugate-transposed products).
//
// Complex products run as four real DMMA products (4M):
//   C.re += A.re B.re - A.im B.im,   C.im += A.re B.im + A.im B.re
// with conjugation and the sign of the second product applied to the register
// fragments.  B200 has no FP64 kind of tcgen05.mma; the warp-level DMMA path
// peaks at the chip's FP64 rate (37 TFLOP/s measured), one CTA of 8 warps per SM
// reaching its 0.25 TFLOP/s share.
//
// A CTA computes one BM x BN output tile.  K is streamed through shared memory
// in BK-element chunks with a 3-stage cp.async ring; the first product's K is
// padded with zeros to a chunk boundary so a chunk never mixes products.
// Shared-memory layouts are XOR-swizzled so the DMMA fragment loads
// (A[g][t] and B[t][g], lane = 4g + t) hit distinct banks:
//   complex (16 B):  A(m,k) -> m*BK + (k ^ ((m&1)<<2)),  B(k,n) -> k*BN + (n ^ ((k&3)<<1))
//   real    ( 8 B):  A(m,k) -> m*BK + (k ^ ((m&3)<<2)),  B(k,n) -> k*BN + (n ^ ((k&3)<<2))
// Global loads are coalesced for either operand form (the fastest-varying
// thread index follows the contiguous source dimension).
#pragma once

#include "common.cuh"

namespace sinvb {

enum : int { kOpN = 0, kOpH = 1 };

template <class T>
struct GemmOp {
  const T* A;
  const T* B;
  const T* D;  // addend, may be null, may alias C
  T* C;
  int lda, ldb, ldd, ldc;
  int M, N, K;
  double alpha, beta;
  int opA, opB;
  const T* A2;  // second product (null: none); op(A2) is M x K2, op(B2) is K2 x N
  const T* B2;
  int lda2, ldb2, K2;
  int opA2, opB2;
  int sign2;  // +1 or -1
};

template <class T>
__host__ __device__ __forceinline__ GemmOp<T> make_op(int M, int N, int K, double alpha, const T* A, int lda,
                                                      const T* B, int ldb, const T* D, int ldd, T* C, int ldc) {
  GemmOp<T> o;
  o.A = A; o.B = B; o.D = D; o.C = C;
  o.lda = lda; o.ldb = ldb; o.ldd = ldd; o.ldc = ldc;
  o.M = M; o.N = N; o.K = K; o.alpha = alpha; o.beta = 1.0;
  o.opA = kOpN; o.opB = kOpN;
  o.A2 = nullptr; o.B2 = nullptr; o.lda2 = 0; o.ldb2 = 0; o.K2 = 0;
  o.opA2 = kOpN; o.opB2 = kOpN; o.sign2 = 1;
  return o;
}

// Adds the second product sign2 * op(A2) op(B2) (K2 = K) to an op.
template <class T>
__host__ __device__ __forceinline__ GemmOp<T> with_second(GemmOp<T> o, const T* A2, int lda2, int opA2, const T* B2,
                                                          int ldb2, int opB2, int sign2 = 1) {
  o.A2 = A2; o.B2 = B2; o.lda2 = lda2; o.ldb2 = ldb2; o.K2 = o.K;
  o.opA2 = opA2; o.opB2 = opB2; o.sign2 = sign2;
  return o;
}

constexpr int kThreads = 256;  // 8 warps per CTA, every kernel of the library
constexpr int kStages = 3;

template <class T> struct GemmCfg;
template <> struct GemmCfg<cplx> {
  static constexpr int BK = 16;
  __device__ static int a_idx(int m, int k) { return m * BK + (k ^ ((m & 1) << 2)); }
  template <int BN> __device__ static int b_idx(int k, int n) { return k * BN + (n ^ ((k & 3) << 1)); }
};
template <> struct GemmCfg<double> {
  static constexpr int BK = 16;
  __device__ static int a_idx(int m, int k) { return m * BK + (k ^ ((m & 3) << 2)); }
  template <int BN> __device__ static int b_idx(int k, int n) { return k * BN + (n ^ ((k & 3) << 2)); }
};

// Shared memory (in elements of T) one CTA tile needs: the K-chunk ring, then
// the addend tile D (rows padded by one element against bank conflicts),
// fetched with the first chunk so the epilogue does not wait on global loads.
template <class T, int BM, int BN>
__host__ __device__ constexpr int gemm_ring_elems() {
  return kStages * (BM * GemmCfg<T>::BK + GemmCfg<T>::BK * BN);
}
template <class T, int BM, int BN>
__host__ __device__ constexpr int gemm_smem_elems() {
  return gemm_ring_elems<T, BM, BN>() + BM * (BN + 1);
}

// K extent of the first product as streamed: padded to whole chunks when a
// second product follows.
template <class T>
__device__ __forceinline__ int k1_padded(const GemmOp<T>& op) {
  constexpr int BK = GemmCfg<T>::BK;
  return op.K2 > 0 ? (op.K + BK - 1) / BK * BK : op.K;
}

template <class T, int BM, int BN>
__device__ __forceinline__ void load_chunk(const GemmOp<T>& op, int row0, int col0, int k0, T* sA, T* sB) {
  constexpr int BK = GemmCfg<T>::BK;
  const int tid = threadIdx.x;
  const int K1p = k1_padded(op);
  const bool second = op.K2 > 0 && k0 >= K1p;
  const T* A = second ? op.A2 : op.A;
  const T* B = second ? op.B2 : op.B;
  const int lda = second ? op.lda2 : op.lda, ldb = second ? op.ldb2 : op.ldb;
  const int opA = second ? op.opA2 : op.opA, opB = second ? op.opB2 : op.opB;
  const int kbase = second ? k0 - K1p : k0;
  const int Klim = second ? op.K2 : op.K;
#pragma unroll
  for (int e = tid; e < BM * BK; e += kThreads) {
    int m, k;
    if (opA == kOpN) { m = e / BK; k = e % BK; } else { k = e / BM; m = e % BM; }
    const int gr = row0 + m, gk = kbase + k;
    const bool v = gr < op.M && gk < Klim;
    const T* src = A;
    if (v) src = opA == kOpN ? A + (size_t)gr * lda + gk : A + (size_t)gk * lda + gr;
    cp_async_elem<T>(sA + GemmCfg<T>::a_idx(m, k), src, v);
  }
#pragma unroll
  for (int e = tid; e < BK * BN; e += kThreads) {
    int k, n;
    if (opB == kOpN) { k = e / BN; n = e % BN; } else { n = e / BK; k = e % BK; }
    const int gk = kbase + k, gc = col0 + n;
    const bool v = gk < Klim && gc < op.N;
    const T* src = B;
    if (v) src = opB == kOpN ? B + (size_t)gk * ldb + gc : B + (size_t)gc * ldb + gk;
    cp_async_elem<T>(sB + GemmCfg<T>::template b_idx<BN>(k, n), src, v);
  }
}

// Warp grid 2 (M) x 4 (N); warp tile (BM/2) x (BN/4) made of MT x NT 8x8 DMMA tiles.
template <int BM, int BN>
struct WarpShape {
  static constexpr int WM = BM / 2, WN = BN / 4;
  static constexpr int MT = WM / 8, NT = WN / 8;
  static_assert(MT >= 1 && NT >= 1, "tile too small for 8 warps");
};

// Fragment signs of a chunk: A.im *= sai (conjugation), B.re *= sbr, B.im *= sbi
// (conjugation and the sign of the second product).
template <int BM, int BN>
__device__ __forceinline__ void mma_chunk(const cplx* sA, const cplx* sB, double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4],
                                          double sai, double sbr, double sbi) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<cplx>::BK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int kk = 0; kk < BK; kk += 4) {
    cplx a[W::MT], b[W::NT];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++) {
      a[mt] = sA[GemmCfg<cplx>::a_idx(wm + mt * 8 + g, kk + t)];
      a[mt].im *= sai;
    }
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) {
      b[nt] = sB[GemmCfg<cplx>::b_idx<BN>(kk + t, wn + nt * 8 + g)];
      b[nt].re *= sbr;
      b[nt].im *= sbi;
    }
    // Two passes so that the two products landing on the same accumulator are
    // MT*NT*2 instructions apart instead of back to back (DMMA latency).
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) {
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].re, b[nt].re);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].re, b[nt].im);
      }
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) {
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].im, -b[nt].im);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].im, b[nt].re);
      }
  }
}

template <int BM, int BN>
__device__ __forceinline__ void mma_chunk(const double* sA, const double* sB, double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4],
                                          double, double sbr, double) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<double>::BK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int kk = 0; kk < BK; kk += 4) {
    double a[W::MT], b[W::NT];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++) a[mt] = sA[GemmCfg<double>::a_idx(wm + mt * 8 + g, kk + t)];
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) b[nt] = sbr * sB[GemmCfg<double>::b_idx<BN>(kk + t, wn + nt * 8 + g)];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt], b[nt]);
  }
}

// The common product (no conjugation, no second product): no sign factors
// on the fragments; -Im B by flipping its sign bit on the integer pipe.
__device__ __forceinline__ double neg_bits(double x) {
  return __hiloint2double(__double2hiint(x) ^ 0x80000000, __double2loint(x));
}
template <int BM, int BN>
__device__ __forceinline__ void mma_chunk_plain(const cplx* sA, const cplx* sB,
                                                double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4]) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<cplx>::BK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int kk = 0; kk < BK; kk += 4) {
    cplx a[W::MT], b[W::NT];
    double nbi[W::NT];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++) a[mt] = sA[GemmCfg<cplx>::a_idx(wm + mt * 8 + g, kk + t)];
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) {
      b[nt] = sB[GemmCfg<cplx>::b_idx<BN>(kk + t, wn + nt * 8 + g)];
      nbi[nt] = neg_bits(b[nt].im);
    }
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) {
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].re, b[nt].re);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].re, b[nt].im);
      }
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) {
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].im, nbi[nt]);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].im, b[nt].re);
      }
  }
}
template <int BM, int BN>
__device__ __forceinline__ void mma_chunk_plain(const double* sA, const double* sB,
                                                double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4]) {
  mma_chunk<BM, BN>(sA, sB, acc, 1.0, 1.0, 1.0);
}

// Epilogue of two adjacent outputs (r, c), (r, c+1): alpha times the
// accumulators plus beta times the addend, whose tile sits in shared memory
// at dtile (row stride ldt, indexed from the tile origin; null: no addend).
template <class T>
__device__ __forceinline__ void store_pair(const GemmOp<T>& op, int r, int c, const T* dtile, int ldt, double v0r,
                                           double v0i, double v1r, double v1i);

template <>
__device__ __forceinline__ void store_pair<cplx>(const GemmOp<cplx>& op, int r, int c, const cplx* dtile, int ldt,
                                                 double v0r, double v0i, double v1r, double v1i) {
  if (r >= op.M) return;
  const double al = op.alpha, be = op.beta;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    int cc = c + j;
    if (cc < op.N) {
      cplx v = j == 0 ? cplx{al * v0r, al * v0i} : cplx{al * v1r, al * v1i};
      if (dtile) {
        cplx d = dtile[j];
        v = be == 1.0 ? d + v : cplx{fma(be, d.re, v.re), fma(be, d.im, v.im)};
      }
      op.C[(size_t)r * op.ldc + cc] = v;
    }
  }
}
template <>
__device__ __forceinline__ void store_pair<double>(const GemmOp<double>& op, int r, int c, const double* dtile, int ldt,
                                                   double v0, double, double v1, double) {
  if (r >= op.M) return;
  const double al = op.alpha, be = op.beta;
  if (c < op.N) {
    double v = al * v0;
    if (dtile) v = fma(be, dtile[0], v);
    op.C[(size_t)r * op.ldc + c] = v;
  }
  if (c + 1 < op.N) {
    double v = al * v1;
    if (dtile) v = fma(be, dtile[1], v);
    op.C[(size_t)r * op.ldc + c + 1] = v;
  }
}

// Asynchronous copy of the addend tile D[row0 .., col0 ..] (the part inside
// M x N) into shared memory, row stride BN + 1; consecutive threads take
// consecutive columns.
template <class T, int BM, int BN>
__device__ __forceinline__ void load_addend(const GemmOp<T>& op, int row0, int col0, T* sD) {
#pragma unroll 4
  for (int e = threadIdx.x; e < BM * BN; e += kThreads) {
    const int r = e / BN, c = e % BN;
    const bool v = row0 + r < op.M && col0 + c < op.N;
    const T* src = v ? op.D + (size_t)(row0 + r) * op.ldd + (col0 + c) : op.D;
    cp_async_elem<T>(sD + r * (BN + 1) + c, src, v);
  }
}

template <class T, int BM, int BN>
__device__ __forceinline__ int op_tiles(const GemmOp<T>& op) {
  if (op.M <= 0 || op.N <= 0) return 0;
  return ((op.M + BM - 1) / BM) * ((op.N + BN - 1) / BN);
}

// One output tile (tile row tm, tile column tn) of op, computed by the whole
// CTA.  K streams through a 3-stage cp.async ring; each chunk's successor
// load is issued after the chunk's multiplications so that the DMMAs start
// right after the barrier.  The addend tile D is fetched into shared memory
// with the first chunk, so the epilogue does not wait on global loads (D may
// alias C: the tile reads its own D before it writes C).  smem:
// gemm_smem_elems<T,BM,BN>() elements.  Ends with the CTA synchronised and
// the tile written.
template <class T, int BM, int BN>
__device__ void cta_gemm_tile(const GemmOp<T>& op, int tm, int tn, T* smem) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<T>::BK;
  T* sA = smem;
  T* sB = smem + kStages * BM * BK;
  T* sD = smem + gemm_ring_elems<T, BM, BN>();
  const int row0 = tm * BM, col0 = tn * BN;
  double acc[W::MT][W::NT][4];
#pragma unroll
  for (int i = 0; i < W::MT; i++)
#pragma unroll
    for (int j = 0; j < W::NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

  const int K1p = k1_padded(op);
  const int nk = (K1p + op.K2 + BK - 1) / BK;
  const int nk1 = (K1p + BK - 1) / BK;  // chunks of the first product
  const bool plain = op.opA == kOpN && op.opB == kOpN;
  // fragment signs per product: conjugation of A / B, sign of the second product
  const double sai1 = op.opA == kOpH ? -1.0 : 1.0, sbi1 = op.opB == kOpH ? -1.0 : 1.0;
  const double s2 = op.sign2 < 0 ? -1.0 : 1.0;
  const double sai2 = op.opA2 == kOpH ? -1.0 : 1.0, sbi2 = (op.opB2 == kOpH ? -1.0 : 1.0) * s2;
  const bool addend = op.D != nullptr;
  if (addend) load_addend<T, BM, BN>(op, row0, col0, sD);  // lands with the first chunk's group
#pragma unroll
  for (int s = 0; s < kStages - 1; s++) {
    if (s < nk) load_chunk<T, BM, BN>(op, row0, col0, s * BK, sA + s * BM * BK, sB + s * BK * BN);
    cp_async_commit();
  }
  for (int kc = 0; kc < nk; kc++) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    const int st = kc % kStages;
    if (kc < nk1) {
      if (plain)
        mma_chunk_plain<BM, BN>(sA + st * BM * BK, sB + st * BK * BN, acc);
      else
        mma_chunk<BM, BN>(sA + st * BM * BK, sB + st * BK * BN, acc, sai1, 1.0, sbi1);
    } else {
      mma_chunk<BM, BN>(sA + st * BM * BK, sB + st * BK * BN, acc, sai2, s2, sbi2);
    }
    // into the stage consumed one chunk ago: every warp is past this chunk's barrier
    const int pf = kc + kStages - 1;
    if (pf < nk) {
      const int sp = pf % kStages;
      load_chunk<T, BM, BN>(op, row0, col0, pf * BK, sA + sp * BM * BK, sB + sp * BK * BN);
    }
    cp_async_commit();
  }
  cp_async_wait<0>();
  __syncthreads();  // the addend tile, copied by every thread, is complete

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) {
      const int lr = wm + mt * 8 + g, lc = wn + nt * 8 + 2 * t;
      store_pair<T>(op, row0 + lr, col0 + lc, addend ? sD + lr * (BN + 1) + lc : nullptr, BN + 1, acc[mt][nt][0],
                    acc[mt][nt][2], acc[mt][nt][1], acc[mt][nt][3]);
    }
  __syncthreads();
}

// All tiles of up to 8 independent GEMMs, spread over the team's CTAs.  The
// caller separates dependent phases with team.sync().
template <class T, int BM, int BN, class Team>
__device__ void team_gemm(Team& team, const GemmOp<T>* ops, int nops, T* smem) {
  int counts[8];
  int total = 0;
  for (int i = 0; i < nops; i++) {
    counts[i] = op_tiles<T, BM, BN>(ops[i]);
    total += counts[i];
  }
  const int rank = team.rank(), size = team.size();
  for (int tile = rank; tile < total; tile += size) {
    int i = 0, local = tile;
    while (local >= counts[i]) local -= counts[i++];
    const GemmOp<T>& op = ops[i];
    int tn_count = (op.N + BN - 1) / BN;
    cta_gemm_tile<T, BM, BN>(op, local / tn_count, local % tn_count, smem);
  }
}

}  // namespace sinvb
