// Block GEMM on the FP64 tensor cores (DMMA, mma.sync m8n8k4.f64).
//
//   C[M x N] = D + alpha * A[M x K] * B[K x N]        (row-major, any sizes)
//
// Complex products run as four real DMMA products (4M):
//   C.re += A.re B.re - A.im B.im,   C.im += A.re B.im + A.im B.re
// B200 has no FP64 kind of tcgen05.mma; the warp-level DMMA path peaks at the
// same 37 TFLOP/s as the chip's FP64 units (measured), one CTA per SM reaching
// its 0.25 TFLOP/s share with 8 warps.
//
// A CTA computes one BM x BN output tile.  K is streamed through shared memory
// in BK-element chunks with a 3-stage cp.async ring.  Shared-memory layouts are
// XOR-swizzled so the DMMA fragment loads (A[g][t] and B[t][g], lane = 4g + t)
// hit distinct banks:
//   complex (16 B):  A(m,k) -> m*BK + (k ^ ((m&1)<<2)),  B(k,n) -> k*BN + (n ^ ((k&3)<<1))
//   real    ( 8 B):  A(m,k) -> m*BK + (k ^ ((m&3)<<2)),  B(k,n) -> k*BN + (n ^ ((k&3)<<2))
#pragma once

#include "common.cuh"

namespace sinvb {

template <class T>
struct GemmOp {
  const T* A;
  const T* B;
  const T* D;  // addend, may be null, may alias C (read before the tile's own write)
  T* C;
  int lda, ldb, ldd, ldc;
  int M, N, K;
  double alpha;
};

template <class T>
__device__ __forceinline__ GemmOp<T> make_op(int M, int N, int K, double alpha, const T* A, int lda,
                                             const T* B, int ldb, const T* D, int ldd, T* C, int ldc) {
  GemmOp<T> o;
  o.A = A; o.B = B; o.D = D; o.C = C;
  o.lda = lda; o.ldb = ldb; o.ldd = ldd; o.ldc = ldc;
  o.M = M; o.N = N; o.K = K; o.alpha = alpha;
  return o;
}

constexpr int kThreads = 256;  // 8 warps per CTA, every kernel of the library
constexpr int kStages = 3;

template <class T> struct GemmCfg;
template <> struct GemmCfg<cplx> {
  static constexpr int BK = 8;
  __device__ static int a_idx(int m, int k) { return m * BK + (k ^ ((m & 1) << 2)); }
  template <int BN> __device__ static int b_idx(int k, int n) { return k * BN + (n ^ ((k & 3) << 1)); }
};
template <> struct GemmCfg<double> {
  static constexpr int BK = 16;
  __device__ static int a_idx(int m, int k) { return m * BK + (k ^ ((m & 3) << 2)); }
  template <int BN> __device__ static int b_idx(int k, int n) { return k * BN + (n ^ ((k & 3) << 2)); }
};

// Shared memory (in elements of T) one CTA tile needs.
template <class T, int BM, int BN>
constexpr int gemm_smem_elems() {
  return kStages * (BM * GemmCfg<T>::BK + GemmCfg<T>::BK * BN);
}

template <class T, int BM, int BN>
__device__ __forceinline__ void load_chunk(const GemmOp<T>& op, int row0, int col0, int k0, T* sA, T* sB) {
  constexpr int BK = GemmCfg<T>::BK;
  const int tid = threadIdx.x;
#pragma unroll
  for (int e = tid; e < BM * BK; e += kThreads) {
    int m = e / BK, k = e % BK;
    int gr = row0 + m, gk = k0 + k;
    bool v = gr < op.M && gk < op.K;
    const T* src = v ? op.A + (size_t)gr * op.lda + gk : op.A;
    cp_async_elem<T>(sA + GemmCfg<T>::a_idx(m, k), src, v);
  }
#pragma unroll
  for (int e = tid; e < BK * BN; e += kThreads) {
    int k = e / BN, n = e % BN;
    int gk = k0 + k, gc = col0 + n;
    bool v = gk < op.K && gc < op.N;
    const T* src = v ? op.B + (size_t)gk * op.ldb + gc : op.B;
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

template <int BM, int BN>
__device__ __forceinline__ void mma_chunk(const cplx* sA, const cplx* sB, double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4]) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<cplx>::BK;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int kk = 0; kk < BK; kk += 4) {
    cplx a[W::MT], b[W::NT];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++) a[mt] = sA[GemmCfg<cplx>::a_idx(wm + mt * 8 + g, kk + t)];
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) b[nt] = sB[GemmCfg<cplx>::b_idx<BN>(kk + t, wn + nt * 8 + g)];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) {
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].re, b[nt].re);
        dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt].im, -b[nt].im);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].re, b[nt].im);
        dmma884(acc[mt][nt][2], acc[mt][nt][3], a[mt].im, b[nt].re);
      }
  }
}

template <int BM, int BN>
__device__ __forceinline__ void mma_chunk(const double* sA, const double* sB, double (&acc)[WarpShape<BM, BN>::MT][WarpShape<BM, BN>::NT][4]) {
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
    for (int nt = 0; nt < W::NT; nt++) b[nt] = sB[GemmCfg<double>::b_idx<BN>(kk + t, wn + nt * 8 + g)];
#pragma unroll
    for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
      for (int nt = 0; nt < W::NT; nt++) dmma884(acc[mt][nt][0], acc[mt][nt][1], a[mt], b[nt]);
  }
}

template <class T>
__device__ __forceinline__ void store_pair(const GemmOp<T>& op, int r, int c, double v0r, double v0i, double v1r, double v1i);

template <>
__device__ __forceinline__ void store_pair<cplx>(const GemmOp<cplx>& op, int r, int c, double v0r, double v0i, double v1r, double v1i) {
  if (r >= op.M) return;
  const double al = op.alpha;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    int cc = c + j;
    if (cc < op.N) {
      cplx v = j == 0 ? cplx{al * v0r, al * v0i} : cplx{al * v1r, al * v1i};
      if (op.D) v = op.D[(size_t)r * op.ldd + cc] + v;
      op.C[(size_t)r * op.ldc + cc] = v;
    }
  }
}
template <>
__device__ __forceinline__ void store_pair<double>(const GemmOp<double>& op, int r, int c, double v0, double, double v1, double) {
  if (r >= op.M) return;
  const double al = op.alpha;
  if (c < op.N) {
    double v = al * v0;
    if (op.D) v += op.D[(size_t)r * op.ldd + c];
    op.C[(size_t)r * op.ldc + c] = v;
  }
  if (c + 1 < op.N) {
    double v = al * v1;
    if (op.D) v += op.D[(size_t)r * op.ldd + c + 1];
    op.C[(size_t)r * op.ldc + c + 1] = v;
  }
}

// One output tile (tile row tm, tile column tn) of op, computed by the whole CTA.
// smem: gemm_smem_elems<T,BM,BN>() elements.  Ends with the CTA synchronised and
// the tile written.
template <class T, int BM, int BN>
__device__ void cta_gemm_tile(const GemmOp<T>& op, int tm, int tn, T* smem) {
  using W = WarpShape<BM, BN>;
  constexpr int BK = GemmCfg<T>::BK;
  T* sA = smem;
  T* sB = smem + kStages * BM * BK;
  const int row0 = tm * BM, col0 = tn * BN;
  double acc[W::MT][W::NT][4];
#pragma unroll
  for (int i = 0; i < W::MT; i++)
#pragma unroll
    for (int j = 0; j < W::NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

  const int nk = (op.K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < kStages - 1; s++) {
    if (s < nk) load_chunk<T, BM, BN>(op, row0, col0, s * BK, sA + s * BM * BK, sB + s * BK * BN);
    cp_async_commit();
  }
  for (int kc = 0; kc < nk; kc++) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    int pf = kc + kStages - 1;
    if (pf < nk) {
      int st = pf % kStages;
      load_chunk<T, BM, BN>(op, row0, col0, pf * BK, sA + st * BM * BK, sB + st * BK * BN);
    }
    cp_async_commit();
    int st = kc % kStages;
    mma_chunk<BM, BN>(sA + st * BM * BK, sB + st * BK * BN, acc);
  }
  cp_async_wait<0>();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * W::WM, wn = (warp & 3) * W::WN;
#pragma unroll
  for (int mt = 0; mt < W::MT; mt++)
#pragma unroll
    for (int nt = 0; nt < W::NT; nt++) {
      int r = row0 + wm + mt * 8 + g;
      int c = col0 + wn + nt * 8 + 2 * t;
      store_pair<T>(op, r, c, acc[mt][nt][0], acc[mt][nt][2], acc[mt][nt][1], acc[mt][nt][3]);
    }
  __syncthreads();
}

template <class T, int BM, int BN>
__device__ __forceinline__ int op_tiles(const GemmOp<T>& op) {
  if (op.M <= 0 || op.N <= 0) return 0;
  return ((op.M + BM - 1) / BM) * ((op.N + BN - 1) / BN);
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
