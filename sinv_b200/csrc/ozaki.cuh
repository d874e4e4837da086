// Complex FP64 block products on the int8 tensor cores (tcgen05.mma kind::i8),
// exact integer accumulation: the Ozaki scheme (Ozaki, Ogita, Oishi, Rump,
// "Error-free transformations of matrix multiplication by using fast routines
// of matrix multiplication and its applications", Numer. Algorithms 59, 2012;
// on integer tensor cores: Ootomo, Ozaki, Yokota, "DGEMM on integer matrix
// multiplication unit", IJHPCA 2024).
//
//   C = beta D + alpha A B,   A: M x K complex, B: K x N complex, FP64 in and out.
//
// Splitting.  Every row i of A is scaled by 2^-e_i (e_i: exponent of the row's
// largest |Re| or |Im|) and every column j of B by 2^-f_j, so all entries lie
// in (-1, 1).  Each scaled value x is cut into S signed 7-bit digits
//   x = sum_t d_t 2^(-6-7(t-1)),  d_t in [-64, 64]  (the first digit carries 6 bits)
// which int8 holds exactly.  Digit products are exact in int32 and so are their
// sums (|sum| <= S * 2K * 64 * 64 < 2^31 for 2K <= 2^14), so the only error is
// the truncation after S digits: levels L = s + t <= S + 1 are kept,
//   C_ij = 2^(e_i + f_j) sum_L 2^(-12-7(L-2)) sum_{s+t=L} (A_s B_t)_ij.
// Complex operands are embedded as real matrices: per 64-row group of A the
// 128 MMA rows are [Re A | -Im A] (64 rows) and [Im A | Re A] (64 rows), B^T
// rows are [Re B(:,j) | Im B(:,j)], so one 128 x 64 x 2K real product gives the
// real and the imaginary parts of a 64 x 64 complex tile in TMEM lanes 0-63 and
// 64-127, and one accumulator of 64 columns holds a level (S levels <= 512
// columns).
//
// Digit planes live in global memory in the canonical K-major core-matrix
// layout of tcgen05 (8 rows x 16 bytes per core matrix): the 64-byte K-block of
// 128 A rows (or 64 B rows) is one contiguous 8 KB (4 KB) run that a single
// bulk copy moves into shared memory.
//   offset(r, k) = ((k/64 * R/8 + r/8) * 4 + (k%64)/16) * 128 + (r%8) * 16 + k%16
#pragma once

#include "block_gemm.cuh"
#include "tc_common.cuh"

namespace sinvb {

constexpr int kOzMaxDigits = 8;
constexpr int kOzTileM = 64;   // complex rows per tile (128 MMA rows)
constexpr int kOzTileN = 64;   // complex columns per tile
constexpr int kOzKBlock = 64;  // bytes of K per pipeline stage
constexpr int kOzStages = 2;

__host__ __device__ inline int oz_pad(int x, int m) { return (x + m - 1) / m * m; }

// Geometry of the digit planes of one operand pair.
struct OzShape {
  int M, N, K;   // complex sizes
  int Mp;        // A-embed rows (multiple of 128)
  int Np;        // B^T rows (multiple of 64)
  int Kp;        // bytes of K' = 2K, multiple of 64
  int S;         // digits
  __host__ __device__ size_t a_plane() const { return (size_t)Mp * Kp; }
  __host__ __device__ size_t b_plane() const { return (size_t)Np * Kp; }
};

__host__ __device__ inline OzShape oz_shape(int M, int N, int K, int S) {
  OzShape s;
  s.M = M; s.N = N; s.K = K; s.S = S;
  s.Mp = oz_pad(M, kOzTileM) * 2;
  s.Np = oz_pad(N, kOzTileN);
  s.Kp = oz_pad(2 * K, kOzKBlock);
  return s;
}

__device__ __forceinline__ size_t oz_off(int r, int k, int R) {
  return ((size_t)((k >> 6) * (R >> 3) + (r >> 3)) * 4 + ((k & 63) >> 4)) * 128 + (r & 7) * 16 + (k & 15);
}

// Digits of x in (-1, 1): d[0] has 6 bits, the rest 7.
__device__ __forceinline__ void oz_digits(double x, int S, int (&d)[kOzMaxDigits]) {
  double v = x * 64.0;
#pragma unroll
  for (int t = 0; t < kOzMaxDigits; t++) {
    if (t < S) {
      double r = rint(v);
      d[t] = (int)r;
      v = (v - r) * 128.0;
    } else {
      d[t] = 0;
    }
  }
}

__device__ __forceinline__ int oz_exponent(double amax) {
  int e = 0;
  if (amax > 0.0) frexp(amax, &e);
  return e;
}

// Writes 16 consecutive K bytes of one digit-plane row.
__device__ __forceinline__ void oz_store16(int8_t* plane, int r, int k16, int R, const int8_t (&v)[16]) {
  int4 w;
  memcpy(&w, v, 16);
  *reinterpret_cast<int4*>(plane + oz_off(r, k16, R)) = w;
}

// A side: exponents e_i and digit planes of the embedded rows, work spread over
// `nthreads_total` threads with global index `gtid` (one warp per complex row).
__device__ inline void oz_slice_a(const cplx* A, int lda, const OzShape& s, int8_t* planes, int* ea, int gwarp,
                           int nwarps) {
  const int lane = threadIdx.x & 31;
  const int K = s.K;
  for (int i = gwarp; i < s.Mp / 2; i += nwarps) {
    const int rre = (i / kOzTileM) * 2 * kOzTileM + (i % kOzTileM), rim = rre + kOzTileM;
    double amax = 0.0;
    if (i < s.M)
      for (int k = lane; k < K; k += 32) {
        cplx v = A[(size_t)i * lda + k];
        amax = fmax(amax, fmax(fabs(v.re), fabs(v.im)));
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const int e = oz_exponent(amax);
    if (lane == 0 && i < s.M) ea[i] = e;
    const double sc = ldexp(1.0, -e);
    // each lane: one 16-byte group of K' for both embedded rows, all planes
    for (int k16 = lane * 16; k16 < s.Kp; k16 += 32 * 16) {
      int8_t re_row[kOzMaxDigits][16], im_row[kOzMaxDigits][16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int kk = k16 + q;
        int dx[kOzMaxDigits], dy[kOzMaxDigits];
        const int k = kk < K ? kk : kk - K;
        double x = 0.0, y = 0.0;
        if (i < s.M && kk < 2 * K) {
          cplx v = A[(size_t)i * lda + k];
          x = v.re * sc;
          y = v.im * sc;
        }
        oz_digits(x, s.S, dx);
        oz_digits(y, s.S, dy);
        const bool first = kk < K;
#pragma unroll
        for (int t = 0; t < kOzMaxDigits; t++) {
          re_row[t][q] = (int8_t)(first ? dx[t] : -dy[t]);  // [Re A | -Im A]
          im_row[t][q] = (int8_t)(first ? dy[t] : dx[t]);   // [Im A |  Re A]
        }
      }
      for (int t = 0; t < s.S; t++) {
        oz_store16(planes + t * s.a_plane(), rre, k16, s.Mp, re_row[t]);
        oz_store16(planes + t * s.a_plane(), rim, k16, s.Mp, im_row[t]);
      }
    }
  }
}

// B side: exponents f_j and digit planes of B^T rows [Re B(:,j) | Im B(:,j)],
// one thread per (column j, 16-byte K group); column maxima first (one thread
// per column).
__device__ inline void oz_slice_b_exponents(const cplx* B, int ldb, const OzShape& s, int* fb, int gtid, int nthreads) {
  for (int j = gtid; j < s.N; j += nthreads) {
    double amax = 0.0;
    for (int k = 0; k < s.K; k++) {
      cplx v = B[(size_t)k * ldb + j];
      amax = fmax(amax, fmax(fabs(v.re), fabs(v.im)));
    }
    fb[j] = oz_exponent(amax);
  }
}

__device__ inline void oz_slice_b_digits(const cplx* B, int ldb, const OzShape& s, int8_t* planes, const int* fb,
                                  int gtid, int nthreads) {
  const int groups = s.Kp / 16;
  const int K = s.K;
  for (int w = gtid; w < s.Np * groups; w += nthreads) {
    const int j = w % s.Np, k16 = (w / s.Np) * 16;  // consecutive threads: consecutive columns (coalesced reads)
    const double sc = j < s.N ? ldexp(1.0, -fb[j]) : 0.0;
    int8_t row[kOzMaxDigits][16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int kk = k16 + q;
      double x = 0.0;
      if (j < s.N && kk < 2 * K) {
        cplx v = B[(size_t)(kk < K ? kk : kk - K) * ldb + j];
        x = (kk < K ? v.re : v.im) * sc;
      }
      int d[kOzMaxDigits];
      oz_digits(x, s.S, d);
#pragma unroll
      for (int t = 0; t < kOzMaxDigits; t++) row[t][q] = (int8_t)d[t];
    }
    for (int t = 0; t < s.S; t++) oz_store16(planes + t * s.b_plane(), j, k16, s.Np, row[t]);
  }
}

// Shared state of the tile routine; lives in shared memory for the whole kernel.
struct OzState {
  uint64_t full[kOzStages];
  uint64_t empty[kOzStages];
  uint64_t done;
  unsigned tmem;       // TMEM base address
  unsigned kblocks;    // k-blocks streamed so far (stage / phase bookkeeping)
  unsigned tiles;      // tiles finished so far (phase of `done`)
};

__host__ __device__ constexpr size_t oz_stage_bytes(int S) { return (size_t)S * (128 + 64) * kOzKBlock; }
__host__ __device__ constexpr size_t oz_smem_bytes(int S) {
  return kOzStages * oz_stage_bytes(S) > (size_t)kOzTileM * kOzTileN * 16 ? kOzStages * oz_stage_bytes(S)
                                                                          : (size_t)kOzTileM * kOzTileN * 16;
}

// One-time set-up by the whole CTA: barriers and a TMEM allocation (warp 0).
__device__ inline void oz_setup(OzState* st) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzStages; s++) {
      mbar_init(&st->full[s], 1);
      mbar_init(&st->empty[s], 1);
    }
    mbar_init(&st->done, 1);
    st->kblocks = 0;
    st->tiles = 0;
    mbar_fence_init();
  }
  if ((threadIdx.x >> 5) == 0) tmem_alloc(&st->tmem, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ inline void oz_teardown(OzState* st) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(st->tmem, 512);
}

struct OzOp {
  const int8_t* a_planes;
  const int8_t* b_planes;
  const int* ea;
  const int* fb;
  OzShape s;
  const cplx* D;
  cplx* C;
  int ldd, ldc;
  double alpha, beta;
};

// One 64 x 64 complex output tile on the tensor cores.  Called by all threads
// of the CTA; returns false when a bounded wait gave up (status reported).
__device__ inline bool oz_tile(const OzOp& op, int tm, int tn, OzState* st, unsigned char* smem, int* status) {
  const OzShape& s = op.s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nkb = s.Kp / kOzKBlock;
  const unsigned kb0 = st->kblocks;
  const size_t stage = oz_stage_bytes(s.S);
  __shared__ int ok_flag;
  if (threadIdx.x == 0) ok_flag = 1;
  __syncthreads();
  if (warp == 0 && lane == 0) {  // producer: bulk copies of the digit tiles
    for (int kb = 0; kb < nkb; kb++) {
      const unsigned g = kb0 + kb, sidx = g % kOzStages, use = g / kOzStages;
      if (use > 0 && !mbar_wait(&st->empty[sidx], (use - 1) & 1, status)) { ok_flag = 0; break; }
      unsigned char* base = smem + sidx * stage;
      mbar_expect_tx(&st->full[sidx], (unsigned)stage);
      const size_t aoff = (size_t)(kb * (s.Mp >> 3) + (tm * 2 * kOzTileM >> 3)) * 512;
      const size_t boff = (size_t)(kb * (s.Np >> 3) + (tn * kOzTileN >> 3)) * 512;
      for (int t = 0; t < s.S; t++) {
        bulk_g2s(base + t * 8192, op.a_planes + t * s.a_plane() + aoff, 8192, &st->full[sidx]);
        bulk_g2s(base + s.S * 8192 + t * 4096, op.b_planes + t * s.b_plane() + boff, 4096, &st->full[sidx]);
      }
    }
  } else if (warp == 1 && lane == 0) {  // MMA issuer
    const uint32_t idesc = idesc_i8(128, 64);
    bool good = true;
    for (int kb = 0; kb < nkb && good; kb++) {
      const unsigned g = kb0 + kb, sidx = g % kOzStages, use = g / kOzStages;
      if (!mbar_wait(&st->full[sidx], use & 1, status)) { good = false; break; }
      tc_fence_after();
      unsigned char* base = smem + sidx * stage;
      for (int L = 2; L <= s.S + 1; L++) {
        const unsigned dcol = st->tmem + (L - 2) * 64;
        for (int a = 1; a < L; a++) {
          const int b = L - a;
          if (a > s.S || b > s.S) continue;
          for (int ks = 0; ks < 2; ks++) {
            const uint64_t ad = sdesc(base + (a - 1) * 8192 + ks * 256, 128, 512);
            const uint64_t bd = sdesc(base + s.S * 8192 + (b - 1) * 4096 + ks * 256, 128, 512);
            const bool first = kb == 0 && a == (L - s.S > 1 ? L - s.S : 1) && ks == 0;
            mma_i8(dcol, ad, bd, idesc, !first);
          }
        }
      }
      mma_commit(&st->empty[sidx]);
    }
    if (good) mma_commit(&st->done);
    else ok_flag = 0;
  }
  // epilogue: TMEM lanes -> FP64, staged in shared memory as a 64 x 64 complex tile
  __syncthreads();
  const bool ok = ok_flag != 0;
  double* ctile = reinterpret_cast<double*>(smem);  // [64][64] complex as interleaved doubles
  if (warp >= 4) {
    bool good = ok && mbar_wait(&st->done, st->tiles & 1, status);
    if (!good) ok_flag = 0;
    tc_fence_after();
    // wait for the producer's last copies too: all MMAs done implies all stages consumed
    const int q = warp - 4;
    const int r = 32 * q + lane;               // MMA row in the tile
    const int i = r & 63, part = r >> 6;       // complex row, 0 = Re, 1 = Im
    double acc[64];
#pragma unroll
    for (int c = 0; c < 64; c++) acc[c] = 0.0;
    if (good) {
      for (int L = 2; L <= s.S + 1; L++) {
        const double scale = ldexp(1.0, -12 - 7 * (L - 2));
#pragma unroll
        for (int h = 0; h < 2; h++) {
          int v[32];
          tmem_ld32(st->tmem + ((unsigned)(32 * q) << 16) + (L - 2) * 64 + h * 32, v);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 32; c++) acc[h * 32 + c] = fma((double)v[c], scale, acc[h * 32 + c]);
        }
      }
    }
    tc_fence_before();
    const int gi = tm * kOzTileM + i;
    const int ei = (gi < s.M) ? op.ea[gi] : 0;
#pragma unroll
    for (int c = 0; c < 64; c++) {
      const int gj = tn * kOzTileN + c;
      const int fj = (gj < s.N) ? op.fb[gj] : 0;
      ctile[(i * 64 + c) * 2 + part] = ldexp(acc[c], ei + fj);
    }
  }
  __syncthreads();
  // coalesced write of the tile: C = beta D + alpha * product
  if (ok_flag) {
    for (int e = threadIdx.x; e < kOzTileM * kOzTileN; e += blockDim.x) {
      const int i = e / kOzTileN, c = e % kOzTileN;
      const int gi = tm * kOzTileM + i, gj = tn * kOzTileN + c;
      if (gi < s.M && gj < s.N) {
        cplx v{op.alpha * ctile[e * 2], op.alpha * ctile[e * 2 + 1]};
        if (op.D) {
          cplx d = op.D[(size_t)gi * op.ldd + gj];
          v = cplx{fma(op.beta, d.re, v.re), fma(op.beta, d.im, v.im)};
        }
        op.C[(size_t)gi * op.ldc + gj] = v;
      }
    }
  }
  fence_proxy_async_smem();  // generic smem writes before the next tile's bulk copies
  __syncthreads();
  if (threadIdx.x == 0) {
    st->kblocks = kb0 + nkb;
    st->tiles += 1;
  }
  __syncthreads();
  return ok_flag != 0;
}

// Scratch one GEMM of the team routine needs: exponents and digit planes.
__host__ __device__ inline size_t oz_op_scratch(int M, int N, int K, int S) {
  const OzShape s = oz_shape(M, N, K, S);
  return (size_t)oz_pad(M * 4, 256) + oz_pad(N * 4, 256) + (size_t)S * (s.a_plane() + s.b_plane());
}

// Up to 2 independent complex block products C = beta D + alpha A B on the
// int8 tensor cores, spread over a team of CTAs (the mixed-precision form of
// team_gemm).  Three phases: digits of every A and exponents of every B;
// digits of every B; output tiles.  The caller synchronises after the last.
// Only plain (non-transposed) operands.  Returns false when a wait gave up.
template <class Team>
__device__ bool team_gemm_ozaki(Team& team, const GemmOp<cplx>* ops, int nops, int S, unsigned char* scratch,
                                OzState* st, unsigned char* smem, int* status) {
  OzOp oz[2];
  unsigned char* p = scratch;
  for (int i = 0; i < nops; i++) {
    const GemmOp<cplx>& g = ops[i];
    OzOp& o = oz[i];
    o.s = oz_shape(g.M, g.N, g.K, S);
    o.ea = reinterpret_cast<int*>(p);
    p += oz_pad(g.M * 4, 256);
    o.fb = reinterpret_cast<int*>(p);
    p += oz_pad(g.N * 4, 256);
    o.a_planes = reinterpret_cast<int8_t*>(p);
    p += (size_t)S * o.s.a_plane();
    o.b_planes = reinterpret_cast<int8_t*>(p);
    p += (size_t)S * o.s.b_plane();
    o.D = g.D;
    o.C = g.C;
    o.ldd = g.ldd;
    o.ldc = g.ldc;
    o.alpha = g.alpha;
    o.beta = g.beta;
  }
  const int warps = blockDim.x >> 5;
  const int gwarp = team.rank() * warps + (threadIdx.x >> 5), nwarps = team.size() * warps;
  const int gtid = team.rank() * blockDim.x + threadIdx.x, nthr = team.size() * blockDim.x;
  for (int i = 0; i < nops; i++) {
    oz_slice_a(ops[i].A, ops[i].lda, oz[i].s, const_cast<int8_t*>(oz[i].a_planes), const_cast<int*>(oz[i].ea),
               gwarp, nwarps);
    oz_slice_b_exponents(ops[i].B, ops[i].ldb, oz[i].s, const_cast<int*>(oz[i].fb), gtid, nthr);
  }
  if (!team.sync()) return false;
  for (int i = 0; i < nops; i++)
    oz_slice_b_digits(ops[i].B, ops[i].ldb, oz[i].s, const_cast<int8_t*>(oz[i].b_planes), oz[i].fb, gtid, nthr);
  fence_proxy_async_smem();
  // digit planes are read by the bulk-copy (async) proxy of other CTAs
  asm volatile("fence.proxy.async.global;" ::: "memory");
  if (!team.sync()) return false;
  // and, on the reading side, after the barrier that made them visible
  asm volatile("fence.proxy.async.global;" ::: "memory");
  int counts[2], total = 0;
  for (int i = 0; i < nops; i++) {
    counts[i] = (oz_pad(oz[i].s.M, kOzTileM) / kOzTileM) * (oz[i].s.Np / kOzTileN);
    total += counts[i];
  }
  for (int t = team.rank(); t < total; t += team.size()) {
    int i = 0, local = t;
    while (local >= counts[i]) local -= counts[i++];
    const int tn_count = oz[i].s.Np / kOzTileN;
    if (!oz_tile(oz[i], local / tn_count, local % tn_count, st, smem, status)) return false;
  }
  return true;
}

}  // namespace sinvb
