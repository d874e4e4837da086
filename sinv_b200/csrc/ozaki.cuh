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
// in (-1, 1).  Each scaled value x is rounded once to a multiple of 2^(1-7S)
// and cut into S signed digits
//   x = sum_t d_t 2^(-6-7(t-1)),  t = 1..S,  d_1 in [-64, 64], d_t in [-64, 63]
// which int8 holds exactly.  Digit products are exact in int32 and so are
// their sums (|sum| <= S * 2K * 2^12 < 2^31 for 2K <= 2^16), so the only
// errors are the rounding of the operands and the levels L = s + t > S + 1
// left out:
//   C_ij = 2^(e_i + f_j) sum_{L=2}^{S+1} 2^(-12-7(L-2)) sum_{s+t=L} (A_s B_t)_ij.
// Complex operands are embedded as real matrices: per 64-row group of A the
// 128 MMA rows are [Re A | -Im A] (64 rows) and [Im A | Re A] (64 rows), B^T
// rows are [Re B(:,j) | Im B(:,j)], so one 128 x 64 x 2K real product gives the
// real and the imaginary parts of a 64 x 64 complex tile in TMEM lanes 0-63 and
// 64-127.  Each level owns 64 TMEM columns (S <= 8 levels in 512 columns);
// the B digits of one A digit s sit next to each other in shared memory, so a
// single MMA with N = 64 * (number of B digits, at most 4) feeds the run of
// levels s+1, s+2, ... at once.
//
// Digit planes live in global memory in the canonical K-major core-matrix
// layout of tcgen05 (8 rows x 16 bytes per core matrix) with 32-byte K-blocks:
// the K-block of 128 A rows (64 B rows) is one contiguous 4 KB (2 KB) run that
// one bulk copy moves into the shared-memory stage ring.
//   offset(r, k) = ((k/32 * R/8 + r/8) * 2 + (k%32)/16) * 128 + (r%8) * 16 + k%16
// The two halves of K' = 2 Kh start at 0 and Kh = K rounded up to 16.
#pragma once

#include "block_gemm.cuh"
#include "tc_common.cuh"

namespace sinvb {

constexpr int kOzMaxDigits = 8;
constexpr int kOzTileM = 64;                          // complex rows per output tile (128 MMA rows)
constexpr int kOzTileN = 64;                          // complex columns per output tile
constexpr int kOzKBlock = 32;                         // K' bytes per pipeline stage (one MMA's K)
constexpr int kOzMaxStages = 4;
constexpr int kOzStageA = 2 * kOzTileM * kOzKBlock;   // 4096 B: one digit of a 128-row A block
constexpr int kOzStageB = kOzTileN * kOzKBlock;       // 2048 B: one digit of a 64-row B^T block
constexpr int kOzEpiCols = 32;                        // output columns per epilogue staging pass
constexpr int kOzEpiStride = 2 * kOzEpiCols + 1;      // doubles per staged row (odd: no bank conflicts)
constexpr size_t kOzEpiBytes = (size_t)kOzTileM * kOzEpiStride * 8;
static_assert(kOzTileN % kOzEpiCols == 0 && (kOzTileM * kOzEpiCols) % 128 == 0, "epilogue passes");

__host__ __device__ inline int oz_pad(int x, int m) { return (x + m - 1) / m * m; }

// Geometry of the digit planes of one operand pair.
struct OzShape {
  int M, N, K;  // complex sizes
  int Kh;       // K rounded up to 16: start of the second half of K'
  int Mp;       // embedded A rows: 2 x (M rounded up to 64)
  int Np;       // B^T rows: N rounded up to 64
  int Kp;       // K' = 2 Kh bytes per digit row (a multiple of 32)
  int S;        // digits
  __host__ __device__ size_t a_plane() const { return (size_t)Mp * Kp; }
  __host__ __device__ size_t b_plane() const { return (size_t)Np * Kp; }
};

__host__ __device__ inline OzShape oz_shape(int M, int N, int K, int S) {
  OzShape s;
  s.M = M; s.N = N; s.K = K; s.S = S;
  s.Kh = oz_pad(K, 16);
  s.Mp = oz_pad(M, kOzTileM) * 2;
  s.Np = oz_pad(N, kOzTileN);
  s.Kp = 2 * s.Kh;
  return s;
}

// Stages of the ring: four, three for 8 digits (shared memory).  A fifth stage
// for 7 digits (with 8-column epilogue passes to make room) measured no faster.
__host__ __device__ constexpr int oz_stages(int S) { return S <= 7 ? 4 : 3; }
__host__ __device__ constexpr size_t oz_stage_bytes(int S) { return (size_t)S * (kOzStageA + kOzStageB); }
// ring, epilogue staging, 128 exponents of the tile being written (the
// slicing phase reuses the same space, see oz_slice_smem)
__host__ __device__ constexpr size_t oz_smem_bytes(int S) {
  return oz_stages(S) * oz_stage_bytes(S) + kOzEpiBytes + 128 * sizeof(int);
}

__host__ __device__ __forceinline__ size_t oz_off(int r, int k, int R) {
  return ((size_t)((k >> 5) * (R >> 3) + (r >> 3)) * 2 + ((k >> 4) & 1)) * 128 + (r & 7) * 16 + (k & 15);
}

// The S digits of x in (-1, 1), d[0] most significant: m = round(x 2^(7S-1))
// cut into base-128 digits with balanced remainders (in [-64, 63]) from the
// bottom up.  m is split in FP64 as H 2^(7L) + Lo (L = S/2 low digits,
// |Lo| <= 2^(7L-1)) so the digit arithmetic runs on 32-bit integers; the
// representation is unique, so the split changes no digit.
template <int S>
__device__ __forceinline__ void oz_split(double x, int (&d)[S]) {
  constexpr int L = S / 2;
  if constexpr (L == 0) {
    d[0] = __double2int_rn(x * 64.0);
  } else {
    const double m = rint(x * (double)(1ull << (7 * S - 1)));
    const double h = rint(m * (1.0 / (double)(1ull << (7 * L))));
    int lo = __double2int_rn(fma(-h, (double)(1ull << (7 * L)), m));
    int hi = __double2int_rn(h);
#pragma unroll
    for (int t = S - 1; t >= S - L; t--) {
      const int r = ((lo + 64) & 127) - 64;
      d[t] = r;
      lo = (lo - r) >> 7;
    }
    hi += lo;  // carry out of the low part: -1, 0 or 1
#pragma unroll
    for (int t = S - L - 1; t >= 1; t--) {
      const int r = ((hi + 64) & 127) - 64;
      d[t] = r;
      hi = (hi - r) >> 7;
    }
    d[0] = hi;
  }
}

__device__ __forceinline__ int oz_exponent(double amax) {
  int e = 0;
  if (amax > 0.0) frexp(amax, &e);
  return e;
}

__device__ __forceinline__ double oz_pow2(int e) {
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

// Four signed bytes (low byte of each argument) packed little-endian.
__device__ __forceinline__ uint32_t oz_pack4(int b0, int b1, int b2, int b3) {
  return __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
}

// A side, by CTAs: CTA-group g holds the 8 complex rows 8g .. 8g+7 (warp w
// loads row 8g + w, lane l the K = 4l + 128m + q, q < 4, so each load of a
// warp is one contiguous 2 KB run), whose embedded rows form two whole 8-row
// groups of the planes.  The digits of a chunk of kOzAChunk K are assembled in
// shared memory as core matrices (8 rows x 16 bytes, padded to 144 bytes so
// the 4-byte writes of a warp hit 32 banks) and copied out with 16-byte
// stores, eight lanes per 128-byte core matrix.  Rows past M are written as
// zeros (they only reach output rows that are never stored).
constexpr int kOzAChunk = 512;                  // K per staging pass (4 x 128)
constexpr int kOzCmStride = 144;                // staged bytes per core matrix
constexpr int kOzACms = kOzAChunk / 16;         // core matrices per (digit, row group, half)
__host__ __device__ constexpr size_t oz_slice_a_smem(int S) { return (size_t)S * 4 * kOzACms * kOzCmStride; }

template <int S>
__device__ inline void oz_slice_a(const cplx* A, int lda, const OzShape& s, int8_t* planes, int* ea, int g0,
                                  int gstep, unsigned char* stage) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int groups = (s.M + 7) / 8;
  for (int g = g0; g < groups; g += gstep) {
    const int i = 8 * g + warp;
    const bool live = i < s.M;
    const cplx* row = A + (size_t)i * lda;
    cplx v[4][4];
    double amax = 0.0;
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int k = 128 * m + 4 * lane + q;
        v[m][q] = (live && k < s.K) ? row[k] : cplx{0.0, 0.0};
        amax = fmax(amax, fmax(fabs(v[m][q].re), fabs(v[m][q].im)));
      }
    for (int k = kOzAChunk + lane; live && k < s.K; k += 32) {
      const cplx w = row[k];
      amax = fmax(amax, fmax(fabs(w.re), fabs(w.im)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const int e = oz_exponent(amax);
    if (lane == 0 && live) ea[i] = e;
    const double sc = ldexp(1.0, -e);
    const int gre = (8 * g / kOzTileM) * 2 * kOzTileM + (8 * g) % kOzTileM;  // first embedded row (Re part)
    for (int k0 = 0; k0 < s.Kh; k0 += kOzAChunk) {
      if (k0 > 0) {
#pragma unroll
        for (int m = 0; m < 4; m++)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int k = k0 + 128 * m + 4 * lane + q;
            v[m][q] = (live && k < s.K) ? row[k] : cplx{0.0, 0.0};
          }
      }
      const int kc = s.Kh - k0 < kOzAChunk ? s.Kh - k0 : kOzAChunk;  // multiple of 16
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int kk = 128 * m + 4 * lane;  // within the chunk
        if (kk < kc) {
          int dx[4][S], dy[4][S];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            oz_split<S>(v[m][q].re * sc, dx[q]);
            oz_split<S>(v[m][q].im * sc, dy[q]);
          }
          // staging index: [digit][group: 0 = Re rows, 1 = Im rows][half][core matrix]
          const int cm = kk >> 4, byte = warp * 16 + (kk & 15);
#pragma unroll
          for (int t = 0; t < S; t++) {
            const uint32_t wr = oz_pack4(dx[0][t], dx[1][t], dx[2][t], dx[3][t]);
            const uint32_t wi = oz_pack4(dy[0][t], dy[1][t], dy[2][t], dy[3][t]);
            unsigned char* b0 = stage + (size_t)t * 4 * kOzACms * kOzCmStride + cm * kOzCmStride + byte;
            *reinterpret_cast<uint32_t*>(b0) = wr;                                        // Re rows, first half
            *reinterpret_cast<uint32_t*>(b0 + 1 * kOzACms * kOzCmStride) = __vsub4(0u, wi);  // Re rows, -Im
            *reinterpret_cast<uint32_t*>(b0 + 2 * kOzACms * kOzCmStride) = wi;            // Im rows, Im
            *reinterpret_cast<uint32_t*>(b0 + 3 * kOzACms * kOzCmStride) = wr;            // Im rows, Re
          }
        }
      }
      __syncthreads();
      // copy out: item = (digit, quarter, core matrix, row); 16 bytes each
      const int ncm = kc / 16, items = S * 4 * ncm * 8;
      for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int r8 = it & 7, rest = it >> 3;
        const int cm = rest % ncm, qt = (rest / ncm) & 3, t = rest / ncm / 4;
        const int rowe = gre + (qt >> 1) * kOzTileM + r8;       // embedded row
        const int kp = (qt & 1) * s.Kh + k0 + 16 * cm;          // K' byte
        const uint4 w = *reinterpret_cast<const uint4*>(stage + ((size_t)(t * 4 + qt) * kOzACms + cm) * kOzCmStride +
                                                        r8 * 16);
        *reinterpret_cast<uint4*>(planes + (size_t)t * s.a_plane() + oz_off(rowe, kp, s.Mp)) = w;
      }
      __syncthreads();
    }
  }
}

// B side for the 32-column blocks cb0, cb0 + cbstep, ... (up to 4 at a time):
// column exponents f_j (warps split the rows, each lane keeps the maxima of
// one column per block, then a reduction in shared memory), then the digit
// planes of the B^T rows [Re B(:,j) | Im B(:,j)] (each thread 16 consecutive K
// of one column, one 16-byte store per digit and half; eight lanes fill one
// 128-byte core matrix).  Called by every thread of the CTA; `red` is
// 4 x blockDim.x doubles of shared memory.  Columns past N are left unwritten
// (they only reach discarded outputs).
template <int S>
__device__ inline void oz_slice_b(const cplx* B, int ldb, const OzShape& s, int8_t* planes, int* fb, int cb0, int cbstep,
                                  double* red) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int blocks = (s.N + 31) / 32;
  for (int cb1 = cb0; cb1 < blocks; cb1 += 4 * cbstep) {
    int js[4];
    double amax[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int cb = cb1 + r * cbstep;
      js[r] = cb < blocks ? cb * 32 + lane : s.N;
      amax[r] = 0.0;
    }
#pragma unroll 4
    for (int k = warp; k < s.K; k += nw) {
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (js[r] < s.N) {
          const cplx v = B[(size_t)k * ldb + js[r]];
          amax[r] = fmax(amax[r], fmax(fabs(v.re), fabs(v.im)));
        }
    }
#pragma unroll
    for (int r = 0; r < 4; r++) red[(r * nw + warp) * 32 + lane] = amax[r];
    __syncthreads();
    if (warp < 4) {  // warp r finishes block r
      const int r = warp;
      double mx = 0.0;
      for (int w = 0; w < nw; w++) mx = fmax(mx, red[(r * nw + w) * 32 + lane]);
      const int f = oz_exponent(mx);
      const int cb = cb1 + r * cbstep, j = cb * 32 + lane;
      if (cb < blocks && j < s.N) fb[j] = f;
      red[4 * nw * 32 + r * 32 + lane] = ldexp(1.0, -f);
    }
    __syncthreads();
    const int per = s.Kh / 16;  // 16-K groups per column
    for (int w = warp; w < 4 * per; w += nw) {
      const int r = w / per, k16 = 16 * (w % per);
      const int j = js[r];
      if (j >= s.N) continue;  // warp-uniform: whole block past N
      const double sc = red[4 * nw * 32 + r * 32 + lane];
      const bool valid = j < s.N;
      cplx v[16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int k = k16 + q;
        v[q] = (valid && k < s.K) ? B[(size_t)k * ldb + j] : cplx{0.0, 0.0};
      }
      uint32_t wr[S][4], wi[S][4];
#pragma unroll
      for (int g = 0; g < 4; g++) {
        int dx[4][S], dy[4][S];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          oz_split<S>(v[4 * g + q].re * sc, dx[q]);
          oz_split<S>(v[4 * g + q].im * sc, dy[q]);
        }
#pragma unroll
        for (int t = 0; t < S; t++) {
          wr[t][g] = oz_pack4(dx[0][t], dx[1][t], dx[2][t], dx[3][t]);
          wi[t][g] = oz_pack4(dy[0][t], dy[1][t], dy[2][t], dy[3][t]);
        }
      }
      if (valid) {
        const size_t o_r = oz_off(j, k16, s.Np), o_i = oz_off(j, s.Kh + k16, s.Np);
#pragma unroll
        for (int t = 0; t < S; t++) {
          int8_t* pl = planes + (size_t)t * s.b_plane();
          *reinterpret_cast<uint4*>(pl + o_r) = make_uint4(wr[t][0], wr[t][1], wr[t][2], wr[t][3]);
          *reinterpret_cast<uint4*>(pl + o_i) = make_uint4(wi[t][0], wi[t][1], wi[t][2], wi[t][3]);
        }
      }
    }
    __syncthreads();  // `red` is reused by the next batch of blocks
  }
}

// Per-CTA state of the tile pipeline; lives in shared memory for the whole kernel.
struct OzState {
  uint64_t full[kOzMaxStages];   // stage filled (bulk copies landed)
  uint64_t empty[kOzMaxStages];  // stage consumed (MMAs done)
  uint64_t tmem_full;            // a tile's accumulators are complete
  uint64_t tmem_empty;           // the epilogue has read them (128 arrivals)
  unsigned tmem;                 // TMEM base address
  unsigned kblocks;              // k-blocks streamed so far (stage index and phases of full / empty)
  unsigned tiles;                // tiles finished so far (phases of tmem_full / tmem_empty)
  int fail;                      // a bounded wait gave up: the pipeline phases are no longer known
};

// One-time set-up by the whole CTA: barriers and a TMEM allocation (warp 0).
__device__ inline void oz_setup(OzState* st) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzMaxStages; s++) {
      mbar_init(&st->full[s], 1);
      mbar_init(&st->empty[s], 1);
    }
    mbar_init(&st->tmem_full, 1);
    mbar_init(&st->tmem_empty, 128);
    st->kblocks = 0;
    st->tiles = 0;
    st->fail = 0;
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

// One product of a tile routine call: digit planes, exponents, output.
struct OzOp {
  const int8_t* a_planes;
  const int8_t* b_planes;
  const int* ea;
  const int* fb;
  OzShape s;
  int tiles;  // (Mp / 128) x (Np / 64) output tiles, numbered row by row
  const cplx* D;
  cplx* C;
  int ldd, ldc;
  double alpha, beta;
};

__host__ __device__ inline int oz_tile_count(const OzShape& s) { return (s.Mp / (2 * kOzTileM)) * (s.Np / kOzTileN); }

// The MMAs of one k-block: for every A digit a, B digits 1 .. S+1-a in runs
// of at most 4 (N <= 256); the run starting at B digit b0 lands in the TMEM
// columns of levels a+b0, a+b0+1, ...  The A digit 1 runs cover every level,
// so on the first k-block of a tile they overwrite the accumulators.
template <int S>
__device__ __forceinline__ void oz_issue_s(uint64_t adesc, uint64_t bdesc, unsigned tmem, bool first) {
#pragma unroll
  for (int a = 1; a <= S; a++) {
#pragma unroll
    for (int b0 = 1; b0 <= S + 1 - a; b0 += 4) {
      const int cnt = (S + 2 - a - b0) < 4 ? (S + 2 - a - b0) : 4;
      mma_i8(tmem + (unsigned)((a + b0 - 2) * 64), adesc + (uint64_t)((a - 1) * (kOzStageA >> 4)),
             bdesc + (uint64_t)((b0 - 1) * (kOzStageB >> 4)), idesc_i8(128, 64 * cnt), !(first && a == 1));
    }
  }
}

__device__ __forceinline__ void oz_issue(int S, uint64_t adesc, uint64_t bdesc, unsigned tmem, bool first) {
  switch (S) {
    case 1: oz_issue_s<1>(adesc, bdesc, tmem, first); break;
    case 2: oz_issue_s<2>(adesc, bdesc, tmem, first); break;
    case 3: oz_issue_s<3>(adesc, bdesc, tmem, first); break;
    case 4: oz_issue_s<4>(adesc, bdesc, tmem, first); break;
    case 5: oz_issue_s<5>(adesc, bdesc, tmem, first); break;
    case 6: oz_issue_s<6>(adesc, bdesc, tmem, first); break;
    case 7: oz_issue_s<7>(adesc, bdesc, tmem, first); break;
    default: oz_issue_s<8>(adesc, bdesc, tmem, first); break;
  }
}

// Barrier 1 of the four epilogue warps (128 threads), and its AND-reduction.
__device__ __forceinline__ void oz_epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ bool oz_epi_all(bool p) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, 128, p;\n\t"
      "selp.b32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((int)p)
      : "memory");
  return r != 0;
}

struct OzTileRef {
  int op, tm, tn;
};
__device__ __forceinline__ OzTileRef oz_tile_ref(const OzOp* ops, int nops, int t) {
  int i = 0;
  while (i + 1 < nops && t >= ops[i].tiles) t -= ops[i].tiles, i++;
  const int tn_count = ops[i].s.Np / kOzTileN;
  return {i, t / tn_count, t % tn_count};
}

// Output tiles t = first, first + stride, ... of the ops (numbered op by op):
// warp 0 streams digit blocks into the stage ring, warp 1 issues the MMAs into
// TMEM, warps 4-7 read the levels back, rebuild FP64 and write C, while the
// MMAs of the next tile already run.  Called by every thread of the CTA with
// the same arguments; all ops have the same digit count.  Returns false when
// a bounded wait gave up (status reported).
__device__ inline bool oz_tiles(const OzOp* ops, int nops, int first, int stride, OzState* st, unsigned char* smem,
                                int* status) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = ops[0].s.S, NS = oz_stages(S);
  const size_t stage = oz_stage_bytes(S);
  int total = 0;
  for (int i = 0; i < nops; i++) total += ops[i].tiles;
  unsigned my_kb = 0, my_tiles = 0;
  for (int t = first; t < total; t += stride) {
    my_kb += ops[oz_tile_ref(ops, nops, t).op].s.Kp / kOzKBlock;
    my_tiles++;
  }
  // the ring area may hold data written through the generic proxy (FP64 tiles)
  fence_proxy_async_smem();
  __syncthreads();
  const unsigned kb0 = st->kblocks, t0 = st->tiles;
  if (st->fail) return false;

  if (warp == 0) {
    if (lane == 0) {  // producer
      unsigned g = kb0;
      bool ok = true;
      for (int t = first; t < total && ok; t += stride) {
        const OzTileRef r = oz_tile_ref(ops, nops, t);
        const OzOp& op = ops[r.op];
        const int nkb = op.s.Kp / kOzKBlock;
        for (int kb = 0; kb < nkb; kb++, g++) {
          const unsigned sidx = g % NS, use = g / NS;
          if (use > 0 && !mbar_wait(&st->empty[sidx], (use - 1) & 1, status)) {
            ok = false;
            break;
          }
          unsigned char* base = smem + sidx * stage;
          mbar_expect_tx(&st->full[sidx], (unsigned)stage);
          const size_t aoff = (size_t)(kb * (op.s.Mp >> 3) + r.tm * 16) * 256;
          const size_t boff = (size_t)(kb * (op.s.Np >> 3) + r.tn * 8) * 256;
          for (int d = 0; d < S; d++) {
            bulk_g2s(base + d * kOzStageA, op.a_planes + d * op.s.a_plane() + aoff, kOzStageA, &st->full[sidx]);
            bulk_g2s(base + S * kOzStageA + d * kOzStageB, op.b_planes + d * op.s.b_plane() + boff, kOzStageB,
                     &st->full[sidx]);
          }
        }
      }
      if (!ok) st->fail = 1;
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      unsigned g = kb0, T = t0;
      bool ok = true;
      const uint64_t d0 = sdesc(smem, 128, 256);
      for (int t = first; t < total && ok; t += stride) {
        const OzOp& op = ops[oz_tile_ref(ops, nops, t).op];
        const int nkb = op.s.Kp / kOzKBlock;
        if (T > 0 && !mbar_wait(&st->tmem_empty, (T - 1) & 1, status)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int kb = 0; kb < nkb; kb++, g++) {
          const unsigned sidx = g % NS, use = g / NS;
          if (!mbar_wait(&st->full[sidx], use & 1, status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = d0 + (uint64_t)((sidx * stage) >> 4);
          oz_issue(S, ad, ad + (uint64_t)((S * kOzStageA) >> 4), st->tmem, kb == 0);
          mma_commit(&st->empty[sidx]);
        }
        if (!ok) break;
        mma_commit(&st->tmem_full);
        T++;
      }
      if (!ok) st->fail = 1;
    }
  } else if (warp >= 4) {  // epilogue: TMEM lanes 32 (warp - 4) ...
    const int et = threadIdx.x - 128;       // 0..127
    const int i = et & 63, part = et >> 6;  // complex row in the tile, 0 = Re / 1 = Im
    const unsigned lane_base = st->tmem + ((unsigned)(32 * (warp - 4)) << 16);
    double* stg = reinterpret_cast<double*>(smem + NS * stage);
    int* exps = reinterpret_cast<int*>(smem + NS * stage + kOzEpiBytes);  // [0,64): f_j, [64,128): e_i
    unsigned T = t0;
    bool ok = true;
    for (int t = first; t < total; t += stride) {
      const OzTileRef r = oz_tile_ref(ops, nops, t);
      const OzOp& op = ops[r.op];
      {  // exponents of the tile's columns and rows, fetched while the MMAs run
        const int g = et < 64 ? r.tn * kOzTileN + et : r.tm * kOzTileM + (et - 64);
        exps[et] = et < 64 ? (g < op.s.N ? op.fb[g] : 0) : (g < op.s.M ? op.ea[g] : 0);
      }
      ok = oz_epi_all(mbar_wait(&st->tmem_full, T & 1, status));  // also orders `exps`
      if (!ok) break;
      tc_fence_after();
      // Horner over the levels, least significant first: acc = sum_L v_L 2^(-7(L-2))
      double acc[kOzTileN];  // the tile's 64 columns, Re or Im part (by `part`)
      {
        int v[32];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          tmem_ld32(lane_base + (unsigned)((S - 1) * 64 + h * 32), v);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 32; c++) acc[h * 32 + c] = (double)v[c];
        }
        for (int L = S; L >= 2; L--) {
#pragma unroll
          for (int h = 0; h < 2; h++) {
            tmem_ld32(lane_base + (unsigned)((L - 2) * 64 + h * 32), v);
            tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 32; c++) acc[h * 32 + c] = fma(acc[h * 32 + c], 0.0078125, (double)v[c]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&st->tmem_empty);  // the next tile's MMAs may overwrite the accumulators
      const int ei = exps[64 + i] - 12;
      const bool addend = op.D != nullptr && op.beta != 0.0;
#pragma unroll
      for (int h = 0; h < kOzTileN / kOzEpiCols; h++) {
#pragma unroll
        for (int c = 0; c < kOzEpiCols; c++)
          stg[i * kOzEpiStride + 2 * c + part] =
              op.alpha * acc[h * kOzEpiCols + c] * oz_pow2(ei + exps[h * kOzEpiCols + c]);
        oz_epi_sync();
        // kPer entries per thread: all addend loads first, then the stores
        constexpr int kPer = kOzTileM * kOzEpiCols / 128;
        cplx dv[kPer];
#pragma unroll
        for (int m = 0; m < kPer; m++) {
          const int e = et + 128 * m, ii = e / kOzEpiCols, c = e % kOzEpiCols;
          const int gi = r.tm * kOzTileM + ii, gj = r.tn * kOzTileN + h * kOzEpiCols + c;
          dv[m] = (addend && gi < op.s.M && gj < op.s.N) ? op.D[(size_t)gi * op.ldd + gj] : cplx{0.0, 0.0};
        }
#pragma unroll
        for (int m = 0; m < kPer; m++) {
          const int e = et + 128 * m, ii = e / kOzEpiCols, c = e % kOzEpiCols;
          const int gi = r.tm * kOzTileM + ii, gj = r.tn * kOzTileN + h * kOzEpiCols + c;
          if (gi < op.s.M && gj < op.s.N) {
            const double re = stg[ii * kOzEpiStride + 2 * c], im = stg[ii * kOzEpiStride + 2 * c + 1];
            op.C[(size_t)gi * op.ldc + gj] = addend ? cplx{fma(op.beta, dv[m].re, re), fma(op.beta, dv[m].im, im)}
                                                    : cplx{re, im};
          }
        }
        oz_epi_sync();
      }
      T++;
    }
    if (!ok && et == 0) st->fail = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && !st->fail) {
    st->kblocks = kb0 + my_kb;
    st->tiles = t0 + my_tiles;
  }
  __syncthreads();
  return st->fail == 0;
}

// Scratch one product of the team routine needs: exponents and digit planes.
__host__ __device__ inline size_t oz_op_scratch(int M, int N, int K, int S) {
  const OzShape s = oz_shape(M, N, K, S);
  return (size_t)oz_pad(M * 4, 256) + oz_pad(N * 4, 256) + (size_t)S * (s.a_plane() + s.b_plane());
}

// Fills an OzOp for C = beta D + alpha A B with its scratch at `p`; returns the
// end of the scratch it took.
__host__ __device__ inline unsigned char* oz_bind(OzOp& o, int M, int N, int K, int S, unsigned char* p, double alpha,
                                                  double beta, const cplx* D, int ldd, cplx* C, int ldc) {
  o.s = oz_shape(M, N, K, S);
  o.tiles = oz_tile_count(o.s);
  o.ea = reinterpret_cast<int*>(p);
  p += oz_pad(M * 4, 256);
  o.fb = reinterpret_cast<int*>(p);
  p += oz_pad(N * 4, 256);
  o.a_planes = reinterpret_cast<int8_t*>(p);
  p += (size_t)S * o.s.a_plane();
  o.b_planes = reinterpret_cast<int8_t*>(p);
  p += (size_t)S * o.s.b_plane();
  o.D = D;
  o.C = C;
  o.ldd = ldd;
  o.ldc = ldc;
  o.alpha = alpha;
  o.beta = beta;
  return p;
}

// Digits and exponents of the operands of `nops` products: A row groups
// a0, a0 + astep, ..., B column blocks b0, b0 + bstep, ...  Called by every
// thread of the CTA; `smem` holds oz_slice_smem(S) bytes.
__host__ __device__ constexpr size_t oz_slice_smem(int S) {
  return oz_slice_a_smem(S) > 4 * 256 * 8 + 4 * 32 * 8 ? oz_slice_a_smem(S) : 4 * 256 * 8 + 4 * 32 * 8;
}

// Operands to slice: bit i of slice_a / slice_b for op i's A / B (an operand
// whose planes are already in place, from an earlier call or another op of
// this one, is skipped).
template <int S>
__device__ inline void oz_slice_ops_s(const GemmOp<cplx>* ops, const OzOp* oz, int nops, unsigned slice_a,
                                      unsigned slice_b, int a0, int astep, int b0, int bstep, unsigned char* smem) {
  for (int i = 0; i < nops; i++) {
    if ((slice_a >> i) & 1u)
      oz_slice_a<S>(ops[i].A, ops[i].lda, oz[i].s, const_cast<int8_t*>(oz[i].a_planes), const_cast<int*>(oz[i].ea),
                    a0, astep, smem);
    if ((slice_b >> i) & 1u)
      oz_slice_b<S>(ops[i].B, ops[i].ldb, oz[i].s, const_cast<int8_t*>(oz[i].b_planes), const_cast<int*>(oz[i].fb),
                    b0, bstep, reinterpret_cast<double*>(smem));
  }
}

__device__ inline void oz_slice_ops(int S, const GemmOp<cplx>* ops, const OzOp* oz, int nops, unsigned slice_a,
                                    unsigned slice_b, int a0, int astep, int b0, int bstep, unsigned char* smem) {
  switch (S) {
    case 1: oz_slice_ops_s<1>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 2: oz_slice_ops_s<2>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 3: oz_slice_ops_s<3>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 4: oz_slice_ops_s<4>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 5: oz_slice_ops_s<5>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 6: oz_slice_ops_s<6>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    case 7: oz_slice_ops_s<7>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
    default: oz_slice_ops_s<8>(ops, oz, nops, slice_a, slice_b, a0, astep, b0, bstep, smem); break;
  }
}

// Operand slots of the team products: scratch holds two A-role slots (row
// exponents and embedded digit planes) and two B-role slots (column exponents
// and digit planes), each for an M x K (K x N) operand; 2 oz_op_scratch(M, N,
// K, S) bytes in all.  A product names the slot of each operand and whether
// the operand is sliced in this call or its planes are reused, so an operand
// shared by consecutive products is sliced once.
struct OzSlots {
  int a[2], b[2];      // slot of op i's A / B operand
  unsigned slice_a;    // bit i: slice op i's A into its slot
  unsigned slice_b;    // bit i: slice op i's B into its slot
};

__host__ __device__ inline size_t oz_slot_a_bytes(const OzShape& s) {
  return (size_t)oz_pad(s.M * 4, 256) + (size_t)s.S * s.a_plane();
}
__host__ __device__ inline size_t oz_slot_b_bytes(const OzShape& s) {
  return (size_t)oz_pad(s.N * 4, 256) + (size_t)s.S * s.b_plane();
}

// Up to 2 independent complex block products C = beta D + alpha A B on the
// int8 tensor cores, spread over a team of CTAs (the mixed-precision form of
// team_gemm).  Two phases: digits and exponents of every operand (A row groups
// and B column blocks over the CTAs of the team), then the output tiles
// (over its CTAs).  The caller synchronises after the second.  Plain
// (non-transposed) operands only.  Returns false when a wait gave up.
//
// The operands of all products of one sweep have the same shape (M = N = K =
// the block size), so one slot size fits every operand; `slots` says which
// operands this call slices and which planes it reuses (OzSlots).
template <class Team>
__device__ bool team_gemm_ozaki(Team& team, const GemmOp<cplx>* ops, int nops, int S, unsigned char* scratch,
                                const OzSlots& slots, OzState* st, unsigned char* smem, int* status) {
  if (st->fail) {  // an earlier wait of this CTA gave up: its pipeline state is unknown
    report(status, SINVB_STATUS_TIMEOUT);
    return false;
  }
  OzOp oz[2];
  const OzShape s0 = oz_shape(ops[0].M, ops[0].N, ops[0].K, S);
  const size_t sa = oz_slot_a_bytes(s0), sb = oz_slot_b_bytes(s0);
  for (int i = 0; i < nops; i++) {
    const GemmOp<cplx>& g = ops[i];
    OzOp& o = oz[i];
    o.s = oz_shape(g.M, g.N, g.K, S);
    o.tiles = oz_tile_count(o.s);
    unsigned char* pa = scratch + (size_t)slots.a[i] * sa;
    unsigned char* pb = scratch + 2 * sa + (size_t)slots.b[i] * sb;
    o.ea = reinterpret_cast<int*>(pa);
    o.a_planes = reinterpret_cast<int8_t*>(pa + oz_pad(g.M * 4, 256));
    o.fb = reinterpret_cast<int*>(pb);
    o.b_planes = reinterpret_cast<int8_t*>(pb + oz_pad(g.N * 4, 256));
    o.D = g.D;
    o.C = g.C;
    o.ldd = g.ldd;
    o.ldc = g.ldc;
    o.alpha = g.alpha;
    o.beta = g.beta;
  }
  oz_slice_ops(S, ops, oz, nops, slots.slice_a, slots.slice_b, team.rank(), team.size(), team.rank(), team.size(),
               smem);
  // the planes are read by the bulk-copy (async) proxy of every CTA of the team
  asm volatile("fence.proxy.async.global;" ::: "memory");
  if (!team.sync()) return false;
  asm volatile("fence.proxy.async.global;" ::: "memory");
  return oz_tiles(oz, nops, team.rank(), team.size(), st, smem, status);
}

}  // namespace sinvb
