// Two-sided RGF selected inversion on one GPU.
//
// Reference: src/sinv/algorithms/rgf/rgf2sided.py:18-274, where two MPI
// processes sweep the upper and the lower half of the block chain towards the
// middle and exchange their connected blocks.  Here the two halves are two
// teams of CTAs of one cooperative launch, so a single large matrix runs two
// dependency chains of about n/2 steps at once instead of one of n:
//
//   left team  (blocks 0 .. m-1, left to right):  g^L_i = (A_ii - A_{i,i-1} g^L_{i-1} A_{i-1,i})^-1
//   right team (blocks n-1 .. m+1, right to left): g^R_i = (A_ii - A_{i,i+1} g^R_{i+1} A_{i+1,i})^-1
//   whole grid, middle block m = (n-1)/2:
//     G_mm = (A_mm - A_{m,m-1} g^L_{m-1} A_{m-1,m} - A_{m,m+1} g^R_{m+1} A_{m+1,m})^-1
//   each team then runs the backward recursion of rgf.py:51-62 outwards from G_mm.
//
// The right half is the left half's code on the block chain read backwards:
// with j = n-1-i its diagonal is A_{n-1-j}, its "upper" block A'_{j,j+1} is
// the original lower block A_{n-1-j,n-2-j}, its "lower" block the original
// upper one, and likewise for the outputs, so every half-sweep routine takes
// block sequences with a signed stride.  The middle product is one GEMM with
// two terms: S = A_mm - L X^L - R X^R with X^L = g^L_{m-1} A_{m-1,m} and
// X^R = g^R_{m+1} A_{m+1,m}, kept from the last forward step of each team.
//
// Storage: as in the one-sided sweep (rgf_sweep.cuh) every half keeps
// X_i = g_i A'_{i,i+1} in G'_lower[i] and P_{i+1} = A'_{i+1,i} g_i in
// G'_upper[i] until its backward step overwrites them, so SAVE_OFFDIAG is
// required; the two halves touch disjoint output blocks.
#include "block_inverse.cuh"
#include "host_util.h"

namespace sinvb {

// Block i of a sequence at base + i * stride (elements; the stride may be negative).
template <class T>
struct Blocks {
  T* base;
  long long stride;
  __device__ __forceinline__ T* operator()(int i) const { return base + (long long)i * stride; }
};

template <class T>
struct HalfSweep {
  Blocks<const T> diag, upper, lower;  // in sweep order: A_ii, A_{i,i+1}, A_{i+1,i}
  Blocks<T> Gd, Gu, Gl;                // G_ii, G_{i,i+1}, G_{i+1,i} in sweep order
  T* T0;                               // b x b ping-pong of the backward sweep
  T* T1;
  T* side;                             // invert_side_elems(b)
  int len;                             // blocks before the middle; block len is the middle
};

template <class T>
struct Rgf2sParams {
  HalfSweep<T> half[2];  // 0: left team, 1: right team
  const T* mid_diag;     // A_mm
  T* mid_G;              // G_mm
  WsHeader* hdr;
  int* status;
  int b;
  unsigned flags;
};

// Forward sweep of one half: g_0 .. g_{len-1} in Gd, then the X / P blocks of
// the step into the middle (X_{len-1} in Gl[len-1], P_len in Gu[len-1]).
template <class T, int BM, int BN, class Team>
__device__ bool half_forward(Team& team, const HalfSweep<T>& h, int b, int* status, T* smem) {
  if (h.len == 0) return true;
  team_copy<T>(team, b, b, h.diag(0), b, h.Gd(0), b);
  if (!team.sync()) return false;
  if (!team_invert<T, BM, BN>(team, h.Gd(0), b, b, h.side, status, smem)) return false;
  for (int i = 1; i <= h.len; i++) {
    const T* g = h.Gd(i - 1);
    {  // X_{i-1} = g_{i-1} U_{i-1},  P_i = L_i g_{i-1}
      GemmOp<T> ops[2];
      ops[0] = make_op<T>(b, b, b, 1.0, g, b, h.upper(i - 1), b, nullptr, 0, h.Gl(i - 1), b);
      ops[1] = make_op<T>(b, b, b, 1.0, h.lower(i - 1), b, g, b, nullptr, 0, h.Gu(i - 1), b);
      team_gemm<T, BM, BN>(team, ops, 2, smem);
    }
    if (!team.sync()) return false;
    if (i == h.len) break;  // the middle block is the whole grid's
    {  // S_i = A_ii - P_i U_{i-1}
      GemmOp<T> op = make_op<T>(b, b, b, -1.0, h.Gu(i - 1), b, h.upper(i - 1), b, h.diag(i), b, h.Gd(i), b);
      team_gemm<T, BM, BN>(team, &op, 1, smem);
    }
    if (!team.sync()) return false;
    if (!team_invert<T, BM, BN>(team, h.Gd(i), b, b, h.side, status, smem)) return false;
  }
  return true;
}

// Backward sweep of one half from G_len = G_mm (in Gd[len]), rgf.py:51-62 in
// the product order of rgf_sweep.cuh.
template <class T, int BM, int BN, class Team>
__device__ bool half_backward(Team& team, const HalfSweep<T>& h, int b, bool sym, T* smem) {
  T* prevT = nullptr;
  int prevI = -1;
  for (int i = h.len - 1; i >= 0; i--) {
    T* Tcur = (i & 1) ? h.T1 : h.T0;
    {  // T = -G_{i+1} P_{i+1} (= G_{i+1,i}); flush the previous T
      GemmOp<T> op = make_op<T>(b, b, b, -1.0, h.Gd(i + 1), b, h.Gu(i), b, nullptr, 0, Tcur, b);
      team_gemm<T, BM, BN>(team, &op, 1, smem);
      if (prevT) {
        team_copy<T>(team, b, b, prevT, b, h.Gl(prevI), b);
        if (sym) team_copy<T>(team, b, b, prevT, b, h.Gu(prevI), b, true);
      }
    }
    if (!team.sync()) return false;
    {  // G_{i,i+1} = -X_i G_{i+1};  G_ii = g_i - X_i T
      GemmOp<T> ops[2];
      int q = 0;
      if (!sym) ops[q++] = make_op<T>(b, b, b, -1.0, h.Gl(i), b, h.Gd(i + 1), b, nullptr, 0, h.Gu(i), b);
      ops[q++] = make_op<T>(b, b, b, -1.0, h.Gl(i), b, Tcur, b, h.Gd(i), b, h.Gd(i), b);
      team_gemm<T, BM, BN>(team, ops, q, smem);
    }
    if (!team.sync()) return false;
    prevT = Tcur;
    prevI = i;
  }
  if (prevT) {
    team_copy<T>(team, b, b, prevT, b, h.Gl(prevI), b);
    if (sym) team_copy<T>(team, b, b, prevT, b, h.Gu(prevI), b, true);
    if (!team.sync()) return false;
  }
  return true;
}

// CTAs [0, G/2) are the left team, [G/2, G) the right team; the whole grid
// meets for the middle block.  Every CTA passes every grid barrier, also
// after its team gave up on a wait, so the others' waits end.
template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) rgf2s_kernel(Rgf2sParams<T> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* smem = reinterpret_cast<T*>(smem_raw);
  const int G = gridDim.x, half = G / 2, me = blockIdx.x;
  const int side = me < half ? 0 : 1;
  TeamDyn all{&p.hdr->barrier_count, p.status, me, G, 0u};
  TeamDyn team{&p.hdr->barrier_half[side], p.status, side ? me - half : me, side ? G - half : half, 0u};
  const HalfSweep<T>& h = p.half[side];
  const bool sym = p.flags & SINVB_SYM;
  const int b = p.b;

  half_forward<T, BM, BN>(team, h, b, p.status, smem);
  if (!all.sync()) return;
  {  // S = A_mm - L X^L - R X^R over the whole grid
    const HalfSweep<T>& l = p.half[0];
    const HalfSweep<T>& r = p.half[1];
    GemmOp<T> op;
    if (l.len > 0 && r.len > 0) {
      op = make_op<T>(b, b, b, -1.0, l.lower(l.len - 1), b, l.Gl(l.len - 1), b, p.mid_diag, b, p.mid_G, b);
      op = with_second<T>(op, r.lower(r.len - 1), b, kOpN, r.Gl(r.len - 1), b, kOpN, 1);
    } else if (l.len > 0) {
      op = make_op<T>(b, b, b, -1.0, l.lower(l.len - 1), b, l.Gl(l.len - 1), b, p.mid_diag, b, p.mid_G, b);
    } else if (r.len > 0) {
      op = make_op<T>(b, b, b, -1.0, r.lower(r.len - 1), b, r.Gl(r.len - 1), b, p.mid_diag, b, p.mid_G, b);
    }
    if (l.len > 0 || r.len > 0)
      team_gemm<T, BM, BN>(all, &op, 1, smem);
    else
      team_copy<T>(all, b, b, p.mid_diag, b, p.mid_G, b);
  }
  if (!all.sync()) return;
  if (!team_invert<T, BM, BN>(all, p.mid_G, b, b, p.half[0].side, p.status, smem)) return;
  half_backward<T, BM, BN>(team, h, b, sym, smem);
}

struct Rgf2sLayout {
  size_t T[4], side[2], total;
};

static Rgf2sLayout rgf2s_layout(int b, size_t es) {
  Rgf2sLayout L{};
  size_t off = sizeof(WsHeader);
  auto take = [&](size_t bytes) {
    size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  for (int k = 0; k < 4; k++) L.T[k] = take((size_t)b * b * es);
  for (int k = 0; k < 2; k++) L.side[k] = take(invert_side_elems(b) * es);
  L.total = off;
  return L;
}

template <class T>
static int rgf2s_run(const void* diag_, const void* upper_, const void* lower_, int n, int b, unsigned flags,
                     void* Gd_, void* Gu_, void* Gl_, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  if (n < 1 || b < 1 || !diag_ || !Gd_ || !workspace) return SINVB_EINVAL;
  if (flags & ~(SINVB_SYM | SINVB_SAVE_OFFDIAG)) return SINVB_EINVAL;
  if (!(flags & SINVB_SAVE_OFFDIAG)) return SINVB_EINVAL;  // the halves keep X / P in G_upper / G_lower
  if (n > 1 && (!upper_ || !lower_ || !Gu_ || !Gl_)) return SINVB_EINVAL;
  for (const void* q : {diag_, upper_, lower_, (const void*)Gd_, (const void*)Gu_, (const void*)Gl_})
    if (q && (uintptr_t)q % sizeof(T)) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  const Rgf2sLayout L = rgf2s_layout(b, sizeof(T));
  if (workspace_bytes < L.total) return SINVB_EWORKSPACE;
  int rc = check_device();
  if (rc) return rc;
  const T* diag = (const T*)diag_;
  const T* upper = (const T*)upper_;
  const T* lower = (const T*)lower_;
  T* Gd = (T*)Gd_;
  T* Gu = (T*)Gu_;
  T* Gl = (T*)Gl_;
  unsigned char* ws = (unsigned char*)workspace;
  const long long bb = (long long)b * b;
  const int m = (n - 1) / 2;
  Rgf2sParams<T> p;
  // left half: blocks 0 .. m-1 in order
  HalfSweep<T>& l = p.half[0];
  l.diag = {diag, bb};
  l.upper = {upper, bb};
  l.lower = {lower, bb};
  l.Gd = {Gd, bb};
  l.Gu = {Gu, bb};
  l.Gl = {Gl, bb};
  l.len = m;
  // right half: blocks n-1 .. m+1, read backwards (upper and lower swap roles)
  HalfSweep<T>& r = p.half[1];
  r.len = n - 1 - m;
  const long long last = n >= 2 ? (long long)(n - 2) * bb : 0;
  r.diag = {diag + (long long)(n - 1) * bb, -bb};
  r.upper = {lower + last, -bb};
  r.lower = {upper + last, -bb};
  r.Gd = {Gd + (long long)(n - 1) * bb, -bb};
  r.Gu = {Gl + last, -bb};
  r.Gl = {Gu + last, -bb};
  for (int k = 0; k < 2; k++) {
    p.half[k].T0 = reinterpret_cast<T*>(ws + L.T[2 * k]);
    p.half[k].T1 = reinterpret_cast<T*>(ws + L.T[2 * k + 1]);
    p.half[k].side = reinterpret_cast<T*>(ws + L.side[k]);
  }
  p.mid_diag = diag + (long long)m * bb;
  p.mid_G = Gd + (long long)m * bb;
  p.hdr = reinterpret_cast<WsHeader*>(ws);
  p.status = &p.hdr->status;
  p.b = b;
  p.flags = flags;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), stream));
  void* args[] = {(void*)&p};
  auto launch = [&](auto kern, size_t smem) -> int {
    SINVB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SINVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    if (per_sm < 1) return SINVB_EUNSUPPORTED;
    const int grid = device_sm_count() * (per_sm > 2 ? 2 : per_sm);
    SINVB_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(kThreads), args, smem, stream));
    return SINVB_OK;
  };
  auto smem_for = [](size_t gemm_elems) {
    const size_t g = gemm_elems * sizeof(T);
    return g > sizeof(GjShared<T>) ? g : sizeof(GjShared<T>);
  };
  if (b <= 32) return launch(rgf2s_kernel<T, 32, 32>, smem_for(gemm_smem_elems<T, 32, 32>()));
  return launch(rgf2s_kernel<T, 64, 64>, smem_for(gemm_smem_elems<T, 64, 64>()));
}

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_rgf2s_workspace_size(int n, int b, int dtype, unsigned flags) {
  (void)n;
  (void)flags;
  if (b < 1 || (dtype != SINVB_C128 && dtype != SINVB_F64)) return 0;
  return rgf2s_layout(b, dtype == SINVB_C128 ? 16 : 8).total;
}

int sinvb_rgf2s_z(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                  void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                  sinvb_stream_t stream) {
  return rgf2s_run<cplx>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                         (cudaStream_t)stream);
}

int sinvb_rgf2s_d(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                  void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                  sinvb_stream_t stream) {
  return rgf2s_run<double>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                           (cudaStream_t)stream);
}

}  // extern "C"
