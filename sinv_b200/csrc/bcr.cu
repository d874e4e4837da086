// Block cyclic reduction (BCR) selected inversion on the whole GPU.
//
// Reference: src/sinv/algorithms/bcr/bcr_serial.py:19-467 with the padding and
// production index sets of src/sinv/algorithms/bcr/bcr_utils.py:17-129.
//
// The reference pads the block count to 2^p - 1 with identity blocks
// (bcr_utils.py:44-71) and works on dense N x N arrays.  Padding rows are
// decoupled from the real rows (zero couplings), so every product they enter is
// an exact zero and every real block comes out the same without them: this
// implementation skips them and keeps only block arrays.  It also keeps
// inv(A_kk) from the reduction instead of recomputing it in the production
// (bcr_serial.py:302, :379); both computations are the same inversion of the
// same block.
//
// Level l (offset o = 2^l) of the reduction eliminates the rows e = o-1 (mod 2o)
// into the kept rows j = 2o-1 (mod 2o); the rows of a level are independent
// (bcr_serial.py:207-212), and so are the produced rows of a production level
// (bcr_serial.py:437-466).  The host turns the whole algorithm into phases of
// independent block operations (executor.cuh) that one cooperative kernel
// runs on every SM:
//
//   reduce l:   Dinv[e] = D[e]^{-1}, one Newton step X0 + X0 (I - D X0) (:121, :148)
//               U_{e,e+o} = Dinv[e] A_{e,e+o},  L_{e+o,e} = A_{e+o,e} Dinv[e]
//               U_{e,e-o} = Dinv[e] A_{e,e-o},  L_{e-o,e} = A_{e-o,e} Dinv[e]  (:124-128, :150-154)
//               D[j] -= L_{j,i} A_{i,j} + L_{j,k} A_{k,j}             (:130-133, :156-159)
//               A_{j,j-2o} = -L_{j,i} A_{i,j-2o},  A_{j,j+2o} = -L_{j,k} A_{k,j+2o}   (:138-142, :164-168)
//   root:       G_rr = D[r]^{-1}, one Newton step                     (:220-249)
//   produce l:  corner / center production                            (:253-383)
//
// Level couplings A_{r,r+o} / A_{r+o,r} (l >= 1) and produced couplings
// G_{r,r+o} / G_{r+o,r} (l >= 1) live in per-level workspace arrays indexed by
// q = (r+1)/o - 1; level 0 couplings are the input and output block arrays.
#include <vector>

#include "host_util.h"
#include "schedule.cuh"

namespace sinvb {

namespace {

struct BcrPlan {
  // data offsets in elements from the data base
  size_t D, Dinv, Ua, Ub, La, Lb, W;
  size_t X0, Ev, eye;  // Newton step: raw inverses, residuals I - D X0, one identity block
  std::vector<size_t> Up, Lo, CU, CL;  // per level (index 0 unused)
  size_t data_elems;
  int height, root;
};

inline int ceil_log2(long long x) {
  int p = 0;
  while ((1LL << p) < x) p++;
  return p;
}

BcrPlan bcr_plan(int n, int b) {
  BcrPlan P{};
  const size_t bb = (size_t)b * b;
  const int p = ceil_log2((long long)n + 1);  // padded count 2^p - 1 (bcr_utils.py:17-40)
  P.height = p - 1;
  P.root = (1 << (p - 1)) - 1;
  size_t off = 0;
  auto take = [&](size_t blocks) {
    size_t at = off;
    off += blocks * bb;
    return at;
  };
  P.D = take(n);
  P.Dinv = take(n);
  P.Ua = take(n);
  P.Ub = take(n);
  P.La = take(n);
  P.Lb = take(n);
  P.X0 = take((size_t)(n / 2 + 2));
  P.Ev = take((size_t)(n / 2 + 2));
  P.eye = take(1);
  P.Up.assign(P.height + 2, 0);
  P.Lo.assign(P.height + 2, 0);
  P.CU.assign(P.height + 2, 0);
  P.CL.assign(P.height + 2, 0);
  for (int l = 1; l <= P.height; l++) {
    size_t cnt = (size_t)(n >> l);
    P.Up[l] = take(cnt);
    P.Lo[l] = take(cnt);
    P.CU[l] = take(cnt);
    P.CL[l] = take(cnt);
  }
  P.W = off;
  off += (size_t)(n / 2 + 2) * invert_side_elems(b);
  P.data_elems = off;
  return P;
}

template <class T>
T bcr_one();
template <>
cplx bcr_one<cplx>() { return cplx{1.0, 0.0}; }
template <>
double bcr_one<double>() { return 1.0; }

// The identity block of the Newton steps (a copy from pageable memory has
// read the host array when cudaMemcpyAsync returns).
template <class T>
int upload_identity(unsigned char* dst, int b, cudaStream_t stream) {
  std::vector<T> eye((size_t)b * b, T{});
  for (int i = 0; i < b; i++) eye[(size_t)i * b + i] = bcr_one<T>();
  SINVB_CUDA(cudaMemcpyAsync(dst, eye.data(), eye.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
  return SINVB_OK;
}

template <class T>
void build_bcr(Sched& s, const BcrPlan& P, int n, int b, const T* diag, const T* upper, const T* lower, T* Gd, T* Gu,
               T* Gl, T* base) {
  const size_t bb = (size_t)b * b;
  auto blk = [&](size_t region, int r) { return base + region + (size_t)r * bb; };
  T* D = base + P.D;
  auto Dk = [&](int r) { return D + (size_t)r * bb; };
  auto Dinv = [&](int r) { return blk(P.Dinv, r); };
  auto Ua = [&](int r) { return blk(P.Ua, r); };
  auto Ub = [&](int r) { return blk(P.Ub, r); };
  auto La = [&](int r) { return blk(P.La, r); };
  auto Lb = [&](int r) { return blk(P.Lb, r); };
  auto q = [](int r, int l) { return (r + 1) / (1 << l) - 1; };
  // level-l couplings of the reduced matrix: A_{r,r+o}, A_{r+o,r}
  auto Up = [&](int l, int r) -> T* { return l == 0 ? const_cast<T*>(upper) + (size_t)r * bb : blk(P.Up[l], q(r, l)); };
  auto Lo = [&](int l, int r) -> T* { return l == 0 ? const_cast<T*>(lower) + (size_t)r * bb : blk(P.Lo[l], q(r, l)); };
  // produced couplings G_{r,r+o}, G_{r+o,r}
  auto CU = [&](int l, int r) -> T* { return l == 0 ? Gu + (size_t)r * bb : blk(P.CU[l], q(r, l)); };
  auto CL = [&](int l, int r) -> T* { return l == 0 ? Gl + (size_t)r * bb : blk(P.CL[l], q(r, l)); };
  std::vector<T*> Wv;
  for (int x = 0; x < n / 2 + 2; x++) Wv.push_back(base + P.W + (size_t)x * invert_side_elems(b));
  auto X0v = [&](size_t x) { return blk(P.X0, (int)x); };
  auto Evv = [&](size_t x) { return blk(P.Ev, (int)x); };
  T* I = base + P.eye;
  // One Newton step on the inverses X0v(x) of raw[x] (pivot-free Gauss-Jordan
  // loses digits on the undamped blocks BCR inverts, which the reference's
  // LAPACK inverse keeps): E = I - D X0, then dst[x] = X0 + X0 E.
  auto newton = [&](const std::vector<T*>& raw, const std::vector<T*>& dst) {
    s.begin();
    for (size_t x = 0; x < raw.size(); x++) s.gemm(b, -1.0, raw[x], X0v(x), I, Evv(x));
    s.begin();
    for (size_t x = 0; x < raw.size(); x++) s.gemm(b, 1.0, X0v(x), Evv(x), X0v(x), dst[x]);
  };

  s.begin();
  s.copy(n * b, b, diag, b, D, b);  // working diagonal (the reference reduces a copy, bcr_utils.py:66-69)
  for (int l = 0; l < P.height; l++) {
    const int o = 1 << l;
    std::vector<int> E;
    for (int e = o - 1; e < n; e += 2 * o) E.push_back(e);
    // Dinv[e] = D[e]^{-1}, refined by one Newton step
    s.begin();
    std::vector<T*> inv, raw, dst;
    for (size_t x = 0; x < E.size(); x++) {
      s.copy(b, b, Dk(E[x]), b, X0v(x), b);
      inv.push_back(X0v(x));
      raw.push_back(Dk(E[x]));
      dst.push_back(Dinv(E[x]));
    }
    invert_many<T>(s, inv, Wv, b);
    newton(raw, dst);
    // U / L factors of every eliminated row
    s.begin();
    for (int e : E) {
      const int a = e - o, c = e + o;
      if (c <= n - 1) {
        s.gemm(b, 1.0, Dinv(e), Up(l, e), nullptr, Ub(e));
        s.gemm(b, 1.0, Lo(l, e), Dinv(e), nullptr, Lb(e));
      }
      if (a >= 0) {
        s.gemm(b, 1.0, Dinv(e), Lo(l, a), nullptr, Ua(e));
        s.gemm(b, 1.0, Up(l, a), Dinv(e), nullptr, La(e));
      }
    }
    // Schur update of the kept rows and the next level's couplings
    s.begin();
    for (int j = 2 * o - 1; j < n; j += 2 * o) {
      const int i = j - o, k = j + o;
      if (k <= n - 1)
        s.gemm(b, -1.0, Lb(i), Up(l, i), Dk(j), Dk(j), La(k), Lo(l, j));
      else
        s.gemm(b, -1.0, Lb(i), Up(l, i), Dk(j), Dk(j));
      const int h = j - 2 * o, r = k + o;
      if (h >= 0) s.gemm(b, -1.0, Lb(i), Lo(l, h), nullptr, Lo(l + 1, h));
      if (r <= n - 1) s.gemm(b, -1.0, La(k), Up(l, k), nullptr, Up(l + 1, j));
    }
  }
  // root, refined by one Newton step
  s.begin();
  s.copy(b, b, Dk(P.root), b, X0v(0), b);
  invert_many<T>(s, std::vector<T*>{X0v(0)}, Wv, b);
  newton(std::vector<T*>{Dk(P.root)}, std::vector<T*>{Gd + (size_t)P.root * bb});
  // production, top level down
  for (int l = P.height - 1; l >= 0; l--) {
    const int o = 1 << l;
    std::vector<int> E;
    for (int e = o - 1; e < n; e += 2 * o) E.push_back(e);
    s.begin();
    for (int e : E) {
      const int a = e - o, c = e + o;
      const bool ha = a >= 0, hc = c <= n - 1;
      T* Gaa = ha ? Gd + (size_t)a * bb : nullptr;
      T* Gcc = hc ? Gd + (size_t)c * bb : nullptr;
      if (ha && hc) {  // center_produce, bcr_serial.py:361-383
        T* Gac = CU(l + 1, a);
        T* Gca = CL(l + 1, a);
        s.gemm(b, -1.0, Gaa, La(e), nullptr, CU(l, a), Gac, Lb(e));
        s.gemm(b, -1.0, Gca, La(e), nullptr, CL(l, e), Gcc, Lb(e));
        s.gemm(b, -1.0, Ua(e), Gaa, nullptr, CL(l, a), Ub(e), Gca);
        s.gemm(b, -1.0, Ua(e), Gac, nullptr, CU(l, e), Ub(e), Gcc);
      } else if (hc) {  // corner_produce from below, bcr_serial.py:291-298
        s.gemm(b, -1.0, Gcc, Lb(e), nullptr, CL(l, e));
        s.gemm(b, -1.0, Ub(e), Gcc, nullptr, CU(l, e));
      } else if (ha) {  // corner_produce from above
        s.gemm(b, -1.0, Gaa, La(e), nullptr, CU(l, a));
        s.gemm(b, -1.0, Ua(e), Gaa, nullptr, CL(l, a));
      }
    }
    s.begin();
    for (int e : E) {
      const int a = e - o, c = e + o;
      const bool ha = a >= 0, hc = c <= n - 1;
      T* Gee = Gd + (size_t)e * bb;
      if (ha && hc)
        s.gemm(b, -1.0, CL(l, a), La(e), Dinv(e), Gee, CU(l, e), Lb(e));
      else if (hc)
        s.gemm(b, -1.0, CU(l, e), Lb(e), Dinv(e), Gee);
      else if (ha)
        s.gemm(b, -1.0, CL(l, a), La(e), Dinv(e), Gee);
    }
  }
  // drop empty phases
  std::vector<ExecPhase> kept;
  for (auto& p : s.phases)
    if (p.units > 0) kept.push_back(p);
  s.phases.swap(kept);
}

struct BcrLayout {
  size_t ops_off, phases_off, data_off, total;
  int nops, nphases;
};

int tile_for(int b) { return b >= 128 ? 64 : 32; }

template <class T>
BcrLayout bcr_layout_and_schedule(int n, int b, const T* diag, const T* upper, const T* lower, T* Gd, T* Gu, T* Gl,
                                  unsigned char* ws, Sched* out) {
  const BcrPlan P = bcr_plan(n, b);
  BcrLayout L{};
  Sched s;
  s.bm = s.bn = tile_for(b);
  // the op table size does not depend on the pointers: build once to size it
  L.ops_off = sizeof(WsHeader);
  build_bcr<T>(s, P, n, b, diag, upper, lower, Gd, Gu, Gl, (T*)nullptr);
  L.nops = (int)s.ops.size();
  L.nphases = (int)s.phases.size();
  L.phases_off = align_up(L.ops_off + (size_t)L.nops * sizeof(ExecOp), 256);
  L.data_off = align_up(L.phases_off + (size_t)L.nphases * sizeof(ExecPhase), 256);
  L.total = align_up(L.data_off + P.data_elems * sizeof(T), 256);
  if (out && ws) {
    out->bm = out->bn = s.bm;
    build_bcr<T>(*out, P, n, b, diag, upper, lower, Gd, Gu, Gl, (T*)(ws + L.data_off));
  }
  return L;
}

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) bcr_kernel(unsigned char* ws, int nphases) {
  run_uploaded_schedule<T, BM, BN>(ws, nphases);
}

template <class T, int BM, int BN>
int launch_bcr(unsigned char* ws, int nphases, cudaStream_t stream) {
  return launch_schedule_kernel<T, BM, BN>(bcr_kernel<T, BM, BN>, ws, nphases, stream);
}

template <class T>
int run_bcr(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags, void* Gd,
            void* Gu, void* Gl, void* workspace, size_t ws_bytes, cudaStream_t stream, int dtype) {
  (void)flags;
  if (n < 1 || b < 1 || !diag || !Gd || !workspace) return SINVB_EINVAL;
  if (n > 1 && (!upper || !lower || !Gu || !Gl)) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  const size_t align = sizeof(T);
  for (const void* p : {diag, upper, lower, (const void*)Gd, (const void*)Gu, (const void*)Gl})
    if (p && (uintptr_t)p % align) return SINVB_EINVAL;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  Sched s;
  BcrLayout L = bcr_layout_and_schedule<T>(n, b, (const T*)diag, (const T*)upper, (const T*)lower, (T*)Gd, (T*)Gu,
                                           (T*)Gl, ws, &s);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  (void)dtype;
  WsHeader h{};
  h.desc_offset = L.ops_off;
  h.items_offset = L.phases_off;
  SINVB_CUDA(cudaMemcpyAsync(ws, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.ops_off, s.ops.data(), s.ops.size() * sizeof(ExecOp), cudaMemcpyHostToDevice,
                             stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.phases_off, s.phases.data(), s.phases.size() * sizeof(ExecPhase),
                             cudaMemcpyHostToDevice, stream));
  rc = upload_identity<T>(ws + L.data_off + bcr_plan(n, b).eye * sizeof(T), b, stream);
  if (rc) return rc;
  if (tile_for(b) == 64) return launch_bcr<T, 64, 64>(ws, (int)s.phases.size(), stream);
  return launch_bcr<T, 32, 32>(ws, (int)s.phases.size(), stream);
}

// ---------------------------------------------------------------------------
// A batch of independent matrices in one launch.  Every matrix keeps its own
// BCR schedule and data region; phase k of the batch is phase k of every
// matrix that has one, so the rows of a level of all matrices share each grid
// barrier and small matrices fill the GPU together.  Matrices are independent,
// so only each matrix's own phase order matters.  Layout: header, one status
// word per matrix (at a fixed offset, so a re-run can clear them without the
// schedule), merged op table, merged phases, then the data regions.
struct BcrBatchLayout {
  size_t ops_off, phases_off, status_off, total;
  std::vector<size_t> data_off;
  int nops, nphases, tile;
};

int batch_tile(const sinvb_batch_desc* d, int count) {
  int bmax = 1;
  for (int k = 0; k < count; k++) bmax = std::max(bmax, d[k].b);
  return tile_for(bmax);
}

// Appends phase k of every part to `out`, tagging each op with its matrix.
void merge_phases(const std::vector<Sched>& parts, Sched& out) {
  size_t np = 0;
  for (const Sched& p : parts) np = std::max(np, p.phases.size());
  for (size_t k = 0; k < np; k++) {
    out.begin();
    for (size_t i = 0; i < parts.size(); i++) {
      if (k >= parts[i].phases.size()) continue;
      const ExecPhase& ph = parts[i].phases[k];
      for (int o = ph.op_begin; o < ph.op_end; o++) {
        ExecOp op = parts[i].ops[o];
        op.inst = (int)i;
        out.push(op);
      }
    }
  }
}

template <class T>
BcrBatchLayout bcr_batch_layout(const sinvb_batch_desc* d, int count, unsigned char* ws, Sched* out) {
  BcrBatchLayout L{};
  L.tile = batch_tile(d, count);
  std::vector<Sched> parts((size_t)count);
  std::vector<BcrPlan> plans;
  plans.reserve((size_t)count);
  for (int k = 0; k < count; k++) {
    plans.push_back(bcr_plan(d[k].n, d[k].b));
    parts[k].bm = parts[k].bn = L.tile;
    build_bcr<T>(parts[k], plans[k], d[k].n, d[k].b, (const T*)d[k].diag, (const T*)d[k].upper,
                 (const T*)d[k].lower, (T*)d[k].G_diag, (T*)d[k].G_upper, (T*)d[k].G_lower, (T*)nullptr);
  }
  Sched merged;
  merged.bm = merged.bn = L.tile;
  merge_phases(parts, merged);
  L.nops = (int)merged.ops.size();
  L.nphases = (int)merged.phases.size();
  L.status_off = sizeof(WsHeader);
  L.ops_off = align_up(L.status_off + (size_t)count * sizeof(int), 256);
  L.phases_off = align_up(L.ops_off + (size_t)L.nops * sizeof(ExecOp), 256);
  size_t off = align_up(L.phases_off + (size_t)L.nphases * sizeof(ExecPhase), 256);
  L.data_off.resize((size_t)count);
  for (int k = 0; k < count; k++) {
    L.data_off[k] = off;
    off = align_up(off + plans[k].data_elems * sizeof(T), 256);
  }
  L.total = off;
  if (out && ws) {
    for (int k = 0; k < count; k++) {
      parts[k] = Sched{};
      parts[k].bm = parts[k].bn = L.tile;
      build_bcr<T>(parts[k], plans[k], d[k].n, d[k].b, (const T*)d[k].diag, (const T*)d[k].upper,
                   (const T*)d[k].lower, (T*)d[k].G_diag, (T*)d[k].G_upper, (T*)d[k].G_lower,
                   (T*)(ws + L.data_off[k]));
    }
    out->bm = out->bn = L.tile;
    merge_phases(parts, *out);
  }
  return L;
}

template <class T>
int run_bcr_batched(const sinvb_batch_desc* d, int count, void* workspace, size_t ws_bytes, int* status,
                    cudaStream_t stream) {
  if (count < 0 || (count > 0 && !d) || !workspace) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  for (int k = 0; k < count; k++) {
    const sinvb_batch_desc& e = d[k];
    if (e.n < 1 || e.b < 1 || !e.diag || !e.G_diag) return SINVB_EINVAL;
    if (e.n > 1 && (!e.upper || !e.lower || !e.G_upper || !e.G_lower)) return SINVB_EINVAL;
    for (const void* p : {e.diag, e.upper, e.lower, (const void*)e.G_diag, (const void*)e.G_upper,
                          (const void*)e.G_lower})
      if (p && (uintptr_t)p % sizeof(T)) return SINVB_EINVAL;
  }
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  if (count == 0) {
    if (ws_bytes < sizeof(WsHeader)) return SINVB_EWORKSPACE;
    SINVB_CUDA(cudaMemsetAsync(ws, 0, sizeof(WsHeader), stream));
    return SINVB_OK;
  }
  Sched s;
  BcrBatchLayout L = bcr_batch_layout<T>(d, count, ws, &s);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  WsHeader h{};
  h.count = count;
  h.desc_offset = L.ops_off;
  h.items_offset = L.phases_off;
  h.slots_offset = L.status_off;
  h.inst_status = status;
  h.sched_phases = L.nphases;
  SINVB_CUDA(cudaMemcpyAsync(ws, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.ops_off, s.ops.data(), s.ops.size() * sizeof(ExecOp), cudaMemcpyHostToDevice,
                             stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.phases_off, s.phases.data(), s.phases.size() * sizeof(ExecPhase),
                             cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemsetAsync(ws + L.status_off, 0, (size_t)count * sizeof(int), stream));
  for (int k = 0; k < count; k++) {
    rc = upload_identity<T>(ws + L.data_off[k] + bcr_plan(d[k].n, d[k].b).eye * sizeof(T), d[k].b, stream);
    if (rc) return rc;
  }
  if (L.tile == 64) return launch_bcr<T, 64, 64>(ws, (int)s.phases.size(), stream);
  return launch_bcr<T, 32, 32>(ws, (int)s.phases.size(), stream);
}

// Re-runs the batch uploaded into ws by run_bcr_batched (same descriptors):
// clears the barrier and status words and launches; the tile comes from the
// block sizes, the phase count from the header.
template <class T>
int rerun_bcr_batched(const sinvb_batch_desc* d, int count, void* workspace, cudaStream_t stream) {
  if (count < 0 || (count > 0 && !d) || !workspace) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  for (int k = 0; k < count; k++)
    if (d[k].n < 1 || d[k].b < 1) return SINVB_EINVAL;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  SINVB_CUDA(cudaMemsetAsync(ws, 0, 16, stream));  // status, barrier counter
  if (count == 0) return SINVB_OK;
  SINVB_CUDA(cudaMemsetAsync(ws + sizeof(WsHeader), 0, (size_t)count * sizeof(int), stream));
  if (batch_tile(d, count) == 64) return launch_bcr<T, 64, 64>(ws, -1, stream);
  return launch_bcr<T, 32, 32>(ws, -1, stream);
}

}  // namespace

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_bcr_workspace_size(int n, int b, int dtype, unsigned flags) {
  (void)flags;
  if (n < 1 || b < 1) return 0;
  if (dtype == SINVB_C128)
    return bcr_layout_and_schedule<cplx>(n, b, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr)
        .total;
  if (dtype == SINVB_F64)
    return bcr_layout_and_schedule<double>(n, b, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                           nullptr)
        .total;
  return 0;
}

int sinvb_bcr_z(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags, void* G_diag,
                void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes, sinvb_stream_t stream) {
  return run_bcr<cplx>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                       (cudaStream_t)stream, SINVB_C128);
}

int sinvb_bcr_d(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags, void* G_diag,
                void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes, sinvb_stream_t stream) {
  return run_bcr<double>(diag, upper, lower, n, b, flags, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                         (cudaStream_t)stream, SINVB_F64);
}

size_t sinvb_bcr_batched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype, unsigned flags) {
  (void)flags;
  if (count < 0 || (count > 0 && !descs)) return 0;
  if (count == 0) return sizeof(WsHeader);
  for (int k = 0; k < count; k++)
    if (descs[k].n < 1 || descs[k].b < 1) return 0;
  if (dtype == SINVB_C128) return bcr_batch_layout<cplx>(descs, count, nullptr, nullptr).total;
  if (dtype == SINVB_F64) return bcr_batch_layout<double>(descs, count, nullptr, nullptr).total;
  return 0;
}

int sinvb_bcr_batched_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  (void)flags;
  return run_bcr_batched<cplx>(descs, count, workspace, workspace_bytes, status, (cudaStream_t)stream);
}

int sinvb_bcr_batched_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream) {
  (void)flags;
  return run_bcr_batched<double>(descs, count, workspace, workspace_bytes, status, (cudaStream_t)stream);
}

int sinvb_bcr_batched_rerun_z(const sinvb_batch_desc* descs, int count, void* workspace, sinvb_stream_t stream) {
  return rerun_bcr_batched<cplx>(descs, count, workspace, (cudaStream_t)stream);
}

int sinvb_bcr_batched_rerun_d(const sinvb_batch_desc* descs, int count, void* workspace, sinvb_stream_t stream) {
  return rerun_bcr_batched<double>(descs, count, workspace, (cudaStream_t)stream);
}

}  // extern "C"
