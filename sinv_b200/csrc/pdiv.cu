// PDIV (pairwise) selected inversion on one GPU.
//
// Reference: src/sinv/algorithms/pdiv/pdiv_localmap.py:27-1436 with the
// partitioning of src/sinv/algorithms/pdiv/pdiv_utils.py:84-171.  The
// reference gives each of P MPI processes (a power of two) one partition of
// the block rows (n // P blocks each, the remainder in the first).  Each
// process inverts its partition densely (:94-116); log2(P) reduction steps
// then merge neighbouring groups of processes through the bridge blocks
// between them, every process keeping twelve b x b "matrix maps" M (how its
// final blocks follow from its local inverse K) and eight "cross maps" C
// (for the bridge blocks of the inverse) (:188-252, :573-900); finally each
// process produces its tridiagonal blocks and the bridges to the next
// partition from K and its maps (:903-1436).
//
// Here the whole algorithm is one executor schedule (schedule.cuh) on every
// SM, the P partitions side by side in each phase:
//
// * K is never formed.  The maps and the production read only K's tridiagonal
//   blocks and its first and last block rows and columns, which one RGF sweep
//   pair over the partition gives.  Forward: g_0 = A_00^{-1},
//   X_i = g_i A_{i,i+1}, P_{i+1} = A_{i+1,i} g_i,
//   g_{i+1} = (A_{i+1,i+1} - P_{i+1} A_{i,i+1})^{-1}, and the running products
//   W_i = (-P_i) ... (-P_1), V_i = (-X_0) ... (-X_{i-1}).  Backward (l the last
//   row): K_ll = g_l, K_{i+1,i} = -K_{i+1,i+1} P_{i+1},
//   K_{i,i+1} = -X_i K_{i+1,i+1}, K_ii = g_i - X_i K_{i+1,i}, the last column
//   K_{i,l} = -X_i K_{i+1,l} and row K_{l,i} = -K_{l,i+1} P_{i+1}; then the
//   first column K_{i,0} = K_ii W_i and row K_{0,j} = V_j K_jj.
// * Every statement of a step's map updates reads maps from before the step
//   (the neighbour's maps are sent before the updates, and within a process
//   no statement reads a map an earlier statement of the step wrote), so the
//   maps are double-buffered by step.  Each update is a chain of four b x b
//   products; the factors a group shares (Bu J12, Bl J21, U0 Bu J12, ...) are
//   formed once per group, so every update is two dependent products.
// * J = [[I, -U3 Bl], [-U2 Bu, I]]^{-1} (get_J, :373-410) is a 2b x 2b
//   pivot-free blocked Gauss-Jordan inversion inside the schedule.
//
// Results agree with the reference's to rounding (the reference inverts each
// partition with LAPACK, partial pivoting, and multiplies in its own order).
#include <cstdint>
#include <vector>

#include "host_util.h"
#include "schedule.cuh"

namespace sinvb {

namespace {

struct PdivPart {
  int s, m;  // first block row, block rows
  size_t Kd, Ku, Kl, Cf, Cl, Rf, Rl, X, Pm, W, V, M[2], C, T, Y, Z, S, Xt, E, side;
};

struct PdivGroup {
  size_t U, UY, J, Jv, Jt, Je, I2, Q, EH, side;
};

struct PdivPlan {
  int n, b, P;
  std::vector<PdivPart> parts;
  std::vector<PdivGroup> groups;  // indexed by the group's middle process
  size_t eye, zero, data_elems;
};

constexpr int kPdivMaxPartitions = 64;

bool power_of_two(int x) { return x > 0 && (x & (x - 1)) == 0; }

PdivPlan pdiv_plan(int n, int b, int P) {
  PdivPlan L{};
  L.n = n;
  L.b = b;
  L.P = P;
  const size_t bb = (size_t)b * b;
  size_t off = 0;
  auto take = [&](size_t blocks) {
    size_t at = off;
    off += blocks * bb;
    return at;
  };
  auto take_elems = [&](size_t elems) {
    size_t at = off;
    off += align_up(elems, 32);
    return at;
  };
  L.eye = take(1);
  L.zero = take(1);
  const int base = n / P;
  int s = 0;
  for (int p = 0; p < P; p++) {
    PdivPart q{};
    q.s = s;
    q.m = p == 0 ? n - base * (P - 1) : base;  // pdiv_utils.py:107-121
    s += q.m;
    const size_t m = (size_t)q.m;
    q.Kd = take(m);
    q.Ku = take(m);
    q.Kl = take(m);
    q.Cf = take(m);
    q.Cl = take(m);
    q.Rf = take(m);
    q.Rl = take(m);
    q.X = take(m);
    q.Pm = take(m);
    q.W = take(m);
    q.V = take(m);
    q.M[0] = take(12);
    q.M[1] = take(12);
    q.C = take(8);
    q.T = take(6);
    q.Y = take(m + 2);
    q.Z = take(m + 2);
    q.S = take(1);
    q.Xt = take(1);
    q.E = take(1);
    q.side = take_elems(invert_side_elems(b));
    L.parts.push_back(q);
  }
  for (int g = 0; g < P; g++) {
    PdivGroup G{};
    G.U = take(6);
    G.UY = take(4);
    G.J = take(4);
    G.Jv = take(4);
    G.Jt = take(4);
    G.Je = take(4);
    G.I2 = take(4);
    G.Q = take(4);
    G.EH = take(4);
    G.side = take_elems(invert_side_elems(2 * b));
    L.groups.push_back(G);
  }
  L.data_elems = off;
  return L;
}

template <class T>
void build_pdiv(Sched& s, const PdivPlan& L, const T* diag, const T* upper, const T* lower, T* Gd, T* Gu, T* Gl,
                T* base) {
  const int b = L.b, P = L.P;
  const size_t bb = (size_t)b * b;
  T* I = base + L.eye;
  T* O = base + L.zero;
  auto Ad = [&](int r) { return diag + (size_t)r * bb; };
  auto Au = [&](int r) { return upper + (size_t)r * bb; };
  auto Al = [&](int r) { return lower + (size_t)r * bb; };
  auto B = [&](size_t region, int k) { return base + region + (size_t)k * bb; };
  const std::vector<PdivPart>& parts = L.parts;
  auto Kd = [&](int p, int i) { return B(parts[p].Kd, i); };
  auto Ku = [&](int p, int i) { return B(parts[p].Ku, i); };
  auto Kl = [&](int p, int i) { return B(parts[p].Kl, i); };
  auto Cf = [&](int p, int i) { return B(parts[p].Cf, i); };
  auto Cl = [&](int p, int i) { return B(parts[p].Cl, i); };
  auto Rf = [&](int p, int i) { return B(parts[p].Rf, i); };
  auto Rl = [&](int p, int i) { return B(parts[p].Rl, i); };
  auto X = [&](int p, int i) { return B(parts[p].X, i); };
  auto Pm = [&](int p, int i) { return B(parts[p].Pm, i); };
  auto W = [&](int p, int i) { return B(parts[p].W, i); };
  auto V = [&](int p, int i) { return B(parts[p].V, i); };
  auto M = [&](int p, int buf, int k) { return B(parts[p].M[buf], k); };
  auto C = [&](int p, int k) { return B(parts[p].C, k); };
  auto Tm = [&](int p, int k) { return B(parts[p].T, k); };
  auto Y = [&](int p, int i) { return B(parts[p].Y, i); };
  auto Z = [&](int p, int i) { return B(parts[p].Z, i); };
  auto side = [&](int p) { return base + parts[p].side; };
  auto last = [&](int p) { return parts[p].m - 1; };
  int mmax = 0;
  for (const PdivPart& q : parts) mmax = std::max(mmax, q.m);

  // ---- every partition's K blocks: forward sweep.  Every block inverse
  // gets one Newton step, X1 = X0 + X0 (I - S X0): a partition's first block
  // is E - H_ii as given (no contact damping), whose leading sub-blocks can be
  // ill conditioned, and the pivot-free blocked Gauss-Jordan loses digits on
  // it that LAPACK's partial pivoting (the reference's inverse) keeps.
  auto Sv = [&](int p) { return B(parts[p].S, 0); };
  auto Xt = [&](int p) { return B(parts[p].Xt, 0); };
  auto Ev = [&](int p) { return B(parts[p].E, 0); };
  std::vector<T*> inv, sides;
  auto newton = [&](const std::vector<int>& ps, int row) {
    inv.clear();
    sides.clear();
    for (int p : ps) {
      inv.push_back(Xt(p));
      sides.push_back(side(p));
    }
    invert_many<T>(s, inv, sides, b);
    s.begin();
    for (int p : ps) s.gemm(b, -1.0, Sv(p), Xt(p), I, Ev(p));  // E = I - S X0
    s.begin();
    for (int p : ps) s.gemm(b, 1.0, Xt(p), Ev(p), Xt(p), Kd(p, row));  // X1 = X0 + X0 E
  };
  s.begin();
  std::vector<int> all;
  for (int p = 0; p < P; p++) {
    s.copy(b, b, Ad(parts[p].s), b, Sv(p), b);
    s.copy(b, b, Ad(parts[p].s), b, Xt(p), b);
    all.push_back(p);
  }
  newton(all, 0);
  for (int i = 0; i + 1 < mmax; i++) {
    s.begin();
    for (int p = 0; p < P; p++) {
      if (i + 1 >= parts[p].m) continue;
      const int r = parts[p].s + i;
      s.gemm(b, 1.0, Kd(p, i), Au(r), nullptr, X(p, i));   // X_i = g_i A_{i,i+1}
      s.gemm(b, 1.0, Al(r), Kd(p, i), nullptr, Pm(p, i));  // P_{i+1} = A_{i+1,i} g_i
    }
    s.begin();
    std::vector<int> live;
    for (int p = 0; p < P; p++) {
      if (i + 1 >= parts[p].m) continue;
      const int r = parts[p].s + i;
      s.gemm(b, -1.0, Pm(p, i), Au(r), Ad(r + 1), Sv(p));                      // S_{i+1}
      s.gemm(b, -1.0, Pm(p, i), Au(r), Ad(r + 1), Xt(p));                      // (inverted in place)
      s.gemm(b, -1.0, Pm(p, i), i == 0 ? I : W(p, i), nullptr, W(p, i + 1));  // W_{i+1} = -P_{i+1} W_i
      s.gemm(b, -1.0, i == 0 ? I : V(p, i), X(p, i), nullptr, V(p, i + 1));   // V_{i+1} = -V_i X_i
      live.push_back(p);
    }
    newton(live, i + 1);
  }
  // ---- backward sweep, row i = m - 2 - t of every partition
  for (int t = 0; t + 1 < mmax; t++) {
    s.begin();
    for (int p = 0; p < P; p++) {
      const int i = parts[p].m - 2 - t;
      if (i < 0) continue;
      const bool nl = i + 1 == last(p);
      s.gemm(b, -1.0, Kd(p, i + 1), Pm(p, i), nullptr, Kl(p, i));                // K_{i+1,i}
      s.gemm(b, -1.0, X(p, i), Kd(p, i + 1), nullptr, Ku(p, i));                 // K_{i,i+1}
      s.gemm(b, -1.0, X(p, i), nl ? Kd(p, i + 1) : Cl(p, i + 1), nullptr, Cl(p, i));  // K_{i,l}
      s.gemm(b, -1.0, nl ? Kd(p, i + 1) : Rl(p, i + 1), Pm(p, i), nullptr, Rl(p, i));  // K_{l,i}
    }
    s.begin();
    for (int p = 0; p < P; p++) {
      const int i = parts[p].m - 2 - t;
      if (i < 0) continue;
      s.gemm(b, -1.0, X(p, i), Kl(p, i), Kd(p, i), Kd(p, i));  // K_ii = g_i - X_i K_{i+1,i}
    }
  }
  // first row and column, the corner copies, and the initial maps
  // (initialize_matrixmaps / initialize_crossmaps, :119-185)
  s.begin();
  for (int p = 0; p < P; p++) {
    const int l = last(p);
    for (int i = 0; i <= l; i++) {
      if (i == 0) {
        s.copy(b, b, Kd(p, 0), b, Cf(p, 0), b);
        s.copy(b, b, Kd(p, 0), b, Rf(p, 0), b);
      } else {
        s.gemm(b, 1.0, Kd(p, i), W(p, i), nullptr, Cf(p, i));  // K_{i,0} = K_ii W_i
        s.gemm(b, 1.0, V(p, i), Kd(p, i), nullptr, Rf(p, i));  // K_{0,i} = V_i K_ii
      }
    }
    s.copy(b, b, Kd(p, l), b, Cl(p, l), b);
    s.copy(b, b, Kd(p, l), b, Rl(p, l), b);
    for (int k = 0; k < 12; k++) s.copy(b, b, (k == 0 || k == 3 || k == 4 || k == 7) ? I : O, b, M(p, 0, k), b);
    for (int k = 0; k < 8; k++) s.copy(b, b, O, b, C(p, k), b);
  }

  // ---- reduction steps (update_maps, :188-252)
  int steps = 0;
  while ((1 << steps) < P) steps++;
  for (int step = 1; step <= steps; step++) {
    const int stride = 1 << step, o = (step - 1) & 1, nw = step & 1;
    struct Grp {
      int start, end, mid;
      const PdivGroup* g;
    };
    std::vector<Grp> grps;
    for (int start = 0; start < P; start += stride)
      grps.push_back({start, start + stride - 1, start + stride / 2 - 1, &L.groups[start + stride / 2 - 1]});
    auto U = [&](const Grp& G, int k) { return B(G.g->U, k); };
    auto UY = [&](const Grp& G, int k) { return B(G.g->UY, k); };
    auto Q = [&](const Grp& G, int k) { return B(G.g->Q, k); };  // QU11, QU12, QL21, QL22
    auto EH = [&](const Grp& G, int k) { return B(G.g->EH, k); };  // Eu, Hu, El, Hl
    auto J = [&](const Grp& G) { return base + G.g->J; };
    // U blocks of the two middle processes (get_U, :279-370), from the maps before the step
    s.begin();
    for (const Grp& G : grps) {
      const int pm = G.mid, pn = G.mid + 1, lm = last(pm), ln = last(pn);
      s.gemm(b, 1.0, M(pm, o, 0), Rf(pm, lm), nullptr, U(G, 0), M(pm, o, 1), Kd(pm, lm));  // toprow
      s.gemm(b, 1.0, Cf(pm, lm), M(pm, o, 4), nullptr, U(G, 1), Kd(pm, lm), M(pm, o, 5));  // leftcol
      s.gemm(b, 1.0, Kd(pn, 0), M(pn, o, 2), nullptr, U(G, 4), Rf(pn, ln), M(pn, o, 3));    // rightcol
      s.gemm(b, 1.0, M(pn, o, 6), Kd(pn, 0), nullptr, U(G, 5), M(pn, o, 7), Cf(pn, ln));    // botrow
      s.gemm(b, 1.0, M(pm, o, 8), Rf(pm, lm), nullptr, UY(G, 0), M(pm, o, 9), Kd(pm, lm));
      s.gemm(b, 1.0, M(pm, o, 10), Rf(pm, lm), nullptr, UY(G, 1), M(pm, o, 11), Kd(pm, lm));
      s.gemm(b, 1.0, M(pn, o, 8), Kd(pn, 0), nullptr, UY(G, 2), M(pn, o, 9), Cf(pn, ln));
      s.gemm(b, 1.0, M(pn, o, 10), Kd(pn, 0), nullptr, UY(G, 3), M(pn, o, 11), Cf(pn, ln));
    }
    s.begin();
    for (const Grp& G : grps) {
      const int pm = G.mid, pn = G.mid + 1, lm = last(pm), ln = last(pn);
      // element(last, last) of the middle process, element(0, 0) of the next
      s.gemm(b, 1.0, Cf(pm, lm), UY(G, 0), Kd(pm, lm), U(G, 2), Kd(pm, lm), UY(G, 1));
      s.gemm(b, 1.0, Kd(pn, 0), UY(G, 2), Kd(pn, 0), U(G, 3), Rf(pn, ln), UY(G, 3));
    }
    // J = [[I, -U3 Bl], [-U2 Bu, I]]^{-1}, Bu / Bl the bridge after the middle
    // process: assembled twice (Jt is inverted in place, Jv kept), one Newton
    // step J = Jt + Jt (I - Jv Jt)
    s.begin();
    std::vector<T*> js, jside;
    const size_t lo = (size_t)b * 2 * b;
    for (const Grp& G : grps) {
      const int r = parts[G.mid + 1].s - 1;
      for (T* j : {base + G.g->Jt, base + G.g->Jv}) {
        s.copy(b, b, I, b, j, 2 * b);
        s.copy(b, b, I, b, j + lo + b, 2 * b);
        s.gemm(b, -1.0, U(G, 3), Al(r), nullptr, j + b, nullptr, nullptr, -1, b, b, b, b, b, 2 * b);
        s.gemm(b, -1.0, U(G, 2), Au(r), nullptr, j + lo, nullptr, nullptr, -1, b, b, b, b, b, 2 * b);
      }
      T* i2 = base + G.g->I2;
      s.copy(b, b, I, b, i2, 2 * b);
      s.copy(b, b, O, b, i2 + b, 2 * b);
      s.copy(b, b, O, b, i2 + lo, 2 * b);
      s.copy(b, b, I, b, i2 + lo + b, 2 * b);
      js.push_back(base + G.g->Jt);
      jside.push_back(base + G.g->side);
    }
    invert_many<T>(s, js, jside, 2 * b);
    s.begin();
    for (const Grp& G : grps)
      s.gemm(2 * b, -1.0, base + G.g->Jv, base + G.g->Jt, base + G.g->I2, base + G.g->Je);
    s.begin();
    for (const Grp& G : grps)
      s.gemm(2 * b, 1.0, base + G.g->Jt, base + G.g->Je, base + G.g->Jt, J(G));
    s.begin();
    for (const Grp& G : grps) {
      const int r = parts[G.mid + 1].s - 1;
      T* j = J(G);
      s.gemm(b, 1.0, Au(r), j, nullptr, Q(G, 0), nullptr, nullptr, -1, b, b, b, b, 2 * b, b);       // Bu J11
      s.gemm(b, 1.0, Au(r), j + b, nullptr, Q(G, 1), nullptr, nullptr, -1, b, b, b, b, 2 * b, b);   // Bu J12
      s.gemm(b, 1.0, Al(r), j + lo, nullptr, Q(G, 2), nullptr, nullptr, -1, b, b, b, b, 2 * b, b);  // Bl J21
      s.gemm(b, 1.0, Al(r), j + lo + b, nullptr, Q(G, 3), nullptr, nullptr, -1, b, b, b, b, 2 * b, b);  // Bl J22
    }
    // first product of every chain: the group's shared factors and each process's own
    s.begin();
    for (const Grp& G : grps) {
      s.gemm(b, 1.0, U(G, 0), Q(G, 1), nullptr, EH(G, 0));  // Eu = UUR Bu J12
      s.gemm(b, 1.0, U(G, 5), Q(G, 3), nullptr, EH(G, 1));  // Hu = DLL Bl J22
      s.gemm(b, 1.0, U(G, 5), Q(G, 2), nullptr, EH(G, 2));  // El = DLL Bl J21
      s.gemm(b, 1.0, U(G, 0), Q(G, 0), nullptr, EH(G, 3));  // Hl = UUR Bu J11
      for (int r = G.start; r <= G.end; r++) {
        if (r <= G.mid) {
          s.gemm(b, 1.0, M(r, o, 2), Q(G, 1), nullptr, Tm(r, 0));  // M2 Bu J12
          s.gemm(b, 1.0, M(r, o, 3), Q(G, 1), nullptr, Tm(r, 1));  // M3 Bu J12
          s.gemm(b, 1.0, M(r, o, 2), Q(G, 0), nullptr, Tm(r, 4));  // M2 Bu J11
          s.gemm(b, 1.0, M(r, o, 3), Q(G, 0), nullptr, Tm(r, 5));  // M3 Bu J11
          if (r < G.mid) {
            s.gemm(b, 1.0, M(r + 1, o, 2), Q(G, 1), nullptr, Tm(r, 2));  // Mn2 Bu J12
            s.gemm(b, 1.0, M(r + 1, o, 3), Q(G, 1), nullptr, Tm(r, 3));  // Mn3 Bu J12
          } else {
            s.gemm(b, 1.0, M(r + 1, o, 4), Q(G, 3), nullptr, Tm(r, 2));  // Mn4 Bl J22
            s.gemm(b, 1.0, M(r + 1, o, 5), Q(G, 3), nullptr, Tm(r, 3));  // Mn5 Bl J22
          }
        } else {
          s.gemm(b, 1.0, M(r, o, 4), Q(G, 2), nullptr, Tm(r, 0));  // M4 Bl J21
          s.gemm(b, 1.0, M(r, o, 5), Q(G, 2), nullptr, Tm(r, 1));  // M5 Bl J21
          s.gemm(b, 1.0, M(r, o, 4), Q(G, 3), nullptr, Tm(r, 4));  // M4 Bl J22
          s.gemm(b, 1.0, M(r, o, 5), Q(G, 3), nullptr, Tm(r, 5));  // M5 Bl J22
          if (r < G.end) {
            s.gemm(b, 1.0, M(r + 1, o, 4), Q(G, 2), nullptr, Tm(r, 2));  // Mn4 Bl J21
            s.gemm(b, 1.0, M(r + 1, o, 5), Q(G, 2), nullptr, Tm(r, 3));  // Mn5 Bl J21
          }
        }
      }
    }
    // cross maps (update_crossmap, :573-744) and the new matrix maps
    // (update_matrixmap, :747-900)
    s.begin();
    for (const Grp& G : grps) {
      T* ULL = U(G, 1);
      T* DUR = U(G, 4);
      for (int r = G.start; r <= G.end; r++) {
        auto Mo = [&](int k) { return M(r, o, k); };
        auto Mn = [&](int k) { return M(r + 1, o, k); };
        auto Nw = [&](int k) { return M(r, nw, k); };
        auto Cx = [&](int k) { return C(r, k); };
        T* t0 = Tm(r, 0);
        T* t1 = Tm(r, 1);
        T* t2 = Tm(r, 2);
        T* t3 = Tm(r, 3);
        T* t4 = Tm(r, 4);
        T* t5 = Tm(r, 5);
        if (r <= G.mid) {
          if (r < G.mid) {  // crossmap_upper, :600-644
            s.gemm(b, -1.0, t0, Mn(6), Cx(0), Cx(0));
            s.gemm(b, -1.0, t0, Mn(7), Cx(1), Cx(1));
            s.gemm(b, -1.0, t1, Mn(6), Cx(2), Cx(2));
            s.gemm(b, -1.0, t1, Mn(7), Cx(3), Cx(3));
          } else {  // crossmap_middle, :647-697
            s.gemm(b, -1.0, t4, Mn(0), Cx(0), Cx(0));
            s.gemm(b, -1.0, t4, Mn(1), Cx(1), Cx(1));
            s.gemm(b, -1.0, t5, Mn(0), Cx(2), Cx(2));
            s.gemm(b, -1.0, t5, Mn(1), Cx(3), Cx(3));
          }
          s.gemm(b, -1.0, t2, Mo(6), Cx(4), Cx(4));
          s.gemm(b, -1.0, t2, Mo(7), Cx(5), Cx(5));
          s.gemm(b, -1.0, t3, Mo(6), Cx(6), Cx(6));
          s.gemm(b, -1.0, t3, Mo(7), Cx(7), Cx(7));
          // matrixmap_upper, :780-830
          s.gemm(b, 1.0, t0, Mo(6), Mo(8), Nw(8));
          s.gemm(b, 1.0, t0, Mo(7), Mo(9), Nw(9));
          s.gemm(b, 1.0, t1, Mo(6), Mo(10), Nw(10));
          s.gemm(b, 1.0, t1, Mo(7), Mo(11), Nw(11));
          s.gemm(b, 1.0, EH(G, 0), Mo(6), Mo(0), Nw(0));
          s.gemm(b, 1.0, EH(G, 0), Mo(7), Mo(1), Nw(1));
          s.gemm(b, 1.0, t0, ULL, Mo(4), Nw(4));
          s.gemm(b, 1.0, t1, ULL, Mo(5), Nw(5));
          s.gemm(b, 1.0, t4, DUR, nullptr, Nw(2));
          s.gemm(b, 1.0, t5, DUR, nullptr, Nw(3));
          s.gemm(b, 1.0, EH(G, 1), Mo(6), nullptr, Nw(6));
          s.gemm(b, 1.0, EH(G, 1), Mo(7), nullptr, Nw(7));
        } else {
          if (r < G.end) {  // crossmap_lower, :700-744
            s.gemm(b, -1.0, t0, Mn(0), Cx(0), Cx(0));
            s.gemm(b, -1.0, t0, Mn(1), Cx(1), Cx(1));
            s.gemm(b, -1.0, t1, Mn(0), Cx(2), Cx(2));
            s.gemm(b, -1.0, t1, Mn(1), Cx(3), Cx(3));
            s.gemm(b, -1.0, t2, Mo(0), Cx(4), Cx(4));
            s.gemm(b, -1.0, t2, Mo(1), Cx(5), Cx(5));
            s.gemm(b, -1.0, t3, Mo(0), Cx(6), Cx(6));
            s.gemm(b, -1.0, t3, Mo(1), Cx(7), Cx(7));
          }
          // matrixmap_lower, :833-900
          s.gemm(b, 1.0, t0, Mo(0), Mo(8), Nw(8));
          s.gemm(b, 1.0, t0, Mo(1), Mo(9), Nw(9));
          s.gemm(b, 1.0, t1, Mo(0), Mo(10), Nw(10));
          s.gemm(b, 1.0, t1, Mo(1), Mo(11), Nw(11));
          s.gemm(b, 1.0, t0, DUR, Mo(2), Nw(2));
          s.gemm(b, 1.0, t1, DUR, Mo(3), Nw(3));
          s.gemm(b, 1.0, t4, ULL, nullptr, Nw(4));
          s.gemm(b, 1.0, t5, ULL, nullptr, Nw(5));
          s.gemm(b, 1.0, EH(G, 2), Mo(0), Mo(6), Nw(6));
          s.gemm(b, 1.0, EH(G, 2), Mo(1), Mo(7), Nw(7));
          s.gemm(b, 1.0, EH(G, 3), Mo(0), nullptr, Nw(0));
          s.gemm(b, 1.0, EH(G, 3), Mo(1), nullptr, Nw(1));
        }
      }
    }
  }

  // ---- production (produce_partition :903-1000, produce_bridges :1297-1436)
  const int f = steps & 1;
  s.begin();
  for (int p = 0; p < P; p++) {
    const int l = last(p);
    for (int c = 0; c <= l; c++) {
      s.gemm(b, 1.0, M(p, f, 8), Rf(p, c), nullptr, Y(p, c), M(p, f, 9), Rl(p, c));
      s.gemm(b, 1.0, M(p, f, 10), Rf(p, c), nullptr, Z(p, c), M(p, f, 11), Rl(p, c));
    }
    if (p + 1 < P) {
      const int q = p + 1, lq = last(q);
      s.gemm(b, 1.0, C(p, 0), Kd(q, 0), nullptr, Y(p, l + 1), C(p, 1), Cf(q, lq));
      s.gemm(b, 1.0, C(p, 2), Kd(q, 0), nullptr, Z(p, l + 1), C(p, 3), Cf(q, lq));
      s.gemm(b, 1.0, C(p, 4), Rf(p, l), nullptr, Y(p, l + 2), C(p, 5), Kd(p, l));
      s.gemm(b, 1.0, C(p, 6), Rf(p, l), nullptr, Z(p, l + 2), C(p, 7), Kd(p, l));
    }
  }
  s.begin();
  for (int p = 0; p < P; p++) {
    const int l = last(p), r0 = parts[p].s;
    // element(M, r, c) = K_rc + K_r0 (M8 K_0c + M9 K_lc) + K_rl (M10 K_0c + M11 K_lc)
    for (int i = 0; i <= l; i++) {
      s.gemm(b, 1.0, Cf(p, i), Y(p, i), Kd(p, i), Gd + (size_t)(r0 + i) * bb, Cl(p, i), Z(p, i));
      if (i < l) {
        s.gemm(b, 1.0, Cf(p, i), Y(p, i + 1), Ku(p, i), Gu + (size_t)(r0 + i) * bb, Cl(p, i), Z(p, i + 1));
        s.gemm(b, 1.0, Cf(p, i + 1), Y(p, i), Kl(p, i), Gl + (size_t)(r0 + i) * bb, Cl(p, i + 1), Z(p, i));
      }
    }
    if (p + 1 < P) {
      const int q = p + 1, lq = last(q), r = r0 + l;
      s.gemm(b, 1.0, Cf(p, l), Y(p, l + 1), nullptr, Gu + (size_t)r * bb, Kd(p, l), Z(p, l + 1));
      s.gemm(b, 1.0, Kd(q, 0), Y(p, l + 2), nullptr, Gl + (size_t)r * bb, Rf(q, lq), Z(p, l + 2));
    }
  }
  std::vector<ExecPhase> kept;
  for (auto& ph : s.phases)
    if (ph.units > 0) kept.push_back(ph);
  s.phases.swap(kept);
}

struct PdivLayout {
  size_t ops_off, phases_off, data_off, total;
  int nops, nphases, tile;
};

int pdiv_tile(int b) { return b >= 128 ? 64 : 32; }

template <class T>
PdivLayout pdiv_layout(const PdivPlan& P, const T* diag, const T* upper, const T* lower, T* Gd, T* Gu, T* Gl,
                       unsigned char* ws, Sched* out) {
  PdivLayout L{};
  L.tile = pdiv_tile(P.b);
  Sched s;
  s.bm = s.bn = L.tile;
  build_pdiv<T>(s, P, diag, upper, lower, Gd, Gu, Gl, (T*)nullptr);
  L.nops = (int)s.ops.size();
  L.nphases = (int)s.phases.size();
  L.ops_off = sizeof(WsHeader);
  L.phases_off = align_up(L.ops_off + (size_t)L.nops * sizeof(ExecOp), 256);
  L.data_off = align_up(L.phases_off + (size_t)L.nphases * sizeof(ExecPhase), 256);
  L.total = align_up(L.data_off + P.data_elems * sizeof(T), 256);
  if (out && ws) {
    out->bm = out->bn = L.tile;
    build_pdiv<T>(*out, P, diag, upper, lower, Gd, Gu, Gl, (T*)(ws + L.data_off));
  }
  return L;
}

template <class T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, 1) pdiv_kernel(unsigned char* ws, int nphases) {
  run_uploaded_schedule<T, BM, BN>(ws, nphases);
}

template <class T>
T host_one();
template <>
cplx host_one<cplx>() { return cplx{1.0, 0.0}; }
template <>
double host_one<double>() { return 1.0; }

template <class T>
int run_pdiv(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, void* Gd,
             void* Gu, void* Gl, void* workspace, size_t ws_bytes, cudaStream_t stream) {
  if (n < 1 || b < 1 || !diag || !Gd || !workspace) return SINVB_EINVAL;
  if (!power_of_two(partitions) || partitions > n || partitions > kPdivMaxPartitions) return SINVB_EINVAL;
  if (n > 1 && (!upper || !lower || !Gu || !Gl)) return SINVB_EINVAL;
  if ((uintptr_t)workspace % 256) return SINVB_EWORKSPACE;
  for (const void* p : {diag, upper, lower, (const void*)Gd, (const void*)Gu, (const void*)Gl})
    if (p && (uintptr_t)p % sizeof(T)) return SINVB_EINVAL;
  int rc = check_device();
  if (rc) return rc;
  unsigned char* ws = (unsigned char*)workspace;
  const PdivPlan P = pdiv_plan(n, b, partitions);
  Sched s;
  PdivLayout L = pdiv_layout<T>(P, (const T*)diag, (const T*)upper, (const T*)lower, (T*)Gd, (T*)Gu, (T*)Gl, ws,
                                &s);
  if (ws_bytes < L.total) return SINVB_EWORKSPACE;
  WsHeader h{};
  h.desc_offset = L.ops_off;
  h.items_offset = L.phases_off;
  h.sched_phases = L.nphases;
  std::vector<T> eye((size_t)b * b, T{});
  for (int i = 0; i < b; i++) eye[(size_t)i * b + i] = host_one<T>();
  T* data = (T*)(ws + L.data_off);
  SINVB_CUDA(cudaMemcpyAsync(ws, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.ops_off, s.ops.data(), s.ops.size() * sizeof(ExecOp), cudaMemcpyHostToDevice,
                             stream));
  SINVB_CUDA(cudaMemcpyAsync(ws + L.phases_off, s.phases.data(), s.phases.size() * sizeof(ExecPhase),
                             cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemcpyAsync(data + P.eye, eye.data(), eye.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
  SINVB_CUDA(cudaMemsetAsync(data + P.zero, 0, eye.size() * sizeof(T), stream));
  // (a copy from pageable memory has read `eye` when cudaMemcpyAsync returns)
  if (L.tile == 64)
    return launch_schedule_kernel<T, 64, 64>(pdiv_kernel<T, 64, 64>, ws, L.nphases, stream);
  return launch_schedule_kernel<T, 32, 32>(pdiv_kernel<T, 32, 32>, ws, L.nphases, stream);
}

template <class T>
size_t pdiv_workspace(int n, int b, int partitions) {
  if (n < 1 || b < 1 || !power_of_two(partitions) || partitions > n || partitions > kPdivMaxPartitions) return 0;
  const PdivPlan P = pdiv_plan(n, b, partitions);
  return pdiv_layout<T>(P, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr).total;
}

}  // namespace

}  // namespace sinvb

using namespace sinvb;

extern "C" {

size_t sinvb_pdiv_workspace_size(int n, int b, int partitions, int dtype, unsigned flags) {
  (void)flags;
  if (dtype == SINVB_C128) return pdiv_workspace<cplx>(n, b, partitions);
  if (dtype == SINVB_F64) return pdiv_workspace<double>(n, b, partitions);
  return 0;
}

int sinvb_pdiv_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions,
                 unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                 sinvb_stream_t stream) {
  (void)flags;
  return run_pdiv<cplx>(diag, upper, lower, n, b, partitions, G_diag, G_upper, G_lower, workspace, workspace_bytes,
                        (cudaStream_t)stream);
}

int sinvb_pdiv_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions,
                 unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                 sinvb_stream_t stream) {
  (void)flags;
  return run_pdiv<double>(diag, upper, lower, n, b, partitions, G_diag, G_upper, G_lower, workspace,
                          workspace_bytes, (cudaStream_t)stream);
}

}  // extern "C"
