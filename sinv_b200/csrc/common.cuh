// Shared device helpers of libsinvb: element types, status words, teams of
// CTAs, asynchronous copies.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sinvb.h"

namespace sinvb {

// ---------------------------------------------------------------------------
// Element types.  Complex values are interleaved (re, im) doubles, 16-byte
// aligned: the numpy / torch complex128 layout.
// ---------------------------------------------------------------------------
struct __align__(16) cplx {
  double re, im;
};

template <class T> struct Elem;
template <> struct Elem<double> {
  static constexpr bool kComplex = false;
  __device__ static double zero() { return 0.0; }
  __device__ static double one() { return 1.0; }
};
template <> struct Elem<cplx> {
  static constexpr bool kComplex = true;
  __device__ static cplx zero() { return {0.0, 0.0}; }
  __device__ static cplx one() { return {1.0, 0.0}; }
};

__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
// a - b*c
__device__ __forceinline__ cplx fms(cplx a, cplx b, cplx c) {
  return {fma(-b.re, c.re, fma(b.im, c.im, a.re)), fma(-b.re, c.im, fma(-b.im, c.re, a.im))};
}
__device__ __forceinline__ double fms(double a, double b, double c) { return fma(-b, c, a); }

// Reciprocal of a pivot.  Complex: conj(p) / |p|^2 with the larger component
// factored out first (Smith's scaling) so |p|^2 cannot overflow.
__device__ __forceinline__ double recip(double p) { return 1.0 / p; }
__device__ __forceinline__ cplx recip(cplx p) {
  if (fabs(p.re) >= fabs(p.im)) {
    double r = p.im / p.re;
    double d = 1.0 / fma(p.im, r, p.re);
    return {d, -r * d};
  } else {
    double r = p.re / p.im;
    double d = 1.0 / fma(p.re, r, p.im);
    return {r * d, -d};
  }
}
__device__ __forceinline__ bool pivot_ok(double p) { return p != 0.0 && isfinite(p); }
__device__ __forceinline__ bool pivot_ok(cplx p) {
  return (p.re != 0.0 || p.im != 0.0) && isfinite(p.re) && isfinite(p.im);
}

// ---------------------------------------------------------------------------
// Workspace header: first 256 bytes of every workspace.
// ---------------------------------------------------------------------------
struct WsHeader {
  int status;                 // SINVB_OK or SINVB_STATUS_* (first failure of the call)
  int reserved;
  unsigned int barrier_count; // grid-team barrier arrivals
  unsigned int queue_head;    // batched work queue
  // batched launches: written by the upload, read by the persistent kernel
  int count;                  // instances
  unsigned int flags;
  unsigned int nslots;        // scratch slots (batched: one per concurrent team)
  unsigned int pad0;
  unsigned long long slot_bytes;
  unsigned long long desc_offset;
  unsigned long long slots_offset;
  int* inst_status;           // caller's per-instance status array (may be null)
  unsigned long long items_offset;
  int total_slots;            // sum of team sizes
  unsigned int slot_bits[8];  // batched: scratch slots in use (bit per slot, up to 256)
  const unsigned int* ready;  // batched, streamed: instance k starts once ready[k] == gen
  unsigned int* done;         // batched, streamed: done[k] = gen when instance k has finished
  unsigned int gen;
  unsigned int barrier_half[2];  // two-sided RGF: the left and right teams' barrier counters
  int sched_phases;              // schedule executor (batched BCR): phases in the uploaded table
  unsigned int pad[27];
};
static_assert(sizeof(WsHeader) == 256, "header is 256 bytes");

// First failure wins; later ones keep the first code.
__device__ __forceinline__ void report(int* status, int code) { atomicCAS(status, 0, code); }


// ---------------------------------------------------------------------------
// Teams: the set of CTAs that cooperate on one matrix.  A team splits each
// phase's tiles among its CTAs and separates dependent phases with sync().
// sync() returns false when a bounded wait gave up; callers then return.
// ---------------------------------------------------------------------------
struct TeamCta {
  __device__ int rank() const { return 0; }
  __device__ int size() const { return 1; }
  __device__ bool sync() const {
    __syncthreads();
    return true;
  }
};

struct TeamCluster {
  __device__ int rank() const {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
  }
  __device__ int size() const {
    unsigned n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return (int)n;
  }
  // Hardware cluster barrier with release/acquire ordering of the CTAs'
  // global-memory writes.
  __device__ bool sync() const {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
    return true;
  }
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Upper bound of every team-barrier wait.  Team members may join late (a
// CTA finishes its previous instance first), so the bound is generous; a wait
// that reaches it reports SINVB_STATUS_TIMEOUT and the team abandons the work.
constexpr unsigned long long kTeamWaitNs = 60ull * 1000000000ull;

// A team of `n` CTAs that meet at a counter in global memory: the CTAs of a
// cooperative launch (the whole GPU on one matrix) or the members of one
// batched work item.  Generation g waits for (g+1) * n arrivals.  All members
// are resident (persistent or cooperative launches), so every wait ends.
struct TeamDyn {
  unsigned* counter;
  int* status;
  int r, n;
  unsigned generation;
  unsigned long long wait_ns = kTeamWaitNs;  // bound of each wait (batched calls may lower it)
  __device__ int rank() const { return r; }
  __device__ int size() const { return n; }
  __device__ bool sync() {
    if (n == 1) {
      __syncthreads();
      return true;
    }
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned target = (generation + 1) * (unsigned)n;
      __threadfence();
      atomicAdd(counter, 1u);
      unsigned seen;
      int good = 1;
      unsigned long long t0 = 0;
      for (unsigned spins = 0;; spins++) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(counter) : "memory");
        if (seen >= target) break;
        if (spins > 64) {
          __nanosleep(64);
          if ((spins & 1023) == 0) {
            unsigned long long now = global_ns();
            if (t0 == 0) t0 = now;
            else if (now - t0 > wait_ns) {
              report(status, SINVB_STATUS_TIMEOUT);
              good = 0;
              break;
            }
          }
        }
      }
      __threadfence();
      ok = good;
    }
    __syncthreads();
    generation++;
    return ok != 0;
  }
};

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (zero-filled when src_bytes == 0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 8 : 0));
}
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem, bool valid);
template <>
__device__ __forceinline__ void cp_async_elem<cplx>(cplx* smem, const cplx* gmem, bool valid) {
  cp_async16(smem, gmem, valid);
}
template <>
__device__ __forceinline__ void cp_async_elem<double>(double* smem, const double* gmem, bool valid) {
  cp_async8(smem, gmem, valid);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N));
}

// FP64 tensor-core MMA: D(8x8) += A(8x4, row) * B(4x8, col).
// Fragment ownership (lane = 4*g + t): A[g][t], B[t][g], C[g][2t], C[g][2t+1].
__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

}  // namespace sinvb
