// Work queue of the persistent batched kernels (batched RGF, batched
// adjoint): per-instance team areas, scratch slots taken from a bitmap,
// streamed ready / done words, all waits bounded.
#pragma once

#include "common.cuh"

namespace sinvb {

// Per-instance meeting point of its team (64 bytes apart).
struct ItemArea {
  unsigned counter;  // team barrier arrivals
  int status;        // device status of the instance
  unsigned char* scratch;  // scratch slot of the team's rank-0 CTA
  int slot_id;       // its index in the slot bitmap (-1: none)
  unsigned left;     // members that have finished with the instance
  unsigned pad[10];
};
static_assert(sizeof(ItemArea) == 64, "64-byte item areas");

// Scratch slots are taken by a team's rank 0 from the bitmap hdr->slot_bits
// (hdr->nslots slots, at least as many as teams that can run at once, so a
// slot is normally free at once; the wait is bounded all the same).
__device__ inline int acquire_scratch(WsHeader* hdr, int* status, unsigned long long wait_ns) {
  const int K = (int)hdr->nslots;
  unsigned long long t0 = 0;
  for (unsigned spins = 0;; spins++) {
    for (int w = 0; w * 32 < K; w++) {
      const unsigned valid = (K - w * 32 >= 32) ? 0xffffffffu : ((1u << (K - w * 32)) - 1u);
      unsigned cur = *((volatile unsigned*)&hdr->slot_bits[w]);
      while (true) {
        const unsigned freeb = ~cur & valid;
        if (!freeb) break;
        const int bit = __ffs(freeb) - 1;
        const unsigned old = atomicOr(&hdr->slot_bits[w], 1u << bit);
        if (!(old & (1u << bit))) return w * 32 + bit;
        cur = old | (1u << bit);
      }
    }
    __nanosleep(256);
    if ((spins & 255) == 255) {
      const unsigned long long now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > wait_ns) {
        report(status, SINVB_STATUS_TIMEOUT);
        return -1;
      }
    }
  }
}
// Streamed batches: the inputs of instance k are in place once ready[k]
// holds this call's generation (written by a copy after the data, in stream
// order); a bounded wait.  Returns false (timeout reported) when the word
// never came; the instance is then skipped.
__device__ inline bool wait_ready(const WsHeader* hdr, int k, int* status, unsigned long long wait_ns) {
  const unsigned gen = hdr->gen;
  unsigned long long t0 = 0;
  for (unsigned spins = 0;; spins++) {
    unsigned v;
    asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(hdr->ready + k) : "memory");
    if (v == gen) return true;
    __nanosleep(512);
    if ((spins & 255) == 255) {
      const unsigned long long now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > wait_ns) {
        report(status, SINVB_STATUS_TIMEOUT);
        return false;
      }
    }
  }
}
// ... and done[k] tells the host that instance k's results may be copied out.
__device__ inline void signal_done(const WsHeader* hdr, int k) {
  if (!hdr->done) return;
  __threadfence_system();
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(hdr->done + k), "r"(hdr->gen) : "memory");
}

__device__ inline void release_scratch(WsHeader* hdr, int id) {
  if (id < 0) return;
  __threadfence();
  atomicAnd(&hdr->slot_bits[id >> 5], ~(1u << (id & 31)));
}

// Called by thread 0 of every member once its CTA is done with the instance
// (after a __syncthreads), on every path out of it: the last member to leave
// returns the scratch slot.  A failed pivot leaves every member running to the
// sweep's final barrier, a wait that gave up lets members leave at different
// times; either way the slot comes free only when no member can touch it.
__device__ inline void leave_item(WsHeader* hdr, ItemArea* item, int team) {
  __threadfence();
  if (atomicAdd(&item->left, 1u) == (unsigned)team - 1) {
    __threadfence();  // rank 0 wrote slot_id before it left
    const int id = *((volatile int*)&item->slot_id);
    release_scratch(hdr, id);
  }
}

// Thread 0 of rank 0: the instance's status to the caller's array and the
// call-wide word, and (streamed calls) its done word.
__device__ inline void finish_item(WsHeader* hdr, ItemArea* item, int orig) {
  const int st = *((volatile int*)&item->status);
  if (hdr->inst_status) hdr->inst_status[orig] = st;
  if (st) report(&hdr->status, st);
  signal_done(hdr, orig);
}

}  // namespace sinvb
