// Shared device helpers: mbarriers, TMA loads, bounded waits, error flag.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.h"

namespace ptb {

// Device-side error word (one per launch, in global memory): bit 0 = a
// bounded wait ran out.  The host reads it after the launch and reports
// LIBPT_ERR_TIMEOUT; the kernel itself returns instead of hanging.
enum : unsigned { ERR_WAIT_TIMEOUT = 1u };

// Wall-clock limit of any single device-side wait.  One GEMM tile finishes in
// well under a millisecond; two seconds only triggers on a logic error.  A
// build may set another limit with -DLIBPT_WAIT_LIMIT_NS=...; mbar_wait also
// takes a per-call limit (the wait probe of the self-test uses a short one).
#ifndef LIBPT_WAIT_LIMIT_NS
#define LIBPT_WAIT_LIMIT_NS 2000000000ull
#endif
constexpr unsigned long long WAIT_LIMIT_NS = LIBPT_WAIT_LIMIT_NS;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count));
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait until the phase with the given parity has completed.  Returns false
// (and raises ERR_WAIT_TIMEOUT in *err) if that takes longer than
// WAIT_LIMIT_NS; callers then stop issuing work and leave the kernel.
__device__ __forceinline__ bool mbar_wait(
    uint64_t *bar, uint32_t parity, unsigned *err,
    unsigned long long limit_ns = WAIT_LIMIT_NS) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > limit_ns) {
      atomicOr(err, ERR_WAIT_TIMEOUT);
      return false;
    }
  }
  return true;
}

// 2-D / 3-D / 4-D tiled TMA loads into shared memory, completing on an
// mbarrier (no multicast).  Coordinates are element indices, innermost first.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map,
                                            uint64_t *bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0),
      "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map,
                                            uint64_t *bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0),
      "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map,
                                            uint64_t *bar, int c0, int c1,
                                            int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0),
      "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}

// ---- CTA pairs (clusters of two) -------------------------------------------

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// All threads of both CTAs of the cluster.
__device__ __forceinline__ void cluster_sync() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Shared::cluster address of the same shared-memory location in CTA `rank`.
__device__ __forceinline__ uint32_t cluster_addr(const void *p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(a)
               : "r"(smem_u32(p)), "r"(rank));
  return a;
}

// Arrive on an mbarrier of either CTA of the cluster (shared::cluster
// address).
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar) {
  asm volatile(
      "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar)
      : "memory");
}

// 5-D tiled TMA load into this CTA's shared memory whose completion is
// counted on an mbarrier of either CTA of the pair (no multicast).
__device__ __forceinline__ void tma_load_5d_pair(void *dst,
                                                 const CUtensorMap *map,
                                                 uint32_t bar, int c0, int c1,
                                                 int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.cta_group::2.shared::cluster.global.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1),
      "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}

// Makes a tensor map that generic-proxy writes (a host copy, or a previous
// plan's maps at the same address) put in device memory visible to the TMA
// unit's tensor-map proxy; issued once per map before this CTA's first TMA
// through it.
__device__ __forceinline__ void tmap_acquire(const CUtensorMap *map) {
  asm volatile(
      "fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(
          reinterpret_cast<uint64_t>(map))
      : "memory");
}

// Remembers which maps of a job's map array this thread has fenced, so each
// map is acquired once per CTA (and again only when the array changes).
struct MapFence {
  const CUtensorMap *base = nullptr;
  unsigned long long mask = 0;
  __device__ __forceinline__ const CUtensorMap *get(const CUtensorMap *b,
                                                    int idx) {
    if (b != base) {
      base = b;
      mask = 0;
    }
    if (!((mask >> idx) & 1ull)) {
      tmap_acquire(b + idx);
      mask |= 1ull << idx;
    }
    return b + idx;
  }
};

// A job's tensor map idx: from the launch's parameter table (PM) or from
// the job's device-memory maps (fenced once per CTA).
template <bool PM>
struct MapSource {
  const LaunchMaps *pm;
  MapFence mf;
  __device__ __forceinline__ explicit MapSource(const LaunchMaps *p) : pm(p) {}
  __device__ __forceinline__ const CUtensorMap *get(const GemmJob &job,
                                                    int idx) {
    if (PM) return &pm->m[job.map0 + idx];
    return mf.get(job.maps, idx);
  }
};

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

// d += a * b on a 16x8x4 FP64 tile (DMMA).  Fragment ownership, lane =
// 4*g + t:  a0 = A[g][t], a1 = A[g+8][t];  b0 = B[t][g];
// d0,d1 = C[g][2t..2t+1], d2,d3 = C[g+8][2t..2t+1].
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0,
                                            double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
      "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ double flip_sign(double x, unsigned long long mask) {
  return __longlong_as_double(__double_as_longlong(x) ^ mask);
}

// Index of the last of `n` entries (sorted by `begin`) whose begin <= x.
template <typename T>
__device__ __forceinline__ int find_entry(const T *v, int n, int x,
                                          int32_t T::*begin) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (v[mid].*begin <= x)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// 1/d for the energy denominators (normal doubles with 2^-1000 <= |d| <=
// 2^1000), within 2 ulp of the correctly rounded reciprocal
// (libpt_selftest_recip measures it against IEEE division):
// the hardware's approximate reciprocal (PTX rcp.approx.ftz.f64, about 20
// correct bits) refined by two Newton-Raphson steps r <- r + r (1 - d r),
// each of which squares the relative error.  The energy epilogues multiply
// by it instead of dividing (an element's energy carries a few more
// rounding errors of 2^-53), in place of the much longer IEEE division
// sequence in kernels whose instruction issue is one of their limits.
__device__ __forceinline__ double recip_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}

// ---- device-resident tile queue ---------------------------------------------
//
// The reference hands triples to OpenMP threads one at a time
// (schedule(dynamic), src/pt.c:228, 353).  Here the CTAs of a persistent
// GEMM launch take output tiles one at a time from the counter in the
// launch's work list (GemmList::next): a CTA's producer thread takes its
// next tile while the current one is still being staged, and hands the
// index to the CTA's other roles through a small ring in shared memory
// (slot `full` barrier: the index is written; `empty` barrier: every
// consumer has read it).  -1 ends the sequence.  Tiles of uneven cost (jobs
// of different K, rounds mixing solves) then spread over the SMs instead of
// being dealt round-robin in advance.  Every wait is bounded.
constexpr int TQ_SLOTS = 4;

struct TileRing {
  uint64_t full[TQ_SLOTS], empty[TQ_SLOTS];
  int tile[TQ_SLOTS];
};

// Thread 0, before the CTA's first barrier: `consumers` arrivals free a slot.
__device__ __forceinline__ void tq_init(TileRing *r, uint32_t consumers) {
  for (int s = 0; s < TQ_SLOTS; ++s) {
    mbar_init(&r->full[s], 1);
    mbar_init(&r->empty[s], consumers);
  }
}

// The next tile of the launch (may be >= ntiles: none left).
__device__ __forceinline__ int tq_take(GemmList *l) {
  return atomicAdd(&l->next, 1);
}

// Producer: publishes tile t (or -1) in the next slot.
__device__ __forceinline__ bool tq_put(TileRing *r, int &slot, uint32_t &ph,
                                       int t, unsigned *err) {
  if (!mbar_wait(&r->empty[slot], ph ^ 1u, err)) return false;
  r->tile[slot] = t;
  mbar_arrive(&r->full[slot]);   // release: the index is visible after it
  if (++slot == TQ_SLOTS) {
    slot = 0;
    ph ^= 1u;
  }
  return true;
}

// Consumer (every thread of a consuming warp calls it; lane 0 frees the
// slot for the warp): the next tile index, -1 at the end or on a timeout.
__device__ __forceinline__ int tq_get(TileRing *r, int &slot, uint32_t &ph,
                                      unsigned *err, bool warp_arrives) {
  if (!mbar_wait(&r->full[slot], ph, err)) return -1;
  const int t = r->tile[slot];
  if (warp_arrives) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&r->empty[slot]);
  } else {
    mbar_arrive(&r->empty[slot]);
  }
  if (++slot == TQ_SLOTS) {
    slot = 0;
    ph ^= 1u;
  }
  return t;
}

// Producer, after its last take: the last CTA of the launch to get here
// resets the list's counters, so the next launch of the same list (a
// replayed graph, repeated self-test launches) starts from tile 0.
__device__ __forceinline__ void tq_finish(GemmList *l) {
  if (atomicAdd(&l->done, 1) == (int)gridDim.x - 1) {
    atomicExch(&l->next, 0);
    atomicExch(&l->done, 0);
  }
}

}  // namespace ptb
