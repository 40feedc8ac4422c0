// Shared device helpers of the flyb200 kernels (sm_100a).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/flyb200.h"

#define FLYB_API extern "C" __attribute__((visibility("default")))

namespace flyb {

// ------------------------------------------------------------------ status words
// status[0]: first error code, status[1]: where (kernel-specific), status[2]: step
__device__ __forceinline__ void set_error(int* status, int code, int where, int step) {
  if (status && atomicCAS(status, 0, code) == 0) {
    status[1] = where;
    status[2] = step;
  }
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------------ grid barrier
// Generation barrier over all blocks of a co-resident (cooperative) grid. sync[0] counts
// arrivals, sync[1] is the generation. Every wait is bounded: after kSpinLimit polls the block
// records FLYB_EBARRIER in status and returns false; callers then return, so a grid that is not
// co-resident ends with an error status instead of hanging.
constexpr long long kSpinLimit = 1ll << 24;   // polls with a 64-256 ns backoff: seconds at most

// Polls *p until it differs from `value`, at most `limit` times (or until status is set).
// Returns false, with FLYB_EBARRIER recorded at `where`, when the limit ran out.
__device__ __forceinline__ bool bounded_wait_ne(const int* p, int value, int* status, long long limit, int where,
                                                int step) {
  long long it = 0;
  unsigned ns = 64;
  while (ld_acquire(p) == value) {
    if (++it > limit || ld_acquire(status) != 0) {
      set_error(status, FLYB_EBARRIER, where, step);
      return false;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
  return true;
}

__device__ __forceinline__ bool grid_barrier(int* sync, int* status, int& generation, int step) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    const int gen = generation;
    __threadfence();
    const int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int arrived = atomicAdd(&sync[0], 1);
    if (arrived == nblocks - 1) {
      sync[0] = 0;
      __threadfence();
      st_release(&sync[1], gen + 1);
    } else if (!bounded_wait_ne(&sync[1], gen, status, kSpinLimit, 1, step)) {
      ok = 0;
    }
    __threadfence();
  }
  __syncthreads();
  generation += 1;
  return ok != 0;
}

// ------------------------------------------------------------------ bulk async copies (no multicast)
// Global <-> shared copies by the async proxy (PTX cp.async.bulk, sm_90 and later), completion of
// loads tracked by an mbarrier transaction count, stores by bulk groups of the issuing thread.
// Addresses 16-byte aligned, sizes multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of async transfer on the barrier's current phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Polls of an mbarrier wait: each try_wait may itself suspend for a short hardware-defined time,
// so this bounds a wait to about a second.
constexpr long long kMbarLimit = 1ll << 20;

// Waits for the phase of `parity` to complete, at most `limit` polls; false (and FLYB_EBARRIER in
// status at `where`) when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status, long long limit,
                                                  int where, int step) {
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  set_error(status, FLYB_EBARRIER, where, step);
  return false;
}

__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst_smem)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src_smem)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The issuing thread's committed bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// ... and have completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic shared-memory writes before later async-proxy reads of them.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
// the 4x32 Philox S-box with the multipliers and Weyl key increments given in that paper.
__device__ __forceinline__ void philox4x32_10(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t& c3,
                                              uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += W0; k1 += W1; }
    const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
    const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
}

// Uniform in [0, 1) with 24 random bits for (seed, step, neuron, fly).
__device__ __forceinline__ float philox_uniform(unsigned long long seed, long long step, uint32_t neuron,
                                                uint32_t fly) {
  uint32_t c0 = (uint32_t)step, c1 = (uint32_t)((unsigned long long)step >> 32), c2 = neuron, c3 = fly;
  philox4x32_10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
  return (float)(c0 >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float clip01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }

}  // namespace flyb

// Host-side helpers
#define FLYB_CHECK_LAUNCH() do { cudaError_t e__ = cudaGetLastError(); if (e__ != cudaSuccess) return (int)e__; } while (0)
