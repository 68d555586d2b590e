// Shared host/device helpers for libsppgpu: status handling, mbarrier and
// bulk-copy (cp.async.bulk) wrappers with bounded waits, device status words.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/sppgpu.h"

namespace spp {

// Records a formatted message for spp_last_error_string() and returns `code`.
int fail(int code, const char* fmt, ...);
// Maps a CUDA error to SPP_ERR_CUDA with context; SPP_OK if e == cudaSuccess.
int cuda_status(cudaError_t e, const char* what);
// Sets cudaFuncAttributeMaxDynamicSharedMemorySize once per (device, kernel).
int set_smem_attr(const void* fn, int64_t bytes);

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
static inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Device status block at the head of every workspace (16 bytes, 4 words):
//   [0] error bits (SPP_DEV_* below), [1] first failing block, [2] detail,
//   [3] reserved.
constexpr int64_t kStatusBytes = 256;  // keeps the data that follows 256-B aligned
// Word of the status block where the float corner turn flags samples that
// are not normal float32 (words 0-3 are the device status).
constexpr int kSpecialWord = 16;
enum : uint32_t {
  SPP_DEV_TIMEOUT = 1u,   // a bounded mbarrier wait expired
  SPP_DEV_RANGE = 2u,     // a delay fell outside the declared range (clamped)
};

}  // namespace spp

// ---------------------------------------------------------------------------
// Device-side helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__

namespace spp {

__device__ __forceinline__ void dev_flag(uint32_t* status, uint32_t bits, uint32_t detail) {
  if (status == nullptr) return;
  uint32_t old = atomicOr(status, bits);
  if (old == 0) {
    status[1] = blockIdx.x + gridDim.x * blockIdx.y;
    status[2] = detail;
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase.  Gives up after ~2 s of wall time (read
// from %globaltimer every 256 polls), flags SPP_DEV_TIMEOUT and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 0 && global_timer_ns() - t0 > 2000000000ull) {
      dev_flag(status, SPP_DEV_TIMEOUT, i);
      return false;
    }
  }
}

// Bounded wait with an explicit limit (nanoseconds), for the self-test.
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, uint32_t* status,
                                             uint64_t limit_ns) {
  const uint64_t t0 = global_timer_ns();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0 && global_timer_ns() - t0 > limit_ns) {
      dev_flag(status, SPP_DEV_TIMEOUT, i);
      return false;
    }
  }
}

// 1-D bulk copy global -> shared, completion signalled on `bar` (transaction
// bytes).  dst/src 16-B aligned, bytes a multiple of 16.  Plain (no cluster
// multicast) copy of this GPU's own memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace spp

#endif  // __CUDACC__
