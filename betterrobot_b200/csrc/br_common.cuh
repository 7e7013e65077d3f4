// br_common.cuh — shared helpers: TMA bulk-store wrappers, shared-memory
// layout arithmetic and per-device launch properties.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/br_b200.h"

namespace br {

constexpr int kWarp = 32;

__host__ __device__ __forceinline__ int round4(int n) { return (n + 3) & ~3; }

// ---- Blackwell bulk async copies (cp.async.bulk, smem -> global) ---------
// Make generic-proxy shared-memory writes visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One contiguous shared -> global copy; both addresses 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(ssrc));
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               :: "l"(gdst), "r"(s), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until every committed bulk group has finished READING shared memory.
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Wait until at most the N most recently committed bulk groups are still reading shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" :: "n"(N) : "memory");
}
// Wait until every committed bulk group has completed (writes performed).
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---- cp.async (16-byte global -> shared copies that do not pass through registers) ----
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(s), "l"(gsrc) : "memory");
}
// Wait for every cp.async this thread issued (the data is then visible to this thread;
// other threads see it after a barrier).
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// One 4-byte global -> shared copy (both addresses 4-byte aligned).
__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(s), "l"(gsrc) : "memory");
}
// Close the group of this thread's cp.async issued since the last commit.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's committed groups are still in flight.
template <int N>
__device__ __forceinline__ void cp_async_wait_groups() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// Warp-cooperative copy of `n` floats from shared to global (fallback when the
// destination block is not 16-byte aligned or its size is not a multiple of 16).
__device__ __forceinline__ void warp_copy(float* __restrict__ g, const float* __restrict__ s, int n, int lane) {
  for (int i = lane; i < n; i += kWarp) g[i] = s[i];
}

// ---- host helpers --------------------------------------------------------
struct DeviceInfo {
  int device = -1;
  int sms = 0;
  int max_smem_optin = 0;
  size_t l2_bytes = 0;
};

// Cached per current device.
// floor(e / d) by a multiply: e * ceil(2^32 / d) >> 32 is exact for 0 <= e < 2^16 and
// 1 <= d <= 128 (the error term e (ceil(2^32/d) d - 2^32) / (d 2^32) stays below 1/d), which
// covers the flattened (item, slot) indices the kernels split.  An integer
// division by a runtime divisor is a ~20-instruction dependent sequence.
struct FastDiv {
  unsigned long long m;
  int d;
  __device__ explicit FastDiv(int d_) : m((0x100000000ull + (unsigned long long)d_ - 1ull) / (unsigned long long)d_), d(d_) {}
  __device__ __forceinline__ int div(int e) const { return (int)(((unsigned long long)e * m) >> 32); }
  __device__ __forceinline__ int mod(int e) const { return e - div(e) * d; }
};

const DeviceInfo& device_info();

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline bool aligned4(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 3u) == 0; }

int validate_tree(const br_tree_t* t);

}  // namespace br
