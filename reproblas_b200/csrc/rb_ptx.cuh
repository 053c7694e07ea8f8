// rb_ptx.cuh -- small inline-PTX helpers shared by the kernels that stream operands through
// shared memory: 16-byte cp.async, mbarriers with bounded waits, and the bulk (TMA) copies
// that complete on an mbarrier. No form here multicasts.
#pragma once
#include <cstdint>

namespace rb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t addr, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// Polls of a bounded wait: ~2 s. Waits for copies or tensor-core work already issued (the
// drains before a CTA exits or frees TMEM) always use this limit.
constexpr long long kWaitPolls = 1ll << 25;

// Bounded wait: gives up after `polls` polls (default ~2 s) and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, unsigned parity,
                                                  long long polls = kWaitPolls) {
  for (long long it = 0; it < polls; it++) {
    if (mbar_try_wait(addr, parity)) return true;
    if (it > 1024) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// TMA: 2-D tile load into shared memory (coordinates innermost first), completion counted
// on an mbarrier. Elements outside the tensor are filled with zeros.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, int c0, int c1,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];"
      :
      : "r"(dst), "l"(tmap), "r"(c0), "r"(c1), "r"(mbar)
      : "memory");
}

// TMA: 1-D tile load (elements outside the tensor are filled with zeros).
__device__ __forceinline__ void tma_load_1d(uint32_t dst, const void* tmap, int c0, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2}], [%3];"
      :
      : "r"(dst), "l"(tmap), "r"(c0), "r"(mbar)
      : "memory");
}

// Contiguous bulk copy global -> shared (both addresses 16-byte aligned, bytes a multiple
// of 16), completion counted on an mbarrier.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :
      : "r"(dst), "l"(src), "r"(bytes), "r"(mbar)
      : "memory");
}

// Barrier over the first `count` threads of the CTA (a multiple of 32), id 1..15.
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

}  // namespace rb
