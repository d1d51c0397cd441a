// Shared helpers for the motionest CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/motionest.h"

namespace me {

typedef long long i64;

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kInvTwoPi = 0.15915494309189533576888376337251;

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
  return make_float2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// a * b + c with four fused multiply-adds
__host__ __device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(-a.y, b.y, fmaf(a.x, b.x, c.x)), fmaf(a.y, b.x, fmaf(a.x, b.y, c.y)));
}
// Division by a divisor 1 <= d < 2^31 fixed at launch, for 0 <= n < 2^31, by the round-up
// multiply-shift method (Granlund and Montgomery, 1994): q = (umulhi(n, m) + n) >> s with
// s = ceil(log2 d) and m = floor(2^32 (2^s - d) / d) + 1.
struct FastDiv {
  unsigned m;
  int s;
  void set(int d) {
    s = 0;
    while ((1LL << s) < d) s++;
    m = (unsigned)(((1ULL << 32) * ((1ULL << s) - (unsigned long long)d)) / (unsigned long long)d + 1);
  }
  __device__ __forceinline__ int div(int n) const {
    return (int)((__umulhi((unsigned)n, m) + (unsigned)n) >> s);
  }
};

// multiply by +i or -i
__host__ __device__ __forceinline__ float2 mul_i(float2 a) { return make_float2(-a.y, a.x); }
__host__ __device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }

// exp(i*phi) with the argument reduced in double precision first, then evaluated in float.
__device__ __forceinline__ float2 expi_reduced(double phi) {
  double r = phi - kTwoPi * rint(phi * kInvTwoPi);
  float s, c;
  sincosf((float)r, &s, &c);
  return make_float2(c, s);
}

// Ampere-style asynchronous global -> shared copies (16 bytes; both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// 8-byte variant (both addresses 8-byte aligned), cached in L1.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// ---- Bulk copies on the TMA engine (non-tensor form) tracked by an mbarrier ----
// A bulk copy moves one contiguous range global -> shared without per-thread load
// instructions: one thread posts the byte count on the barrier and issues the copies, every
// consumer waits on the barrier's phase.  Both addresses must be 16-byte aligned and the size
// a multiple of 16 bytes (the callers check this on the host and otherwise use cp.async).
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// makes the initialised barrier visible to the async proxy (the copy engine)
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// orders this thread's earlier generic-proxy shared-memory accesses (made visible to it by a
// CTA barrier) before the async-proxy writes of the copies it issues next
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Tiled tensor copies (TMA, no multicast) through a tensor map held in kernel parameter space
// (__grid_constant__), between this GPU's global memory and this CTA's shared memory.  The
// load completes on an mbarrier; stores are tracked by bulk groups of the issuing thread.
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const void* tmap, int c0, int c1,
                                            int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* smem_dst, const void* tmap, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const void* tmap, const void* smem_src, int c0,
                                             int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
          tmap),
      "r"(smem_u32(smem_src)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const void* tmap, const void* smem_src, int c0,
                                             int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];\n" ::"l"(
          tmap),
      "r"(smem_u32(smem_src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// the issuing thread's committed stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// the issuing thread's committed stores have completed
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// Every wait on a barrier is bounded: after `limit` clock cycles (about a second for the
// default) the waiting thread gives up, records the fault in this translation unit's flag
// (read and cleared on the host by me_wait_status) and carries on with whatever the buffer
// holds, so the kernel still ends and the context stays usable.  Once any wait has timed
// out, later waits give up at once instead of each spending their own limit.
constexpr long long kWaitCycles = 1LL << 31;
static __device__ unsigned g_wait_fault;  // one per translation unit (internal linkage)

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned code,
                                                  long long limit = kWaitCycles) {
  if (mbar_try_wait(bar, parity)) return true;
  if (*(volatile unsigned*)&g_wait_fault) return false;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) {
      atomicOr(&g_wait_fault, code);
      return false;
    }
  }
  return true;
}

// Host side: read and clear this translation unit's wait-fault flag (synchronises the device).
#define ME_WAIT_FAULT_ACCESSOR(fn)                                                      \
  int fn(unsigned* out) {                                                               \
    unsigned v = 0, zero = 0;                                                           \
    cudaError_t e = cudaDeviceSynchronize();                                            \
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&v, g_wait_fault, sizeof(unsigned)); \
    if (e == cudaSuccess && v) e = cudaMemcpyToSymbol(g_wait_fault, &zero, sizeof(unsigned)); \
    *out = v;                                                                           \
    return check_cuda(e, "wait status");                                                \
  }

// Fault codes recorded by the bounded waits (bits, OR-ed together).
enum WaitFault : unsigned {
  WF_SENSE_FWD = 1u,
  WF_SENSE_ADJ = 2u,
  WF_LINE_PASS = 4u,
  WF_SELFTEST = 0x100u,
};

// Allow `bytes` of dynamic shared memory for `kernel` (only needed above the 48 KB default).
template <typename K>
inline cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Count of kernel launches issued by the library (reported by me_launch_count).
void count_launch();
void count_launches(long long n);  // n kernels of a graph launch

// Error state of the library (per host thread).
void set_error(const std::string& msg);
int fail(const std::string& msg);  // sets the error, returns ME_ERR_INVALID
int check_cuda(cudaError_t e, const char* what);  // returns ME_OK or ME_ERR_CUDA

}  // namespace me
