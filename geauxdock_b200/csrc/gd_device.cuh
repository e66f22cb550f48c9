// gd_device.cuh -- device helpers shared by the kernels: Philox, fast special
// functions, warp reductions, bulk (TMA) copies into shared memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gd {

// ---------------------------------------------------------------- Philox --
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with Weyl key
// increments.  Stateless: the stream position is the counter, so resuming a
// run and re-running a replica alone or in a batch give identical draws.
struct Philox4 {
  uint32_t v[4];
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                           uint32_t k0, uint32_t k1)
{
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int round = 0; round < 10; ++round) {
    if (round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  Philox4 r;
  r.v[0] = c0; r.v[1] = c1; r.v[2] = c2; r.v[3] = c3;
  return r;
}

// 32-bit draw -> uniform in (0, 1]: the reference draws curand_uniform(),
// whose range is (0, 1] (src/backend_gpu/kernel_cuda_l2_util.cu:16-26).
__host__ __device__ __forceinline__ float u01(uint32_t x)
{
  return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

// --------------------------------------------- special functions (FP32) --
// Documented PTX approximations (PTX ISA, "Floating-Point Instructions"):
// one MUFU operation each, relative error a few 2^-23.
__device__ __forceinline__ float rsqrt_approx(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x)
{
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x)
{
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------- reductions --
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Compensated butterfly: each level adds two partial sums with Knuth's
// TwoSum and carries the rounding error; the result is (sum, compensation).
__device__ __forceinline__ float warp_sum_comp(float s, float c)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float so = __shfl_xor_sync(0xffffffffu, s, o);
    const float co = __shfl_xor_sync(0xffffffffu, c, o);
    const float t = s + so;
    const float bp = t - s;
    const float err = (s - (t - bp)) + (so - bp);
    s = t;
    c = c + co + err;
  }
  return s + c;
}

// Kahan/Neumaier accumulation of x into (s, c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float x)
{
  const float t = s + x;
  if (fabsf(s) >= fabsf(x))
    c += (s - t) + x;
  else
    c += (x - t) + s;
  s = t;
}

// ------------------------------------------------- bulk copy (TMA, 1-D) --
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Non-multicast 1-D bulk copy global -> this CTA's shared memory, completing
// on `bar`.  dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Nanoseconds of the GPU's global timer (%globaltimer).
__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Remove `bytes` from the transaction count of the barrier's current phase
// (bytes announced by expect_tx that no copy will deliver).
__device__ __forceinline__ void mbar_complete_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Bounded wait for phase `parity` of `bar` to complete.  Returns false once
// `limit_ns` nanoseconds of the global timer have passed instead of spinning
// forever.  The result is per thread: a caller that must act on it as a CTA
// combines it with __syncthreads_and.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

}  // namespace gd
