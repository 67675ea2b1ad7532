// hvdg_common.cuh -- device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hvdg_internal.h"

namespace hvdg {

// ---- complex float2 arithmetic --------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) {
  return make_float2(a.x * s, a.y * s);
}
__device__ __forceinline__ float cnorm(float2 a) { return a.x * a.x + a.y * a.y; }
// Re[a * b]
__device__ __forceinline__ float re_mul(float2 a, float2 b) { return a.x * b.x - a.y * b.y; }

// Carrier at (line phasor, column phasor, V-switch sign): c = L * P, and
// -conj(c) on switched lines (MakeCarrierPal, ntsc_geometry.cpp:438-456).
__device__ __forceinline__ float2 carrier(float2 L, float2 P, float sw) {
  float2 c = cmul(L, P);
  return sw < 0.0f ? make_float2(-c.x, c.y) : c;
}

// ---- warp reductions --------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;  // valid in lane 0
}
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_allmax(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Order-preserving map float -> uint32 (for radix selection).
__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}

// Exact k-th smallest (0-based) of n floats in shared memory by the whole
// block: 4-pass 8-bit radix select on order-preserving keys. `hist` is
// 256 unsigned ints of shared scratch, `bcast` 2 unsigned ints. All threads
// must call. Equivalent to std::nth_element(v, v + k, v + n); v[k].
__device__ inline float block_select_kth(const float* v, int n, int k, unsigned* hist,
                                         unsigned* bcast) {
  uint32_t prefix = 0, mask = 0;
  int kk = k;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    // four elements' loads in flight per thread (the values may sit in
    // global memory), then their bins in turn; lanes counting into the same
    // bin add once through their lowest lane (the keys of one selection
    // crowd a few bins: without this the shared-memory atomics of a warp
    // serialise)
    const int step = blockDim.x;
    for (int i0 = threadIdx.x; i0 - (int)threadIdx.x < n; i0 += 4 * step) {
      float x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = i0 + q * step < n ? v[i0 + q * step] : 0.0f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t key = float_key(x[q]);
        const unsigned bin = i0 + q * step < n && (key & mask) == prefix ? (key >> shift) & 255u
                                                                         : 256u;
        const unsigned peers = __match_any_sync(__activemask(), bin);
        if (bin < 256u && (int)(__ffs(peers) - 1) == (int)(threadIdx.x & 31))
          atomicAdd(&hist[bin], (unsigned)__popc(peers));
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      // the bin holding the kk-th key: lane l owns bins 8 l .. 8 l + 7; an
      // exclusive scan of the lanes' totals gives each lane its base, and
      // the lane whose bins cross kk names the bin (counts are exact)
      const int l = threadIdx.x;
      unsigned cnt[8], tot = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        cnt[q] = hist[8 * l + q];
        tot += cnt[q];
      }
      unsigned incl = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (l >= o) incl += v;
      }
      unsigned acc = incl - tot;
      if (acc <= (unsigned)kk && (unsigned)kk < incl) {
        int b = 8 * l;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (b == 8 * l + q && acc + cnt[q] <= (unsigned)kk) {
            acc += cnt[q];
            ++b;
          }
        }
        bcast[0] = (unsigned)b;
        bcast[1] = acc;
      }
    }
    __syncthreads();
    const uint32_t b = bcast[0];
    kk -= (int)bcast[1];
    prefix |= b << shift;
    mask |= 255u << shift;
    __syncthreads();
  }
  return key_float(prefix);
}

// Bounded spin on a device-scope flag: returns true when *flag >= target
// within the iteration budget, false on timeout (caller reports an error;
// nothing traps or spins forever).
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ bool wait_at_least(const int* flag, int target,
                                              long long limit = kSpinLimit) {
  long long n = 0;
  while (ld_acquire(flag) < target) {
    if (++n > limit) return false;
    __nanosleep(256);
  }
  return true;
}


// ---- TMA bulk copies + mbarriers (sm_90+ async proxy) -----------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase; false on timeout.
constexpr long long kMbarSpinLimit = 1LL << 24;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  long long n = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++n > kMbarSpinLimit) return false;
  }
  return true;
}
// 1-D TMA bulk copy global -> shared (16-byte aligned, size multiple of 16),
// completion counted on `bar` in bytes.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace hvdg
