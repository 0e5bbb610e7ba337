// Device-side building blocks shared by the sort engine's kernels: key order
// transforms, bounded spin helpers and the TMA bulk-copy / mbarrier wrappers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "engine_types.h"

namespace mgs {

enum KeyKind : int { kUnsignedKey = 0, kSignedKey = 1, kFloatKey = 2 };

// Radix order of a key, as CUB DeviceRadixSort 2.8.2 defines it for thrust::sort
// on arithmetic keys (the sort behind src/tanasic_sort.cuh:264): unsigned keys
// as they are; signed keys with the sign bit flipped; IEEE-754 keys with -0.0
// first mapped to +0.0, then the sign bit flipped for positive values and every
// bit flipped for negative values. NaNs thereby order by their bit pattern.
// The engine keeps the original bits in memory and derives digits and
// comparisons from this order, so -0.0 and +0.0 survive unchanged and keep
// their input order (the sort is stable).
template <typename BitsT, int KIND>
struct KeyTraits {
  using Bits = BitsT;
  static constexpr int kKind = KIND;
  static constexpr int kBits = int(sizeof(BitsT) * 8);
  static constexpr int kPasses = int(sizeof(BitsT));  // 8-bit digits
  static constexpr BitsT kSign = BitsT(1) << (kBits - 1);

  __host__ __device__ __forceinline__ static BitsT Ordered(BitsT b) {
    if (KIND == kUnsignedKey) return b;
    if (KIND == kSignedKey) return b ^ kSign;
    if (b == kSign) b = 0;
    const BitsT neg = BitsT(0) - (b >> (kBits - 1));  // all ones when the sign bit is set
    return b ^ (neg | kSign);
  }
  __host__ __device__ __forceinline__ static uint32_t Digit(BitsT b, int pass) {
#ifdef __CUDA_ARCH__
    // byte `pass` of a 4-byte key, zero-extended, in one byte-permute
    if constexpr (sizeof(BitsT) == 4) return __byte_perm(uint32_t(Ordered(b)), 0u, 0x4440u | uint32_t(pass));
#endif
    return uint32_t(Ordered(b) >> (pass * 8)) & 0xFFu;
  }
  // Strict "a before b" in radix order (equal keys are not before each other).
  __host__ __device__ __forceinline__ static bool Less(BitsT a, BitsT b) { return Ordered(a) < Ordered(b); }
};

// Digit extraction of the radix passes.
//   PlainDigits: the 8-bit digits of the whole ordered key, ascending (the
//                thrust::sort / CUB SortKeys order).
//   RangeDigits: the 8-bit digits of bits [begin, end) of the ordered key (the
//                last digit narrower when end - begin is not a multiple of 8),
//                each reversed when descending (CUB's begin_bit / end_bit and
//                SortKeysDescending). Passes beyond the range give every key
//                digit 0, so the sort skips them as identities; the passes stay
//                stable, so keys equal on the range keep their input order.
//                Zeros of IEEE keys follow CUB's onesweep (every CUB sort of
//                more than one tile of keys): ascending, both -0.0 and +0.0
//                take the ordered pattern of +0.0; descending, both take that
//                of -0.0. Over the whole key the two patterns are neighbours
//                and the choice never shows; on a partial bit range it decides
//                where zeros go.
struct PlainDigits {
  template <class Tr>
  __device__ __forceinline__ uint32_t digit(typename Tr::Bits k, int pass) const {
    return Tr::Digit(k, pass);
  }
};
struct RangeDigits {
  int begin, end, descending;
  template <class Tr>
  __device__ __forceinline__ uint32_t digit(typename Tr::Bits k, int pass) const {
    const int shift = begin + 8 * pass;
    const int width = min(max(end - shift, 0), 8);
    if (width == 0) return 0u;  // shift < end <= key bits whenever width > 0
    const uint32_t mask = (1u << width) - 1u;
    typename Tr::Bits o = Tr::Ordered(k);
    if (Tr::kKind == kFloatKey && descending && o == Tr::kSign) o = Tr::kSign - 1;  // zeros as -0.0
    const uint32_t d = uint32_t(o >> shift) & mask;
    return descending ? (mask ^ d) : d;
  }
};

// Digits of the ordered key minus `base`, for keys whose ordered values all lie
// in [base, base + 2^(8 * passes)): a set of keys that spans a narrow range (a
// k-way merge tile, a segment) is sorted by that many passes. B is the key's
// bit type.
template <typename B>
struct OffsetDigits {
  B base;
  template <class Tr>
  __device__ __forceinline__ uint32_t digit(typename Tr::Bits k, int pass) const {
    static_assert(sizeof(typename Tr::Bits) == sizeof(B), "base of the key's width");
    return uint32_t((B(Tr::Ordered(k)) - base) >> (8 * pass)) & 0xFFu;
  }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t lanemask_gt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_gt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_volatile_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.volatile.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Streaming 16-byte load (data is touched once per pass).
__device__ __forceinline__ uint4 ld_stream_v4(const uint4* p) { return __ldcs(p); }

// ---- TMA bulk copy (cp.async.bulk, no tensor map, no multicast) ----------
// Local-HBM -> shared-memory bulk copies completed on an mbarrier. Both
// addresses must be 16-byte aligned and the byte count a multiple of 16.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_parity(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait on an mbarrier phase; false when the bound ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_tries) {
  for (uint32_t i = 0; i < max_tries; ++i) {
    if (mbar_try_wait_parity(bar, parity)) return true;
  }
  return false;
}

// Block-wide exclusive scan of one uint32 per thread (BLOCK a multiple of 32,
// at most 1024). `warp_tmp` needs BLOCK/32 + 1 words. Returns the exclusive prefix
// and writes the block total to *total.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tmp, uint32_t* total) {
  constexpr int kWarps = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tmp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kWarps ? warp_tmp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kWarps) warp_tmp[lane] = wi - w;  // exclusive warp offsets
    if (lane == kWarps - 1) warp_tmp[kWarps] = wi;
  }
  __syncthreads();
  const uint32_t r = warp_tmp[warp] + incl - v;
  *total = warp_tmp[kWarps];
  __syncthreads();
  return r;
}

}  // namespace mgs
