// dfc_device.cuh — device helpers: PTX wrappers (TMA bulk copies, mbarriers,
// 128-bit CAS), value decoding, order-preserving encodings, hashing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dfc_internal.h"

namespace dfc {

// ---------------------------------------------------------------------------
// Shared-memory addresses, mbarriers and bulk (TMA) copies.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
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

// Bounded wait on an mbarrier phase: gives up after `limit` polls (each poll
// is itself a hardware-timed try_wait) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// Atomics.
// ---------------------------------------------------------------------------
// 128-bit compare-and-swap (sm_90+): {lo, hi} at addr.
__device__ __forceinline__ void cas128(void* addr, uint64_t cmp_lo, uint64_t cmp_hi, uint64_t new_lo,
                                       uint64_t new_hi, uint64_t& old_lo, uint64_t& old_hi) {
  asm volatile(
      "{\n\t.reg .b128 c, n, o;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 n, {%4, %5};\n\t"
      "atom.global.cas.b128 o, [%6], c, n;\n\t"
      "mov.b128 {%0, %1}, o;\n\t}"
      : "=l"(old_lo), "=l"(old_hi)
      : "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi), "l"(addr)
      : "memory");
}

__device__ __forceinline__ uint64_t ld_cg_u64(const void* p) {
  return __ldcg(reinterpret_cast<const unsigned long long*>(p));
}
// A load every iteration of a spin wait issues afresh (never hoisted).
__device__ __forceinline__ uint64_t ld_relaxed_u64(const void* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_cg_u32(const void* p) {
  return __ldcg(reinterpret_cast<const unsigned int*>(p));
}

__device__ __forceinline__ void red_add_u32(void* p, uint32_t v) {
  atomicAdd(reinterpret_cast<unsigned int*>(p), v);
}
__device__ __forceinline__ void red_min_u32(void* p, uint32_t v) {
  atomicMin(reinterpret_cast<unsigned int*>(p), v);
}
__device__ __forceinline__ void red_or_u32(void* p, uint32_t v) {
  atomicOr(reinterpret_cast<unsigned int*>(p), v);
}
__device__ __forceinline__ void red_add_u64(void* p, uint64_t v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void red_min_u64(void* p, uint64_t v) {
  atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void red_max_u64(void* p, uint64_t v) {
  atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void red_add_f64(void* p, double v) { atomicAdd(reinterpret_cast<double*>(p), v); }

// Record updates in either space: kShared selects explicit shared-memory
// atomics (a generic pointer into shared memory would take the generic path).
__device__ __forceinline__ uint32_t shared_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
template <bool kShared>
__device__ __forceinline__ void rec_add_u32(void* p, uint32_t v) {
  if constexpr (kShared) asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(shared_addr(p)), "r"(v) : "memory");
  else red_add_u32(p, v);
}
template <bool kShared>
__device__ __forceinline__ void rec_or_u32(void* p, uint32_t v) {
  if constexpr (kShared) asm volatile("red.shared.or.b32 [%0], %1;" ::"r"(shared_addr(p)), "r"(v) : "memory");
  else red_or_u32(p, v);
}
template <bool kShared>
__device__ __forceinline__ void rec_max_u32(void* p, uint32_t v) {
  if constexpr (kShared) asm volatile("red.shared.max.u32 [%0], %1;" ::"r"(shared_addr(p)), "r"(v) : "memory");
  else atomicMax(reinterpret_cast<unsigned int*>(p), v);
}
template <bool kShared>
__device__ __forceinline__ void rec_add_u64(void* p, uint64_t v) {
  if constexpr (kShared) asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(shared_addr(p)), "l"(v) : "memory");
  else red_add_u64(p, v);
}
template <bool kShared>
__device__ __forceinline__ uint64_t rec_fetch_add_u64(void* p, uint64_t v) {
  if constexpr (kShared) {
    uint64_t old;
    asm volatile("atom.shared.add.u64 %0, [%1], %2;" : "=l"(old) : "r"(shared_addr(p)), "l"(v) : "memory");
    return old;
  } else {
    return atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
  }
}
template <bool kShared>
__device__ __forceinline__ void rec_max_u64(void* p, uint64_t v) {
  if constexpr (kShared) asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(shared_addr(p)), "l"(v) : "memory");
  else red_max_u64(p, v);
}
template <bool kShared>
__device__ __forceinline__ void rec_add_f64(void* p, double v) {
  if constexpr (kShared) asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(shared_addr(p)), "d"(v) : "memory");
  else red_add_f64(p, v);
}
template <bool kShared>
__device__ __forceinline__ uint64_t rec_cas_u64(void* p, uint64_t cmp, uint64_t val) {
  if constexpr (kShared) {
    uint64_t old;
    asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "r"(shared_addr(p)), "l"(cmp), "l"(val) : "memory");
    return old;
  } else {
    return atomicCAS(reinterpret_cast<unsigned long long*>(p), (unsigned long long)cmp, (unsigned long long)val);
  }
}

// ---------------------------------------------------------------------------
// Values.
// ---------------------------------------------------------------------------
// Distributed shared memory: explicit .shared::cluster accesses on 32-bit
// cluster addresses (mapa of a local shared address to a CTA rank).
__device__ __forceinline__ uint32_t dsm_map(const void* local, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(local)), "r"(rank));
  return a;
}
__device__ __forceinline__ uint32_t dsm_ld_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.relaxed.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t dsm_ld_u64(uint32_t a) {
  uint64_t v;
  asm volatile("ld.relaxed.cluster.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t dsm_add_u32(uint32_t a, uint32_t v) {
  uint32_t old;
  asm volatile("atom.shared::cluster.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void dsm_max_u32(uint32_t a, uint32_t v) {
  asm volatile("red.shared::cluster.max.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void dsm_or_b32(uint32_t a, uint32_t v) {
  asm volatile("red.shared::cluster.or.b32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t dsm_add_u64(uint32_t a, uint64_t v) {
  uint64_t old;
  asm volatile("atom.shared::cluster.add.u64 %0, [%1], %2;" : "=l"(old) : "r"(a), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ void dsm_add_f64(uint32_t a, double v) {
  asm volatile("red.shared::cluster.add.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ uint64_t dsm_cas_u64(uint32_t a, uint64_t cmp, uint64_t val) {
  uint64_t old;
  asm volatile("atom.shared::cluster.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "r"(a), "l"(cmp), "l"(val) : "memory");
  return old;
}

__device__ __forceinline__ bool dt_float(int dt) { return dt == DFC_FLOAT32 || dt == DFC_FLOAT64; }
__device__ __forceinline__ bool dt_unsigned(int dt) {
  return dt == DFC_UINT8 || dt == DFC_UINT16 || dt == DFC_UINT32 || dt == DFC_UINT64;
}

// Raw bits of element i (zero-extended).
__device__ __forceinline__ uint64_t load_bits(const void* base, int size, uint64_t i) {
  switch (size) {
    case 1: return reinterpret_cast<const uint8_t*>(base)[i];
    case 2: return reinterpret_cast<const uint16_t*>(base)[i];
    case 4: return reinterpret_cast<const uint32_t*>(base)[i];
    default: return reinterpret_cast<const uint64_t*>(base)[i];
  }
}

// Signed value of integer bits (sign-extends signed types).
__device__ __forceinline__ int64_t bits_to_i64(uint64_t b, int dt) {
  switch (dt) {
    case DFC_INT8: return (int8_t)b;
    case DFC_INT16: return (int16_t)b;
    case DFC_INT32: return (int32_t)b;
    default: return (int64_t)b;  // INT64 and every unsigned type (zero-extended)
  }
}

__device__ __forceinline__ double bits_to_f64(uint64_t b, int dt) {
  if (dt == DFC_FLOAT32) return (double)__uint_as_float((uint32_t)b);
  return __longlong_as_double((long long)b);
}

__device__ __forceinline__ double bits_as_double(uint64_t b, int dt) {
  if (dt_float(dt)) return bits_to_f64(b, dt);
  if (dt == DFC_UINT64) return (double)b;
  return (double)bits_to_i64(b, dt);
}

// Order-preserving u64 encoding of a value (min/max by unsigned atomics).
// Floats: +0 and -0 encode alike (their tie is settled by the first zero's row).
__device__ __forceinline__ uint64_t order_encode(uint64_t b, int dt) {
  if (dt_float(dt)) {
    double d = bits_to_f64(b, dt);
    uint64_t u = (d == 0.0) ? 0ull : (uint64_t)__double_as_longlong(d);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
  }
  if (dt_unsigned(dt)) return b;
  return (uint64_t)bits_to_i64(b, dt) ^ 0x8000000000000000ull;
}

// Inverse of order_encode into the raw bits of `dt` (floats via Float64).
__device__ __forceinline__ uint64_t order_decode(uint64_t e, int dt) {
  if (dt_float(dt)) {
    uint64_t u = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFull) : ~e;
    double d = __longlong_as_double((long long)u);
    if (dt == DFC_FLOAT32) return __float_as_uint((float)d);
    return u;
  }
  if (dt_unsigned(dt)) return e;
  return e ^ 0x8000000000000000ull;
}

// Equality word of a key cell: floats canonical (every NaN one value,
// -0.0 == 0.0), integers their value bits.
__device__ __forceinline__ uint64_t key_cell(uint64_t b, int dt) {
  if (dt == DFC_FLOAT32) {
    float f = __uint_as_float((uint32_t)b);
    if (f != f) return 0x7FC00000u;
    if (f == 0.0f) return 0;
    return b;
  }
  if (dt == DFC_FLOAT64) {
    double d = __longlong_as_double((long long)b);
    if (d != d) return kCanonNaN;
    if (d == 0.0) return 0;
    return b;
  }
  return b;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__device__ __forceinline__ bool bit_valid(const uint32_t* words, uint64_t i) {
  return (words[i >> 5] >> (i & 31)) & 1u;
}

}  // namespace dfc
