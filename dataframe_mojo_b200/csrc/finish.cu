// finish.cu — group order and finalisation of the filtered hash group-by.
//
// Groups are emitted in first-appearance order among the rows the filter kept
// (maintain_order=True; dataframe/aggregation/state.mojo:267-330 merges the
// partitions' first-row runs): every live record sets the bit of its first
// row in a rows-long bitmap; a popcount prefix over the bitmap words gives
// each group its rank, and perm[rank] = record.  The output kernel then walks
// the groups in rank order, finishing every column (function.mojo:2516-2918,
// reducer.mojo:3391-3599) and packing validity bits with warp ballots.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dfc_device.cuh"
#include "dfc_internal.h"
#include "kernels.h"

namespace dfc {

__device__ __forceinline__ unsigned char* record_at(const ScanParams& p, uint32_t gid) {
  return p.records + (size_t)gid * (size_t)p.rec_stride;
}

__device__ __forceinline__ uint64_t records_handed_out(const ScanParams& p) {
  const uint32_t a = *p.alloc;
  return a < p.recs_total ? a : p.recs_total;
}

// A record is live when a claim set its first row (stored as ~row; 0 = hole).
__device__ __forceinline__ bool live_record(const ScanParams& p, uint64_t i, uint32_t& first) {
  const uint32_t enc = *reinterpret_cast<const uint32_t*>(record_at(p, (uint32_t)i) + kRecFirst);
  first = ~enc;
  return enc != 0;
}

// Marks each live record's first row in the bitmap and keeps the first rows
// densely (firsts[i], ~0 for a hole) so the rank pass reads 4 bytes per
// record instead of a record sector.
__global__ void finish_mark(const __grid_constant__ FinishParams f) {
  const ScanParams& p = f.scan;
  const uint64_t n = records_handed_out(p);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t first;
    const bool live = live_record(p, i, first);
    if (live && first >= p.rows) {
      atomicOr(p.status + 2, CHK_FIRST);
      f.firsts[i] = 0xFFFFFFFFu;
      continue;
    }
    f.firsts[i] = live ? first : 0xFFFFFFFFu;
    if (live) {
      const uint32_t bit = 1u << (first & 31);
      if (atomicOr(&f.order_bits[first >> 5], bit) & bit) atomicOr(p.status + 2, CHK_DUP);
    }
  }
}

constexpr int kScanChunk = kFinishChunk;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    uint32_t s = lane < nw ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  const uint32_t before = warp > 0 ? warp_sums[warp - 1] : 0u;
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

// Popcount of each chunk of bitmap words.
__global__ void finish_chunk_sums(const __grid_constant__ FinishParams f) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t s = 0;
  for (uint64_t w = base + threadIdx.x; w < base + kScanChunk && w < f.words; w += blockDim.x) s += __popc(f.order_bits[w]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ uint32_t partial[32];
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += partial[i];
    f.block_sums[blockIdx.x] = t;
  }
}

// Exclusive scan of the chunk sums (one block; chunks <= a few thousand).
__global__ void finish_scan_chunks(const __grid_constant__ FinishParams f, uint32_t chunks) {
  uint32_t carry = 0;
  for (uint32_t base = 0; base < chunks; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < chunks ? f.block_sums[i] : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, &total);
    if (i < chunks) f.block_sums[i] = carry + ex;
    carry += total;
  }
  // Ungrouped reductions (no key columns) give one row even when no row was
  // kept: the identity record (every state at zero).
  if (threadIdx.x == 0 && f.scan.n_keys == 0 && carry == 0) {
    carry = 1;
    f.perm[0] = kIdentityRecord;
  }
  if (threadIdx.x == 0) f.groups[0] = carry;
}

// Word-level exclusive prefix inside each chunk.
__global__ void finish_word_prefix(const __grid_constant__ FinishParams f) {
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t carry = f.block_sums[blockIdx.x];
  for (uint64_t off = 0; off < kScanChunk; off += blockDim.x) {
    const uint64_t w = base + off + threadIdx.x;
    const uint32_t v = w < f.words ? __popc(f.order_bits[w]) : 0u;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(v, &total);
    if (w < f.words) f.word_prefix[w] = carry + ex;
    carry += total;
  }
}

__global__ void finish_rank(const __grid_constant__ FinishParams f) {
  const ScanParams& p = f.scan;
  const uint64_t n = records_handed_out(p);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t first = f.firsts[i];
    if (first == 0xFFFFFFFFu) continue;
    const uint32_t w = first >> 5;
    const uint32_t rank = f.word_prefix[w] + __popc(f.order_bits[w] & ((1u << (first & 31)) - 1u));
    f.perm[rank] = (uint32_t)i;
  }
}

__device__ __forceinline__ void store_bits(void* base, int dt, uint64_t i, uint64_t b) {
  switch (dt) {
    case DFC_INT8: case DFC_UINT8: reinterpret_cast<uint8_t*>(base)[i] = (uint8_t)b; break;
    case DFC_INT16: case DFC_UINT16: reinterpret_cast<uint16_t*>(base)[i] = (uint16_t)b; break;
    case DFC_INT32: case DFC_UINT32: case DFC_FLOAT32: reinterpret_cast<uint32_t*>(base)[i] = (uint32_t)b; break;
    default: reinterpret_cast<uint64_t*>(base)[i] = b; break;
  }
}

__device__ __forceinline__ bool fits_sum(int odt, __int128 v) {
  switch (odt) {
    case DFC_INT32: return v >= (__int128)INT32_MIN && v <= (__int128)INT32_MAX;
    case DFC_UINT32: return v >= 0 && v <= (__int128)UINT32_MAX;
    case DFC_INT64: return v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX;
    case DFC_UINT64: return v >= 0 && v <= (__int128)UINT64_MAX;
    default: return true;
  }
}

__device__ __forceinline__ __int128 int_sum(const ValField& vf, const unsigned char* rec) {
  if (vf.sum_kind == SUM_I64) return (__int128)*reinterpret_cast<const long long*>(rec + vf.off_sum);
  const uint64_t lo = *reinterpret_cast<const uint64_t*>(rec + vf.off_sum);
  const uint64_t hi = *reinterpret_cast<const uint64_t*>(rec + vf.off_sum + 8);
  return (__int128)(((unsigned __int128)hi << 64) | lo);
}

// One output cell: returns its raw bits; *ok is its validity.
__device__ uint64_t output_cell(const FinishParams& f, const OutCol& oc, const unsigned char* rec, bool* ok) {
  const ScanParams& p = f.scan;
  *ok = true;
  if (oc.kind == OUT_KEY) {
    const KeyField& kf = p.keys[oc.index];
    const DevColumn& col = p.cols[kf.input];
    const bool gather = p.key_mode == KEY_TICKET || kf.dtype == DFC_FLOAT32 || kf.dtype == DFC_FLOAT64;
    if (gather) {
      const uint32_t row = ~*reinterpret_cast<const uint32_t*>(rec + kRecFirst);
      if (row >= p.rows) {
        atomicOr(p.status + 2, CHK_FIRST);
        *ok = false;
        return 0;
      }
      if (col.validity && !bit_valid(col.validity, row)) {
        *ok = false;
        return 0;
      }
      return load_bits(col.values, col.size, row);
    }
    const uint64_t kw = *reinterpret_cast<const uint64_t*>(rec + kRecKey);
    if (kf.null_bit >= 0 && ((kw >> kf.null_bit) & 1ull)) {
      *ok = false;
      return 0;
    }
    return kf.bits == 64 ? kw : ((kw >> kf.shift) & ((1ull << kf.bits) - 1ull));
  }
  const ValField& vf = p.vals[oc.val];
  const uint32_t count = *reinterpret_cast<const uint32_t*>(rec + vf.off_count);
  const int idt = vf.dtype;
  const bool isf = dt_float(idt);
  switch (oc.op) {
    case DFC_AGG_COUNT: return count;
    case DFC_AGG_LEN: return *reinterpret_cast<const uint32_t*>(rec + p.off_len);
    case DFC_AGG_NULL_COUNT: return *reinterpret_cast<const uint32_t*>(rec + p.off_len) - count;
    case DFC_AGG_SUM: {
      *ok = (int64_t)count >= (int64_t)oc.min_count;
      if (isf) {
        const double s = *ok ? *reinterpret_cast<const double*>(rec + vf.off_sum) : 0.0;
        if (oc.dtype == DFC_FLOAT32) return __float_as_uint((float)s);
        return (uint64_t)__double_as_longlong(s);
      }
      if (!*ok) return 0;
      const __int128 s = int_sum(vf, rec);
      if (!fits_sum(oc.dtype, s)) {
        atomicMin(f.overflow_agg, (uint32_t)oc.index);
        atomicOr(p.status, ST_OVERFLOW);
        return 0;
      }
      return (uint64_t)s;
    }
    case DFC_AGG_MEAN: {
      *ok = count > 0;
      if (!*ok) return 0;
      double total;
      if (isf) total = *reinterpret_cast<const double*>(rec + vf.off_sum);
      else total = (double)int_sum(vf, rec);
      return (uint64_t)__double_as_longlong(total / (double)count);
    }
    case DFC_AGG_MIN:
    case DFC_AGG_MAX: {
      const bool is_max = oc.op == DFC_AGG_MAX;
      // Stored: the maximum's code, the minimum's complemented code; 0 = none.
      const uint64_t stored = *reinterpret_cast<const uint64_t*>(rec + (is_max ? vf.off_max : vf.off_min));
      const uint64_t e = is_max ? stored : ~stored;
      const bool seen = isf ? stored != 0ull : count > 0;
      const uint32_t flags = *reinterpret_cast<const uint32_t*>(rec + kRecFlags) >> (3 * oc.val);
      if (!seen) {
        // NaN only when every valid value is NaN (reducer.mojo:3576-3583).
        if (isf && (flags & 1u)) return idt == DFC_FLOAT32 ? 0x7FC00000ull : kCanonNaN;
        *ok = false;
        return 0;
      }
      uint64_t b = order_decode(e, idt);
      if (isf) {
        const bool zero = idt == DFC_FLOAT32 ? ((uint32_t)b & 0x7FFFFFFFu) == 0 : (b & 0x7FFFFFFFFFFFFFFFull) == 0;
        if (zero) {
          // A zero extremum keeps the sign of the group's first zero (ties keep
          // the earlier value, function.mojo:1213-1236).  With one sign seen
          // that is the sign; with both the CPU adjudicates.
          const bool pos = (flags >> 1) & 1u, neg = (flags >> 2) & 1u;
          if (pos && neg) atomicOr(p.status, ST_ZERO_FAULT);
          b = idt == DFC_FLOAT32 ? (neg ? 0x80000000ull : 0ull) : (neg ? 0x8000000000000000ull : 0ull);
        }
      }
      return b;
    }
    case DFC_AGG_FIRST:
    case DFC_AGG_LAST: {
      // The value at the group's first (last) kept row, null when that
      // row's value is; the identity record has neither row.
      const uint32_t r = oc.op == DFC_AGG_FIRST ? ~*reinterpret_cast<const uint32_t*>(rec + kRecFirst)
                                                 : *reinterpret_cast<const uint32_t*>(rec + p.off_last) - 1u;
      const DevColumn& col = p.cols[vf.input];
      if (r >= p.rows || (col.validity && !bit_valid(col.validity, r))) {
        *ok = false;
        return 0;
      }
      return load_bits(col.values, col.size, r);
    }
    case DFC_AGG_VAR:
    case DFC_AGG_STD: {
      const int64_t n = (int64_t)count;
      *ok = n - (int64_t)oc.ddof > 0;
      if (!*ok) return 0;
      const double K =
          __longlong_as_double((long long)(*reinterpret_cast<const uint64_t*>(rec + vf.off_shift) ^ kShiftTag));
      const double S2 = *reinterpret_cast<const double*>(rec + vf.off_m2);
      double S1;
      if (isf) {
        S1 = *reinterpret_cast<const double*>(rec + vf.off_sum) - (double)n * K;
      } else {
        S1 = (double)(int_sum(vf, rec) - (__int128)n * (__int128)K);
      }
      double M2 = S2 - S1 * (S1 / (double)n);
      if (M2 < 0.0) M2 = 0.0;
      // Conditioning.  (a) Our own error: S2 and the sum are atomically
      // accumulated FP64 (relative error ~ 8 sqrt(n) eps with high
      // confidence); |S1| <= sqrt(n S2) and sum |x| <= sqrt(n S2) + n|K|.
      // When that bound exceeds half the 1e-10 (1 + |var|) budget the result
      // is not trusted.  (b) The reference's Welford recurrence loses about
      // eps |mean| / sigma: for a mean more than 2^32 spreads from zero (the
      // [2^60, 2^60 + 256] example of docs/design/metal-moments.md:139-147)
      // its value is its own, and the CPU adjudicates (data fault).
      if (S2 == S2 && K == K && n >= 2) {
        const double eps = 1.1102230246251565e-16;
        const double dn = (double)n;
        const double g = 8.0 * sqrt(dn) * eps;
        const double sum_abs = sqrt(dn * S2) + dn * fabs(K);
        const double bound = g * S2 + 2.0 * fabs(S1) / dn * (g * sum_abs + eps * dn * fabs(K));
        const double budget = 0.5e-10 * (M2 + (double)(n - (int64_t)oc.ddof));
        const double mean = K + S1 / dn;
        const double sigma = sqrt(M2 / dn);
        const bool cpu_off = sigma > 0.0 && fabs(mean) > 4294967296.0 * sigma;
        if (bound > budget || cpu_off) atomicOr(p.status, ST_FAULT);
      }
      const double var = M2 / (double)(n - (int64_t)oc.ddof);
      const double out = oc.op == DFC_AGG_STD ? sqrt(var) : var;
      return (uint64_t)__double_as_longlong(out);
    }
  }
  *ok = false;
  return 0;
}

// A warp finishes 32 groups at a time, in rank order.  Their records lie
// at random places of `records`, so the warp first copies the 32 records
// whole into its slab of shared memory (16-byte loads, all issued before the
// first store) and finishes every column from there: one round trip to HBM
// per record instead of one per dependent field load.  A slab slot is the
// record stride + 8 bytes, so the lanes' 8-byte field reads of one offset
// fall on distinct banks.  Dynamic shared memory: finish_output_smem().
//
// Output columns with any null are noted per block in shared memory and
// reported with one global atomicOr per block and column (a per-warp atomic
// on the same word serialises in L2 when most warps hold a null group).
__global__ void finish_output(const __grid_constant__ FinishParams f) {
  const ScanParams& p = f.scan;
  extern __shared__ __align__(16) unsigned char slabs[];
  __shared__ uint32_t block_nulls[kMaxOut];
  for (int c = threadIdx.x; c < kMaxOut; c += blockDim.x) block_nulls[c] = 0;
  __syncthreads();
  const uint32_t G = f.groups[0];
  const uint64_t handed = records_handed_out(p);
  const uint32_t R = (uint32_t)p.rec_stride;  // a multiple of 16
  const uint32_t slot = R + 8;
  const uint32_t chunks = R / 16;  // 16-byte pieces per record
  const uint32_t pieces = 32 * chunks;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t gwarp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char* slab = slabs + (size_t)(threadIdx.x >> 5) * 32 * slot;
  for (uint64_t wbase = gwarp * 32; wbase < G; wbase += warps * 32) {
    const uint64_t i = wbase + lane;
    bool active = i < G;
    const uint32_t gid = active ? f.perm[i] : 0u;
    // The identity record (no group seen, no keys) finishes from zeros.
    const bool identity = active && gid == kIdentityRecord && p.n_keys == 0;
    if (active && !identity && gid >= handed) {
      atomicOr(p.status + 2, CHK_PERM);
      active = false;
    }
    const bool fetch = active && !identity;
    for (uint32_t base = 0; base < pieces; base += 128) {
      uint4 v[4];
      uint32_t at[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t idx = base + (uint32_t)k * 32 + (uint32_t)lane;
        const uint32_t j = idx / chunks, c = idx - j * chunks;
        const uint32_t g = __shfl_sync(0xffffffffu, gid, (int)(j & 31));
        const bool want = __shfl_sync(0xffffffffu, fetch, (int)(j & 31));
        at[k] = idx < pieces ? j * slot + c * 16 : 0xFFFFFFFFu;
        v[k] = make_uint4(0u, 0u, 0u, 0u);
        if (idx < pieces && want) v[k] = __ldg(reinterpret_cast<const uint4*>(record_at(p, g) + (size_t)c * 16));
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (at[k] == 0xFFFFFFFFu) continue;
        uint2* d = reinterpret_cast<uint2*>(slab + at[k]);
        d[0] = make_uint2(v[k].x, v[k].y);
        d[1] = make_uint2(v[k].z, v[k].w);
      }
    }
    __syncwarp();
    const unsigned char* rec = slab + (size_t)lane * slot;
    for (int c = 0; c < f.n_out; ++c) {
      const OutCol& oc = f.out[c];
      bool ok = false;
      uint64_t b = 0;
      if (active) b = output_cell(f, oc, rec, &ok);
      if (active) store_bits(oc.values, oc.dtype, i, b);
      const uint32_t bits = __ballot_sync(0xffffffffu, active && ok);
      if (lane == 0) {
        oc.validity[wbase >> 5] = bits;
        const uint32_t want = (G - wbase >= 32) ? 0xffffffffu : ((1u << (G - wbase)) - 1u);
        if (bits != want) block_nulls[c] = 1u;
      }
    }
    __syncwarp();  // the slab is refilled next
  }
  __syncthreads();
  for (int c = threadIdx.x; c < f.n_out; c += blockDim.x)
    if (block_nulls[c]) atomicOr(&f.has_nulls[c], 1u);
}

}  // namespace dfc

