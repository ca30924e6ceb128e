// column.cu — device side of the column handoff: validity normalisation and
// value ranges of resident columns.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dfc_device.cuh"
#include "dfc_internal.h"
#include "kernels.h"

namespace dfc {

// Normalises an Arrow LSB-first bitmap window starting at bit `off` into
// 32-bit words from bit 0 (bits past `rows` cleared) and counts valid rows.
// `nbytes` bounds the source: ceil((off + rows) / 8).
__global__ void normalize_validity(const uint8_t* src, uint64_t nbytes, uint64_t off, uint64_t rows, uint32_t* dst,
                                   unsigned long long* valid_rows) {
  const uint64_t words = (rows + 31) / 32;
  unsigned long long local = 0;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t bit = off + w * 32;
    const uint64_t b0 = bit >> 3;
    uint64_t window = 0;
    for (int k = 0; k < 5; ++k)
      if (b0 + k < nbytes) window |= (uint64_t)src[b0 + k] << (8 * k);
    uint32_t out = (uint32_t)(window >> (bit & 7));
    const uint64_t left = rows - w * 32;
    if (left < 32) out &= (1u << left) - 1u;
    dst[w] = out;
    local += __popc(out);
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(valid_rows, local);
}

// One HyperLogLog update: register = the hash's top kHllBits bits, value =
// the position of the first set bit of the rest.
__device__ __forceinline__ void hll_add(uint32_t* local, uint64_t h) {
  const uint32_t reg = (uint32_t)(h >> (64 - kHllBits));
  const uint64_t rest = h << kHllBits;
  const uint32_t rho = rest == 0 ? (65 - kHllBits) : (uint32_t)__clzll(rest) + 1;
  if (rho > local[reg]) atomicMax(&local[reg], rho);
}

// The rows of column_stats for one column type: DT is the dtype, U the
// unsigned integer of its size, so that every per-row dtype test folds away.
template <int DT, typename U>
__device__ __forceinline__ void stats_rows(const DevColumn& c, uint64_t rows, uint32_t* local, unsigned long long& lo,
                                           unsigned long long& hi) {
  constexpr bool kFloat = DT == DFC_FLOAT32 || DT == DFC_FLOAT64;
  const U* vals = static_cast<const U*>(c.values);
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base < rows; base += step * kStatsUnroll) {
    uint64_t b[kStatsUnroll];
    bool ok[kStatsUnroll];
#pragma unroll
    for (int j = 0; j < kStatsUnroll; ++j) {
      const uint64_t i = base + j * step;
      ok[j] = i < rows && (!c.validity || bit_valid(c.validity, i));
      b[j] = ok[j] ? (uint64_t)vals[i] : 0ull;
    }
#pragma unroll
    for (int j = 0; j < kStatsUnroll; ++j) {
      if (!ok[j]) continue;
      hll_add(local, mix64(key_cell(b[j], DT) ^ 0xD6E8FEB86659FD93ull));
      if (kFloat) {
        const double d = bits_to_f64(b[j], DT);
        if (d != d) continue;
      }
      const uint64_t e = order_encode(b[j], DT);
      lo = e < lo ? e : lo;
      hi = e > hi ? e : hi;
    }
  }
}

// Statistics of a column in one pass: the order-encoded minimum and maximum
// of its valid values (mm[0] = min, mm[1] = max; NaN skipped), which bound a
// key's domain when the planner sizes the group table, and the HyperLogLog
// sketch (2^kHllBits registers) of its distinct valid values under group
// equality (floats canonical).  Each thread loads kStatsUnroll rows, a grid
// stride apart, before it uses any of them, so that enough loads are in
// flight to stream the column at HBM rate; each block keeps its registers in
// shared memory and merges them into `regs` with atomicMax.
__global__ void column_stats(DevColumn c, uint64_t rows, unsigned long long* mm, uint32_t* regs) {
  __shared__ uint32_t local[1u << kHllBits];
  for (uint32_t i = threadIdx.x; i < (1u << kHllBits); i += blockDim.x) local[i] = 0;
  __syncthreads();
  unsigned long long lo = ~0ull, hi = 0ull;
  switch (c.dtype) {
    case DFC_INT8: stats_rows<DFC_INT8, uint8_t>(c, rows, local, lo, hi); break;
    case DFC_INT16: stats_rows<DFC_INT16, uint16_t>(c, rows, local, lo, hi); break;
    case DFC_INT32: stats_rows<DFC_INT32, uint32_t>(c, rows, local, lo, hi); break;
    case DFC_INT64: stats_rows<DFC_INT64, uint64_t>(c, rows, local, lo, hi); break;
    case DFC_UINT8: stats_rows<DFC_UINT8, uint8_t>(c, rows, local, lo, hi); break;
    case DFC_UINT16: stats_rows<DFC_UINT16, uint16_t>(c, rows, local, lo, hi); break;
    case DFC_UINT32: stats_rows<DFC_UINT32, uint32_t>(c, rows, local, lo, hi); break;
    case DFC_UINT64: stats_rows<DFC_UINT64, uint64_t>(c, rows, local, lo, hi); break;
    case DFC_FLOAT32: stats_rows<DFC_FLOAT32, uint32_t>(c, rows, local, lo, hi); break;
    case DFC_FLOAT64: stats_rows<DFC_FLOAT64, uint64_t>(c, rows, local, lo, hi); break;
    default: break;  // the host registers only the types above
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < (1u << kHllBits); i += blockDim.x)
    if (local[i]) atomicMax(&regs[i], local[i]);
}

// HyperLogLog registers of the query's key words over all rows: the packed
// key word (keys <= 64 bits) or the 64-bit key hash, both as the scan forms
// them.  The group count of a multi-key query is estimated from these
// directly instead of from the product of the columns' distinct counts.
// The query's key word of row i (packed keys) or its 64-bit key hash (ticket
// keys), as the scan forms them.
__device__ __forceinline__ uint64_t query_key_word(const ScanParams& p, uint64_t i) {
  const bool packed = p.key_mode == KEY_PACKED;
  uint64_t kw = packed ? 0ull : 0x243F6A8885A308D3ull;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    const DevColumn& c = p.cols[f.input];
    const bool ok = !c.validity || bit_valid(c.validity, i);
    const uint64_t cell = ok ? key_cell(load_bits(c.values, c.size, i), f.dtype) : 0ull;
    if (packed) {
      if (!ok) kw |= 1ull << f.null_bit;
      else kw |= (f.bits == 64) ? cell : (cell << f.shift);
    } else {
      const uint64_t v = ok ? cell + 1 : 0x9E3779B97F4A7C15ull;
      kw = mix64(kw ^ (v * 0x9E3779B97F4A7C15ull + (uint64_t)k));
    }
  }
  return kw;
}

// Rows are loaded kKeysUnroll at a time per thread (all key columns of
// each) before any register update, as in column_stats.
__global__ void keys_hll(const __grid_constant__ ScanParams p, uint32_t* regs) {
  __shared__ uint32_t local[1u << kHllBits];
  for (uint32_t i = threadIdx.x; i < (1u << kHllBits); i += blockDim.x) local[i] = 0;
  __syncthreads();
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base < p.rows; base += step * kKeysUnroll) {
    uint64_t kw[kKeysUnroll];
#pragma unroll
    for (int j = 0; j < kKeysUnroll; ++j) {
      const uint64_t i = base + j * step;
      kw[j] = i < p.rows ? query_key_word(p, i) : 0ull;
    }
#pragma unroll
    for (int j = 0; j < kKeysUnroll; ++j)
      if (base + j * step < p.rows) hll_add(local, mix64(kw[j] ^ 0xD6E8FEB86659FD93ull));
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < (1u << kHllBits); i += blockDim.x)
    if (local[i]) atomicMax(&regs[i], local[i]);
}

// Key words of the rows i * stride, i < n (a sample for the planner's skew
// estimate); the caller keeps (n - 1) * stride below the row count.
__global__ void keys_sample(const __grid_constant__ ScanParams p, unsigned long long* out, uint32_t n, uint64_t stride) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = query_key_word(p, (uint64_t)i * stride);
}

}  // namespace dfc
