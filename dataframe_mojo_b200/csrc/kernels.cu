// kernels.cu — the filtered hash group-by on sm_100a.
//
// scan_kernel: one pass over the rows.  A producer warp streams each tile of
// every column the query touches (values + validity words) into a ring of
// shared-memory stages with 1-D TMA bulk copies (cp.async.bulk, no multicast)
// completing on mbarriers; consumer warps evaluate the filter program, pack the
// key, probe the global open-addressing key table (claims by 128-bit CAS that
// publish key and group id together) and fold the row into its group record
// with fire-and-forget atomics.  The group semantics restate
// dataframe/aggregation/function.mojo:1143-1236 (`_scatter`) for a table all
// workers share: integer sums exact in 128 bits, FP64 sums, min/max with the
// NaN flag and first-zero sign, and the second moment as a shifted sum of
// squares (K = the first value the group saw), finished into M2 = S2 - S1^2/n.
//
// finish kernels: groups ranked by first selected row through a row bitmap and
// its popcount prefix (first-appearance order of maintain_order=True,
// dataframe/aggregation/state.mojo:267-330), then every output column written
// in that order with its validity bitmap (function.mojo:2516-2918,
// reducer.mojo:3391-3599).
#include <cuda_runtime.h>
#include <stdint.h>

#include "dfc_device.cuh"
#include "dfc_internal.h"
#include "kernels.h"

namespace dfc {

constexpr uint32_t kWaitLimit = 1u << 22;   // try_wait polls before a stage wait gives up
constexpr uint32_t kSpinLimit = 1u << 20;   // re-reads of a key entry before giving up
constexpr uint32_t kNoGid = 0xFFFFFFFFu;

// Where one tile's column data is: a shared-memory stage, or global memory
// for the ragged last tile.
struct TileView {
  const unsigned char* vals[kMaxInputs];
  const uint32_t* valid[kMaxInputs];
};

__device__ __forceinline__ bool view_valid(const TileView& v, int c, uint32_t r) {
  const uint32_t* w = v.valid[c];
  return w == nullptr || ((w[r >> 5] >> (r & 31)) & 1u);
}

__device__ __forceinline__ uint64_t view_bits(const ScanParams& p, const TileView& v, int c, uint32_t r) {
  return load_bits(v.vals[c], p.cols[c].size, r);
}

// ---------------------------------------------------------------------------
// Filter program (postfix, Kleene): value and known bits kept as two stacks
// packed in registers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool cmp_i64(int op, int64_t a, int64_t b) {
  switch (op) {
    case DFC_LT: return a < b;
    case DFC_LE: return a <= b;
    case DFC_GT: return a > b;
    case DFC_GE: return a >= b;
    case DFC_EQ: return a == b;
    default: return a != b;
  }
}
__device__ __forceinline__ bool cmp_u64(int op, uint64_t a, uint64_t b) {
  switch (op) {
    case DFC_LT: return a < b;
    case DFC_LE: return a <= b;
    case DFC_GT: return a > b;
    case DFC_GE: return a >= b;
    case DFC_EQ: return a == b;
    default: return a != b;
  }
}
template <typename F>
__device__ __forceinline__ bool cmp_f(int op, F a, F b) {
  switch (op) {
    case DFC_LT: return a < b;
    case DFC_LE: return a <= b;
    case DFC_GT: return a > b;
    case DFC_GE: return a >= b;
    case DFC_EQ: return a == b;
    default: return !(a == b);
  }
}

__device__ __forceinline__ bool eval_filter(const ScanParams& p, const TileView& v, uint32_t r) {
  if (p.n_pred == 0) return true;
  uint32_t sv = 0, sk = 0;
  for (int i = 0; i < p.n_pred; ++i) {
    const PredOp& op = p.pred[i];
    switch (op.kind) {
      case DFC_PRED_CMP: {
        int c = op.input;
        bool known = view_valid(v, c, r);
        bool val = false;
        if (known) {
          uint64_t b = view_bits(p, v, c, r);
          int dt = p.cols[c].dtype;
          if (dt == DFC_FLOAT64) val = cmp_f<double>(op.cmp, bits_to_f64(b, dt), op.lit.f);
          else if (dt == DFC_FLOAT32) val = cmp_f<float>(op.cmp, __uint_as_float((uint32_t)b), (float)op.lit.f);
          else if (dt == DFC_UINT64) val = cmp_u64(op.cmp, b, op.lit.u);
          else val = cmp_i64(op.cmp, bits_to_i64(b, dt), op.lit.i);
        }
        sv = (sv << 1) | (uint32_t)val;
        sk = (sk << 1) | (uint32_t)known;
        break;
      }
      case DFC_PRED_IS_NULL:
        sv = (sv << 1) | (uint32_t)(!view_valid(v, op.input, r));
        sk = (sk << 1) | 1u;
        break;
      case DFC_PRED_IS_NOT_NULL:
        sv = (sv << 1) | (uint32_t)view_valid(v, op.input, r);
        sk = (sk << 1) | 1u;
        break;
      case DFC_PRED_TRUE:
        sv = (sv << 1) | 1u;
        sk = (sk << 1) | 1u;
        break;
      case DFC_PRED_NOT:
        sv ^= 1u;
        break;
      case DFC_PRED_AND: {
        uint32_t bv = sv & 1u, bk = sk & 1u;
        sv >>= 1;
        sk >>= 1;
        uint32_t av = sv & 1u, ak = sk & 1u;
        uint32_t false_known = (ak & (av ^ 1u)) | (bk & (bv ^ 1u));
        uint32_t rv = (false_known ^ 1u) & ak & bk & av & bv;
        uint32_t rk = false_known | (ak & bk);
        sv = (sv & ~1u) | rv;
        sk = (sk & ~1u) | rk;
        break;
      }
      case DFC_PRED_OR: {
        uint32_t bv = sv & 1u, bk = sk & 1u;
        sv >>= 1;
        sk >>= 1;
        uint32_t av = sv & 1u, ak = sk & 1u;
        uint32_t true_known = (ak & av) | (bk & bv);
        uint32_t rk = true_known | (ak & bk);
        sv = (sv & ~1u) | true_known;
        sk = (sk & ~1u) | rk;
        break;
      }
    }
  }
  return (sv & sk & 1u) != 0;
}

// ---------------------------------------------------------------------------
// Keys.
// ---------------------------------------------------------------------------
// Packed mode: every key column's bits (and null flags) side by side in one
// 64-bit word, compared exactly.  Ticket mode: the word is a 64-bit hash and
// equality is checked on the key columns at the row that claimed the group.
__device__ __forceinline__ uint64_t key_word(const ScanParams& p, const TileView& v, uint32_t r) {
  if (p.key_mode == KEY_PACKED) {
    uint64_t kw = 0;
    for (int k = 0; k < p.n_keys; ++k) {
      const KeyField& f = p.keys[k];
      if (f.null_bit >= 0 && !view_valid(v, f.input, r)) {
        kw |= 1ull << f.null_bit;
      } else {
        uint64_t cell = key_cell(view_bits(p, v, f.input, r), f.dtype);
        kw |= (f.bits == 64) ? cell : (cell << f.shift);
      }
    }
    return kw;
  }
  uint64_t h = 0x243F6A8885A308D3ull;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    uint64_t cell = view_valid(v, f.input, r) ? key_cell(view_bits(p, v, f.input, r), f.dtype) + 1
                                              : 0x9E3779B97F4A7C15ull;
    h = mix64(h ^ (cell * 0x9E3779B97F4A7C15ull + (uint64_t)k));
  }
  return h == kEmpty ? kEmpty - 1 : h;
}

// Ticket mode: key columns of global rows a and b equal under group equality.
__device__ __forceinline__ bool rows_key_equal(const ScanParams& p, uint64_t a, uint64_t b) {
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    const DevColumn& c = p.cols[f.input];
    bool va = c.validity == nullptr || bit_valid(c.validity, a);
    bool vb = c.validity == nullptr || bit_valid(c.validity, b);
    if (va != vb) return false;
    if (va && key_cell(load_bits(c.values, c.size, a), f.dtype) != key_cell(load_bits(c.values, c.size, b), f.dtype))
      return false;
  }
  return true;
}

__device__ __forceinline__ unsigned char* record_at(const ScanParams& p, uint32_t gid) {
  return p.records + (size_t)gid * (size_t)p.rec_stride;
}

// Writes a fresh record: the identity template, then key and rows.
__device__ __forceinline__ void init_record(const ScanParams& p, unsigned char* rec, uint64_t kw, uint32_t row) {
  const uint4* src = reinterpret_cast<const uint4*>(p.rec_template);
  uint4* dst = reinterpret_cast<uint4*>(rec);
  for (int i = 0; i < p.rec_words / 2; ++i) dst[i] = src[i];
  *reinterpret_cast<unsigned long long*>(rec + kRecKey) = kw;
  *reinterpret_cast<uint32_t*>(rec + kRecFirst) = row;
  *reinterpret_cast<uint32_t*>(rec + kRecClaim) = row;
}

// Record numbers are handed out by CTA tickets: ticket t falls in the CTA's
// chunk k = t / chunk, whose base the holder of the chunk's first ticket draws
// from the global counter and publishes (tagged with k) in a small ring.
constexpr int kChunkRing = 64;

struct ClaimState {
  uint32_t ticket;
  unsigned long long ring[kChunkRing];
};

// Reserves a record for a claim attempt.  kNoGid when the records ran out.
__device__ __forceinline__ uint32_t reserve_record(const ScanParams& p, ClaimState* cs) {
  const uint32_t t = atomicAdd(&cs->ticket, 1u);
  const uint32_t k = t / p.chunk, off = t % p.chunk;
  volatile unsigned long long* slot = &cs->ring[k % kChunkRing];
  if (off == 0) {
    const uint32_t base = atomicAdd(p.alloc, p.chunk);
    *slot = ((unsigned long long)k << 32) | base;
  }
  unsigned long long e = *slot;
  for (uint32_t i = 0; (uint32_t)(e >> 32) != k; ++i) {
    if (i == kSpinLimit) {
      atomicOr(p.status, ST_TIMEOUT);
      return kNoGid;
    }
    e = *slot;
  }
  const uint32_t base = (uint32_t)e;
  if (base >= p.recs_total || off >= p.recs_total - base) {
    atomicOr(p.status, ST_CAPACITY);
    return kNoGid;
  }
  return base + off;
}

// At CTA exit: the unused tail of the CTA's last chunk becomes holes.
__device__ __forceinline__ void retire_chunk(const ScanParams& p, ClaimState* cs) {
  const uint32_t t = cs->ticket;
  if (t % p.chunk == 0) return;
  const uint32_t k = t / p.chunk;
  const unsigned long long e = cs->ring[k % kChunkRing];
  if ((uint32_t)(e >> 32) != k) return;
  const uint32_t base = (uint32_t)e;
  for (uint32_t off = t % p.chunk + threadIdx.x; off < p.chunk; off += blockDim.x) {
    if (base < p.recs_total && off < p.recs_total - base)
      *reinterpret_cast<uint32_t*>(p.records + (size_t)(base + off) * p.rec_stride + kRecFirst) = kNoRow;
  }
}

// Re-reads an entry until its meta word is published (a claim publishes key
// and meta in one 128-bit CAS, so this only spins on a torn read).
__device__ __forceinline__ uint64_t entry_meta(const ScanParams& p, KeyEntry* e) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    uint64_t m = ld_cg_u64(&e->meta);
    if (m != kEmpty) return m;
  }
  atomicOr(p.status, ST_TIMEOUT);
  return kEmpty;
}

// Finds the group of key word kw (row `row`), claiming a new one if needed.
__device__ uint32_t find_or_claim(const ScanParams& p, uint64_t kw, uint32_t row, ClaimState* cs) {
  const uint64_t slots = p.table_mask + 1;
  if (kw == kEmpty) {
    // The all-ones key has its own entry after the table.
    KeyEntry* e = p.table + slots;
    uint64_t m = ld_cg_u64(&e->meta);
    if (m != kEmpty) return (uint32_t)m;
    uint32_t gid = reserve_record(p, cs);
    if (gid == kNoGid) return kNoGid;
    unsigned char* rec = record_at(p, gid);
    init_record(p, rec, kw, row);
    __threadfence();
    uint64_t ok, om;
    cas128(e, kEmpty, kEmpty, kEmpty, (uint64_t)gid | ((uint64_t)row << 32), ok, om);
    if (om == kEmpty) return gid;
    *reinterpret_cast<uint32_t*>(rec + kRecFirst) = kNoRow;  // lost the race: a hole
    return (uint32_t)om;
  }
  uint64_t slot = mix64(kw ^ 0x632BE59BD9B4E019ull) & p.table_mask;
  uint32_t gid_reserved = kNoGid;
  for (uint64_t probe = 0; probe < slots; ++probe) {
    KeyEntry* e = p.table + slot;
    uint64_t k = ld_cg_u64(&e->key);
    if (k == kw) {
      uint64_t m = entry_meta(p, e);
      if (m == kEmpty) break;
      if (p.key_mode == KEY_PACKED || rows_key_equal(p, row, (uint32_t)(m >> 32))) {
        if (gid_reserved != kNoGid) *reinterpret_cast<uint32_t*>(record_at(p, gid_reserved) + kRecFirst) = kNoRow;
        return (uint32_t)m;
      }
    } else if (k == kEmpty) {
      if (gid_reserved == kNoGid) {
        gid_reserved = reserve_record(p, cs);
        if (gid_reserved == kNoGid) return kNoGid;
        init_record(p, record_at(p, gid_reserved), kw, row);
        __threadfence();
      }
      uint64_t ok, om;
      cas128(e, kEmpty, kEmpty, kw, (uint64_t)gid_reserved | ((uint64_t)row << 32), ok, om);
      if (ok == kEmpty && om == kEmpty) return gid_reserved;
      if (ok == kw && (p.key_mode == KEY_PACKED || rows_key_equal(p, row, (uint32_t)(om >> 32)))) {
        *reinterpret_cast<uint32_t*>(record_at(p, gid_reserved) + kRecFirst) = kNoRow;
        return (uint32_t)om;
      }
    }
    slot = (slot + 1) & p.table_mask;
  }
  if (gid_reserved != kNoGid) *reinterpret_cast<uint32_t*>(record_at(p, gid_reserved) + kRecFirst) = kNoRow;
  atomicOr(p.status, ST_CAPACITY);
  return kNoGid;
}

// Folds one selected row into its group record.
__device__ __forceinline__ void update_record(const ScanParams& p, unsigned char* rec, const TileView& v, uint32_t r,
                                              uint32_t row) {
  if (p.track_first) red_min_u32(rec + kRecFirst, row);
  if (p.track_len) red_add_u32(rec + kRecLen, 1u);
  for (int j = 0; j < p.n_vals; ++j) {
    const ValField& f = p.vals[j];
    const int c = f.input;
    if (!view_valid(v, c, r)) continue;
    const int dt = f.dtype;
    const uint64_t b = view_bits(p, v, c, r);
    red_add_u32(rec + f.off_count, 1u);
    const bool isf = dt_float(dt);
    const double xd = isf ? bits_to_f64(b, dt) : 0.0;
    const bool nan = isf && (xd != xd);
    if (f.off_sum >= 0) {
      if (f.sum_kind == SUM_F64) {
        red_add_f64(rec + f.off_sum, xd);
      } else if (f.sum_kind == SUM_I64) {
        red_add_u64(rec + f.off_sum, (uint64_t)bits_to_i64(b, dt));
      } else {
        const bool uns = dt == DFC_UINT64;
        const uint64_t x = uns ? b : (uint64_t)bits_to_i64(b, dt);
        const uint64_t neg = (!uns && (int64_t)x < 0) ? ~0ull : 0ull;
        const uint64_t old = atomicAdd(reinterpret_cast<unsigned long long*>(rec + f.off_sum), x);
        const uint64_t carry = (old + x) < old ? 1ull : 0ull;
        const uint64_t hi = neg + carry;
        if (hi) red_add_u64(rec + f.off_sum + 8, hi);
      }
    }
    if (f.off_min >= 0 || f.off_max >= 0) {
      if (nan) {
        red_or_u32(rec + kRecFlags, 1u << f.nan_bit);
      } else {
        const uint64_t e = order_encode(b, dt);
        if (f.off_min >= 0) red_min_u64(rec + f.off_min, e);
        if (f.off_max >= 0) red_max_u64(rec + f.off_max, e);
        if (f.off_zero >= 0 && xd == 0.0)
          red_min_u64(rec + f.off_zero, ((uint64_t)row << 1) | (uint64_t)(__double_as_longlong(xd) < 0));
      }
    }
    if (f.off_m2 >= 0) {
      const double x = isf ? xd : bits_as_double(b, dt);
      const uint64_t xb = (x != x) ? kCanonNaN : (uint64_t)__double_as_longlong(x);
      uint64_t kb = ld_cg_u64(rec + f.off_shift);
      if (kb == kShiftUnset) {
        const uint64_t prev =
            atomicCAS(reinterpret_cast<unsigned long long*>(rec + f.off_shift), kShiftUnset, xb);
        kb = (prev == kShiftUnset) ? xb : prev;
      }
      const double d = x - __longlong_as_double((long long)kb);
      red_add_f64(rec + f.off_m2, d * d);
    }
  }
}

__device__ __forceinline__ void process_row(const ScanParams& p, const TileView& v, uint64_t tile_start, uint32_t r,
                                            ClaimState* cs) {
  if (!eval_filter(p, v, r)) return;
  const uint32_t row = (uint32_t)(tile_start + r);
  const uint64_t kw = key_word(p, v, r);
  const uint32_t gid = find_or_claim(p, kw, row, cs);
  if (gid == kNoGid) return;
  update_record(p, record_at(p, gid), v, r, row);
}

__global__ void __launch_bounds__(kScanThreads, 1) scan_kernel(const __grid_constant__ ScanParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
  uint64_t* empty = full + S;
  __shared__ ClaimState s_claim;
  __shared__ volatile uint32_t s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kScanConsumerWarps);
    }
    fence_mbar_init();
    s_claim.ticket = 0;
    s_abort = 0;
  }
  if (threadIdx.x < kChunkRing) s_claim.ring[threadIdx.x] = ~0ull;
  __syncthreads();

  const uint64_t T = (uint64_t)p.tile_rows;
  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (uint64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
        const uint32_t s = it % S, ph = (it / S) & 1u;
        if (it >= (uint32_t)S && !mbar_wait_bounded(&empty[s], ph ^ 1u, kWaitLimit)) {
          atomicOr(p.status, ST_TIMEOUT);
          s_abort = 1;
          break;
        }
        if (s_abort) break;
        if (p.use_tma && t < p.full_tiles) {
          unsigned char* stage = smem + (size_t)s * p.stage_bytes;
          mbar_arrive_expect_tx(&full[s], (uint32_t)p.stage_tx);
          for (int c = 0; c < p.n_stage; ++c) {
            const DevColumn& col = p.cols[c];
            bulk_g2s(stage + p.stage_off[c], static_cast<const unsigned char*>(col.values) + t * T * col.size,
                     (uint32_t)(T * col.size), &full[s]);
            if (p.stage_voff[c] >= 0)
              bulk_g2s(stage + p.stage_voff[c], col.validity + t * (T / 32), (uint32_t)(T / 8), &full[s]);
          }
        } else {
          mbar_arrive(&full[s]);
        }
      }
      // Every issued stage must have landed before the CTA may exit.
      if (s_abort) {
        uint32_t first = it > (uint32_t)S ? it - S : 0;
        for (uint32_t j = first; j < it; ++j) mbar_wait_bounded(&full[j % S], (j / S) & 1u, kWaitLimit);
      }
    }
  } else {
    const uint32_t ct = threadIdx.x - 32;
    uint32_t it = 0;
    TileView view;
    for (uint64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const uint32_t s = it % S, ph = (it / S) & 1u;
      if (!mbar_wait_bounded(&full[s], ph, kWaitLimit)) {
        atomicOr(p.status, ST_TIMEOUT);
        s_abort = 1;
        break;
      }
      const uint64_t start = t * T;
      if (p.use_tma && t < p.full_tiles) {
        const unsigned char* stage = smem + (size_t)s * p.stage_bytes;
        for (int c = 0; c < p.n_stage; ++c) {
          view.vals[c] = stage + p.stage_off[c];
          view.valid[c] = p.stage_voff[c] >= 0 ? reinterpret_cast<const uint32_t*>(stage + p.stage_voff[c]) : nullptr;
        }
      } else {
        for (int c = 0; c < p.n_stage; ++c) {
          const DevColumn& col = p.cols[c];
          view.vals[c] = static_cast<const unsigned char*>(col.values) + start * col.size;
          view.valid[c] = col.validity ? col.validity + start / 32 : nullptr;
        }
      }
      const uint64_t left = p.rows - start;
      const uint32_t n = (uint32_t)(left < T ? left : T);
      for (uint32_t r = ct; r < n; r += kScanConsumerThreads) process_row(p, view, start, r, &s_claim);
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (s_abort) break;
    }
  }
  __syncthreads();
  retire_chunk(p, &s_claim);
}

// ---------------------------------------------------------------------------
// Finish.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t records_handed_out(const ScanParams& p) {
  const uint32_t a = *p.alloc;
  return a < p.recs_total ? a : p.recs_total;
}

__device__ __forceinline__ bool live_record(const ScanParams& p, uint64_t i, uint32_t& first) {
  first = *reinterpret_cast<const uint32_t*>(record_at(p, (uint32_t)i) + kRecFirst);
  return first != kNoRow;
}

__global__ void finish_mark(const __grid_constant__ FinishParams f) {
  const ScanParams& p = f.scan;
  const uint64_t n = records_handed_out(p);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t first;
    if (live_record(p, i, first)) atomicOr(&f.order_bits[first >> 5], 1u << (first & 31));
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
    uint32_t first;
    if (!live_record(p, i, first)) continue;
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
      const uint32_t row = *reinterpret_cast<const uint32_t*>(rec + kRecFirst);
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
    case DFC_AGG_LEN: return *reinterpret_cast<const uint32_t*>(rec + kRecLen);
    case DFC_AGG_NULL_COUNT: return *reinterpret_cast<const uint32_t*>(rec + kRecLen) - count;
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
      const uint64_t e = *reinterpret_cast<const uint64_t*>(rec + (is_max ? vf.off_max : vf.off_min));
      bool seen;
      if (isf) seen = is_max ? (e != 0ull) : (e != ~0ull);
      else seen = count > 0;
      if (!seen) {
        const uint32_t flags = *reinterpret_cast<const uint32_t*>(rec + kRecFlags);
        if (isf && ((flags >> vf.nan_bit) & 1u)) return idt == DFC_FLOAT32 ? 0x7FC00000ull : kCanonNaN;
        *ok = false;
        return 0;
      }
      uint64_t b = order_decode(e, idt);
      if (isf && vf.off_zero >= 0) {
        const bool zero = idt == DFC_FLOAT32 ? ((uint32_t)b & 0x7FFFFFFFu) == 0 : (b & 0x7FFFFFFFFFFFFFFFull) == 0;
        if (zero) {
          const uint64_t z = *reinterpret_cast<const uint64_t*>(rec + vf.off_zero);
          const bool neg = (z & 1ull) != 0;
          b = idt == DFC_FLOAT32 ? (neg ? 0x80000000ull : 0ull) : (neg ? 0x8000000000000000ull : 0ull);
        }
      }
      return b;
    }
    case DFC_AGG_VAR:
    case DFC_AGG_STD: {
      const int64_t n = (int64_t)count;
      *ok = n - (int64_t)oc.ddof > 0;
      if (!*ok) return 0;
      const double K = *reinterpret_cast<const double*>(rec + vf.off_shift);
      const double S2 = *reinterpret_cast<const double*>(rec + vf.off_m2);
      double S1;
      if (isf) {
        S1 = *reinterpret_cast<const double*>(rec + vf.off_sum) - (double)n * K;
      } else {
        S1 = (double)(int_sum(vf, rec) - (__int128)n * (__int128)K);
      }
      double M2 = S2 - S1 * (S1 / (double)n);
      if (M2 < 0.0) M2 = 0.0;
      // Conditioning: results the reference CPU's Welford recurrence cannot
      // reproduce within 1e-10 (a mean far from zero relative to the spread),
      // or that cancel too much here, are handed back as a data fault.
      const double mean = K + S1 / (double)n;
      const double var_pop = M2 / (double)n;
      if (S2 == S2 && mean == mean && n >= 2) {
        const bool far_mean = fabs(mean) > 1.0e6 * sqrt(var_pop);
        const bool cancels = S2 > 1.0e4 * M2;
        if ((far_mean && mean != 0.0 && (M2 > 0.0 || S2 > 0.0)) || (cancels && S2 > 0.0)) {
          atomicOr(p.status, ST_FAULT);
        }
      }
      const double var = M2 / (double)(n - (int64_t)oc.ddof);
      const double out = oc.op == DFC_AGG_STD ? sqrt(var) : var;
      return (uint64_t)__double_as_longlong(out);
    }
  }
  *ok = false;
  return 0;
}

__global__ void finish_output(const __grid_constant__ FinishParams f) {
  const ScanParams& p = f.scan;
  const uint32_t G = f.groups[0];
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t gwarp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (uint64_t wbase = gwarp * 32; wbase < G; wbase += warps * 32) {
    const uint64_t i = wbase + lane;
    const bool active = i < G;
    const unsigned char* rec = active ? record_at(p, f.perm[i]) : nullptr;
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
        if (bits != want) atomicOr(&f.has_nulls[c], 1u);
      }
    }
  }
}

}  // namespace dfc

// ---------------------------------------------------------------------------
// Column handoff helpers.
// ---------------------------------------------------------------------------
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

// Order-encoded minimum and maximum of the valid values of a column
// (out[0] = min, out[1] = max; NaN skipped).  Used to bound key domains.
__global__ void column_minmax(DevColumn c, uint64_t rows, unsigned long long* out) {
  unsigned long long lo = ~0ull, hi = 0ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < rows; i += (uint64_t)gridDim.x * blockDim.x) {
    if (c.validity && !bit_valid(c.validity, i)) continue;
    const uint64_t b = load_bits(c.values, c.size, i);
    if (dt_float(c.dtype)) {
      const double d = bits_to_f64(b, c.dtype);
      if (d != d) continue;
    }
    const uint64_t e = order_encode(b, c.dtype);
    lo = e < lo ? e : lo;
    hi = e > hi ? e : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = a < lo ? a : lo;
    hi = b > hi ? b : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], lo);
    atomicMax(&out[1], hi);
  }
}

}  // namespace dfc
