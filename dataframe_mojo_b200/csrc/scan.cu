// scan.cu — the fused filter + key + aggregate pass of the filtered hash
// group-by on sm_100a.
//
// One persistent CTA per SM slot.  Warp 0 is the producer: for every tile of
// `tile_rows` rows it streams each column the query touches (values and
// validity words) into a ring of shared-memory stages with 1-D TMA bulk
// copies (cp.async.bulk, no multicast) that complete on mbarriers.  The other
// eight warps consume two tiles per step, column at a time:
//   1. selection: the filter program per row, one warp ballot per 32 rows;
//   2. compaction: the selected rows' indices, densely, in shared memory, so
//      every lane of the later phases holds a selected row;
//   3. keys: each key column packed into the rows' key words (packed mode) or
//      hashed (ticket mode);
//   4. groups: with few groups a CTA-local shared-memory table, duplicate keys
//      of a warp collapsed with __match_any_sync into one leader update;
//      with up to 32K groups the CTAs of a cluster pool their shared memory
//      into one table; otherwise the global open-addressing table, probed
//      two entries per round in warp-synchronous rounds, a new group claimed
//      by a CAS of its key word, then its record published in the entry;
//   5. states: each aggregated column's read-set (first row, K, min, max) for
//      all rows, then fire-and-forget atomics (counts, sums, the shifted
//      square sum; first row / min / max only when the row improves them).
// Type dispatch happens once per column per step, outside the row loops.
// Group records start all-zero (stream-ordered memset), so a claim needs no
// initialisation and no fence: first row is stored as ~row, the minimum as
// ~code (both raised by atomicMax), K xor a tag (0 = unset).
// Semantics restated from dataframe/aggregation/function.mojo:1143-1236
// (`_scatter`) and :1559-1779 (`combine`): integer sums exact in 128 bits,
// FP64 float sums, min/max skip NaN (flag) and keep the earlier value on
// ties, moments from shifted sums (finished into M2 = S2 - S1^2/n, the
// mergeable equivalent of the reference's Welford state,
// dataframe/aggregation/scalar_states.mojo:104-145).
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "dfc_device.cuh"
#include "dfc_internal.h"
#include "kernels.h"

namespace dfc {

constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait polls before a stage wait gives up
constexpr uint32_t kSpinLimit = 1u << 20;  // re-reads before a publication wait gives up
constexpr uint32_t kNoGid = 0xFFFFFFFFu;
constexpr int kR = kScanRowsPerThread;                  // rows a thread holds per pass
constexpr int kTilesPerStep = 2;                         // tiles a consumer step covers
constexpr int kMaxTileRows = 1024;
constexpr int kStepRows = kTilesPerStep * kMaxTileRows;  // compacted rows at most per step
constexpr int kPassRows = kScanConsumerThreads * kR;     // compacted rows per pass

// Barrier of the consumer warps only (named barrier 1); returns whether any
// of them passed `flag`, so every consumer warp takes the same decision.
__device__ __forceinline__ bool consumer_sync_or(bool flag) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)flag), "n"(kScanConsumerThreads)
      : "memory");
  return out != 0;
}

// The tiles of one consumer step: each in a shared-memory stage or, for the
// ragged last tile, in global memory.
struct Step {
  const unsigned char* stage[kTilesPerStep];
  uint64_t start[kTilesPerStep];
  bool staged[kTilesPerStep];
  uint32_t n[kTilesPerStep];  // rows of each tile (0: absent)
};

__device__ __forceinline__ const unsigned char* col_values(const ScanParams& p, const Step& s, int tile, int c) {
  return s.staged[tile] ? s.stage[tile] + p.stage_off[c]
                        : static_cast<const unsigned char*>(p.cols[c].values) + s.start[tile] * (uint64_t)p.cols[c].size;
}

__device__ __forceinline__ const uint32_t* col_valid(const ScanParams& p, const Step& s, int tile, int c) {
  if (s.staged[tile])
    return p.stage_voff[c] >= 0 ? reinterpret_cast<const uint32_t*>(s.stage[tile] + p.stage_voff[c]) : nullptr;
  return p.cols[c].validity ? p.cols[c].validity + s.start[tile] / 32 : nullptr;
}

__device__ __forceinline__ bool valid_at(const uint32_t* w, uint32_t r) {
  return w == nullptr || ((w[r >> 5] >> (r & 31)) & 1u);
}

__device__ __forceinline__ unsigned char* record_at(const ScanParams& p, uint32_t gid) {
  return p.records + (size_t)gid * (size_t)p.rec_stride;
}

template <typename T>
__device__ __forceinline__ T load_as(const unsigned char* base, uint32_t r) {
  return reinterpret_cast<const T*>(base)[r];
}

// A row of the step: tile index and row inside the tile.
struct RowRef {
  uint32_t tile;
  uint32_t r;
  bool on;
};

// Per-column pointers of the step, resolved once per column.
struct ColRef {
  const unsigned char* vals[kTilesPerStep];
  const uint32_t* valid[kTilesPerStep];
};

__device__ __forceinline__ ColRef col_ref(const ScanParams& p, const Step& s, int c) {
  ColRef cr;
#pragma unroll
  for (int t = 0; t < kTilesPerStep; ++t) {
    cr.vals[t] = col_values(p, s, t, c);
    cr.valid[t] = col_valid(p, s, t, c);
  }
  return cr;
}

__device__ __forceinline__ const unsigned char* rv(const ColRef& cr, const RowRef& x) {
  return x.tile ? cr.vals[1] : cr.vals[0];
}
__device__ __forceinline__ bool rvalid(const ColRef& cr, const RowRef& x) {
  return valid_at(x.tile ? cr.valid[1] : cr.valid[0], x.r);
}

// ---------------------------------------------------------------------------
// 1. Selection.
// ---------------------------------------------------------------------------
template <typename F>
__device__ __forceinline__ bool cmp_op(int op, F a, F b) {
  switch (op) {
    case DFC_LT: return a < b;
    case DFC_LE: return a <= b;
    case DFC_GT: return a > b;
    case DFC_GE: return a >= b;
    case DFC_EQ: return a == b;
    default: return !(a == b);
  }
}

// One comparison on a row (known = not null).
__device__ __forceinline__ bool cmp_row(const PredOp& op, int dt, int size, const unsigned char* vals, uint32_t r) {
  const uint64_t b = load_bits(vals, size, r);
  if (dt == DFC_FLOAT64) return cmp_op<double>(op.cmp, __longlong_as_double((long long)b), op.lit.f);
  if (dt == DFC_FLOAT32) return cmp_op<float>(op.cmp, __uint_as_float((uint32_t)b), (float)op.lit.f);
  if (dt == DFC_UINT64) return cmp_op<uint64_t>(op.cmp, b, op.lit.u);
  return cmp_op<int64_t>(op.cmp, bits_to_i64(b, dt), op.lit.i);
}

// The general filter program for one row: value and known bits as two
// register stacks (postfix, Kleene logic).
__device__ bool program_row(const ScanParams& p, const Step& s, int tile, uint32_t r) {
  uint32_t sv = 0, sk = 0;
  for (int i = 0; i < p.n_pred; ++i) {
    const PredOp& op = p.pred[i];
    switch (op.kind) {
      case DFC_PRED_CMP: {
        const int c = op.input;
        const bool known = valid_at(col_valid(p, s, tile, c), r);
        const bool v = known && cmp_row(op, p.cols[c].dtype, p.cols[c].size, col_values(p, s, tile, c), r);
        sv = (sv << 1) | (uint32_t)v;
        sk = (sk << 1) | (uint32_t)known;
        break;
      }
      case DFC_PRED_IS_NULL:
      case DFC_PRED_IS_NOT_NULL: {
        const bool is_valid = valid_at(col_valid(p, s, tile, op.input), r);
        sv = (sv << 1) | (uint32_t)(op.kind == DFC_PRED_IS_NULL ? !is_valid : is_valid);
        sk = (sk << 1) | 1u;
        break;
      }
      case DFC_PRED_TRUE:
        sv = (sv << 1) | 1u;
        sk = (sk << 1) | 1u;
        break;
      case DFC_PRED_NOT:
        sv ^= sk & 1u;
        break;
      default: {  // AND / OR
        const uint32_t bv = sv & 1u, bk = sk & 1u;
        sv >>= 1;
        sk >>= 1;
        const uint32_t av = sv & 1u, ak = sk & 1u;
        uint32_t rv, rk;
        if (op.kind == DFC_PRED_AND) {
          const uint32_t false_known = (ak & (av ^ 1u)) | (bk & (bv ^ 1u));
          rk = false_known | (ak & bk);
          rv = (false_known ^ 1u) & ak & bk & av & bv;
        } else {
          const uint32_t true_known = (ak & av) | (bk & bv);
          rk = true_known | (ak & bk);
          rv = true_known;
        }
        sv = (sv & ~1u) | rv;
        sk = (sk & ~1u) | rk;
      }
    }
  }
  return (sv & sk & 1u) != 0;
}

template <typename T>
__device__ __forceinline__ uint32_t select_word_cmp(const PredOp& op, const unsigned char* vals, const uint32_t* valid,
                                                    uint32_t r, bool in) {
  bool v = false;
  if (in && valid_at(valid, r)) {
    const T x = load_as<T>(vals, r);
    if constexpr (sizeof(T) == 8 && T(-1) > T(0)) v = cmp_op<uint64_t>(op.cmp, (uint64_t)x, op.lit.u);
    else if constexpr (std::is_floating_point<T>::value) v = cmp_op<T>(op.cmp, x, (T)op.lit.f);
    else v = cmp_op<int64_t>(op.cmp, (int64_t)x, op.lit.i);
  }
  return __ballot_sync(0xffffffffu, v);
}

// The selection words of a tile: warp w computes words w, w + 8, ...; each
// lane holds one row of a word.  Returns, per word, the bits of selected rows.
__device__ __forceinline__ uint32_t select_word(const ScanParams& p, const Step& s, int tile, uint32_t word) {
  const uint32_t r = word * 32 + (threadIdx.x & 31);
  const bool in = r < s.n[tile];
  if (p.n_pred == 0) return __ballot_sync(0xffffffffu, in);
  const PredOp& op = p.pred[0];
  if (p.n_pred == 1 && op.kind == DFC_PRED_CMP) {
    const int c = op.input;
    const unsigned char* vals = col_values(p, s, tile, c);
    const uint32_t* valid = col_valid(p, s, tile, c);
    switch (p.cols[c].dtype) {
      case DFC_INT8: return select_word_cmp<int8_t>(op, vals, valid, r, in);
      case DFC_INT16: return select_word_cmp<int16_t>(op, vals, valid, r, in);
      case DFC_INT32: return select_word_cmp<int32_t>(op, vals, valid, r, in);
      case DFC_INT64: return select_word_cmp<int64_t>(op, vals, valid, r, in);
      case DFC_UINT8: return select_word_cmp<uint8_t>(op, vals, valid, r, in);
      case DFC_UINT16: return select_word_cmp<uint16_t>(op, vals, valid, r, in);
      case DFC_UINT32: return select_word_cmp<uint32_t>(op, vals, valid, r, in);
      case DFC_UINT64: return select_word_cmp<uint64_t>(op, vals, valid, r, in);
      case DFC_FLOAT32: return select_word_cmp<float>(op, vals, valid, r, in);
      default: return select_word_cmp<double>(op, vals, valid, r, in);
    }
  }
  return __ballot_sync(0xffffffffu, in && program_row(p, s, tile, r));
}

// ---------------------------------------------------------------------------
// 3. Keys.
// ---------------------------------------------------------------------------
template <typename T, int R>
__device__ __forceinline__ void key_field(const ColRef& cr, const RowRef (&x)[R], bool packed, const KeyField& f,
                                          int k, uint64_t (&kw)[R]) {
#pragma unroll
  for (int j = 0; j < R; ++j) {
    if (!x[j].on) continue;
    const bool ok = rvalid(cr, x[j]);
    uint64_t cell = 0;
    if (ok) {
      const T v = load_as<T>(rv(cr, x[j]), x[j].r);
      if constexpr (std::is_same<T, float>::value) cell = key_cell(__float_as_uint(v), DFC_FLOAT32);
      else if constexpr (std::is_same<T, double>::value) cell = key_cell((uint64_t)__double_as_longlong(v), DFC_FLOAT64);
      else cell = (uint64_t)(typename std::make_unsigned<T>::type)v;
    }
    if (packed) {
      if (!ok) kw[j] |= 1ull << f.null_bit;
      else kw[j] |= (sizeof(T) == 8) ? cell : (cell << f.shift);
    } else {
      const uint64_t c = ok ? cell + 1 : 0x9E3779B97F4A7C15ull;
      kw[j] = mix64(kw[j] ^ (c * 0x9E3779B97F4A7C15ull + (uint64_t)k));
    }
  }
}

template <int R = kR>
__device__ __forceinline__ void key_words(const ScanParams& p, const Step& s, const RowRef (&x)[R], uint64_t (&kw)[R]) {
  const bool packed = p.key_mode == KEY_PACKED;
#pragma unroll
  for (int j = 0; j < R; ++j) kw[j] = packed ? 0ull : 0x243F6A8885A308D3ull;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    const ColRef cr = col_ref(p, s, f.input);
    switch (f.dtype) {
      case DFC_INT8: key_field<int8_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_INT16: key_field<int16_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_INT32: key_field<int32_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_INT64: key_field<int64_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_UINT8: key_field<uint8_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_UINT16: key_field<uint16_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_UINT32: key_field<uint32_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_UINT64: key_field<uint64_t, R>(cr, x, packed, f, k, kw); break;
      case DFC_FLOAT32: key_field<float, R>(cr, x, packed, f, k, kw); break;
      default: key_field<double, R>(cr, x, packed, f, k, kw); break;
    }
  }
  if (!packed) {
#pragma unroll
    for (int j = 0; j < R; ++j)
      if (kw[j] == kEmpty) kw[j] = kEmpty - 1;
  }
}

// Ticket mode: key columns of global rows a and b equal under group equality.
__device__ __forceinline__ bool rows_key_equal(const ScanParams& p, uint64_t a, uint64_t b) {
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    const DevColumn& c = p.cols[f.input];
    const bool va = c.validity == nullptr || bit_valid(c.validity, a);
    const bool vb = c.validity == nullptr || bit_valid(c.validity, b);
    if (va != vb) return false;
    if (va && key_cell(load_bits(c.values, c.size, a), f.dtype) != key_cell(load_bits(c.values, c.size, b), f.dtype))
      return false;
  }
  return true;
}

__device__ __forceinline__ uint64_t slot_of(const ScanParams& p, uint64_t kw) {
  return mix64(kw ^ 0x632BE59BD9B4E019ull) & p.table_mask;
}

// ---------------------------------------------------------------------------
// 4. Groups: claims in the global table.
// ---------------------------------------------------------------------------
// Record numbers are handed out by CTA tickets: ticket t falls in the CTA's
// chunk k = t / chunk, whose base the holder of the chunk's first ticket draws
// from the global counter and publishes (tagged with k) in a small ring.
// Records stay all-zero until used; one reserved and never used (a lost
// race of the per-lane claims below) is a hole the finish skips.
constexpr int kChunkRing = 64;

struct ClaimState {
  uint32_t ticket;
  unsigned long long ring[kChunkRing];
};

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

// The winner of a claim writes the group's key word and, without
// maintain_order, its claim row (the group's row for keys and order).
__device__ __forceinline__ void claimed(const ScanParams& p, uint32_t gid, uint64_t kw, uint32_t row) {
  unsigned char* rec = record_at(p, gid);
  *reinterpret_cast<unsigned long long*>(rec + kRecKey) = kw;
  if (!p.track_first) *reinterpret_cast<uint32_t*>(rec + kRecFirst) = ~row;
}

// Re-reads an entry's meta word until published (a claim writes key and meta
// in one 128-bit CAS, so this only loops on a torn read).
__device__ __forceinline__ uint64_t entry_meta(const ScanParams& p, const KeyEntry* e) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    const uint64_t m = ld_relaxed_u64(&e->meta);
    if (m != kEmpty) return m;
  }
  atomicOr(p.status, ST_TIMEOUT);
  return kEmpty;
}

// The group of key word kw at row `row`, claiming a new record if the key is
// new: the per-lane path for ticket keys and the all-ones key word (one-step
// claims: a 128-bit CAS of key and reserved record; a lost race leaves the
// reserved record unused).
// Visits slots in the same order as the lock-step rounds.  kNoGid when
// records or table slots ran out (ST_CAPACITY set).
__device__ __noinline__ uint32_t find_or_claim(const ScanParams& p, uint64_t kw, uint32_t row, ClaimState* cs) {
  const uint64_t slots = p.table_mask + 1;
  if (kw == kEmpty) {  // the all-ones key word has its own entry after the table
    KeyEntry* e = p.table + slots;
    const uint64_t m = ld_cg_u64(&e->meta);
    if (m != kEmpty) return (uint32_t)m;
    const uint32_t gid = reserve_record(p, cs);
    if (gid == kNoGid) return kNoGid;
    uint64_t ok, om;
    cas128(e, kEmpty, kEmpty, kEmpty, (uint64_t)gid | ((uint64_t)row << 32), ok, om);
    if (om == kEmpty) {
      claimed(p, gid, kw, row);
      return gid;
    }
    return (uint32_t)om;
  }
  uint64_t slot = slot_of(p, kw);
  uint32_t reserved = kNoGid;
  for (uint64_t probe = 0; probe < slots; ++probe) {
    KeyEntry* e = p.table + slot;
    const uint64_t k = ld_cg_u64(&e->key);
    if (k == kw) {
      const uint64_t m = entry_meta(p, e);
      if (m == kEmpty) return kNoGid;
      if (p.key_mode == KEY_PACKED || rows_key_equal(p, row, (uint32_t)(m >> 32))) return (uint32_t)m;
    } else if (k == kEmpty) {
      if (reserved == kNoGid) {
        reserved = reserve_record(p, cs);
        if (reserved == kNoGid) return kNoGid;
      }
      uint64_t ok, om;
      cas128(e, kEmpty, kEmpty, kw, (uint64_t)reserved | ((uint64_t)row << 32), ok, om);
      if (ok == kEmpty && om == kEmpty) {
        claimed(p, reserved, kw, row);
        return reserved;
      }
      if (ok == kw && (p.key_mode == KEY_PACKED || rows_key_equal(p, row, (uint32_t)(om >> 32)))) return (uint32_t)om;
    }
    slot = (slot + 1) & p.table_mask;
  }
  atomicOr(p.status, ST_CAPACITY);
  return kNoGid;
}

// Packed keys: all rows of the warp resolved together.  Each round a pending
// row looks at two consecutive entries of its probe sequence: its key ->
// found; empty -> claim it (CAS); both others -> the next two.  Rounds run in
// lock-step so the warp's loads and claims overlap.
__device__ __forceinline__ void resolve_packed(const ScanParams& p, const uint32_t (&rows)[kR], bool (&sel)[kR],
                                               const uint64_t (&kw)[kR], uint32_t (&gid)[kR], ClaimState* cs) {
  uint64_t slot[kR];
  ulonglong2 e0[kR], e1[kR];
  bool pend[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    gid[j] = kNoGid;
    pend[j] = sel[j];
    slot[j] = 0;
    if (pend[j] && kw[j] == kEmpty) {
      gid[j] = find_or_claim(p, kw[j], rows[j], cs);
      pend[j] = false;
    }
    if (pend[j]) {
      slot[j] = slot_of(p, kw[j]);
      e0[j] = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + slot[j]));
      e1[j] = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + ((slot[j] + 1) & p.table_mask)));
    }
  }
  for (uint32_t round = 0;; ++round) {
    bool any = false;
#pragma unroll
    for (int j = 0; j < kR; ++j) any |= pend[j];
    if (!__any_sync(0xffffffffu, any)) break;
    if (round > (p.table_mask >> 1) + 2) {  // every slot seen: the table is full
#pragma unroll
      for (int j = 0; j < kR; ++j) pend[j] = false;
      atomicOr(p.status, ST_CAPACITY);
      break;
    }
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      if (!pend[j]) continue;
      int step = 0;  // entries of this round consumed without a result
      for (int h = 0; h < 2 && pend[j]; ++h) {
        const ulonglong2 e = h ? e1[j] : e0[j];
        const uint64_t s = (slot[j] + h) & p.table_mask;
        if (e.x == kw[j]) {
          if (e.y != kEmpty) {
            gid[j] = (uint32_t)e.y;
            pend[j] = false;
          }
          break;  // claimed, not yet published: look at this entry again
        }
        if (e.x == kEmpty) {
          // Two steps: a CAS of the key word claims the entry, then the
          // winner reserves a record and publishes it in the meta word.  Only
          // winners reserve, so no record is left unused.  Rows that find the
          // key unpublished read the entry again next round (no waiting here).
          KeyEntry* en = p.table + s;
          const unsigned long long prev = atomicCAS(&en->key, kEmpty, kw[j]);
          if (prev == kEmpty) {
            const uint32_t g = reserve_record(p, cs);
            if (g != kNoGid) {
              claimed(p, g, kw[j], rows[j]);
              atomicExch(&en->meta, (unsigned long long)g | ((unsigned long long)rows[j] << 32));
              gid[j] = g;
            }
            pend[j] = false;
            break;
          }
          if (prev == kw[j]) break;  // another row's claim of this key: read it again
          step = h + 1;              // taken by another key: go on past it
          continue;
        }
        step = h + 1;
      }
      if (pend[j]) {
        slot[j] = (slot[j] + step) & p.table_mask;
        e0[j] = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + slot[j]));
        e1[j] = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + ((slot[j] + 1) & p.table_mask)));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kR; ++j) sel[j] = sel[j] && gid[j] != kNoGid;
}

// Thread-block cluster helpers.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_ranks() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_index() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
// Every thread of every CTA of the cluster; release/acquire at cluster scope
// orders the CTAs' global-memory work on the shared table across phases.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t ld_cluster_u32(const void* local, uint32_t rank) {
  uint32_t a, v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(local)), "r"(rank));
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
  return v;
}

// ---------------------------------------------------------------------------
// 4'. Shared-memory regime (few groups): each CTA keeps its own key table and
// all-zero group records in shared memory -- or, with smem_cluster > 1, the
// CTAs of a thread-block cluster pool their tables into one, each key living
// in one CTA's share and reached through distributed shared memory; duplicate
// keys inside a warp are collapsed with __match_any_sync so one leader lane
// applies the combined update; each CTA merges its share into the global
// table when the cluster is done.  Rows whose key finds no room take the
// global path.
// ---------------------------------------------------------------------------
struct SmemTable {
  unsigned long long* keys;  // smem_slots, kEmpty = free
  unsigned char* recs;       // smem_slots records of rec_stride bytes
  uint32_t* used;            // claimed slots
  uint32_t ranks;            // CTAs sharing the table (power of two)
};

// A group record of a shared-memory table as group_update sees it: in this
// CTA's own table (generic address, native atomics) or in a cluster table
// (the owner CTA's record as a .shared::cluster address, explicit-space
// atomics).  On B200 a native 64-bit atomic maximum through a generic address
// into another CTA's shared memory lost updates in this library's tests, so
// cluster records raise 64-bit maxima by compare-and-swap.
struct OwnRec {
  unsigned char* p;
  __device__ __forceinline__ void max_u32(int off, uint32_t v) const { atomicMax(reinterpret_cast<uint32_t*>(p + off), v); }
  __device__ __forceinline__ void add_u32(int off, uint32_t v) const { atomicAdd(reinterpret_cast<uint32_t*>(p + off), v); }
  __device__ __forceinline__ void or_u32(int off, uint32_t v) const { atomicOr(reinterpret_cast<uint32_t*>(p + off), v); }
  __device__ __forceinline__ uint64_t add_u64(int off, uint64_t v) const {
    return atomicAdd(reinterpret_cast<unsigned long long*>(p + off), (unsigned long long)v);
  }
  __device__ __forceinline__ void add_f64(int off, double v) const { atomicAdd(reinterpret_cast<double*>(p + off), v); }
  __device__ __forceinline__ uint64_t ld_u64(int off) const {
    return *reinterpret_cast<const volatile unsigned long long*>(p + off);
  }
  __device__ __forceinline__ uint64_t cas_u64(int off, uint64_t cmp, uint64_t val) const {
    return atomicCAS(reinterpret_cast<unsigned long long*>(p + off), (unsigned long long)cmp, (unsigned long long)val);
  }
  __device__ __forceinline__ bool max_u64(int off, uint64_t v) const {
    atomicMax(reinterpret_cast<unsigned long long*>(p + off), (unsigned long long)v);
    return true;
  }
};

struct ClusterRec {
  uint32_t a;
  __device__ __forceinline__ void max_u32(int off, uint32_t v) const { dsm_max_u32(a + off, v); }
  __device__ __forceinline__ void add_u32(int off, uint32_t v) const { dsm_add_u32(a + off, v); }
  __device__ __forceinline__ void or_u32(int off, uint32_t v) const { dsm_or_b32(a + off, v); }
  __device__ __forceinline__ uint64_t add_u64(int off, uint64_t v) const { return dsm_add_u64(a + off, v); }
  __device__ __forceinline__ void add_f64(int off, double v) const { dsm_add_f64(a + off, v); }
  __device__ __forceinline__ uint64_t ld_u64(int off) const { return dsm_ld_u64(a + off); }
  __device__ __forceinline__ uint64_t cas_u64(int off, uint64_t cmp, uint64_t val) const {
    return dsm_cas_u64(a + off, cmp, val);
  }
  // False when the retries ran out.
  __device__ __forceinline__ bool max_u64(int off, uint64_t v) const {
    uint64_t old = dsm_ld_u64(a + off);
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
      if (old >= v) return true;
      const uint64_t seen = dsm_cas_u64(a + off, old, v);
      if (seen == old) return true;
      old = seen;
    }
    return false;
  }
};

// The direct-addressed slot of packed key word `kw` (ScanParams::direct).
__device__ __forceinline__ uint32_t direct_slot(const ScanParams& p, uint64_t kw) {
  uint32_t s = 0;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& kf = p.keys[k];
    if (kf.null_bit >= 0 && ((kw >> kf.null_bit) & 1ull)) continue;  // null: field 0
    const uint64_t mask = kf.bits == 64 ? ~0ull : ((1ull << kf.bits) - 1ull);
    const uint64_t raw = (kw >> kf.shift) & mask;
    // The key's own wrap-around subtraction: values lie in [dmin, dmin + span).
    s += (uint32_t)(((raw - p.dmin[k]) & mask) + 1ull) << p.dshift[k];
  }
  return s;
}

// The record of key word `kw` in this CTA's own table (claimed if new);
// false when the key is absent and the table is three-quarters full.
// Direct-addressed tables hold every key's slot, so they never fill.
__device__ __forceinline__ bool smem_probe(const ScanParams& p, const SmemTable& st, uint64_t kw, OwnRec& rec) {
  if (kw == kEmpty) return false;
  if (p.direct) {
    const uint32_t s = direct_slot(p, kw);
    if (s >= p.smem_slots) return false;  // outside the planned ranges: the global path
    unsigned long long* key = &st.keys[s];
    const unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(key);
    if (k != kw) {
      if (k != kEmpty) return false;
      const unsigned long long prev = atomicCAS(key, kEmpty, kw);
      if (prev == kEmpty) atomicAdd(st.used, 1u);
      else if (prev != kw) return false;
    }
    rec.p = st.recs + (size_t)s * p.rec_stride;
    return true;
  }
  const uint32_t mask = p.smem_slots - 1;
  uint32_t s = (uint32_t)mix64(kw ^ 0x9FB21C651E98DF25ull) & mask;
  for (int probe = 0; probe < 32; ++probe) {
    const unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(&st.keys[s]);
    bool hit = k == kw;
    if (!hit && k == kEmpty) {
      // At most three-quarters full, so probes stay short.
      if (*reinterpret_cast<volatile uint32_t*>(st.used) >= p.smem_slots - p.smem_slots / 4) return false;
      const unsigned long long prev = atomicCAS(&st.keys[s], kEmpty, kw);
      if (prev == kEmpty) atomicAdd(st.used, 1u);
      hit = prev == kEmpty || prev == kw;
    }
    if (hit) {
      rec.p = st.recs + (size_t)s * p.rec_stride;
      return true;
    }
    s = (s + 1) & mask;
  }
  return false;
}

// The same in a cluster table: the hash's high bits pick the owner CTA, its
// low bits the first slot of the owner's share; probes stay inside the share
// and the fill limit is the owner's.
__device__ __forceinline__ bool smem_probe(const ScanParams& p, const SmemTable& st, uint64_t kw, ClusterRec& rec) {
  if (kw == kEmpty) return false;
  const uint64_t h = mix64(kw ^ 0x9FB21C651E98DF25ull);
  const uint32_t r = (uint32_t)(h >> 40) & (st.ranks - 1);
  const uint32_t keys = dsm_map(st.keys, r), recs = dsm_map(st.recs, r), used = dsm_map(st.used, r);
  const uint32_t mask = p.smem_slots - 1;
  uint32_t s = (uint32_t)h & mask;
  for (int probe = 0; probe < 32; ++probe) {
    const uint64_t k = dsm_ld_u64(keys + s * 8u);
    bool hit = k == kw;
    if (!hit && k == kEmpty) {
      if (dsm_ld_u32(used) >= p.smem_slots - p.smem_slots / 4) return false;
      const uint64_t prev = dsm_cas_u64(keys + s * 8u, kEmpty, kw);
      if (prev == kEmpty) dsm_add_u32(used, 1u);
      hit = prev == kEmpty || prev == kw;
    }
    if (hit) {
      rec.a = recs + s * (uint32_t)p.rec_stride;
      return true;
    }
    s = (s + 1) & mask;
  }
  return false;
}

// Compensated FP32 pairs {s, c} (Neumaier's variant of Kahan summation; the
// value is s + c): `x` with its low part `xc` added to the pair.  A sum that
// leaves the FP32 range from finite operands sets `range` (the host reruns
// the query in FP64); non-finite sums keep the compensation unchanged, so
// +-inf and NaN propagate through s alone.
__device__ __forceinline__ void pair_add(float& s, float& c, float x, float xc, bool& range) {
  const float t = s + x;
  if (isfinite(t)) {
    const float e = fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
    c += e + xc;
  } else if (isfinite(s) && isfinite(x)) {
    range = true;
  }
  s = t;
}

// The pair sum of each lane's group (members in lane order), as group_reduce.
__device__ __forceinline__ void group_pair(uint32_t grp, int maxpop, float ms, float mc, bool take, float& s, float& c,
                                           bool& range, bool one = false) {
  if (one) {
    s = take ? ms : 0.f;
    c = take ? mc : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float os = __shfl_xor_sync(0xffffffffu, s, o), oc = __shfl_xor_sync(0xffffffffu, c, o);
      pair_add(s, c, os, oc, range);
    }
    return;
  }
  s = 0.f;
  c = 0.f;
  uint32_t left = grp;
  const int lane = threadIdx.x & 31;
  for (int i = 0; i < maxpop; ++i) {
    const int src = left ? __ffs(left) - 1 : lane;
    const float vs = __shfl_sync(0xffffffffu, take ? ms : 0.f, src);
    const float vc = __shfl_sync(0xffffffffu, take ? mc : 0.f, src);
    if (left) {
      pair_add(s, c, vs, vc, range);
      left &= left - 1;
    }
  }
}

// Adds {x, xc} to the pair at byte `off` of a record by compare-and-swap;
// false when the retries ran out.
template <typename Rec>
__device__ __forceinline__ bool pair_cas_add(const Rec& rec, int off, float x, float xc, bool& range) {
  uint64_t old = rec.ld_u64(off);
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    float s = __uint_as_float((uint32_t)old), c = __uint_as_float((uint32_t)(old >> 32));
    bool r = false;
    pair_add(s, c, x, xc, r);
    const uint64_t nw = ((uint64_t)__float_as_uint(c) << 32) | __float_as_uint(s);
    const uint64_t seen = rec.cas_u64(off, old, nw);
    if (seen == old) {
      range = range || r;
      return true;
    }
    old = seen;
  }
  return false;
}

// The FP64 value of a pair (s alone when it is not finite).
__device__ __forceinline__ double pair_value(const unsigned char* at) {
  const float s = *reinterpret_cast<const float*>(at), c = *reinterpret_cast<const float*>(at + 4);
  return isfinite(s) ? (double)s + (double)c : (double)s;
}

// The lane holding the i-th member of `grp` (lanes outside return their own).
__device__ __forceinline__ int nth_lane(uint32_t grp, int i) {
  for (int k = 0; k < i; ++k) grp &= grp - 1;
  return grp ? __ffs(grp) - 1 : (int)(threadIdx.x & 31);
}

// Full-warp butterfly reductions (every lane gets the result).
__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}
__device__ __forceinline__ __int128 warp_sum_i128(__int128 v) {
  uint64_t lo = (uint64_t)v, hi = (uint64_t)((unsigned __int128)v >> 64);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t olo = __shfl_xor_sync(0xffffffffu, lo, o), ohi = __shfl_xor_sync(0xffffffffu, hi, o);
    const uint64_t nlo = lo + olo;
    hi = hi + ohi + (nlo < lo ? 1ull : 0ull);
    lo = nlo;
  }
  return (__int128)(((unsigned __int128)hi << 64) | lo);
}

// Reduction over each lane's group, members in lane order; shuffles run on
// the full warp, one per member of the largest group.  `one`: every lane in
// a group is in the same one, reduced by a five-step butterfly instead.
template <typename V, typename Op>
__device__ __forceinline__ V group_reduce(uint32_t grp, int maxpop, V mine, V identity, bool take, Op op,
                                          bool one = false) {
  if (one) {
    V acc = take ? mine : identity;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = op(acc, __shfl_xor_sync(0xffffffffu, acc, o));
    return acc;
  }
  V acc = identity;
  uint32_t left = grp;
  const int lane = threadIdx.x & 31;
  for (int i = 0; i < maxpop; ++i) {
    const V v = __shfl_sync(0xffffffffu, take ? mine : identity, left ? __ffs(left) - 1 : lane);
    if (left) {
      acc = op(acc, v);
      left &= left - 1;
    }
  }
  return acc;
}

// One warp's rows folded into their records, rows of one record first
// reduced across lanes: `grp` the lanes sharing this lane's record `rec` (0
// for a lane outside), `maxpop` the largest group in the warp.  The group's
// lowest lane (the leader) applies one atomic per field.  `get(v, ok, b)`
// gives the lane's validity and raw bits of value column v.  `Rec`: OwnRec or
// ClusterRec.
template <typename Rec, typename Get>
__device__ __forceinline__ void group_update(const ScanParams& p, const Rec& rec, uint32_t grp, int maxpop, bool loc,
                                             uint32_t row, Get&& get) {
  const int lane = threadIdx.x & 31;
  {
    const bool leader = loc && lane == __ffs(grp) - 1;
    // All rows of the warp in one group (a hot key): butterfly reductions.
    const bool one = maxpop > 4 && maxpop == __popc(__ballot_sync(0xffffffffu, loc));
    // The group's earliest row.  A CTA record always keeps its first row:
    // it is the claim row when the record is merged into the global table.
    const uint32_t first =
        group_reduce<uint32_t>(grp, maxpop, row, 0xFFFFFFFFu, loc, [](uint32_t a, uint32_t b2) { return a < b2 ? a : b2; },
                               one);
    // The group's latest row + 1 (LAST; 0 = none).
    const uint32_t last = p.off_last >= 0 ? group_reduce<uint32_t>(grp, maxpop, row + 1u, 0u, loc,
                                                                   [](uint32_t a, uint32_t b2) { return a > b2 ? a : b2; }, one)
                                          : 0u;
    if (leader) {
      rec.max_u32(kRecFirst, ~first);
      if (p.off_len >= 0) rec.add_u32(p.off_len, (uint32_t)__popc(grp));
      if (p.off_last >= 0) rec.max_u32(p.off_last, last);
    }
    for (int v = 0; v < p.n_vals; ++v) {
      const ValField& f = p.vals[v];
      const int dt = f.dtype;
      const bool isf = dt_float(dt);
      bool ok = false;
      uint64_t b = 0;
      if (loc) get(v, ok, b);
      if (!ok) b = 0;
      const double xd = isf ? bits_to_f64(b, dt) : bits_as_double(b, dt);
      const bool nan = ok && isf && xd != xd;
      const uint32_t vmask = grp & __ballot_sync(0xffffffffu, ok);
      // NaN and signed-zero flags: float columns only (isf is warp-uniform).
      uint32_t nanmask = 0, pz = 0, nz = 0;
      if (isf) {
        nanmask = grp & __ballot_sync(0xffffffffu, nan);
        pz = grp & __ballot_sync(0xffffffffu, ok && xd == 0.0 && __double_as_longlong(xd) >= 0);
        nz = grp & __ballot_sync(0xffffffffu, ok && xd == 0.0 && __double_as_longlong(xd) < 0);
      }
      if (leader && vmask) rec.add_u32(f.off_count, (uint32_t)__popc(vmask));
      const bool comp = (p.comp_mask >> v) & 1u;
      bool range = false, stuck = false;
      if (f.off_sum >= 0) {
        if (comp) {
          float ps, pc;
          group_pair(grp, maxpop, (float)xd, 0.f, ok, ps, pc, range, one);
          if (leader && vmask) stuck = !pair_cas_add(rec, f.off_sum, ps, pc, range);
        } else if (f.sum_kind == SUM_F64) {
          const double sm = group_reduce<double>(grp, maxpop, xd, 0.0, ok, [](double a, double b2) { return a + b2; }, one);
          if (leader && vmask) rec.add_f64(f.off_sum, sm);
        } else {
          // The group's partial sum, exact in 128 bits.
          const bool uns = dt == DFC_UINT64;
          const uint64_t xv = ok ? (uns ? b : (uint64_t)bits_to_i64(b, dt)) : 0ull;
          const uint64_t xhi = (!uns && (int64_t)xv < 0) ? ~0ull : 0ull;
          __int128 exact = 0;
          uint32_t left = one ? 0u : grp;
          if (one) exact = warp_sum_i128(ok ? (__int128)(((unsigned __int128)xhi << 64) | xv) : (__int128)0);
          for (int i = 0; i < (one ? 0 : maxpop); ++i) {
            const int src = left ? __ffs(left) - 1 : lane;
            const uint64_t vlo = __shfl_sync(0xffffffffu, xv, src);
            const uint64_t vhi = __shfl_sync(0xffffffffu, xhi, src);
            if (left) {
              exact += (__int128)(((unsigned __int128)vhi << 64) | vlo);
              left &= left - 1;
            }
          }
          if (leader && vmask) {
            if (f.sum_kind == SUM_I64) {
              rec.add_u64(f.off_sum, (uint64_t)(int64_t)exact);
            } else {
              const uint64_t add_lo = (uint64_t)exact, add_hi = (uint64_t)(exact >> 64);
              const uint64_t old = rec.add_u64(f.off_sum, add_lo);
              const uint64_t hi_add = add_hi + ((old + add_lo) < old ? 1ull : 0ull);
              if (hi_add) rec.add_u64(f.off_sum + 8, hi_add);
            }
          }
        }
      }
      if (f.off_min >= 0 || f.off_max >= 0) {
        const bool ordinary = ok && !nan;
        const uint64_t e = ordinary ? order_encode(b, dt) : 0ull;
        if (f.off_min >= 0) {
          const unsigned long long m = group_reduce<unsigned long long>(
              grp, maxpop, ~e, 0ull, ordinary, [](unsigned long long a, unsigned long long b2) { return a > b2 ? a : b2; },
              one);
          if (leader && m && !rec.max_u64(f.off_min, m)) stuck = true;
        }
        if (f.off_max >= 0) {
          const unsigned long long m = group_reduce<unsigned long long>(
              grp, maxpop, e, 0ull, ordinary, [](unsigned long long a, unsigned long long b2) { return a > b2 ? a : b2; },
              one);
          if (leader && m && !rec.max_u64(f.off_max, m)) stuck = true;
        }
        if (leader) {
          uint32_t bits = 0;
          if (nanmask) bits |= 1u << (3 * v);
          if (pz) bits |= 1u << (3 * v + 1);
          if (nz) bits |= 1u << (3 * v + 2);
          if (bits) rec.or_u32(kRecFlags, bits);
        }
      }
      if (f.off_m2 >= 0) {
        // The group's shift K: set once, by the first valid value of a leader.
        const uint64_t xbits = (xd != xd) ? kCanonNaN : (uint64_t)__double_as_longlong(xd);
        const uint64_t cand = __shfl_sync(0xffffffffu, xbits, vmask ? __ffs(vmask) - 1 : lane);
        uint64_t ks = 0;
        if (leader && vmask) {
          ks = rec.ld_u64(f.off_shift);
          if (ks == 0) {
            const uint64_t prev = rec.cas_u64(f.off_shift, 0ull, cand ^ kShiftTag);
            ks = prev == 0 ? (cand ^ kShiftTag) : prev;
          }
        }
        ks = __shfl_sync(0xffffffffu, ks, grp ? __ffs(grp) - 1 : lane);
        const double kd = __longlong_as_double((long long)(ks ^ kShiftTag));
        if (comp) {
          // d = x - K exactly as dh + dl (Knuth's TwoSum; K is a Float32 value),
          // d^2 as dh^2 (rounded) + its FMA residue + 2 dh dl.
          const float xf = (float)xd, kf = (float)kd;
          const float dh = xf - kf;
          const float bb = dh - xf;
          const float dl = (xf - (dh - bb)) + (-kf - bb);
          const float sq = dh * dh;
          const float sq_lo = fmaf(2.f * dh, dl, fmaf(dh, dh, -sq));
          if (ok && isfinite(xf) && isfinite(kf) && !isfinite(sq)) range = true;
          float ps, pc;
          group_pair(grp, maxpop, sq, isfinite(sq) ? sq_lo : 0.f, ok, ps, pc, range, one);
          if (leader && vmask && !stuck) stuck = !pair_cas_add(rec, f.off_m2, ps, pc, range);
        } else {
          const double d = xd - kd;
          const double s2 = group_reduce<double>(grp, maxpop, d * d, 0.0, ok, [](double a, double b2) { return a + b2; }, one);
          if (leader && vmask) rec.add_f64(f.off_m2, s2);
        }
      }
      if (range) atomicOr(p.status, ST_F32_RANGE);
      if (stuck) atomicOr(p.status, ST_TIMEOUT);
    }
  }
}

template <typename Rec>
__device__ __forceinline__ void smem_rows_in(const ScanParams& p, const Step& s, const SmemTable& st,
                                             const RowRef (&x)[kR], const uint32_t (&rows)[kR], bool (&sel)[kR],
                                             const uint64_t (&kw)[kR]) {
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    Rec rec{};
    const bool loc = sel[j] && smem_probe(p, st, kw[j], rec);
    uint32_t grp = __match_any_sync(0xffffffffu, kw[j]) & __ballot_sync(0xffffffffu, loc);
    if (!loc) grp = 0;
    const int maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    if (maxpop == 0) continue;
    group_update(p, rec, grp, maxpop, loc, rows[j], [&](int v, bool& ok, uint64_t& b) {
      const int c = p.vals[v].input;
      const ColRef cr = col_ref(p, s, c);
      ok = rvalid(cr, x[j]);
      b = ok ? load_bits(rv(cr, x[j]), p.cols[c].size, x[j].r) : 0ull;
    });
    sel[j] = sel[j] && !loc;  // the rest take the global path
  }
}


// Folds the lanes of the warp's largest group -- `grp` is each lane's group
// mask (0 outside), `maxpop` its size -- into the group's record (`rec`, the
// lane's own record pointer) with one atomic per field: every field reduced
// over the group by a five-step butterfly, whatever the group's size.  Same
// state updates as group_update.  Every lane calls it; returns whether this
// lane was folded.  `get(v, ok, b)` gives the lane's value of column v.
template <typename Get>
__device__ bool collapse_largest(const ScanParams& p, unsigned char* rec, uint32_t grp, int maxpop, bool on, uint32_t row,
                                 Get&& get) {
  const int lane = threadIdx.x & 31;
  const uint32_t cand = __ballot_sync(0xffffffffu, on && __popc(grp) == maxpop);
  const int lead = __ffs(cand) - 1;  // the lowest lane of a largest group: its leader
  const uint32_t big = __shfl_sync(0xffffffffu, grp, lead);
  const bool in = (big >> lane) & 1u;
  const bool leader = lane == lead;
  unsigned char* const grec = reinterpret_cast<unsigned char*>(
      __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(rec), lead));
  const uint32_t first = __reduce_min_sync(0xffffffffu, in ? row : 0xFFFFFFFFu);
  const uint32_t last = __reduce_max_sync(0xffffffffu, in ? row + 1u : 0u);
  if (leader) {
    atomicMax(reinterpret_cast<uint32_t*>(grec + kRecFirst), ~first);
    if (p.off_len >= 0) atomicAdd(reinterpret_cast<uint32_t*>(grec + p.off_len), (uint32_t)__popc(big));
    if (p.off_last >= 0) atomicMax(reinterpret_cast<uint32_t*>(grec + p.off_last), last);
  }
  for (int v = 0; v < p.n_vals; ++v) {
    const ValField& f = p.vals[v];
    const int dt = f.dtype;
    const bool isf = dt_float(dt);
    bool ok = false;
    uint64_t b = 0;
    if (in) get(v, ok, b);
    ok = ok && in;
    if (!ok) b = 0;
    const double xd = isf ? bits_to_f64(b, dt) : bits_as_double(b, dt);
    const bool nan = ok && isf && xd != xd;
    const uint32_t vmask = __ballot_sync(0xffffffffu, ok);
    if (leader && vmask) atomicAdd(reinterpret_cast<uint32_t*>(grec + f.off_count), (uint32_t)__popc(vmask));
    if (f.off_sum >= 0) {
      if (f.sum_kind == SUM_F64) {
        const double sm = warp_sum_f64(ok ? xd : 0.0);
        if (leader && vmask) atomicAdd(reinterpret_cast<double*>(grec + f.off_sum), sm);
      } else {
        const bool uns = dt == DFC_UINT64;
        const __int128 xv = !ok ? (__int128)0 : (uns ? (__int128)b : (__int128)bits_to_i64(b, dt));
        const __int128 exact = warp_sum_i128(xv);
        if (leader && vmask) {
          if (f.sum_kind == SUM_I64) {
            atomicAdd(reinterpret_cast<unsigned long long*>(grec + f.off_sum), (unsigned long long)(long long)exact);
          } else {
            const uint64_t add_lo = (uint64_t)exact, add_hi = (uint64_t)(exact >> 64);
            const uint64_t old = atomicAdd(reinterpret_cast<unsigned long long*>(grec + f.off_sum), add_lo);
            const uint64_t hi_add = add_hi + ((old + add_lo) < old ? 1ull : 0ull);
            if (hi_add) atomicAdd(reinterpret_cast<unsigned long long*>(grec + f.off_sum + 8), hi_add);
          }
        }
      }
    }
    if (f.off_min >= 0 || f.off_max >= 0) {
      const bool ordinary = ok && !nan;
      const uint64_t e = ordinary ? order_encode(b, dt) : 0ull;
      if (f.off_min >= 0) {
        const unsigned long long m = warp_max_u64(ordinary ? ~e : 0ull);
        if (leader && m) atomicMax(reinterpret_cast<unsigned long long*>(grec + f.off_min), m);
      }
      if (f.off_max >= 0) {
        const unsigned long long m = warp_max_u64(e);
        if (leader && m) atomicMax(reinterpret_cast<unsigned long long*>(grec + f.off_max), m);
      }
      const uint32_t nanmask = __ballot_sync(0xffffffffu, nan);
      const uint32_t pz = __ballot_sync(0xffffffffu, ok && isf && xd == 0.0 && __double_as_longlong(xd) >= 0);
      const uint32_t nz = __ballot_sync(0xffffffffu, ok && isf && xd == 0.0 && __double_as_longlong(xd) < 0);
      if (leader) {
        uint32_t bits = 0;
        if (nanmask) bits |= 1u << (3 * v);
        if (pz) bits |= 1u << (3 * v + 1);
        if (nz) bits |= 1u << (3 * v + 2);
        if (bits) atomicOr(reinterpret_cast<uint32_t*>(grec + kRecFlags), bits);
      }
    }
    if (f.off_m2 >= 0 && vmask) {
      // The group's shift K: set once, by the first valid value of a leader.
      const uint64_t xbits = (xd != xd) ? kCanonNaN : (uint64_t)__double_as_longlong(xd);
      const uint64_t candk = __shfl_sync(0xffffffffu, xbits, __ffs(vmask) - 1);
      uint64_t ks = 0;
      if (leader) {
        ks = *reinterpret_cast<volatile unsigned long long*>(grec + f.off_shift);
        if (ks == 0) {
          const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(grec + f.off_shift), 0ull, candk ^ kShiftTag);
          ks = prev == 0 ? (candk ^ kShiftTag) : prev;
        }
      }
      ks = __shfl_sync(0xffffffffu, ks, lead);
      const double d = xd - __longlong_as_double((long long)(ks ^ kShiftTag));
      const double s2 = warp_sum_f64(ok ? d * d : 0.0);
      if (leader) atomicAdd(reinterpret_cast<double*>(grec + f.off_m2), s2);
    }
  }
  return in;
}


// ---------------------------------------------------------------------------
// 5. States in the global records.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T from_bits(uint64_t b) {
  if constexpr (std::is_same<T, float>::value) return __uint_as_float((uint32_t)b);
  else if constexpr (std::is_same<T, double>::value) return __longlong_as_double((long long)b);
  else return (T)b;
}

// The rows' updates of one aggregated column: `recs` the rows' group records,
// `ok` whether the row holds a valid value, `vb` the value's raw bits.
// kShared: the records are in shared memory (generic loads, not .cg).
template <typename T, bool kShared = false, int R = kR>
__device__ __forceinline__ void update_rows(const ScanParams& p, const ValField& f, int v, unsigned char* const (&recs)[R],
                                            const bool (&ok)[R], const uint64_t (&vb)[R]) {
  constexpr bool kFloat = std::is_floating_point<T>::value;
  T val[R];
  uint64_t lo[R], hi[R], ks[R];
  // Values and the read-set of every row, loads in flight together.
#pragma unroll
  for (int j = 0; j < R; ++j) {
    val[j] = ok[j] ? from_bits<T>(vb[j]) : T(0);
    lo[j] = hi[j] = ks[j] = 0;
    if (!ok[j]) continue;
    const unsigned char* rec = recs[j];
    auto ld = [&](int off) -> uint64_t {
      if constexpr (kShared) return *reinterpret_cast<const volatile unsigned long long*>(rec + off);
      else return ld_cg_u64(rec + off);
    };
    if (f.off_min >= 0) lo[j] = ld(f.off_min);
    if (f.off_max >= 0) hi[j] = ld(f.off_max);
    if (f.off_m2 >= 0) ks[j] = ld(f.off_shift);
  }
#pragma unroll
  for (int j = 0; j < R; ++j) {
    if (!ok[j]) continue;
    unsigned char* rec = recs[j];
    rec_add_u32<kShared>(rec + f.off_count, 1u);
    const double xd = (double)val[j];
    const bool nan = kFloat && xd != xd;
    if (f.off_sum >= 0) {
      if constexpr (kFloat) {
        rec_add_f64<kShared>(rec + f.off_sum, xd);
      } else if (std::is_same<T, uint64_t>::value) {
        const uint64_t xv = (uint64_t)val[j];
        const uint64_t old = rec_fetch_add_u64<kShared>(rec + f.off_sum, xv);
        if (old + xv < old) rec_add_u64<kShared>(rec + f.off_sum + 8, 1ull);
      } else {
        const int64_t xv = (int64_t)val[j];
        if (f.sum_kind == SUM_I64) {
          rec_add_u64<kShared>(rec + f.off_sum, (uint64_t)xv);
        } else {
          const uint64_t old = rec_fetch_add_u64<kShared>(rec + f.off_sum, (uint64_t)xv);
          const uint64_t hi_add = (xv < 0 ? ~0ull : 0ull) + ((old + (uint64_t)xv) < old ? 1ull : 0ull);
          if (hi_add) rec_add_u64<kShared>(rec + f.off_sum + 8, hi_add);
        }
      }
    }
    if (f.off_min >= 0 || f.off_max >= 0) {
      if (nan) {
        rec_or_u32<kShared>(rec + kRecFlags, 1u << (3 * v));
      } else {
        // order_encode of the value, by its compile-time type.
        uint64_t e;
        if constexpr (kFloat) {
          const uint64_t u = xd == 0.0 ? 0ull : (uint64_t)__double_as_longlong(xd);
          e = (u >> 63) ? ~u : (u | 0x8000000000000000ull);
        } else if constexpr (std::is_unsigned<T>::value) {
          e = (uint64_t)val[j];
        } else {
          e = (uint64_t)(int64_t)val[j] ^ 0x8000000000000000ull;
        }
        if (f.off_min >= 0 && ~e > lo[j]) rec_max_u64<kShared>(rec + f.off_min, ~e);
        if (f.off_max >= 0 && e > hi[j]) rec_max_u64<kShared>(rec + f.off_max, e);
        if (kFloat && xd == 0.0) rec_or_u32<kShared>(rec + kRecFlags, 1u << (3 * v + (signbit(xd) ? 2 : 1)));
      }
    }
    if (f.off_m2 >= 0) {
      const uint64_t xbits = nan ? kCanonNaN : (uint64_t)__double_as_longlong(xd);
      uint64_t k = ks[j];
      if (k == 0) {
        const uint64_t prev = rec_cas_u64<kShared>(rec + f.off_shift, 0ull, xbits ^ kShiftTag);
        k = prev == 0 ? (xbits ^ kShiftTag) : prev;
      }
      const double d = xd - __longlong_as_double((long long)(k ^ kShiftTag));
      rec_add_f64<kShared>(rec + f.off_m2, d * d);
    }
  }
}

// The rows' values of one aggregated column from the step, then update_rows.
template <typename T>
__device__ __forceinline__ void update_column(const ScanParams& p, const ValField& f, int v, const ColRef& cr,
                                              const RowRef (&x)[kR], const bool (&sel)[kR], const uint32_t (&gid)[kR]) {
  unsigned char* recs[kR];
  bool ok[kR];
  uint64_t vb[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    ok[j] = sel[j] && rvalid(cr, x[j]);
    recs[j] = ok[j] ? record_at(p, gid[j]) : p.records;
    vb[j] = 0;
    if (ok[j]) {
      const T val = load_as<T>(rv(cr, x[j]), x[j].r);
      if constexpr (std::is_same<T, float>::value) vb[j] = __float_as_uint(val);
      else if constexpr (std::is_same<T, double>::value) vb[j] = (uint64_t)__double_as_longlong(val);
      else vb[j] = (uint64_t)(typename std::make_unsigned<T>::type)val;
    }
  }
  update_rows<T>(p, f, v, recs, ok, vb);
}

__device__ void merge_into(const ScanParams& p, const unsigned char* src, uint32_t gid);

// One pass over up to kPassRows compacted rows of a step.
template <int R>
__device__ __forceinline__ void consume_rows(const ScanParams& p, const Step& s, const uint16_t* idx, uint32_t nsel,
                                             uint32_t base, uint32_t shift, ClaimState* cs, const SmemTable* st) {
  const uint32_t ct = threadIdx.x - 32;
  RowRef x[kR];
  uint32_t rows[kR];
  bool sel[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    const uint32_t i = base + ct + (uint32_t)j * kScanConsumerThreads;
    x[j].on = i < nsel;
    const uint32_t e = x[j].on ? idx[i] : 0u;
    x[j].tile = e >> shift;
    x[j].r = e & ((1u << shift) - 1u);
    rows[j] = (uint32_t)(s.start[x[j].tile] + x[j].r);
    sel[j] = x[j].on;
  }
  uint64_t kw[kR];
  key_words(p, s, x, kw);
  if (R != kScanGlobal && st) {
    if constexpr (R == kScanCluster) smem_rows_in<ClusterRec>(p, s, *st, x, rows, sel, kw);
    else if constexpr (R == kScanOwn) smem_rows_in<OwnRec>(p, s, *st, x, rows, sel, kw);
    // Every row found its shared-memory record: nothing is left for the
    // global table (a warp-uniform exit).
    bool left = false;
#pragma unroll
    for (int j = 0; j < kR; ++j) left |= sel[j];
    if (!__any_sync(0xffffffffu, left)) return;
  }

  uint32_t gid[kR];
  if (p.key_mode == KEY_PACKED) {
    resolve_packed(p, rows, sel, kw, gid, cs);
  } else {
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      gid[j] = sel[j] ? find_or_claim(p, kw[j], rows[j], cs) : kNoGid;
      sel[j] = sel[j] && gid[j] != kNoGid;
    }
  }

  // Hot keys: a warp's largest set of rows of one group (up to two sets per
  // row slot) folds into the record by butterfly, one atomic per field.
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    // Record numbers stay below 2^32 - 32 (the planner caps them), so a lane
    // without a row gets a tag no record has.
    const uint32_t tag = sel[j] ? gid[j] : (0xFFFFFFE0u | (uint32_t)lane);
    uint32_t grp = __match_any_sync(0xffffffffu, tag) & __ballot_sync(0xffffffffu, sel[j]);
    if (!sel[j]) grp = 0;
    int maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    for (int round = 0; round < 2 && maxpop >= p.collapse_min; ++round) {
      unsigned char* rec = record_at(p, sel[j] ? gid[j] : 0u);
      const RowRef xr = x[j];
      if (collapse_largest(p, rec, grp, maxpop, sel[j], rows[j], [&](int v, bool& ok, uint64_t& b) {
            const int c = p.vals[v].input;
            const ColRef cr = col_ref(p, s, c);
            ok = rvalid(cr, xr);
            b = ok ? load_bits(rv(cr, xr), p.cols[c].size, xr.r) : 0ull;
          })) {
        sel[j] = false;
        grp = 0;
      }
      maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    }
  }

  if (p.track_first) {
    uint32_t first[kR];
#pragma unroll
    for (int j = 0; j < kR; ++j) first[j] = sel[j] ? ld_cg_u32(record_at(p, gid[j]) + kRecFirst) : ~0u;
#pragma unroll
    for (int j = 0; j < kR; ++j)
      if (sel[j] && ~rows[j] > first[j]) atomicMax(reinterpret_cast<uint32_t*>(record_at(p, gid[j]) + kRecFirst), ~rows[j]);
  }
  if (p.off_len >= 0) {
#pragma unroll
    for (int j = 0; j < kR; ++j)
      if (sel[j]) red_add_u32(record_at(p, gid[j]) + p.off_len, 1u);
  }
  if (p.off_last >= 0) {
#pragma unroll
    for (int j = 0; j < kR; ++j)
      if (sel[j]) atomicMax(reinterpret_cast<uint32_t*>(record_at(p, gid[j]) + p.off_last), rows[j] + 1u);
  }
  for (int v = 0; v < p.n_vals; ++v) {
    const ValField& f = p.vals[v];
    const ColRef cr = col_ref(p, s, f.input);
    switch (f.dtype) {
      case DFC_INT8: update_column<int8_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_INT16: update_column<int16_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_INT32: update_column<int32_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_INT64: update_column<int64_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_UINT8: update_column<uint8_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_UINT16: update_column<uint16_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_UINT32: update_column<uint32_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_UINT64: update_column<uint64_t>(p, f, v, cr, x, sel, gid); break;
      case DFC_FLOAT32: update_column<float>(p, f, v, cr, x, sel, gid); break;
      default: update_column<double>(p, f, v, cr, x, sel, gid); break;
    }
  }
}

// A consumer's ring position: its tile count modulo 2S, so that the slot is
// the position modulo S and the phase is whether it is >= S, advanced by at
// most two tiles at a time with no division by the runtime stage count.
__device__ __forceinline__ uint32_t ring_pos(uint32_t it, uint32_t k, uint32_t S) {
  const uint32_t x = it + k;
  return x >= 2 * S ? x - 2 * S : x;
}
__device__ __forceinline__ uint32_t ring_slot(uint32_t x, uint32_t S) { return x >= S ? x - S : x; }
__device__ __forceinline__ uint32_t ring_phase(uint32_t x, uint32_t S) { return x >= S ? 1u : 0u; }

// The producer (one thread): every tile of this CTA (t = blockIdx.x, +
// gridDim.x, ...) into the ring of S stages, as bulk copies of the first
// n_stage staged columns (tile_tx bytes a full tile) completing on full[s];
// a stage is refilled after its consumers arrive on empty[s].  All
// waits are bounded; on a timeout the producer raises ST_TIMEOUT, sets
// *abort and waits for the copies it issued before returning.
__device__ void produce_tiles(const ScanParams& p, unsigned char* smem, uint64_t* full, uint64_t* empty,
                              volatile uint32_t* abort, int n_stage, uint32_t tile_tx) {
  const int S = p.stages;
  const uint64_t T = (uint64_t)p.tile_rows;
  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
    const uint32_t s = it % S, ph = (it / S) & 1u;
    if (it >= (uint32_t)S && !mbar_wait_bounded(&empty[s], ph ^ 1u, kWaitLimit)) {
      atomicOr(p.status, ST_TIMEOUT);
      *abort = 1;
      break;
    }
    if (*abort) break;
    if (p.use_tma && t < p.full_tiles) {
      unsigned char* stage = smem + (size_t)s * p.stage_bytes;
      mbar_arrive_expect_tx(&full[s], tile_tx);
      for (int c = 0; c < n_stage; ++c) {
        const DevColumn& col = p.cols[c];
        bulk_g2s(stage + p.stage_off[c], static_cast<const unsigned char*>(col.values) + t * T * col.size,
                 (uint32_t)(T * col.size), &full[s]);
        if (p.stage_voff[c] >= 0)
          bulk_g2s(stage + p.stage_voff[c], col.validity + t * (T / 32), (uint32_t)(T / 8), &full[s]);
      }
    } else {
      mbar_arrive(&full[s]);  // ragged tail: consumers read global memory
    }
  }
  // Every issued stage must have landed before the CTA may exit.
  if (*abort) {
    const uint32_t first = it > (uint32_t)S ? it - S : 0;
    for (uint32_t j = first; j < it; ++j) mbar_wait_bounded(&full[j % S], (j / S) & 1u, kWaitLimit);
  }
}

// ---------------------------------------------------------------------------
// The quad row path (ScanParams::fast_rows).  Consumer thread g of a step
// takes rows 4 (g % 256) .. + 3 of the step's tile g / 256 (1024-row tiles),
// reading each column's four values with one or two vector loads from the
// stage; the filter is one range test per row and each key column is packed
// by its size, with no per-row type dispatch.
// ---------------------------------------------------------------------------
static_assert(kTilesPerStep * kMaxTileRows / 4 == kPartConsumerThreads, "one quad per consumer thread and step");

struct Quad {
  int tile;                    // the step's tile, -1: none
  uint32_t r0;                 // first row inside the tile
  uint32_t in;                 // rows inside the tile (bits 0..3)
  bool staged;
  const unsigned char* stage;  // the tile's stage (staged tiles)
  uint64_t start;              // the tile's first row
};

// The tile fields are chosen with compile-time indices (a runtime index
// into Step would put it in local memory).
__device__ __forceinline__ Quad quad_of(const Step& s, int nt) {
  const uint32_t g = threadIdx.x - 32;
  Quad q;
  q.tile = (int)(g >> 8);
  q.r0 = (g & 255u) * 4;
  const bool second = q.tile != 0;
  q.staged = second ? s.staged[1] : s.staged[0];
  q.stage = second ? s.stage[1] : s.stage[0];
  q.start = second ? s.start[1] : s.start[0];
  const uint32_t n = second ? s.n[1] : s.n[0];
  if (q.tile >= nt) {
    q.tile = -1;
    q.in = 0;
    return q;
  }
  const uint32_t left = n > q.r0 ? n - q.r0 : 0u;
  q.in = left >= 4 ? 0xFu : (1u << left) - 1u;
  return q;
}

// Raw bits (zero-extended) of the quad's rows of column c.
__device__ __forceinline__ void quad_load(const ScanParams& p, const Quad& q, int c, uint64_t (&x)[4]) {
  const int size = p.cols[c].size;
  if (q.staged) {
    const unsigned char* at = q.stage + p.stage_off[c] + (size_t)q.r0 * size;
    switch (size) {
      case 8: {
        const ulonglong2 a = reinterpret_cast<const ulonglong2*>(at)[0], b = reinterpret_cast<const ulonglong2*>(at)[1];
        x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
        return;
      }
      case 4: {
        const uint4 a = *reinterpret_cast<const uint4*>(at);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        return;
      }
      case 2: {
        const uint2 a = *reinterpret_cast<const uint2*>(at);
        x[0] = a.x & 0xFFFFu; x[1] = a.x >> 16; x[2] = a.y & 0xFFFFu; x[3] = a.y >> 16;
        return;
      }
      default: {
        const uint32_t a = *reinterpret_cast<const uint32_t*>(at);
        x[0] = a & 0xFFu; x[1] = (a >> 8) & 0xFFu; x[2] = (a >> 16) & 0xFFu; x[3] = a >> 24;
        return;
      }
    }
  }
  const unsigned char* vals = static_cast<const unsigned char*>(p.cols[c].values) + q.start * (uint64_t)size;
#pragma unroll
  for (int i = 0; i < 4; ++i) x[i] = ((q.in >> i) & 1u) ? load_bits(vals, size, q.r0 + i) : 0ull;
}

// Validity bits of the quad's rows of column c (bits 0..3, rows outside the
// tile 0).
__device__ __forceinline__ uint32_t quad_valid(const ScanParams& p, const Quad& q, int c) {
  const uint32_t* w;
  if (q.staged) w = p.stage_voff[c] >= 0 ? reinterpret_cast<const uint32_t*>(q.stage + p.stage_voff[c]) : nullptr;
  else w = p.cols[c].validity ? p.cols[c].validity + q.start / 32 : nullptr;
  if (w == nullptr || q.in == 0) return q.in;
  return (w[q.r0 >> 5] >> (q.r0 & 31u)) & q.in;
}

// Selected rows of the quad (bits 0..3).
__device__ __forceinline__ uint32_t quad_select(const ScanParams& p, const Quad& q) {
  if (p.fast_col < 0 || q.in == 0) return q.in;
  const int c = p.fast_col;
  uint64_t x[4];
  quad_load(p, q, c, x);
  const uint32_t valid = quad_valid(p, q, c);
  const int dt = p.cols[c].dtype;
  const int sh = 64 - 8 * p.cols[c].size;
  uint32_t sel = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    bool v;
    if (p.fast_kind == FAST_FLOAT) {
      const double d = bits_to_f64(x[i], dt);
      v = d >= p.fast_lo.f && d <= p.fast_hi.f;
    } else if (p.fast_kind == FAST_UNSIGNED) {
      v = x[i] >= p.fast_lo.u && x[i] <= p.fast_hi.u;
    } else {
      const int64_t xi = (int64_t)(x[i] << sh) >> sh;  // sign-extended from the column's size
      v = xi >= p.fast_lo.i && xi <= p.fast_hi.i;
    }
    sel |= (uint32_t)(v != (p.fast_neg != 0)) << i;
  }
  return sel & valid;
}

// ---------------------------------------------------------------------------
// Ungrouped queries in registers (kScanReduce).  With no key every kept row
// belongs to one group, and per-row atomics on one record serialise.  Each
// consumer thread instead keeps the group's state for its own rows in
// registers (the reference's Metal reductions keep per-thread partials too,
// dataframe_metal/accelerator/gpu/filter_sum.mojo:1-20): count, exact
// integer or FP64 sum, extrema codes, NaN and signed-zero flags, and shifted
// moments about the thread's first value K_t.  A warp folds its lanes' states
// by shuffles (moments re-centred on one lane's K), each warp folds its state
// into the CTA's one shared-memory record with one atomic per field, and the
// CTA's record merges into the global record as an own table does.
// ---------------------------------------------------------------------------
struct ReduceField {
  uint32_t n, flags;
  double sf;       // Float sum
  __int128 si;     // integer sum
  uint64_t emin;   // the largest complemented code (the minimum), 0 = none
  uint64_t emax;   // the largest code, 0 = none
  uint64_t k;      // K_t ^ kShiftTag, 0 = unset
  double s1, s2;   // sums of (x - K_t) and (x - K_t)^2
};
struct ReduceState {
  uint32_t first, last, len;  // least kept row, largest kept row + 1, kept rows
  ReduceField f[kReduceVals];
};

__device__ __forceinline__ void reduce_init(ReduceState& st) {
  st.first = 0xFFFFFFFFu;
  st.last = st.len = 0;
#pragma unroll
  for (int v = 0; v < kReduceVals; ++v) {
    ReduceField& f = st.f[v];
    f.n = f.flags = 0;
    f.sf = f.s1 = f.s2 = 0.0;
    f.si = 0;
    f.emin = f.emax = f.k = 0;
  }
}

// A step's selection words of this warp: word w of tile k at [k * kRedWords +
// i], w = warp - 1 + i * kScanConsumerWarps.
constexpr int kRedWords = 4;  // 1,024-row tiles: 32 words over 8 consumer warps
static_assert(kRedWords * kScanConsumerWarps * 32 >= kMaxTileRows, "a step's words per warp");

// One valid value of type T folded into `f`.
template <typename T>
__device__ __forceinline__ void reduce_one(const T x, bool want_sum, bool want_ext, bool want_m2, ReduceField& f) {
  constexpr bool kFloat = std::is_floating_point<T>::value;
  const double xd = (double)x;
  const bool nan = kFloat && xd != xd;
  ++f.n;
  if (want_sum) {
    if constexpr (kFloat) f.sf += xd;
    else f.si += (__int128)x;
  }
  if (want_ext) {
    if (nan) {
      f.flags |= 1u;
    } else {
      uint64_t e;
      if constexpr (kFloat) {
        const uint64_t u = xd == 0.0 ? 0ull : (uint64_t)__double_as_longlong(xd);
        e = (u >> 63) ? ~u : (u | 0x8000000000000000ull);
        if (xd == 0.0) f.flags |= signbit(xd) ? 4u : 2u;
      } else if constexpr (std::is_unsigned<T>::value) {
        e = (uint64_t)x;
      } else {
        e = (uint64_t)(int64_t)x ^ 0x8000000000000000ull;
      }
      if (~e > f.emin) f.emin = ~e;
      if (e > f.emax) f.emax = e;
    }
  }
  if (want_m2) {
    if (f.k == 0) f.k = (nan ? kCanonNaN : (uint64_t)__double_as_longlong(xd)) ^ kShiftTag;
    const double d = xd - __longlong_as_double((long long)(f.k ^ kShiftTag));
    f.s1 += d;
    f.s2 += d * d;
  }
}

// The quad path (ScanParams::fast_rows, 1,024-row tiles): consumer thread g
// takes rows 4g .. 4g + 3 of each of the step's tiles, the filter as one
// range test per row and four values per column from one vector load.
template <typename T>
__device__ __forceinline__ void reduce_quad_field(const ValField& vf, uint32_t ok, const uint64_t (&x)[4],
                                                  ReduceField& f) {
  const bool want_sum = vf.off_sum >= 0, want_ext = vf.off_min >= 0 || vf.off_max >= 0, want_m2 = vf.off_m2 >= 0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if ((ok >> i) & 1u) reduce_one<T>(from_bits<T>(x[i]), want_sum, want_ext, want_m2, f);
}

__device__ __forceinline__ void reduce_step_quad(const ScanParams& p, const Step& s, int nt, ReduceState& st) {
  const uint32_t g = threadIdx.x - 32;
#pragma unroll
  for (int k = 0; k < kTilesPerStep; ++k) {
    if (k >= nt) break;
    Quad q;
    q.tile = k;
    q.r0 = g * 4;
    q.staged = k ? s.staged[1] : s.staged[0];
    q.stage = k ? s.stage[1] : s.stage[0];
    q.start = k ? s.start[1] : s.start[0];
    const uint32_t n = k ? s.n[1] : s.n[0];
    const uint32_t left = n > q.r0 ? n - q.r0 : 0u;
    q.in = left >= 4 ? 0xFu : (1u << left) - 1u;
    const uint32_t sel = quad_select(p, q);
    if (!sel) continue;
    const uint32_t row0 = (uint32_t)(q.start + q.r0);
    st.first = min(st.first, row0 + (uint32_t)(__ffs(sel) - 1));
    st.last = max(st.last, row0 + (uint32_t)(32 - __clz(sel)));
    st.len += (uint32_t)__popc(sel);
#pragma unroll
    for (int v = 0; v < kReduceVals; ++v) {
      if (v >= p.n_vals) break;
      const ValField& vf = p.vals[v];
      uint64_t x[4];
      quad_load(p, q, vf.input, x);
      const uint32_t ok = quad_valid(p, q, vf.input) & sel;
      switch (vf.dtype) {
        case DFC_INT8: reduce_quad_field<int8_t>(vf, ok, x, st.f[v]); break;
        case DFC_INT16: reduce_quad_field<int16_t>(vf, ok, x, st.f[v]); break;
        case DFC_INT32: reduce_quad_field<int32_t>(vf, ok, x, st.f[v]); break;
        case DFC_INT64: reduce_quad_field<int64_t>(vf, ok, x, st.f[v]); break;
        case DFC_UINT8: reduce_quad_field<uint8_t>(vf, ok, x, st.f[v]); break;
        case DFC_UINT16: reduce_quad_field<uint16_t>(vf, ok, x, st.f[v]); break;
        case DFC_UINT32: reduce_quad_field<uint32_t>(vf, ok, x, st.f[v]); break;
        case DFC_UINT64: reduce_quad_field<uint64_t>(vf, ok, x, st.f[v]); break;
        case DFC_FLOAT32: reduce_quad_field<float>(vf, ok, x, st.f[v]); break;
        default: reduce_quad_field<double>(vf, ok, x, st.f[v]); break;
      }
    }
  }
}

// The lane's kept rows of value column v (type T) folded into `f`: one dtype
// dispatch per step instead of one per row.
template <typename T>
__device__ __forceinline__ void reduce_words(const ScanParams& p, const Step& s, int nt, int v,
                                             const uint32_t (&selw)[2 * kRedWords], ReduceField& f) {
  const ValField& vf = p.vals[v];
  const int c = vf.input;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool want_sum = vf.off_sum >= 0, want_ext = vf.off_min >= 0 || vf.off_max >= 0, want_m2 = vf.off_m2 >= 0;
#pragma unroll
  for (int k = 0; k < kTilesPerStep; ++k) {
    if (k >= nt) break;
    const unsigned char* vals = col_values(p, s, k, c);
    const uint32_t* valid = col_valid(p, s, k, c);
#pragma unroll
    for (int i = 0; i < kRedWords; ++i) {
      if (!((selw[k * kRedWords + i] >> lane) & 1u)) continue;
      const uint32_t r = (uint32_t)(warp - 1 + i * kScanConsumerWarps) * 32u + (uint32_t)lane;
      if (!valid_at(valid, r)) continue;
      reduce_one<T>(load_as<T>(vals, r), want_sum, want_ext, want_m2, f);
    }
  }
}

// The warp's words of this step: selection, row bookkeeping, then each value
// column by its type.
__device__ __forceinline__ void reduce_step(const ScanParams& p, const Step& s, int nt, uint32_t words,
                                            ReduceState& st) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t selw[2 * kRedWords];
#pragma unroll
  for (int k = 0; k < kTilesPerStep; ++k) {
#pragma unroll
    for (int i = 0; i < kRedWords; ++i) {
      const uint32_t w = (uint32_t)(warp - 1 + i * kScanConsumerWarps);
      selw[k * kRedWords + i] = (k < nt && w < words) ? select_word(p, s, k, w) : 0u;
      if ((selw[k * kRedWords + i] >> lane) & 1u) {
        const uint32_t row = (uint32_t)(s.start[k] + w * 32u + (uint32_t)lane);
        st.first = min(st.first, row);
        st.last = max(st.last, row + 1u);
        ++st.len;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < kReduceVals; ++v) {
    if (v >= p.n_vals) break;
    switch (p.vals[v].dtype) {
      case DFC_INT8: reduce_words<int8_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_INT16: reduce_words<int16_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_INT32: reduce_words<int32_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_INT64: reduce_words<int64_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_UINT8: reduce_words<uint8_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_UINT16: reduce_words<uint16_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_UINT32: reduce_words<uint32_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_UINT64: reduce_words<uint64_t>(p, s, nt, v, selw, st.f[v]); break;
      case DFC_FLOAT32: reduce_words<float>(p, s, nt, v, selw, st.f[v]); break;
      default: reduce_words<double>(p, s, nt, v, selw, st.f[v]); break;
    }
  }
}

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) { return __reduce_add_sync(0xffffffffu, v); }

// The warp's states folded into the CTA's record `rec` (every lane calls it).
__device__ __forceinline__ void reduce_flush(const ScanParams& p, ReduceState& st, const OwnRec& rec) {
  const int lane = threadIdx.x & 31;
  const uint32_t first = __reduce_min_sync(0xffffffffu, st.first);
  const uint32_t last = __reduce_max_sync(0xffffffffu, st.last);
  const uint32_t len = warp_sum_u32(st.len);
  if (len == 0) return;  // warp-uniform
  if (lane == 0) {
    rec.max_u32(kRecFirst, ~first);
    if (p.off_len >= 0) rec.add_u32(p.off_len, len);
    if (p.off_last >= 0) rec.max_u32(p.off_last, last);
  }
#pragma unroll
  for (int v = 0; v < kReduceVals; ++v) {
    if (v >= p.n_vals) break;
    const ValField& vf = p.vals[v];
    ReduceField& f = st.f[v];
    const uint32_t n = warp_sum_u32(f.n);
    const uint32_t flags = __reduce_or_sync(0xffffffffu, f.flags);
    if (lane == 0) {
      if (n) rec.add_u32(vf.off_count, n);
      if (flags) rec.or_u32(kRecFlags, flags << (3 * v));
    }
    if (vf.off_sum >= 0) {
      if (dt_float(vf.dtype)) {
        const double sm = warp_sum_f64(f.sf);
        if (lane == 0 && n) rec.add_f64(vf.off_sum, sm);
      } else {
        const __int128 exact = warp_sum_i128(f.si);
        if (lane == 0 && n) {
          if (vf.sum_kind == SUM_I64) {
            rec.add_u64(vf.off_sum, (uint64_t)(int64_t)exact);
          } else {
            const uint64_t add_lo = (uint64_t)exact, add_hi = (uint64_t)(exact >> 64);
            const uint64_t old = rec.add_u64(vf.off_sum, add_lo);
            const uint64_t hi_add = add_hi + ((old + add_lo) < old ? 1ull : 0ull);
            if (hi_add) rec.add_u64(vf.off_sum + 8, hi_add);
          }
        }
      }
    }
    if (vf.off_min >= 0) {
      const uint64_t m = warp_max_u64(f.emin);
      if (lane == 0 && m) rec.max_u64(vf.off_min, m);
    }
    if (vf.off_max >= 0) {
      const uint64_t m = warp_max_u64(f.emax);
      if (lane == 0 && m) rec.max_u64(vf.off_max, m);
    }
    if (vf.off_m2 >= 0) {
      // Moments re-centred on the first lane's K (sum (x - K)^2 = S2_t +
      // 2 d S1_t + n_t d^2, d = K_t - K), then on the record's.
      const uint32_t has = __ballot_sync(0xffffffffu, f.k != 0);
      if (has) {
        const uint64_t kw = __shfl_sync(0xffffffffu, f.k, __ffs(has) - 1);
        double s1 = 0.0, s2 = 0.0;
        if (f.k != 0) {
          const double d = __longlong_as_double((long long)(f.k ^ kShiftTag)) -
                           __longlong_as_double((long long)(kw ^ kShiftTag));
          const double dn = (double)f.n;
          s1 = d == 0.0 ? f.s1 : f.s1 + dn * d;
          s2 = d == 0.0 ? f.s2 : f.s2 + 2.0 * d * f.s1 + dn * d * d;
        }
        s1 = warp_sum_f64(s1);
        s2 = warp_sum_f64(s2);
        if (lane == 0) {
          uint64_t kr = rec.ld_u64(vf.off_shift);
          if (kr == 0) {
            const uint64_t prev = rec.cas_u64(vf.off_shift, 0ull, kw);
            kr = prev == 0 ? kw : prev;
          }
          const double d = __longlong_as_double((long long)(kw ^ kShiftTag)) -
                           __longlong_as_double((long long)(kr ^ kShiftTag));
          const double dn = (double)n;
          rec.add_f64(vf.off_m2, d == 0.0 ? s2 : s2 + 2.0 * d * s1 + dn * d * d);
        }
      }
    }
  }
}

// The scan body, specialised by table regime R (kScan*): each regime's
// kernel carries only its own table code, which keeps the instruction
// footprint of the hot loop small.
template <int R>
__device__ __forceinline__ void scan_body(const ScanParams& p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
  uint64_t* empty = full + S;
  __shared__ ClaimState s_claim;
  __shared__ volatile uint32_t s_abort;
  __shared__ uint32_t s_used;
  // Compacted rows of a step, three buffers: a step's count is reset two
  // steps ahead of its reuse, between barriers.
  __shared__ uint32_t s_nsel[3];
  __shared__ uint16_t s_idx[3][kStepRows];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kScanConsumerWarps);
    }
    fence_mbar_init();
    s_claim.ticket = 0;
    s_abort = 0;
    s_used = 0;
    s_nsel[0] = s_nsel[1] = s_nsel[2] = 0;
  }
  if (threadIdx.x < kChunkRing) s_claim.ring[threadIdx.x] = ~0ull;
  SmemTable st{nullptr, nullptr, &s_used, R == kScanCluster ? p.smem_cluster : 1u};
  if (R != kScanGlobal && p.smem_slots) {
    st.keys = reinterpret_cast<unsigned long long*>(smem + p.smem_keys_off);
    st.recs = smem + p.smem_recs_off;
    for (uint32_t s = threadIdx.x; s < p.smem_slots; s += blockDim.x) st.keys[s] = kEmpty;
    uint4* recs = reinterpret_cast<uint4*>(st.recs);
    const uint32_t n16 = p.smem_slots * (uint32_t)p.rec_stride / 16;
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) recs[i] = make_uint4(0, 0, 0, 0);
    // No key: the one group's key word is 0, its record slot 0.
    if (R == kScanReduce && threadIdx.x == 0) st.keys[0] = 0ull;
  }
  __syncthreads();
  // A cluster table: every share is initialised before any CTA probes it.
  if (R == kScanCluster) cluster_sync_all();

  const uint64_t T = (uint64_t)p.tile_rows;
  if (warp == 0) {
    if (lane == 0) produce_tiles(p, smem, full, empty, &s_abort, p.n_stage, (uint32_t)p.stage_tx);
  } else {
    const uint32_t shift = 31 - __clz((uint32_t)p.tile_rows);
    const uint32_t words = (uint32_t)(T / 32);
    uint32_t it = 0;   // tiles consumed
    uint32_t stp = 0;  // steps
    ReduceState red;
    if (R == kScanReduce) reduce_init(red);
    for (uint64_t t = blockIdx.x; t < p.tiles; t += (uint64_t)kTilesPerStep * gridDim.x, ++stp) {
      Step s;
      int nt = 0;
      bool failed = false;
#pragma unroll
      for (int k = 0; k < kTilesPerStep; ++k) {
        const uint64_t tk = t + (uint64_t)k * gridDim.x;
        s.n[k] = 0;
        s.start[k] = 0;
        s.staged[k] = false;
        s.stage[k] = smem;
        if (tk >= p.tiles || failed) continue;
        const uint32_t x = ring_pos(it, (uint32_t)k, (uint32_t)S), sid = ring_slot(x, (uint32_t)S), ph = ring_phase(x, (uint32_t)S);
        if (!mbar_wait_bounded(&full[sid], ph, kWaitLimit)) {
          atomicOr(p.status, ST_TIMEOUT);
          s_abort = 1;
          failed = true;
          continue;
        }
        s.stage[k] = smem + (size_t)sid * p.stage_bytes;
        s.start[k] = tk * T;
        s.staged[k] = p.use_tma && tk < p.full_tiles;
        const uint64_t left = p.rows - s.start[k];
        s.n[k] = (uint32_t)(left < T ? left : T);
        ++nt;
      }
      if constexpr (R == kScanReduce) {
        // Each lane folds its kept rows into registers.
        if (!failed) {
          if (p.fast_rows) reduce_step_quad(p, s, nt, red);
          else reduce_step(p, s, nt, words, red);
        }
        if (consumer_sync_or(failed || s_abort)) {
          s_abort = 1;
          break;
        }
        __syncwarp();
        for (int k = 0; k < nt; ++k)
          if (lane == 0) mbar_arrive(&empty[ring_slot(ring_pos(it, (uint32_t)k, (uint32_t)S), (uint32_t)S)]);
        it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
        continue;
      }
      // 1 + 2: selection words and compaction into s_idx[b].
      const uint32_t b = stp % 3u;
      if (!failed) {
        for (int k = 0; k < nt; ++k) {
          for (uint32_t w = (uint32_t)(warp - 1); w < words; w += kScanConsumerWarps) {
            const uint32_t bits = select_word(p, s, k, w);
            uint32_t off = 0;
            if (lane == 0 && bits) off = atomicAdd(&s_nsel[b], (uint32_t)__popc(bits));
            off = __shfl_sync(0xffffffffu, off, 0);
            if ((bits >> lane) & 1u)
              s_idx[b][off + __popc(bits & ((1u << lane) - 1u))] = (uint16_t)(((uint32_t)k << shift) | (w * 32 + lane));
          }
        }
      }
      // Every consumer warp takes the same exit decision at this barrier.
      const bool stop = consumer_sync_or(failed || s_abort);
      const uint32_t nsel = s_nsel[b];
      if (threadIdx.x == 32) s_nsel[(b + 2u) % 3u] = 0;  // read last step, written two steps on
      if (stop) {
        s_abort = 1;
        break;
      }
      // 3 - 5 over the compacted rows.
      for (uint32_t base = 0; base < nsel; base += kPassRows)
        consume_rows<R>(p, s, s_idx[b], nsel, base, shift, &s_claim, p.smem_slots ? &st : nullptr);
      __syncwarp();
      for (int k = 0; k < nt; ++k)
        if (lane == 0) mbar_arrive(&empty[ring_slot(ring_pos(it, (uint32_t)k, (uint32_t)S), (uint32_t)S)]);
      it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
    }
    if (R == kScanReduce && p.smem_slots && !s_abort) reduce_flush(p, red, OwnRec{st.recs});
  }
  __syncthreads();
  // A cluster table: no CTA touches another's share after this barrier, so
  // each merges its own share and may exit.
  if (R == kScanCluster) cluster_sync_all();
  if (R != kScanGlobal && p.smem_slots && !s_abort) {
    // The share's records find their global records through the same
    // warp-synchronous claim rounds as the rows (packed keys only; no thread
    // waits on another's claim).  Every thread runs the same passes, kR slots
    // each; CTAs start at different slots (every table hashes a key to the
    // same slot), so fewer of them meet on one global record at a time.
    const uint32_t mask = p.smem_slots - 1;
    const uint32_t rot = (uint32_t)mix64(blockIdx.x + 0x51ull) & mask;
    const uint32_t per = blockDim.x * (uint32_t)kR;
    for (uint32_t base = 0; base < p.smem_slots; base += per) {
      uint32_t rows[kR], gid[kR], slot[kR];
      uint64_t kw[kR];
      bool sel[kR];
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        const uint32_t i = base + threadIdx.x + (uint32_t)j * blockDim.x;
        slot[j] = (i + rot) & mask;
        kw[j] = i < p.smem_slots ? st.keys[slot[j]] : kEmpty;
        const uint32_t first_enc =
            kw[j] != kEmpty ? *reinterpret_cast<const uint32_t*>(st.recs + (size_t)slot[j] * p.rec_stride + kRecFirst) : 0u;
        sel[j] = first_enc != 0;
        rows[j] = ~first_enc;
      }
      resolve_packed(p, rows, sel, kw, gid, &s_claim);
#pragma unroll
      for (int j = 0; j < kR; ++j)
        if (sel[j]) merge_into(p, st.recs + (size_t)slot[j] * p.rec_stride, gid[j]);
    }
  }
}

__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel_global(const __grid_constant__ ScanParams p) {
  scan_body<kScanGlobal>(p);
}
__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel_own(const __grid_constant__ ScanParams p) {
  scan_body<kScanOwn>(p);
}
__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel_cluster(const __grid_constant__ ScanParams p) {
  scan_body<kScanCluster>(p);
}
__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel_reduce(const __grid_constant__ ScanParams p) {
  scan_body<kScanReduce>(p);
}

// Merges one shared-memory record into global record `gid` (function.mojo:
// 1559-1779 `combine`; the shifted square sums are re-centred on the global
// record's K; compensated FP32 pairs enter as FP64 values).
__device__ void merge_into(const ScanParams& p, const unsigned char* src, uint32_t gid) {
  const uint32_t first_enc = *reinterpret_cast<const uint32_t*>(src + kRecFirst);
  unsigned char* dst = record_at(p, gid);
  if (p.track_first) atomicMax(reinterpret_cast<uint32_t*>(dst + kRecFirst), first_enc);
  if (p.off_len >= 0) red_add_u32(dst + p.off_len, *reinterpret_cast<const uint32_t*>(src + p.off_len));
  if (p.off_last >= 0) atomicMax(reinterpret_cast<uint32_t*>(dst + p.off_last), *reinterpret_cast<const uint32_t*>(src + p.off_last));
  const uint32_t flags = *reinterpret_cast<const uint32_t*>(src + kRecFlags);
  if (flags) red_or_u32(dst + kRecFlags, flags);
  for (int v = 0; v < p.n_vals; ++v) {
    const ValField& f = p.vals[v];
    const uint32_t n = *reinterpret_cast<const uint32_t*>(src + f.off_count);
    if (f.off_min >= 0) {
      const uint64_t m = *reinterpret_cast<const uint64_t*>(src + f.off_min);
      if (m) red_max_u64(dst + f.off_min, m);
    }
    if (f.off_max >= 0) {
      const uint64_t m = *reinterpret_cast<const uint64_t*>(src + f.off_max);
      if (m) red_max_u64(dst + f.off_max, m);
    }
    if (n == 0) continue;
    red_add_u32(dst + f.off_count, n);
    const bool comp = (p.comp_mask >> v) & 1u;
    if (f.off_sum >= 0) {
      if (comp) {
        red_add_f64(dst + f.off_sum, pair_value(src + f.off_sum));
      } else if (f.sum_kind == SUM_F64) {
        red_add_f64(dst + f.off_sum, *reinterpret_cast<const double*>(src + f.off_sum));
      } else if (f.sum_kind == SUM_I64) {
        red_add_u64(dst + f.off_sum, *reinterpret_cast<const uint64_t*>(src + f.off_sum));
      } else {
        const uint64_t lo = *reinterpret_cast<const uint64_t*>(src + f.off_sum);
        const uint64_t hi = *reinterpret_cast<const uint64_t*>(src + f.off_sum + 8);
        const uint64_t old = atomicAdd(reinterpret_cast<unsigned long long*>(dst + f.off_sum), lo);
        const uint64_t hi_add = hi + ((old + lo) < old ? 1ull : 0ull);
        if (hi_add) red_add_u64(dst + f.off_sum + 8, hi_add);
      }
    }
    if (f.off_m2 >= 0) {
      // sum (x - K)^2 = S2_l + 2 d S1_l + n d^2,  d = K_l - K,  S1_l = sum x - n K_l.
      const uint64_t kl_enc = *reinterpret_cast<const uint64_t*>(src + f.off_shift);
      uint64_t kg_enc = ld_cg_u64(dst + f.off_shift);
      if (kg_enc == 0) {
        const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(dst + f.off_shift), 0ull, kl_enc);
        kg_enc = prev == 0 ? kl_enc : prev;
      }
      const double kl = __longlong_as_double((long long)(kl_enc ^ kShiftTag));
      const double kg = __longlong_as_double((long long)(kg_enc ^ kShiftTag));
      const double dn = (double)n;
      double s1;
      if (dt_float(f.dtype)) {
        s1 = (comp ? pair_value(src + f.off_sum) : *reinterpret_cast<const double*>(src + f.off_sum)) - dn * kl;
      } else {
        __int128 isum;
        if (f.sum_kind == SUM_I64) isum = (__int128)*reinterpret_cast<const long long*>(src + f.off_sum);
        else isum = (__int128)(((unsigned __int128)*reinterpret_cast<const uint64_t*>(src + f.off_sum + 8) << 64) |
                               *reinterpret_cast<const uint64_t*>(src + f.off_sum));
        s1 = (double)(isum - (__int128)n * (__int128)kl);
      }
      const double d = kl - kg;
      const double s2 = comp ? pair_value(src + f.off_m2) : *reinterpret_cast<const double*>(src + f.off_m2);
      red_add_f64(dst + f.off_m2, d == 0.0 ? s2 : s2 + 2.0 * d * s1 + dn * d * d);
    }
  }
}

// ===========================================================================
// Radix-partitioned regime (many groups).
//
// With millions of groups the global table and records outgrow L2, and every
// probe, read-set load and atomic of the global regime is an HBM round trip
// (HBM serves about 50 G random 16-byte loads and 25 G random atomics a
// second).  This regime turns the group-by into streaming passes and on-chip
// work:
//   count    the key and filter columns only: the selected rows per
//            partition (shared-memory counters, one global add per CTA and
//            partition at the end);
//   offsets  the partitions' exclusive prefix: each partition's range of
//            part_buf;
//   pass A   every column: each selected row is written to the next place of
//            its partition's range; a warp's rows of one partition reserve
//            their places with one atomic on the partition's cursor.  The
//            cursors of all partitions are a few tens of KB, so they and the
//            partitions' write frontiers stay in L2, which merges the rows
//            into whole lines before they reach HBM;
//   pass B   one partition at a time per CTA: its rows (read once, streaming)
//            fold into a shared-memory table sized so a partition's groups
//            fit it; the live records are then appended to `records`.
// Partitions are sized from the group estimate; a partition whose groups do
// not fit the table raises CAP_AGG_TABLE and the host reruns with more.
// ===========================================================================

__device__ __forceinline__ void part_check(const ScanParams& p, uint32_t code) { atomicOr(p.status + 2, code); }

// The key word folded to 32 bits (its high half multiplied in), shared by the
// partition hash and pass B's slot hash.
__device__ __forceinline__ uint32_t fold_key(uint64_t kw) {
  return (uint32_t)kw ^ ((uint32_t)(kw >> 32) * 0x9E3779B1u);
}

// Partition: the top part_bits bits of a multiplicative hash of the folded
// key word (one multiply per row in the streaming passes).
__device__ __forceinline__ uint32_t partition_of(const ScanParams& p, uint64_t kw) {
  return (fold_key(kw) * 0x85EBCA77u) >> (32 - p.part_bits);
}

__device__ __forceinline__ void raise_capacity(const ScanParams& p, uint32_t what) {
  atomicOr(p.status, ST_CAPACITY);
  atomicOr(p.status + 1, what);
}

// The partition passes need no compaction: consumer warp w owns words
// w, w + 16, ... of every tile (kPR of them at most), and each lane handles
// its own row of each word.  Selection is a ballot per word; unselected rows
// are masked off.  The warps pass no CTA barrier while streaming.
constexpr int kPR = kMaxTileRows / 32 / kPartWarps;  // rows a lane holds per tile
static_assert(kPR >= 1, "a consumer warp owns whole words");

constexpr int kSR = kPR * kTilesPerStep;  // rows a lane holds per step (two tiles)

// Waits for the tiles of one step (this CTA's tiles t and t + gridDim.x,
// its it-th and it+1-th): false when a wait gave up (ST_TIMEOUT raised).
__device__ __forceinline__ bool step_wait(const ScanParams& p, unsigned char* smem, uint64_t* full, uint64_t t,
                                          uint32_t it, volatile uint32_t* s_abort, Step& s, int& nt) {
  const int S = p.stages;
  const uint64_t T = (uint64_t)p.tile_rows;
  nt = 0;
#pragma unroll
  for (int k = 0; k < kTilesPerStep; ++k) {
    const uint64_t tk = t + (uint64_t)k * gridDim.x;
    s.n[k] = 0;
    s.start[k] = 0;
    s.staged[k] = false;
    s.stage[k] = smem;
    if (tk >= p.tiles) continue;
    const uint32_t x = ring_pos(it, (uint32_t)k, (uint32_t)S), sid = ring_slot(x, (uint32_t)S), ph = ring_phase(x, (uint32_t)S);
    if (*s_abort || !mbar_wait_bounded(&full[sid], ph, kWaitLimit)) {
      atomicOr(p.status, ST_TIMEOUT);
      *s_abort = 1;
      return false;
    }
    s.stage[k] = smem + (size_t)sid * p.stage_bytes;
    s.start[k] = tk * T;
    s.staged[k] = p.use_tma && tk < p.full_tiles;
    const uint64_t left = p.rows - s.start[k];
    s.n[k] = (uint32_t)(left < T ? left : T);
    ++nt;
  }
  return true;
}

// This lane's rows of the step: tile j / kPR, word (warp - 1) + (j % kPR) * 16.
__device__ __forceinline__ void step_rows(const ScanParams& p, const Step& s, int nt, RowRef (&x)[kSR],
                                          uint32_t (&bits)[kSR]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t words = (uint32_t)p.tile_rows / 32;
#pragma unroll
  for (int j = 0; j < kSR; ++j) {
    const int tile = j / kPR;
    const uint32_t w = (uint32_t)(warp - 1) + (uint32_t)(j % kPR) * kPartWarps;
    bits[j] = (w < words && tile < nt) ? select_word(p, s, tile, w) : 0u;
    x[j].tile = (uint32_t)tile;
    x[j].r = w * 32 + lane;
    x[j].on = (bits[j] >> lane) & 1u;
  }
}

// Releases the step's stages (each consumer warp arrives once per tile).
__device__ __forceinline__ void step_release(const ScanParams& p, uint64_t* empty, uint32_t it, int nt) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < nt; ++k) mbar_arrive(&empty[ring_slot(ring_pos(it, (uint32_t)k, (uint32_t)p.stages), (uint32_t)p.stages)]);
}

// Ring set-up shared by the counting pass and pass A.
__device__ __forceinline__ void ring_init(int S, uint64_t* full, uint64_t* empty, volatile uint32_t* s_abort) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kPartWarps);
    }
    fence_mbar_init();
    *s_abort = 0;
  }
  __syncthreads();
}


// Packed key words of the quad's rows (packed key mode).
__device__ __forceinline__ void quad_keys(const ScanParams& p, const Quad& q, uint64_t (&kw)[4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) kw[i] = 0;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    uint64_t x[4];
    quad_load(p, q, f.input, x);
    const uint32_t valid = f.null_bit >= 0 ? quad_valid(p, q, f.input) : 0xFu;
#pragma unroll
    for (int i = 0; i < 4; ++i) kw[i] |= ((valid >> i) & 1u) ? (x[i] << f.shift) : (1ull << f.null_bit);
  }
}

// Counting pass.  Dynamic shared memory: the ring (p.stages stages of
// p.stage_bytes, only the key and filter columns staged), its mbarriers,
// then one counter per partition.
template <bool kQuad>
__device__ __forceinline__ void count_body(const ScanParams& p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
  uint64_t* empty = full + S;
  uint32_t* s_count = reinterpret_cast<uint32_t*>(empty + S);
  __shared__ volatile uint32_t s_abort;
  const uint32_t nparts = 1u << p.part_bits;
  for (uint32_t q = threadIdx.x; q < nparts; q += blockDim.x) s_count[q] = 0;
  ring_init(S, full, empty, &s_abort);
  if ((threadIdx.x >> 5) == 0) {
    if ((threadIdx.x & 31) == 0) produce_tiles(p, smem, full, empty, &s_abort, p.n_stage_count, (uint32_t)p.stage_tx_count);
  } else {
    uint32_t it = 0;
    for (uint64_t t = blockIdx.x; t < p.tiles; t += (uint64_t)kTilesPerStep * gridDim.x) {
      Step s;
      int nt;
      if (!step_wait(p, smem, full, t, it, &s_abort, s, nt)) break;
      if constexpr (kQuad) {
        const Quad q = quad_of(s, nt);
        uint32_t sel = 0;
        uint64_t kw[4];
        if (q.tile >= 0) {
          sel = quad_select(p, q);
          quad_keys(p, q, kw);
        }
        step_release(p, empty, it, nt);
        it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if ((sel >> i) & 1u) atomicAdd(&s_count[partition_of(p, kw[i])], 1u);
      } else {
        RowRef x[kSR];
        uint32_t bits[kSR];
        uint64_t kw[kSR];
        step_rows(p, s, nt, x, bits);
        key_words<kSR>(p, s, x, kw);
        step_release(p, empty, it, nt);
        it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
#pragma unroll
        for (int j = 0; j < kSR; ++j)
          if (x[j].on) atomicAdd(&s_count[partition_of(p, kw[j])], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < nparts; q += blockDim.x) {
    const uint32_t c = s_count[q];
    if (c) atomicAdd(&p.part_totals[q], c);
  }
}

__global__ void __launch_bounds__(kPartThreads, 1) partition_count(const __grid_constant__ ScanParams p) {
  count_body<false>(p);
}
__global__ void __launch_bounds__(kPartThreads, 1) partition_count_quad(const __grid_constant__ ScanParams p) {
  count_body<true>(p);
}

// The partitions' exclusive prefix (one CTA of 1024 threads), and pass B's
// order: partitions holding more than four times the average rows (hot keys)
// first, so none of them starts late and leaves one CTA working alone at the
// end.  Both walk the partitions in rows of 1024 (thread t takes partition
// r * 1024 + t), so every load and store of a warp is one contiguous run:
// a block scan per row with a running carry, then one shared-memory atomic
// per warp and class for the order, the lanes ranked by their ballot.
__global__ void __launch_bounds__(1024) partition_offsets(const __grid_constant__ ScanParams p) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_next_big, s_small;
  const uint32_t nparts = 1u << p.part_bits;
  const uint32_t B = blockDim.x;  // 1024: a multiple of 32
  const uint32_t nw = B / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t below = (1u << lane) - 1u;
  uint32_t carry = 0;  // rows of the partitions before this row of partitions
  for (uint32_t r0 = 0; r0 < nparts; r0 += B) {
    const uint32_t q = r0 + threadIdx.x;
    const uint32_t v = q < nparts ? p.part_totals[q] : 0u;
    uint32_t x = v;  // inclusive prefix inside the warp
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const uint32_t w = lane < (int)nw ? s_warp[lane] : 0u;
      uint32_t z = w;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      if (lane < (int)nw) s_warp[lane] = z - w;  // exclusive over the warps
    }
    __syncthreads();
    const uint32_t ex = carry + s_warp[warp] + x - v;
    if (q < nparts) {
      p.part_start[q] = ex;
      p.part_range[q] = make_uint2(ex, v);
    }
    // The next row's carry: the last thread's inclusive prefix (after every
    // thread has read its warp's offset).
    __syncthreads();
    if (threadIdx.x == B - 1) s_warp[0] = ex + v;
    __syncthreads();
    carry = s_warp[0];
    __syncthreads();
  }
  const uint32_t total = carry;
  if (threadIdx.x == 0) {
    *p.part_kept = total;
    s_next_big = 0;
  }
  const uint64_t big_rows = 4ull * total / nparts;
  uint32_t nbig = 0;
  for (uint32_t q = threadIdx.x; q < nparts; q += B)
    if (p.part_totals[q] > big_rows) ++nbig;
  nbig = __reduce_add_sync(0xffffffffu, nbig);
  if (lane == 0) s_warp[warp] = nbig;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t w = 0; w < nw; ++w) t += s_warp[w];
    s_small = t;  // the small partitions follow the big ones
  }
  __syncthreads();
  for (uint32_t r0 = 0; r0 < nparts; r0 += B) {
    const uint32_t q = r0 + threadIdx.x;
    const bool valid = q < nparts;
    const bool big = valid && p.part_totals[q] > big_rows;
    const uint32_t mb = __ballot_sync(0xffffffffu, big), ms = __ballot_sync(0xffffffffu, valid && !big);
    uint32_t bb = 0, bs = 0;
    if (lane == 0) {
      if (mb) bb = atomicAdd(&s_next_big, (uint32_t)__popc(mb));
      if (ms) bs = atomicAdd(&s_small, (uint32_t)__popc(ms));
    }
    bb = __shfl_sync(0xffffffffu, bb, 0);
    bs = __shfl_sync(0xffffffffu, bs, 0);
    if (!valid) continue;
    const uint32_t at = big ? bb + (uint32_t)__popc(mb & below) : bs + (uint32_t)__popc(ms & below);
    if (at < nparts) p.part_order[at] = q;
    else part_check(p, CHK_PART);
  }
}

// Pass A.  Dynamic shared memory: the ring of every staged column and its
// mbarriers.  Each selected row goes to part_start[q] + a place reserved on
// q's cursor by one atomic per row; the reservations of all of a lane's row
// slots are in flight at once.  (With thousands of partitions the lanes of a
// warp rarely share one, and reserving per warp group with __match_any_sync
// cost more than it saved: 1.91 against 1.69 ms on 100M rows.)
// RS row slots per lane: kSR rows (generic path) or a quad.
template <int RS>
__device__ __forceinline__ void place_rows(const ScanParams& p, const bool (&on)[RS], const uint64_t (&kw)[RS],
                                           unsigned long long* (&dst)[RS]) {
  const uint32_t nparts = 1u << p.part_bits;
  uint32_t q[RS], base[RS];
#pragma unroll
  for (int j = 0; j < RS; ++j) q[j] = on[j] ? partition_of(p, kw[j]) : 0u;
#pragma unroll
  for (int j = 0; j < RS; ++j) base[j] = on[j] && q[j] < nparts ? atomicAdd(&p.part_cursor[q[j]], 1u) : 0u;
#pragma unroll
  for (int j = 0; j < RS; ++j) {
    dst[j] = nullptr;
    if (!on[j]) continue;
    const uint32_t at = base[j];
    const uint2 range = q[j] < nparts ? __ldg(p.part_range + q[j]) : make_uint2(0u, 0u);  // {start, total}
    if (q[j] >= nparts || at >= range.y) {
      part_check(p, CHK_RANGE);
      continue;
    }
    dst[j] = p.part_buf + ((uint64_t)range.x + at) * p.part_words;
  }
}

// The row's key word, row word and first value, stored together once the
// row's place is known (the other value columns are already written):
// consecutive stores to one row let L2 merge them before the line leaves.
// 24-byte rows (one value column) take two stores: of consecutive rows one
// starts on a 16-byte boundary (its first two words go as one vector) and the
// next on 8 mod 16 (its last two words do).  part_buf is 256-byte aligned.
__device__ __forceinline__ void write_row(const ScanParams& p, unsigned long long* dst, uint64_t kw, uint32_t vflags,
                                          uint32_t row, uint64_t val0) {
  const uint64_t w1 = (uint64_t)row | ((uint64_t)vflags << 32);
  if (p.part_words == 3) {
    if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
      *reinterpret_cast<ulonglong2*>(dst) = make_ulonglong2(kw, w1);
      dst[2] = val0;
    } else {
      dst[0] = kw;
      *reinterpret_cast<ulonglong2*>(dst + 1) = make_ulonglong2(w1, val0);
    }
    return;
  }
  dst[0] = kw;
  dst[1] = w1;
  if (p.n_vals > 0) dst[2] = val0;
}

template <bool kQuad>
__device__ __forceinline__ void place_body(const ScanParams& p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
  uint64_t* empty = full + S;
  __shared__ volatile uint32_t s_abort;
  ring_init(S, full, empty, &s_abort);
  if ((threadIdx.x >> 5) == 0) {
    if ((threadIdx.x & 31) == 0) produce_tiles(p, smem, full, empty, &s_abort, p.n_stage, (uint32_t)p.stage_tx);
    return;
  }
  uint32_t it = 0;
  for (uint64_t t = blockIdx.x; t < p.tiles; t += (uint64_t)kTilesPerStep * gridDim.x) {
    Step s;
    int nt = 0;
    if (!step_wait(p, smem, full, t, it, &s_abort, s, nt)) break;
    if constexpr (kQuad) {
      const Quad q = quad_of(s, nt);
      uint32_t sel = 0;
      uint64_t kw[4] = {0, 0, 0, 0};
      if (q.tile >= 0) {
        sel = quad_select(p, q);
        if (sel) quad_keys(p, q, kw);
      }
      bool on[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) on[i] = (sel >> i) & 1u;
      unsigned long long* dst[4];
      place_rows<4>(p, on, kw, dst);
      uint32_t vflags[4] = {0, 0, 0, 0};
      uint64_t val0[4] = {0, 0, 0, 0};  // the first value column, written with the row's first words
      if (sel) {
        for (int v = 0; v < p.n_vals; ++v) {
          const int c = p.vals[v].input;
          uint64_t x[4];
          quad_load(p, q, c, x);
          const uint32_t valid = quad_valid(p, q, c);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            if (!dst[i]) continue;
            const bool ok = (valid >> i) & 1u;
            vflags[i] |= (uint32_t)ok << v;
            if (v == 0) val0[i] = ok ? x[i] : 0ull;
            else dst[i][2 + v] = ok ? x[i] : 0ull;
          }
        }
      }
      const uint64_t row0 = q.start + q.r0;
      step_release(p, empty, it, nt);
      it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (dst[i]) write_row(p, dst[i], kw[i], vflags[i], (uint32_t)(row0 + i), val0[i]);
    } else {
      RowRef x[kSR];
      uint32_t bits[kSR];
      uint64_t kw[kSR];
      step_rows(p, s, nt, x, bits);
      key_words<kSR>(p, s, x, kw);
      bool on[kSR];
#pragma unroll
      for (int j = 0; j < kSR; ++j) on[j] = x[j].on;
      unsigned long long* dst[kSR];
      place_rows<kSR>(p, on, kw, dst);
      uint32_t vflags[kSR] = {};
      uint64_t val0[kSR] = {};
      for (int v = 0; v < p.n_vals; ++v) {
        const int c = p.vals[v].input;
        const ColRef cr = col_ref(p, s, c);
        const int size = p.cols[c].size;
#pragma unroll
        for (int j = 0; j < kSR; ++j) {
          if (!dst[j]) continue;
          const bool ok = rvalid(cr, x[j]);
          vflags[j] |= (uint32_t)ok << v;
          const uint64_t b = ok ? load_bits(rv(cr, x[j]), size, x[j].r) : 0ull;
          if (v == 0) val0[j] = b;
          else dst[j][2 + v] = b;
        }
      }
      step_release(p, empty, it, nt);
      it = ring_pos(it, (uint32_t)nt, (uint32_t)p.stages);
#pragma unroll
      for (int j = 0; j < kSR; ++j)
        if (dst[j]) write_row(p, dst[j], kw[j], vflags[j], (uint32_t)(s.start[x[j].tile] + x[j].r), val0[j]);
    }
  }
}

__global__ void __launch_bounds__(kPartThreads, 1) partition_kernel(const __grid_constant__ ScanParams p) {
  place_body<false>(p);
}
__global__ void __launch_bounds__(kPartThreads, 1) partition_kernel_quad(const __grid_constant__ ScanParams p) {
  place_body<true>(p);
}

// ---------------------------------------------------------------------------
// Pass B.  The table: agg_slots records (any count) in dynamic shared memory,
// the key word at kRecKey (all ones = free), every other field at its
// identity (zero), and one more record for the all-ones key word.  Records
// are rec_stride bytes, laid out agg_stride() = rec_stride + 8 bytes apart: a
// stride of 8 mod 16 bytes spreads the same field of random slots over every
// bank pair (a 64-byte stride put all of a warp's accesses to one field in
// two banks).  A row finds its record by linear probing from a hash of its
// key word (independent of the partition hash).  A record is live once a row
// set its first row; every claimed slot is, and claims append their slot to
// a list after the table (S entries), so the copy-out visits only them.
// ---------------------------------------------------------------------------
__device__ __forceinline__ size_t agg_stride(const ScanParams& p) { return (size_t)p.rec_stride + 8; }

__device__ __forceinline__ void reset_record(unsigned char* rec, size_t rs) {
  unsigned long long* r = reinterpret_cast<unsigned long long*>(rec);
  r[0] = kEmpty;
  for (size_t q = 1; q < rs / 8; ++q) r[q] = 0ull;
}

// The shared-memory record of key word `kw` (claimed if new); false when the
// table is seven-eighths full and the key is not in it.  Below that fill a
// free slot always exists, so the probe ends within agg_slots steps.
__device__ __forceinline__ bool agg_probe(const ScanParams& p, unsigned char* table, uint32_t* used, uint32_t* live,
                                          uint64_t kw, unsigned char*& rec) {
  const uint32_t S = p.agg_slots;
  const size_t rs = agg_stride(p);
  if (kw == kEmpty) {
    rec = table + (size_t)S * rs;
    return true;
  }
  uint32_t h = fold_key(kw) ^ 0x632BE59Bu;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  // First slot: the hash scaled to [0, S) (S need not be a power of two).
  uint32_t s = (uint32_t)(((uint64_t)h * S) >> 32);
  for (uint32_t probe = 0; probe < S; ++probe) {
    unsigned long long* key = reinterpret_cast<unsigned long long*>(table + (size_t)s * rs + kRecKey);
    const unsigned long long k = *reinterpret_cast<volatile unsigned long long*>(key);
    bool hit = k == kw;
    if (!hit && k == kEmpty) {
      if (*reinterpret_cast<volatile uint32_t*>(used) >= S - S / 8) return false;
      const unsigned long long prev = atomicCAS(key, kEmpty, kw);
      if (prev == kEmpty) {
        // Each slot is claimed once, so fewer than S claims exist.
        const uint32_t at = atomicAdd(used, 1u);
        if (at < S) live[at] = s;
        else part_check(p, CHK_SLOT);
      }
      hit = prev == kEmpty || prev == kw;
    }
    if (hit) {
      rec = table + (size_t)s * rs;
      return true;
    }
    s = s + 1 == S ? 0u : s + 1;
  }
  return false;
}

constexpr int kBR = 2;  // rows a pass B thread holds in flight

// kBR rows of a partition per thread: rows first + j * stride (< n).  Each
// row updates its shared-memory record with per-lane atomics (the global
// regime's update_rows on shared records); a warp's largest group of rows on
// one record (a hot key) is first folded by butterflies (collapse_largest),
// one atomic per field.
__device__ __forceinline__ void fold_rows(const ScanParams& p, unsigned char* table, uint32_t* used, uint32_t* live,
                                          const unsigned long long* rows, uint32_t n, uint32_t first, uint32_t stride) {
  const uint32_t W = p.part_words;
  bool on[kBR];
  uint64_t kw[kBR], v0[kBR];
  uint32_t row[kBR], vf[kBR];
  const unsigned long long* src[kBR];
#pragma unroll
  for (int j = 0; j < kBR; ++j) {
    const uint32_t i = first + (uint32_t)j * stride;
    on[j] = i < n;
    src[j] = rows + (uint64_t)(on[j] ? i : 0) * W;
    kw[j] = v0[j] = 0;
    row[j] = vf[j] = 0;
    if (!on[j]) continue;
    uint64_t w1;
    if (W == 3) {
      // 24-byte rows: a 16-byte load of the aligned word pair and one 8-byte load.
      if ((reinterpret_cast<uintptr_t>(src[j]) & 15u) == 0) {
        const ulonglong2 a = __ldcs(reinterpret_cast<const ulonglong2*>(src[j]));
        kw[j] = a.x;
        w1 = a.y;
        v0[j] = __ldcs(src[j] + 2);
      } else {
        kw[j] = __ldcs(src[j]);
        const ulonglong2 b = __ldcs(reinterpret_cast<const ulonglong2*>(src[j] + 1));
        w1 = b.x;
        v0[j] = b.y;
      }
    } else {
      kw[j] = __ldcs(src[j]);
      w1 = __ldcs(src[j] + 1);
      if (p.n_vals > 0) v0[j] = __ldcs(src[j] + 2);  // the first value column, loaded with the rest
    }
    row[j] = (uint32_t)w1;
    vf[j] = (uint32_t)(w1 >> 32);
  }
  unsigned char* recs[kBR];
  bool lost = false;
#pragma unroll
  for (int j = 0; j < kBR; ++j) {
    recs[j] = table;
    const bool hit = on[j] && agg_probe(p, table, used, live, kw[j], recs[j]);
    lost |= on[j] && !hit;
    on[j] = hit;
  }
  if (lost) raise_capacity(p, CAP_AGG_TABLE);
  // Hot keys: the warp's largest group per row slot folds by butterflies.
#pragma unroll
  for (int j = 0; j < kBR; ++j) {
    // Rows of one key found the same record: match the record's offset in
    // the table (32 bits) rather than the 64-bit key word.
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t tag = on[j] ? (uint32_t)(recs[j] - table) : (0x80000000u | lane);
    uint32_t grp = __match_any_sync(0xffffffffu, tag);
    if (!on[j]) grp = 0;
    int maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    for (int round = 0; round < 2 && maxpop >= p.agg_collapse_min; ++round) {
      const unsigned long long* sp = src[j];
      const uint32_t flags = vf[j];
      const uint64_t first_val = v0[j];
      if (collapse_largest(p, recs[j], grp, maxpop, on[j], row[j], [&](int v, bool& ok, uint64_t& b) {
            ok = (flags >> v) & 1u;
            b = ok ? (v == 0 ? first_val : __ldcs(sp + 2 + v)) : 0ull;
          })) {
        on[j] = false;
        grp = 0;
      }
      maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    }
  }
  // A partition's rows arrive roughly in row order, so most rows do not
  // lower their group's first row: the atomic only when they do (a new
  // record's 0 always takes it).
  uint32_t first_seen[kBR];
#pragma unroll
  for (int j = 0; j < kBR; ++j)
    first_seen[j] = on[j] ? *reinterpret_cast<const volatile uint32_t*>(recs[j] + kRecFirst) : ~0u;
#pragma unroll
  for (int j = 0; j < kBR; ++j) {
    if (!on[j]) continue;
    if (~row[j] > first_seen[j]) rec_max_u32<true>(recs[j] + kRecFirst, ~row[j]);
    if (p.off_len >= 0) rec_add_u32<true>(recs[j] + p.off_len, 1u);
    if (p.off_last >= 0) rec_max_u32<true>(recs[j] + p.off_last, row[j] + 1u);
  }
  for (int v = 0; v < p.n_vals; ++v) {
    bool ok[kBR];
    uint64_t vb[kBR];
#pragma unroll
    for (int j = 0; j < kBR; ++j) {
      ok[j] = on[j] && ((vf[j] >> v) & 1u);
      vb[j] = ok[j] ? (v == 0 ? v0[j] : __ldcs(src[j] + 2 + v)) : 0ull;
    }
    const ValField& f = p.vals[v];
    switch (f.dtype) {
      case DFC_INT8: update_rows<int8_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_INT16: update_rows<int16_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_INT32: update_rows<int32_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_INT64: update_rows<int64_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_UINT8: update_rows<uint8_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_UINT16: update_rows<uint16_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_UINT32: update_rows<uint32_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_UINT64: update_rows<uint64_t, true, kBR>(p, f, v, recs, ok, vb); break;
      case DFC_FLOAT32: update_rows<float, true, kBR>(p, f, v, recs, ok, vb); break;
      default: update_rows<double, true, kBR>(p, f, v, recs, ok, vb); break;
    }
  }
}

__global__ void __launch_bounds__(kAggThreads, 2) partition_aggregate(const __grid_constant__ ScanParams p) {
  extern __shared__ __align__(16) unsigned char table[];
  __shared__ uint32_t s_next, s_used, s_base, s_hole_lo, s_hole_hi, s_chunk_next, s_chunk_end;
  const uint32_t nparts = 1u << p.part_bits;
  const uint32_t S = p.agg_slots;
  const size_t rs = agg_stride(p);
  const size_t rw = (size_t)p.rec_stride / 8;  // words of a record
  uint32_t* const live = reinterpret_cast<uint32_t*>(table + (size_t)(S + 1) * rs);  // claimed slots, in claim order
  unsigned char* const ones = table + (size_t)S * rs;  // the all-ones key word's record
  for (uint32_t s = threadIdx.x; s <= S; s += blockDim.x) reset_record(table + (size_t)s * rs, p.rec_stride);
  if (threadIdx.x == 0) {
    s_next = atomicAdd(p.part_next, 1u);
    s_used = 0;
    s_chunk_next = s_chunk_end = 0;
  }
  __syncthreads();
  for (;;) {
    const uint32_t pick = s_next;
    if (pick >= nparts) break;
    const uint32_t part = p.part_order[pick];
    if (part >= nparts) {  // uniform over the CTA
      if (threadIdx.x == 0) part_check(p, CHK_PART);
      break;
    }
    __syncthreads();  // every thread read s_next
    // The next partition is fetched while this one folds.
    if (threadIdx.x == 0) s_next = atomicAdd(p.part_next, 1u);
    const uint32_t n = p.part_totals[part];
    if (threadIdx.x == 0 && p.part_cursor[part] != n) part_check(p, CHK_RANGE);
    const unsigned long long* rows = p.part_buf + (uint64_t)p.part_start[part] * p.part_words;
    const uint32_t per = blockDim.x * (uint32_t)kBR;
    for (uint32_t base = 0; base < n; base += per)
      fold_rows(p, table, &s_used, live, rows, n, base + threadIdx.x, blockDim.x);
    __syncthreads();
    // Live records: the claimed slots and the all-ones record when a row
    // reached it.  Reserve (chunks of kRecChunk from p.alloc), copy out and
    // reset.
    const uint32_t n_live = min(s_used, S);
    const bool ones_live = *reinterpret_cast<const uint32_t*>(ones + kRecFirst) != 0u;
    if (threadIdx.x == 0) {
      const uint32_t tot = n_live + (ones_live ? 1u : 0u);
      s_hole_lo = s_hole_hi = 0;
      if (tot > s_chunk_end - s_chunk_next) {
        // The rest of the current chunk stays unused: holes for the finish.
        s_hole_lo = s_chunk_next;
        s_hole_hi = s_chunk_end;
        const uint32_t grab = tot > kRecChunk ? tot : kRecChunk;
        s_chunk_next = atomicAdd(p.alloc, grab);
        s_chunk_end = s_chunk_next + grab;
        if ((uint64_t)s_chunk_next + grab > p.recs_total) raise_capacity(p, CAP_RECORDS);
      }
      s_base = s_chunk_next;
      s_chunk_next += tot;
    }
    __syncthreads();
    for (uint32_t r = s_hole_lo + threadIdx.x; r < s_hole_hi; r += blockDim.x)
      if (r < p.recs_total) *reinterpret_cast<uint32_t*>(record_at(p, r) + kRecFirst) = 0u;
    const uint32_t base_rec = s_base;
    auto copy_out = [&](unsigned char* rec, uint32_t dst) {
      if (dst < p.recs_total) {
        // Records are a multiple of 16 bytes and 16-byte aligned in the
        // global array: 16-byte stores (the table's stride is 8 mod 16).
        ulonglong2* out = reinterpret_cast<ulonglong2*>(record_at(p, dst));
        const unsigned long long* in = reinterpret_cast<const unsigned long long*>(rec);
        for (size_t q = 0; q + 1 < rw; q += 2) out[q / 2] = make_ulonglong2(in[q], in[q + 1]);
      }
      reset_record(rec, p.rec_stride);
    };
    for (uint32_t i = threadIdx.x; i < n_live; i += blockDim.x) {
      const uint32_t s = live[i];
      if (s < S) copy_out(table + (size_t)s * rs, base_rec + i);
      else part_check(p, CHK_SLOT);
    }
    if (ones_live && threadIdx.x == blockDim.x - 1) copy_out(ones, base_rec + n_live);
    __syncthreads();  // s_base, the list and the table are reused for the next partition
    if (threadIdx.x == 0) s_used = 0;
  }
  // The unused rest of the last chunk: holes.
  for (uint32_t r = s_chunk_next + threadIdx.x; r < s_chunk_end; r += blockDim.x)
    if (r < p.recs_total) *reinterpret_cast<uint32_t*>(record_at(p, r) + kRecFirst) = 0u;
}

}  // namespace dfc
