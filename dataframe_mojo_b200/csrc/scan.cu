// scan.cu — the fused filter + key + aggregate pass of the filtered hash
// group-by on sm_100a.
//
// One persistent CTA per SM slot.  Warp 0 is the producer: for every tile of
// `tile_rows` rows it streams each column the query touches (values and
// validity words) into a ring of shared-memory stages with 1-D TMA bulk
// copies (cp.async.bulk, no multicast) that complete on mbarriers.  The other
// warps consume a stage with every thread holding kScanRowsPerThread rows at
// once, so the rows' independent probes and record reads overlap:
//   1. the filter program (postfix, Kleene logic) over the thread's rows;
//   2. the key word (packed key columns, or a 64-bit hash in ticket mode);
//   3. with few groups, the CTA's shared-memory table: duplicate keys of a
//      warp collapse with __match_any_sync into one leader update;
//   4. otherwise one 16-byte probe load per row in the global open-addressing
//      table; misses resolve in warp-synchronous rounds in which new groups
//      are claimed by a 128-bit CAS that publishes key and group id together;
//   5. the group record's read-set (first row, K, min, max), then
//      fire-and-forget atomics: counts, sums, the shifted square sum; first
//      row / min / max only when the row improves them.
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

#include "dfc_device.cuh"
#include "dfc_internal.h"
#include "kernels.h"

namespace dfc {

constexpr uint32_t kWaitLimit = 1u << 22;  // try_wait polls before a stage wait gives up
constexpr uint32_t kSpinLimit = 1u << 20;  // re-reads before a publication wait gives up
constexpr uint32_t kNoGid = 0xFFFFFFFFu;
constexpr int kR = kScanRowsPerThread;

// Where a tile's data is: a shared-memory stage (staged) or global memory.
struct Tile {
  const unsigned char* stage;
  uint64_t start;
  bool staged;
};

__device__ __forceinline__ const unsigned char* col_values(const ScanParams& p, const Tile& t, int c) {
  return t.staged ? t.stage + p.stage_off[c]
                  : static_cast<const unsigned char*>(p.cols[c].values) + t.start * (uint64_t)p.cols[c].size;
}

__device__ __forceinline__ const uint32_t* col_valid(const ScanParams& p, const Tile& t, int c) {
  if (t.staged) return p.stage_voff[c] >= 0 ? reinterpret_cast<const uint32_t*>(t.stage + p.stage_voff[c]) : nullptr;
  return p.cols[c].validity ? p.cols[c].validity + t.start / 32 : nullptr;
}

__device__ __forceinline__ bool valid_at(const uint32_t* w, uint32_t r) {
  return w == nullptr || ((w[r >> 5] >> (r & 31)) & 1u);
}

__device__ __forceinline__ unsigned char* record_at(const ScanParams& p, uint32_t gid) {
  return p.records + (size_t)gid * (size_t)p.rec_stride;
}

// ---------------------------------------------------------------------------
// Filter program over the thread's rows: value and known bits as two
// register stacks per row.
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

__device__ __forceinline__ void filter_rows(const ScanParams& p, const Tile& t, const uint32_t (&rr)[kR],
                                            bool (&sel)[kR]) {
  if (p.n_pred == 0) return;
  uint32_t sv[kR], sk[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) sv[j] = sk[j] = 0;
  for (int i = 0; i < p.n_pred; ++i) {
    const PredOp& op = p.pred[i];
    if (op.kind == DFC_PRED_CMP) {
      const int c = op.input, dt = p.cols[c].dtype, size = p.cols[c].size;
      const unsigned char* vals = col_values(p, t, c);
      const uint32_t* valid = col_valid(p, t, c);
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        bool known = false, v = false;
        if (sel[j]) {
          known = valid_at(valid, rr[j]);
          const uint64_t b = load_bits(vals, size, rr[j]);
          if (dt == DFC_FLOAT64) v = cmp_op<double>(op.cmp, __longlong_as_double((long long)b), op.lit.f);
          else if (dt == DFC_FLOAT32) v = cmp_op<float>(op.cmp, __uint_as_float((uint32_t)b), (float)op.lit.f);
          else if (dt == DFC_UINT64) v = cmp_op<uint64_t>(op.cmp, b, op.lit.u);
          else v = cmp_op<int64_t>(op.cmp, bits_to_i64(b, dt), op.lit.i);
          v = v && known;
        }
        sv[j] = (sv[j] << 1) | (uint32_t)v;
        sk[j] = (sk[j] << 1) | (uint32_t)known;
      }
    } else if (op.kind == DFC_PRED_IS_NULL || op.kind == DFC_PRED_IS_NOT_NULL) {
      const uint32_t* valid = col_valid(p, t, op.input);
      const bool want_null = op.kind == DFC_PRED_IS_NULL;
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        const bool is_valid = sel[j] ? valid_at(valid, rr[j]) : true;
        sv[j] = (sv[j] << 1) | (uint32_t)(want_null ? !is_valid : is_valid);
        sk[j] = (sk[j] << 1) | 1u;
      }
    } else if (op.kind == DFC_PRED_TRUE) {
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        sv[j] = (sv[j] << 1) | 1u;
        sk[j] = (sk[j] << 1) | 1u;
      }
    } else if (op.kind == DFC_PRED_NOT) {
#pragma unroll
      for (int j = 0; j < kR; ++j) sv[j] ^= sk[j] & 1u;
    } else {  // AND / OR
      const bool is_and = op.kind == DFC_PRED_AND;
#pragma unroll
      for (int j = 0; j < kR; ++j) {
        const uint32_t bv = sv[j] & 1u, bk = sk[j] & 1u;
        sv[j] >>= 1;
        sk[j] >>= 1;
        const uint32_t av = sv[j] & 1u, ak = sk[j] & 1u;
        uint32_t rv, rk;
        if (is_and) {
          const uint32_t false_known = (ak & (av ^ 1u)) | (bk & (bv ^ 1u));
          rk = false_known | (ak & bk);
          rv = (false_known ^ 1u) & ak & bk & av & bv;
        } else {
          const uint32_t true_known = (ak & av) | (bk & bv);
          rk = true_known | (ak & bk);
          rv = true_known;
        }
        sv[j] = (sv[j] & ~1u) | rv;
        sk[j] = (sk[j] & ~1u) | rk;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kR; ++j) sel[j] = sel[j] && ((sv[j] & sk[j] & 1u) != 0);
}

// ---------------------------------------------------------------------------
// Keys.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void key_words(const ScanParams& p, const Tile& t, const uint32_t (&rr)[kR],
                                          const bool (&sel)[kR], uint64_t (&kw)[kR]) {
  const bool packed = p.key_mode == KEY_PACKED;
#pragma unroll
  for (int j = 0; j < kR; ++j) kw[j] = packed ? 0ull : 0x243F6A8885A308D3ull;
  for (int k = 0; k < p.n_keys; ++k) {
    const KeyField& f = p.keys[k];
    const int size = p.cols[f.input].size;
    const unsigned char* vals = col_values(p, t, f.input);
    const uint32_t* valid = col_valid(p, t, f.input);
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      if (!sel[j]) continue;
      const bool ok = valid_at(valid, rr[j]);
      const uint64_t cell = ok ? key_cell(load_bits(vals, size, rr[j]), f.dtype) : 0ull;
      if (packed) {
        if (!ok) kw[j] |= 1ull << f.null_bit;
        else kw[j] |= (f.bits == 64) ? cell : (cell << f.shift);
      } else {
        const uint64_t c = ok ? cell + 1 : 0x9E3779B97F4A7C15ull;
        kw[j] = mix64(kw[j] ^ (c * 0x9E3779B97F4A7C15ull + (uint64_t)k));
      }
    }
  }
  if (!packed) {
#pragma unroll
    for (int j = 0; j < kR; ++j)
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
// Claims.
// ---------------------------------------------------------------------------
// Record numbers are handed out by CTA tickets: ticket t falls in the CTA's
// chunk k = t / chunk, whose base the holder of the chunk's first ticket draws
// from the global counter and publishes (tagged with k) in a small ring.  A
// reserved record that loses its claim race stays all-zero: a hole.
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
    const uint64_t m = ld_cg_u64(&e->meta);
    if (m != kEmpty) return m;
  }
  atomicOr(p.status, ST_TIMEOUT);
  return kEmpty;
}

// The group of key word kw at row `row`, claiming a new record if the key is
// new: the per-lane path for ticket keys, the all-ones key word and merges.
// kNoGid when records or table slots ran out (ST_CAPACITY set).
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

// Packed keys: every lane's rows resolved together.  Each round a pending
// row looks at its current entry: its key -> found; empty -> claim it (CAS);
// another key -> step to the next slot and reload.  All lanes run the rounds
// in lock-step, so a warp's claims share their latency.
__device__ __forceinline__ void resolve_packed(const ScanParams& p, const uint32_t (&rows)[kR], bool (&sel)[kR],
                                               const uint64_t (&kw)[kR], uint32_t (&gid)[kR], ClaimState* cs) {
  uint64_t slot[kR];
  unsigned long long ek[kR], em[kR];
  bool pend[kR];
  uint32_t res[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    gid[j] = kNoGid;
    res[j] = kNoGid;
    pend[j] = sel[j];
    slot[j] = 0;
    ek[j] = em[j] = 0;
    if (pend[j] && kw[j] == kEmpty) {
      gid[j] = find_or_claim(p, kw[j], rows[j], cs);
      pend[j] = false;
    }
    if (pend[j]) {
      slot[j] = slot_of(p, kw[j]);
      const ulonglong2 e = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + slot[j]));
      ek[j] = e.x;
      em[j] = e.y;
    }
  }
  for (uint32_t round = 0;; ++round) {
    bool any = false;
#pragma unroll
    for (int j = 0; j < kR; ++j) any |= pend[j];
    if (!__any_sync(0xffffffffu, any)) break;
    if (round > p.table_mask + 2) {  // every slot seen: the table is full
#pragma unroll
      for (int j = 0; j < kR; ++j) pend[j] = false;
      atomicOr(p.status, ST_CAPACITY);
      break;
    }
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      if (!pend[j]) continue;
      bool reload = false;
      if (ek[j] == kw[j]) {
        if (em[j] != kEmpty) {
          gid[j] = (uint32_t)em[j];
          pend[j] = false;
        } else {
          reload = true;  // torn read of a fresh claim
        }
      } else if (ek[j] == kEmpty) {
        // A record reserved for a claim that lost its race is kept for this
        // row's next attempt; one never used stays all-zero (a hole).
        if (res[j] == kNoGid) res[j] = reserve_record(p, cs);
        const uint32_t r = res[j];
        if (r == kNoGid) {
          pend[j] = false;
          continue;
        }
        uint64_t ok, om;
        cas128(p.table + slot[j], kEmpty, kEmpty, kw[j], (uint64_t)r | ((uint64_t)rows[j] << 32), ok, om);
        if (ok == kEmpty && om == kEmpty) {
          claimed(p, r, kw[j], rows[j]);
          gid[j] = r;
          pend[j] = false;
        } else if (ok == kw[j]) {
          gid[j] = (uint32_t)om;
          pend[j] = false;
        } else {
          slot[j] = (slot[j] + 1) & p.table_mask;
          reload = true;
        }
      } else {
        slot[j] = (slot[j] + 1) & p.table_mask;
        reload = true;
      }
      if (reload) {
        const ulonglong2 e = __ldcg(reinterpret_cast<const ulonglong2*>(p.table + slot[j]));
        ek[j] = e.x;
        em[j] = e.y;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kR; ++j) sel[j] = sel[j] && gid[j] != kNoGid;
}

// ---------------------------------------------------------------------------
// Shared-memory regime (few groups): each CTA keeps its own key table and
// all-zero group records in shared memory; duplicate keys inside a warp are
// collapsed with __match_any_sync so one leader lane applies the combined
// update; the CTA's records are merged into the global table when it exits.
// Rows whose key finds no room in the CTA table take the global path.
// ---------------------------------------------------------------------------
struct SmemTable {
  unsigned long long* keys;  // smem_slots, kEmpty = free
  unsigned char* recs;       // smem_slots records of rec_stride bytes
  uint32_t* used;            // claimed slots
};

__device__ __forceinline__ int smem_probe(const ScanParams& p, const SmemTable& st, uint64_t kw) {
  if (kw == kEmpty) return -1;
  const uint32_t mask = p.smem_slots - 1;
  uint32_t s = (uint32_t)mix64(kw ^ 0x9FB21C651E98DF25ull) & mask;
  for (int probe = 0; probe < 32; ++probe) {
    const unsigned long long k = st.keys[s];
    if (k == kw) return (int)s;
    if (k == kEmpty) {
      // At most three-quarters full, so probes stay short.
      if (*(volatile uint32_t*)st.used >= p.smem_slots - p.smem_slots / 4) return -1;
      const unsigned long long prev = atomicCAS(&st.keys[s], kEmpty, kw);
      if (prev == kEmpty) {
        atomicAdd(st.used, 1u);
        return (int)s;
      }
      if (prev == kw) return (int)s;
    }
    s = (s + 1) & mask;
  }
  return -1;
}

// The lane holding the i-th member of `grp` (lanes outside return their own).
__device__ __forceinline__ int nth_lane(uint32_t grp, int i) {
  for (int k = 0; k < i; ++k) grp &= grp - 1;
  return grp ? __ffs(grp) - 1 : (int)(threadIdx.x & 31);
}

// Reduction over each lane's group; shuffles run on the full warp.
template <typename V, typename Op>
__device__ __forceinline__ V group_reduce(uint32_t grp, int maxpop, V mine, V identity, bool take, Op op) {
  V acc = identity;
  for (int i = 0; i < maxpop; ++i) {
    const V v = __shfl_sync(0xffffffffu, take ? mine : identity, nth_lane(grp, i));
    if (i < __popc(grp)) acc = op(acc, v);
  }
  return acc;
}

__device__ __forceinline__ void smem_rows(const ScanParams& p, const Tile& t, const SmemTable& st,
                                          const uint32_t (&rr)[kR], bool (&sel)[kR], const uint64_t (&kw)[kR]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    const int ls = sel[j] ? smem_probe(p, st, kw[j]) : -1;
    const bool loc = ls >= 0;
    uint32_t grp = __match_any_sync(0xffffffffu, kw[j]) & __ballot_sync(0xffffffffu, loc);
    if (!loc) grp = 0;
    const int maxpop = __reduce_max_sync(0xffffffffu, (unsigned)__popc(grp));
    if (maxpop == 0) continue;
    const bool leader = loc && lane == __ffs(grp) - 1;
    unsigned char* rec = loc ? st.recs + (size_t)ls * p.rec_stride : nullptr;
    if (leader) {
      // The leader is the group's lowest lane, hence its earliest row.  The
      // CTA record always keeps its first row: it is the claim row when the
      // record is merged into the global table.
      atomicMax(reinterpret_cast<uint32_t*>(rec + kRecFirst), ~(uint32_t)(t.start + rr[j]));
      if (p.off_len >= 0) atomicAdd(reinterpret_cast<uint32_t*>(rec + p.off_len), (uint32_t)__popc(grp));
    }
    for (int v = 0; v < p.n_vals; ++v) {
      const ValField& f = p.vals[v];
      const int c = f.input, dt = f.dtype;
      const bool isf = dt_float(dt);
      const bool ok = loc && valid_at(col_valid(p, t, c), rr[j]);
      const uint64_t b = ok ? load_bits(col_values(p, t, c), p.cols[c].size, rr[j]) : 0ull;
      const double xd = isf ? bits_to_f64(b, dt) : bits_as_double(b, dt);
      const bool nan = ok && isf && xd != xd;
      const uint32_t vmask = grp & __ballot_sync(0xffffffffu, ok);
      const uint32_t nanmask = grp & __ballot_sync(0xffffffffu, nan);
      const uint32_t pz = grp & __ballot_sync(0xffffffffu, ok && isf && xd == 0.0 && __double_as_longlong(xd) >= 0);
      const uint32_t nz = grp & __ballot_sync(0xffffffffu, ok && isf && xd == 0.0 && __double_as_longlong(xd) < 0);
      if (leader && vmask) atomicAdd(reinterpret_cast<uint32_t*>(rec + f.off_count), (uint32_t)__popc(vmask));
      if (f.off_sum >= 0) {
        if (f.sum_kind == SUM_F64) {
          const double s = group_reduce<double>(grp, maxpop, xd, 0.0, ok, [](double a, double b2) { return a + b2; });
          if (leader && vmask) atomicAdd(reinterpret_cast<double*>(rec + f.off_sum), s);
        } else {
          // The group's partial sum, exact in 128 bits.
          const bool uns = dt == DFC_UINT64;
          const uint64_t x = ok ? (uns ? b : (uint64_t)bits_to_i64(b, dt)) : 0ull;
          const uint64_t xhi = (!uns && (int64_t)x < 0) ? ~0ull : 0ull;
          __int128 exact = 0;
          for (int i = 0; i < maxpop; ++i) {
            const int src = nth_lane(grp, i);
            const uint64_t vlo = __shfl_sync(0xffffffffu, x, src);
            const uint64_t vhi = __shfl_sync(0xffffffffu, xhi, src);
            if (i < __popc(grp)) exact += (__int128)(((unsigned __int128)vhi << 64) | vlo);
          }
          if (leader && vmask) {
            if (f.sum_kind == SUM_I64) {
              atomicAdd(reinterpret_cast<unsigned long long*>(rec + f.off_sum), (unsigned long long)(long long)exact);
            } else {
              const uint64_t add_lo = (uint64_t)exact, add_hi = (uint64_t)(exact >> 64);
              const uint64_t old = atomicAdd(reinterpret_cast<unsigned long long*>(rec + f.off_sum), add_lo);
              const uint64_t hi_add = add_hi + ((old + add_lo) < old ? 1ull : 0ull);
              if (hi_add) atomicAdd(reinterpret_cast<unsigned long long*>(rec + f.off_sum + 8), hi_add);
            }
          }
        }
      }
      if (f.off_min >= 0 || f.off_max >= 0) {
        const bool ordinary = ok && !nan;
        const uint64_t e = ordinary ? order_encode(b, dt) : 0ull;
        if (f.off_min >= 0) {
          const unsigned long long m = group_reduce<unsigned long long>(
              grp, maxpop, ~e, 0ull, ordinary, [](unsigned long long a, unsigned long long b2) { return a > b2 ? a : b2; });
          if (leader && m) atomicMax(reinterpret_cast<unsigned long long*>(rec + f.off_min), m);
        }
        if (f.off_max >= 0) {
          const unsigned long long m = group_reduce<unsigned long long>(
              grp, maxpop, e, 0ull, ordinary, [](unsigned long long a, unsigned long long b2) { return a > b2 ? a : b2; });
          if (leader && m) atomicMax(reinterpret_cast<unsigned long long*>(rec + f.off_max), m);
        }
        if (leader) {
          uint32_t bits = 0;
          if (nanmask) bits |= 1u << (3 * v);
          if (pz) bits |= 1u << (3 * v + 1);
          if (nz) bits |= 1u << (3 * v + 2);
          if (bits) atomicOr(reinterpret_cast<uint32_t*>(rec + kRecFlags), bits);
        }
      }
      if (f.off_m2 >= 0) {
        // The group's shift K: set once, by the first valid value of a leader.
        const uint64_t xbits = (xd != xd) ? kCanonNaN : (uint64_t)__double_as_longlong(xd);
        const uint64_t cand = __shfl_sync(0xffffffffu, xbits, vmask ? __ffs(vmask) - 1 : lane);
        uint64_t ks = 0;
        if (leader && vmask) {
          ks = *reinterpret_cast<volatile unsigned long long*>(rec + f.off_shift);
          if (ks == 0) {
            const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(rec + f.off_shift), 0ull, cand ^ kShiftTag);
            ks = prev == 0 ? (cand ^ kShiftTag) : prev;
          }
        }
        ks = __shfl_sync(0xffffffffu, ks, grp ? __ffs(grp) - 1 : lane);
        const double d = xd - __longlong_as_double((long long)(ks ^ kShiftTag));
        const double s2 = group_reduce<double>(grp, maxpop, d * d, 0.0, ok, [](double a, double b2) { return a + b2; });
        if (leader && vmask) atomicAdd(reinterpret_cast<double*>(rec + f.off_m2), s2);
      }
    }
    sel[j] = sel[j] && !loc;  // the rest take the global path
  }
}

__device__ void merge_record(const ScanParams& p, const unsigned char* src, uint64_t kw, ClaimState* cs);

// ---------------------------------------------------------------------------
// A tile's rows for one consumer thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void consume_tile(const ScanParams& p, const Tile& t, uint32_t n, uint32_t ct,
                                             ClaimState* cs, const SmemTable* st) {
  uint32_t rr[kR], rows[kR];
  bool sel[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    rr[j] = ct + (uint32_t)j * kScanConsumerThreads;
    rows[j] = (uint32_t)(t.start + rr[j]);
    sel[j] = rr[j] < n;
  }
  filter_rows(p, t, rr, sel);
  uint64_t kw[kR];
  key_words(p, t, rr, sel, kw);
  if (st) smem_rows(p, t, *st, rr, sel, kw);

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

  // Read-set of every row (first row, then per column K, min, max), loads in
  // flight together, then the atomics.
  uint32_t first[kR];
#pragma unroll
  for (int j = 0; j < kR; ++j) first[j] = (sel[j] && p.track_first) ? ld_cg_u32(record_at(p, gid[j]) + kRecFirst) : ~0u;
#pragma unroll
  for (int j = 0; j < kR; ++j) {
    if (!sel[j]) continue;
    unsigned char* rec = record_at(p, gid[j]);
    if (p.track_first && ~rows[j] > first[j]) atomicMax(reinterpret_cast<uint32_t*>(rec + kRecFirst), ~rows[j]);
    if (p.off_len >= 0) red_add_u32(rec + p.off_len, 1u);
  }

  for (int v = 0; v < p.n_vals; ++v) {
    const ValField& f = p.vals[v];
    const int c = f.input, dt = f.dtype, size = p.cols[c].size;
    const unsigned char* vals = col_values(p, t, c);
    const uint32_t* valid = col_valid(p, t, c);
    const bool isf = dt_float(dt);
    bool ok[kR];
    uint64_t b[kR], lo[kR], hi[kR], ks[kR];
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      ok[j] = sel[j] && valid_at(valid, rr[j]);
      b[j] = ok[j] ? load_bits(vals, size, rr[j]) : 0ull;
      lo[j] = ~0ull;
      hi[j] = ~0ull;
      ks[j] = 1ull;
      if (!ok[j]) continue;
      const unsigned char* rec = record_at(p, gid[j]);
      if (f.off_min >= 0) lo[j] = ld_cg_u64(rec + f.off_min);
      if (f.off_max >= 0) hi[j] = ld_cg_u64(rec + f.off_max);
      if (f.off_m2 >= 0) ks[j] = ld_cg_u64(rec + f.off_shift);
    }
#pragma unroll
    for (int j = 0; j < kR; ++j) {
      if (!ok[j]) continue;
      unsigned char* rec = record_at(p, gid[j]);
      red_add_u32(rec + f.off_count, 1u);
      const double xd = isf ? bits_to_f64(b[j], dt) : 0.0;
      if (f.off_sum >= 0) {
        if (f.sum_kind == SUM_F64) {
          red_add_f64(rec + f.off_sum, xd);
        } else if (f.sum_kind == SUM_I64) {
          red_add_u64(rec + f.off_sum, (uint64_t)bits_to_i64(b[j], dt));
        } else {
          const bool uns = dt == DFC_UINT64;
          const uint64_t x = uns ? b[j] : (uint64_t)bits_to_i64(b[j], dt);
          const uint64_t neg = (!uns && (int64_t)x < 0) ? ~0ull : 0ull;
          const uint64_t old = atomicAdd(reinterpret_cast<unsigned long long*>(rec + f.off_sum), x);
          const uint64_t hi_add = neg + ((old + x) < old ? 1ull : 0ull);
          if (hi_add) red_add_u64(rec + f.off_sum + 8, hi_add);
        }
      }
      if (f.off_min >= 0 || f.off_max >= 0) {
        if (isf && xd != xd) {
          red_or_u32(rec + kRecFlags, 1u << (3 * v));
        } else {
          const uint64_t e = order_encode(b[j], dt);
          if (f.off_min >= 0 && ~e > lo[j]) red_max_u64(rec + f.off_min, ~e);
          if (f.off_max >= 0 && (e > hi[j] || hi[j] == ~0ull)) red_max_u64(rec + f.off_max, e);
          if (isf && xd == 0.0)
            red_or_u32(rec + kRecFlags, 1u << (3 * v + ((__double_as_longlong(xd) < 0) ? 2 : 1)));
        }
      }
      if (f.off_m2 >= 0) {
        const double x = isf ? xd : bits_as_double(b[j], dt);
        const uint64_t xbits = (x != x) ? kCanonNaN : (uint64_t)__double_as_longlong(x);
        uint64_t k = ks[j];
        if (k == 0) {
          const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long*>(rec + f.off_shift), 0ull, xbits ^ kShiftTag);
          k = prev == 0 ? (xbits ^ kShiftTag) : prev;
        }
        const double d = x - __longlong_as_double((long long)(k ^ kShiftTag));
        red_add_f64(rec + f.off_m2, d * d);
      }
    }
  }
}

__global__ void __launch_bounds__(kScanThreads, 2) scan_kernel(const __grid_constant__ ScanParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = p.stages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * p.stage_bytes);
  uint64_t* empty = full + S;
  __shared__ ClaimState s_claim;
  __shared__ volatile uint32_t s_abort;
  __shared__ uint32_t s_used;
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
  }
  if (threadIdx.x < kChunkRing) s_claim.ring[threadIdx.x] = ~0ull;
  SmemTable st{nullptr, nullptr, &s_used};
  if (p.smem_slots) {
    st.keys = reinterpret_cast<unsigned long long*>(smem + p.smem_keys_off);
    st.recs = smem + p.smem_recs_off;
    for (uint32_t s = threadIdx.x; s < p.smem_slots; s += blockDim.x) st.keys[s] = kEmpty;
    uint4* recs = reinterpret_cast<uint4*>(st.recs);
    const uint32_t n16 = p.smem_slots * (uint32_t)p.rec_stride / 16;
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) recs[i] = make_uint4(0, 0, 0, 0);
  }
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
          mbar_arrive(&full[s]);  // ragged tail: consumers read global memory
        }
      }
      // Every issued stage must have landed before the CTA may exit.
      if (s_abort) {
        const uint32_t first = it > (uint32_t)S ? it - S : 0;
        for (uint32_t j = first; j < it; ++j) mbar_wait_bounded(&full[j % S], (j / S) & 1u, kWaitLimit);
      }
    }
  } else {
    const uint32_t ct = threadIdx.x - 32;
    uint32_t it = 0;
    for (uint64_t t = blockIdx.x; t < p.tiles; t += gridDim.x, ++it) {
      const uint32_t s = it % S, ph = (it / S) & 1u;
      if (!mbar_wait_bounded(&full[s], ph, kWaitLimit)) {
        atomicOr(p.status, ST_TIMEOUT);
        s_abort = 1;
        break;
      }
      const Tile tile{smem + (size_t)s * p.stage_bytes, t * T, p.use_tma && t < p.full_tiles};
      const uint64_t left = p.rows - tile.start;
      const uint32_t n = (uint32_t)(left < T ? left : T);
      for (uint32_t base = 0; base < n; base += kScanConsumerThreads * kR)
        consume_tile(p, tile, n, ct + base, &s_claim, p.smem_slots ? &st : nullptr);
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (s_abort) break;
    }
  }
  __syncthreads();
  if (p.smem_slots && !s_abort) {
    for (uint32_t s = threadIdx.x; s < p.smem_slots; s += blockDim.x)
      if (st.keys[s] != kEmpty) merge_record(p, st.recs + (size_t)s * p.rec_stride, st.keys[s], &s_claim);
  }
}

// Merges one CTA-table record into the global table (function.mojo:1559-1779
// `combine`; the shifted square sums are re-centred on the global record's K).
__device__ void merge_record(const ScanParams& p, const unsigned char* src, uint64_t kw, ClaimState* cs) {
  const uint32_t first_enc = *reinterpret_cast<const uint32_t*>(src + kRecFirst);
  if (first_enc == 0) return;
  const uint32_t gid = find_or_claim(p, kw, ~first_enc, cs);
  if (gid == kNoGid) return;
  unsigned char* dst = record_at(p, gid);
  if (p.track_first) atomicMax(reinterpret_cast<uint32_t*>(dst + kRecFirst), first_enc);
  if (p.off_len >= 0) red_add_u32(dst + p.off_len, *reinterpret_cast<const uint32_t*>(src + p.off_len));
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
    if (f.off_sum >= 0) {
      if (f.sum_kind == SUM_F64) {
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
        s1 = *reinterpret_cast<const double*>(src + f.off_sum) - dn * kl;
      } else {
        __int128 isum;
        if (f.sum_kind == SUM_I64) isum = (__int128)*reinterpret_cast<const long long*>(src + f.off_sum);
        else isum = (__int128)(((unsigned __int128)*reinterpret_cast<const uint64_t*>(src + f.off_sum + 8) << 64) |
                               *reinterpret_cast<const uint64_t*>(src + f.off_sum));
        s1 = (double)(isum - (__int128)n * (__int128)kl);
      }
      const double d = kl - kg;
      const double s2 = *reinterpret_cast<const double*>(src + f.off_m2);
      red_add_f64(dst + f.off_m2, d == 0.0 ? s2 : s2 + 2.0 * d * s1 + dn * d * d);
    }
  }
}

}  // namespace dfc
