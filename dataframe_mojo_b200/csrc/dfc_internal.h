// dfc_internal.h — descriptors shared by the planner (host) and the kernels.
//
// Data layout in HBM for one query:
//   inputs    resident columns: values (unpadded, 16-byte aligned) and a
//             validity bitmap normalised to bit offset 0, 32-bit words, padded
//   table     open-addressing key table, `slots` entries of 16 bytes
//             {key word, gid | claim row << 32}; all-ones = empty
//   records   dense group records, `stride` bytes each; CTAs draw chunks of
//             record numbers from one global counter
//   order     first-row bitmap (rows bits) + per-word popcount prefix + perm
//   outputs   one values buffer and one validity bitmap per output column
#pragma once

#include <stdint.h>

#include "../../include/dfcuda.h"

namespace dfc {

constexpr int kMaxInputs = 16;
constexpr int kMaxKeys = 4;
constexpr int kMaxVals = 8;
constexpr int kMaxPred = 32;
constexpr int kMaxAggs = 32;
constexpr int kMaxOut = kMaxKeys + kMaxAggs;
constexpr int kMaxRecWords = 64;  // 512-byte records at most

constexpr uint64_t kEmpty = ~0ull;
constexpr uint32_t kNoRow = 0xFFFFFFFFu;
// Shift K of the shifted second moment before any value set it: a signalling
// NaN payload; data NaNs are stored canonical (0x7FF8...) so they never match.
constexpr uint64_t kShiftUnset = 0x7FF40000000D0FC5ull;
constexpr uint64_t kCanonNaN = 0x7FF8000000000000ull;

// Status bits raised by kernels.
enum StatusBits : uint32_t {
  ST_CAPACITY = 1u,   // a CTA ran out of records or a probe wrapped
  ST_TIMEOUT = 2u,    // a bounded wait gave up
  ST_OVERFLOW = 4u,   // a checked integer sum does not fit
  ST_FAULT = 8u,      // ill-conditioned moments: CPU adjudicates
};

enum KeyMode : int32_t { KEY_PACKED = 0, KEY_TICKET = 1 };

enum SumKind : int32_t { SUM_NONE = 0, SUM_I64 = 1, SUM_I128 = 2, SUM_F64 = 3 };

// Record header (bytes).
constexpr int kRecKey = 0;    // u64 key word (packed key or 64-bit hash)
constexpr int kRecFirst = 8;  // u32 first row (claim row until updated)
constexpr int kRecFlags = 12; // u32 per-value NaN-seen bits
constexpr int kRecLen = 16;   // u32 rows of the group
constexpr int kRecClaim = 20; // u32 row that claimed the group
constexpr int kRecHeader = 24;

struct DevColumn {
  const void* values;
  const uint32_t* validity;  // nullptr: every row valid
  int32_t dtype;
  int32_t size;
};

struct KeyField {
  int32_t input;
  int32_t dtype;
  int32_t shift;     // bit position of the value bits inside the key word
  int32_t bits;      // 8, 16, 32 or 64
  int32_t null_bit;  // bit position of the null flag, -1: the column has no nulls
  int32_t pad;
};

struct ValField {
  int32_t input;
  int32_t dtype;
  int32_t sum_kind;
  int32_t off_count;  // u32 valid values (always present)
  int32_t off_sum;    // i64 / i128 (lo, hi) / f64, -1 absent
  int32_t off_min;    // u64 order-preserving encoding, -1 absent
  int32_t off_max;
  int32_t off_zero;   // u64 (row << 1 | sign) of the first zero, float min/max only
  int32_t off_m2;     // f64 sum of (x - K)^2, -1 absent
  int32_t off_shift;  // f64 K
  int32_t nan_bit;    // bit in the record flags
  int32_t pad;
};

struct PredOp {
  int32_t kind;
  int32_t input;
  int32_t cmp;
  int32_t pad;
  union {
    int64_t i;
    uint64_t u;
    double f;
  } lit;
};

struct KeyEntry {
  unsigned long long key;
  unsigned long long meta;
};

struct ScanParams {
  DevColumn cols[kMaxInputs];
  int32_t n_cols;
  // Columns staged per tile: values at stage_off, validity words at stage_voff.
  int32_t n_stage;
  int32_t stage_col[kMaxInputs];
  int32_t stage_off[kMaxInputs];
  int32_t stage_voff[kMaxInputs];  // -1: no validity
  int32_t stage_bytes;  // ring stride (128-byte aligned)
  int32_t stage_tx;     // bytes the bulk copies of one full tile deliver
  int32_t tile_rows;
  int32_t stages;
  int32_t use_tma;
  uint64_t rows;
  uint64_t tiles;       // ceil(rows / tile_rows)
  uint64_t full_tiles;  // rows / tile_rows
  // Keys.
  int32_t key_mode;
  int32_t n_keys;
  KeyField keys[kMaxKeys];
  // Filter program.
  int32_t n_pred;
  int32_t pad0;
  PredOp pred[kMaxPred];
  // Value states.
  int32_t n_vals;
  int32_t rec_stride;
  ValField vals[kMaxVals];
  int32_t track_first;  // maintain_order: first row by atomic min
  int32_t track_len;
  int32_t rec_words;    // stride / 8
  int32_t pad1;
  unsigned long long rec_template[kMaxRecWords];
  // Tables.
  KeyEntry* table;
  uint64_t table_mask;
  unsigned char* records;
  uint32_t recs_total;   // records allocated
  uint32_t chunk;        // records a CTA draws from `alloc` at a time (power of two)
  uint32_t* alloc;       // [0] records handed out (may exceed recs_total)
  uint32_t* status;      // [0] status bits
};

struct OutCol {
  void* values;
  uint32_t* validity;  // always allocated; has_nulls tells whether any bit is 0
  int32_t dtype;
  int32_t kind;        // OUT_KEY / OUT_AGG
  int32_t index;       // key field or aggregation index
  int32_t val;         // ValField index (aggregations)
  int32_t op;
  int32_t ddof;
  int32_t min_count;
  int32_t pad;
};

enum OutKind : int32_t { OUT_KEY = 0, OUT_AGG = 1 };

struct FinishParams {
  ScanParams scan;  // layout of the records and keys
  uint32_t* order_bits;    // rows bits
  uint32_t* word_prefix;   // exclusive popcount prefix per 32-bit word
  uint32_t* block_sums;    // scratch of the prefix scan
  uint32_t* perm;          // rank -> gid
  uint32_t* groups;        // [0] number of groups
  uint32_t* has_nulls;     // per output column
  uint32_t* overflow_agg;  // [0] lowest aggregation index that overflowed
  uint64_t words;          // ceil(rows / 32)
  int32_t n_out;
  int32_t pad;
  OutCol out[kMaxOut];
};

}  // namespace dfc
