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

#include "dfcuda.h"

namespace dfc {

constexpr int kMaxInputs = 16;
constexpr int kMaxKeys = 4;
constexpr int kMaxVals = 8;
constexpr int kMaxPred = 32;
constexpr int kMaxAggs = 32;
constexpr int kMaxOut = kMaxKeys + kMaxAggs;
constexpr int kMaxRecWords = 64;  // 512-byte records at most

constexpr uint64_t kEmpty = ~0ull;
// The shift K of the shifted second moment is stored xor this tag, so an
// all-zero record means "unset".  The tag is a signalling-NaN payload; data
// NaNs are stored canonical (0x7FF8...), so no value stores as zero.
constexpr uint64_t kShiftTag = 0x7FF40000000D0FC5ull;
constexpr uint64_t kCanonNaN = 0x7FF8000000000000ull;
// perm entry of the identity record: the one output row of an ungrouped
// query that kept no row (record numbers stay below 2^32 - 32).
constexpr uint32_t kIdentityRecord = 0xFFFFFFFFu;

// Status bits raised by kernels.
enum StatusBits : uint32_t {
  ST_CAPACITY = 1u,    // records or table slots ran out
  ST_TIMEOUT = 2u,     // a bounded wait gave up
  ST_OVERFLOW = 4u,    // a checked integer sum does not fit
  ST_FAULT = 8u,       // ill-conditioned moments: the CPU adjudicates
  ST_ZERO_FAULT = 16u, // a zero extremum seen with both signs: the CPU adjudicates
  ST_F32_RANGE = 32u,  // a compensated FP32 partial left the FP32 range: rerun in FP64
};

enum KeyMode : int32_t { KEY_PACKED = 0, KEY_TICKET = 1 };

enum SumKind : int32_t { SUM_NONE = 0, SUM_I64 = 1, SUM_I128 = 2, SUM_F64 = 3 };

// Group record (bytes).  Every field's identity is zero, so records are
// initialised by a memset: first row stored as ~row and the minimum as ~code
// (both raised by atomicMax), the maximum as its code, K xor kShiftTag.
// Value fields follow the header: u32 length and counts, then per aggregated
// column the read-set (K, min, max) and the sums.
constexpr int kRecKey = 0;    // u64 key word (packed key or 64-bit hash)
constexpr int kRecFirst = 8;  // u32 ~first row; 0 = a hole (reserved, never claimed)
constexpr int kRecFlags = 12; // u32, per value column v: bit 3v NaN seen, 3v+1 +0 seen, 3v+2 -0 seen
constexpr int kRecHeader = 16;

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
  int32_t off_m2;     // f64 sum of (x - K)^2, -1 absent
  int32_t off_shift;  // f64 K, the first value the group saw
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
  // Shared-memory regime: CTA key table (smem_slots, power of two; 0 = off)
  // and records at these byte offsets of the dynamic shared memory.  With
  // smem_cluster > 1 the tables of a cluster's CTAs form one table of
  // smem_cluster * smem_slots entries (a key lives in one CTA's share, reached
  // through distributed shared memory).
  uint32_t smem_slots;
  uint32_t smem_keys_off;
  uint32_t smem_recs_off;
  uint32_t smem_cluster;  // CTAs sharing one table; 0 or 1: each CTA its own
  int32_t track_first;  // maintain_order: first row lowered by atomic min
  int32_t off_len;      // u32 rows of the group, -1 absent
  int32_t off_last;     // u32 the group's latest row + 1 (LAST), -1 absent
  int32_t rec_words;    // stride / 8
  // Value fields (bit v) whose sum and shifted square sum accumulate in the
  // shared-memory tables as compensated FP32 pairs {s, c} (Float32 columns),
  // merged into the FP64 global records; rows on the global path add in FP64.
  uint32_t comp_mask;
  // Direct addressing of own tables (integer keys whose ranges together fit
  // the table, dataframe/aggregation/perfect_hash.mojo:1-50): a key's slot is
  // the sum over key columns of (value - dmin + 1, or 0 for null) << dshift;
  // no hashing and no probing.  0: hashed tables.
  int32_t direct;
  // Ungrouped queries (no key) whose value columns fit the register path:
  // scan_kernel_reduce instead of the own-table scan.
  int32_t reduce;
  int32_t dshift[kMaxKeys];
  uint64_t dmin[kMaxKeys];  // each key's least value, as raw bits of its width
  // Tables.
  KeyEntry* table;
  uint64_t table_mask;
  unsigned char* records;
  uint32_t recs_total;   // records allocated
  uint32_t chunk;        // records a CTA draws from `alloc` at a time (power of two)
  uint32_t* alloc;       // [0] records handed out (may exceed recs_total)
  uint32_t* status;      // [0] status bits, [1] CapacityBits, [2] partition-pass checks
  // Radix-partitioned regime (partition = the top part_bits bits of a hash
  // of the key word).  A counting pass stages only the key and filter columns
  // (the first n_stage_count staged columns, stage_tx_count bytes a full
  // tile) and counts the selected rows per partition into part_totals; their
  // exclusive prefix (part_start) gives every partition its range of
  // part_buf.  Pass A stages every column and places each selected row at
  // part_start[q] + the partition's cursor, raised by one atomic per warp and
  // partition, as part_words 8-byte words {key word, row | value validity
  // << 32, values...}.  Pass B folds one partition at a time per CTA into a
  // shared-memory table of agg_slots records and appends its live records to
  // `records` in chunks drawn from `alloc`.
  int32_t n_stage_count;   // staged columns the counting pass needs
  int32_t stage_tx_count;  // bytes of one full tile of those columns
  uint32_t part_bits;      // log2 partitions, 0 = regime off
  uint32_t part_words;
  unsigned long long* part_buf;
  uint32_t* part_totals;   // [partition] selected rows
  uint32_t* part_start;    // [partition] first row of the partition in part_buf
  uint2* part_range;       // [partition] {part_start, part_totals}: pass A reads both with one load
  uint32_t* part_cursor;   // [partition] rows pass A placed (zeroed before pass A)
  uint32_t* part_order;    // pass B's order of the partitions: the large ones first
  uint32_t agg_slots;      // pass B table slots
  uint32_t* part_next;     // pass B work counter
  uint32_t* part_kept;     // rows the counting pass kept (written by partition_offsets)
  int32_t agg_collapse_min;  // pass B: group size in a warp from which its rows fold by butterflies
  int32_t collapse_min;      // the global-table scan: the same threshold
  // The quad row path of the counting pass and pass A (fast_rows = 1): every
  // lane takes four consecutive rows of a 1024-row tile with vector loads.
  // It needs integer key columns and no filter or one comparison, held in
  // range form: a row is selected when its filter value x (valid, read as
  // fast_kind) satisfies (fast_lo <= x <= fast_hi) != fast_neg.
  int32_t fast_rows;
  int32_t fast_col;   // the compared column's slot, -1: no filter
  int32_t fast_kind;  // FAST_SIGNED (sign-extended int64), FAST_UNSIGNED (zero-extended uint64) or FAST_FLOAT (double)
  int32_t fast_neg;
  union {
    int64_t i;
    uint64_t u;
    double f;
  } fast_lo, fast_hi;
};

enum FastKind : int32_t { FAST_SIGNED = 0, FAST_UNSIGNED = 1, FAST_FLOAT = 2 };

// Which capacity ran out (status word 1), so the host grows only that.
enum CapacityBits : uint32_t { CAP_RECORDS = 1u, CAP_AGG_TABLE = 2u };

// Index and consistency checks (status word 2).  A failed check skips the
// access it guards; the host fails the query with the code.
enum CheckBits : uint32_t {
  CHK_PART = 4u,      // a partition number out of range
  CHK_RANGE = 8u,     // pass A placed a row beyond its partition's count
  CHK_SLOT = 16u,     // a table slot out of range
  CHK_FIRST = 128u,   // a record's first row beyond the rows
  CHK_DUP = 256u,     // two records with the same first row
  CHK_PERM = 512u,    // a rank naming no record
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
  uint32_t* firsts;        // first row per record (~0: hole)
  uint32_t* groups;        // [0] number of groups
  uint32_t* has_nulls;     // per output column
  uint32_t* overflow_agg;  // [0] lowest aggregation index that overflowed
  uint64_t words;          // ceil(rows / 32)
  int32_t n_out;
  int32_t pad;
  OutCol out[kMaxOut];
};

}  // namespace dfc
