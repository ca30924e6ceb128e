// oracle.cpp — CPU restatement of dataframe_mojo's filtered grouped reduction.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker of the CUDA provider
// (tests/, __graft_entry__.smoke) and the CPU baseline that bench.py times;
// the product (dataframe_mojo_b200/) never links or calls it.
//
// What it restates, by reference file:line (paths inside dataframe_mojo):
//   filter: a null predicate drops the row; comparisons are IEEE
//     (dataframe/kernels/fused_compare.mojo:31-183, kernels/binary.mojo:2172-2187)
//   key equality: nulls equal each other, every NaN is one value, -0.0 == 0.0
//     (dataframe/aggregation/reducer.mojo:869-875 float_key;
//      dataframe/kernels/partition.mojo:42-60)
//   group order with maintain_order: first occurrence among the rows the
//     filter kept (dataframe/aggregation/hash_table.mojo:2850-3153,
//     dataframe/aggregation/state.mojo:267-330)
//   state updates (dataframe/aggregation/function.mojo:1143-1236 `_scatter`):
//     integer sums exact in 128 bits; float sums FP64 in input order;
//     min/max keep the earlier value on ties and skip NaN (flag 2);
//     moments by Welford (scalar_states.mojo:104-145 VarState.add)
//   merges (function.mojo:1559-1779 `combine`; Chan's update at 1736-1758)
//   finalisation (function.mojo:2374-2432, 2516-2805, 2891-2918;
//     reducer.mojo:3391-3599): COUNT/LEN/NULL_COUNT Int64; SUM in the input's
//     sum type (dtype.mojo:838-849), null when count < min_count, overflow
//     raises "Int64 expression sum overflow" / "<type> expression sum
//     overflow"; Float32 sums rounded from the FP64 total; MEAN Float64,
//     null when count == 0; MIN/MAX in the input type, NaN only when every
//     valid value is NaN; VAR/STD M2/(n-ddof), null when n <= ddof.

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <queue>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

namespace {

thread_local std::string g_error;

int fail(int status, const std::string& msg) {
  g_error = msg;
  return status;
}

size_t dtype_size(int dt) {
  switch (dt) {
    case DFC_INT8: case DFC_UINT8: return 1;
    case DFC_INT16: case DFC_UINT16: return 2;
    case DFC_INT32: case DFC_UINT32: case DFC_FLOAT32: return 4;
    case DFC_INT64: case DFC_UINT64: case DFC_FLOAT64: return 8;
  }
  return 0;
}
bool is_float(int dt) { return dt == DFC_FLOAT32 || dt == DFC_FLOAT64; }
const char* dtype_name(int dt) {
  // DataType.name() of a numeric type is its storage DType's text
  // (dataframe/dtype.mojo:662-665).
  switch (dt) {
    case DFC_INT8: return "int8";
    case DFC_INT16: return "int16";
    case DFC_INT32: return "int32";
    case DFC_INT64: return "int64";
    case DFC_UINT8: return "uint8";
    case DFC_UINT16: return "uint16";
    case DFC_UINT32: return "uint32";
    case DFC_UINT64: return "uint64";
    case DFC_FLOAT32: return "float32";
    case DFC_FLOAT64: return "float64";
  }
  return "?";
}

bool col_valid(const orc_column& c, uint64_t row) {
  if (!c.validity) return true;
  uint64_t bit = c.bit_offset + row;
  return (c.validity[bit >> 3] >> (bit & 7)) & 1;
}

int64_t col_int(const orc_column& c, uint64_t row) {
  switch (c.dtype) {
    case DFC_INT8: return ((const int8_t*)c.values)[row];
    case DFC_INT16: return ((const int16_t*)c.values)[row];
    case DFC_INT32: return ((const int32_t*)c.values)[row];
    case DFC_INT64: return ((const int64_t*)c.values)[row];
    case DFC_UINT8: return ((const uint8_t*)c.values)[row];
    case DFC_UINT16: return ((const uint16_t*)c.values)[row];
    case DFC_UINT32: return ((const uint32_t*)c.values)[row];
    case DFC_UINT64: return (int64_t)((const uint64_t*)c.values)[row];
  }
  return 0;
}
uint64_t col_u64(const orc_column& c, uint64_t row) { return ((const uint64_t*)c.values)[row]; }
double col_float(const orc_column& c, uint64_t row) {
  if (c.dtype == DFC_FLOAT32) return (double)((const float*)c.values)[row];
  return ((const double*)c.values)[row];
}
// Any numeric value as Float64 (the moments and means read integers as their value).
double col_as_double(const orc_column& c, uint64_t row) {
  if (is_float(c.dtype)) return col_float(c, row);
  if (c.dtype == DFC_UINT64) return (double)col_u64(c, row);
  return (double)col_int(c, row);
}

// Equality key of one key cell (reducer.mojo:869-875 for floats).
uint64_t key_word(const orc_column& c, uint64_t row) {
  if (is_float(c.dtype)) {
    double v = col_float(c, row);
    if (std::isnan(v)) return 0x7FF8000000000000ull;
    if (v == 0) return 0;
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
  }
  if (c.dtype == DFC_UINT64) return col_u64(c, row);
  return (uint64_t)col_int(c, row);
}

// ---------------------------------------------------------------------------
// Predicate: Kleene logic over (value, known) pairs.
// ---------------------------------------------------------------------------
struct Tri {
  bool value;
  bool known;
};

template <typename T>
bool compare(int cmp, T a, T b) {
  switch (cmp) {
    case DFC_LT: return a < b;
    case DFC_LE: return a <= b;
    case DFC_GT: return a > b;
    case DFC_GE: return a >= b;
    case DFC_EQ: return a == b;
    case DFC_NE: return !(a == b);  // IEEE: NaN != NaN (kernels/binary.mojo:2186)
  }
  return false;
}

bool eval_predicate(const orc_query& q, uint64_t row) {
  if (q.n_pred == 0) return true;
  Tri stack[64];
  int sp = 0;
  for (int i = 0; i < q.n_pred; ++i) {
    const dfc_pred_op& op = q.pred[i];
    switch (op.kind) {
      case DFC_PRED_CMP: {
        const orc_column& c = q.inputs[op.column];
        if (!col_valid(c, row)) {
          stack[sp++] = {false, false};
          break;
        }
        bool r;
        if (is_float(c.dtype)) {
          double v = col_float(c, row);
          double lit = op.lit.f;
          if (c.dtype == DFC_FLOAT32) {
            // The literal is bound to Float32 like the column.
            float fv = (float)v, fl = (float)lit;
            r = compare<float>(op.cmp, fv, fl);
          } else {
            r = compare<double>(op.cmp, v, lit);
          }
        } else if (c.dtype == DFC_UINT64) {
          r = compare<uint64_t>(op.cmp, col_u64(c, row), op.lit.u);
        } else {
          r = compare<int64_t>(op.cmp, col_int(c, row), op.lit.i);
        }
        stack[sp++] = {r, true};
        break;
      }
      case DFC_PRED_IS_NULL:
        stack[sp++] = {!col_valid(q.inputs[op.column], row), true};
        break;
      case DFC_PRED_IS_NOT_NULL:
        stack[sp++] = {col_valid(q.inputs[op.column], row), true};
        break;
      case DFC_PRED_TRUE:
        stack[sp++] = {true, true};
        break;
      case DFC_PRED_NOT: {
        Tri a = stack[sp - 1];
        stack[sp - 1] = {!a.value, a.known};
        break;
      }
      case DFC_PRED_AND: {
        Tri b = stack[--sp], a = stack[--sp];
        Tri r;
        if ((a.known && !a.value) || (b.known && !b.value)) r = {false, true};
        else if (a.known && b.known) r = {true, true};
        else r = {false, false};
        stack[sp++] = r;
        break;
      }
      case DFC_PRED_OR: {
        Tri b = stack[--sp], a = stack[--sp];
        Tri r;
        if ((a.known && a.value) || (b.known && b.value)) r = {true, true};
        else if (a.known && b.known) r = {false, true};
        else r = {false, false};
        stack[sp++] = r;
        break;
      }
    }
  }
  return sp > 0 && stack[sp - 1].known && stack[sp - 1].value;
}

// ---------------------------------------------------------------------------
// Per-group, per-value-column state: every word any aggregation over that
// column needs (the reference keeps one slot per reduction; sum and mean of
// one column hold identical FLOAT_SUM / INT_SUM states, so sharing is exact).
// ---------------------------------------------------------------------------
struct ValueState {
  int64_t count = 0;      // _K_COUNT / sum counts
  __int128 isum = 0;      // _K_INT_SUM / _K_NARROW_SUM total
  double fsum = 0.0;      // _K_FLOAT_SUM total
  bool seen = false;      // MIN/MAX flag 1
  bool nan_seen = false;  // MIN/MAX flag 2
  // Best values in the canonical domain: ints as __int128, floats as double.
  __int128 min_i = 0, max_i = 0;
  double min_f = 0, max_f = 0;
  int64_t wn = 0;         // Welford count / mean / m2
  double wmean = 0, wm2 = 0;
  // N_UNIQUE (_K_DISTINCT, function.mojo:620-625): the distinct valid values
  // by key equality (key_word) and whether a null was seen (null counts as a
  // value, tests/public_contracts/test_approx_n_unique.mojo:60-80).
  std::unordered_set<uint64_t> uniq;
  bool uniq_null = false;
};

struct Group {
  uint64_t first_row;
  uint64_t last_row = 0;  // LAST: the group's latest kept row (function.mojo:1586-1600)
  int64_t len;
  std::vector<ValueState> vals;
};

struct GroupKey {
  uint64_t w[4];
  uint32_t nulls;
  bool operator==(const GroupKey& o) const {
    return nulls == o.nulls && w[0] == o.w[0] && w[1] == o.w[1] && w[2] == o.w[2] && w[3] == o.w[3];
  }
};

uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}
uint64_t hash_key(const GroupKey& k) {
  uint64_t h = mix64(k.nulls + 0x9E3779B97F4A7C15ull);
  for (int i = 0; i < 4; ++i) h = mix64(h ^ (k.w[i] + 0x9E3779B97F4A7C15ull * (i + 1)));
  return h;
}

// Open-addressing map from GroupKey to a group index (insertion order =
// first-occurrence order within the rows one worker saw).
struct GroupTable {
  std::vector<int64_t> slots;
  std::vector<GroupKey> keys;
  std::vector<Group> groups;
  uint64_t mask = 0;
  GroupTable() { rehash(1024); }
  void rehash(size_t cap) {
    slots.assign(cap, -1);
    mask = cap - 1;
    for (size_t g = 0; g < keys.size(); ++g) {
      uint64_t s = hash_key(keys[g]) & mask;
      while (slots[s] >= 0) s = (s + 1) & mask;
      slots[s] = (int64_t)g;
    }
  }
  // Returns the group index; `created` tells whether the key was new.
  int64_t find_or_insert(const GroupKey& k, uint64_t h, bool& created) {
    uint64_t s = h & mask;
    while (true) {
      int64_t g = slots[s];
      if (g < 0) break;
      if (keys[g] == k) {
        created = false;
        return g;
      }
      s = (s + 1) & mask;
    }
    created = true;
    int64_t g = (int64_t)keys.size();
    keys.push_back(k);
    slots[s] = g;
    if (keys.size() * 2 > slots.size()) rehash(slots.size() * 2);
    return g;
  }
};

struct Plan {
  std::vector<int> value_cols;      // distinct input indices that aggregations read
  std::vector<int> agg_value_slot;  // per aggregation, index into value_cols
  std::vector<bool> uniq;           // per value column: an N_UNIQUE reads it
};

Plan make_plan(const orc_query& q) {
  Plan p;
  for (int a = 0; a < q.n_aggs; ++a) {
    int col = q.aggs[a].column;
    int slot = -1;
    for (size_t i = 0; i < p.value_cols.size(); ++i)
      if (p.value_cols[i] == col) slot = (int)i;
    if (slot < 0) {
      slot = (int)p.value_cols.size();
      p.value_cols.push_back(col);
    }
    p.agg_value_slot.push_back(slot);
  }
  p.uniq.assign(p.value_cols.size(), false);
  for (int a = 0; a < q.n_aggs; ++a)
    if (q.aggs[a].op == DFC_AGG_N_UNIQUE) p.uniq[p.agg_value_slot[a]] = true;
  return p;
}

GroupKey make_key(const orc_query& q, uint64_t row) {
  GroupKey k{};
  for (int i = 0; i < q.n_keys; ++i) {
    const orc_column& c = q.inputs[q.keys[i]];
    if (!col_valid(c, row)) {
      k.nulls |= 1u << i;
      k.w[i] = 0;
    } else {
      k.w[i] = key_word(c, row);
    }
  }
  return k;
}

// `_scatter` for one valid value (function.mojo:1143-1236).
void update_value(ValueState& s, const orc_column& c, uint64_t row) {
  s.count += 1;
  if (is_float(c.dtype)) {
    double x = col_float(c, row);
    s.fsum += x;
    if (std::isnan(x)) {
      s.nan_seen = true;
    } else {
      if (!s.seen || x < s.min_f) s.min_f = x;
      if (!s.seen || x > s.max_f) s.max_f = x;
      s.seen = true;
    }
  } else {
    __int128 x = (c.dtype == DFC_UINT64) ? (__int128)col_u64(c, row) : (__int128)col_int(c, row);
    s.isum += x;
    if (!s.seen || x < s.min_i) s.min_i = x;
    if (!s.seen || x > s.max_i) s.max_i = x;
    s.seen = true;
  }
  // Welford (scalar_states.mojo:123-127).
  double x = col_as_double(c, row);
  s.wn += 1;
  double delta = x - s.wmean;
  s.wmean += delta / (double)s.wn;
  s.wm2 += delta * (x - s.wmean);
}

// `combine` of one value column's state (function.mojo:1559-1779): `b` holds
// rows that come after `a`'s in input order.
void combine_value(ValueState& a, const ValueState& b, bool floating) {
  a.count += b.count;
  a.isum += b.isum;
  a.fsum += b.fsum;
  a.nan_seen = a.nan_seen || b.nan_seen;
  if (b.seen) {
    if (floating) {
      if (!a.seen || b.min_f < a.min_f) a.min_f = b.min_f;
      if (!a.seen || b.max_f > a.max_f) a.max_f = b.max_f;
    } else {
      if (!a.seen || b.min_i < a.min_i) a.min_i = b.min_i;
      if (!a.seen || b.max_i > a.max_i) a.max_i = b.max_i;
    }
    a.seen = true;
  }
  // Chan's update (function.mojo:1736-1758).
  if (b.wn == 0) return;
  if (a.wn == 0) {
    a.wn = b.wn;
    a.wmean = b.wmean;
    a.wm2 = b.wm2;
    return;
  }
  int64_t total = a.wn + b.wn;
  double delta = b.wmean - a.wmean;
  double mean = a.wmean + delta * ((double)b.wn / (double)total);
  double m2 = a.wm2 + b.wm2 + delta * delta * (double)a.wn * (double)b.wn / (double)total;
  a.wn = total;
  a.wmean = mean;
  a.wm2 = m2;
}

// ---------------------------------------------------------------------------
// Results.
// ---------------------------------------------------------------------------
struct OutColumn {
  int dtype;
  std::vector<uint8_t> bytes;
  std::vector<uint8_t> valid;
};

}  // namespace

struct orc_result {
  uint64_t rows = 0;
  std::vector<OutColumn> cols;
  std::vector<uint64_t> first_rows;
};

namespace {

int sum_dtype(int dt) {
  // dtype.mojo:838-849: 8- and 16-bit integers widen to Int64.
  if (dt == DFC_INT8 || dt == DFC_INT16 || dt == DFC_UINT8 || dt == DFC_UINT16) return DFC_INT64;
  return dt;
}

template <typename T>
void put(OutColumn& c, size_t i, T v) {
  std::memcpy(c.bytes.data() + i * sizeof(T), &v, sizeof(T));
}

void put_typed(OutColumn& c, size_t i, int dt, __int128 vi, double vf) {
  switch (dt) {
    case DFC_INT8: put<int8_t>(c, i, (int8_t)vi); break;
    case DFC_INT16: put<int16_t>(c, i, (int16_t)vi); break;
    case DFC_INT32: put<int32_t>(c, i, (int32_t)vi); break;
    case DFC_INT64: put<int64_t>(c, i, (int64_t)vi); break;
    case DFC_UINT8: put<uint8_t>(c, i, (uint8_t)vi); break;
    case DFC_UINT16: put<uint16_t>(c, i, (uint16_t)vi); break;
    case DFC_UINT32: put<uint32_t>(c, i, (uint32_t)vi); break;
    case DFC_UINT64: put<uint64_t>(c, i, (uint64_t)vi); break;
    case DFC_FLOAT32: put<float>(c, i, (float)vf); break;
    case DFC_FLOAT64: put<double>(c, i, vf); break;
  }
}

// Range of a sum type (function.mojo:2891-2918; reducer.mojo:3391-3416).
bool fits(int dt, __int128 v) {
  switch (dt) {
    case DFC_INT32: return v >= INT32_MIN && v <= INT32_MAX;
    case DFC_UINT32: return v >= 0 && v <= (__int128)UINT32_MAX;
    case DFC_INT64: return v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX;
    case DFC_UINT64: return v >= 0 && v <= (__int128)UINT64_MAX;
  }
  return true;
}

std::string overflow_message(int input_dtype) {
  // Int64 inputs raise the IntSumState text (scalar_states.mojo:39,
  // function.mojo:2798); other integer inputs their sum type's name
  // (function.mojo:2914, reducer.mojo:3412).
  if (input_dtype == DFC_INT64) return "Int64 expression sum overflow";
  return std::string(dtype_name(sum_dtype(input_dtype))) + " expression sum overflow";
}

int finalize(const orc_query& q, const Plan& plan, const std::vector<Group>& groups,
             const std::vector<GroupKey>& keys, const std::vector<uint64_t>& key_rows,
             orc_result* r) {
  size_t G = groups.size();
  r->rows = G;
  r->first_rows.resize(G);
  for (size_t g = 0; g < G; ++g) r->first_rows[g] = groups[g].first_row;
  // Key columns: the value at the group's first row (the group row keeps the
  // first row's key words; a float key's FIRST state, group_by.mojo:319-329).
  for (int k = 0; k < q.n_keys; ++k) {
    const orc_column& c = q.inputs[q.keys[k]];
    OutColumn out;
    out.dtype = c.dtype;
    size_t sz = dtype_size(c.dtype);
    out.bytes.assign(G * sz, 0);
    out.valid.assign(G, 0);
    for (size_t g = 0; g < G; ++g) {
      uint64_t row = key_rows[g];
      bool valid = !((keys[g].nulls >> k) & 1);
      out.valid[g] = valid;
      if (valid) std::memcpy(out.bytes.data() + g * sz, (const uint8_t*)c.values + row * sz, sz);
    }
    r->cols.push_back(std::move(out));
  }
  for (int a = 0; a < q.n_aggs; ++a) {
    const dfc_agg& agg = q.aggs[a];
    const orc_column& c = q.inputs[agg.column];
    int slot = plan.agg_value_slot[a];
    bool floating = is_float(c.dtype);
    OutColumn out;
    int odt;
    switch (agg.op) {
      case DFC_AGG_COUNT: case DFC_AGG_LEN: case DFC_AGG_NULL_COUNT: case DFC_AGG_N_UNIQUE: odt = DFC_INT64; break;
      case DFC_AGG_SUM: odt = sum_dtype(c.dtype); break;
      case DFC_AGG_MIN: case DFC_AGG_MAX: case DFC_AGG_FIRST: case DFC_AGG_LAST: odt = c.dtype; break;
      default: odt = DFC_FLOAT64; break;
    }
    out.dtype = odt;
    out.bytes.assign(G * dtype_size(odt), 0);
    out.valid.assign(G, 0);
    if (agg.op == DFC_AGG_FIRST || agg.op == DFC_AGG_LAST) {
      // The value at the group's first (last) kept row, null when that row's
      // value is null (function.mojo:997-1013, 2637-2650).
      const size_t sz = dtype_size(c.dtype);
      for (size_t g = 0; g < G; ++g) {
        const uint64_t row = agg.op == DFC_AGG_FIRST ? groups[g].first_row : groups[g].last_row;
        const bool valid = groups[g].len > 0 && col_valid(c, row);
        out.valid[g] = valid;
        if (valid) std::memcpy(out.bytes.data() + g * sz, (const uint8_t*)c.values + row * sz, sz);
      }
      r->cols.push_back(std::move(out));
      continue;
    }
    if (agg.op == DFC_AGG_N_UNIQUE) {
      for (size_t g = 0; g < G; ++g) {
        const ValueState& s = groups[g].vals[slot];
        const int64_t n = (int64_t)s.uniq.size() + (s.uniq_null ? 1 : 0);
        std::memcpy(out.bytes.data() + g * 8, &n, 8);
        out.valid[g] = 1;
      }
      r->cols.push_back(std::move(out));
      continue;
    }
    for (size_t g = 0; g < G; ++g) {
      const ValueState& s = groups[g].vals[slot];
      bool ok = true;
      __int128 vi = 0;
      double vf = 0;
      switch (agg.op) {
        case DFC_AGG_COUNT: vi = s.count; break;
        case DFC_AGG_LEN: vi = groups[g].len; break;
        case DFC_AGG_NULL_COUNT: vi = groups[g].len - s.count; break;
        case DFC_AGG_SUM:
          ok = s.count >= agg.min_count;
          if (floating) {
            vf = ok ? s.fsum : 0.0;
          } else {
            vi = ok ? s.isum : 0;
            if (ok && !fits(odt, vi)) return fail(DFC_DATA_OVERFLOW, overflow_message(c.dtype));
          }
          break;
        case DFC_AGG_MEAN:
          ok = s.count > 0;
          if (ok) vf = floating ? s.fsum / (double)s.count : (double)s.isum / (double)s.count;
          break;
        case DFC_AGG_MIN: case DFC_AGG_MAX: {
          bool is_max = agg.op == DFC_AGG_MAX;
          if (floating) {
            if (s.seen) vf = is_max ? s.max_f : s.min_f;
            else if (s.nan_seen) vf = std::nan("");
            else ok = false;
          } else {
            ok = s.seen;
            vi = ok ? (is_max ? s.max_i : s.min_i) : 0;
          }
          break;
        }
        case DFC_AGG_VAR: case DFC_AGG_STD: {
          ok = s.wn - (int64_t)agg.ddof > 0;
          if (ok) {
            double var = s.wm2 / (double)(s.wn - (int64_t)agg.ddof);
            vf = agg.op == DFC_AGG_STD ? std::sqrt(var) : var;
          }
          break;
        }
        default:
          return fail(DFC_UNSUPPORTED, "unsupported aggregation");
      }
      out.valid[g] = ok;
      if (ok || agg.op == DFC_AGG_SUM) put_typed(out, g, odt, vi, vf);
      if (agg.op == DFC_AGG_COUNT || agg.op == DFC_AGG_LEN || agg.op == DFC_AGG_NULL_COUNT)
        out.valid[g] = 1;
    }
    r->cols.push_back(std::move(out));
  }
  return DFC_OK;
}

int validate(const orc_query* q) {
  if (!q || q->n_keys < 0 || q->n_keys > 4 || q->n_inputs < 1) return fail(DFC_INVALID, "bad query");
  uint64_t rows = q->inputs[0].rows;
  for (int i = 0; i < q->n_inputs; ++i)
    if (q->inputs[i].rows != rows) return fail(DFC_INVALID, "row counts differ");
  for (int a = 0; a < q->n_aggs; ++a)
    if (q->aggs[a].column < 0 || q->aggs[a].column >= q->n_inputs) return fail(DFC_INVALID, "bad agg column");
  return DFC_OK;
}

// One worker's pass over rows [lo, hi): groups in first-row order.
void scan_range(const orc_query& q, const Plan& plan, uint64_t lo, uint64_t hi, GroupTable& t,
                std::vector<uint64_t>& key_rows) {
  size_t nv = plan.value_cols.size();
  for (uint64_t row = lo; row < hi; ++row) {
    if (!eval_predicate(q, row)) continue;
    GroupKey k = make_key(q, row);
    bool created;
    int64_t g = t.find_or_insert(k, hash_key(k), created);
    if (created) {
      Group grp;
      grp.first_row = row;
      grp.len = 0;
      grp.vals.resize(nv);
      t.groups.push_back(std::move(grp));
      key_rows.push_back(row);
    }
    Group& grp = t.groups[g];
    grp.len += 1;
    grp.last_row = row;
    for (size_t v = 0; v < nv; ++v) {
      const orc_column& c = q.inputs[plan.value_cols[v]];
      const bool valid = col_valid(c, row);
      if (valid) update_value(grp.vals[v], c, row);
      if (plan.uniq[v]) {
        if (valid) grp.vals[v].uniq.insert(key_word(c, row));
        else grp.vals[v].uniq_null = true;
      }
    }
  }
}

// Ungrouped reductions (no key columns; the filtered reduction region
// SCAN_FRAME -> FILTER* -> SELECT, dataframe_metal/filter_plan.mojo:149-200)
// always have one row: with no row kept it holds the reductions of nothing,
// the states at their initial values (function.mojo:187-254), finished as
// for an empty group (sum 0 unless min_count > 0, mean/min/max/var null).
void ungrouped_row(const orc_query& q, const Plan& plan, std::vector<Group>& groups, std::vector<GroupKey>& keys,
                   std::vector<uint64_t>& key_rows) {
  if (q.n_keys != 0 || !groups.empty()) return;
  Group g;
  g.first_row = 0;
  g.len = 0;
  g.vals.resize(plan.value_cols.size());
  groups.push_back(std::move(g));
  keys.push_back(GroupKey{});
  key_rows.push_back(0);
}

}  // namespace

extern "C" {

int32_t orc_groupby(const orc_query* q, orc_result** out) {
  int st = validate(q);
  if (st) return st;
  Plan plan = make_plan(*q);
  GroupTable t;
  std::vector<uint64_t> key_rows;
  scan_range(*q, plan, 0, q->inputs[0].rows, t, key_rows);
  ungrouped_row(*q, plan, t.groups, t.keys, key_rows);
  auto r = std::make_unique<orc_result>();
  st = finalize(*q, plan, t.groups, t.keys, key_rows, r.get());
  if (st) return st;
  *out = r.release();
  return DFC_OK;
}

int32_t orc_groupby_parallel(const orc_query* q, int32_t threads, orc_result** out) {
  int st = validate(q);
  if (st) return st;
  Plan plan = make_plan(*q);
  int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  uint64_t rows = q->inputs[0].rows;
  // Phase 1: each worker reduces a contiguous morsel range into its own table
  // (hash_table.mojo:11-47: per-worker partial tables).
  std::vector<GroupTable> tables(T);
  std::vector<std::vector<uint64_t>> krows(T);
  {
    std::vector<std::thread> ws;
    for (int t = 0; t < T; ++t)
      ws.emplace_back([&, t] {
        uint64_t lo = rows * t / T, hi = rows * (t + 1) / T;
        scan_range(*q, plan, lo, hi, tables[t], krows[t]);
      });
    for (auto& w : ws) w.join();
  }
  // Phase 2: partition-wise merge.  Groups go to P partitions by key hash;
  // each partition folds the workers' groups in worker order, so a
  // partition's groups stay in first-row order (hash_table.mojo:2850-3153).
  const int P = 64;
  std::vector<std::vector<Group>> pgroups(P);
  std::vector<std::vector<GroupKey>> pkeys(P);
  std::vector<std::vector<uint64_t>> prows(P);
  {
    std::vector<std::vector<std::vector<int64_t>>> parts(T, std::vector<std::vector<int64_t>>(P));
    std::vector<std::thread> ws;
    for (int t = 0; t < T; ++t)
      ws.emplace_back([&, t] {
        for (size_t g = 0; g < tables[t].keys.size(); ++g)
          parts[t][(hash_key(tables[t].keys[g]) >> 58) & (P - 1)].push_back((int64_t)g);
      });
    for (auto& w : ws) w.join();
    ws.clear();
    std::vector<bool> floating(plan.value_cols.size());
    for (size_t v = 0; v < plan.value_cols.size(); ++v) floating[v] = is_float(q->inputs[plan.value_cols[v]].dtype);
    for (int t = 0; t < T; ++t)
      ws.emplace_back([&, t] {
        for (int p = t; p < P; p += T) {
          GroupTable merged;
          for (int w = 0; w < T; ++w)
            for (int64_t g : parts[w][p]) {
              const GroupKey& k = tables[w].keys[g];
              bool created;
              int64_t m = merged.find_or_insert(k, hash_key(k), created);
              Group& src = tables[w].groups[g];
              if (created) {
                merged.groups.push_back(src);
                prows[p].push_back(krows[w][g]);
              } else {
                Group& dst = merged.groups[m];
                dst.len += src.len;
                dst.last_row = std::max(dst.last_row, src.last_row);
                for (size_t v = 0; v < dst.vals.size(); ++v) {
                  dst.vals[v].uniq.insert(src.vals[v].uniq.begin(), src.vals[v].uniq.end());
                  dst.vals[v].uniq_null = dst.vals[v].uniq_null || src.vals[v].uniq_null;
                }
                for (size_t v = 0; v < dst.vals.size(); ++v) combine_value(dst.vals[v], src.vals[v], floating[v]);
              }
            }
          pgroups[p] = std::move(merged.groups);
          pkeys[p] = std::move(merged.keys);
        }
      });
    for (auto& w : ws) w.join();
  }
  // Phase 3: the partitions' ascending first-row runs merged into one
  // first-occurrence order (state.mojo:267-330).
  std::vector<Group> groups;
  std::vector<GroupKey> keys;
  std::vector<uint64_t> key_rows;
  size_t total = 0;
  for (int p = 0; p < P; ++p) total += pgroups[p].size();
  groups.reserve(total);
  keys.reserve(total);
  key_rows.reserve(total);
  using Item = std::pair<uint64_t, int>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  std::vector<size_t> at(P, 0);
  for (int p = 0; p < P; ++p)
    if (!pgroups[p].empty()) heap.push({pgroups[p][0].first_row, p});
  while (!heap.empty()) {
    int p = heap.top().second;
    heap.pop();
    size_t i = at[p]++;
    groups.push_back(std::move(pgroups[p][i]));
    keys.push_back(pkeys[p][i]);
    key_rows.push_back(prows[p][i]);
    if (at[p] < pgroups[p].size()) heap.push({pgroups[p][at[p]].first_row, p});
  }
  ungrouped_row(*q, plan, groups, keys, key_rows);
  auto r = std::make_unique<orc_result>();
  st = finalize(*q, plan, groups, keys, key_rows, r.get());
  if (st) return st;
  *out = r.release();
  return DFC_OK;
}

uint64_t orc_result_rows(const orc_result* r) { return r->rows; }
int32_t orc_result_columns(const orc_result* r) { return (int32_t)r->cols.size(); }
int32_t orc_result_dtype(const orc_result* r, int32_t i) { return r->cols[i].dtype; }
const void* orc_result_values(const orc_result* r, int32_t i) { return r->cols[i].bytes.data(); }
const uint8_t* orc_result_valid(const orc_result* r, int32_t i) { return r->cols[i].valid.data(); }
const uint64_t* orc_result_first_rows(const orc_result* r) { return r->first_rows.data(); }
void orc_result_free(orc_result* r) { delete r; }
const char* orc_error(void) { return g_error.c_str(); }

}  // extern "C"
