// runtime.cu — host side of libdfcuda.so: the C ABI of include/dfcuda.h, the
// resident-column registry, the query planner (key packing, group-record
// layout, shared-memory stage layout, table capacity), launches, bounded
// waits, capacity regrowth and results.
//
// Behaviour mirrors the reference provider contract
// (docs/design/accelerator-contract.md): unsupported work is rejected before
// anything is submitted; errors after submission propagate; checked sums
// report the CPU's exact overflow text; nothing is retried on the CPU.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "dfcuda.h"
#include "dfc_internal.h"
#include "kernels.h"

using namespace dfc;

struct dfc_column {
  uint64_t serial = 0;  // registration number: identifies the column for learned group counts
  int32_t device = 0;
  dfc_dtype dtype = DFC_INT64;
  uint64_t rows = 0;
  void* values = nullptr;        // device
  bool owns_values = false;
  uint32_t* validity = nullptr;  // device, normalised; nullptr when no row is null
  uint64_t null_count = 0;
  // Statistics, computed the first time the column is a key: order-encoded
  // value range and a HyperLogLog estimate of its distinct valid values.
  bool have_stats = false;
  uint64_t min_enc = ~0ull, max_enc = 0;
  double distinct = 0;
};

struct ResultCol {
  dfc_dtype dtype;
  void* values = nullptr;
  uint32_t* validity = nullptr;
  bool has_nulls = false;
};

struct dfc_result {
  int32_t device = 0;
  uint64_t rows = 0;
  std::vector<ResultCol> cols;
  void* slab = nullptr;  // every column's buffers, carved from one allocation
  std::atomic<int> refs{1};
};

namespace {

thread_local std::string t_error;
thread_local dfc_timings t_timings{};

dfc_status fail(dfc_status st, const std::string& msg) {
  t_error = msg;
  return st;
}

dfc_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail(DFC_OOM, std::string("device memory exhausted: ") + what);
  }
  return fail(DFC_DEVICE, std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " +
                              what);
}

#define CK(call, what)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, what);   \
  } while (0)

int dtype_size(int dt) {
  switch (dt) {
    case DFC_INT8: case DFC_UINT8: return 1;
    case DFC_INT16: case DFC_UINT16: return 2;
    case DFC_INT32: case DFC_UINT32: case DFC_FLOAT32: return 4;
    case DFC_INT64: case DFC_UINT64: case DFC_FLOAT64: return 8;
  }
  return 0;
}
bool is_float(int dt) { return dt == DFC_FLOAT32 || dt == DFC_FLOAT64; }
bool is_unsigned(int dt) { return dt == DFC_UINT8 || dt == DFC_UINT16 || dt == DFC_UINT32 || dt == DFC_UINT64; }
const char* dtype_name(int dt) {
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

// Result type of a sum (dataframe/dtype.mojo:838-849).
int sum_dtype(int dt) {
  if (dt == DFC_INT8 || dt == DFC_INT16 || dt == DFC_UINT8 || dt == DFC_UINT16) return DFC_INT64;
  return dt;
}

// Overflow text of the CPU provider (function.mojo:2798 for Int64 inputs,
// :2914 / reducer.mojo:3412 for the others).
std::string overflow_message(int input_dtype) {
  if (input_dtype == DFC_INT64) return "Int64 expression sum overflow";
  return std::string(dtype_name(sum_dtype(input_dtype))) + " expression sum overflow";
}

// The scan kernels (one per table regime) share this signature.
using ScanFn = void (*)(ScanParams);

// The scan kernel for a planned query's table regime.
ScanFn scan_fn(const ScanParams& sp) {
  if (!sp.smem_slots) return scan_kernel_global;
  if (sp.reduce) return scan_kernel_reduce;
  return sp.smem_cluster > 1 ? scan_kernel_cluster : scan_kernel_own;
}

struct DeviceState {
  bool ready = false;
  int sms = 0;
  size_t smem_optin = 0;       // scan_kernel's dynamic shared memory limit
  size_t smem_half = 0;        // scan_kernel's dynamic shared memory at two CTAs per SM
  size_t part_smem_optin = 0;  // partition_kernel's
  size_t count_smem_optin = 0; // partition_count's
  size_t agg_smem_optin = 0;   // partition_aggregate's, one CTA per SM
  size_t agg_smem_half = 0;    // partition_aggregate's at two CTAs per SM
  int scan_occupancy = 1;
};
std::mutex g_dev_mu;
std::map<int, DeviceState> g_dev;

// Group counts seen per query shape (key columns and filter program, literals
// included): a repeat of the same query sizes its table from them (the
// reference sizes from column statistics, dataframe/aggregation/hash_table.mojo:699-714).
// Joint distinct counts of multi-key sets over all rows, per key-column set.
std::mutex g_learn_mu;
std::map<std::vector<uint64_t>, uint64_t> g_learned;
std::map<std::vector<uint64_t>, double> g_joint;
// Key skew per key-column set: {top-1 share, top-kHotSlots share} of a sample.
std::map<std::vector<uint64_t>, std::pair<double, double>> g_skew;
std::atomic<uint64_t> g_column_serial{0};

// dfc_set_memory_limit: the most bytes one query may hold on a device
// (working memory and result columns); <= 0 none.
std::atomic<int64_t> g_memory_limit[64];

// Host-side fault injection (DFCUDA_FAULT, read on every call): `alloc` fails
// the query's working-memory allocation, `capacity` makes the first attempt
// report a full table (the regrowth path reruns it), `timeout` makes the
// host's bounded wait give up at once, `overflow` reports a checked integer
// sum overflow.  Nothing is injected on the GPU.
bool fault_is(const char* what) {
  const char* f = getenv("DFCUDA_FAULT");
  return f && strcmp(f, what) == 0;
}

// The library's own stream-ordered memory pool per device.  Freed query
// memory stays cached in it (queries reuse it without returning to the
// driver); the device's default pool, which other code in the process may
// use, keeps its own release threshold.
constexpr int kMaxDevices = 64;
cudaMemPool_t g_pools[kMaxDevices] = {};

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t stream) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool = dev >= 0 && dev < kMaxDevices ? g_pools[dev] : nullptr;
  if (!pool) return cudaMallocAsync(p, bytes, stream);
  return cudaMallocFromPoolAsync(p, bytes, pool, stream);
}

dfc_status device_ready(int dev, DeviceState** out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (dev < 0 || dev >= kMaxDevices) return fail(DFC_INVALID, "device ordinal out of range");
  DeviceState& d = g_dev[dev];
  if (!d.ready) {
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
    if (prop.major < 10) return fail(DFC_NO_DEVICE, "device is not sm_100 class");
    // Function attributes apply to the current device: set it for the
    // set-up and give the caller's back afterwards.
    int prev = -1;
    cudaGetDevice(&prev);
    CK(cudaSetDevice(dev), "cudaSetDevice");
    struct Restore {
      int prev;
      ~Restore() {
        if (prev >= 0) cudaSetDevice(prev);
      }
    } restore{prev};
    d.sms = prop.multiProcessorCount;
    d.smem_optin = prop.sharedMemPerBlockOptin;
    if (!g_pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t pool;
      CK(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
      uint64_t threshold = UINT64_MAX;
      CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
      g_pools[dev] = pool;
    }
    // Dynamic shared memory may use what the kernel's static buffers leave.
    cudaFuncAttributes fa;
    size_t scan_static = 0;
    for (ScanFn f : {scan_kernel_global, scan_kernel_own, scan_kernel_cluster, scan_kernel_reduce}) {
      CK(cudaFuncGetAttributes(&fa, f), "cudaFuncGetAttributes");
      scan_static = std::max(scan_static, fa.sharedSizeBytes);
    }
    d.smem_optin = prop.sharedMemPerBlockOptin - scan_static;
    d.smem_half = (prop.sharedMemPerMultiprocessor - 2 * prop.reservedSharedMemPerBlock) / 2 - scan_static;
    for (ScanFn f : {scan_kernel_global, scan_kernel_own, scan_kernel_cluster, scan_kernel_reduce})
      CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.smem_optin),
         "cudaFuncSetAttribute");
    // Cluster tables pool the shared memory of up to 16 CTAs.
    CK(cudaFuncSetAttribute(scan_kernel_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
       "cudaFuncSetAttribute");
    // The partition passes: the counting pass and pass A at one CTA per SM,
    // pass B at two when its table fits half an SM.
    d.part_smem_optin = prop.sharedMemPerBlockOptin;
    for (auto f : {partition_kernel, partition_kernel_quad}) {
      CK(cudaFuncGetAttributes(&fa, f), "cudaFuncGetAttributes");
      d.part_smem_optin = std::min(d.part_smem_optin, prop.sharedMemPerBlockOptin - fa.sharedSizeBytes);
    }
    for (auto f : {partition_kernel, partition_kernel_quad})
      CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.part_smem_optin),
         "cudaFuncSetAttribute");
    d.count_smem_optin = prop.sharedMemPerBlockOptin;
    for (auto f : {partition_count, partition_count_quad}) {
      CK(cudaFuncGetAttributes(&fa, f), "cudaFuncGetAttributes");
      d.count_smem_optin = std::min(d.count_smem_optin, prop.sharedMemPerBlockOptin - fa.sharedSizeBytes);
    }
    for (auto f : {partition_count, partition_count_quad})
      CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.count_smem_optin),
         "cudaFuncSetAttribute");
    CK(cudaFuncGetAttributes(&fa, partition_aggregate), "cudaFuncGetAttributes");
    d.agg_smem_optin = prop.sharedMemPerBlockOptin - fa.sharedSizeBytes;
    d.agg_smem_half = (prop.sharedMemPerMultiprocessor - 2 * prop.reservedSharedMemPerBlock) / 2 - fa.sharedSizeBytes;
    CK(cudaFuncSetAttribute(partition_aggregate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.agg_smem_optin),
       "cudaFuncSetAttribute");
    // The output kernel stages each warp's records in shared memory.
    CK(cudaFuncSetAttribute(finish_output, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)finish_output_smem(kMaxRecWords * 8)),
       "cudaFuncSetAttribute");
    d.ready = true;
  }
  *out = &d;
  return DFC_OK;
}

// One non-blocking stream per thread and device, for calls without a stream
// (or the stream the thread chose with dfc_set_thread_stream).
thread_local std::map<int, cudaStream_t> t_streams;
thread_local std::map<int, cudaStream_t> t_chosen;

cudaStream_t thread_stream(int dev) {
  auto c = t_chosen.find(dev);
  if (c != t_chosen.end()) return c->second;
  auto it = t_streams.find(dev);
  if (it != t_streams.end()) return it->second;
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  t_streams[dev] = s;
  return s;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

double wait_limit_seconds() {
  const char* s = getenv("DFC_WAIT_TIMEOUT_S");
  if (s) {
    double v = atof(s);
    if (v > 0) return v;
  }
  return 300.0;
}

// Host-side bounded wait on the stream's work (cudaEventQuery polling).
dfc_status wait_bounded(cudaStream_t stream) {
  if (fault_is("timeout")) return fail(DFC_TIMEOUT, "device work did not finish within the wait limit (injected by DFCUDA_FAULT=timeout)");
  // One completion event per thread and device, created on first use.
  thread_local std::map<int, cudaEvent_t> events;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaEvent_t& ev = events[dev];
  if (!ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
  cudaError_t e = cudaEventRecord(ev, stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  const auto t0 = std::chrono::steady_clock::now();
  const double limit = wait_limit_seconds();
  while (true) {
    e = cudaEventQuery(ev);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(e, "query execution");
    // Poll without sleeping for the first 2 ms (most queries end sooner, and
    // a sleep overshoots by tens of microseconds), then every 20 us.
    const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (waited > limit) return fail(DFC_TIMEOUT, "device work did not finish within the wait limit");
    if (waited > 2e-3) std::this_thread::sleep_for(std::chrono::microseconds(20));
    else std::this_thread::yield();
  }
  return DFC_OK;
}

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Global-table slots per estimated group: the table's load stays at most
// 1/factor of the estimate, and record capacity follows the estimate, not the
// table.  DFC_TABLE_FACTOR=<2,4,8,16> sets it; by default 16 while such a
// table stays within kRoomyTableBytes, else 8.  On the 100M-row, 7.4M-group
// workload the scan took 7.17 ms at 16, 7.48 at 8, 8.10 at 4 and 9.35 at 2:
// shorter probe chains outweigh the table's size.
constexpr uint64_t kRoomyTableBytes = 4ull << 30;

uint64_t table_factor_setting() {
  static const uint64_t f = [] {
    const char* env = getenv("DFC_TABLE_FACTOR");
    const long v = env && *env ? atol(env) : 0;
    return (v == 2 || v == 4 || v == 8 || v == 16) ? (uint64_t)v : 0ull;
  }();
  return f;
}

uint64_t table_factor_for(uint64_t est) {
  if (const uint64_t f = table_factor_setting()) return f;
  return next_pow2(std::max<uint64_t>(1024, est * 16)) * sizeof(KeyEntry) <= kRoomyTableBytes ? 16 : 8;
}

// Host decoding of the order encoding (kernels' order_encode) for integer ranges.
__int128 order_value(uint64_t e, int dt) {
  if (is_unsigned(dt)) return (__int128)e;
  return (__int128)(int64_t)(e ^ 0x8000000000000000ull);
}

// ---------------------------------------------------------------------------
// Planning.
// ---------------------------------------------------------------------------
struct Plan {
  ScanParams sp{};
  FinishParams fp{};
  int n_out = 0;
  int out_dtype[kMaxOut];
  int out_agg_input_dtype[kMaxOut];  // for overflow messages, by aggregation index
  int tile_rows = 1024;
  size_t smem = 0;
  int device = 0;
  uint64_t rows = 0;
  uint64_t est_groups = 0;
  std::vector<uint64_t> key_sig;  // registration numbers of the key columns
  std::vector<uint64_t> shape_sig;  // key_sig, then the filter program (columns by registration number)
  // Key skew from a 16K-row sample of the key words (-1: not measured): the
  // most frequent key's share and the share of the kHotSlots most frequent.
  double top1 = -1, top_hot = -1;
  // Slots a direct-addressed own table needs (plan_direct; 0: not eligible).
  uint64_t direct_slots = 0;
};

// The stage ring for tiles of `tile` rows (a power of two >= 128, so every
// values block (tile * size) and validity block (tile / 8) is a multiple of
// 16 bytes, as bulk copies require): per column its values then validity
// words, the key and filter columns first; 4 stages.  Sets the tile fields
// of P.sp and P.smem (the ring and its mbarriers); returns one stage's bytes.
size_t layout_ring(Plan& P, int tile) {
  ScanParams& sp = P.sp;
  size_t b = 0, stage_tx_count = 0;
  for (int c = 0; c < sp.n_stage; ++c) {
    if (c == sp.n_stage_count) stage_tx_count = b;
    sp.stage_off[c] = (int)b;
    b += (size_t)tile * sp.cols[c].size;
    if (sp.cols[c].validity) {
      sp.stage_voff[c] = (int)b;
      b += (size_t)tile / 8;
    } else {
      sp.stage_voff[c] = -1;
    }
  }
  if (sp.n_stage_count == sp.n_stage) stage_tx_count = b;
  sp.stage_tx = (int)b;
  sp.stage_tx_count = (int)stage_tx_count;
  b = (b + 127) & ~(size_t)127;
  sp.stage_bytes = (int)b;
  sp.tile_rows = tile;
  sp.stages = 4;
  sp.tiles = (P.rows + tile - 1) / tile;
  sp.full_tiles = P.rows / tile;
  P.tile_rows = tile;
  P.smem = (size_t)sp.stages * b + 2 * sp.stages * sizeof(uint64_t);
  return b;
}

dfc_status plan_query(const dfc_query* q, Plan& P) {
  if (!q) return fail(DFC_INVALID, "null query");
  if (q->abi_version != DFC_ABI_VERSION) return fail(DFC_INVALID, "ABI version mismatch");
  if (q->n_inputs < 1 || q->n_inputs > kMaxInputs || !q->inputs)
    return fail(DFC_UNSUPPORTED, "between 1 and 16 input columns are supported");
  if (q->n_keys < 0 || q->n_keys > kMaxKeys || (q->n_keys > 0 && !q->keys))
    return fail(DFC_UNSUPPORTED, "at most 4 keys are supported");
  if (q->n_aggs < 0 || q->n_aggs > kMaxAggs || (q->n_aggs > 0 && !q->aggs))
    return fail(DFC_UNSUPPORTED, "at most 32 aggregations are supported");
  if (q->n_pred < 0 || q->n_pred > kMaxPred || (q->n_pred > 0 && !q->pred))
    return fail(DFC_UNSUPPORTED, "filter programs of at most 32 operations are supported");
  for (int i = 0; i < q->n_inputs; ++i)
    if (!q->inputs[i]) return fail(DFC_INVALID, "null input column");
  const dfc_column* c0 = q->inputs[0];
  P.device = c0->device;
  P.rows = c0->rows;
  for (int i = 1; i < q->n_inputs; ++i) {
    if (q->inputs[i]->rows != P.rows) return fail(DFC_INVALID, "input columns differ in length");
    if (q->inputs[i]->device != P.device) return fail(DFC_UNSUPPORTED, "input columns live on different devices");
  }
  if (P.rows >= 0xFFFFFFFFull) return fail(DFC_UNSUPPORTED, "at most 2^32-2 rows per query");

  ScanParams& sp = P.sp;
  // Slots: the columns the query touches, staged per tile.
  int slot_of[kMaxInputs];
  for (int i = 0; i < kMaxInputs; ++i) slot_of[i] = -1;
  int n_slots = 0;
  auto use = [&](int input) -> int {
    if (slot_of[input] < 0) {
      slot_of[input] = n_slots;
      const dfc_column* c = q->inputs[input];
      DevColumn& dc = sp.cols[n_slots];
      dc.values = c->values;
      dc.validity = c->validity;
      dc.dtype = c->dtype;
      dc.size = dtype_size(c->dtype);
      ++n_slots;
    }
    return slot_of[input];
  };

  // Keys.
  int total_bits = 0;
  sp.n_keys = q->n_keys;
  for (int k = 0; k < q->n_keys; ++k) {
    int in = q->keys[k];
    if (in < 0 || in >= q->n_inputs) return fail(DFC_INVALID, "key index out of range");
    for (int j = 0; j < k; ++j)
      if (q->keys[j] == in) return fail(DFC_INVALID, "duplicate key column");
    const dfc_column* c = q->inputs[in];
    KeyField& f = sp.keys[k];
    f.input = use(in);
    f.dtype = c->dtype;
    f.bits = 8 * dtype_size(c->dtype);
    total_bits += f.bits + (c->validity ? 1 : 0);
    P.key_sig.push_back(c->serial);
  }
  if (total_bits <= 64) {
    sp.key_mode = KEY_PACKED;
    int at = 0;
    for (int k = 0; k < q->n_keys; ++k) {
      KeyField& f = sp.keys[k];
      f.shift = at;
      at += f.bits;
      f.null_bit = -1;
      if (q->inputs[q->keys[k]]->validity) f.null_bit = at++;
    }
  } else {
    sp.key_mode = KEY_TICKET;
    for (int k = 0; k < q->n_keys; ++k) {
      sp.keys[k].shift = 0;
      sp.keys[k].null_bit = -1;
    }
  }

  // Filter program (stack discipline checked here, before submission).
  sp.n_pred = q->n_pred;
  int depth = 0;
  for (int i = 0; i < q->n_pred; ++i) {
    const dfc_pred_op& op = q->pred[i];
    PredOp& d = sp.pred[i];
    d.kind = op.kind;
    d.cmp = op.cmp;
    d.lit.u = op.lit.u;
    d.input = 0;
    switch (op.kind) {
      case DFC_PRED_CMP:
        if (op.cmp < DFC_LT || op.cmp > DFC_NE) return fail(DFC_INVALID, "bad comparison operator");
        /* fallthrough */
      case DFC_PRED_IS_NULL:
      case DFC_PRED_IS_NOT_NULL:
        if (op.column < 0 || op.column >= q->n_inputs) return fail(DFC_INVALID, "filter column out of range");
        d.input = use(op.column);
        ++depth;
        break;
      case DFC_PRED_TRUE:
        ++depth;
        break;
      case DFC_PRED_NOT:
        if (depth < 1) return fail(DFC_INVALID, "malformed filter program");
        break;
      case DFC_PRED_AND:
      case DFC_PRED_OR:
        if (depth < 2) return fail(DFC_INVALID, "malformed filter program");
        --depth;
        break;
      default:
        return fail(DFC_UNSUPPORTED, "unsupported filter operation");
    }
    if (depth > 32) return fail(DFC_UNSUPPORTED, "filter program too deep");
  }
  if (q->n_pred > 0 && depth != 1) return fail(DFC_INVALID, "malformed filter program");
  P.shape_sig = P.key_sig;
  P.shape_sig.push_back(~0ull);
  for (int i = 0; i < q->n_pred; ++i) {
    const dfc_pred_op& op = q->pred[i];
    const bool has_col = op.kind == DFC_PRED_CMP || op.kind == DFC_PRED_IS_NULL || op.kind == DFC_PRED_IS_NOT_NULL;
    P.shape_sig.push_back(((uint64_t)(uint32_t)op.kind << 32) | (uint32_t)op.cmp);
    P.shape_sig.push_back(has_col ? q->inputs[op.column]->serial : 0);
    P.shape_sig.push_back(op.kind == DFC_PRED_CMP ? op.lit.u : 0);
  }
  // Key and filter columns hold the first slots: the partition counting pass
  // stages only those.
  sp.n_stage_count = n_slots;

  // Value states: one ValField per distinct aggregated column.
  struct Need {
    int input;
    bool sum = false, mn = false, mx = false, m2 = false;
  };
  std::vector<Need> needs;
  int val_of_agg[kMaxAggs];
  bool track_len = false, track_first_row = false, track_last = false;
  for (int a = 0; a < q->n_aggs; ++a) {
    const dfc_agg& ag = q->aggs[a];
    if (ag.column < 0 || ag.column >= q->n_inputs) return fail(DFC_INVALID, "aggregation column out of range");
    if (ag.op == DFC_AGG_N_UNIQUE)
      return fail(DFC_UNSUPPORTED, "n_unique runs through dfc_groupby (two device group-bys)");
    if (ag.op < DFC_AGG_COUNT || ag.op > DFC_AGG_LAST) return fail(DFC_UNSUPPORTED, "unsupported aggregation");
    if ((ag.op == DFC_AGG_VAR || ag.op == DFC_AGG_STD) && ag.ddof < 0) return fail(DFC_INVALID, "negative ddof");
    int v = -1;
    for (size_t j = 0; j < needs.size(); ++j)
      if (needs[j].input == ag.column) v = (int)j;
    if (v < 0) {
      if (needs.size() >= (size_t)kMaxVals) return fail(DFC_UNSUPPORTED, "at most 8 aggregated columns");
      v = (int)needs.size();
      needs.push_back(Need{ag.column});
    }
    val_of_agg[a] = v;
    Need& n = needs[v];
    switch (ag.op) {
      case DFC_AGG_SUM: case DFC_AGG_MEAN: n.sum = true; break;
      case DFC_AGG_MIN: n.mn = true; break;
      case DFC_AGG_MAX: n.mx = true; break;
      case DFC_AGG_VAR: case DFC_AGG_STD: n.m2 = true; n.sum = true; break;
      case DFC_AGG_LEN: case DFC_AGG_NULL_COUNT: track_len = true; break;
      case DFC_AGG_FIRST: track_first_row = true; break;
      case DFC_AGG_LAST: track_last = true; break;
      default: break;
    }
  }
  // Group record: header, u32 length and counts, then per column the
  // read-set (K, min, max: read before the atomics that may improve them)
  // and the sums.  The common single-column float record (count, sum, K,
  // min, max, S2) is exactly 64 bytes: one pair of 32-byte sectors.
  sp.n_vals = (int)needs.size();
  int off = kRecHeader;
  sp.off_len = -1;
  if (track_len) {
    sp.off_len = off;
    off += 4;
  }
  sp.off_last = -1;
  if (track_last) {
    sp.off_last = off;
    off += 4;
  }
  for (int j = 0; j < sp.n_vals; ++j) {
    ValField& f = sp.vals[j];
    f.input = use(needs[j].input);
    f.dtype = q->inputs[needs[j].input]->dtype;
    f.off_count = off;
    off += 4;
  }
  off = (off + 7) & ~7;
  for (int j = 0; j < sp.n_vals; ++j) {
    ValField& f = sp.vals[j];
    const Need& n = needs[j];
    const int sz = dtype_size(f.dtype);
    f.sum_kind = SUM_NONE;
    f.off_sum = f.off_min = f.off_max = f.off_m2 = f.off_shift = -1;
    if (n.m2) { f.off_shift = off; off += 8; }
    if (n.mn) { f.off_min = off; off += 8; }
    if (n.mx) { f.off_max = off; off += 8; }
    if (n.sum) {
      if (is_float(f.dtype)) f.sum_kind = SUM_F64;
      else if (sz <= 2 || (sz == 4 && P.rows < (1ull << 31))) f.sum_kind = SUM_I64;
      else f.sum_kind = SUM_I128;
      off = (f.sum_kind == SUM_I128) ? ((off + 15) & ~15) : off;
      f.off_sum = off;
      off += f.sum_kind == SUM_I128 ? 16 : 8;
    }
    if (n.m2) { f.off_m2 = off; off += 8; }
  }
  sp.rec_stride = (off + 15) & ~15;
  if (sp.rec_stride > kMaxRecWords * 8) return fail(DFC_UNSUPPORTED, "group record too wide");
  sp.comp_mask = 0;
  if (q->flags & DFC_Q_FLOAT32_COMPENSATED)
    for (int j = 0; j < sp.n_vals; ++j)
      if (sp.vals[j].dtype == DFC_FLOAT32 && sp.vals[j].off_sum >= 0) sp.comp_mask |= 1u << j;
  sp.rec_words = sp.rec_stride / 8;
  // Group sizes in a warp from which the rows of one key fold by butterflies
  // (one atomic per field) instead of per-lane atomics: the table scans and
  // pass B.  DFC_COLLAPSE_MIN / DFC_AGG_COLLAPSE_MIN=<n> (tuning; 33: never).
  sp.collapse_min = 4;
  sp.agg_collapse_min = 12;
  if (const char* env = getenv("DFC_COLLAPSE_MIN"))
    if (atoi(env) > 0) sp.collapse_min = atoi(env);
  if (const char* env = getenv("DFC_AGG_COLLAPSE_MIN"))
    if (atoi(env) > 0) sp.agg_collapse_min = atoi(env);
  // FIRST reads the group's earliest kept row, which maintain_order tracks.
  sp.track_first = ((q->flags & DFC_Q_MAINTAIN_ORDER) || track_first_row) ? 1 : 0;

  // Output columns: keys, then one per aggregation.
  FinishParams& fp = P.fp;
  int n_out = 0;
  for (int k = 0; k < q->n_keys; ++k) {
    OutCol& oc = fp.out[n_out];
    oc.kind = OUT_KEY;
    oc.index = k;
    oc.dtype = q->inputs[q->keys[k]]->dtype;
    P.out_dtype[n_out++] = oc.dtype;
  }
  for (int a = 0; a < q->n_aggs; ++a) {
    const dfc_agg& ag = q->aggs[a];
    const int idt = q->inputs[ag.column]->dtype;
    OutCol& oc = fp.out[n_out];
    oc.kind = OUT_AGG;
    oc.index = a;
    oc.val = val_of_agg[a];
    oc.op = ag.op;
    oc.ddof = ag.ddof;
    oc.min_count = ag.min_count;
    switch (ag.op) {
      case DFC_AGG_COUNT: case DFC_AGG_LEN: case DFC_AGG_NULL_COUNT: oc.dtype = DFC_INT64; break;
      case DFC_AGG_SUM: oc.dtype = sum_dtype(idt); break;
      case DFC_AGG_MIN: case DFC_AGG_MAX: case DFC_AGG_FIRST: case DFC_AGG_LAST: oc.dtype = idt; break;
      default: oc.dtype = DFC_FLOAT64; break;
    }
    P.out_agg_input_dtype[a] = idt;
    P.out_dtype[n_out++] = oc.dtype;
  }
  fp.n_out = n_out;
  P.n_out = n_out;

  // Stage layout: the largest tile whose 4-stage ring fits in 96 KB.
  sp.n_stage = n_slots;
  sp.n_cols = n_slots;
  sp.rows = P.rows;
  bool aligned = true;
  for (int c = 0; c < n_slots; ++c)
    if (((uintptr_t)sp.cols[c].values & 15u) != 0) aligned = false;
  sp.use_tma = aligned ? 1 : 0;
  int tile = 1024;
  while (tile >= 128 && layout_ring(P, tile) * 4 > 96 * 1024) tile >>= 1;
  if (tile < 128) return fail(DFC_UNSUPPORTED, "too many input columns for the stage ring");
  return DFC_OK;
}

// Estimated number of groups: what the last query on these keys found, else
// the product of the key columns' value ranges, capped by the row count.
// Column statistics, computed once per column on its first use as a key.
std::mutex g_stats_mu;

// HyperLogLog estimate (Flajolet et al. 2007) with the linear-counting
// correction for small cardinalities.
double hll_estimate(const std::vector<uint32_t>& regs) {
  double sum = 0;
  int zeros = 0;
  for (uint32_t r : regs) {
    sum += std::ldexp(1.0, -(int)r);
    zeros += r == 0;
  }
  const double m = (double)regs.size(), alpha = 0.7213 / (1.0 + 1.079 / m);
  double est = alpha * m * m / sum;
  if (est <= 2.5 * m && zeros > 0) est = m * std::log(m / zeros);
  return est;
}

// Resident 256-thread blocks per SM of a statistics kernel (cached): its
// grid-stride loop then runs in one wave.
unsigned stats_blocks_per_sm(const void* fn) {
  static std::mutex mu;
  static std::map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(fn);
  if (it != cache.end()) return (unsigned)it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 256, 0) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = 4;
  }
  cache[fn] = n;
  return (unsigned)n;
}

// Distinct key words of the query over all rows (HyperLogLog; 0 on failure).
double joint_key_estimate(const Plan& P, DeviceState* ds, cudaStream_t stream) {
  const uint32_t nreg = 1u << kHllBits;
  uint32_t* d_regs = nullptr;
  std::vector<uint32_t> regs(nreg);
  cudaError_t e = pool_alloc((void**)&d_regs, nreg * 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_regs, 0, nreg * 4, stream);
  if (e == cudaSuccess) {
    const unsigned blocks = (unsigned)std::min<uint64_t>((P.rows + 255) / 256, (uint64_t)ds->sms * stats_blocks_per_sm((const void*)keys_hll));
    keys_hll<<<std::max(1u, blocks), 256, 0, stream>>>(P.sp, d_regs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(regs.data(), d_regs, nreg * 4, cudaMemcpyDeviceToHost, stream);
  if (d_regs) cudaFreeAsync(d_regs, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return hll_estimate(regs) * 1.05 + 16;  // ~1.6% standard error at 4096 registers: keep a margin
}

dfc_status ensure_stats(dfc_column* c, DeviceState* ds, cudaStream_t stream) {
  std::lock_guard<std::mutex> lk(g_stats_mu);
  if (c->have_stats || c->rows == 0) return DFC_OK;
  const uint32_t nreg = 1u << kHllBits;
  unsigned long long* d_mm = nullptr;
  uint32_t* d_regs = nullptr;
  unsigned long long h_mm[2] = {~0ull, 0ull};
  std::vector<uint32_t> regs(nreg);
  cudaError_t e = pool_alloc((void**)&d_mm, 16, stream);
  if (e == cudaSuccess) e = pool_alloc((void**)&d_regs, nreg * 4, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_mm, h_mm, 16, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_regs, 0, nreg * 4, stream);
  if (e == cudaSuccess) {
    DevColumn dc{c->values, c->validity, c->dtype, dtype_size(c->dtype)};
    const unsigned blocks = (unsigned)std::min<uint64_t>((c->rows + 255) / 256, (uint64_t)ds->sms * stats_blocks_per_sm((const void*)column_stats));
    column_stats<<<std::max(1u, blocks), 256, 0, stream>>>(dc, c->rows, d_mm, d_regs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_mm, d_mm, 16, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(regs.data(), d_regs, nreg * 4, cudaMemcpyDeviceToHost, stream);
  if (d_mm) cudaFreeAsync(d_mm, stream);
  if (d_regs) cudaFreeAsync(d_regs, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "column statistics");
  const double est = hll_estimate(regs);
  c->min_enc = h_mm[0];
  c->max_enc = h_mm[1];
  c->distinct = est;
  c->have_stats = true;
  return DFC_OK;
}

// Estimated number of groups: what the last query of the same shape found
// (when `learned`), else the product of the key columns' distinct estimates
// (capped by their value ranges), capped by the row count.  The statistics
// describe all rows, so for a filtered query they bound the count from above.
uint64_t estimate_groups(const dfc_query* q, const Plan& P, DeviceState* ds, cudaStream_t stream, bool learned = true) {
  if (learned) {
    // DFC_GROUPS_ESTIMATE=<n> replaces the first estimate (capacity regrowth tests).
    if (const char* env = getenv("DFC_GROUPS_ESTIMATE")) {
      const long long v = atoll(env);
      if (v > 0) return (uint64_t)v;
    }
    std::lock_guard<std::mutex> lk(g_learn_mu);
    auto it = g_learned.find(P.shape_sig);
    if (it != g_learned.end()) return it->second;
  }
  double prod = 1.0;
  for (int k = 0; k < q->n_keys; ++k) {
    dfc_column* c = q->inputs[q->keys[k]];
    double d = (double)c->rows;
    if (ensure_stats(c, ds, stream) == DFC_OK && c->have_stats) {
      // HyperLogLog's standard error at 4096 registers is ~1.6%: keep a margin.
      d = std::min(d, c->distinct * 1.1 + 16);
      if (!is_float(c->dtype) && c->min_enc <= c->max_enc) {
        const __int128 span = order_value(c->max_enc, c->dtype) - order_value(c->min_enc, c->dtype) + 1;
        if (span > 0 && (double)span < d) d = (double)span;
      }
    }
    if (c->validity) d += 1;
    prod *= d;
  }
  // Several keys: the product bounds the group count loosely (correlated
  // keys, Zipf pairs); the key words' own distinct count is the estimate.
  if (q->n_keys > 1 && prod > 65536 && P.rows > 0) {
    double joint = 0;
    {
      std::lock_guard<std::mutex> lk(g_learn_mu);
      auto it = g_joint.find(P.key_sig);
      if (it != g_joint.end()) joint = it->second;
    }
    if (joint <= 0) {
      joint = joint_key_estimate(P, ds, stream);
      std::lock_guard<std::mutex> lk(g_learn_mu);
      if (joint > 0) g_joint[P.key_sig] = joint;
    }
    if (joint > 0) prod = std::min(prod, joint);
  }
  double est = std::min(prod, (double)P.rows);
  return (uint64_t)std::max(1.0, est);
}

// Direct addressing (dataframe/aggregation/perfect_hash.mojo:1-50): integer
// keys whose exact value ranges are known, each taking bit_width(range)
// bits (0 for null, value - min + 1 otherwise), at most kDirectBits in all,
// the first key highest.  Sets the kernel's fields and P.direct_slots; an
// own table the regime picks then uses them instead of hashing.
constexpr int kDirectBits = 12;
void plan_direct(const dfc_query* q, Plan& P, DeviceState* ds, cudaStream_t stream) {
  ScanParams& sp = P.sp;
  sp.direct = 0;
  P.direct_slots = 0;
  if (sp.key_mode != KEY_PACKED || q->n_keys <= 0 || getenv("DFC_NO_DIRECT")) return;
  int total = 0;
  int shift[kMaxKeys] = {};
  uint64_t mins[kMaxKeys] = {};
  for (int k = q->n_keys - 1; k >= 0; --k) {
    dfc_column* c = q->inputs[q->keys[k]];
    if (is_float(c->dtype) || c->rows == 0) return;
    if (ensure_stats(c, ds, stream) != DFC_OK || !c->have_stats || c->min_enc > c->max_enc) return;
    const __int128 lo = order_value(c->min_enc, c->dtype);
    const __int128 span = order_value(c->max_enc, c->dtype) - lo + 1;  // fields 1..span; 0 is null
    if (span <= 0 || span >= ((__int128)1 << 31)) return;
    int bits = 0;
    while (((__int128)1 << bits) <= span) ++bits;
    shift[k] = total;
    total += bits;
    if (total > kDirectBits) return;
    mins[k] = (uint64_t)lo;  // two's complement: the kernel subtracts in the key's width
  }
  for (int k = 0; k < q->n_keys; ++k) {
    sp.dshift[k] = shift[k];
    sp.dmin[k] = mins[k];
  }
  P.direct_slots = 1ull << total;
}

// Per-CTA hot-key tables: slots, and the sampled share of rows their keys
// must cover to be used when the groups do not fit a CTA.
constexpr uint64_t kHotSlots = 512;
constexpr double kHotCoverage = 0.6;
constexpr uint64_t kOwnAlwaysGroups = 256;  // own tables whatever the skew
constexpr double kSkewedTop1 = 0.01;        // own tables up to 4096 groups

// The key skew of the query's key columns over all rows (the filter is not
// applied), from the key words of 16K evenly spaced rows (sorted on the host:
// about 1 ms; the decisions compare shares against 1% and 60%); cached per
// key set.
void measure_skew(Plan& P, DeviceState* ds, cudaStream_t stream) {
  {
    std::lock_guard<std::mutex> lk(g_learn_mu);
    auto it = g_skew.find(P.key_sig);
    if (it != g_skew.end()) {
      P.top1 = it->second.first;
      P.top_hot = it->second.second;
      return;
    }
  }
  if (P.rows == 0) return;
  const uint32_t n = (uint32_t)std::min<uint64_t>(P.rows, 16384);
  const uint64_t stride = P.rows / n;
  unsigned long long* d = nullptr;
  std::vector<unsigned long long> h(n);
  cudaError_t e = pool_alloc((void**)&d, (size_t)n * 8, stream);
  if (e == cudaSuccess) {
    keys_sample<<<std::max(1u, std::min((n + 255) / 256, (uint32_t)ds->sms * 4)), 256, 0, stream>>>(P.sp, d, n, stride);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, (size_t)n * 8, cudaMemcpyDeviceToHost, stream);
  if (d) cudaFreeAsync(d, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  // Rows per distinct key word (open addressing over at least 2n slots),
  // then a histogram of those counts: the largest count, and the rows the
  // kHotSlots most frequent keys cover, without sorting the sample.
  const uint32_t cap = (uint32_t)next_pow2(2ull * n);
  std::vector<unsigned long long> keys(cap);
  std::vector<uint32_t> count(cap, 0);
  const int shift = 64 - __builtin_ctzll(cap);
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t slot = shift >= 64 ? 0 : (uint32_t)((h[i] * 0x9E3779B97F4A7C15ull) >> shift);
    while (count[slot] && keys[slot] != h[i]) slot = (slot + 1) & (cap - 1);
    keys[slot] = h[i];
    count[slot] += 1;
  }
  std::vector<uint32_t> keys_with(n + 1, 0);
  for (uint32_t c : count)
    if (c) keys_with[c] += 1;
  uint32_t top = n;
  while (top > 1 && keys_with[top] == 0) --top;
  uint64_t hot = 0, taken = 0;
  for (uint32_t c = top; c >= 1 && taken < kHotSlots; --c) {
    const uint64_t k = std::min<uint64_t>(keys_with[c], kHotSlots - taken);
    hot += k * c;
    taken += k;
  }
  P.top1 = (double)top / n;
  P.top_hot = (double)hot / n;
  std::lock_guard<std::mutex> lk(g_learn_mu);
  g_skew[P.key_sig] = {P.top1, P.top_hot};
}

void learn_groups(const Plan& P, uint64_t groups) {
  std::lock_guard<std::mutex> lk(g_learn_mu);
  g_learned[P.shape_sig] = groups;
}

// Occupancy answers per (kernel, cluster size, shared memory), cached: the
// queries ask the same few shapes again and again.
std::mutex g_occ_mu;
std::map<std::tuple<const void*, uint32_t, size_t>, int> g_occ;

// Co-resident clusters of `ranks` scan CTAs with `smem` dynamic bytes each.
int scan_clusters_uncached(uint32_t ranks, size_t smem);
int scan_clusters(uint32_t ranks, size_t smem) {
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple((const void*)scan_kernel_cluster, ranks + 64u * (uint32_t)dev, smem);
  {
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) return it->second;
  }
  const int n = scan_clusters_uncached(ranks, smem);
  std::lock_guard<std::mutex> lk(g_occ_mu);
  g_occ[key] = n;
  return n;
}

int scan_clusters_uncached(uint32_t ranks, size_t smem) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ranks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(ranks);
  cfg.blockDim = dim3(kScanThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (void*)scan_kernel_cluster, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Shared-memory tables for an estimate of `est` groups at the current ring.
// `own`: each CTA keeps its own table at load <= 1/2 (up to 4096 groups).
// Otherwise the CTAs of a thread-block cluster (2..16) pool their shared
// memory into one table (up to 32K groups), each share at average load
// <= 0.7: the smallest cluster whose shares fit at two CTAs per SM, else the
// smallest at one.  Cluster tables are chosen only where on-chip partials are
// required (compensated FP32 fields) or asked for (DFC_Q_FORCE_SHARED,
// DFC_SMEM_CLUSTER=<2..16>, which also picks the size): on B200, 100M rows
// over 10K uniform keys took 31 ms in a cluster table against 4.6 ms in the
// global table in L2.  Sets P.sp's shared-memory fields and P.smem; false:
// none fits.
constexpr uint64_t kOwnTableGroups = 4096;
constexpr uint64_t kClusterTableGroups = 32768;
bool plan_shared_at(Plan& P, DeviceState* ds, uint64_t est, uint32_t flags, bool own) {
  ScanParams& sp = P.sp;
  const bool force = (flags & DFC_Q_FORCE_SHARED) != 0;
  const size_t ring = P.smem;
  const size_t keys_off = (ring + 15) & ~(size_t)15;
  auto recs_at = [&](uint64_t sslots) { return (keys_off + sslots * 8 + 15) & ~(size_t)15; };
  auto total_for = [&](uint64_t sslots) { return recs_at(sslots) + sslots * (size_t)sp.rec_stride; };
  auto take = [&](uint64_t sslots, uint32_t ranks) {
    sp.smem_slots = (uint32_t)sslots;
    sp.smem_cluster = ranks;
    sp.smem_keys_off = (uint32_t)keys_off;
    sp.smem_recs_off = (uint32_t)recs_at(sslots);
    P.smem = total_for(sslots);
    return true;
  };
  uint32_t want = 0;
  if (const char* env = getenv("DFC_SMEM_CLUSTER")) want = (uint32_t)atoi(env);
  if (own) {
    // Own tables: always for a few groups; up to 4096 groups when the keys
    // are skewed (a hot key's updates stay in each CTA instead of meeting on
    // one global record); beyond that a kHotSlots table that caches the keys
    // that come first (the hot ones) when those cover enough of the rows.
    // Measured on B200 (512 queries of 1K-20M rows): uniform keys over 300 to
    // 4K groups ran 1.5-2.5x faster in the global table, skewed ones up to
    // 1.4x faster in own tables, and Zipf keys over 8K-300K groups about 1.7x
    // faster with a 512-slot hot table; the 100M-row query over 7.4M (Int32
    // Zipf, code) pairs, whose 512 most frequent keys cover 31% of the rows,
    // ran 3x slower with one (misses probe a full table).  DFC_HOT_SLOTS=<n>
    // forces an n-slot hot table (tuning).
    uint64_t hot = 0;
    if (const char* env = getenv("DFC_HOT_SLOTS"))
      if (atoll(env) > 0) hot = next_pow2(std::max<uint64_t>(64, (uint64_t)atoll(env)));
    const bool skewed = P.top1 >= kSkewedTop1;
    // Compensated FP32 fields need on-chip partials: own tables whenever they fit.
    const bool sized = est <= kOwnAlwaysGroups || ((skewed || sp.comp_mask) && est <= kOwnTableGroups);
    if (!force && !hot && !sized && est > kOwnTableGroups && P.top_hot >= kHotCoverage) hot = kHotSlots;
    if (want >= 2 || (!force && !hot && !sized)) return false;
    const uint64_t sslots =
        hot ? hot : next_pow2(std::max<uint64_t>(64, std::min<uint64_t>(est, kOwnTableGroups) * 2));
    if (!hot && P.direct_slots > 0) {
      // Direct addressing: every possible key its own slot, when that table
      // still fits two CTAs per SM or is no larger than the hashed one.
      const uint64_t dslots = std::max<uint64_t>(64, P.direct_slots);
      if (total_for(dslots) <= ds->smem_optin && (total_for(dslots) <= ds->smem_half || dslots <= sslots)) {
        sp.direct = 1;
        return take(dslots, 1);
      }
    }
    // smem_optin already excludes the kernel's static shared memory.
    return total_for(sslots) <= ds->smem_optin && take(sslots, 1);
  }
  auto share = [&](uint32_t ranks) {
    return next_pow2(std::max<uint64_t>(64, (uint64_t)std::ceil((double)std::max<uint64_t>(est, 1) * 1.4 / ranks)));
  };
  if (want >= 2) {
    if (want > 16 || (want & (want - 1))) return false;
    const uint64_t sslots = share(want);
    if (total_for(sslots) > ds->smem_optin || scan_clusters(want, total_for(sslots)) < 1) return false;
    return take(sslots, want);
  }
  if (!force && (est > kClusterTableGroups || sp.comp_mask == 0)) return false;
  for (size_t budget : {ds->smem_half, ds->smem_optin}) {
    for (uint32_t ranks = 2; ranks <= 16; ranks *= 2) {
      const uint64_t sslots = share(ranks);
      const size_t total = total_for(sslots);
      if (total > budget || scan_clusters(ranks, total) < 1) continue;
      return take(sslots, ranks);
    }
  }
  return false;
}

bool plan_quad(ScanParams& sp);

// Own tables, then cluster tables, each with the query's ring or else with
// smaller tiles (down to 256 rows) that leave the tables more room; the ring
// is restored when nothing fits.  Packed keys only; false: the global table
// alone.
bool plan_shared(Plan& P, DeviceState* ds, uint64_t est, uint32_t flags) {
  ScanParams& sp = P.sp;
  sp.smem_slots = 0;
  sp.smem_cluster = 1;
  sp.direct = 0;
  sp.reduce = 0;
  if ((flags & DFC_Q_FORCE_GLOBAL) || sp.key_mode != KEY_PACKED) return false;
  if (sp.n_keys == 0) {
    // No key: one small own table, so the stage ring may take most of the
    // shared memory of two CTAs per SM.  Narrow columns need the depth: a
    // 4-stage ring of 4 KB tiles keeps too few bytes in flight per SM.
    const size_t table = 64 * (8 + (size_t)sp.rec_stride) + 64;
    const size_t per = (size_t)sp.stage_bytes + 2 * sizeof(uint64_t);
    const size_t budget = ds->smem_half > table ? ds->smem_half - table : 0;
    sp.stages = (int)std::max<size_t>(4, std::min<size_t>(16, budget / per));
    P.smem = (size_t)sp.stages * per;
  }
  const int tile0 = sp.tile_rows;
  for (bool own : {true, false}) {
    for (int tile = tile0; tile >= std::min(tile0, 256); tile >>= 1) {
      if (tile != sp.tile_rows) layout_ring(P, tile);
      if (plan_shared_at(P, ds, est, flags, own)) {
        // No key, an own table and value columns that fit the register
        // path: per-thread states instead of per-row updates of one record.
        // DFC_NO_REDUCE=1 keeps the per-row path (tuning).
        sp.reduce = sp.n_keys == 0 && sp.smem_cluster <= 1 && sp.comp_mask == 0 && sp.n_vals <= kReduceVals &&
                    !getenv("DFC_NO_REDUCE");
        // Its rows four at a time when the filter is one range test
        // (fast_rows; DFC_NO_QUAD=1 keeps one row per lane).
        if (sp.reduce && !(plan_quad(sp) && !getenv("DFC_NO_QUAD"))) sp.fast_rows = 0;
        return true;
      }
    }
  }
  if (sp.tile_rows != tile0) layout_ring(P, tile0);
  return false;
}

// CTAs of the scan per SM at P.smem (cluster launches: co-resident CTAs in
// whole clusters).
uint64_t scan_capacity(const Plan& P, DeviceState* ds) {
  if (P.sp.smem_cluster > 1)
    return (uint64_t)std::max(1, scan_clusters(P.sp.smem_cluster, P.smem)) * P.sp.smem_cluster;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple((const void*)scan_fn(P.sp), 64u * (uint32_t)dev, P.smem);
  int occ = -1;
  {
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) occ = it->second;
  }
  if (occ < 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, scan_fn(P.sp), kScanThreads, P.smem) != cudaSuccess) {
      cudaGetLastError();
      occ = 1;
    }
    std::lock_guard<std::mutex> lk(g_occ_mu);
    g_occ[key] = occ;
  }
  return (uint64_t)ds->sms * std::max(1, occ);
}

// The scan's persistent grid: every co-resident CTA, at most one per tile
// (cluster launches: whole clusters).
uint64_t scan_grid(const Plan& P, DeviceState* ds) {
  const uint64_t tiles = std::max<uint64_t>(1, P.sp.tiles);
  const uint64_t cap = scan_capacity(P, ds);
  if (P.sp.smem_cluster > 1) {
    const uint64_t r = P.sp.smem_cluster;
    return std::min<uint64_t>(cap / r, (tiles + r - 1) / r) * r;
  }
  return std::max<uint64_t>(1, std::min<uint64_t>(cap, tiles));
}

cudaError_t launch_scan(const ScanParams& sp, uint64_t ncta, size_t smem, cudaStream_t stream) {
  const ScanFn fn = scan_fn(sp);
  if (fn != scan_kernel_cluster) {
    fn<<<(unsigned)ncta, kScanThreads, smem, stream>>>(sp);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = sp.smem_cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)ncta);
  cfg.blockDim = dim3(kScanThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, scan_kernel_cluster, sp);
}

// A query's output columns, sized for out_rows groups, carved from one
// stream-ordered allocation (256-byte aligned pieces: each column's values,
// then its validity words).  One allocation instead of two per column.
cudaError_t alloc_result_cols(const Plan& P, uint64_t out_rows, std::vector<ResultCol>& rc, void** slab,
                              cudaStream_t stream) {
  rc.assign(P.n_out, ResultCol{});
  auto piece = [](uint64_t bytes) { return (std::max<uint64_t>(bytes, 256) + 255) & ~(uint64_t)255; };
  std::vector<uint64_t> off(2 * (size_t)P.n_out);
  uint64_t total = 0;
  for (int c = 0; c < P.n_out; ++c) {
    off[2 * c] = total;
    total += piece(out_rows * dtype_size(P.out_dtype[c]));
    off[2 * c + 1] = total;
    total += piece(((out_rows + 31) / 32) * 4);
  }
  cudaError_t e = pool_alloc(slab, std::max<uint64_t>(total, 256), stream);
  if (e != cudaSuccess) {
    *slab = nullptr;
    cudaGetLastError();
    return e;
  }
  unsigned char* base = static_cast<unsigned char*>(*slab);
  for (int c = 0; c < P.n_out; ++c) {
    rc[c].dtype = (dfc_dtype)P.out_dtype[c];
    rc[c].values = base + off[2 * c];
    rc[c].validity = reinterpret_cast<uint32_t*>(base + off[2 * c + 1]);
  }
  return cudaSuccess;
}

// Releases output columns that did not become a result.
void release_result_cols(std::vector<ResultCol>& rc, void*& slab, cudaStream_t stream) {
  if (slab) cudaFreeAsync(slab, stream);
  slab = nullptr;
  for (auto& r : rc) r.values = nullptr, r.validity = nullptr;
}

// A query's working buffers carved from one stream-ordered allocation:
// alloc() records each request (256-byte aligned), commit() allocates the
// block and sets every recorded pointer.
struct Scratch {
  cudaStream_t stream = nullptr;
  void* block = nullptr;
  std::vector<std::pair<void**, size_t>> wants;
  size_t total = 0;
  dfc_status alloc(void** p, size_t bytes, const char*) {
    wants.push_back({p, total});
    total += (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
    *p = nullptr;
    return DFC_OK;
  }
  dfc_status commit(const char* what) {
    if (fault_is("alloc")) return fail(DFC_OOM, std::string(what) + ": allocation failed (injected by DFCUDA_FAULT=alloc)");
    cudaError_t e = pool_alloc(&block, std::max<size_t>(total, 256), stream);
    if (e != cudaSuccess) {
      block = nullptr;
      return cuda_fail(e, what);
    }
    for (auto& w : wants) *w.first = static_cast<unsigned char*>(block) + w.second;
    return DFC_OK;
  }
  void release() {
    if (block) cudaFreeAsync(block, stream);
    block = nullptr;
    wants.clear();
    total = 0;
  }
};

// The attempt's timing events, created once per thread and device.
cudaEvent_t* attempt_events(int device) {
  thread_local std::map<int, std::array<cudaEvent_t, 6>> events;
  auto it = events.find(device);
  if (it == events.end()) {
    std::array<cudaEvent_t, 6> ev{};
    for (auto& x : ev) cudaEventCreate(&x);
    it = events.emplace(device, ev).first;
  }
  return it->second.data();
}

// Control block copied back after every attempt.
struct Control {
  uint32_t status[4];  // [0] StatusBits, [1] CapacityBits, [2] partition-pass index checks
  uint32_t groups;
  uint32_t overflow_agg;
  uint32_t alloc;
  uint32_t part_next;
  uint32_t part_kept;  // radix-partitioned regime: rows the filter kept (the counting pass's total)
  uint32_t pad[3];
  uint32_t has_nulls[kMaxOut];
};

// Radix-partitioned regime sizing (the ScanParams fields of that name).
struct PartPlan {
  uint32_t bits = 0;
  uint32_t words = 0;
  uint32_t agg_slots = 0;
  uint64_t recs = 0;
  int count_stages = 0;       // counting pass ring stages
  int count_stage_bytes = 0;  // and their stride (the key and filter columns only)
  int stages = 0;             // pass A ring stages (every staged column)
  size_t count_smem = 0;      // counting pass dynamic shared memory
  size_t smem = 0;            // pass A
  size_t agg_smem = 0;        // pass B
  uint64_t ctas = 0;          // counting pass and pass A grid: one CTA per SM
  uint64_t agg_ctas = 0;      // pass B grid: every resident CTA
};

// A pass B table holds a partition's groups at load <= kAggLoad on average
// (partitions take groups by a hash, so their sizes vary by a few percent).
// A warp's probe lasts as long as its longest chain, so the load is kept low:
// on the 100M-row, 7.4M-group workload pass B took 7.8, 4.7 and 3.6 ms at
// loads of 0.51, 0.26 and 0.13.
constexpr double kAggLoad = 0.25;
constexpr uint32_t kPartMinBits = 10;  // at least 1024 partitions: pass B balances over them

// Sizes the regime for `est` groups with at least 2^min_bits partitions;
// false when it does not apply (keys wider than 64 bits, records too wide
// for a shared-memory table, more groups than 2^15 tables hold).
bool plan_partitions(const Plan& P, const DeviceState* ds, uint64_t est, PartPlan& pp, uint32_t min_bits = 0) {
  const ScanParams& sp = P.sp;
  if (sp.key_mode != KEY_PACKED || P.rows == 0 || P.rows >= 0xFFFFFFFFull) return false;
  pp.words = 2 + (uint32_t)sp.n_vals;
  const size_t rs = (size_t)sp.rec_stride + 8;  // the shared-memory record stride (scan.cu agg_stride)
  const double groups = (double)std::max<uint64_t>(est, 1);
  // Slots of a table in `bytes` (any count, a multiple of 32), besides the
  // record of the all-ones key word; each slot also takes a 4-byte entry of
  // the claimed-slot list.
  auto slots_in = [&](size_t bytes) {
    return bytes > rs ? (uint64_t)((bytes - rs) / (rs + 4)) & ~(uint64_t)31 : 0ull;
  };
  // DFC_PART_MIN_BITS=<n> raises the least partition count (tuning).
  if (const char* env = getenv("DFC_PART_MIN_BITS"))
    if (atoi(env) > 0) min_bits = std::max<uint32_t>(min_bits, (uint32_t)atoi(env));
  // DFC_AGG_LOAD=<x> (tuning) replaces kAggLoad.
  double load = kAggLoad;
  if (const char* env = getenv("DFC_AGG_LOAD"))
    if (atof(env) > 0.0 && atof(env) < 0.875) load = atof(env);
  auto bits_for = [&](uint64_t slots) {
    uint32_t b = std::max(kPartMinBits, min_bits);
    while (b < (uint32_t)kPartMaxBits && groups / (double)(1ull << b) > (double)slots * load) ++b;
    return b;
  };
  // Two pass B CTAs per SM when their tables hold the groups, else one CTA
  // per SM with twice the table.
  uint64_t slots = slots_in(ds->agg_smem_half);
  uint32_t bits = bits_for(slots);
  const bool two = slots >= 256 && groups / (double)(1ull << bits) <= (double)slots * load;
  if (!two) {
    slots = slots_in(ds->agg_smem_optin);
    bits = bits_for(slots);
  }
  if (slots < 64 || bits > (uint32_t)kPartMaxBits || groups / (double)(1ull << bits) > (double)slots * load)
    return false;
  pp.bits = bits;
  pp.agg_slots = (uint32_t)slots;
  pp.agg_smem = (slots + 1) * rs + slots * 4;
  pp.agg_ctas = (uint64_t)ds->sms * (two ? 2 : 1);
  // Counting pass: a ring of the key and filter columns only (they hold the
  // first bytes of every stage), then one counter per partition.
  const size_t mbar = 2 * sizeof(uint64_t);
  pp.count_stage_bytes = (int)(((size_t)sp.stage_tx_count + 127) & ~(size_t)127);
  const size_t counters = (size_t)4 << bits;
  if (ds->count_smem_optin <= counters) return false;
  pp.count_stages = (int)std::min<size_t>(16, (ds->count_smem_optin - counters) / (pp.count_stage_bytes + mbar));
  if (pp.count_stages < 4) return false;
  pp.count_smem = (size_t)pp.count_stages * (pp.count_stage_bytes + mbar) + counters;
  // Pass A: a ring of every staged column.
  pp.stages = (int)std::min<size_t>(8, ds->part_smem_optin / ((size_t)sp.stage_bytes + mbar));
  if (pp.stages < 4) return false;
  pp.smem = (size_t)pp.stages * ((size_t)sp.stage_bytes + mbar);
  pp.ctas = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ds->sms, sp.tiles));
  // Every group once, plus the unused tail of each pass B CTA's last chunk.
  pp.recs = std::min<uint64_t>(0xFFFFFFDFull, (uint64_t)(groups * 1.25) + 4096 + pp.agg_ctas * kRecChunk);
  return true;
}

// The quad row path of the partition passes (ScanParams::fast_rows): staged
// 1024-row tiles, integer key columns, and no filter or one comparison, put
// in range form here: the row is selected when its valid value x satisfies
// (lo <= x <= hi) != neg, with the comparison semantics of the kernels'
// select_word_cmp (floats in their own type, UInt64 unsigned, other integers
// as Int64).  False leaves the generic row path.
bool plan_quad(ScanParams& sp) {
  sp.fast_rows = 0;
  sp.fast_col = -1;
  sp.fast_neg = 0;
  sp.fast_kind = FAST_SIGNED;
  if (sp.tile_rows != 1024 || !sp.use_tma || sp.key_mode != KEY_PACKED) return false;
  for (int k = 0; k < sp.n_keys; ++k)
    if (is_float(sp.keys[k].dtype)) return false;
  if (sp.n_pred == 0) {
    sp.fast_rows = 1;
    return true;
  }
  if (sp.n_pred != 1 || sp.pred[0].kind != DFC_PRED_CMP) return false;
  const PredOp& op = sp.pred[0];
  const int dt = sp.cols[op.input].dtype;
  const int cmp = op.cmp;
  sp.fast_col = op.input;
  sp.fast_neg = cmp == DFC_NE ? 1 : 0;
  if (is_float(dt)) {
    sp.fast_kind = FAST_FLOAT;
    const double inf = std::numeric_limits<double>::infinity();
    double lit = op.lit.f, below, above;
    if (dt == DFC_FLOAT32) {
      const float lf = (float)lit;
      lit = lf;
      below = std::nextafter(lf, -std::numeric_limits<float>::infinity());
      above = std::nextafter(lf, std::numeric_limits<float>::infinity());
    } else {
      below = std::nextafter(lit, -inf);
      above = std::nextafter(lit, inf);
    }
    double lo = -inf, hi = inf;
    switch (cmp) {
      case DFC_LT: hi = below; if (lit == -inf) { lo = 1; hi = 0; } break;
      case DFC_LE: hi = lit; break;
      case DFC_GT: lo = above; if (lit == inf) { lo = 1; hi = 0; } break;
      case DFC_GE: lo = lit; break;
      default: lo = hi = lit; break;  // EQ, NE (a NaN literal matches nothing)
    }
    sp.fast_lo.f = lo;
    sp.fast_hi.f = hi;
  } else if (dt == DFC_UINT64) {
    sp.fast_kind = FAST_UNSIGNED;
    const uint64_t lit = op.lit.u;
    uint64_t lo = 0, hi = UINT64_MAX;
    switch (cmp) {
      case DFC_LT: if (lit == 0) { lo = 1; hi = 0; } else hi = lit - 1; break;
      case DFC_LE: hi = lit; break;
      case DFC_GT: if (lit == UINT64_MAX) { lo = 1; hi = 0; } else lo = lit + 1; break;
      case DFC_GE: lo = lit; break;
      default: lo = hi = lit; break;
    }
    sp.fast_lo.u = lo;
    sp.fast_hi.u = hi;
  } else {
    const int64_t lit = op.lit.i;
    int64_t lo = INT64_MIN, hi = INT64_MAX;
    bool empty = false;
    switch (cmp) {
      case DFC_LT: if (lit == INT64_MIN) empty = true; else hi = lit - 1; break;
      case DFC_LE: hi = lit; break;
      case DFC_GT: if (lit == INT64_MAX) empty = true; else lo = lit + 1; break;
      case DFC_GE: lo = lit; break;
      default: lo = hi = lit; break;
    }
    if (is_unsigned(dt)) {
      // Zero-extended values up to 32 bits: the range clipped to x >= 0.
      sp.fast_kind = FAST_UNSIGNED;
      if (empty || hi < 0) {
        sp.fast_lo.u = 1;
        sp.fast_hi.u = 0;
      } else {
        sp.fast_lo.u = (uint64_t)std::max<int64_t>(lo, 0);
        sp.fast_hi.u = (uint64_t)hi;
      }
    } else {
      sp.fast_kind = FAST_SIGNED;
      sp.fast_lo.i = empty ? 1 : lo;
      sp.fast_hi.i = empty ? 0 : hi;
    }
  }
  sp.fast_rows = 1;
  return true;
}

// The automatic choice of the radix-partitioned regime: the estimated
// groups' records take more than kPartitionRecordBytes (half the L2) and
// the sampled hottest key holds under kPartitionTop1 of the rows.
// DFC_PARTITION_MIN_GROUPS=<n> replaces the record test by est >= n (tuning).
constexpr double kPartitionRecordBytes = 64.0 * 1024 * 1024;
constexpr double kPartitionTop1 = 0.01;
bool partition_by_default(const Plan& P, uint64_t est) {
  if (P.sp.key_mode != KEY_PACKED || P.top1 < 0 || P.top1 >= kPartitionTop1) return false;
  if (const char* env = getenv("DFC_PARTITION_MIN_GROUPS"))
    if (atoll(env) > 0) return est >= (uint64_t)atoll(env);
  return (double)est * P.sp.rec_stride > kPartitionRecordBytes;
}

// One attempt of the query at the given capacities: the global or
// shared-memory regime (`pp` null; `slots` key-table entries) or the
// radix-partitioned regime (`pp`).  *grow: a capacity ran out; the caller
// regrows it (host_ctl->status[1] says which in the partitioned regime) and
// retries.
dfc_status run_attempt(const dfc_query* q, Plan& P, DeviceState* ds, cudaStream_t stream, uint64_t slots,
                       uint64_t factor, const PartPlan* pp, dfc_result** out, bool* grow, Control* host_ctl) {
  *grow = false;
  ScanParams& sp = P.sp;
  FinishParams& fp = P.fp;
  Scratch S;
  S.stream = stream;

  const uint64_t ncta = pp ? pp->ctas : scan_grid(P, ds);
  uint64_t chunk = 64, recs;
  if (pp) {
    // Pass B appends every group once, in chunks of kRecChunk per CTA.
    recs = std::max<uint64_t>(1, pp->recs);
  } else {
    // Records: the groups the table may hold (load factor <= 1/table_factor:
    // the lock-step probe rounds run as long as a warp's longest chain) plus
    // every CTA's partly used last chunk.
    const uint64_t groups_cap = std::min<uint64_t>(P.rows, slots / factor);
    while (chunk < 1024 && chunk * ncta * 8 < groups_cap) chunk <<= 1;
    // Slack for holes: records reserved by claims that lost a race.
    recs = groups_cap + groups_cap / 8 + chunk * ncta;
  }
  if (recs >= 0xFFFFFFE0ull) return fail(DFC_CAPACITY, "group capacity exceeds 2^32 - 32 records");

  void *table = nullptr, *records, *ctl, *bits, *prefix, *bsums, *perm, *firsts;
  void *part_buf = nullptr, *part_totals = nullptr, *part_start = nullptr, *part_cursor = nullptr, *part_order = nullptr,
       *part_range = nullptr;
  const uint64_t words = (P.rows + 31) / 32;
  const uint64_t chunks = std::max<uint64_t>(1, (words + kFinishChunk - 1) / kFinishChunk);
  const uint64_t nparts = pp ? (1ull << pp->bits) : 0;
  dfc_status st;
  if (pp) {
    // Every row may pass the filter: part_buf holds all of them.
    if ((st = S.alloc(&part_buf, P.rows * pp->words * 8, "partition rows"))) return S.release(), st;
    if ((st = S.alloc(&part_totals, nparts * 4, "partition totals"))) return S.release(), st;
    if ((st = S.alloc(&part_start, nparts * 4, "partition starts"))) return S.release(), st;
    if ((st = S.alloc(&part_range, nparts * 8, "partition ranges"))) return S.release(), st;
    if ((st = S.alloc(&part_cursor, nparts * 4, "partition cursors"))) return S.release(), st;
    if ((st = S.alloc(&part_order, nparts * 4, "partition order"))) return S.release(), st;
  } else {
    if ((st = S.alloc(&table, (slots + 1) * sizeof(KeyEntry), "key table"))) return S.release(), st;
  }
  if ((st = S.alloc(&records, recs * sp.rec_stride, "group records"))) return S.release(), st;
  if ((st = S.alloc(&ctl, sizeof(Control), "control block"))) return S.release(), st;
  if ((st = S.alloc(&bits, words * 4 + 16, "order bitmap"))) return S.release(), st;
  if ((st = S.alloc(&prefix, words * 4 + 16, "order prefix"))) return S.release(), st;
  if ((st = S.alloc(&bsums, chunks * 4, "prefix chunks"))) return S.release(), st;
  if ((st = S.alloc(&perm, recs * 4, "group permutation"))) return S.release(), st;
  if ((st = S.alloc(&firsts, recs * 4, "first rows"))) return S.release(), st;
  // Output columns sized for the group capacity (the group count is known
  // only on the device; the host reads it once, at the end).
  // Ungrouped reductions always give one row.
  const uint64_t out_rows = std::max<uint64_t>(P.sp.n_keys == 0 ? 1 : 0, std::min<uint64_t>(P.rows, recs));
  // The device's memory limit (DATAFRAME_ACCEL_MEMORY_LIMIT through
  // dfc_set_memory_limit): rejected before the query's kernels are submitted.
  if (const int64_t limit = g_memory_limit[P.device].load(); limit > 0) {
    uint64_t need = S.total;
    for (int c = 0; c < P.n_out; ++c) need += out_rows * dtype_size(P.out_dtype[c]) + ((out_rows + 31) / 32) * 4 + 512;
    if (need > (uint64_t)limit) {
      S.release();
      char msg[200];
      snprintf(msg, sizeof msg, "the query needs %llu bytes of device memory; the memory limit is %lld",
               (unsigned long long)need, (long long)limit);
      return fail(DFC_UNSUPPORTED, msg);
    }
  }
  if ((st = S.commit("query working memory"))) return S.release(), st;
  std::vector<ResultCol> rc;
  void* out_slab = nullptr;
  {
    const cudaError_t e = alloc_result_cols(P, out_rows, rc, &out_slab, stream);
    if (e != cudaSuccess) {
      S.release();
      return cuda_fail(e, "output columns");
    }
  }
  auto free_outputs = [&]() { release_result_cols(rc, out_slab, stream); };

  Control* dctl = static_cast<Control*>(ctl);
  cudaError_t e;
  if (pp) {
    // Pass B writes every record it hands out (holes included); the counting
    // pass and pass A add into zeroed counters.
    e = cudaMemsetAsync(part_totals, 0, nparts * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(part_cursor, 0, nparts * 4, stream);
  } else {
    e = cudaMemsetAsync(table, 0xFF, (slots + 1) * sizeof(KeyEntry), stream);
    // Group records start all-zero: every field's identity (dfc_internal.h).
    if (e == cudaSuccess) e = cudaMemsetAsync(records, 0, recs * sp.rec_stride, stream);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(ctl, 0, sizeof(Control), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(&dctl->overflow_agg, 0xFF, 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(bits, 0, words * 4 + 16, stream);
  if (e != cudaSuccess) {
    free_outputs();
    S.release();
    return cuda_fail(e, "scratch initialisation");
  }

  sp.table = static_cast<KeyEntry*>(table);
  sp.table_mask = pp ? 0 : slots - 1;
  sp.records = static_cast<unsigned char*>(records);
  sp.recs_total = (uint32_t)recs;
  sp.chunk = (uint32_t)chunk;
  sp.alloc = &dctl->alloc;
  sp.status = dctl->status;
  sp.part_bits = pp ? pp->bits : 0;
  if (pp) {
    sp.part_words = pp->words;
    sp.part_buf = static_cast<unsigned long long*>(part_buf);
    sp.part_totals = static_cast<uint32_t*>(part_totals);
    sp.part_start = static_cast<uint32_t*>(part_start);
    sp.part_range = static_cast<uint2*>(part_range);
    sp.part_cursor = static_cast<uint32_t*>(part_cursor);
    sp.part_order = static_cast<uint32_t*>(part_order);
    sp.agg_slots = pp->agg_slots;
    sp.part_next = &dctl->part_next;
    sp.part_kept = &dctl->part_kept;
  }

  cudaEvent_t* ev = attempt_events(P.device);
  cudaEventRecord(ev[0], stream);
  if (pp) {
    // The counting pass streams the key and filter columns through a deeper
    // ring of narrower stages (their bytes lead every stage).
    const bool quad = plan_quad(sp) && !getenv("DFC_NO_QUAD");
    ScanParams spc = sp;
    spc.stages = pp->count_stages;
    spc.stage_bytes = pp->count_stage_bytes;
    (quad ? partition_count_quad : partition_count)<<<(unsigned)ncta, kPartThreads, pp->count_smem, stream>>>(spc);
    cudaEventRecord(ev[4], stream);
    partition_offsets<<<1, 1024, 0, stream>>>(sp);
    cudaEventRecord(ev[5], stream);
    ScanParams spa = sp;
    spa.stages = pp->stages;
    (quad ? partition_kernel_quad : partition_kernel)<<<(unsigned)ncta, kPartThreads, pp->smem, stream>>>(spa);
    cudaEventRecord(ev[3], stream);
    partition_aggregate<<<(unsigned)std::min<uint64_t>(pp->agg_ctas, nparts), kAggThreads, pp->agg_smem, stream>>>(sp);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      free_outputs();
      S.release();
      return cuda_fail(e, "partition pass launch");
    }
    t_timings.launches += 4;
  } else {
    if (P.rows > 0) {
      e = launch_scan(sp, ncta, P.smem, stream);
      if (e != cudaSuccess) {
        free_outputs();
        S.release();
        return cuda_fail(e, "scan launch");
      }
      t_timings.launches += 1;
    }
    cudaEventRecord(ev[3], stream);
  }
  cudaEventRecord(ev[1], stream);

  fp.scan = sp;
  fp.order_bits = static_cast<uint32_t*>(bits);
  fp.word_prefix = static_cast<uint32_t*>(prefix);
  fp.block_sums = static_cast<uint32_t*>(bsums);
  fp.perm = static_cast<uint32_t*>(perm);
  fp.firsts = static_cast<uint32_t*>(firsts);
  fp.groups = &dctl->groups;
  fp.has_nulls = dctl->has_nulls;
  fp.overflow_agg = &dctl->overflow_agg;
  fp.words = words;
  for (int c = 0; c < P.n_out; ++c) {
    fp.out[c].values = rc[c].values;
    fp.out[c].validity = rc[c].validity;
  }
  const unsigned rec_blocks = (unsigned)std::min<uint64_t>((recs + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
  finish_mark<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
  finish_chunk_sums<<<(unsigned)chunks, kFinishThreads, 0, stream>>>(fp);
  finish_scan_chunks<<<1, 1024, 0, stream>>>(fp, (uint32_t)chunks);
  finish_word_prefix<<<(unsigned)chunks, 1024, 0, stream>>>(fp);
  finish_rank<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
  const unsigned out_blocks = (unsigned)std::min<uint64_t>((out_rows + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
  finish_output<<<std::max(1u, out_blocks), kFinishThreads, finish_output_smem(fp.scan.rec_stride), stream>>>(fp);
  t_timings.launches += 6;
  cudaEventRecord(ev[2], stream);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_ctl, ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
  S.release();
  if (e != cudaSuccess) {
    free_outputs();
    return cuda_fail(e, "kernel launch");
  }
  st = wait_bounded(stream);
  if (st) {
    free_outputs();
    return st;
  }
  float ms_scan = 0, ms_agg = 0, ms_finish = 0, ms_count = 0, ms_offsets = 0;
  cudaEventElapsedTime(&ms_scan, ev[0], ev[3]);
  if (pp) {
    cudaEventElapsedTime(&ms_count, ev[0], ev[4]);
    cudaEventElapsedTime(&ms_offsets, ev[4], ev[5]);
  }
  cudaEventElapsedTime(&ms_agg, ev[3], ev[1]);
  cudaEventElapsedTime(&ms_finish, ev[1], ev[2]);
  t_timings.scan_ns += ms_scan * 1e6;
  t_timings.aggregate_ns += ms_agg * 1e6;
  t_timings.finish_ns += ms_finish * 1e6;
  t_timings.table_slots = pp ? (uint64_t)pp->agg_slots : slots;
  t_timings.partitions = pp ? (int32_t)nparts : 0;
  if (pp) {
    t_timings.count_ns += ms_count * 1e6;
    t_timings.place_ns += (ms_scan - ms_count - ms_offsets) * 1e6;
    t_timings.kept_rows = host_ctl->part_kept;
    t_timings.placed_row_bytes = 8u * pp->words;
  }
  if (getenv("DFC_TRACE")) {
    fprintf(stderr,
            "dfc attempt: rows=%llu regime=%s slots=%llu recs=%llu smem_slots=%u x%u tile=%d top1=%.4f hot=%.3f ctas=%llu "
            "parts=%llu agg_slots=%u agg_ctas=%llu stages=%d/%d | status=%#x cap=%#x check=%#x alloc=%u groups=%u ms "
            "scan=%.3f (count=%.3f offsets=%.3f) agg=%.3f fin=%.3f\n",
            (unsigned long long)P.rows, pp ? "partitioned" : "table", (unsigned long long)slots,
            (unsigned long long)recs, sp.smem_slots, std::max(1u, sp.smem_cluster), sp.tile_rows, P.top1, P.top_hot,
            (unsigned long long)ncta, (unsigned long long)nparts, pp ? pp->agg_slots : 0u,
            (unsigned long long)(pp ? pp->agg_ctas : 0), pp ? pp->count_stages : 0, pp ? pp->stages : 0,
            host_ctl->status[0], host_ctl->status[1], host_ctl->status[2], host_ctl->alloc, host_ctl->groups, ms_scan,
            ms_count, ms_offsets, ms_agg, ms_finish);
  }
  if (host_ctl->status[2] && !(host_ctl->status[0] & ST_TIMEOUT)) {
    free_outputs();
    char msg[128];
    snprintf(msg, sizeof msg, "an internal index or consistency check failed (code %#x)", host_ctl->status[2]);
    return fail(DFC_DEVICE, msg);
  }

  const uint32_t status = host_ctl->status[0];
  if (status & ST_TIMEOUT) {
    free_outputs();
    return fail(DFC_TIMEOUT, "a bounded device wait gave up");
  }
  if (status & (ST_CAPACITY | ST_F32_RANGE)) {
    // Out of capacity, or a compensated FP32 partial out of range (the caller
    // reruns in FP64).
    free_outputs();
    *grow = true;
    return DFC_CAPACITY;
  }
  if (status & ST_OVERFLOW) {
    free_outputs();
    const uint32_t a = host_ctl->overflow_agg;
    const int idt = (a < (uint32_t)q->n_aggs) ? P.out_agg_input_dtype[a] : DFC_INT64;
    return fail(DFC_DATA_OVERFLOW, overflow_message(idt));
  }
  if (status & ST_FAULT) {
    free_outputs();
    return fail(DFC_DATA_FAULT,
                "Mojo GPU data fault: variance of a group whose mean is far from its spread; the CPU adjudicates");
  }
  if (status & ST_ZERO_FAULT) {
    free_outputs();
    return fail(DFC_DATA_FAULT, "Mojo GPU data fault: mixed signed-zero extrema; the CPU adjudicates");
  }
  auto* r = new dfc_result();
  r->device = P.device;
  r->rows = host_ctl->groups;
  for (int c = 0; c < P.n_out; ++c) rc[c].has_nulls = host_ctl->has_nulls[c] != 0;
  r->cols = std::move(rc);
  r->slab = out_slab;
  *out = r;
  return DFC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI.
// ---------------------------------------------------------------------------
extern "C" {

DFC_API uint32_t dfc_version(void) { return DFC_ABI_VERSION; }

DFC_API int32_t dfc_installed(void) {
  // No driver call: the library exists (it was loaded) and a device node is present.
  return access("/dev/nvidiactl", F_OK) == 0 ? 1 : 0;
}

DFC_API int32_t dfc_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int usable = 0;
  for (int i = 0; i < n; ++i) {
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, i);
    if (major >= 10) ++usable;
  }
  return usable;
}

DFC_API dfc_status dfc_device_info_get(int32_t ordinal, dfc_device_info* out) {
  if (!out) return fail(DFC_INVALID, "null output");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || ordinal < 0 || ordinal >= n) {
    cudaGetLastError();
    return fail(DFC_NO_DEVICE, "no such device");
  }
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, ordinal), "cudaGetDeviceProperties");
  memset(out, 0, sizeof(*out));
  out->ordinal = ordinal;
  out->sm_count = prop.multiProcessorCount;
  out->cc_major = prop.major;
  out->cc_minor = prop.minor;
  out->total_bytes = prop.totalGlobalMem;
  out->budget_bytes = -1;
  if (ordinal < 64 && g_memory_limit[ordinal].load() > 0) out->budget_bytes = g_memory_limit[ordinal].load();
  const char* lim = out->budget_bytes > 0 ? nullptr : getenv("DATAFRAME_ACCEL_MEMORY_LIMIT");
  if (lim && *lim) {
    char* end = nullptr;
    long long v = strtoll(lim, &end, 10);
    if (end && *end == 0 && v > 0) out->budget_bytes = v;
  }
  snprintf(out->name, sizeof(out->name), "%s", prop.name);
  return DFC_OK;
}

DFC_API dfc_status dfc_measure_transfer(int32_t device, uint64_t bytes, dfc_byte_cost* to_device,
                                        dfc_byte_cost* to_host) {
  if (!to_device || !to_host) return fail(DFC_INVALID, "null output");
  const uint64_t small = 4096;
  if (bytes < 2 * small) return fail(DFC_INVALID, "measure at least 8 KiB");
  DeviceState* ds;
  dfc_status st = device_ready(device, &ds);
  if (st) return st;
  DeviceGuard guard(device);
  cudaStream_t stream = thread_stream(device);
  void* host = nullptr;
  void* dev = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto done = [&](dfc_status s) {
    if (dev) cudaFreeAsync(dev, stream);
    cudaStreamSynchronize(stream);
    if (host) cudaFreeHost(host);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return s;
  };
  cudaError_t e = cudaHostAlloc(&host, bytes, cudaHostAllocDefault);
  if (e == cudaSuccess) e = pool_alloc(&dev, bytes, stream);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) return done(cuda_fail(e, "transfer buffers"));
  memset(host, 0, bytes);
  // The best of three timed copies (after one untimed) of n bytes.
  auto best_ms = [&](uint64_t n, bool h2d, float& out) -> cudaError_t {
    out = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaError_t r = cudaEventRecord(e0, stream);
      if (r == cudaSuccess)
        r = h2d ? cudaMemcpyAsync(dev, host, n, cudaMemcpyHostToDevice, stream)
                : cudaMemcpyAsync(host, dev, n, cudaMemcpyDeviceToHost, stream);
      if (r == cudaSuccess) r = cudaEventRecord(e1, stream);
      if (r == cudaSuccess) r = cudaEventSynchronize(e1);
      float ms = 0;
      if (r == cudaSuccess) r = cudaEventElapsedTime(&ms, e0, e1);
      if (r != cudaSuccess) return r;
      if (rep > 0) out = std::min(out, ms);
    }
    return cudaSuccess;
  };
  for (int dir = 0; dir < 2; ++dir) {
    float t_small = 0, t_large = 0;
    e = best_ms(small, dir == 0, t_small);
    if (e == cudaSuccess) e = best_ms(bytes, dir == 0, t_large);
    if (e != cudaSuccess) return done(cuda_fail(e, "transfer measurement"));
    dfc_byte_cost& c = dir == 0 ? *to_device : *to_host;
    c.ns_per_byte = std::max(0.0, ((double)t_large - (double)t_small) * 1e6 / (double)(bytes - small));
    c.fixed_ns = std::max(0.0, (double)t_small * 1e6 - c.ns_per_byte * (double)small);
  }
  return done(DFC_OK);
}

DFC_API dfc_status dfc_set_memory_limit(int32_t device, int64_t bytes) {
  if (device < 0 || device >= 64) return fail(DFC_INVALID, "device ordinal out of range");
  g_memory_limit[device].store(bytes > 0 ? bytes : 0);
  return DFC_OK;
}

// Whether `p` is device memory of `device` (not host, managed or another
// GPU's memory): the kernels stream borrowed columns with bulk copies, which
// must read this GPU's own memory.
bool device_memory_of(const void* p, int device) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

DFC_API dfc_status dfc_column_register(int32_t device, dfc_dtype dtype, uint64_t rows, const void* values,
                                       const uint8_t* validity, uint64_t validity_bit_offset, uint32_t flags,
                                       dfc_column** out) {
  if (!out) return fail(DFC_INVALID, "null output");
  *out = nullptr;
  const int sz = dtype_size(dtype);
  if (sz == 0) return fail(DFC_UNSUPPORTED, "unsupported column type");
  if (rows > 0 && !values) return fail(DFC_INVALID, "null values");
  if (flags != DFC_COLUMN_HOST && flags != DFC_COLUMN_DEVICE) return fail(DFC_INVALID, "bad column flags");
  DeviceState* ds;
  dfc_status st = device_ready(device, &ds);
  if (st) return st;
  if (flags == DFC_COLUMN_DEVICE && rows > 0 && (!device_memory_of(values, device) || !device_memory_of(validity, device)))
    return fail(DFC_INVALID, "DFC_COLUMN_DEVICE values and validity must be device memory of the column's device "
                             "(host, managed or another GPU's memory is not accepted)");
  DeviceGuard guard(device);
  if (flags == DFC_COLUMN_DEVICE && rows > 0) {
    // A borrowed column may have been written on any stream of the device,
    // none of which orders before this thread's non-blocking stream (the
    // validity bitmap is read here, the values by later queries): wait for
    // the device's queued work first.
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "device column producer");
  }
  cudaStream_t stream = thread_stream(device);
  auto* c = new dfc_column();
  c->serial = ++g_column_serial;
  c->device = device;
  c->dtype = dtype;
  c->rows = rows;
  const size_t bytes = (size_t)rows * sz;
  auto bail = [&](dfc_status s) {
    if (c->owns_values && c->values) cudaFreeAsync(c->values, stream);
    if (c->validity) cudaFreeAsync(c->validity, stream);
    cudaStreamSynchronize(stream);
    delete c;
    return s;
  };
  if (flags == DFC_COLUMN_HOST) {
    cudaError_t e = pool_alloc(&c->values, std::max<size_t>(256, (bytes + 255) & ~(size_t)255), stream);
    if (e != cudaSuccess) return bail(cuda_fail(e, "column values"));
    c->owns_values = true;
    if (bytes) {
      e = cudaMemcpyAsync(c->values, values, bytes, cudaMemcpyHostToDevice, stream);
      if (e != cudaSuccess) return bail(cuda_fail(e, "column upload"));
    }
  } else {
    c->values = const_cast<void*>(values);
  }
  if (validity && rows > 0) {
    const uint64_t nbytes = (validity_bit_offset + rows + 7) / 8;
    const uint64_t words = (rows + 31) / 32;
    cudaError_t e = pool_alloc((void**)&c->validity, ((words * 4 + 255) & ~(uint64_t)255), stream);
    if (e != cudaSuccess) return bail(cuda_fail(e, "validity bitmap"));
    const uint8_t* src = validity;
    void* staging = nullptr;
    unsigned long long* d_count = nullptr;
    e = pool_alloc((void**)&d_count, 8, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, 8, stream);
    if (e == cudaSuccess && flags == DFC_COLUMN_HOST) {
      e = pool_alloc(&staging, nbytes, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(staging, validity, nbytes, cudaMemcpyHostToDevice, stream);
      src = static_cast<const uint8_t*>(staging);
    }
    if (e == cudaSuccess) {
      unsigned blocks = (unsigned)std::min<uint64_t>((words + 255) / 256, (uint64_t)ds->sms * 8);
      normalize_validity<<<std::max(1u, blocks), 256, 0, stream>>>(src, nbytes, validity_bit_offset, rows, c->validity,
                                                                  d_count);
      e = cudaGetLastError();
    }
    unsigned long long valid_rows = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&valid_rows, d_count, 8, cudaMemcpyDeviceToHost, stream);
    if (staging) cudaFreeAsync(staging, stream);
    if (d_count) cudaFreeAsync(d_count, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return bail(cuda_fail(e, "validity normalisation"));
    c->null_count = rows - valid_rows;
    if (c->null_count == 0) {
      cudaFreeAsync(c->validity, stream);
      c->validity = nullptr;
    }
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return bail(cuda_fail(e, "column upload"));
  *out = c;
  return DFC_OK;
}

DFC_API dfc_status dfc_column_release(dfc_column* column) {
  if (!column) return DFC_OK;
  DeviceGuard guard(column->device);
  // Stream-ordered: queued work on this thread's stream that reads the column
  // finishes before the memory is reused.
  cudaStream_t stream = thread_stream(column->device);
  if (column->owns_values && column->values) cudaFreeAsync(column->values, stream);
  if (column->validity) cudaFreeAsync(column->validity, stream);
  delete column;
  return DFC_OK;
}

DFC_API uint64_t dfc_column_rows(const dfc_column* column) { return column ? column->rows : 0; }
DFC_API int32_t dfc_column_null_count(const dfc_column* column) {
  return column ? (int32_t)std::min<uint64_t>(column->null_count, INT32_MAX) : 0;
}

}  // extern "C"

namespace {

// One group-by through the planner (every aggregation but N_UNIQUE).
dfc_status groupby_one(const dfc_query* query, dfc_result** out) {
  if (!out) return fail(DFC_INVALID, "null output");
  *out = nullptr;
  t_timings = dfc_timings{};
  const auto t0 = std::chrono::steady_clock::now();
  Plan P;
  dfc_status st = plan_query(query, P);
  if (st) return st;
  DeviceState* ds;
  st = device_ready(P.device, &ds);
  if (st) return st;
  DeviceGuard guard(P.device);
  cudaStream_t stream = query->stream ? static_cast<cudaStream_t>(query->stream) : thread_stream(P.device);
  thread_local Control* host_ctl = nullptr;
  if (!host_ctl) CK(cudaMallocHost((void**)&host_ctl, sizeof(Control)), "pinned control block");
  const auto t_est = std::chrono::steady_clock::now();
  uint64_t est = estimate_groups(query, P, ds, stream);
  plan_direct(query, P, ds, stream);
  const auto t_skew = std::chrono::steady_clock::now();
  // Regime: per-CTA shared-memory tables when the estimated groups fit in
  // shared memory at load <= 1/2 (two CTAs per SM if possible, else one);
  // otherwise the global table alone.  Rows whose key finds no room in a CTA
  // table take the global path, so a low estimate costs speed, not results.
  P.sp.smem_slots = 0;
  // The radix-partitioned regime: on request, or when the estimated groups'
  // records outgrow the L2-sized budget (the global table's probes and
  // atomics would then miss L2) and no key is hot enough to leave one pass B
  // CTA with much more than its share of the rows.
  PartPlan pp;
  bool partitioned = false;
  const bool forced_off = (query->flags & (DFC_Q_FORCE_GLOBAL | DFC_Q_FORCE_SHARED)) != 0;
  if (P.sp.key_mode == KEY_PACKED && est > kOwnAlwaysGroups && !(query->flags & DFC_Q_FORCE_GLOBAL))
    measure_skew(P, ds, stream);
  if (!forced_off && ((query->flags & DFC_Q_FORCE_PARTITIONED) || partition_by_default(P, est)))
    partitioned = plan_partitions(P, ds, est, pp);
  if (!partitioned) plan_shared(P, ds, est, query->flags);
  const auto t_plan = std::chrono::steady_clock::now();
  if (getenv("DFC_TRACE")) {
    auto us = [](auto a, auto b) { return std::chrono::duration<double, std::micro>(b - a).count(); };
    fprintf(stderr, "dfc plan: est=%llu prepare_us=%.1f estimate_us=%.1f skew+regime_us=%.1f\n", (unsigned long long)est,
            us(t0, t_est), us(t_est, t_skew), us(t_skew, t_plan));
  }
  // The query keeps its table factor through regrowth.
  const uint64_t factor = table_factor_for(est);
  uint64_t slots = next_pow2(std::max<uint64_t>(1024, est * factor));
  const uint64_t max_slots = next_pow2(std::max<uint64_t>(1024, P.rows * factor));
  slots = std::min(slots, max_slots);
  for (int attempt = 0; attempt < 6; ++attempt) {
    bool grow = false;
    st = run_attempt(query, P, ds, stream, slots, factor, partitioned ? &pp : nullptr, out, &grow, host_ctl);
    if (st == DFC_OK && attempt == 0 && fault_is("capacity")) {
      // Injected: the first attempt reports a full table and is regrown.
      dfc_result_free(*out);
      *out = nullptr;
      host_ctl->status[0] = ST_CAPACITY;
      host_ctl->status[1] = partitioned ? CAP_AGG_TABLE : 0u;
      grow = true;
      st = DFC_CAPACITY;
    }
    if (!grow) break;
    t_timings.retries += 1;
    if (host_ctl->status[0] & ST_F32_RANGE) {
      // A compensated FP32 partial left the FP32 range: FP64 throughout.
      P.sp.comp_mask = 0;
      if (!(host_ctl->status[0] & ST_CAPACITY)) continue;
    }
    if (partitioned) {
      // A partition's groups did not fit its table (the estimate was low):
      // more partitions, sized from the column statistics, twice the last
      // estimate and twice the records already handed out.  Records ran out:
      // twice the records.  When the plan cannot grow, the global regime
      // takes the query.
      const uint32_t why = host_ctl->status[1];
      const PartPlan last = pp;
      if (why & CAP_AGG_TABLE) {
        const uint64_t stats = estimate_groups(query, P, ds, stream, false);
        est = std::min<uint64_t>(P.rows, std::max<uint64_t>({stats, est * 2, (uint64_t)host_ctl->alloc * 2}));
        if (last.bits < (uint32_t)kPartMaxBits && plan_partitions(P, ds, est, pp, last.bits + 1)) {
          pp.recs = std::max(pp.recs, last.recs);
          continue;
        }
      } else if (why & CAP_RECORDS) {
        pp.recs = std::min<uint64_t>(0xFFFFFFDFull, last.recs * 2);
        if (pp.recs > last.recs) continue;
      }
      partitioned = false;
      plan_shared(P, ds, est, query->flags);
      slots = std::min(next_pow2(std::max<uint64_t>(1024, est * factor)), max_slots);
      continue;
    }
    if (slots >= max_slots) return fail(DFC_CAPACITY, "group table could not grow further");
    slots = std::min(slots * 8, max_slots);
  }
  if (st == DFC_CAPACITY) return fail(DFC_CAPACITY, "group table capacity exhausted after regrowth");
  if (st) return st;
  if (fault_is("overflow")) {
    // Injected: the first integer sum reports the CPU's overflow error.
    for (int a = 0; a < query->n_aggs; ++a) {
      const int idt = P.out_agg_input_dtype[a];
      if (query->aggs[a].op == DFC_AGG_SUM && !is_float(idt)) {
        dfc_result_free(*out);
        *out = nullptr;
        return fail(DFC_DATA_OVERFLOW, overflow_message(idt));
      }
    }
  }
  learn_groups(P, (*out)->rows);
  t_timings.groups = (*out)->rows;
  t_timings.regime = partitioned ? 2 : (P.sp.smem_slots ? (P.sp.reduce ? 3 : 1) : 0);
  t_timings.cluster_ctas = P.sp.smem_slots ? (int32_t)std::max(1u, P.sp.smem_cluster) : 0;
  t_timings.compensated = P.sp.smem_slots ? (int32_t)P.sp.comp_mask : 0;
  t_timings.direct_slots = P.sp.smem_slots && P.sp.direct ? P.sp.smem_slots : 0;
  t_timings.total_ns = std::chrono::duration<double, std::nano>(std::chrono::steady_clock::now() - t0).count();
  return DFC_OK;
}

// A result column as a query input, read in place (result validity is
// already 32-bit words at bit offset 0, the normalised form).
dfc_column result_input(const dfc_result* r, int i) {
  dfc_column c;
  c.serial = ++g_column_serial;
  c.device = r->device;
  c.dtype = r->cols[i].dtype;
  c.rows = r->rows;
  c.values = r->cols[i].values;
  c.validity = r->cols[i].has_nulls ? r->cols[i].validity : nullptr;
  c.null_count = r->cols[i].has_nulls ? 1 : 0;
  return c;
}

// N_UNIQUE(v) by two device group-bys: the distinct (keys, v) tuples of the
// kept rows, then the rows of that result per key tuple (LEN).  Both run in
// first-appearance order: a group's first tuple comes at the group's first
// row, so the second result's rows line up with the main query's groups.
// The main query (maintain_order forced) gives the keys and every other
// aggregation; the result is assembled in the query's column order.
dfc_status groupby_with_n_unique(const dfc_query* q, dfc_result** out) {
  *out = nullptr;
  if (q->n_aggs < 0 || q->n_aggs > kMaxAggs || !q->aggs) return fail(DFC_INVALID, "bad aggregation list");
  std::vector<dfc_agg> main_aggs;
  std::vector<int> where(q->n_aggs), nu_cols;
  for (int a = 0; a < q->n_aggs; ++a) {
    if (q->aggs[a].op != DFC_AGG_N_UNIQUE) {
      where[a] = (int)main_aggs.size();
      main_aggs.push_back(q->aggs[a]);
      continue;
    }
    const int v = q->aggs[a].column;
    if (v < 0 || v >= q->n_inputs) return fail(DFC_INVALID, "aggregation column out of range");
    int slot = -1;
    for (size_t u = 0; u < nu_cols.size(); ++u)
      if (nu_cols[u] == v) slot = (int)u;
    if (slot < 0) {
      slot = (int)nu_cols.size();
      nu_cols.push_back(v);
    }
    where[a] = -1 - slot;
  }
  if (main_aggs.empty()) main_aggs.push_back(dfc_agg{DFC_AGG_LEN, q->n_keys > 0 ? q->keys[0] : 0, 0, 0});
  dfc_query q0 = *q;
  q0.flags |= DFC_Q_MAINTAIN_ORDER;
  q0.aggs = main_aggs.data();
  q0.n_aggs = (int32_t)main_aggs.size();
  dfc_result* r0 = nullptr;
  dfc_status st = groupby_one(&q0, &r0);
  if (st) return st;
  const dfc_timings main_timings = t_timings;
  int launches = t_timings.launches;
  std::vector<dfc_result*> counts(nu_cols.size(), nullptr);
  auto release = [&]() {
    dfc_result_free(r0);
    for (dfc_result* r : counts) dfc_result_free(r);
  };
  const uint32_t regime_flags = q->flags & (DFC_Q_FORCE_GLOBAL | DFC_Q_FORCE_SHARED | DFC_Q_FORCE_PARTITIONED);
  for (size_t u = 0; u < nu_cols.size(); ++u) {
    const int v = nu_cols[u];
    int keys1[kMaxKeys + 1];
    int n1 = 0, vpos = -1;
    for (int k = 0; k < q->n_keys; ++k) {
      keys1[n1++] = q->keys[k];
      if (q->keys[k] == v) vpos = k;
    }
    if (vpos < 0) {
      if (n1 >= kMaxKeys) {
        release();
        return fail(DFC_UNSUPPORTED, "n_unique of a non-key column with four keys");
      }
      vpos = n1;
      keys1[n1++] = v;
    }
    dfc_query q1 = *q;
    q1.flags = DFC_Q_MAINTAIN_ORDER | regime_flags;
    q1.keys = keys1;
    q1.n_keys = n1;
    q1.aggs = nullptr;
    q1.n_aggs = 0;
    dfc_result* r1 = nullptr;
    if ((st = groupby_one(&q1, &r1))) {
      release();
      return st;
    }
    launches += t_timings.launches;
    dfc_column c1[kMaxKeys + 1];
    dfc_column* p1[kMaxKeys + 1];
    int keys2[kMaxKeys];
    for (int i = 0; i < n1; ++i) {
      c1[i] = result_input(r1, i);
      p1[i] = &c1[i];
    }
    for (int k = 0; k < q->n_keys; ++k) keys2[k] = k;
    const dfc_agg len{DFC_AGG_LEN, vpos, 0, 0};
    dfc_query q2 = {};
    q2.abi_version = DFC_ABI_VERSION;
    q2.flags = DFC_Q_MAINTAIN_ORDER | regime_flags;
    q2.n_inputs = n1;
    q2.n_keys = q->n_keys;
    q2.inputs = p1;
    q2.keys = keys2;
    q2.n_aggs = 1;
    q2.aggs = &len;
    q2.stream = q->stream;
    st = groupby_one(&q2, &counts[u]);
    launches += t_timings.launches;
    dfc_result_free(r1);
    if (st) {
      release();
      return st;
    }
    if (counts[u]->rows != r0->rows) {
      release();
      return fail(DFC_DEVICE, "n_unique: the distinct-value counts do not line up with the groups");
    }
  }
  // The result: keys and aggregations in the query's order, each column
  // copied into one new allocation.
  auto* r = new dfc_result();
  r->device = r0->device;
  r->rows = r0->rows;
  DeviceGuard guard(r0->device);
  cudaStream_t stream = q->stream ? static_cast<cudaStream_t>(q->stream) : thread_stream(r0->device);
  std::vector<const ResultCol*> src;
  for (int k = 0; k < q->n_keys; ++k) src.push_back(&r0->cols[k]);
  for (int a = 0; a < q->n_aggs; ++a)
    src.push_back(where[a] >= 0 ? &r0->cols[q->n_keys + where[a]] : &counts[-1 - where[a]]->cols[q->n_keys]);
  auto piece = [](uint64_t bytes) { return (std::max<uint64_t>(bytes, 256) + 255) & ~(uint64_t)255; };
  const uint64_t rows = r->rows, vwords = (rows + 31) / 32;
  uint64_t total = 0;
  for (const ResultCol* c : src) total += piece(rows * dtype_size(c->dtype)) + piece(vwords * 4);
  cudaError_t e = pool_alloc(&r->slab, std::max<uint64_t>(total, 256), stream);
  unsigned char* at = static_cast<unsigned char*>(r->slab);
  for (const ResultCol* c : src) {
    if (e != cudaSuccess) break;
    ResultCol rc;
    rc.dtype = c->dtype;
    rc.has_nulls = c->has_nulls;
    rc.values = at;
    at += piece(rows * dtype_size(c->dtype));
    rc.validity = reinterpret_cast<uint32_t*>(at);
    at += piece(vwords * 4);
    if (rows) e = cudaMemcpyAsync(rc.values, c->values, rows * dtype_size(c->dtype), cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess && rows) e = cudaMemcpyAsync(rc.validity, c->validity, vwords * 4, cudaMemcpyDeviceToDevice, stream);
    r->cols.push_back(rc);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  release();
  if (e != cudaSuccess) {
    dfc_result_free(r);
    return cuda_fail(e, "n_unique result assembly");
  }
  t_timings = main_timings;
  t_timings.launches = launches;
  *out = r;
  return DFC_OK;
}

}  // namespace

extern "C" {

DFC_API dfc_status dfc_groupby(const dfc_query* query, dfc_result** out) {
  if (!out) return fail(DFC_INVALID, "null output");
  *out = nullptr;
  if (query && query->aggs)
    for (int a = 0; a < query->n_aggs && a < kMaxAggs; ++a)
      if (query->aggs[a].op == DFC_AGG_N_UNIQUE) return groupby_with_n_unique(query, out);
  return groupby_one(query, out);
}

DFC_API uint64_t dfc_result_rows(const dfc_result* result) { return result ? result->rows : 0; }
DFC_API int32_t dfc_result_columns(const dfc_result* result) { return result ? (int32_t)result->cols.size() : 0; }

DFC_API dfc_status dfc_result_column(const dfc_result* result, int32_t i, dfc_dtype* dtype, const void** device_values,
                                     const uint8_t** device_validity) {
  if (!result || i < 0 || i >= (int32_t)result->cols.size()) return fail(DFC_INVALID, "bad result column");
  const ResultCol& c = result->cols[i];
  if (dtype) *dtype = c.dtype;
  if (device_values) *device_values = c.values;
  if (device_validity) *device_validity = c.has_nulls ? reinterpret_cast<const uint8_t*>(c.validity) : nullptr;
  return DFC_OK;
}

DFC_API dfc_status dfc_result_copy_to_host(const dfc_result* result, int32_t i, void* values, uint8_t* validity) {
  if (!result || i < 0 || i >= (int32_t)result->cols.size()) return fail(DFC_INVALID, "bad result column");
  const ResultCol& c = result->cols[i];
  DeviceGuard guard(result->device);
  cudaStream_t stream = thread_stream(result->device);
  const size_t n = result->rows;
  if (values && n) CK(cudaMemcpyAsync(values, c.values, n * dtype_size(c.dtype), cudaMemcpyDeviceToHost, stream), "result copy");
  if (validity && n) {
    if (c.has_nulls) CK(cudaMemcpyAsync(validity, c.validity, (n + 7) / 8, cudaMemcpyDeviceToHost, stream), "result copy");
    else memset(validity, 0xFF, (n + 7) / 8);
  }
  CK(cudaStreamSynchronize(stream), "result copy");
  return DFC_OK;
}

DFC_API dfc_status dfc_result_copy_to_device(const dfc_result* result, int32_t i, void* values, uint8_t* validity) {
  if (!result || i < 0 || i >= (int32_t)result->cols.size()) return fail(DFC_INVALID, "bad result column");
  const ResultCol& c = result->cols[i];
  DeviceGuard guard(result->device);
  const size_t n = result->rows;
  if (n && (!device_memory_of(values, result->device) || !device_memory_of(validity, result->device)))
    return fail(DFC_INVALID, "result copy targets must be device memory of the result's device");
  cudaStream_t stream = thread_stream(result->device);
  if (values && n)
    CK(cudaMemcpyAsync(values, c.values, n * dtype_size(c.dtype), cudaMemcpyDeviceToDevice, stream), "result copy");
  if (validity && n) {
    if (c.has_nulls) CK(cudaMemcpyAsync(validity, c.validity, (n + 7) / 8, cudaMemcpyDeviceToDevice, stream), "result copy");
    else CK(cudaMemsetAsync(validity, 0xFF, (n + 7) / 8, stream), "result copy");
  }
  CK(cudaStreamSynchronize(stream), "result copy");
  return DFC_OK;
}

DFC_API void dfc_result_free(dfc_result* result) {
  if (!result) return;
  if (result->refs.fetch_sub(1) != 1) return;
  DeviceGuard guard(result->device);
  cudaStream_t stream = thread_stream(result->device);
  if (result->slab) {
    cudaFreeAsync(result->slab, stream);
  } else {
    for (auto& c : result->cols) {
      if (c.values) cudaFreeAsync(c.values, stream);
      if (c.validity) cudaFreeAsync(c.validity, stream);
    }
  }
  delete result;
}

struct Residence {
  dfc_result* result;
  int32_t column;
  bool validity;  // the column's LSB-first validity bitmap instead of its values
};

DFC_API void* dfc_result_residence(dfc_result* result, int32_t i) {
  if (!result || i < 0 || i >= (int32_t)result->cols.size()) return nullptr;
  result->refs.fetch_add(1);
  return new Residence{result, i, false};
}

DFC_API void* dfc_result_validity_residence(dfc_result* result, int32_t i) {
  if (!result || i < 0 || i >= (int32_t)result->cols.size() || !result->cols[i].has_nulls) return nullptr;
  result->refs.fetch_add(1);
  return new Residence{result, i, true};
}

DFC_API int32_t dfc_residence_to_host(void* ctx, void* host_dst, int64_t bytes) {
  auto* r = static_cast<Residence*>(ctx);
  if (!r || !host_dst || bytes < 0) return 1;
  const ResultCol& c = r->result->cols[r->column];
  const uint64_t rows = r->result->rows;
  const int64_t have = r->validity ? (int64_t)((rows + 7) / 8) : (int64_t)(rows * dtype_size(c.dtype));
  if (bytes > have) return 1;
  DeviceGuard guard(r->result->device);
  const void* src = r->validity ? static_cast<const void*>(c.validity) : c.values;
  if (bytes && cudaMemcpy(host_dst, src, (size_t)bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  return 0;
}

DFC_API void dfc_residence_release(void* ctx) {
  auto* r = static_cast<Residence*>(ctx);
  if (!r) return;
  dfc_result_free(r->result);
  delete r;
}

DFC_API dfc_status dfc_last_timings(dfc_timings* out) {
  if (!out) return fail(DFC_INVALID, "null output");
  *out = t_timings;
  return DFC_OK;
}

DFC_API dfc_status dfc_set_thread_stream(int32_t device, void* stream) {
  if (device < 0) return fail(DFC_INVALID, "bad device");
  if (stream) t_chosen[device] = static_cast<cudaStream_t>(stream);
  else t_chosen.erase(device);
  return DFC_OK;
}

DFC_API const char* dfc_last_error(void) { return t_error.c_str(); }

DFC_API const char* dfc_status_name(dfc_status status) {
  switch (status) {
    case DFC_OK: return "ok";
    case DFC_UNSUPPORTED: return "unsupported";
    case DFC_INVALID: return "invalid";
    case DFC_DATA_OVERFLOW: return "data overflow";
    case DFC_DATA_FAULT: return "data fault";
    case DFC_CAPACITY: return "capacity";
    case DFC_OOM: return "out of device memory";
    case DFC_TIMEOUT: return "timeout";
    case DFC_DEVICE: return "device error";
    case DFC_NO_DEVICE: return "no device";
  }
  return "unknown";
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dfc_groupby_noalloc: the query with all of its working memory in one fixed
// array, for callers that cannot allocate device memory.
// ---------------------------------------------------------------------------

// The array every GPU that loads this library holds until the process exits.
// In host code its name is only a stand-in for the symbol, not a device
// address: noalloc_scratch() asks the runtime for the address once per device.
static __device__ __align__(256) unsigned char dfc_noalloc_scratch[DFC_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_addr_mu;
unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {};
// One call at a time per device: the calls share the array.
std::mutex g_noalloc_run_mu[kNoAllocMaxDevices];

// Device address of the array on `dev`; `dev` must be the current device.
dfc_status noalloc_scratch(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_addr_mu);
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, dfc_noalloc_scratch), "cudaGetSymbolAddress of the fixed scratch array");
    g_noalloc_base[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_base[dev];
  return DFC_OK;
}

// Bounded wait for `stream` that creates nothing (no event).
dfc_status noalloc_wait(cudaStream_t stream) {
  const auto t0 = std::chrono::steady_clock::now();
  const double limit = wait_limit_seconds();
  for (int spins = 0;; ++spins) {
    const cudaError_t e = cudaStreamQuery(stream);
    if (e == cudaSuccess) return DFC_OK;
    if (e != cudaErrorNotReady) return cuda_fail(e, "query execution");
    if (spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(20));
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit)
      return fail(DFC_TIMEOUT, "device work did not finish within the wait limit");
  }
}

// Hands out 256-byte-aligned pieces of the array; `used` is the total asked
// for, which may exceed the array (checked before any piece is used).
struct Carve {
  unsigned char* base;
  size_t used = 0;
  void* take(size_t bytes) {
    void* p = base + used;
    used += (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
    return p;
  }
};

}  // namespace

extern "C" {

DFC_API dfc_status dfc_groupby_noalloc(const dfc_query* query, int32_t device, uint64_t rows,
                                       const dfc_device_column* columns, uint64_t capacity,
                                       dfc_device_output* outputs, uint64_t* groups) {
  if (!query || !columns || !outputs || !groups) return fail(DFC_INVALID, "null argument");
  *groups = 0;
  t_timings = dfc_timings{};
  if (device < 0 || device >= kNoAllocMaxDevices) return fail(DFC_INVALID, "device ordinal out of range");
  if (query->n_inputs < 1 || query->n_inputs > kMaxInputs)
    return fail(DFC_UNSUPPORTED, "between 1 and 16 input columns are supported");
  // Host-side descriptors over the caller's device memory (no copies).
  dfc_column cols[kMaxInputs];
  dfc_column* col_ptrs[kMaxInputs];
  for (int i = 0; i < query->n_inputs; ++i) {
    const dfc_device_column& d = columns[i];
    if (dtype_size(d.dtype) == 0) return fail(DFC_UNSUPPORTED, "unsupported column type");
    if (rows > 0 && !d.values) return fail(DFC_INVALID, "null values");
    if (((uintptr_t)d.values & 15u) != 0 || ((uintptr_t)d.validity & 15u) != 0)
      return fail(DFC_INVALID, "column values and validity must be 16-byte aligned");
    if (rows > 0 && (!device_memory_of(d.values, device) || !device_memory_of(d.validity, device)))
      return fail(DFC_INVALID, "column values and validity must be device memory of `device` "
                               "(host, managed or another GPU's memory is not accepted)");
    cols[i].device = device;
    cols[i].dtype = (dfc_dtype)d.dtype;
    cols[i].rows = rows;
    cols[i].values = const_cast<void*>(d.values);
    cols[i].validity = const_cast<uint32_t*>(d.validity);
    col_ptrs[i] = &cols[i];
  }
  dfc_query q = *query;
  q.inputs = col_ptrs;
  Plan P;
  dfc_status st = plan_query(&q, P);
  if (st) return st;
  for (int c = 0; c < P.n_out; ++c) {
    if (capacity > 0 && (!outputs[c].values || !outputs[c].validity)) return fail(DFC_INVALID, "null output buffer");
    if (capacity > 0 && (!device_memory_of(outputs[c].values, device) || !device_memory_of(outputs[c].validity, device)))
      return fail(DFC_INVALID, "output buffers must be device memory of `device`");
  }
  DeviceState* ds;
  if ((st = device_ready(P.device, &ds))) return st;
  DeviceGuard guard(P.device);
  std::lock_guard<std::mutex> run_lock(g_noalloc_run_mu[device]);
  unsigned char* base;
  if ((st = noalloc_scratch(P.device, &base))) return st;
  cudaStream_t stream = query->stream ? static_cast<cudaStream_t>(query->stream) : cudaStreamPerThread;
  ScanParams& sp = P.sp;
  FinishParams& fp = P.fp;

  // Regime and table size from the caller's capacity (no statistics pass,
  // so no skew sample): per-CTA shared-memory tables up to the group count
  // dfc_groupby takes them for whatever the skew (kOwnAlwaysGroups), up to
  // kOwnTableGroups for compensated FP32 fields (they need on-chip partials)
  // or on DFC_Q_FORCE_SHARED; the global table otherwise.  The
  // radix-partitioned regime is never used here (DFC_Q_FORCE_PARTITIONED is
  // ignored): its partition buffers would not fit the array.
  const uint64_t est = std::min<uint64_t>(capacity, P.rows);
  sp.smem_slots = 0;
  const bool own_tables = (query->flags & DFC_Q_FORCE_SHARED) || est <= kOwnAlwaysGroups ||
                          (sp.comp_mask != 0 && est <= kOwnTableGroups);
  if (!(query->flags & DFC_Q_FORCE_GLOBAL) && sp.key_mode == KEY_PACKED && own_tables) {
    const uint64_t sslots = next_pow2(std::max<uint64_t>(64, std::min<uint64_t>(est, 4096) * 2));
    const size_t keys_off = (P.smem + 15) & ~(size_t)15;
    const size_t recs_off = (keys_off + sslots * 8 + 15) & ~(size_t)15;
    const size_t total = recs_off + sslots * (size_t)sp.rec_stride;
    if (total <= ds->smem_optin) {
      sp.smem_slots = (uint32_t)sslots;
      sp.smem_keys_off = (uint32_t)keys_off;
      sp.smem_recs_off = (uint32_t)recs_off;
      P.smem = total;
    }
  }
  const uint64_t slots = std::min(next_pow2(std::max<uint64_t>(1024, est * 2)),
                                  next_pow2(std::max<uint64_t>(1024, P.rows * 2)));
  int occ = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, scan_fn(P.sp), kScanThreads, P.smem), "occupancy");
  occ = std::max(1, occ);
  uint64_t ncta = (uint64_t)ds->sms * (uint64_t)occ;
  ncta = std::max<uint64_t>(1, std::min<uint64_t>(ncta, std::max<uint64_t>(1, sp.tiles)));
  const uint64_t groups_cap = std::min<uint64_t>(P.rows, slots / 2);
  uint64_t chunk = 64;
  while (chunk < 1024 && chunk * ncta * 8 < groups_cap) chunk <<= 1;
  const uint64_t words = (P.rows + 31) / 32;
  const uint64_t chunks = std::max<uint64_t>(1, (words + kFinishChunk - 1) / kFinishChunk);
  // Every group holds a table entry, so the table bounds the group count.
  const uint64_t out_rows = std::max<uint64_t>(P.sp.n_keys == 0 ? 1 : 0, std::min<uint64_t>(P.rows, slots + 1));

  // Working memory, carved from the array: the fixed parts, then as many
  // group records as the rest holds.  Besides the groups, records go to
  // claims that lost a race (many with hot keys) and to partly used chunks;
  // a row reserves one record at most, so more than rows + chunks of slack
  // is never needed.  Outputs are staged here and copied out once the group
  // count is known to fit the caller's buffers.
  Carve cv{base};
  void* table = cv.take((slots + 1) * sizeof(KeyEntry));
  Control* dctl = static_cast<Control*>(cv.take(sizeof(Control)));
  void* bits = cv.take(words * 4 + 16);
  void* prefix = cv.take(words * 4 + 16);
  void* bsums = cv.take(chunks * 4);
  void* perm = cv.take(out_rows * 4);
  void* out_vals[kMaxOut];
  uint32_t* out_valid[kMaxOut];
  for (int c = 0; c < P.n_out; ++c) {
    out_vals[c] = cv.take(out_rows * 8);
    out_valid[c] = static_cast<uint32_t*>(cv.take(((out_rows + 31) / 32) * 4));
  }
  const uint64_t per_record = (uint64_t)sp.rec_stride + 4;  // record + its first row
  const uint64_t min_recs = groups_cap + groups_cap / 8 + chunk * ncta;
  const uint64_t left = cv.used + 512 < DFC_NOALLOC_SCRATCH_BYTES ? DFC_NOALLOC_SCRATCH_BYTES - cv.used - 512 : 0;
  const uint64_t useful = std::max<uint64_t>(min_recs, P.rows + chunk * ncta);
  const uint64_t recs = std::min<uint64_t>({useful, left / per_record, 0xFFFFFFDFull});
  if (recs < min_recs) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "dfc_groupby_noalloc: this query needs %llu bytes of working memory; the fixed scratch array holds %llu "
             "(fewer rows or a smaller capacity fit)",
             (unsigned long long)(cv.used + 512 + min_recs * per_record), (unsigned long long)DFC_NOALLOC_SCRATCH_BYTES);
    return fail(DFC_CAPACITY, msg);
  }
  void* records = cv.take(recs * sp.rec_stride);
  void* firsts = cv.take(recs * 4);

  // The array keeps the previous call's contents: clear what starts known.
  // A compensated FP32 partial that leaves the FP32 range (ST_F32_RANGE)
  // makes dfc_groupby rerun the query in FP64; here the rerun happens in the
  // same array, once, after the first attempt has finished on the GPU.
  Control hc;
  for (int attempt = 0;; ++attempt) {
    cudaError_t e = cudaMemsetAsync(table, 0xFF, (slots + 1) * sizeof(KeyEntry), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(records, 0, recs * sp.rec_stride, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dctl, 0, sizeof(Control), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&dctl->overflow_agg, 0xFF, 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(bits, 0, words * 4 + 16, stream);
    if (e != cudaSuccess) return cuda_fail(e, "scratch initialisation");

    sp.table = static_cast<KeyEntry*>(table);
    sp.table_mask = slots - 1;
    sp.records = static_cast<unsigned char*>(records);
    sp.recs_total = (uint32_t)recs;
    sp.chunk = (uint32_t)chunk;
    sp.alloc = &dctl->alloc;
    sp.status = dctl->status;
    if (P.rows > 0) {
      scan_fn(sp)<<<(unsigned)ncta, kScanThreads, P.smem, stream>>>(sp);
      t_timings.launches += 1;
    }
    fp.scan = sp;
    fp.order_bits = static_cast<uint32_t*>(bits);
    fp.word_prefix = static_cast<uint32_t*>(prefix);
    fp.block_sums = static_cast<uint32_t*>(bsums);
    fp.perm = static_cast<uint32_t*>(perm);
    fp.firsts = static_cast<uint32_t*>(firsts);
    fp.groups = &dctl->groups;
    fp.has_nulls = dctl->has_nulls;
    fp.overflow_agg = &dctl->overflow_agg;
    fp.words = words;
    for (int c = 0; c < P.n_out; ++c) {
      fp.out[c].values = out_vals[c];
      fp.out[c].validity = out_valid[c];
    }
    const unsigned rec_blocks =
        (unsigned)std::min<uint64_t>((recs + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
    finish_mark<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
    finish_chunk_sums<<<(unsigned)chunks, kFinishThreads, 0, stream>>>(fp);
    finish_scan_chunks<<<1, 1024, 0, stream>>>(fp, (uint32_t)chunks);
    finish_word_prefix<<<(unsigned)chunks, 1024, 0, stream>>>(fp);
    finish_rank<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
    const unsigned out_blocks =
        (unsigned)std::min<uint64_t>((out_rows + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
    finish_output<<<std::max(1u, out_blocks), kFinishThreads, finish_output_smem(fp.scan.rec_stride), stream>>>(fp);
    t_timings.launches += 6;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    if ((st = noalloc_wait(stream))) return st;
    CK(cudaMemcpyAsync(&hc, dctl, sizeof(Control), cudaMemcpyDeviceToHost, stream), "control block");
    if ((st = noalloc_wait(stream))) return st;
    if (attempt == 0 && (hc.status[0] & ST_F32_RANGE) && !(hc.status[0] & ST_TIMEOUT) && !hc.status[2]) {
      sp.comp_mask = 0;
      t_timings.retries += 1;
      continue;
    }
    break;
  }

  const uint32_t status = hc.status[0];
  if (hc.status[2]) {
    char msg[128];
    snprintf(msg, sizeof msg, "an internal index or consistency check failed (code %#x)", hc.status[2]);
    return fail(DFC_DEVICE, msg);
  }
  if (status & ST_TIMEOUT) return fail(DFC_TIMEOUT, "a bounded device wait gave up");
  if (status & ST_CAPACITY) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "dfc_groupby_noalloc: more groups than the table sized for this capacity holds "
             "(%u of %llu records handed out, %llu table slots)",
             hc.alloc, (unsigned long long)recs, (unsigned long long)slots);
    return fail(DFC_CAPACITY, msg);
  }
  if (status & ST_OVERFLOW) {
    const uint32_t a = hc.overflow_agg;
    const int idt = (a < (uint32_t)query->n_aggs) ? P.out_agg_input_dtype[a] : DFC_INT64;
    return fail(DFC_DATA_OVERFLOW, overflow_message(idt));
  }
  if (status & ST_FAULT)
    return fail(DFC_DATA_FAULT,
                "Mojo GPU data fault: variance of a group whose mean is far from its spread; the CPU adjudicates");
  if (status & ST_ZERO_FAULT)
    return fail(DFC_DATA_FAULT, "Mojo GPU data fault: mixed signed-zero extrema; the CPU adjudicates");
  const uint64_t G = hc.groups;
  if (G > capacity) {
    char msg[160];
    snprintf(msg, sizeof msg, "dfc_groupby_noalloc: the query has %llu groups; the outputs hold %llu",
             (unsigned long long)G, (unsigned long long)capacity);
    return fail(DFC_CAPACITY, msg);
  }
  for (int c = 0; c < P.n_out; ++c) {
    outputs[c].dtype = P.out_dtype[c];
    outputs[c].has_nulls = hc.has_nulls[c] != 0 ? 1 : 0;
    if (G == 0) continue;
    cudaError_t e = cudaMemcpyAsync(outputs[c].values, out_vals[c], G * dtype_size(P.out_dtype[c]), cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(outputs[c].validity, out_valid[c], ((G + 31) / 32) * 4, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "output copy");
  }
  if ((st = noalloc_wait(stream))) return st;
  *groups = G;
  t_timings.groups = G;
  t_timings.table_slots = slots;
  t_timings.regime = sp.smem_slots ? 1 : 0;
  t_timings.compensated = sp.smem_slots ? (int32_t)sp.comp_mask : 0;
  return DFC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dfc_groupby_batch: many queries in one submission.
// ---------------------------------------------------------------------------
namespace {

constexpr int kBatchStreams = 8;
constexpr int kFullGridAhead = 2;  // served form: full-grid requests in flight at most
thread_local std::vector<std::string> t_batch_errors;

// The batch's streams on `dev`, created once per thread.
const std::vector<cudaStream_t>& batch_streams(int dev) {
  thread_local std::map<int, std::vector<cudaStream_t>> streams;
  auto& v = streams[dev];
  if (v.empty()) {
    v.resize(kBatchStreams);
    for (auto& s : v) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  }
  return v;
}

// One query of a batch: its plan and where its working memory lies.
struct BatchItem {
  Plan P;
  dfc_status st = DFC_OK;
  uint64_t slots = 0, recs = 0, chunk = 64, ncta = 1, words = 0, chunks = 1, out_rows = 0;
  bool full_grid = false;  // the scan's grid fills every SM
  size_t off_table = 0, off_records = 0, off_bits = 0, off_prefix = 0, off_bsums = 0, off_perm = 0, off_firsts = 0;
  std::vector<ResultCol> rc;
  void* slab = nullptr;  // rc's buffers
};

// The stream of a sized query: a scan whose grid fills every SM runs on
// stream 0, one after another (two such scans side by side only interleave
// and share L2 between their tables); smaller queries spread over the rest.
int item_stream(const BatchItem& it, int& k) {
  if (it.full_grid) return 0;
  return 1 + (k++ % (kBatchStreams - 1));
}

size_t arena_take(size_t& used, size_t bytes) {
  const size_t at = used;
  used += (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255;
  return at;
}

// Regime and capacities of one planned query; its working memory is laid
// out from `used` on (256-byte aligned pieces).
dfc_status size_item(const dfc_query* q, BatchItem& it, DeviceState* ds, cudaStream_t stream, size_t& used) {
  Plan& P = it.P;
  const uint64_t est = estimate_groups(q, P, ds, stream);
  plan_direct(q, P, ds, stream);
  if (P.sp.key_mode == KEY_PACKED && est > kOwnAlwaysGroups && !(q->flags & DFC_Q_FORCE_GLOBAL))
    measure_skew(P, ds, stream);
  plan_shared(P, ds, est, q->flags);
  const uint64_t factor = table_factor_for(est);
  it.slots = std::min(next_pow2(std::max<uint64_t>(1024, est * factor)),
                      next_pow2(std::max<uint64_t>(1024, P.rows * factor)));
  it.ncta = scan_grid(P, ds);
  it.full_grid = it.ncta >= scan_capacity(P, ds);
  const uint64_t groups_cap = std::min<uint64_t>(P.rows, it.slots / factor);
  it.chunk = 64;
  while (it.chunk < 1024 && it.chunk * it.ncta * 8 < groups_cap) it.chunk <<= 1;
  it.recs = groups_cap + groups_cap / 8 + it.chunk * it.ncta;
  if (it.recs >= 0xFFFFFFE0ull) return fail(DFC_CAPACITY, "group capacity exceeds 2^32 - 32 records");
  it.words = (P.rows + 31) / 32;
  it.chunks = std::max<uint64_t>(1, (it.words + kFinishChunk - 1) / kFinishChunk);
  it.out_rows = std::max<uint64_t>(P.sp.n_keys == 0 ? 1 : 0, std::min<uint64_t>(P.rows, it.recs));
  it.off_table = arena_take(used, (it.slots + 1) * sizeof(KeyEntry));
  it.off_records = arena_take(used, it.recs * P.sp.rec_stride);
  it.off_bits = arena_take(used, it.words * 4 + 16);
  it.off_prefix = arena_take(used, it.words * 4 + 16);
  it.off_bsums = arena_take(used, it.chunks * 4);
  it.off_perm = arena_take(used, it.recs * 4);
  it.off_firsts = arena_take(used, it.recs * 4);
  return DFC_OK;
}

// Output columns of a sized query (one stream-ordered allocation).
dfc_status alloc_outputs(BatchItem& it, cudaStream_t stream) {
  if (alloc_result_cols(it.P, it.out_rows, it.rc, &it.slab, stream) != cudaSuccess)
    return fail(DFC_OOM, "output columns");
  return DFC_OK;
}

// The result of a finished query from its control block, or its error.
dfc_status finish_item(const dfc_query* q, BatchItem& it, const Control& c, int device, dfc_result** out) {
  const uint32_t status = c.status[0];
  if (c.status[2] && !(status & ST_TIMEOUT)) {
    char msg[128];
    snprintf(msg, sizeof msg, "an internal index or consistency check failed (code %#x)", c.status[2]);
    return fail(DFC_DEVICE, msg);
  }
  if (status & ST_TIMEOUT) return fail(DFC_TIMEOUT, "a bounded device wait gave up");
  if (status & (ST_CAPACITY | ST_F32_RANGE)) return DFC_CAPACITY;  // rerun alone
  if (status & ST_OVERFLOW) {
    const uint32_t a = c.overflow_agg;
    const int idt = (a < (uint32_t)q->n_aggs) ? it.P.out_agg_input_dtype[a] : DFC_INT64;
    return fail(DFC_DATA_OVERFLOW, overflow_message(idt));
  }
  if (status & ST_FAULT)
    return fail(DFC_DATA_FAULT, "Mojo GPU data fault: variance of a group whose mean is far from its spread; the CPU adjudicates");
  if (status & ST_ZERO_FAULT)
    return fail(DFC_DATA_FAULT, "Mojo GPU data fault: mixed signed-zero extrema; the CPU adjudicates");
  auto* r = new dfc_result();
  r->device = device;
  r->rows = c.groups;
  for (int col = 0; col < it.P.n_out; ++col) it.rc[col].has_nulls = c.has_nulls[col] != 0;
  r->cols = std::move(it.rc);
  r->slab = it.slab;
  it.slab = nullptr;
  *out = r;
  learn_groups(it.P, c.groups);
  return DFC_OK;
}

// The launches of one planned query (global or shared-memory regime) on
// `stream`, working memory at `base`, control block `dctl`.
void launch_item(BatchItem& it, DeviceState* ds, unsigned char* base, Control* dctl, cudaStream_t stream) {
  ScanParams& sp = it.P.sp;
  FinishParams& fp = it.P.fp;
  void* table = base + it.off_table;
  void* records = base + it.off_records;
  cudaMemsetAsync(table, 0xFF, (it.slots + 1) * sizeof(KeyEntry), stream);
  cudaMemsetAsync(records, 0, it.recs * sp.rec_stride, stream);
  cudaMemsetAsync(dctl, 0, sizeof(Control), stream);
  cudaMemsetAsync(&dctl->overflow_agg, 0xFF, 4, stream);
  cudaMemsetAsync(base + it.off_bits, 0, it.words * 4 + 16, stream);
  sp.table = static_cast<KeyEntry*>(table);
  sp.table_mask = it.slots - 1;
  sp.records = static_cast<unsigned char*>(records);
  sp.recs_total = (uint32_t)it.recs;
  sp.chunk = (uint32_t)it.chunk;
  sp.alloc = &dctl->alloc;
  sp.status = dctl->status;
  sp.part_bits = 0;
  if (it.P.rows > 0) launch_scan(sp, it.ncta, it.P.smem, stream);
  fp.scan = sp;
  fp.order_bits = reinterpret_cast<uint32_t*>(base + it.off_bits);
  fp.word_prefix = reinterpret_cast<uint32_t*>(base + it.off_prefix);
  fp.block_sums = reinterpret_cast<uint32_t*>(base + it.off_bsums);
  fp.perm = reinterpret_cast<uint32_t*>(base + it.off_perm);
  fp.firsts = reinterpret_cast<uint32_t*>(base + it.off_firsts);
  fp.groups = &dctl->groups;
  fp.has_nulls = dctl->has_nulls;
  fp.overflow_agg = &dctl->overflow_agg;
  fp.words = it.words;
  for (int c = 0; c < it.P.n_out; ++c) {
    fp.out[c].values = it.rc[c].values;
    fp.out[c].validity = it.rc[c].validity;
  }
  const unsigned rec_blocks = (unsigned)std::min<uint64_t>((it.recs + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
  finish_mark<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
  finish_chunk_sums<<<(unsigned)it.chunks, kFinishThreads, 0, stream>>>(fp);
  finish_scan_chunks<<<1, 1024, 0, stream>>>(fp, (uint32_t)it.chunks);
  finish_word_prefix<<<(unsigned)it.chunks, 1024, 0, stream>>>(fp);
  finish_rank<<<std::max(1u, rec_blocks), kFinishThreads, 0, stream>>>(fp);
  const unsigned out_blocks = (unsigned)std::min<uint64_t>((it.out_rows + kFinishThreads - 1) / kFinishThreads, (uint64_t)ds->sms * 16);
  finish_output<<<std::max(1u, out_blocks), kFinishThreads, finish_output_smem(fp.scan.rec_stride), stream>>>(fp);
}

}  // namespace

extern "C" {

DFC_API const char* dfc_batch_error(int32_t i) {
  if (i < 0 || (size_t)i >= t_batch_errors.size()) return "";
  return t_batch_errors[i].c_str();
}

DFC_API dfc_status dfc_groupby_batch(const dfc_query* const* queries, int32_t n, dfc_result** results,
                                     dfc_status* statuses) {
  if (n < 0 || (n > 0 && (!queries || !results || !statuses))) return fail(DFC_INVALID, "null argument");
  t_batch_errors.assign((size_t)n, std::string());
  const auto t0 = std::chrono::steady_clock::now();
  dfc_timings bt{};
  for (int i = 0; i < n; ++i) {
    results[i] = nullptr;
    statuses[i] = DFC_OK;
  }
  if (n == 0) return DFC_OK;
  std::vector<BatchItem> items((size_t)n);
  auto reject = [&](int i, dfc_status st) {
    items[i].st = st;
    statuses[i] = st;
    t_batch_errors[i] = t_error;
  };
  int device = -1;
  DeviceState* ds = nullptr;
  for (int i = 0; i < n; ++i) {
    dfc_status st = plan_query(queries[i], items[i].P);
    if (st) {
      reject(i, st);
      continue;
    }
    if (device < 0) {
      device = items[i].P.device;
      if ((st = device_ready(device, &ds))) return st;
    } else if (items[i].P.device != device) {
      fail(DFC_UNSUPPORTED, "a batch runs on one device");
      reject(i, DFC_UNSUPPORTED);
    }
  }
  if (device < 0) return DFC_OK;  // nothing to run
  DeviceGuard guard(device);
  cudaStream_t main = thread_stream(device);
  const auto& streams = batch_streams(device);

  // Plans: regime and capacities per query, working memory in one arena.
  const auto t_plan = std::chrono::steady_clock::now();
  size_t used = 0;
  for (int i = 0; i < n; ++i) {
    BatchItem& it = items[i];
    if (it.st) continue;
    const dfc_status st = size_item(queries[i], it, ds, main, used);
    if (st) reject(i, st);
  }
  const auto t_alloc = std::chrono::steady_clock::now();
  unsigned char* arena = nullptr;
  Control* dctl = nullptr;
  cudaError_t e = pool_alloc((void**)&arena, std::max<size_t>(used, 256), main);
  if (e == cudaSuccess) e = pool_alloc((void**)&dctl, (size_t)n * sizeof(Control), main);
  if (e != cudaSuccess) {
    if (arena) cudaFreeAsync(arena, main);
    return cuda_fail(e, "batch working memory");
  }
  auto free_outputs = [&](BatchItem& it) { release_result_cols(it.rc, it.slab, main); };
  for (int i = 0; i < n; ++i) {
    BatchItem& it = items[i];
    if (it.st) continue;
    if (alloc_outputs(it, main)) {
      free_outputs(it);
      reject(i, DFC_OOM);
    }
  }

  // Launch: queries round-robin over the batch streams, forked from and
  // joined back to the thread's stream; no synchronisation in between.
  cudaEvent_t fork;
  cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  cudaEventRecord(fork, main);
  std::vector<cudaEvent_t> joins(streams.size());
  for (size_t s = 0; s < streams.size(); ++s) {
    cudaStreamWaitEvent(streams[s], fork, 0);
    cudaEventCreateWithFlags(&joins[s], cudaEventDisableTiming);
  }
  const auto t_launch = std::chrono::steady_clock::now();
  // Two phases: the smaller queries side by side on streams 1-7, then the
  // full-grid ones one after another on stream 0.  A persistent scan sized to
  // every SM runs late on the SMs other kernels still hold, so it never runs
  // beside the small ones.
  int k = 0;
  for (int phase = 0; phase < 2; ++phase) {
    for (int i = 0; i < n; ++i) {
      if (items[i].st || items[i].full_grid != (phase == 1)) continue;
      launch_item(items[i], ds, arena, dctl + i, streams[item_stream(items[i], k)]);
      bt.launches += items[i].P.rows > 0 ? 7 : 6;
    }
    if (phase == 0)
      for (size_t s = 1; s < streams.size(); ++s) {
        cudaEventRecord(joins[s], streams[s]);
        cudaStreamWaitEvent(streams[0], joins[s], 0);
      }
  }
  for (size_t s = 0; s < streams.size(); ++s) {
    cudaEventRecord(joins[s], streams[s]);
    cudaStreamWaitEvent(main, joins[s], 0);
  }
  thread_local std::vector<Control> hctl;
  thread_local Control* pinned = nullptr;
  thread_local size_t pinned_n = 0;
  if (pinned_n < (size_t)n) {
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    if (cudaMallocHost((void**)&pinned, (size_t)n * sizeof(Control)) != cudaSuccess) pinned = nullptr;
    pinned_n = pinned ? (size_t)n : 0;
  }
  e = cudaGetLastError();
  if (e == cudaSuccess && pinned) e = cudaMemcpyAsync(pinned, dctl, (size_t)n * sizeof(Control), cudaMemcpyDeviceToHost, main);
  const auto t_wait = std::chrono::steady_clock::now();
  dfc_status st = e == cudaSuccess ? wait_bounded(main) : cuda_fail(e, "batch launch");
  const auto t_done = std::chrono::steady_clock::now();
  if (st == DFC_OK && !pinned) st = fail(DFC_OOM, "pinned batch control blocks");
  cudaEventDestroy(fork);
  for (auto& j : joins) cudaEventDestroy(j);
  cudaFreeAsync(arena, main);
  cudaFreeAsync(dctl, main);
  if (st) {
    for (auto& it : items) free_outputs(it);
    return st;
  }

  // Results; a query that ran out of capacity reruns alone with regrowth.
  for (int i = 0; i < n; ++i) {
    BatchItem& it = items[i];
    if (it.st) continue;
    const Control& c = pinned[i];
    dfc_status qs = finish_item(queries[i], it, c, device, &results[i]);
    if (qs == DFC_CAPACITY) {
      // Ran out of capacity: alone, with regrowth.
      free_outputs(it);
      const dfc_timings keep = bt;
      qs = dfc_groupby(queries[i], &results[i]);
      bt = keep;
      bt.retries += 1;
    } else if (qs == DFC_OK) {
      bt.groups += c.groups;
    } else {
      free_outputs(it);
    }
    statuses[i] = qs;
    if (qs) t_batch_errors[i] = t_error;
  }
  bt.total_ns = std::chrono::duration<double, std::nano>(std::chrono::steady_clock::now() - t0).count();
  if (getenv("DFC_TRACE")) {
    auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    fprintf(stderr, "dfc batch: n=%d arena=%zu MB plan=%.2f alloc=%.2f launch=%.2f wait=%.2f results=%.2f ms retries=%d\n",
            n, used >> 20, ms(t_plan, t_alloc), ms(t_alloc, t_launch), ms(t_launch, t_wait), ms(t_wait, t_done),
            ms(t_done, std::chrono::steady_clock::now()), bt.retries);
  }
  t_timings = bt;
  return DFC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The served form: a request loop with continuous batching.
// ---------------------------------------------------------------------------
namespace {

// A query description the server owns (dfc_query holds borrowed pointers).
struct OwnedQuery {
  dfc_query q{};
  std::vector<dfc_column*> inputs;
  std::vector<int32_t> keys;
  std::vector<dfc_pred_op> pred;
  std::vector<dfc_agg> aggs;
  void take(const dfc_query* src) {
    q = *src;
    inputs.assign(src->inputs, src->inputs + std::max(0, src->n_inputs));
    keys.assign(src->keys, src->keys + std::max(0, src->n_keys));
    pred.assign(src->pred, src->pred + std::max(0, src->n_pred));
    aggs.assign(src->aggs, src->aggs + std::max(0, src->n_aggs));
    q.inputs = inputs.data();
    q.keys = keys.data();
    q.pred = pred.empty() ? nullptr : pred.data();
    q.aggs = aggs.empty() ? nullptr : aggs.data();
    q.stream = nullptr;
  }
};

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t tag = 0;
  OwnedQuery oq;
  Clock::time_point submitted, admitted;
  BatchItem item;
  size_t bytes = 0;  // device memory it holds while in flight
  unsigned char* arena = nullptr;
  size_t arena_size = 0;
  Control* dctl = nullptr;
  int slot = -1;     // pinned control slot
  bool full = false; // its scan fills every SM
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

}  // namespace

struct dfc_server {
  int device = 0;
  DeviceState* ds = nullptr;
  int max_inflight = 64;
  int64_t budget = 0;       // device bytes in flight at most
  int64_t held = 0;
  int full_inflight = 0;  // admitted requests whose scan fills every SM
  int full_ahead = kFullGridAhead;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::vector<Request*> inflight;
  std::deque<dfc_completion> done;
  std::atomic<int64_t> ready{0};  // completions in `done`
  std::vector<cudaStream_t> streams;
  cudaStream_t plan_stream = nullptr;
  // Working arenas of finished requests, by size, kept for later ones (worker
  // thread only): requests of several GB each otherwise make the memory pool
  // map new memory whenever two of them are in flight.
  std::multimap<size_t, unsigned char*> arenas;
  size_t arena_bytes = 0;
  Control* pinned = nullptr;  // max_inflight control slots
  std::vector<int> free_slots;
  bool stop = false;
  uint64_t submitted = 0, completed = 0, admitted_total = 0;
  int max_seen_inflight = 0;
  std::thread worker;
};

namespace {

void server_complete(dfc_server* sv, Request* r, dfc_status st, dfc_result* res, const std::string& msg) {
  dfc_completion c{};
  c.tag = r->tag;
  c.status = st;
  c.result = res;
  const auto now = Clock::now();
  c.latency_ns = std::chrono::duration<double, std::nano>(now - r->submitted).count();
  c.queue_ns = std::chrono::duration<double, std::nano>(r->admitted - r->submitted).count();
  snprintf(c.message, sizeof c.message, "%s", msg.c_str());
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->done.push_back(c);
  sv->ready.fetch_add(1, std::memory_order_release);
  sv->completed += 1;
  sv->cv_done.notify_all();
}

// A working arena of at least `need` bytes for `r`: the smallest kept one,
// else a new one (64 MiB granules).
cudaError_t arena_get(dfc_server* sv, size_t need, cudaStream_t stream, Request* r) {
  auto it = sv->arenas.lower_bound(need);
  if (it != sv->arenas.end()) {
    r->arena = it->second;
    r->arena_size = it->first;
    sv->arena_bytes -= it->first;
    sv->arenas.erase(it);
    return cudaSuccess;
  }
  const size_t size = (need + (64u << 20) - 1) & ~(size_t)((64u << 20) - 1);
  r->arena_size = size;
  return pool_alloc((void**)&r->arena, size, stream);
}

// Keeps a finished request's arena (at most a quarter of the budget in all,
// the largest released first).
void arena_put(dfc_server* sv, Request* r) {
  sv->arenas.emplace(r->arena_size, r->arena);
  sv->arena_bytes += r->arena_size;
  while (sv->arena_bytes > (size_t)std::max<int64_t>(0, sv->budget / 4) && !sv->arenas.empty()) {
    auto last = std::prev(sv->arenas.end());
    cudaFreeAsync(last->second, r->stream);
    sv->arena_bytes -= last->first;
    sv->arenas.erase(last);
  }
  r->arena = nullptr;
}

// Plans, sizes and launches one request; false when it must wait for memory
// (nothing done) or failed (completed with its error).
bool server_launch(dfc_server* sv, Request* r, int& k) {
  const auto t_start = Clock::now();
  r->item = BatchItem{};  // a request that waited for memory is planned afresh
  BatchItem& it = r->item;
  dfc_status st = plan_query(&r->oq.q, it.P);
  if (!st && it.P.device != sv->device) st = fail(DFC_UNSUPPORTED, "the request's columns live on another device");
  size_t used = 0;
  // Statistics kernels (first use of a key column) run on their own stream,
  // so waiting for them does not wait for requests in flight.
  if (!st) st = size_item(&r->oq.q, it, sv->ds, sv->plan_stream, used);
  cudaStream_t stream = sv->streams[st ? 0 : item_stream(it, k)];
  if (st) {
    r->admitted = Clock::now();
    server_complete(sv, r, st, nullptr, t_error);
    delete r;
    return true;
  }
  // Output bytes count against the budget too (they live until released).
  size_t out_bytes = 0;
  for (int c = 0; c < it.P.n_out; ++c) out_bytes += it.out_rows * 8 + ((it.out_rows + 31) / 32) * 4 + 512;
  r->bytes = used + out_bytes + sizeof(Control);
  r->full = it.full_grid;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->held > 0 && sv->held + (int64_t)r->bytes > sv->budget) return false;  // wait for memory
    // A scan that fills every SM runs after the ones queued before it: with
    // kFullGridAhead of them in flight the device stays busy, and admitting
    // more would only hold their memory early.
    if (r->full && sv->full_inflight >= sv->full_ahead) return false;
    sv->held += (int64_t)r->bytes;
    sv->full_inflight += r->full ? 1 : 0;
  }
  r->admitted = Clock::now();
  r->stream = stream;
  cudaError_t e = arena_get(sv, std::max<size_t>(used, 256), stream, r);
  if (e == cudaSuccess) e = pool_alloc((void**)&r->dctl, sizeof(Control), stream);
  if (e == cudaSuccess && alloc_outputs(it, stream)) e = cudaErrorMemoryAllocation;
  if (e != cudaSuccess) {
    cudaGetLastError();
    release_result_cols(it.rc, it.slab, stream);
    if (r->arena) arena_put(sv, r);
    if (r->dctl) cudaFreeAsync(r->dctl, stream);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->held -= (int64_t)r->bytes;
      sv->full_inflight -= r->full ? 1 : 0;
    }
    server_complete(sv, r, DFC_OOM, nullptr, "device memory for the request");
    delete r;
    return true;
  }
  launch_item(it, sv->ds, r->arena, r->dctl, stream);
  r->slot = sv->free_slots.back();
  sv->free_slots.pop_back();
  cudaMemcpyAsync(sv->pinned + r->slot, r->dctl, sizeof(Control), cudaMemcpyDeviceToHost, stream);
  cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming);
  cudaEventRecord(r->done, stream);
  sv->inflight.push_back(r);
  if (getenv("DFC_TRACE"))
    fprintf(stderr, "dfc serve launch tag=%llu full=%d slots=%llu recs=%llu bytes=%zu smem=%u plan+launch_us=%.1f queued_us=%.1f\n",
            (unsigned long long)r->tag, (int)r->full, (unsigned long long)it.slots, (unsigned long long)it.recs, r->bytes,
            it.P.sp.smem_slots, std::chrono::duration<double, std::micro>(Clock::now() - t_start).count(),
            std::chrono::duration<double, std::micro>(r->admitted - r->submitted).count());
  return true;
}

// Finishes a request whose work is done on the device.
void server_finish(dfc_server* sv, Request* r) {
  const auto t_start = Clock::now();
  dfc_result* res = nullptr;
  const Control c = sv->pinned[r->slot];
  sv->free_slots.push_back(r->slot);
  cudaEventDestroy(r->done);
  arena_put(sv, r);  // its work is done: any later request may reuse it
  cudaFreeAsync(r->dctl, r->stream);
  dfc_status st = finish_item(&r->oq.q, r->item, c, sv->device, &res);
  std::string msg = st ? t_error : std::string();
  if (st) release_result_cols(r->item.rc, r->item.slab, r->stream);
  if (st == DFC_CAPACITY) {  // alone, with regrowth
    st = dfc_groupby(&r->oq.q, &res);
    msg = st ? t_error : std::string();
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->held -= (int64_t)r->bytes;
    sv->full_inflight -= r->full ? 1 : 0;
  }
  if (getenv("DFC_TRACE"))
    fprintf(stderr, "dfc serve finish tag=%llu st=%d groups=%u status=%#x run_us=%.1f finish_us=%.1f\n",
            (unsigned long long)r->tag, (int)st, c.groups, c.status[0],
            std::chrono::duration<double, std::micro>(t_start - r->admitted).count(),
            std::chrono::duration<double, std::micro>(Clock::now() - t_start).count());
  server_complete(sv, r, st, res, msg);
  delete r;
}

bool pending_empty(dfc_server* sv) {
  std::lock_guard<std::mutex> lk(sv->mu);
  return sv->pending.empty();
}

void server_loop(dfc_server* sv) {
  DeviceGuard guard(sv->device);
  int k = 0;
  bool mem_blocked = false;  // the head request waits for memory: retry after a completion
  for (;;) {
    // Admit what arrived, as in-flight slots and memory allow.
    std::vector<Request*> take;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      if (sv->pending.empty() && sv->inflight.empty()) {
        if (sv->stop) return;
        sv->cv_work.wait_for(lk, std::chrono::milliseconds(5));
      }
      while (!mem_blocked && !sv->pending.empty() && (int)(sv->inflight.size() + take.size()) < sv->max_inflight) {
        take.push_back(sv->pending.front());
        sv->pending.pop_front();
      }
    }
    for (size_t i = 0; i < take.size(); ++i) {
      if (!server_launch(sv, take[i], k)) {
        // Not enough memory now: back to the front, in order.
        std::lock_guard<std::mutex> lk(sv->mu);
        for (size_t j = take.size(); j-- > i;) sv->pending.push_front(take[j]);
        mem_blocked = true;
        break;
      }
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->admitted_total += 1;
      sv->max_seen_inflight = std::max(sv->max_seen_inflight, (int)sv->inflight.size());
    }
    // Finish what the device completed.
    bool progressed = false;
    for (size_t i = 0; i < sv->inflight.size();) {
      Request* r = sv->inflight[i];
      const cudaError_t q = cudaEventQuery(r->done);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      sv->inflight.erase(sv->inflight.begin() + (long)i);
      progressed = true;
      if (q != cudaSuccess) {
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          sv->held -= (int64_t)r->bytes;
          sv->full_inflight -= r->full ? 1 : 0;
        }
        server_complete(sv, r, cuda_fail(q, "request execution"), nullptr, t_error);
        delete r;
        continue;
      }
      server_finish(sv, r);
    }
    if (progressed) mem_blocked = false;
    if (!progressed && take.empty()) {
      // Nothing to admit and nothing done: wait for the oldest request in
      // flight (bounded), or briefly when none is.
      if (!sv->inflight.empty() && (mem_blocked || pending_empty(sv))) {
        const auto until = Clock::now() + std::chrono::milliseconds(2);
        while (cudaEventQuery(sv->inflight.front()->done) == cudaErrorNotReady && Clock::now() < until &&
               (mem_blocked || pending_empty(sv)))
          std::this_thread::yield();
      } else {
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      }
    }
  }
}

}  // namespace

extern "C" {

DFC_API dfc_status dfc_server_create(int32_t device, int32_t max_inflight, int64_t memory_budget, dfc_server** out) {
  if (!out) return fail(DFC_INVALID, "null output");
  *out = nullptr;
  DeviceState* ds;
  dfc_status st = device_ready(device, &ds);
  if (st) return st;
  DeviceGuard guard(device);
  auto* sv = new dfc_server();
  sv->device = device;
  sv->ds = ds;
  sv->max_inflight = std::max(1, max_inflight);
  if (memory_budget <= 0) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    memory_budget = (int64_t)(free_b * 0.8);
  }
  sv->budget = memory_budget;
  // DFC_SERVER_FULL_AHEAD=<n>: full-grid requests in flight at most (tuning).
  if (const char* env = getenv("DFC_SERVER_FULL_AHEAD"))
    if (atoi(env) > 0) sv->full_ahead = atoi(env);
  sv->streams.resize(kBatchStreams);
  for (auto& s : sv->streams) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&sv->plan_stream, cudaStreamNonBlocking);
  if (cudaMallocHost((void**)&sv->pinned, sizeof(Control) * sv->max_inflight) != cudaSuccess) {
    for (auto& s : sv->streams) cudaStreamDestroy(s);
    cudaStreamDestroy(sv->plan_stream);
    delete sv;
    return fail(DFC_OOM, "pinned control slots");
  }
  for (int i = sv->max_inflight - 1; i >= 0; --i) sv->free_slots.push_back(i);
  // Grow the device memory pool by a quarter of the budget now (allocated
  // and freed at once; the pool keeps it), so the first requests in flight
  // side by side do not pay for mapping new memory (up to 0.6 s for 8 GB).
  {
    void* warm = nullptr;
    if (pool_alloc(&warm, (size_t)(sv->budget / 4), sv->streams[0]) == cudaSuccess) {
      cudaFreeAsync(warm, sv->streams[0]);
      cudaStreamSynchronize(sv->streams[0]);
    }
    cudaGetLastError();
  }
  sv->worker = std::thread(server_loop, sv);
  *out = sv;
  return DFC_OK;
}

DFC_API dfc_status dfc_server_submit(dfc_server* sv, const dfc_query* query, uint64_t tag) {
  if (!sv || !query) return fail(DFC_INVALID, "null argument");
  if (query->n_inputs < 0 || query->n_keys < 0 || query->n_pred < 0 || query->n_aggs < 0 ||
      (query->n_inputs > 0 && !query->inputs) || (query->n_keys > 0 && !query->keys) ||
      (query->n_pred > 0 && !query->pred) || (query->n_aggs > 0 && !query->aggs))
    return fail(DFC_INVALID, "malformed query");
  auto* r = new Request();
  r->tag = tag;
  r->oq.take(query);
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
      delete r;
      return fail(DFC_INVALID, "the server is stopping");
    }
    sv->pending.push_back(r);
    sv->submitted += 1;
  }
  sv->cv_work.notify_one();
  return DFC_OK;
}

DFC_API int32_t dfc_server_poll(dfc_server* sv, dfc_completion* out, int32_t max, int32_t wait_ms) {
  if (!sv || !out || max <= 0) return 0;
  // A caller that polls in a tight loop must not contend for the worker's
  // lock while nothing is ready.
  if (wait_ms <= 0 && sv->ready.load(std::memory_order_acquire) == 0) return 0;
  std::unique_lock<std::mutex> lk(sv->mu);
  if (sv->done.empty() && wait_ms > 0) sv->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms));
  int32_t n = 0;
  while (n < max && !sv->done.empty()) {
    out[n++] = sv->done.front();
    sv->done.pop_front();
  }
  sv->ready.fetch_sub(n, std::memory_order_release);
  return n;
}

DFC_API dfc_status dfc_server_stats_get(dfc_server* sv, dfc_server_stats* out) {
  if (!sv || !out) return fail(DFC_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  out->submitted = sv->submitted;
  out->completed = sv->completed;
  out->pending = sv->pending.size();
  out->inflight = sv->inflight.size();
  out->max_inflight_seen = sv->max_seen_inflight;
  out->bytes_held = sv->held;
  out->budget = sv->budget;
  return DFC_OK;
}

DFC_API void dfc_server_destroy(dfc_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  sv->worker.join();  // the loop drains pending and in-flight requests first
  for (auto& c : sv->done)
    if (c.result) dfc_result_free(c.result);
  DeviceGuard guard(sv->device);
  for (auto& s : sv->streams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  cudaStreamSynchronize(sv->plan_stream);
  cudaStreamDestroy(sv->plan_stream);
  for (auto& a : sv->arenas) cudaFree(a.second);
  cudaFreeHost(sv->pinned);
  delete sv;
}

}  // extern "C"
