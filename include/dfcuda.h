/*
 * dfcuda.h — C ABI of libdfcuda.so, a B200 (sm_100a) accelerator provider for
 * dataframe_mojo's filtered hash group-by:
 *
 *     filter(predicate) -> group_by(keys, maintain_order) -> agg(...)
 *
 * The reference reaches an accelerator through thirteen provider functions
 * re-exported by dataframe/_accel_provider.mojo:10-27 (contract:
 * docs/design/accelerator-contract.md:22-70).  Those functions take Mojo
 * objects (LazyFrame, DataFrame).  A provider package written in Mojo
 * marshals them into the plain descriptors below and calls this library
 * through external_call / OwnedDLHandle, the pattern the reference already
 * uses for its native Parquet shim (dataframe/io/native_library.mojo:38-90,
 * native/dfparquet/dfparquet.sym).  Nothing here names a Mojo or torch type.
 *
 * Threading: every entry point is thread-safe.  One CUDA context per device
 * (the primary context); a query runs on the caller's stream or on a stream
 * owned by the library; the resident-column registry is guarded by a lock.
 *
 * Errors: every call that can fail returns a dfc_status; the text of the last
 * failure on the calling thread is dfc_last_error().  Checked integer sums
 * report DFC_DATA_OVERFLOW with the reference CPU's exact message
 * ("Int64 expression sum overflow", "int32 expression sum overflow", ...:
 * dataframe/aggregation/function.mojo:2798, 2914).
 */
#ifndef DFCUDA_H
#define DFCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFC_ABI_VERSION 1u

#if defined(__GNUC__)
#define DFC_API __attribute__((visibility("default")))
#else
#define DFC_API
#endif

/* ------------------------------------------------------------------------ */
/* Status codes.                                                             */
/* ------------------------------------------------------------------------ */
typedef enum dfc_status {
  DFC_OK = 0,
  /* Rejected before anything was submitted (contract: "Raises for
   * unsupported work before submitting anything",
   * docs/design/accelerator-contract.md:28). */
  DFC_UNSUPPORTED = 1,
  /* Malformed arguments (null pointers, mismatched row counts, ...). */
  DFC_INVALID = 2,
  /* A checked integer sum does not fit its result type; dfc_last_error()
   * holds the CPU provider's message. */
  DFC_DATA_OVERFLOW = 3,
  /* A value-dependent result the CPU must adjudicate (the reference's data
   * fault, dataframe_metal/accelerator/faults.mojo:1-18). */
  DFC_DATA_FAULT = 4,
  /* The group table could not grow far enough (after the bounded retries). */
  DFC_CAPACITY = 5,
  /* Device memory could not be allocated. */
  DFC_OOM = 6,
  /* A bounded device wait gave up. */
  DFC_TIMEOUT = 7,
  /* A CUDA call failed. */
  DFC_DEVICE = 8,
  /* No usable sm_100 device. */
  DFC_NO_DEVICE = 9
} dfc_status;

/* ------------------------------------------------------------------------ */
/* Column types (numeric storage types of dataframe/dtype.mojo).             */
/* ------------------------------------------------------------------------ */
typedef enum dfc_dtype {
  DFC_INT8 = 1,
  DFC_INT16 = 2,
  DFC_INT32 = 3,
  DFC_INT64 = 4,
  DFC_UINT8 = 5,
  DFC_UINT16 = 6,
  DFC_UINT32 = 7, /* also a categorical's dictionary codes */
  DFC_UINT64 = 8,
  DFC_FLOAT32 = 9,
  DFC_FLOAT64 = 10
} dfc_dtype;

/* ------------------------------------------------------------------------ */
/* Devices (reference: dataframe/devices.mojo:64-141; provider functions     */
/* devices() and transfer_model()).  Neither call creates a context.        */
/* ------------------------------------------------------------------------ */
typedef struct dfc_device_info {
  int32_t ordinal;
  int32_t sm_count;
  int32_t cc_major;
  int32_t cc_minor;
  uint64_t total_bytes;  /* HBM capacity */
  int64_t budget_bytes;  /* bytes the planner may hold there; -1 = no limit */
  char name[96];
} dfc_device_info;

/* Library ABI version (DFC_ABI_VERSION).  Mirrors the version probe of the
 * reference's native shim (native/dfparquet/dfparquet.sym). */
DFC_API uint32_t dfc_version(void);

/* Whether this library can run here: built for sm_100a and an NVIDIA device
 * node is present.  Opens no driver and creates no context (provider
 * installed(), dataframe/_accel_provider.mojo:11;
 * docs/design/accelerator-contract.md:27). */
DFC_API int32_t dfc_installed(void);

/* Number of sm_100 devices; reads driver metadata only (provider devices(),
 * docs/design/accelerator-contract.md:40). */
DFC_API int32_t dfc_device_count(void);
DFC_API dfc_status dfc_device_info_get(int32_t ordinal, dfc_device_info* out);

/* A copy's cost, `fixed_ns + ns_per_byte * bytes` nanoseconds (the
 * reference's ByteCost, dataframe/devices.mojo:44-56). */
typedef struct dfc_byte_cost {
  double fixed_ns;
  double ns_per_byte;
} dfc_byte_cost;

/* Measures pinned host <-> device copies on `device` (provider
 * transfer_model(), dataframe/devices.mojo:59-80): the best of three copies
 * of 4 KiB and of `bytes` each way, timed by CUDA events, fitted to a fixed
 * cost and a cost per byte.  Creates the device's context. */
DFC_API dfc_status dfc_measure_transfer(int32_t device, uint64_t bytes, dfc_byte_cost* to_device,
                                        dfc_byte_cost* to_host);

/* ------------------------------------------------------------------------ */
/* Device column handoff: typed values plus an Arrow LSB-first validity     */
/* bitmap, resident in HBM across queries.                                  */
/* Reference: Column[T] = value buffer + validity bits + offset window,     */
/* dataframe/storage/column.mojo:1-32, dataframe/storage/bitmap.mojo:1-76;  */
/* device residence: dataframe/storage/residence.mojo:20-72.                */
/* ------------------------------------------------------------------------ */
typedef struct dfc_column dfc_column;

/* The most bytes one query may hold on `device` (its working memory and its
 * result columns); a query that would need more is rejected with
 * DFC_UNSUPPORTED before its kernels are submitted.  <= 0: no limit.  The
 * provider sets it from DATAFRAME_ACCEL_MEMORY_LIMIT, the name the
 * reference's contract keeps (docs/design/accelerator-contract.md:168-171);
 * dfc_device_info_get reports it as budget_bytes. */
DFC_API dfc_status dfc_set_memory_limit(int32_t device, int64_t bytes);

/* values/validity point to host memory: the library copies them into HBM
 * (validity normalised to bit offset 0) and keeps them resident. */
#define DFC_COLUMN_HOST 0u
/* values (and validity, when given) point to device memory the caller owns
 * and keeps alive until dfc_column_release; only the validity bitmap is
 * copied (normalised).  Both must be device memory of `device`
 * (cudaPointerGetAttributes): host, managed or another GPU's memory is
 * rejected with DFC_INVALID.  Registration first waits for the device's
 * queued work (cudaDeviceSynchronize), so values written on any stream
 * before the call are the ones read; writes after it must be ordered before
 * the query's stream (dfc_query.stream) by the caller. */
#define DFC_COLUMN_DEVICE 1u

/* validity may be NULL (every row valid).  validity_bit_offset is the bit
 * of row 0 inside validity (an Arrow window's offset). */
DFC_API dfc_status dfc_column_register(int32_t device, dfc_dtype dtype,
                                       uint64_t rows, const void* values,
                                       const uint8_t* validity,
                                       uint64_t validity_bit_offset,
                                       uint32_t flags, dfc_column** out);
DFC_API dfc_status dfc_column_release(dfc_column* column);
DFC_API uint64_t dfc_column_rows(const dfc_column* column);
DFC_API int32_t dfc_column_null_count(const dfc_column* column);

/* ------------------------------------------------------------------------ */
/* The query: a bound SCAN -> FILTER* -> AGG region                          */
/* (dataframe/query_execution/placement.mojo:74-94).                        */
/* ------------------------------------------------------------------------ */

/* Predicate program, postfix.  Comparisons follow IEEE rules for floats
 * (NaN compares false except !=) and a null operand makes the comparison
 * null; AND/OR/NOT are Kleene; a row is kept only when the program is true
 * (dataframe/kernels/fused_compare.mojo:31-183; kernels/binary.mojo:2172). */
typedef enum dfc_pred_kind {
  DFC_PRED_CMP = 1,         /* inputs[column] <cmp> literal */
  DFC_PRED_IS_NULL = 2,     /* inputs[column] is null */
  DFC_PRED_IS_NOT_NULL = 3, /* inputs[column] is not null */
  DFC_PRED_AND = 4,
  DFC_PRED_OR = 5,
  DFC_PRED_NOT = 6,
  DFC_PRED_TRUE = 7
} dfc_pred_kind;

typedef enum dfc_cmp { DFC_LT = 1, DFC_LE = 2, DFC_GT = 3, DFC_GE = 4, DFC_EQ = 5, DFC_NE = 6 } dfc_cmp;

/* The literal is already bound to the column's type (binding happens in the
 * core before a backend is chosen, docs/design/accelerator-contract.md:75):
 * integer columns read lit.i (signed) or lit.u (UINT64), float columns lit.f. */
typedef struct dfc_pred_op {
  int32_t kind;   /* dfc_pred_kind */
  int32_t column; /* index into dfc_query.inputs (CMP / IS_NULL / IS_NOT_NULL) */
  int32_t cmp;    /* dfc_cmp (CMP) */
  int32_t reserved;
  union {
    int64_t i;
    uint64_t u;
    double f;
  } lit;
} dfc_pred_op;

/* Aggregations (dataframe/expr.mojo reduction ops; state kinds
 * dataframe/aggregation/function.mojo:187-254). */
typedef enum dfc_agg_op {
  DFC_AGG_COUNT = 1,      /* valid values, Int64, never null */
  DFC_AGG_SUM = 2,        /* sum type of the input; null when count < min_count */
  DFC_AGG_MEAN = 3,       /* Float64; null when count == 0 */
  DFC_AGG_MIN = 4,        /* input type; NaN only when every valid value is NaN */
  DFC_AGG_MAX = 5,
  DFC_AGG_VAR = 6,        /* Float64, M2 / (n - ddof); null when n <= ddof */
  DFC_AGG_STD = 7,
  DFC_AGG_LEN = 8,        /* rows of the group, Int64 */
  DFC_AGG_NULL_COUNT = 9, /* null values, Int64 */
  /* The value at the group's first (last) row among the rows the filter
   * kept, null when that row's value is null; the input type
   * (dataframe/aggregation/function.mojo:997-1013, 1586-1600, 2637-2650). */
  DFC_AGG_FIRST = 10,
  DFC_AGG_LAST = 11,
  /* Distinct values of the group, Int64: null counts as one value, every
   * NaN is one value and -0.0 == 0.0, the key equality
   * (function.mojo:620-625; tests/public_contracts/test_approx_n_unique.mojo:60-80). */
  DFC_AGG_N_UNIQUE = 12
} dfc_agg_op;

typedef struct dfc_agg {
  int32_t op;        /* dfc_agg_op */
  int32_t column;    /* index into dfc_query.inputs */
  int32_t ddof;      /* VAR / STD (reference default 1, dataframe/expr.mojo:2904-2910) */
  int32_t min_count; /* SUM (reference default 0) */
} dfc_agg;

/* Query flags. */
#define DFC_Q_MAINTAIN_ORDER 1u    /* groups in first-occurrence order of the rows the filter kept */
#define DFC_Q_FORCE_GLOBAL 2u      /* skip the shared-memory table regime */
#define DFC_Q_FORCE_SHARED 4u      /* use the shared-memory table regime regardless of estimates */
#define DFC_Q_FLOAT32_COMPENSATED 8u /* Float32 sums and variances: compensated FP32 partials in the shared-memory
                                        tables, merged in FP64 (default: FP64 accumulation throughout) */
#define DFC_Q_FORCE_PARTITIONED 16u /* use the radix-partitioned regime regardless of estimates (keys <= 64 bits) */

typedef struct dfc_query {
  uint32_t abi_version; /* DFC_ABI_VERSION */
  uint32_t flags;       /* DFC_Q_* */
  int32_t n_inputs;     /* columns the query reads; all have the same row count */
  int32_t n_keys;       /* 0..4; 0: ungrouped reductions, one output row even when no row is kept */
  dfc_column* const* inputs;
  const int32_t* keys;  /* n_keys indices into inputs */
  int32_t n_pred;       /* 0 keeps every row */
  int32_t n_aggs;       /* 0..32 */
  const dfc_pred_op* pred;
  const dfc_agg* aggs;
  void* stream;         /* cudaStream_t, or NULL for the library's per-thread stream */
} dfc_query;

/* ------------------------------------------------------------------------ */
/* Results: n_keys key columns then one column per aggregation, resident    */
/* on the device until dfc_result_free.                                     */
/* ------------------------------------------------------------------------ */
typedef struct dfc_result dfc_result;

/* Runs the query and waits for it.  On DFC_OK *out holds the result.
 * Provider execute()/handoff_execute() (docs/design/accelerator-contract.md:
 * 28, 32) reduce to this call. */
DFC_API dfc_status dfc_groupby(const dfc_query* query, dfc_result** out);

/* ------------------------------------------------------------------------ */
/* Many queries in one submission (the batched form).  The reference core   */
/* issues one execute() per region; a server or a pipeline with many small  */
/* regions pays a host round trip and a device synchronisation per query.   */
/* This plans every query, takes their working memory from one arena,       */
/* spreads their launches over several streams with no synchronisation in   */
/* between, and reads every control block back at once.  statuses[i] and    */
/* results[i] are query i's outcome (dfc_batch_error(i) its message); a     */
/* query that outgrows its capacity estimate reruns alone with regrowth.    */
/* Returns DFC_OK when the batch ran (look at statuses), else the failure   */
/* that stopped all of it.  The radix-partitioned regime is not used here.  */
/* ------------------------------------------------------------------------ */
DFC_API dfc_status dfc_groupby_batch(const dfc_query* const* queries, int32_t n, dfc_result** results,
                                     dfc_status* statuses);
DFC_API const char* dfc_batch_error(int32_t i);

/* ------------------------------------------------------------------------ */
/* The served form: a request loop with continuous batching.  The reference */
/* has no server (its core runs one query per collect()); this serves many  */
/* clients over resident tables.  A worker thread admits submitted requests */
/* while fewer than max_inflight are on the device and their working memory */
/* fits memory_budget (<= 0: 80% of the free HBM at creation), launches     */
/* each on one of several streams without waiting for the others, and       */
/* finishes each as its device work completes: requests that arrive while   */
/* others run are admitted as slots and memory free up, and their work      */
/* overlaps.  The columns a request names must stay registered until its    */
/* completion is polled.                                                    */
/* ------------------------------------------------------------------------ */
typedef struct dfc_server dfc_server;

typedef struct dfc_completion {
  uint64_t tag;          /* as submitted */
  int32_t status;        /* dfc_status */
  int32_t reserved;
  dfc_result* result;    /* on DFC_OK: the caller frees it */
  double latency_ns;     /* submission to completion */
  double queue_ns;       /* submission to admission */
  char message[160];     /* the error text when status != DFC_OK */
} dfc_completion;

typedef struct dfc_server_stats {
  uint64_t submitted;
  uint64_t completed;
  uint64_t pending;
  uint64_t inflight;
  int64_t max_inflight_seen;
  int64_t bytes_held;
  int64_t budget;
} dfc_server_stats;

DFC_API dfc_status dfc_server_create(int32_t device, int32_t max_inflight, int64_t memory_budget,
                                     dfc_server** out);
/* Copies the query description; returns at once. */
DFC_API dfc_status dfc_server_submit(dfc_server* server, const dfc_query* query, uint64_t tag);
/* Up to max completions, waiting up to wait_ms for the first; returns how many. */
DFC_API int32_t dfc_server_poll(dfc_server* server, dfc_completion* out, int32_t max, int32_t wait_ms);
DFC_API dfc_status dfc_server_stats_get(dfc_server* server, dfc_server_stats* out);
/* Finishes every submitted request, frees unpolled results, stops. */
DFC_API void dfc_server_destroy(dfc_server* server);

/* ------------------------------------------------------------------------ */
/* The same query without any device allocation.  No counterpart in the    */
/* reference: it is for callers that cannot call cudaMalloc -- code running  */
/* under an allocator that owns the device heap (a host framework's caching */
/* pool or a fixed memory budget), or code that must not allocate while it  */
/* holds a lock or serves latency-bound requests.  They pass device inputs  */
/* and device output buffers they already own; the working memory (key      */
/* table, group records, order bitmaps, staged outputs) comes from one       */
/* fixed array of DFC_NOALLOC_SCRATCH_BYTES that every GPU loading this     */
/* library holds until the process exits.                                   */
/*                                                                          */
/* - A query whose working memory exceeds the array is rejected with        */
/*   DFC_CAPACITY and a message giving the bytes it needs; nothing runs.    */
/*   Roughly: rows/4 bytes of bitmaps plus, per group of capacity, 32 to 64 */
/*   bytes of table, 16 to 32 bytes per output column and one group record; */
/*   what is left of the array goes to records for claims that lose a race. */
/*   A query whose racing claims use up those records fails with           */
/*   DFC_CAPACITY too (hot keys over many groups); dfc_groupby regrows.     */
/* - The first call on a device looks up the array's device address (with  */
/*   that device current); make that first call before any stream capture. */
/* - Every call shares the array, which keeps the last call's contents;     */
/*   each call clears what must start at zero.  The library runs one call   */
/*   per device at a time and waits for its work, but work that is still on */
/*   the GPU when the next call starts (after a DFC_TIMEOUT, say) races     */
/*   with it and corrupts both: calls must not overlap on the GPU.          */
/* - Results are the same as dfc_groupby's.  Groups come back in the same   */
/*   order; floating sums and moments may differ in the last bits, as      */
/*   between two dfc_groupby calls.  A compensated FP32 partial that leaves */
/*   the FP32 range reruns the query in FP64 in the same array, as          */
/*   dfc_groupby reruns it.                                                 */
/* - The table regime comes from `capacity` alone (no statistics pass):     */
/*   per-CTA shared-memory tables up to 256 groups (4096 with               */
/*   DFC_Q_FLOAT32_COMPENSATED, any count with DFC_Q_FORCE_SHARED), the    */
/*   global table otherwise; DFC_Q_FORCE_PARTITIONED is ignored.            */
/* - dfc_last_timings reports this call's groups, table slots, regime,      */
/*   launches, retries and compensated fields; no phase times.              */
/* ------------------------------------------------------------------------ */
#define DFC_NOALLOC_SCRATCH_BYTES (64ull << 20)

/* A column in device memory, read in place. */
typedef struct dfc_device_column {
  int32_t dtype;            /* dfc_dtype */
  int32_t reserved;         /* 0 */
  const void* values;       /* rows values, 16-byte aligned */
  const uint32_t* validity; /* LSB-first bitmap at bit offset 0 in ceil(rows/32) 32-bit words,
                               16-byte aligned; NULL when every row is valid */
} dfc_device_column;

/* An output column in device memory the caller owns. */
typedef struct dfc_device_output {
  void* values;       /* capacity * 8 bytes at least (any output type fits) */
  uint32_t* validity; /* ceil(capacity / 32) 32-bit words, LSB first */
  int32_t dtype;      /* set by the call: the column's dfc_dtype */
  int32_t has_nulls;  /* set by the call: 1 when some validity bit is 0 */
} dfc_device_output;

/* Runs `query` over `columns` (query->n_inputs entries, all `rows` long, on
 * `device`; query->inputs is not read) and writes n_keys + n_aggs columns
 * (keys, then one per aggregation) into `outputs`, *groups rows each.
 * `capacity` is the most groups the outputs hold: more groups fail with
 * DFC_CAPACITY.  It waits for the work on query->stream, or on the calling
 * thread's default stream when that is NULL. */
DFC_API dfc_status dfc_groupby_noalloc(const dfc_query* query, int32_t device, uint64_t rows,
                                       const dfc_device_column* columns, uint64_t capacity,
                                       dfc_device_output* outputs, uint64_t* groups);

DFC_API uint64_t dfc_result_rows(const dfc_result* result);
DFC_API int32_t dfc_result_columns(const dfc_result* result);
/* Device pointers of column i; *device_validity is NULL when the column has
 * no nulls. */
DFC_API dfc_status dfc_result_column(const dfc_result* result, int32_t i, dfc_dtype* dtype,
                                     const void** device_values,
                                     const uint8_t** device_validity);
/* Copies column i to host memory: values (rows * size of dtype bytes) and,
 * when validity is not NULL, an LSB-first bitmap of ceil(rows / 8) bytes
 * (all ones when the column has no nulls). */
DFC_API dfc_status dfc_result_copy_to_host(const dfc_result* result, int32_t i, void* values,
                                           uint8_t* validity);
/* The same into device memory of the result's device (a following device
 * step's buffers, e.g. the sharded group-by's exchange): device-to-device
 * copies, waited for. */
DFC_API dfc_status dfc_result_copy_to_device(const dfc_result* result, int32_t i, void* values,
                                             uint8_t* validity);
DFC_API void dfc_result_free(dfc_result* result);

/* Residence callbacks in the shape of the reference's _DeviceResidence
 * (dataframe/storage/residence.mojo:20-22): ctx is a dfc_result column
 * handle made by dfc_result_residence(result, i). to_host returns 0 on
 * success; release frees the handle (the result keeps its own reference). */
DFC_API void* dfc_result_residence(dfc_result* result, int32_t i);
/* The same for column i's validity bitmap (ceil(rows / 8) LSB-first bytes);
 * NULL when the column has no nulls. */
DFC_API void* dfc_result_validity_residence(dfc_result* result, int32_t i);
DFC_API int32_t dfc_residence_to_host(void* ctx, void* host_dst, int64_t bytes);
DFC_API void dfc_residence_release(void* ctx);

/* Per-phase device timings of the last query on this thread, nanoseconds
 * (the provider's report frame; dataframe/execution_observation.mojo:6-83). */
typedef struct dfc_timings {
  double scan_ns;
  double finish_ns;
  double total_ns;
  uint64_t groups;
  uint64_t table_slots;
  int32_t regime;   /* 0 global table, 1 shared-memory tables, 2 radix-partitioned, 3 ungrouped in registers */
  int32_t retries;  /* capacity regrowths */
  int32_t launches; /* kernels this library launched for the query */
  int32_t partitions;  /* radix-partitioned regime: partitions (else 0) */
  double aggregate_ns; /* radix-partitioned regime: the per-partition aggregation pass (scan_ns: the partition pass) */
  int32_t cluster_ctas; /* shared-memory regime: CTAs pooling one table (1: each CTA its own) */
  int32_t compensated;  /* value fields accumulated as compensated FP32 partials (bit per field) */
  double count_ns;      /* radix-partitioned regime: the counting pass (part of scan_ns) */
  double place_ns;      /* radix-partitioned regime: the pass placing rows into partitions (part of scan_ns) */
  uint64_t kept_rows;        /* radix-partitioned regime: rows the filter kept (each placed once) */
  uint64_t placed_row_bytes; /* radix-partitioned regime: bytes of one placed row */
  uint64_t direct_slots;     /* shared-memory regime: slots of own tables addressed by key value (0: hashed) */
} dfc_timings;
DFC_API dfc_status dfc_last_timings(dfc_timings* out);

/* Makes `stream` (a cudaStream_t; NULL restores the library's own) the
 * stream this thread's calls on `device` use when they are not given one:
 * column registration, queries without dfc_query.stream, result copies. */
DFC_API dfc_status dfc_set_thread_stream(int32_t device, void* stream);

/* Text of the last failing call on this thread ("" when none). */
DFC_API const char* dfc_last_error(void);
DFC_API const char* dfc_status_name(dfc_status status);

#ifdef __cplusplus
}
#endif

#endif /* DFCUDA_H */
