/*
 * oracle.h — CPU restatement of dataframe_mojo's filtered grouped reduction
 * (filter -> group_by(keys, maintain_order) -> agg), used ONLY as test
 * infrastructure: the parity checker of the CUDA path (tests/, smoke()) and
 * the timed CPU baseline of bench.py.  The product never links it.
 *
 * Pinning: the restatement is checked against the reference's own
 * known-answer fixtures and generator models (tests/golden/, see
 * tests/test_oracle_golden.py), transcribed from
 *   tests/execution_modes/test_metal_grouped_reductions.mojo:317-560,
 *   tests/support/aggregate_table_reference.mojo:1-330,
 *   tests/public_contracts/test_grouping.mojo:71-105,
 *   benchmarks/bench_gpu_groupby_engine.mojo:12-58,
 *   docs/design/metal-moments.md:139-147 (the Welford example).
 *
 * The query descriptors are the library's own (include/dfcuda.h); columns
 * are host arrays here.
 */
#ifndef DFC_ORACLE_H
#define DFC_ORACLE_H

#include <stdint.h>

#include "../include/dfcuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_column {
  int32_t dtype;            /* dfc_dtype */
  uint64_t rows;
  const void* values;
  const uint8_t* validity;  /* LSB-first, NULL = all valid */
  uint64_t bit_offset;
} orc_column;

typedef struct orc_query {
  uint32_t flags;           /* DFC_Q_MAINTAIN_ORDER honoured; others ignored */
  int32_t n_inputs;
  int32_t n_keys;
  const orc_column* inputs;
  const int32_t* keys;
  int32_t n_pred;
  int32_t n_aggs;
  const dfc_pred_op* pred;
  const dfc_agg* aggs;
} orc_query;

typedef struct orc_result orc_result;

/* Sequential restatement: rows in input order, one worker; equals the
 * reference at DATAFRAME_THREADS=1 for every output (floats bit-for-bit).
 * Returns a dfc_status; on failure orc_error() holds the message. */
int32_t orc_groupby(const orc_query* q, orc_result** out);

/* Multithreaded restatement of the reference's parallel aggregate table
 * (dataframe/aggregation/hash_table.mojo:1-52): per-worker tables over
 * contiguous morsels, hash partitions merged partition-wise (Welford states
 * by Chan's update, function.mojo:1736-1758), then the partitions' runs
 * merged by first row.  threads <= 0 uses every hardware thread. */
int32_t orc_groupby_parallel(const orc_query* q, int32_t threads, orc_result** out);

uint64_t orc_result_rows(const orc_result* r);
int32_t orc_result_columns(const orc_result* r);
int32_t orc_result_dtype(const orc_result* r, int32_t i);
/* Values (rows * size of dtype) and one validity byte per row. */
const void* orc_result_values(const orc_result* r, int32_t i);
const uint8_t* orc_result_valid(const orc_result* r, int32_t i);
/* First selected row of each group (the order key of maintain_order). */
const uint64_t* orc_result_first_rows(const orc_result* r);
void orc_result_free(orc_result* r);
const char* orc_error(void);

#ifdef __cplusplus
}
#endif

#endif
