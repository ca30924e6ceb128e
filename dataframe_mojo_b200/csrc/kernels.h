// kernels.h — kernel entry points and launch constants.
#pragma once

#include "dfc_internal.h"

namespace dfc {

constexpr int kScanRowsPerThread = 4;  // rows each consumer thread holds in flight
constexpr int kScanConsumerWarps = 8;
constexpr int kScanConsumerThreads = kScanConsumerWarps * 32;
constexpr int kScanThreads = kScanConsumerThreads + 32;  // + one producer warp
constexpr int kFinishThreads = 256;
// finish_output's dynamic shared memory: one slab slot (record stride + 8
// bytes) per thread.
inline size_t finish_output_smem(int rec_stride) { return (size_t)kFinishThreads * ((size_t)rec_stride + 8); }
constexpr int kFinishChunk = 4096;  // bitmap words per prefix-scan block

// The scan, one kernel per table regime: the global table only, per-CTA
// shared-memory tables, shared-memory tables pooled over a thread-block
// cluster (launched with a cluster dimension of ScanParams::smem_cluster).
// kScanReduce: ungrouped queries (no key), every consumer thread folding its
// rows into registers (ScanParams::reduce).
enum ScanRegime : int { kScanGlobal = 0, kScanOwn = 1, kScanCluster = 2, kScanReduce = 3 };
__global__ void scan_kernel_global(const __grid_constant__ ScanParams p);
__global__ void scan_kernel_own(const __grid_constant__ ScanParams p);
__global__ void scan_kernel_cluster(const __grid_constant__ ScanParams p);
__global__ void scan_kernel_reduce(const __grid_constant__ ScanParams p);
constexpr int kReduceVals = 2;  // value columns the register path holds
// Radix-partitioned regime: the counting pass, the partition starts, pass A
// (filter, keys, placement into partitions) and pass B (per-partition
// aggregation in a shared-memory table, kAggThreads threads per CTA).
constexpr int kAggThreads = 512;
constexpr int kPartMaxBits = 15;  // partitions at most: 2^15
// The partition passes: one producer warp and kPartWarps consumer warps.
constexpr int kPartWarps = 16;
constexpr int kPartConsumerThreads = kPartWarps * 32;
constexpr int kPartThreads = kPartConsumerThreads + 32;
constexpr uint32_t kRecChunk = 4096;  // records pass B draws from `alloc` at a time
__global__ void partition_count(const __grid_constant__ ScanParams p);
__global__ void partition_count_quad(const __grid_constant__ ScanParams p);  // the quad row path (fast_rows)
__global__ void partition_offsets(const __grid_constant__ ScanParams p);
__global__ void partition_kernel(const __grid_constant__ ScanParams p);
__global__ void partition_kernel_quad(const __grid_constant__ ScanParams p);
__global__ void partition_aggregate(const __grid_constant__ ScanParams p);
__global__ void finish_mark(const __grid_constant__ FinishParams f);
__global__ void finish_chunk_sums(const __grid_constant__ FinishParams f);
__global__ void finish_scan_chunks(const __grid_constant__ FinishParams f, uint32_t chunks);
__global__ void finish_word_prefix(const __grid_constant__ FinishParams f);
__global__ void finish_rank(const __grid_constant__ FinishParams f);
__global__ void finish_output(const __grid_constant__ FinishParams f);

}  // namespace dfc

namespace dfc {
__global__ void normalize_validity(const uint8_t* src, uint64_t nbytes, uint64_t off, uint64_t rows, uint32_t* dst,
                                   unsigned long long* valid_rows);
constexpr int kHllBits = 12;
constexpr int kStatsUnroll = 8;  // rows in flight per thread in column_stats
constexpr int kKeysUnroll = 4;   // and in keys_hll (each row loads every key column)
__global__ void column_stats(DevColumn c, uint64_t rows, unsigned long long* mm, uint32_t* regs);
__global__ void keys_hll(const __grid_constant__ ScanParams p, uint32_t* regs);
__global__ void keys_sample(const __grid_constant__ ScanParams p, unsigned long long* out, uint32_t n, uint64_t stride);
}  // namespace dfc
