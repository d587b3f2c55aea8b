// Internal interface between the host runtime (C++) and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace q1 {

// Input layouts the scan kernel understands (column order inside a tile in brackets).
enum ScanLayout : int {
    kLayPair = 0,        // [ship u16, qty u8, disc u8, tax u8, price u32, pair code 2b]
    kLayPairFilter = 1,  // [filter 1b, qty, disc, tax, price, pair code 2b]
    kLaySep = 2,         // [ship u16, qty, disc, tax, price, rf 2b, ls 1b]
    kLaySepFilter = 3,   // [filter 1b, qty, disc, tax, price, rf 2b, ls 1b]
    kLayUncomp = 4,      // [ship i32, qty i64, disc i64, tax i64, price i64, rf char, ls char]
    kNumScanLayouts = 5
};

// Table placements (same numbering as q1_placement in include/q1.h).
enum ScanPlacement : int {
    kPlaceInRegisters = 0,
    kPlaceInRegistersPerThread = 1,
    kPlaceLocalMem = 2,
    kPlaceSharedMemPerThread = 3,
    kPlaceGlobal = 4,
};

// Consumer warps per CTA (plus one producer warp), per input layout and placement, as measured on
// the 600 M-row table (100 M uncompressed). More warps per SM sub-partition hide more of the decode's
// issue latency where the registers allow. 12 warps leave 128 registers a thread (13 warps, which the
// allocator rounds up to 16 warps' worth): the pair layouts' kernels fit (in_registers_per_thread
// 0.909 -> 0.871 ms; in_registers, shared and global 5-20% faster), and so do the separate-flag
// layouts' register placements, which keep only four groups' planes in registers (A/O and R/O go
// to the CTA's shared table: per-thread 1.129 ms with 8 warps and six planes, 1.044 with 10, 0.980
// with 12; global 1.31 -> 1.22 -> 1.16). Their shared placement runs 10 (3.04 -> 2.71 ms), and so
// does the uncompressed layout, which needs up to 168 registers (per-thread 0.625 -> 0.600 ms
// although one register spills; shared 0.670 -> 0.548). local_mem keeps 8 with compressed rows
// (its per-thread tables run out of L1 with more threads: pair 2.83 -> 3.06 ms), and so does the
// separate layout's in_registers (3.58 -> 3.65 ms with 10).
template <int L, int P>
inline constexpr uint32_t kConsumerWarps =
    (L == kLayPair || L == kLayPairFilter) ? (P == kPlaceLocalMem ? 8u : 12u)
    : (L == kLaySep || L == kLaySepFilter)
        ? ((P == kPlaceLocalMem || P == kPlaceInRegisters) ? 8u
                                                           : ((P == kPlaceSharedMemPerThread) ? 10u : 12u))
        : 10u;
// Rows per tile (one bulk copy per column per tile): a multiple of 128, so that every column slice
// of every tile starts on a 16-byte boundary down to 1-bit columns, and of the consumer threads x
// the rows of a step, so that a tile's steps divide evenly among the consumer threads.
template <int L, int P>
inline constexpr uint32_t kTileRows =
    (L == kLayUncomp) ? 128u * kConsumerWarps<L, P> : (kConsumerWarps<L, P> == 8u ? 4096u : 384u * kConsumerWarps<L, P>);
// Shared-memory ring depth.
template <int L, int P>
inline constexpr uint32_t kStages = (P == kPlaceSharedMemPerThread) ? 3u : 4u;
// Tiles a warp of the global placement write-combines in registers between its atomic adds into
// the global table (12 or 16 rows per thread of a compressed tile, so 49,152 or 65,536 rows per warp
// between flushes; a few flushes per warp over 600 M rows). Measured on 600 M rows (8 warps,
// 4096-row tiles): 1 tile 12.94 ms (same-address L2 atomics serialise: 7.1 M atomic requests per
// 100 M rows), 4 tiles 4.05 ms, 16 tiles 1.95 ms, 64 tiles 1.22 ms, 128 tiles 1.08 ms. A 64-bit
// warp sum bounds the rows a thread may buffer (the kernel's static_assert).
#ifndef Q1_GLOBAL_FLUSH_TILES
#define Q1_GLOBAL_FLUSH_TILES 128
#endif
inline constexpr uint32_t kGlobalFlushTiles = Q1_GLOBAL_FLUSH_TILES;

struct ScanParams {
    const uint8_t* col[7];      // column base pointers in tile order; 16-byte aligned
    uint64_t rows;              // rows to aggregate (<= 2^31 per launch)
    int32_t cutoff;             // compressed: cutoff_day - 727563; uncompressed: cutoff_day
    uint32_t qty_scale;         // 100 when quantity is stored in whole units, else 1
    uint8_t pair_group[4];      // pair layouts: code -> group
    unsigned long long* out;    // [6 groups][6 aggregates][lo, hi]
    uint32_t* status;           // device status word (kStatus* bits); may be null
    unsigned long long* records;  // null: atomics into `out`. Otherwise each CTA writes its own
                                  // [6][6][lo, hi] record at records[blockIdx.x] and leaves `out`
                                  // alone (used by the allocation-free entry point)
};

// Launch the scan kernel for one layout x placement. max_blocks <= 0: one CTA per SM.
cudaError_t launch_scan(int layout, int placement, const ScanParams& prm, int sm_count, int max_blocks,
                        cudaStream_t stream);
// Rows per tile of the layout x placement (a multiple of 128).
uint32_t scan_tile_rows(int layout, int placement);
// Grid size launch_scan uses for `rows` rows of the layout x placement.
uint32_t scan_grid_blocks(int layout, int placement, uint64_t rows, int sm_count, int max_blocks);
// Most rows one launch may take so that no consumer thread adds more than 2^15 rows (which keeps
// its 32-bit and 64-bit partial sums exact) and per-launch sums stay below 2^31 rows.
uint64_t scan_max_rows_per_launch(int layout, int placement, uint32_t grid);

// Group-key aggregation (groupkey_kernels.cu). cols: ship, qty, disc, tax, price, key.
cudaError_t launch_groupkey(int placement, const uint8_t* const cols[6], uint64_t rows, int32_t cutoff_rel,
                            uint32_t num_groups, unsigned long long* scratch, unsigned long long* out,
                            uint32_t* status, int sm_count, int max_blocks, cudaStream_t stream);
uint64_t groupkey_scratch_bytes(uint32_t num_groups);
// High-cardinality path of the shared_mem_per_thread placement (groupkey_part.cu): a radix
// partition by key, then per-partition shared-memory slot tables. acc: num_groups x 8 u64
// (zeroed by the caller); workspace: groupkey_part_workspace_bytes(), 256-byte aligned. When
// `mode` is set, every kernel of the path returns at once unless *mode == kModePartitioned.
enum GroupKeyMode : uint32_t { kModeSinglePass = 1, kModePartitioned = 2, kModeGlobalPath = 3 };
cudaError_t launch_groupkey_part(const uint8_t* const cols[6], uint64_t rows, int32_t cutoff_rel,
                                 uint32_t num_groups, unsigned long long* acc, uint8_t* workspace,
                                 const uint32_t* mode, uint32_t* status, int sm_count, int max_blocks,
                                 cudaStream_t stream);
uint64_t groupkey_part_workspace_bytes();
// byte offset of a spare word in the workspace (the mode word of launch_groupkey)
uint64_t groupkey_part_mode_offset();
// fewest groups for which the shared placement has the partitioned path
uint32_t groupkey_part_min_groups();
cudaError_t launch_generate_keys(uint64_t seed, uint64_t first_row, uint64_t rows, uint32_t num_groups,
                                 const uint32_t* dev_cdf, uint32_t* dev_keys, cudaStream_t stream);

// lineitem text parsing (tbl_kernels.cu). tile_lines: tbl_tiles(bytes) + 1 words; after
// launch_tbl_count it holds the newlines before each 64 KB tile and, last, the total.
uint64_t tbl_tiles(uint64_t bytes);
cudaError_t launch_tbl_count(const char* text, uint64_t bytes, unsigned long long* tile_lines, cudaStream_t stream);
// bad: [malformed lines, byte offset of the first] (caller sets 0 and ~0)
cudaError_t launch_tbl_parse(const char* text, uint64_t bytes, const unsigned long long* tile_first,
                             int32_t* ship, int64_t* qty, int64_t* price, int64_t* disc, int64_t* tax, char* rf,
                             char* ls, uint64_t capacity, unsigned long long* bad, cudaStream_t stream);

// Utility kernels (util_kernels.cu).
struct GenCompressedOut {
    uint16_t* shipdate;
    uint8_t* discount;
    uint32_t* extendedprice;
    uint8_t* tax;
    uint8_t* quantity;
    uint32_t* flags;        // pair codes (may be null)
    uint32_t* returnflag;   // separate containers (may be null)
    uint32_t* linestatus;
};
cudaError_t launch_generate_compressed(uint64_t seed, uint64_t first_row, uint64_t rows, const GenCompressedOut& out,
                                       cudaStream_t stream);
// One thread waits on an mbarrier nothing completes, bounded by limit_ns; on expiry it records
// kStatusWaitTimeout in *status and returns (the bounded-wait self-test).
cudaError_t launch_wait_selftest(uint64_t limit_ns, uint32_t* status, cudaStream_t stream);
cudaError_t launch_precompute_filter(const uint16_t* shipdate, uint64_t rows, int32_t cutoff_rel, uint32_t* bitmap,
                                     cudaStream_t stream);

}  // namespace q1
