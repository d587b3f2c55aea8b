/*
 * q1.h -- C ABI of the B200-native TPC-H Query 1 filter + group-by aggregation path.
 *
 * Every entry point is plain C: integers, pointers and sizes; no C++ or torch types.
 * Every call returns a q1_status; nothing throws across this boundary.
 *
 * Each declaration names the reference interface it replaces (paths are relative to
 * the diegomestre2/tpchQ01_GPU source tree).
 *
 * Fixed-point conventions (identical to the reference CPU kernels, cpu/kernel_hyper.hpp:18-64):
 *   quantity, discount, tax      Decimal(15,2): hundredths          (cpu/tpch_kit.hpp:42-83)
 *   extendedprice                cents (hundredths)
 *   disc_price = (100 - d) * p   scale 1e-4
 *   charge = disc_price*(100+t)  scale 1e-6
 *   shipdate                     MonetDB day number (cpu/monetdb.cpp:62-78); 727563 = 1992-01-01
 * All sums are exact two's-complement 128-bit integers.
 */
#ifndef Q1_H_
#define Q1_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status codes                                                                                 */
/* ------------------------------------------------------------------------------------------ */

typedef enum q1_status {
    Q1_OK                   = 0,
    Q1_ERR_INVALID_ARGUMENT = 1,  /* bad parameter combination (src/main.cu:255-360 validation) */
    Q1_ERR_CUDA             = 2,  /* a CUDA runtime call failed; see q1_last_error()            */
    Q1_ERR_OUT_OF_MEMORY    = 3,  /* device or pinned allocation failed                          */
    Q1_ERR_NOT_LOADED       = 4,  /* q1_run before q1_load_columns                              */
    Q1_ERR_UNSUPPORTED      = 5,  /* layout / placement combination not offered                 */
    Q1_ERR_DOMAIN           = 6,  /* a value does not fit the compressed column types, or a
                                     reference-typed row's int64 products overflow (the
                                     reference's handle_overflow)                              */
    Q1_ERR_DEVICE_TIMEOUT   = 7,  /* a bounded device-side wait expired; the context stays usable */
    Q1_ERR_BUSY             = 8,  /* serving: admission refused (slots or memory budget)         */
    Q1_ERR_CPU_WORKER       = 9,  /* a coprocessing CPU worker failed                            */
    Q1_ERR_INTERNAL         = 10
} q1_status;

/* Human-readable text of the last error raised on the calling thread (never NULL). */
const char* q1_last_error(void);
/* Name of a status code. */
const char* q1_status_string(q1_status s);

/* ------------------------------------------------------------------------------------------ */
/* Constants                                                                                    */
/* ------------------------------------------------------------------------------------------ */

enum {
    Q1_NUM_POTENTIAL_GROUPS   = 6,       /* 3 return flags x 2 line stati (src/constants.hpp:56) */
    Q1_NUM_AGGREGATES         = 6,       /* count, qty, base_price, disc, disc_price, charge     */
    Q1_SHIP_DATE_FRAME        = 727563,  /* 1992-01-01 (src/constants.hpp:50)                   */
    Q1_DEFAULT_CUTOFF_DAY     = 729999,  /* 1998-12-01 minus 90 days (cpu/common.cpp:60)        */
    Q1_MAX_KEY_GROUPS         = 65536    /* group-key aggregation (synthetic uint32 key)          */
};

/* Order of the six aggregates inside one group's record of the device aggregate buffer. */
typedef enum q1_aggregate {
    Q1_AGG_COUNT          = 0,
    Q1_AGG_SUM_QTY        = 1,  /* hundredths                */
    Q1_AGG_SUM_BASE_PRICE = 2,  /* cents                     */
    Q1_AGG_SUM_DISC       = 3,  /* hundredths, sum of d      */
    Q1_AGG_SUM_DISC_PRICE = 4,  /* 1e-4                      */
    Q1_AGG_SUM_CHARGE     = 5   /* 1e-6                      */
} q1_aggregate;

/* Hash-table placements of src/main.cu:166-191 (README spelling in comments). */
typedef enum q1_placement {
    Q1_PLACEMENT_IN_REGISTERS            = 0, /* "in-registers": warp-lane tables (ht_in_registers.cuh)   */
    Q1_PLACEMENT_IN_REGISTERS_PER_THREAD = 1, /* default (ht_in_registers_per_thread.cuh)                  */
    Q1_PLACEMENT_LOCAL_MEM               = 2, /* "local-mem" (ht_in_local_mem.cuh)                          */
    Q1_PLACEMENT_SHARED_MEM_PER_THREAD   = 3, /* "per-thread-shared-mem" (ht_in_shared_mem_per_thread.cuh) */
    Q1_PLACEMENT_GLOBAL                  = 4, /* "global" (ht_in_global_mem.hpp)                           */
    Q1_NUM_PLACEMENTS                    = 5
} q1_placement;

/* Parse a placement name; accepts both the code spelling (in_registers_per_thread, local_mem,
 * shared_mem_per_thread, ...) and the README spelling (in-registers, local-mem,
 * per-thread-shared-mem, ...). Returns Q1_ERR_INVALID_ARGUMENT for unknown names. */
q1_status q1_placement_from_name(const char* name, q1_placement* out);
const char* q1_placement_name(q1_placement p);

typedef enum q1_layout {
    Q1_LAYOUT_UNCOMPRESSED = 0,  /* reference-typed columns, 38 B/row (src/data_types.h:19-25)        */
    Q1_LAYOUT_COMPRESSED   = 1   /* uint16 day offset, uint8 qty/disc/tax, uint32 cents, packed flags */
} q1_layout;

typedef enum q1_flag_packing {
    Q1_FLAGS_PAIR_2BIT = 0,      /* (returnflag, linestatus) pair dictionary, 2 bits/row: 9.25 B/row   */
    Q1_FLAGS_SEPARATE  = 1       /* returnflag 2 bits + linestatus 1 bit (src/main.cu:787-790): 9.375  */
} q1_flag_packing;

typedef enum q1_residency {
    Q1_RESIDENCY_HBM         = 0, /* columns copied once into device memory                         */
    Q1_RESIDENCY_PINNED_HOST = 1  /* columns stay in pinned host memory; every run streams them      */
} q1_residency;

/* ------------------------------------------------------------------------------------------ */
/* Column sets                                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* Uncompressed lineitem columns with the reference's element types (src/data_types.h:19-25,
 * cpu/tpch_kit.hpp:135-149). Host or device pointers depending on the call. */
typedef struct q1_columns {
    const int32_t* shipdate;       /* MonetDB day number      */
    const int64_t* discount;       /* hundredths              */
    const int64_t* extendedprice;  /* cents                   */
    const int64_t* tax;            /* hundredths              */
    const int64_t* quantity;       /* hundredths              */
    const char*    returnflag;     /* 'A' | 'N' | 'R'         */
    const char*    linestatus;     /* 'F' | 'O'               */
} q1_columns;

/* Compressed columns (src/main.cu:773-803, namespace compressed in src/data_types.h:37-44).
 * Bit containers are uint32 words, element i at word i/(32/b), bit b*(i%(32/b)), LSB first
 * (src/bit_operations.hpp:60-154). */
typedef struct q1_compressed_columns {
    const uint16_t* shipdate;      /* day - 727563, at most 32767 (dates up to 2081-09-19)      */
    const uint8_t*  discount;      /* hundredths, 0..100                                        */
    const uint32_t* extendedprice; /* cents                                                     */
    const uint8_t*  tax;           /* hundredths                                                */
    const uint8_t*  quantity;      /* whole units (reference divides by 100, src/main.cu:783)   */
    const uint32_t* flags;         /* Q1_FLAGS_PAIR_2BIT: 2-bit pair codes                      */
    const uint32_t* returnflag;    /* Q1_FLAGS_SEPARATE: 2-bit codes A=0 N=1 R=2               */
    const uint32_t* linestatus;    /* Q1_FLAGS_SEPARATE: 1-bit codes F=0 O=1                   */
    const uint32_t* filter;        /* optional precomputed predicate bitmap, 1 bit/row          */
    int32_t         flag_packing;  /* q1_flag_packing                                           */
    uint32_t        num_pair_codes;/* PAIR_2BIT: number of dictionary entries (1..4)            */
    uint8_t         pair_group[4]; /* PAIR_2BIT: code -> group index (rf_code<<1 | ls_code)     */
} q1_compressed_columns;

/* Column statistics produced by the compressor (the analogue of cpu/tpch_kit.hpp:95-108 MinMax). */
typedef struct q1_column_stats {
    uint64_t rows;
    int32_t  min_shipdate, max_shipdate;
    uint32_t max_quantity, max_discount, max_tax;
    uint32_t max_extendedprice;
    uint32_t num_pair_codes;
    uint8_t  pair_group[4];
    uint32_t group_present_mask;   /* bit g set if group g occurs */
} q1_column_stats;

/* Host-side compressor: reference-typed columns -> compressed columns (src/main.cu:773-803).
 * Output buffers are caller-owned host memory: shipdate[rows], discount[rows], tax[rows],
 * quantity[rows], extendedprice[rows]; for PAIR_2BIT flags[ceil(rows/16)];
 * for SEPARATE returnflag[ceil(rows/16)] and linestatus[ceil(rows/32)].
 * Fails with Q1_ERR_DOMAIN if a value does not fit (the reference asserts at :789-800);
 * in addition discount must be <= 100 and quantity a whole number of units. */
typedef struct q1_compressed_host_out {
    uint16_t* shipdate;
    uint8_t*  discount;
    uint32_t* extendedprice;
    uint8_t*  tax;
    uint8_t*  quantity;
    uint32_t* flags;
    uint32_t* returnflag;
    uint32_t* linestatus;
} q1_compressed_host_out;

q1_status q1_compress_host(const q1_columns* in, uint64_t rows, q1_flag_packing packing,
                           const q1_compressed_host_out* out, q1_column_stats* stats);

/* Filter precomputation: bitmap[i/32] bit i%32 = (shipdate[i] <= cutoff - 727563)
 * (src/main.cu:362-389). Host version writes ceil(rows/32) words. */
q1_status q1_precompute_filter_host(const uint16_t* shipdate, uint64_t rows, int32_t cutoff_day,
                                    uint32_t* bitmap);

/* ------------------------------------------------------------------------------------------ */
/* Results                                                                                      */
/* ------------------------------------------------------------------------------------------ */

/* Two's-complement 128-bit integer. */
typedef struct q1_i128 {
    uint64_t lo;
    uint64_t hi;
} q1_i128;

typedef struct q1_group_result {
    int32_t  group;            /* rf_code<<1 | ls_code (src/kernels/ht_in_global_mem.hpp:41-42) */
    char     returnflag;       /* decoded 'A' 'N' 'R'                                          */
    char     linestatus;       /* decoded 'F' 'O'                                              */
    uint64_t count;
    q1_i128  sum_qty;          /* hundredths */
    q1_i128  sum_base_price;   /* cents      */
    q1_i128  sum_disc;         /* hundredths */
    q1_i128  sum_disc_price;   /* 1e-4       */
    q1_i128  sum_charge;       /* 1e-6       */
    /* Averages from the exact sums, C integer division (truncation toward zero) as in
     * Decimal64::GetInt/GetFrac (cpu/tpch_kit.hpp:54-60), each carrying two extra decimals:
     * avg_qty = sum_qty*100/count (1e-4 units), likewise avg_price and avg_disc. 0 if count==0. */
    int64_t  avg_qty_e4;
    int64_t  avg_price_e4;
    int64_t  avg_disc_e4;
} q1_group_result;

typedef struct q1_result {
    uint32_t        num_groups;     /* always Q1_NUM_POTENTIAL_GROUPS                  */
    q1_group_result groups[Q1_NUM_POTENTIAL_GROUPS];
    uint64_t        rows_total;
    uint64_t        rows_gpu;       /* rows aggregated on the GPU                      */
    uint64_t        rows_cpu;       /* rows aggregated by the coprocessing CPU share   */
    double          ms_last_run;    /* wall-clock of the last run (src/main.cu:893-905) */
    double          ms_gpu_last_run;/* CUDA-event time of the GPU part of the last run */
} q1_result;

/* Convert a device aggregate buffer (num_groups records of Q1_NUM_AGGREGATES q1_i128, laid out
 * [group][aggregate]) into per-group results with averages. */
q1_status q1_finalize_groups(const q1_i128* aggregates_host, uint32_t num_groups,
                             q1_group_result* out);

/* ------------------------------------------------------------------------------------------ */
/* Query context: the reference's tpch_01 driver (src/main.cu:738-916) as a library             */
/* ------------------------------------------------------------------------------------------ */

typedef struct q1_ctx q1_ctx;

typedef struct q1_device_opts {
    int32_t device;          /* CUDA device ordinal (the reference always uses the current one) */
    int32_t cpu_threads;     /* coprocessing pool size; 0 = hardware_concurrency/2 - 1
                                (cpu/kernel_x100.hpp:535-548 with wo_core0 = true)              */
} q1_device_opts;

/* Replaces main()'s device setup (src/main.cu:738-878). */
q1_status q1_open(q1_ctx** ctx, const q1_device_opts* opts);
q1_status q1_close(q1_ctx* ctx);

/* Load a table. Replaces load_table_columns_from_files + the compression loop + device
 * allocation (src/main.cu:391-476, :773-878). `layout` selects what the GPU scans:
 * UNCOMPRESSED keeps the reference-typed columns, COMPRESSED runs q1_compress_host first.
 * HBM residency copies the columns to device memory once; PINNED_HOST keeps them in pinned
 * host memory and every run streams them chunk by chunk (src/main.cu:567-719). */
q1_status q1_load_columns(q1_ctx* ctx, const q1_columns* host_columns, uint64_t rows,
                          q1_layout layout, q1_flag_packing packing, q1_residency residency);

/* Load already-compressed host columns (e.g. a column cache) without recompressing. */
q1_status q1_load_compressed(q1_ctx* ctx, const q1_compressed_columns* host_columns,
                             uint64_t rows, q1_residency residency);

/* Generate `rows` rows of the seeded synthetic lineitem generator into the context, starting at
 * row index `first_row` (a multiple of 32). Compressed tables are generated on the device: for
 * HBM residency straight into place, for PINNED_HOST residency chunk by chunk and copied into
 * pinned host memory. Uncompressed tables are generated on the host and loaded. */
q1_status q1_generate_table(q1_ctx* ctx, uint64_t seed, uint64_t first_row, uint64_t rows,
                            q1_layout layout, q1_flag_packing packing, q1_residency residency);

/* Run parameters: mirror of q1_params_t (src/main.cu:205-240). */
typedef struct q1_params {
    int32_t placement;            /* q1_placement; --hash-table-placement                        */
    int32_t apply_compression;    /* --apply-compression: must match the loaded layout          */
    int32_t use_filter_pushdown;  /* --use-filter-pushdown (requires compression)               */
    int32_t use_coprocessing;     /* --use-coprocessing                                          */
    double  cpu_fraction;         /* --cpu-fraction, 0..1 (default 0.5)                          */
    int32_t streams;              /* --streams (default 4)                                        */
    int32_t threads_per_block;    /* --threads-per-block, multiple of 32; 0 = tuned default     */
    int32_t tuples_per_thread;    /* --tuples-per-thread; 0 = tuned default                     */
    int64_t tuples_per_launch;    /* --tuples-per-kernel-launch (default 1<<21)                 */
    int32_t runs;                 /* --runs (default 5); q1_run executes this many times        */
    int32_t cutoff_day;           /* WHERE l_shipdate <= cutoff_day (default 729999)           */
} q1_params;

/* Fill with the reference defaults (src/constants.hpp:7-40). */
void q1_params_default(q1_params* p);

/* Validate like parse_command_line (src/main.cu:325-358). */
q1_status q1_params_validate(const q1_params* p);

/* Device (or, for PINNED_HOST residency, pinned host) column pointers of the loaded table, for
 * use with the kernel-level calls below. Exactly one of the two views is filled, by layout. */
q1_status q1_table_columns(q1_ctx* ctx, q1_compressed_columns* compressed, q1_columns* uncompressed,
                           uint64_t* rows, q1_layout* layout, q1_residency* residency);

/* Column statistics of the loaded table. */
q1_status q1_table_stats(q1_ctx* ctx, q1_column_stats* stats);

/* Wall-clock and GPU times (ms) of the runs of the last q1_run (src/main.cu:881-905 writes the
 * wall-clock ones to results.csv). */
q1_status q1_run_times(q1_ctx* ctx, double* wall_ms, double* gpu_ms, int32_t capacity, int32_t* count);

/* Execute the query `runs` times (src/main.cu:893-905 loop, execute_query_1_once :498-736).
 * The result of the last run is written to `out`. */
q1_status q1_run(q1_ctx* ctx, const q1_params* p, q1_result* out);

/* ------------------------------------------------------------------------------------------ */
/* Kernel-level ABI: the reference's __global__ kernels (src/kernels/) launched on caller-owned */
/* device memory. Aggregates accumulate into a caller-zeroed buffer of                          */
/* Q1_NUM_POTENTIAL_GROUPS * Q1_NUM_AGGREGATES q1_i128 ([group][aggregate]), just as the         */
/* reference kernels atomicAdd into caller-zeroed arrays.                                      */
/* ------------------------------------------------------------------------------------------ */

typedef struct q1_launch_config {
    int32_t threads_per_block;   /* 0 = tuned default */
    int32_t tuples_per_thread;   /* 0 = tuned default */
    int32_t blocks;              /* 0 = tuned default (multiple of the SM count) */
} q1_launch_config;

/* Replaces the kernels_compressed / kernels_filter_pushdown tables (src/main.cu:175-191):
 * K2, K3, K5, K6, K8, K9, K11, K12, K14, K15. `use_filter` reads cols->filter instead of
 * cols->shipdate. `status_word` (device, may be NULL) receives a nonzero code if a bounded
 * device wait expired. */
q1_status q1_launch_compressed(q1_placement placement, const q1_compressed_columns* dev_cols,
                               uint64_t rows, int32_t cutoff_day, int32_t use_filter,
                               const q1_launch_config* cfg, q1_i128* dev_aggregates,
                               void* cuda_stream);

/* Allocation-free variant of q1_launch_compressed (no counterpart in the reference).
 * For callers that must not allocate device memory: a host that owns every byte of device
 * memory through its own pool or runs under a hard memory cap, or a latency-critical loop in
 * which cudaMalloc/cudaFree must never run. q1_launch_compressed allocates a small status word on
 * first use of a device; this call allocates nothing. Its scratch is a static device array of
 * 147,712 bytes that every GPU loading the library holds until exit: a status word plus one
 * partial-sum record per CTA, which a second kernel adds into dev_aggregates (accumulating, like
 * q1_launch_compressed). Limit: at most 256 CTAs per launch (one per SM is used by default, 148
 * on a B200); larger grids are rejected with Q1_ERR_INVALID_ARGUMENT. The first call on a device,
 * and the first after that device's context was reset, looks up the array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture. The call is
 * synchronous: it waits for
 * `cuda_stream` and returns Q1_ERR_DOMAIN / Q1_ERR_DEVICE_TIMEOUT itself. All calls share the
 * array, so calls whose GPU work overlaps (other threads or streams of the same device) race. */
q1_status q1_launch_compressed_noalloc(q1_placement placement, const q1_compressed_columns* dev_cols,
                                       uint64_t rows, int32_t cutoff_day, int32_t use_filter,
                                       const q1_launch_config* cfg, q1_i128* dev_aggregates,
                                       void* cuda_stream);

/* Replaces the kernels table (src/main.cu:166-173): K1, K4, K7, K10, K13. Takes any int64
 * values, like the reference's CPU kernels: rows in the fast domain (discount 0..100, tax 0..255,
 * quantity and price 0..2^32-1) are summed by the placement's tables, any other passing row
 * exactly by a signed 128-bit path; a passing row whose int64 products overflow is reported as
 * Q1_ERR_DOMAIN by q1_sync_check (KernelHyPer's handle_overflow, cpu/kernel_hyper.hpp:65-91). */
q1_status q1_launch_uncompressed(q1_placement placement, const q1_columns* dev_cols,
                                 uint64_t rows, int32_t cutoff_day,
                                 const q1_launch_config* cfg, q1_i128* dev_aggregates,
                                 void* cuda_stream);

/* The kernel-level calls are asynchronous. This synchronises `cuda_stream` and converts the
 * current device's kernel status word (bounded-wait expiry, out-of-domain rows) into a status
 * code, clearing it. Replaces the reference's reliance on cuda-api-wrappers exceptions. */
q1_status q1_sync_check(void* cuda_stream);

/* ------------------------------------------------------------------------------------------ */
/* Group-key aggregation: the same predicate and aggregates, grouped by a uint32 key column     */
/* (key < num_groups <= Q1_MAX_KEY_GROUPS) instead of (returnflag, linestatus). Generalises the  */
/* reference's 6-entry group table (src/constants.hpp:56) to many groups.                      */
/* ------------------------------------------------------------------------------------------ */

/* Bytes of device scratch q1_launch_groupkey needs for num_groups groups: 64 per group, plus 256
 * above 256 groups and about 1.1 GB of partition workspace above 4096 groups (independent of
 * the row count). */
uint64_t q1_groupkey_scratch_bytes(uint32_t num_groups);

/* Placements: IN_REGISTERS_PER_THREAD (num_groups <= 8; per-thread byte-plane sums),
 * SHARED_MEM_PER_THREAD (per-CTA shared-memory tables: (group, discount, tax) cells for
 * num_groups <= 64, (group, discount) cells for <= 1024, one slot per group for <= 4096; above
 * 256 groups a kernel reads 8192 sample rows and picks on the device the shared-table pass (keys
 * >= 4096 into global atomics), the global path (few passing rows over spread keys) or, above
 * 4096 groups, a two-pass radix partition of the passing rows into 8-byte records, 2^27 rows at
 * a time, aggregated per 4096-key partition in a shared slot table; every path gives the same
 * result), GLOBAL (global atomics for every row). Reads ship, qty, disc, tax, price of dev_cols
 * and dev_keys; the result accumulates into dev_aggregates[num_groups][6] (caller-zeroed
 * int128). dev_scratch: device memory of q1_groupkey_scratch_bytes(num_groups), owned by the
 * caller; calls on different streams need different scratch. A key >= num_groups in a passing
 * row is reported as Q1_ERR_DOMAIN by q1_sync_check. */
q1_status q1_launch_groupkey(q1_placement placement, const q1_compressed_columns* dev_cols,
                             const uint32_t* dev_keys, uint32_t num_groups, uint64_t rows,
                             int32_t cutoff_day, const q1_launch_config* cfg, void* dev_scratch,
                             q1_i128* dev_aggregates, void* cuda_stream);

/* Zipf(s) inverse-CDF thresholds over ranks 1..num_groups (key = rank - 1): cdf[k] =
 * floor(2^32 * P(rank <= k+1)), clamped to 0xFFFFFFFF, last entry 0xFFFFFFFF. */
q1_status q1_zipf_cdf(uint32_t num_groups, double s, uint32_t* cdf_out);

/* Group keys of the seeded generator for rows [first_row, first_row+rows): uniform over
 * [0, num_groups) if dev_cdf is NULL, else the smallest k with bits <= dev_cdf[k]. */
q1_status q1_generate_group_keys_device(uint64_t seed, uint64_t first_row, uint64_t rows,
                                        uint32_t num_groups, const uint32_t* dev_cdf,
                                        uint32_t* dev_keys, void* cuda_stream);

/* ------------------------------------------------------------------------------------------ */
/* Batched aggregation: many independent group-key instances (each its own table, cutoff and    */
/* group count) in one persistent kernel over a device work queue of row tiles, replayed as a   */
/* CUDA graph. Replaces one launch per instance (the reference launches one kernel per chunk,   */
/* src/main.cu:567-719). Results equal q1_launch_groupkey's for every instance, bit for bit.    */
/* ------------------------------------------------------------------------------------------ */

typedef struct q1_batch_instance {
    q1_compressed_columns cols;   /* device: shipdate, discount, extendedprice, tax, quantity   */
    const uint32_t* keys;         /* device group keys, < num_groups                            */
    uint64_t rows;
    int32_t  cutoff_day;
    uint32_t num_groups;          /* 1..65536                                                   */
    q1_i128* aggregates;          /* device [num_groups][6] result table                        */
} q1_batch_instance;

typedef struct q1_batch_opts {
    int32_t use_graph;            /* capture one execution as a CUDA graph and replay it        */
    int32_t accumulate;           /* 0: each run overwrites the result tables; 1: adds to them  */
    int32_t chunk_tiles;          /* work-item size in 2048-row tiles; 0 = heuristic / tuner    */
    int32_t tune;                 /* 0 heuristic placements; 1 autotune, reuse the cache file;
                                     2 autotune and re-measure every class                      */
    const char* tune_cache;       /* autotuner cache file (NULL: kept in memory only)           */
} q1_batch_opts;

typedef struct q1_batch_desc {
    uint32_t instances, items, chunk_tiles, tile_rows, grid, uses_graph, tuned_classes;
    uint32_t mode_count[3];       /* instances per placement: registers, shared table, global  */
    uint64_t total_rows, total_groups;
} q1_batch_desc;

typedef struct q1_batch q1_batch;

/* Build a batch (descriptors, work queue, scratch; autotuning runs here, on cuda_stream). The
 * instance arrays must stay valid while the batch is used. */
q1_status q1_batch_create(const q1_batch_instance* instances, uint32_t n, const q1_batch_opts* opts,
                          void* cuda_stream, q1_batch** out);
/* One execution of every instance (asynchronous; q1_sync_check reports device errors). */
q1_status q1_batch_run(q1_batch* b, void* cuda_stream);
q1_status q1_batch_describe(q1_batch* b, q1_batch_desc* out);
/* Placement chosen for instance i: 0 registers (num_groups <= 4), 1 shared table, 2 global. */
q1_status q1_batch_instance_mode(q1_batch* b, uint32_t i, int32_t* mode);
q1_status q1_batch_destroy(q1_batch* b);

/* Device filter precomputation (GPU version of src/main.cu:362-389). */
q1_status q1_precompute_filter(const uint16_t* dev_shipdate, uint64_t rows, int32_t cutoff_day,
                               uint32_t* dev_bitmap, void* cuda_stream);

/* ------------------------------------------------------------------------------------------ */
/* Binary column cache: the reference's on-disk format (src/file_access.hpp:19-61, written and  */
/* read by src/main.cu:405-474). A directory holds one raw native-endian array per column:     */
/* shipdate.bin (int32 day numbers), returnflag.bin, linestatus.bin (char), discount.bin,       */
/* tax.bin, extendedprice.bin, quantity.bin (int64 hundredths / cents).                          */
/* ------------------------------------------------------------------------------------------ */

/* Writable reference-typed host columns (the output side of q1_columns). */
typedef struct q1_columns_out {
    int32_t* shipdate;
    char*    returnflag;
    char*    linestatus;
    int64_t* discount;
    int64_t* tax;
    int64_t* extendedprice;
    int64_t* quantity;
} q1_columns_out;

/* Writes `rows` rows of host columns as a cache directory (created if missing). */
q1_status q1_cache_write(const char* dir, const q1_columns* host_columns, uint64_t rows);

/* Rows of a cache directory: shipdate.bin's size / 4, every other file checked against it
 * (Q1_ERR_INVALID_ARGUMENT on a missing or mis-sized file). Unlike src/main.cu:412-414, an
 * SF-1-sized cache is never rescaled by a scale factor. */
q1_status q1_cache_rows(const char* dir, uint64_t* rows);

/* Reads a cache directory of exactly `rows` rows into caller-owned host columns. */
q1_status q1_cache_read(const char* dir, uint64_t rows, q1_columns_out* out);

/* Loads a cache directory into the context (compressing it when layout is COMPRESSED), like
 * q1_load_columns; the row count is returned in rows_out (may be NULL). */
q1_status q1_cache_load(q1_ctx* ctx, const char* dir, q1_layout layout, q1_flag_packing packing,
                        q1_residency residency, uint64_t* rows_out);

/* ------------------------------------------------------------------------------------------ */
/* lineitem text (dbgen .tbl) ingestion on the GPU: replaces lineitem::FromFile                 */
/* (cpu/tpch_kit.cpp:155-172, TableReader at :10-99), which the reference runs when no column   */
/* cache exists (src/main.cu:441-475). One row per '\n'-terminated line (the last '\n' may be    */
/* missing), fields separated by '|'; fields 5-11 are read: quantity, extendedprice, discount,  */
/* tax as "[+-]int[.frac]" -> 100*int + frac (Decimal<15,2>), returnflag and linestatus as one  */
/* character, shipdate as "year-month-day" -> MonetDB day number (Date, monetdb.cpp todate).    */
/* ------------------------------------------------------------------------------------------ */

/* Rows in a device text buffer (16-byte aligned for full speed). Synchronous on cuda_stream. */
q1_status q1_tbl_count_device(const char* dev_text, uint64_t bytes, uint64_t* rows, void* cuda_stream);

/* Parses a device text buffer into reference-typed device columns of `capacity` rows (row i =
 * line i). Synchronous; *rows_out = the rows in the text. Q1_ERR_INVALID_ARGUMENT when the text
 * holds more rows than `capacity` or has malformed lines (their count and the first one's byte
 * offset in q1_last_error(); those rows are written as zeros). */
q1_status q1_tbl_parse_device(const char* dev_text, uint64_t bytes, const q1_columns_out* dev_out,
                              uint64_t capacity, uint64_t* rows_out, void* cuda_stream);

/* Reads a .tbl file through the GPU parser (256 MB chunks of whole lines, on the current
 * device) into caller-owned host columns of `capacity` rows; out == NULL only counts the rows. */
q1_status q1_tbl_read_file(const char* path, q1_columns_out* out, uint64_t capacity, uint64_t* rows_out);

/* Loads a .tbl file into the context like q1_load_columns (src/main.cu:441-475). */
q1_status q1_tbl_load(q1_ctx* ctx, const char* path, q1_layout layout, q1_flag_packing packing,
                      q1_residency residency, uint64_t* rows_out);

/* Writes host columns as .tbl text (the inverse of the parser, two decimals per value, ISO
 * dates); the fields Q1 does not read get deterministic placeholders derived from
 * first_row + i. buf == NULL: only *bytes_out (the text's size) is set. Multi-threaded. */
q1_status q1_tbl_format(const q1_columns* host_columns, uint64_t first_row, uint64_t rows, char* buf,
                        uint64_t capacity, uint64_t* bytes_out);

/* ------------------------------------------------------------------------------------------ */
/* Synthetic data generator (stands in for dbgen, scripts/genlineitem.sh)                       */
/* ------------------------------------------------------------------------------------------ */

/* Host generator: rows [first_row, first_row+rows) of the seeded counter-based generator into
 * reference-typed columns. Any NULL output column is skipped. */
q1_status q1_generate_host(uint64_t seed, uint64_t first_row, uint64_t rows, q1_columns* out);

/* Device generator writing compressed columns into caller-owned device buffers sized as for
 * q1_compress_host; the pair dictionary is fixed to {AF, NF, NO, RF}. `stats` may be NULL. */
q1_status q1_generate_compressed_device(uint64_t seed, uint64_t first_row, uint64_t rows,
                                        q1_flag_packing packing,
                                        const q1_compressed_host_out* dev_out,
                                        void* cuda_stream);

/* ------------------------------------------------------------------------------------------ */
/* Serving: a request loop with continuous batching. No reference counterpart: the reference    */
/* answers one query per process run (src/main.cu:520-760); its per-query path stays available  */
/* as q1_server_plain, and every served response equals it bit for bit.                          */
/*                                                                                              */
/* The server keeps one resident table in HBM (the seeded generator's rows, compressed, plus a   */
/* uint32 key column uniform over Q1_SERVE_RESIDENT_KEY_GROUPS groups) together with its partial */
/* aggregates per ship day (cumulative over days, per (returnflag, linestatus) group and per key */
/* group), so a resident request is answered from those without a scan. Ad-hoc requests name a  */
/* table of their own: adhoc_rows rows of the generator under adhoc_seed with its grouping. It   */
/* is generated on the device into an arena of hbm_budget_bytes on first use and stays there     */
/* (least recently used tables not in use are evicted when a new one does not fit). A dispatcher */
/* thread forms rounds from the queue (FIFO) while a slot is free and the next request's table   */
/* is or can be made resident; one round = missing tables generated, all ad-hoc requests of the */
/* round aggregated together in one persistent batch launch, resident answers looked up, all     */
/* responses copied back. Requests that arrive during a round join the next one.                */
/* Q1_SERVE_PLAIN runs the same loop with one request per round through the plain launch.       */
/* ------------------------------------------------------------------------------------------ */

#define Q1_SERVE_MAX_GROUPS 64
#define Q1_SERVE_RESIDENT_KEY_GROUPS 64

typedef enum q1_request_kind {
    Q1_REQ_RESIDENT = 0,   /* query the server's resident table */
    Q1_REQ_ADHOC    = 1    /* query a table of adhoc_rows rows generated under adhoc_seed */
} q1_request_kind;

typedef enum q1_grouping {
    Q1_GROUP_FLAGS = 0,    /* group by (l_returnflag, l_linestatus): 6 slots, 4 live (the Q1 grouping) */
    Q1_GROUP_KEYS  = 1     /* group by a uniform synthetic key in [0, num_groups) */
} q1_grouping;

typedef struct q1_request {
    int32_t  kind;          /* q1_request_kind */
    int32_t  grouping;      /* q1_grouping */
    uint32_t num_groups;    /* Q1_GROUP_KEYS: 1..64 (resident: exactly 64); ignored for FLAGS */
    int32_t  cutoff_day;    /* l_shipdate <= cutoff_day (day number) */
    uint64_t adhoc_rows;    /* Q1_REQ_ADHOC: (adhoc_seed, adhoc_rows, grouping, num_groups) */
    uint64_t adhoc_seed;    /* name the table; keys come from the same seed */
} q1_request;

typedef struct q1_response {
    uint64_t ticket;
    int32_t  status;        /* q1_status of the request */
    uint32_t num_groups;    /* group slots filled: 6 (FLAGS) or num_groups (KEYS) */
    double   latency_ms;    /* submission -> response ready */
    double   queue_ms;      /* submission -> admission into a round */
    /* [group][6]: count, sum_qty (hundredths), sum_base_price, sum_disc, sum_disc_price,
     * sum_charge, the int128 table of q1_launch_groupkey */
    q1_i128  aggregates[Q1_SERVE_MAX_GROUPS * 6];
} q1_response;

typedef enum q1_serve_mode {
    Q1_SERVE_BATCHED = 0,   /* continuous batching into rounds */
    Q1_SERVE_PLAIN   = 1    /* one request per round, one plain launch each (the comparison) */
} q1_serve_mode;

typedef struct q1_server_opts {
    int32_t  device;
    uint32_t max_inflight;       /* requests per round (response slots of a round lane) */
    int32_t  mode;               /* q1_serve_mode */
    uint32_t max_rounds_in_flight;  /* round lanes: rounds on the GPU at once, 1..8 (0 = 2);
                                       Q1_SERVE_PLAIN always runs one */
    uint64_t seed;               /* resident table seed */
    uint64_t resident_rows;      /* rows of the resident table */
    uint64_t hbm_budget_bytes;   /* arena of resident ad-hoc tables (13 B per row + alignment) */
    uint64_t max_adhoc_rows;     /* larger ad-hoc requests are refused at submission */
} q1_server_opts;

typedef struct q1_server_stats {
    uint64_t completed;
    uint64_t failed;
    uint64_t rounds;
    uint64_t pending;            /* submitted, not yet admitted */
    uint64_t logical_rows;       /* rows of all completed requests' tables */
    uint64_t scanned_rows;       /* rows actually scanned (ad-hoc tables) */
    uint64_t generated_rows;     /* ad-hoc rows generated (table cache misses) */
    uint64_t cache_hits, cache_misses, evictions;
    uint64_t cached_tables, cached_bytes;
    double   wall_ms;            /* first completed request's submission -> last completion */
    double   mean_round_size;
    double   p50_ms, p90_ms, p99_ms, max_ms, mean_ms;   /* latency of completed requests */
    uint64_t overlapped_rounds;  /* rounds enqueued while another round was on the GPU */
    uint32_t max_rounds_in_flight;  /* most rounds on the GPU at once */
    uint32_t reserved;
} q1_server_stats;

typedef struct q1_server q1_server;

/* Defaults: device 0, 256 slots, batched, seed 20260104, 600M resident rows, 120 GiB budget,
 * 100M rows per ad-hoc table. */
void q1_server_opts_default(q1_server_opts* opts);

/* Builds the resident table and its per-day aggregates on the device, allocates the arena and
 * starts the dispatcher. */
q1_status q1_server_open(const q1_server_opts* opts, q1_server** out);

/* Queues a request. Q1_ERR_INVALID_ARGUMENT for a malformed request, Q1_ERR_BUSY when its
 * table can never fit the budget. Thread-safe. */
q1_status q1_server_submit(q1_server* server, const q1_request* req, uint64_t* ticket);

/* Waits for a ticket (timeout_ms < 0: no limit; Q1_ERR_BUSY on expiry, the ticket stays
 * valid) and releases it into `out`. Thread-safe. */
q1_status q1_server_wait(q1_server* server, uint64_t ticket, int32_t timeout_ms, q1_response* out);

q1_status q1_server_stats_get(q1_server* server, q1_server_stats* out);
q1_status q1_server_reset_stats(q1_server* server);

/* The plain path for one request: one scan launch over its table (q1_launch_compressed for
 * resident FLAGS requests, q1_launch_groupkey otherwise; ad-hoc FLAGS tables are generated in
 * the compressed pair layout for it), synchronous, on a stream of its own. The arbiter of every
 * served response. */
q1_status q1_server_plain(q1_server* server, const q1_request* req, q1_response* out);

/* Device pointers to the resident table (pair layout) and its key column. */
q1_status q1_server_resident_columns(q1_server* server, q1_compressed_columns* cols,
                                     const uint32_t** dev_keys, uint64_t* rows);

/* Finishes queued requests, stops the dispatcher and frees everything. */
q1_status q1_server_close(q1_server* server);

/* ------------------------------------------------------------------------------------------ */
/* Failure detection. No reference counterpart (the reference exits on any error,                */
/* src/main.cu:260-339). Faults are injected on the host; the device side is exercised by a wait */
/* that nothing completes, bounded like every wait of the kernels.                              */
/* ------------------------------------------------------------------------------------------ */

typedef enum q1_fault {
    Q1_FAULT_NONE         = 0,   /* clears every pending fault */
    Q1_FAULT_CPU_WORKER   = 1,   /* the next CPU pool jobs raise (Q1_ERR_CPU_WORKER from q1_run) */
    Q1_FAULT_DEVICE_ALLOC = 2,   /* the next context, .tbl reader and server device allocations fail
                                    (Q1_ERR_OUT_OF_MEMORY) */
    Q1_FAULT_PINNED_ALLOC = 3,   /* the next context, .tbl reader and server pinned host allocations fail */
    Q1_FAULT_SERVE_ROUND  = 4    /* the next serving rounds fail to enqueue (Q1_ERR_INTERNAL): the
                                    server fails that round, the rounds behind it and every queued
                                    request, and refuses later submissions */
} q1_fault;

/* Makes the next `count` events of `kind` fail (process-wide; for tests of error paths). */
q1_status q1_inject_fault(q1_fault kind, uint32_t count);

/* Launches one thread that waits on an mbarrier nothing completes, bounded by limit_us
 * (1 us .. 2 s): the wait expires, the kernel records the timeout in the device status word and
 * returns, and q1_sync_check(cuda_stream) then reports Q1_ERR_DEVICE_TIMEOUT with the context
 * still usable. */
q1_status q1_selftest_wait_timeout(uint32_t limit_us, void* cuda_stream);

/* Runs the coprocessing mode's CPU share (the host kernel q1_run gives its CPU fraction) on the
 * calling thread over rows [begin, end) of compressed columns in HOST memory (the filter field is
 * not used), adding into aggregates[6][6] (int128, caller-zeroed; same layout as q1_result's
 * sums, quantity in hundredths). Returns Q1_ERR_DOMAIN when a passing row is outside the kernels'
 * domain. Needs no GPU; for tests of the host kernel. */
q1_status q1_selftest_cpu_share(const q1_compressed_columns* host_cols, uint64_t begin, uint64_t end,
                                int32_t cutoff_day, void* aggregates);
/* The same for reference-typed (uncompressed) columns in host memory: any int64 values, summed
 * exactly; Q1_ERR_DOMAIN when a passing row's int64 products overflow. */
q1_status q1_selftest_cpu_share_uncompressed(const q1_columns* host_cols, uint64_t begin, uint64_t end,
                                             int32_t cutoff_day, void* aggregates);

/* Reads `bytes` of host memory at host_buf on `threads` host threads (a contiguous slice each,
 * 16-byte vector loads reduced into a value that is kept) and returns the rate in *gb_per_s
 * (bytes / wall time, 1e9 bytes per GB). A measurement helper with no reference counterpart: the
 * host-streamed mode (PINNED_HOST residency, coprocessing) reads every row from host memory, on
 * the CPU share's cores or by the GPU's copy engines, so this read rate bounds it next to the
 * PCIe copy rate. Needs no GPU. */
q1_status q1_measure_host_read(const void* host_buf, uint64_t bytes, int32_t threads, double* gb_per_s);

/* One-line description of a CUDA device (name, compute capability, SMs, memory, L2) into buf.
 * Replaces get_device_properties / --device (src/helper.hpp:18-48, src/main.cu:266-268). */
q1_status q1_device_describe(int32_t device, char* buf, size_t buf_len);

/* Library version string. */
const char* q1_version(void);

#ifdef __cplusplus
}
#endif

#endif /* Q1_H_ */
