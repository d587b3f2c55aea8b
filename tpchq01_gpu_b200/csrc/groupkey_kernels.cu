// Group-key aggregation for sm_100a: the Q1 predicate and aggregates, grouped by a synthetic
// uint32 key (up to 65,536 groups) instead of the (returnflag, linestatus) pair.
//
// The per-row arithmetic is the reference's (src/kernels/ht_in_global_mem.hpp:31-49); only the
// group index changes: group = key[i] (< num_groups) instead of (rf << 1) + ls.
//
// Input tile (2048 rows): ship u16 | qty u8 | disc u8 | tax u8 | price u32 | key u32 (13 B/row),
// streamed with one cp.async.bulk per column into a 4-stage shared-memory ring exactly like the
// scan kernel (scan_kernels.cu); 8 consumer warps decode 4 rows per step (q1_keyagg.cuh).
//
// Placements:
//   in_registers_per_thread  num_groups <= 8: per-thread dp4a byte planes (PlaneRegs<4|8>)
//   shared_mem_per_thread    num_groups <= 64: shared (group, discount, tax) cells
//                            (Cube3Table); <= 1024: shared (group, discount) cells (CubeTable,
//                            3-stage ring above 768 groups); <= 4096: shared per-group slots
//                            (SlotTable, 3-stage ring above 2048 groups), or, above 4096, this
//                            kernel with keys < 4096 in
//                            slots and larger keys reduced straight into the global
//                            accumulators, or the two-pass partitioned path of
//                            groupkey_part.cu; above 256 groups the path (and the global
//                            placement's, when few rows pass over spread keys) is chosen on the
//                            device from a sample of the rows (q1_groupkey_choose)
//   global                   every passing row reduces into the global accumulators
//
// Accumulators live in scratch memory (per launch, zeroed first): per group 8 x u64 (see
// q1_keyagg.cuh); a finalize kernel folds them into the caller's int128 table [group][6] with
// 128-bit atomics (so, like the reference kernels, results accumulate into a caller-zeroed
// buffer). Launches are capped at 2^31 rows so every u64 scratch sum stays exact.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <cstring>

#include "q1_common.cuh"
#include "q1_keyagg.cuh"
#include "q1_kernels.h"
#include "q1_ptx.cuh"

namespace q1 {

using namespace ptx;

namespace gk {

constexpr uint32_t kMaxStages = 4;    // ring stages (3 when the table needs the room)
constexpr uint32_t kWideSlots = 4096; // slot-table keys of the single-pass kernel
constexpr uint32_t kChooseAbove = 256; // the shared placement's path is chosen on the device above
constexpr uint32_t kMaxDynSmem = 227 * 1024;
// Consumer warps: 16 for the shared-table and global placements, whose atomics need many warps in
// flight to hide their latency; 8 for the register planes, or 12 for four groups' planes on a large
// table (kWide: their 127 registers a thread fit the 128 that 13 warps leave, and a third warp per
// scheduler hides more of the planes' issue latency: 600 M rows 1.49 -> 1.24 ms, 80% -> 96% of HBM).
template <int P, int NG, bool kWide>
__host__ __device__ constexpr uint32_t consumer_warps() {
    return P == kPlaceInRegistersPerThread ? ((NG <= 4 && kWide) ? 12u : 8u) : 16u;
}
// Rows per tile: 2048, or 3072 with 12 warps, so that every consumer thread takes two quads of a
// tile (at most 8 rows, which the planes' flush cadence assumes).
template <int P, int NG, bool kWide>
__host__ __device__ constexpr uint32_t tile_rows() { return consumer_warps<P, NG, kWide>() == 12u ? 3072u : ka::R; }
template <int P, int NG, bool kWide>
__host__ __device__ constexpr uint32_t stage_bytes() { return ka::TileLayout<tile_rows<P, NG, kWide>()>::kStageBytes; }

// Table engine of the shared_mem_per_thread placement.
enum TableKind : uint32_t { kTableNone = 0, kTableCube = 1, kTableSlots = 2, kTableCube3 = 3 };

__host__ __device__ constexpr uint32_t table_kind(int placement, uint32_t num_groups) {
    return placement != kPlaceSharedMemPerThread
               ? kTableNone
               : (num_groups <= ka::kCube3MaxGroups ? kTableCube3
                                                    : (num_groups <= ka::kCubeMaxGroups ? kTableCube : kTableSlots));
}
__host__ __device__ constexpr uint32_t table_bytes(uint32_t kind, uint32_t num_groups) {
    return kind == kTableCube3 ? ka::cube3_bytes(num_groups)
                               : (kind == kTableCube ? ka::cube_bytes(num_groups)
                                                     : (kind == kTableSlots ? ka::slot_bytes(num_groups < kWideSlots
                                                                                                 ? num_groups
                                                                                                 : kWideSlots)
                                                                            : 0u));
}
// (tables live only beside 2048-row stages; the register planes' 3072-row stages take 4 x 39 KB)
__host__ __device__ constexpr uint32_t ring_stages(uint32_t kind, uint32_t num_groups) {
    return kMaxStages * ka::kStageBytes + table_bytes(kind, num_groups) <= kMaxDynSmem ? kMaxStages : kMaxStages - 1;
}
static_assert(kMaxStages * ka::TileLayout<3072>::kStageBytes + 512 <= kMaxDynSmem, "register-plane ring");
// the largest tables fit beside a 3-stage ring, with room left for the static shared memory
static_assert((kMaxStages - 1) * ka::kStageBytes + ka::cube_bytes(ka::kCubeMaxGroups) + 512 <= kMaxDynSmem,
              "1024-group cells");
static_assert((kMaxStages - 1) * ka::kStageBytes + ka::slot_bytes(kWideSlots) + 512 <= kMaxDynSmem, "slot table");

}  // namespace gk

struct GroupKeyParams {
    const uint8_t* col[6];          // ship, qty, disc, tax, price, key (16-byte aligned)
    uint64_t rows;
    int32_t cutoff;                 // cutoff_day - 727563
    uint32_t num_groups;
    uint32_t table;                 // gk::TableKind
    uint32_t stages;                // ring stages
    unsigned long long* acc;        // scratch: num_groups x 8 u64, zeroed
    uint32_t* status;
    const uint32_t* mode;           // when set, the kernel runs only if *mode == mode_want
    uint32_t mode_want;
};

// P: placement; NG: plane groups of in_registers_per_thread (4 or 8); kWide: 12 consumer warps
// over 3072-row tiles for four groups' planes.
template <int P, int NG, bool kWide = false>
__global__ void __launch_bounds__((gk::consumer_warps<P, NG, kWide>() + 1) * 32, 1)
    q1_groupkey_kernel(const __grid_constant__ GroupKeyParams prm) {
    using namespace gk;
    constexpr uint32_t W = consumer_warps<P, NG, kWide>();
    constexpr uint32_t R = tile_rows<P, NG, kWide>();
    constexpr uint32_t kStage = stage_bytes<P, NG, kWide>();
    constexpr uint32_t kSteps = R / 4;   // 4 rows per consumer step
    static_assert(kSteps % (W * 32) == 0 && kSteps / (W * 32) * 4 <= 8, "two quads per consumer thread at most");
    static_assert(P == kPlaceInRegistersPerThread || R == ka::R, "tables beside 2048-row stages only");
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[kMaxStages];
    __shared__ __align__(8) uint64_t empty_bar[kMaxStages];
    __shared__ __align__(8) uint64_t cons_bar;
    if (prm.mode && *prm.mode != prm.mode_want) return;   // the other path of a chosen pair runs
    const uint32_t S = prm.stages;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint64_t num_tiles = prm.rows / R;
    const uint32_t ring = smem_addr(smem);
    const uint32_t G = prm.num_groups;
    ka::Cube3Table cube3;
    ka::CubeTableT<true> cube;
    ka::SlotTable slots;
    const uint32_t hot = G < kWideSlots ? G : kWideSlots;
    if (P == kPlaceSharedMemPerThread) {
        if (prm.table == kTableCube3) cube3.bind(smem + S * kStage, G);
        else if (prm.table == kTableCube) cube.bind(smem + S * kStage, G);
        else slots.bind(smem + S * kStage, hot);
    }

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        mbar_init(smem_addr(&cons_bar), W);
        fence_mbar_init();
    }
    if (P == kPlaceSharedMemPerThread) {
        if (prm.table == kTableCube3) cube3.zero(threadIdx.x, blockDim.x);
        else if (prm.table == kTableCube) cube.zero(threadIdx.x, blockDim.x);
        else slots.zero(threadIdx.x, blockDim.x);
    }
    __syncthreads();

    if (warp == W) {
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            // stage s and phase ph of tile k, stepped rather than divided (S is a launch parameter)
            uint32_t k = 0, s = 0, ph = 0;
            for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
                if (!mbar_wait(smem_addr(&empty_bar[s]), ph ^ 1u, prm.status)) break;
                const uint32_t fb = smem_addr(&full_bar[s]);
                mbar_arrive_expect_tx(fb, kStage);
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    bulk_g2s(ring + s * kStage + ka::TileLayout<R>::col_off(c),
                             prm.col[c] + t * (uint64_t)ka::TileLayout<R>::col_bytes(c),
                             ka::TileLayout<R>::col_bytes(c), fb, pol);
                if (++s == S) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
    } else {
        const uint32_t ctid = threadIdx.x;
        ka::PlaneRegs<NG> regs;
        if (P == kPlaceInRegistersPerThread) regs.zero();
        ka::ConsumerBarrier cb{smem_addr(&cons_bar), 0};
        uint32_t bad = 0;
        uint32_t tiles_since = 0;
        uint64_t rows_since = 0;

        // one decoded quad into the placement's engine
        auto add_quad = [&](const ka::KeyQuad& x) {
            if constexpr (P == kPlaceInRegistersPerThread) {
                regs.add(x, G, prm.acc, bad);
            } else if constexpr (P == kPlaceSharedMemPerThread) {
                if (prm.table == kTableCube3) ka::table_quad(cube3, x, G, G, prm.acc, bad);
                else if (prm.table == kTableCube) ka::table_quad(cube, x, G, G, prm.acc, bad);
                else ka::table_quad(slots, x, G, hot, prm.acc, bad);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    if (!((x.PM >> (8 * r)) & 1u)) continue;
                    const uint32_t key = x.k[r];
                    if (key >= G) {
                        bad = 1u;
                        continue;
                    }
                    ka::scratch_row(prm.acc, key, (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu,
                                    (x.X >> (8 * r)) & 0xFFu, x.p[r]);
                }
            }
        };
        auto table_flush = [&]() {
            cb.sync(lane, prm.status);
            if (prm.table == kTableCube3) cube3.flush(prm.acc, G, ctid, W * 32);
            else if (prm.table == kTableCube) cube.flush(prm.acc, G, ctid, W * 32);
            else slots.flush(prm.acc, ctid, W * 32);
            cb.sync(lane, prm.status);
        };

        bool ok = true;
        uint32_t s = 0, ph = 0;   // stage and phase of the current tile
        for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x) {
            const bool landed = mbar_wait(smem_addr(&full_bar[s]), ph, prm.status);
            if (!__all_sync(0xffffffffu, landed)) {
                ok = false;
                break;
            }
            if (P == kPlaceInRegistersPerThread && tiles_since >= ka::kPlaneFlushTiles) {
                regs.flush(prm.acc, G, lane);
                tiles_since = 0;
            }
            if (P == kPlaceSharedMemPerThread && rows_since + R > ka::kTableFlushRows) {
                table_flush();
                rows_since = 0;
            }
            ++tiles_since;
            rows_since += R;
            const uint32_t base = ring + s * kStage;
#pragma unroll
            for (uint32_t it = 0; it < kSteps / (W * 32); ++it)
                add_quad(ka::load_quad<R>(base, ctid + it * (W * 32), prm.cutoff, bad));
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
            if (++s == S) {
                s = 0;
                ph ^= 1u;
            }
        }
        // the rows after the last full tile, by one CTA straight from global memory
        if (ok && blockIdx.x == (uint32_t)(num_tiles % gridDim.x) && num_tiles * R < prm.rows) {
            if (P == kPlaceSharedMemPerThread && rows_since + R > ka::kTableFlushRows) table_flush();
            // every lane runs every round (the table engines vote across the warp)
            for (uint64_t i0 = num_tiles * R; i0 < prm.rows; i0 += W * 32) {
                const uint64_t i = i0 + ctid;
                add_quad(i < prm.rows ? ka::load_row(prm.col, i, prm.cutoff, bad) : ka::empty_quad());
            }
        }
        if (bad && prm.status) atomicOr(prm.status, kStatusDomain);
        if (P == kPlaceInRegistersPerThread) regs.flush(prm.acc, G, lane);
    }
    __syncthreads();
    if (P == kPlaceSharedMemPerThread) {
        if (prm.table == kTableCube3) cube3.flush(prm.acc, G, threadIdx.x, blockDim.x);
        else if (prm.table == kTableCube) cube.flush(prm.acc, G, threadIdx.x, blockDim.x);
        else slots.flush(prm.acc, threadIdx.x, blockDim.x);
    }
}

// acc (num_groups x 8 u64) -> out[group][6] int128 (+=), quantity scaled to hundredths.
__global__ void __launch_bounds__(256) q1_groupkey_finalize(const unsigned long long* __restrict__ acc,
                                                            uint32_t num_groups, unsigned long long* out) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= num_groups) return;
    const unsigned long long* a = acc + 8ull * g;
    if (!a[0]) return;
    unsigned long long* o = out + 12ull * g;
    atomic_add_u128(o + 2 * kAggCount, a[0], 0);
    const unsigned __int128 q = (unsigned __int128)a[1] * 100u;
    atomic_add_u128(o + 2 * kAggQty, (uint64_t)q, (uint64_t)(q >> 64));
    atomic_add_u128(o + 2 * kAggBasePrice, a[3], 0);
    atomic_add_u128(o + 2 * kAggDisc, a[2], 0);
    const unsigned __int128 dp = (unsigned __int128)a[4] + ((unsigned __int128)a[5] << 32);
    atomic_add_u128(o + 2 * kAggDiscPrice, (uint64_t)dp, (uint64_t)(dp >> 64));
    const unsigned __int128 ch = (unsigned __int128)a[6] + ((unsigned __int128)a[7] << 32);
    atomic_add_u128(o + 2 * kAggCharge, (uint64_t)ch, (uint64_t)(ch >> 64));
}

template <int P, int NG, bool kWide = false>
static cudaError_t launch_gk(const GroupKeyParams& prm, int sm_count, int max_blocks, cudaStream_t st) {
    using namespace gk;
    constexpr uint32_t R = tile_rows<P, NG, kWide>();
    const uint32_t dyn = prm.stages * stage_bytes<P, NG, kWide>() + table_bytes(prm.table, prm.num_groups);
    cudaError_t e = cudaFuncSetAttribute(q1_groupkey_kernel<P, NG, kWide>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = prm.rows / R;
    uint64_t blocks = tiles ? tiles : 1;
    uint64_t cap = (uint64_t)sm_count;
    if (max_blocks > 0 && (uint64_t)max_blocks < cap) cap = (uint64_t)max_blocks;
    if (blocks > cap) blocks = cap;
    q1_groupkey_kernel<P, NG, kWide><<<(unsigned)blocks, (consumer_warps<P, NG, kWide>() + 1) * 32, dyn, st>>>(prm);
    return cudaGetLastError();
}

static uint64_t acc_bytes(uint32_t num_groups) { return 64ull * num_groups; }
// The shared placement chooses its path on the device above 256 groups.
static bool chosen_on_device(int placement, uint32_t num_groups) {
    return placement == kPlaceSharedMemPerThread && num_groups > gk::kChooseAbove;
}

// Chooses the path of the shared placement for more than 256 groups from 8192 evenly spaced
// sample rows and writes it to *mode (every path gives identical results):
//   kModeGlobalPath   every passing row straight into the global accumulators, when fewer than
//                     2% of the rows pass and no key occurs more than 3 times among the sampled
//                     passing rows (global atomics on spread keys do not contend: 1.29 ms per
//                     600 M rows at 1% pass, against 2.0 ms for the slot table; frequent keys make
//                     them contend, 11.7 ms for Zipf keys at 1% pass);
//   kModeSinglePass   the group-key kernel: keys < 4096 in a shared slot table, passing rows of
//                     larger ("cold") keys straight into the global accumulators;
//   kModePartitioned  (more than 4096 groups) the two-pass radix partition (groupkey_part.cu).
// Between the last two, a cost model fitted to both paths on a B200 (ms per 600 M rows; c =
// fraction of the rows that pass with a cold key, p = fraction that pass): single pass 2.2 + 20 c
// + 0.3 p; partitioned 1.7 + 4.3 c + 5.65 (p - c), the hot rows costing more there because skewed
// keys contend for the same ring counters and slots. The single pass wins when
// 21.35 c - 5.35 p < -0.5: skewed keys with many passing rows.
__global__ void __launch_bounds__(256) q1_groupkey_choose(const uint16_t* __restrict__ ship,
                                                          const uint32_t* __restrict__ keys, uint64_t rows,
                                                          int32_t cutoff, uint32_t hot, uint32_t allow_part,
                                                          uint32_t force, uint32_t* mode) {
    constexpr uint32_t K = 8192, kList = 512;
    if (force) {
        if (threadIdx.x == 0) *mode = force;
        return;
    }
    __shared__ uint32_t cnt[4];       // passing, cold, listed, largest key multiplicity
    __shared__ uint32_t list[kList];  // keys of the sampled passing rows
    if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
    __syncthreads();
    uint32_t pass = 0, cold = 0;
    for (uint32_t j = threadIdx.x; j < K; j += blockDim.x) {
        const uint64_t i = (uint64_t)j * rows / K;
        if ((int32_t)ship[i] <= cutoff) {
            const uint32_t key = keys[i];
            ++pass;
            cold += key >= hot ? 1u : 0u;
            const uint32_t at = atomicAdd(&cnt[2], 1u);
            if (at < kList) list[at] = key;
        }
    }
    atomicAdd(&cnt[0], pass);
    atomicAdd(&cnt[1], cold);
    __syncthreads();
    const uint32_t P = cnt[0], C = cnt[1], L = cnt[2] < kList ? cnt[2] : kList;
    const bool few = (uint64_t)P * 50 < K && cnt[2] <= kList;
    if (few) {
        for (uint32_t e = threadIdx.x; e < L; e += blockDim.x) {
            uint32_t m = 0;
            for (uint32_t x = 0; x < L; ++x) m += list[x] == list[e] ? 1u : 0u;
            atomicMax(&cnt[3], m);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (few && cnt[3] <= 3) {
            *mode = kModeGlobalPath;
        } else if (!allow_part) {
            *mode = kModeSinglePass;
        } else {
            const int64_t score = 2135ll * C - 535ll * P;   // 100 x (21.35 c - 5.35 p) x K
            *mode = score < -50ll * K ? kModeSinglePass : kModePartitioned;
        }
    }
}

cudaError_t launch_groupkey(int placement, const uint8_t* const cols[6], uint64_t rows, int32_t cutoff_rel,
                            uint32_t num_groups, unsigned long long* scratch, unsigned long long* out,
                            uint32_t* status, int sm_count, int max_blocks, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, acc_bytes(num_groups), stream);
    if (e != cudaSuccess) return e;
    uint8_t* workspace = reinterpret_cast<uint8_t*>(scratch) + ((acc_bytes(num_groups) + 255) & ~255ull);
    const bool choose = chosen_on_device(placement, num_groups);
    const bool part = num_groups >= groupkey_part_min_groups();
    uint32_t* mode = choose ? reinterpret_cast<uint32_t*>(workspace + groupkey_part_mode_offset()) : nullptr;
    // Q1_GROUPKEY_PATH=single|partitioned|global overrides the sample-based choice (tests, tuning)
    uint32_t force = 0;
    if (const char* env = std::getenv("Q1_GROUPKEY_PATH")) {
        if (!std::strcmp(env, "single")) force = kModeSinglePass;
        else if (!std::strcmp(env, "partitioned") && part) force = kModePartitioned;
        else if (!std::strcmp(env, "global")) force = kModeGlobalPath;
    }
    const uint64_t kMaxRows = 1ull << 31;
    for (uint64_t off = 0; off < rows; off += kMaxRows) {
        GroupKeyParams prm{};
        const uint64_t n = rows - off < kMaxRows ? rows - off : kMaxRows;
        const uint32_t bytes[6] = {2, 1, 1, 1, 4, 4};
        for (int c = 0; c < 6; ++c) prm.col[c] = cols[c] + off * bytes[c];
        prm.rows = n;
        prm.cutoff = cutoff_rel;
        prm.num_groups = num_groups;
        prm.table = gk::table_kind(placement, num_groups);
        prm.stages = gk::ring_stages(prm.table, num_groups);
        prm.acc = scratch;
        prm.status = status;
        if (mode) {
            q1_groupkey_choose<<<1, 256, 0, stream>>>(reinterpret_cast<const uint16_t*>(prm.col[0]),
                                                      reinterpret_cast<const uint32_t*>(prm.col[5]), n, cutoff_rel,
                                                      gk::kWideSlots, part ? 1u : 0u, force, mode);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            prm.mode = mode;
            prm.mode_want = kModeSinglePass;
            // the global path of the choice (returns at once unless chosen)
            GroupKeyParams g = prm;
            g.table = gk::kTableNone;
            g.stages = gk::kMaxStages;
            g.mode_want = kModeGlobalPath;
            if ((e = launch_gk<kPlaceGlobal, 4>(g, sm_count, max_blocks, stream)) != cudaSuccess) return e;
        }
        switch (placement) {
            case kPlaceInRegistersPerThread: {
                // The wide tiles on a table of at least 32 tiles per CTA of the grid (14.5 M rows on
                // 148 SMs): one such scan is up to 20% faster (50 M rows 136 -> 115 us), but a queue
                // of launches on tables of a few million rows ran slower with them (256 launches on
                // 10^4..5*10^7 rows: 10.72 ms with 2048-row tiles throughout, 11.56 ms with the wide
                // ones from 2 tiles per CTA, 10.78 ms from 32).
                const uint64_t grid = (max_blocks > 0 && max_blocks < sm_count) ? (uint64_t)max_blocks : (uint64_t)sm_count;
                const bool wide = n >= 32 * grid * gk::tile_rows<kPlaceInRegistersPerThread, 4, true>();
                e = num_groups > 4 ? launch_gk<kPlaceInRegistersPerThread, 8>(prm, sm_count, max_blocks, stream)
                    : wide         ? launch_gk<kPlaceInRegistersPerThread, 4, true>(prm, sm_count, max_blocks, stream)
                                   : launch_gk<kPlaceInRegistersPerThread, 4>(prm, sm_count, max_blocks, stream);
                break;
            }
            case kPlaceSharedMemPerThread: e = launch_gk<kPlaceSharedMemPerThread, 4>(prm, sm_count, max_blocks, stream); break;
            case kPlaceGlobal: e = launch_gk<kPlaceGlobal, 4>(prm, sm_count, max_blocks, stream); break;
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        if (mode && part) {
            e = launch_groupkey_part(prm.col, n, cutoff_rel, num_groups, scratch, workspace, mode, status, sm_count,
                                     max_blocks, stream);
            if (e != cudaSuccess) return e;
        }
        // fold after every 2^31-row launch so the scratch sums stay exact
        q1_groupkey_finalize<<<(num_groups + 255) / 256, 256, 0, stream>>>(scratch, num_groups, out);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (off + kMaxRows < rows) {
            e = cudaMemsetAsync(scratch, 0, acc_bytes(num_groups), stream);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// The accumulators; above 256 groups also the mode word of the shared placement's path choice,
// and above 4096 groups the partition workspace (which holds that word).
uint64_t groupkey_scratch_bytes(uint32_t num_groups) {
    const uint64_t a = (acc_bytes(num_groups) + 255) & ~255ull;
    if (num_groups >= groupkey_part_min_groups()) return a + groupkey_part_workspace_bytes();
    if (num_groups > gk::kChooseAbove) return a + 256;   // the path choice's mode word
    return acc_bytes(num_groups);
}

// Group keys of the seeded generator: uniform over [0, G) (cdf == nullptr) or by inverse CDF.
__global__ void __launch_bounds__(256) generate_keys_kernel(uint64_t key, uint64_t first_row, uint64_t rows,
                                                            uint32_t num_groups, const uint32_t* __restrict__ cdf,
                                                            uint32_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    out[i] = cdf ? gen_group_key_cdf(key, first_row + i, cdf, num_groups)
                 : gen_group_key_uniform(key, first_row + i, num_groups);
}

cudaError_t launch_generate_keys(uint64_t seed, uint64_t first_row, uint64_t rows, uint32_t num_groups,
                                 const uint32_t* dev_cdf, uint32_t* dev_keys, cudaStream_t stream) {
    if (!rows) return cudaSuccess;
    generate_keys_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(gen_key(seed), first_row, rows, num_groups,
                                                                          dev_cdf, dev_keys);
    return cudaGetLastError();
}

}  // namespace q1
