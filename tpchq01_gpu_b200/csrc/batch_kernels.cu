// Batched Q1 aggregation: many independent instances (each its own table, cutoff and group count)
// in ONE persistent kernel over a device-side queue of row tiles.
//
// Each instance is a group-key table (ship u16, qty u8, disc u8, tax u8, price u32, key u32;
// 13 B/row) aggregated exactly as q1_launch_groupkey does (groupkey_kernels.cu): the per-row
// arithmetic is the reference's (src/kernels/ht_in_global_mem.hpp:31-49) with group = key.
//
// Work queue: the host splits every instance into items of at most `chunk` tiles of 2048 rows
// (the autotuner chooses the chunk); CTAs claim items with an atomic cursor, so small and large
// instances balance across the GPU without one launch per instance.
//
// Per CTA: one producer warp claims items, and for every tile of the item writes the stage's
// metadata (instance, first row, row count) and streams the six column slices with
// cp.async.bulk into a 4-stage shared-memory ring (a partial last tile is read by the consumers
// straight from global memory instead). Eight consumer warps aggregate every tile; when the
// instance changes they flush their accumulators into the instance's scratch (red.global.add),
// according to the instance's placement mode:
//   kModeRegisters  num_groups <= 4: per-thread dp4a byte planes (ka::PlaneRegs<4>)
//   kModeShared     num_groups <= 64: shared (group, discount, tax) cells (ka::Cube3Table);
//                   <= 256: shared (group, discount) cells (ka::CubeTable); more groups:
//                   shared slots for keys < 2048 (ka::SlotTable), the rest spilled
//   kModeGlobal     every passing row reduces straight into the scratch accumulators
// (engines in q1_keyagg.cuh). Scratch per instance: num_groups x 8 u64, folded into the
// caller's int128 table by batch_finalize.
// All waits are bounded (q1_ptx.cuh); on expiry the kernel records a status bit and leaves.
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_batch.h"
#include "q1_common.cuh"
#include "q1_keyagg.cuh"
#include "q1_ptx.cuh"

namespace q1 {

using namespace ptx;

namespace bk {

constexpr uint32_t R = ka::R;   // 2048 rows per tile
constexpr uint32_t S = 4;
constexpr uint32_t W = 8;
constexpr uint32_t kStage = ka::kStageBytes;
constexpr uint32_t kSteps = R / 4;
constexpr uint32_t kKindFull = 0, kKindPartial = 1, kKindEnd = 2;
// shared table region: the larger of the cube (256 groups) and the slot table (2048 slots)
constexpr uint32_t cmax(uint32_t a, uint32_t b) { return a > b ? a : b; }
constexpr uint32_t kTableBytes =
    cmax(ka::cube3_bytes(ka::kCube3MaxGroups), cmax(ka::cube_bytes(ka::kCubeMaxGroups), ka::slot_bytes(ka::kSlots)));

struct StageMeta {
    uint32_t instance;
    uint32_t kind;
    uint32_t rows;     // rows in this tile
    uint32_t pad;
    uint64_t row0;     // first row of the tile within the instance
};

}  // namespace bk

__global__ void __launch_bounds__((bk::W + 1) * 32, 1) q1_batch_kernel(const __grid_constant__ BatchParams prm) {
    using namespace bk;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ StageMeta meta[S];
    __shared__ __align__(8) uint64_t consumers_bar;   // barrier of the 8 consumer warps (bounded wait)

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t ring = smem_addr(smem);
    uint8_t* const tab = smem + S * kStage;   // shared table, all zero between instances

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        mbar_init(smem_addr(&consumers_bar), W);
        fence_mbar_init();
    }
    for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(tab)[i] = 0;
    __syncthreads();

    if (warp == W) {
        // ------------------------------ producer ----------------------------------------
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            uint32_t k = 0;
            bool ok = true;
            for (;;) {
                const uint32_t item_idx = atomicAdd(prm.cursor, 1u);
                if (item_idx >= prm.num_items) break;
                const BatchItem it = prm.items[item_idx];
                const BatchInstanceDev& in = prm.inst[it.instance];
                for (uint32_t tt = 0; tt < it.num_tiles && ok; ++tt, ++k) {
                    const uint32_t s = k % S;
                    if (!mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) {
                        ok = false;
                        break;
                    }
                    const uint64_t tile = (uint64_t)it.first_tile + tt;
                    const uint64_t row0 = tile * R;
                    const uint32_t n = (uint32_t)(in.rows - row0 < R ? in.rows - row0 : R);
                    meta[s].instance = it.instance;
                    meta[s].row0 = row0;
                    meta[s].rows = n;
                    const uint32_t fb = smem_addr(&full_bar[s]);
                    if (n == R) {
                        meta[s].kind = kKindFull;
                        mbar_arrive_expect_tx(fb, kStage);
#pragma unroll
                        for (int c = 0; c < 6; ++c)
                            bulk_g2s(ring + s * kStage + ka::col_off(c), in.col[c] + tile * (uint64_t)ka::col_bytes(c),
                                     ka::col_bytes(c), fb, pol);
                    } else {
                        meta[s].kind = kKindPartial;
                        mbar_arrive(fb);
                    }
                }
                if (!ok) break;
            }
            // end marker for the consumers
            if (ok) {
                const uint32_t s = k % S;
                if (mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) {
                    meta[s].kind = kKindEnd;
                    mbar_arrive(smem_addr(&full_bar[s]));
                    ++k;
                }
            }
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
    } else {
        // ------------------------------ consumers ---------------------------------------
        const uint32_t ctid = threadIdx.x;
        uint32_t cur = 0xFFFFFFFFu;
        // The instance's descriptor stays in global memory (read through the L1 when a flush or a
        // partial tile needs it); only the fields of the row loop live in registers.
        const BatchInstanceDev* in = nullptr;
        uint32_t num_groups = 0;
        int32_t cutoff = 0;
        uint32_t mode = kModeGlobal;
        uint32_t table = 0;   // 0 slots, 1 (group, discount) cube, 2 (group, discount, tax) cube
        uint32_t hot = 0;
        ka::PlaneRegs<4> regs;
        regs.zero();
        ka::Cube3Table cube3;
        ka::CubeTable cube;
        ka::SlotTable slots;
        cube3.bind(tab, 0);
        cube.bind(tab, 0);
        slots.bind(tab, 0);
        ka::ConsumerBarrier cb{smem_addr(&consumers_bar), 0};
        uint32_t bad = 0;
        // Tiles / rows added since the last flush (the same in every consumer thread): plane
        // partials are flushed every ka::kPlaneFlushTiles tiles, shared tables before they would
        // exceed ka::kTableFlushRows rows, and both whenever the instance changes. A flush of a
        // shared table leaves it all zero.
        uint32_t tiles_since = 0;
        uint64_t rows_since = 0;
        auto flush = [&]() {
            tiles_since = 0;
            rows_since = 0;
            if (cur == 0xFFFFFFFFu) return;
            if (mode == kModeRegisters) {
                regs.flush(in->acc, num_groups, lane);
            } else if (mode == kModeShared) {
                cb.sync(lane, prm.status);
                if (table == 2) cube3.flush(in->acc, num_groups, ctid, W * 32);
                else if (table == 1) cube.flush(in->acc, num_groups, ctid, W * 32);
                else slots.flush(in->acc, ctid, W * 32);
                cb.sync(lane, prm.status);
            }
        };
        auto add = [&](const ka::KeyQuad& x) {
            if (mode == kModeRegisters) {
                regs.add(x, num_groups, bad);
            } else if (mode == kModeShared) {
                if (table == 2) ka::table_quad(cube3, x, num_groups, hot, in->acc, bad);
                else if (table == 1) ka::table_quad(cube, x, num_groups, hot, in->acc, bad);
                else ka::table_quad(slots, x, num_groups, hot, in->acc, bad);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    if (!((x.PM >> (8 * r)) & 1u)) continue;
                    const uint32_t key = x.k[r];
                    if (key >= num_groups) {
                        bad = 1u;
                        continue;
                    }
                    ka::scratch_row(in->acc, key, (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu,
                                    (x.X >> (8 * r)) & 0xFFu, x.p[r]);
                }
            }
        };

        uint32_t k = 0;
        for (;; ++k) {
            const uint32_t s = k % S;
            const bool landed = mbar_wait(smem_addr(&full_bar[s]), (k / S) & 1u, prm.status);
            if (!__all_sync(0xffffffffu, landed)) break;
            const StageMeta m = meta[s];
            if (m.kind == kKindEnd) break;
            if (m.instance != cur) {
                flush();
                cur = m.instance;
                in = prm.inst + cur;
                mode = in->mode;
                num_groups = in->num_groups;
                cutoff = in->cutoff;
                if (mode == kModeRegisters && num_groups > 4) mode = kModeShared;   // planes hold 4 groups
                table = num_groups <= ka::kCube3MaxGroups ? 2u : (num_groups <= ka::kCubeMaxGroups ? 1u : 0u);
                hot = table ? num_groups : (num_groups < ka::kSlots ? num_groups : ka::kSlots);
                if (table == 2) cube3.bind(tab, num_groups);
                else if (table == 1) cube.bind(tab, num_groups);
                else slots.bind(tab, hot);
            } else if ((mode == kModeRegisters && tiles_since >= ka::kPlaneFlushTiles) ||
                       (mode == kModeShared && rows_since + m.rows > ka::kTableFlushRows)) {
                flush();
            }
            ++tiles_since;
            rows_since += m.rows;
            if (m.kind == kKindFull) {
                // one engine per tile: the mode test stays out of the row loop
                const uint32_t base = ring + s * kStage;
                if (mode == kModeRegisters) {
#pragma unroll 1
                    for (uint32_t itx = 0; itx < kSteps / (W * 32); ++itx)
                        regs.add(ka::load_quad(base, ctid + itx * (W * 32), cutoff, bad), num_groups, bad);
                } else if (mode == kModeShared && table == 2) {
#pragma unroll
                    for (uint32_t itx = 0; itx < kSteps / (W * 32); ++itx)
                        ka::table_quad(cube3, ka::load_quad(base, ctid + itx * (W * 32), cutoff, bad), num_groups,
                                       hot, in->acc, bad);
                } else {
#pragma unroll
                    for (uint32_t itx = 0; itx < kSteps / (W * 32); ++itx)
                        add(ka::load_quad(base, ctid + itx * (W * 32), cutoff, bad));
                }
            } else {
                for (uint32_t i = ctid; i < m.rows; i += W * 32) add(ka::load_row(in->col, m.row0 + i, cutoff, bad));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
        }
        flush();
        if (bad && prm.status) atomicOr(prm.status, kStatusDomain);
    }
    __syncthreads();
}

// scratch of every instance -> its int128 table (+=); one thread per (instance, group).
__global__ void __launch_bounds__(256) q1_batch_finalize(const BatchInstanceDev* __restrict__ inst,
                                                         const uint64_t* __restrict__ group_base, uint32_t ninst,
                                                         uint64_t total_groups) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total_groups) return;
    uint32_t lo = 0, hi = ninst;   // instance with group_base[i] <= t < group_base[i+1]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (group_base[mid] <= t) lo = mid; else hi = mid;
    }
    const BatchInstanceDev& in = inst[lo];
    const uint32_t g = (uint32_t)(t - group_base[lo]);
    const unsigned long long* a = in.acc + 8ull * g;
    if (!a[0]) return;
    unsigned long long* o = in.out + 12ull * g;
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

// Zero every instance's int128 result table; one thread per (instance, group).
__global__ void __launch_bounds__(256) q1_batch_zero_outputs(const BatchInstanceDev* __restrict__ inst,
                                                             const uint64_t* __restrict__ group_base, uint32_t ninst,
                                                             uint64_t total_groups) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total_groups) return;
    uint32_t lo = 0, hi = ninst;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (group_base[mid] <= t) lo = mid; else hi = mid;
    }
    unsigned long long* o = inst[lo].out + 12ull * (t - group_base[lo]);
#pragma unroll
    for (int i = 0; i < 12; ++i) o[i] = 0;
}

cudaError_t launch_batch_zero_outputs(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                      uint64_t total_groups, cudaStream_t stream) {
    if (!total_groups) return cudaSuccess;
    q1_batch_zero_outputs<<<(unsigned)((total_groups + 255) / 256), 256, 0, stream>>>(inst, group_base, ninst,
                                                                                    total_groups);
    return cudaGetLastError();
}

uint32_t batch_smem_bytes() { return bk::S * bk::kStage + bk::kTableBytes; }

cudaError_t batch_prepare_launch() {
    return cudaFuncSetAttribute(q1_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem_bytes());
}

cudaError_t launch_batch(const BatchParams& prm, uint32_t grid, cudaStream_t stream) {
    q1_batch_kernel<<<grid, (bk::W + 1) * 32, batch_smem_bytes(), stream>>>(prm);
    return cudaGetLastError();
}

cudaError_t launch_batch_finalize(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                  uint64_t total_groups, cudaStream_t stream) {
    if (!total_groups) return cudaSuccess;
    q1_batch_finalize<<<(unsigned)((total_groups + 255) / 256), 256, 0, stream>>>(inst, group_base, ninst, total_groups);
    return cudaGetLastError();
}

}  // namespace q1
