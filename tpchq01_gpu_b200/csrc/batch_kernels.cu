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
// cp.async.bulk into a shared-memory ring of 4 stages (3 in the table kernel, whose table takes
// the room of the fourth; a partial last tile is read by the consumers
// straight from global memory instead). Eight consumer warps aggregate every tile; when the
// instance changes they flush their accumulators into the instance's scratch (red.global.add),
// according to the instance's placement mode:
//   kModeRegisters  num_groups <= 4: per-thread dp4a byte planes (ka::PlaneRegs<4>)
//   kModeShared     num_groups <= 64: shared (group, discount, tax) cells (ka::Cube3Table);
//                   <= 1024: shared (group, discount) cells (ka::CubeTable); more groups:
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
// ring stages: 4 in the register-planes kernel, 3 in the table kernel
template <bool kRegs>
__host__ __device__ constexpr uint32_t stages() { return kRegs ? 4u : 3u; }
// consumer warps: 8 in the register-planes kernel (128 registers a thread), 16 in the table
// kernel, whose shared-memory atomics need more warps in flight
template <bool kRegs>
__host__ __device__ constexpr uint32_t consumer_warps() { return kRegs ? 8u : 16u; }
constexpr uint32_t kStage = ka::kStageBytes;
constexpr uint32_t kSteps = R / 4;
constexpr uint32_t kKindFull = 0, kKindPartial = 1, kKindEnd = 2;
// shared table region: the largest of the cubes (64 and 1024 groups) and the slot table (2048 slots)
constexpr uint32_t cmax(uint32_t a, uint32_t b) { return a > b ? a : b; }
constexpr uint32_t kTableBytes =
    cmax(ka::cube3_bytes(ka::kCube3MaxGroups), cmax(ka::cube_bytes(ka::kCubeMaxGroups), ka::slot_bytes(ka::kSlots)));
// the table kernel's ring and table, with room left for its static shared memory (< 1 KB)
static_assert(3 * kStage + kTableBytes + 512 <= 227 * 1024, "table kernel shared memory");

struct __align__(16) StageMeta {
    uint32_t instance;
    uint32_t kind;
    uint32_t rows;     // rows in this tile
    uint32_t pad;
    uint64_t row0;     // first row of the tile within the instance
};

}  // namespace bk

namespace bk {

// The instance fields the row loop needs, kept in registers while an instance is current; the
// descriptor itself stays in global memory (read through the L1 for flushes and partial tiles).
struct Current {
    const BatchInstanceDev* in;
    unsigned long long* acc;   // the instance's scratch accumulators
    uint32_t id;          // instance index, 0xFFFFFFFF before the first
    uint32_t num_groups;
    uint32_t hot;         // keys below `hot` go to the shared table
    int32_t cutoff;
};

// Consumer side of one engine: processes stages until the producer's end-of-engine marker,
// flushing the engine's accumulators whenever the instance changes and at the end. `k` is the
// running stage counter shared by all engines of the CTA; returns false if a bounded wait
// expired (the kernel then stops).
template <int E, uint32_t W, uint32_t S>
__device__ __forceinline__ bool consume_engine(const BatchParams& prm, uint32_t ring, uint8_t* tab, uint64_t* full_bar,
                                               uint64_t* empty_bar, const StageMeta* meta, uint32_t& k,
                                               ka::ConsumerBarrier& cb, uint32_t& bad) {
    const uint32_t lane = threadIdx.x & 31u, ctid = threadIdx.x;
    ka::PlaneRegs<4> regs;
    ka::Cube3Table cube3;
    ka::CubeTableT<false> cube;
    ka::SlotTable slots;
    if constexpr (E == kEngRegisters) regs.zero();
    Current c{nullptr, nullptr, 0xFFFFFFFFu, 0, 0, 0};
    uint32_t tiles_since = 0;
    uint64_t rows_since = 0;
    bool ok = true;

    auto flush = [&]() {
        tiles_since = 0;
        rows_since = 0;
        if (c.id == 0xFFFFFFFFu) return;
        if constexpr (E == kEngRegisters) {
            regs.flush(c.acc, c.num_groups, lane);
        } else if constexpr (E != kEngGlobal) {
            cb.sync(lane, prm.status);
            if constexpr (E == kEngCube3) cube3.flush(c.acc, c.num_groups, ctid, W * 32);
            else if constexpr (E == kEngCube) cube.flush(c.acc, c.num_groups, ctid, W * 32);
            else slots.flush(c.acc, ctid, W * 32);
            cb.sync(lane, prm.status);
        }
    };
    auto add = [&](const ka::KeyQuad& x) {
        if constexpr (E == kEngRegisters) {
            regs.add(x, c.num_groups, c.acc, bad);
        } else if constexpr (E == kEngCube3) {
            ka::table_quad(cube3, x, c.num_groups, c.hot, c.acc, bad);
        } else if constexpr (E == kEngCube) {
            ka::table_quad(cube, x, c.num_groups, c.hot, c.acc, bad);
        } else if constexpr (E == kEngSlots) {
            ka::table_quad(slots, x, c.num_groups, c.hot, c.acc, bad);
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (!((x.PM >> (8 * r)) & 1u)) continue;
                const uint32_t key = x.k[r];
                if (key >= c.num_groups) {
                    bad = 1u;
                    continue;
                }
                ka::scratch_row(c.acc, key, (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu,
                                (x.X >> (8 * r)) & 0xFFu, x.p[r]);
            }
        }
    };

    uint32_t s = k % S, ph = (k / S) & 1u;   // stage and phase of stage counter k, stepped below
    for (;; ++k) {
        const bool landed = mbar_wait(smem_addr(&full_bar[s]), ph, prm.status);
        if (!__all_sync(0xffffffffu, landed)) {
            ok = false;
            break;
        }
        // instance, kind and row count in one 16-byte load (row0 only for a partial tile)
        const uint4 mh = *reinterpret_cast<const uint4*>(&meta[s]);
        const StageMeta m{mh.x, mh.y, mh.z, 0u, 0ull};
        if (m.kind == kKindEnd) {
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
            ++k;
            break;
        }
        if (m.instance != c.id) {
            flush();
            c.id = m.instance;
            c.in = prm.inst + m.instance;
            c.acc = c.in->acc;
            c.num_groups = c.in->num_groups;
            c.cutoff = c.in->cutoff;
            c.hot = (E == kEngSlots && c.num_groups > ka::kSlots) ? ka::kSlots : c.num_groups;
            if constexpr (E == kEngCube3) cube3.bind(tab, c.num_groups);
            if constexpr (E == kEngCube) cube.bind(tab, c.num_groups);
            if constexpr (E == kEngSlots) slots.bind(tab, c.hot);
        } else if ((E == kEngRegisters && tiles_since >= ka::kPlaneFlushTiles) ||
                   (E != kEngRegisters && E != kEngGlobal && rows_since + m.rows > ka::kTableFlushRows)) {
            flush();
        }
        ++tiles_since;
        rows_since += m.rows;
        if (m.kind == kKindFull) {
            const uint32_t base = ring + s * kStage;
#pragma unroll
            for (uint32_t itx = 0; itx < kSteps / (W * 32); ++itx)
                add(ka::load_quad(base, ctid + itx * (W * 32), c.cutoff, bad));
        } else {
            // every lane runs every round (the table engines vote across the warp)
            for (uint32_t i0 = 0; i0 < m.rows; i0 += W * 32) {
                const uint32_t i = i0 + ctid;
                add(i < m.rows ? ka::load_row(c.in->col, meta[s].row0 + i, c.cutoff, bad) : ka::empty_quad());
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
        if (++s == S) {
            s = 0;
            ph ^= 1u;
        }
    }
    flush();
    return ok;
}

// Engine queue processed at step `step` of a CTA, and the engine code that processes it. The
// register-planes kernel has one step (queue 0). The table kernel starts at its role's queue
// among 1..4 (grid ranges role_end), visits the others in turn, then helps with queue 0 through
// the (group, discount, tax) cells, which hold any instance of <= 4 groups.
template <bool kRegs>
__device__ __forceinline__ uint32_t queue_at(const BatchParams& prm, uint32_t step) {
    if (kRegs) return kEngRegisters;
    uint32_t e0 = 1;
    while (e0 + 1 < kEngines && blockIdx.x >= prm.role_end[e0]) ++e0;
    return step < kEngines - 1 ? 1u + (e0 - 1u + step) % (kEngines - 1u) : (uint32_t)kEngRegisters;
}
template <bool kRegs>
__host__ __device__ constexpr uint32_t steps() { return kRegs ? 1u : kEngines; }

}  // namespace bk

template <bool kRegs>
__global__ void __launch_bounds__((bk::consumer_warps<kRegs>() + 1) * 32, 1)
    q1_batch_kernel(const __grid_constant__ BatchParams prm) {
    using namespace bk;
    constexpr uint32_t W = consumer_warps<kRegs>();
    constexpr uint32_t S = stages<kRegs>();
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ StageMeta meta[S];
    __shared__ __align__(8) uint64_t consumers_bar;   // barrier of the consumer warps (bounded wait)

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t ring = smem_addr(smem);
    uint8_t* const tab = smem + S * kStage;   // shared table (table kernel), all zero between instances

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        mbar_init(smem_addr(&consumers_bar), W);
        fence_mbar_init();
    }
    if (!kRegs)
        for (uint32_t i = threadIdx.x; i < kTableBytes / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(tab)[i] = 0;
    __syncthreads();

    if (warp == W) {
        // ------------------------------ producer ----------------------------------------
        // Per step, claim items from that queue until it is empty, stream their tiles, then post
        // an end-of-queue marker.
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            uint32_t k = 0;
            bool ok = true;
            for (uint32_t step = 0; step < steps<kRegs>() && ok; ++step) {
                const uint32_t e = queue_at<kRegs>(prm, step);
                const uint32_t count = prm.item_begin[e + 1] - prm.item_begin[e];
                for (;;) {
                    const uint32_t idx = count ? atomicAdd(prm.cursor + e, 1u) : count;
                    if (idx >= count) break;
                    const BatchItem it = prm.items[prm.item_begin[e] + idx];
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
                if (!ok) break;
                const uint32_t s = k % S;
                if (!mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) {
                    ok = false;
                    break;
                }
                meta[s].kind = kKindEnd;
                mbar_arrive(smem_addr(&full_bar[s]));
                ++k;
            }
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
    } else {
        // ------------------------------ consumers ---------------------------------------
        // The same queue order; each engine's loop keeps only its own accumulators live.
        ka::ConsumerBarrier cb{smem_addr(&consumers_bar), 0};
        uint32_t bad = 0, k = 0;
        for (uint32_t step = 0; step < steps<kRegs>(); ++step) {
            const uint32_t e = queue_at<kRegs>(prm, step);
            bool ok;
            if constexpr (kRegs) {
                ok = consume_engine<kEngRegisters, W, S>(prm, ring, tab, full_bar, empty_bar, meta, k, cb, bad);
            } else {
                switch (e) {
                    case kEngCube: ok = consume_engine<kEngCube, W, S>(prm, ring, tab, full_bar, empty_bar, meta, k, cb, bad); break;
                    case kEngSlots: ok = consume_engine<kEngSlots, W, S>(prm, ring, tab, full_bar, empty_bar, meta, k, cb, bad); break;
                    case kEngGlobal: ok = consume_engine<kEngGlobal, W, S>(prm, ring, tab, full_bar, empty_bar, meta, k, cb, bad); break;
                    default:   // queues 1 and 0
                        ok = consume_engine<kEngCube3, W, S>(prm, ring, tab, full_bar, empty_bar, meta, k, cb, bad);
                        break;
                }
            }
            if (!ok) break;
        }
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

uint32_t batch_smem_bytes() { return bk::stages<false>() * bk::kStage + bk::kTableBytes; }
// The register-planes kernel needs only the ring; asking for more than half the SM's shared
// memory keeps it at one CTA per SM, like the table kernel.
static uint32_t batch_regs_smem_bytes() { return 120u * 1024u; }

cudaError_t batch_prepare_launch() {
    cudaError_t e = cudaFuncSetAttribute(q1_batch_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)batch_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(q1_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)batch_regs_smem_bytes());
}

cudaError_t launch_batch(const BatchParams& prm, uint32_t grid_regs, uint32_t grid_tables, cudaStream_t stream,
                         cudaStream_t aux, cudaEvent_t fork, cudaEvent_t join) {
    cudaError_t e = cudaSuccess;
    const bool both = grid_regs && grid_tables;
    if (both) {
        if ((e = cudaEventRecord(fork, stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(aux, fork, 0)) != cudaSuccess) return e;
    }
    if (grid_regs) {
        q1_batch_kernel<true><<<grid_regs, (bk::consumer_warps<true>() + 1) * 32, batch_regs_smem_bytes(),
                                both ? aux : stream>>>(prm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (grid_tables) {
        q1_batch_kernel<false><<<grid_tables, (bk::consumer_warps<false>() + 1) * 32, batch_smem_bytes(), stream>>>(prm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (both) {
        if ((e = cudaEventRecord(join, aux)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(stream, join, 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_batch_finalize(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                  uint64_t total_groups, cudaStream_t stream) {
    if (!total_groups) return cudaSuccess;
    q1_batch_finalize<<<(unsigned)((total_groups + 255) / 256), 256, 0, stream>>>(inst, group_base, ninst, total_groups);
    return cudaGetLastError();
}

}  // namespace q1
