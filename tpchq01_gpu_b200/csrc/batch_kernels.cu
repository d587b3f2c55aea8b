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
//   kModeRegisters  num_groups <= 8: per-thread registers, predicated by one-hot key bits
//   kModeShared     a shared-memory table for keys < 2048 (shared atomics), the rest spilled
//   kModeGlobal     every passing row reduces straight into the scratch accumulators
// Scratch per instance: num_groups x 8 u64 (count, qty, disc, price, disc_price lo32/hi32 sums,
// charge lo32/hi32 sums), folded into the caller's int128 table by batch_finalize.
// All waits are bounded (q1_ptx.cuh); on expiry the kernel records a status bit and leaves.
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_batch.h"
#include "q1_common.cuh"
#include "q1_ptx.cuh"

namespace q1 {

using namespace ptx;

namespace bk {

constexpr uint32_t R = kBatchTileRows;   // 2048
constexpr uint32_t S = 4;
constexpr uint32_t W = 8;
constexpr uint32_t kStage = R * 13;
constexpr uint32_t kOffShip = 0, kOffQty = 2 * R, kOffDisc = 3 * R, kOffTax = 4 * R, kOffPrice = 5 * R, kOffKey = 9 * R;
__host__ __device__ constexpr uint32_t col_bytes(int c) { return c == 0 ? 2 * R : (c < 4 ? R : 4 * R); }
__host__ __device__ constexpr uint32_t col_off(int c) {
    return c == 0 ? kOffShip : (c == 1 ? kOffQty : (c == 2 ? kOffDisc : (c == 3 ? kOffTax : (c == 4 ? kOffPrice : kOffKey))));
}
constexpr uint32_t kSteps = R / 4;
constexpr uint32_t kHotSlots = 2048;
constexpr uint32_t kKindFull = 0, kKindPartial = 1, kKindEnd = 2;

struct StageMeta {
    uint32_t instance;
    uint32_t kind;
    uint32_t rows;     // rows in this tile
    uint32_t pad;
    uint64_t row0;     // first row of the tile within the instance
};

__device__ __forceinline__ void red_add(unsigned long long* p, uint64_t v) {
    if (v) asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void scratch_add(unsigned long long* acc, uint32_t g, uint64_t cnt, uint64_t q, uint64_t d,
                                            uint64_t p, uint64_t dp, uint64_t ch) {
    unsigned long long* a = acc + 8ull * g;
    red_add(a + 0, cnt);
    red_add(a + 1, q);
    red_add(a + 2, d);
    red_add(a + 3, p);
    red_add(a + 4, dp & 0xFFFFFFFFull);
    red_add(a + 5, dp >> 32);
    red_add(a + 6, ch & 0xFFFFFFFFull);
    red_add(a + 7, ch >> 32);
}

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
    // shared table (52 B per slot): count u32; qty, disc, price, disc_price, charge low 32 bits,
    // charge high bits as u64 -- exact for 2^25 rows between flushes
    uint32_t* t_cnt = reinterpret_cast<uint32_t*>(smem + S * kStage);
    unsigned long long* t_q = reinterpret_cast<unsigned long long*>(smem + S * kStage + 4 * kHotSlots);
    unsigned long long* t_d = t_q + kHotSlots;
    unsigned long long* t_p = t_d + kHotSlots;
    unsigned long long* t_dp = t_p + kHotSlots;
    unsigned long long* t_chl = t_dp + kHotSlots;
    unsigned long long* t_chh = t_chl + kHotSlots;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        mbar_init(smem_addr(&consumers_bar), W);
        fence_mbar_init();
    }
    for (uint32_t i = threadIdx.x; i < kHotSlots; i += blockDim.x) {
        t_cnt[i] = 0;
        t_q[i] = t_d[i] = t_p[i] = t_dp[i] = t_chl[i] = t_chh[i] = 0;
    }
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
                            bulk_g2s(ring + s * kStage + col_off(c), in.col[c] + tile * (uint64_t)col_bytes(c),
                                     col_bytes(c), fb, pol);
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
        BatchInstanceDev in{};
        uint32_t mode = kModeGlobal;
        // registers mode: 8 groups
        uint64_t rp[8], rdp[8], rch[8];
        uint32_t rc[8], rq[8], rd[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) rp[i] = rdp[i] = rch[i] = 0, rc[i] = rq[i] = rd[i] = 0;
        uint32_t bad = 0;

        // Rows added since the last flush (the same count in every consumer thread): registers
        // are flushed every 2^19 rows (per-thread sums x 32 lanes stay below 2^64), the shared
        // table every 2^25 rows, and both whenever the instance changes.
        uint64_t since = 0;
        // Barrier of the consumer warps only (the producer keeps streaming): one arrive per warp,
        // bounded wait; every consumer passes the same sequence of barriers, so a local phase
        // counter tracks the barrier's parity.
        uint32_t sync_phase = 0;
        auto consumers_sync = [&]() {
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&consumers_bar));
            mbar_wait(smem_addr(&consumers_bar), sync_phase & 1u, prm.status);
            ++sync_phase;
        };
        auto flush = [&]() {
            since = 0;
            if (cur == 0xFFFFFFFFu) return;
            if (mode == kModeRegisters) {
#pragma unroll
                for (int g = 0; g < 8; ++g) {
                    const uint64_t v[6] = {rc[g], rq[g], rd[g], rp[g], rdp[g], rch[g]};
                    uint64_t s6[6];
#pragma unroll
                    for (int a = 0; a < 6; ++a) s6[a] = warp_sum_u64(v[a]);
                    if (lane == 0 && (uint32_t)g < in.num_groups && s6[0])
                        scratch_add(in.acc, g, s6[0], s6[1], s6[2], s6[3], s6[4], s6[5]);
                    rp[g] = rdp[g] = rch[g] = 0;
                    rc[g] = rq[g] = rd[g] = 0;
                }
            } else if (mode == kModeShared) {
                const uint32_t hot = in.num_groups < kHotSlots ? in.num_groups : kHotSlots;
                consumers_sync();
                for (uint32_t g = ctid; g < hot; g += W * 32) {
                    if (t_cnt[g]) {
                        unsigned long long* a = in.acc + 8ull * g;
                        red_add(a + 0, t_cnt[g]);
                        red_add(a + 1, t_q[g]);
                        red_add(a + 2, t_d[g]);
                        red_add(a + 3, t_p[g]);
                        red_add(a + 4, t_dp[g] & 0xFFFFFFFFull);
                        red_add(a + 5, t_dp[g] >> 32);
                        red_add(a + 6, t_chl[g]);
                        red_add(a + 7, t_chh[g]);
                    }
                    t_cnt[g] = 0;
                    t_q[g] = t_d[g] = t_p[g] = t_dp[g] = t_chl[g] = t_chh[g] = 0;
                }
                consumers_sync();
            }
        };

        auto row = [&](uint32_t key, bool pass, uint32_t q, uint32_t d, uint32_t t, uint32_t p) {
            if (pass && key >= in.num_groups) bad = 1;
            if (!pass || key >= in.num_groups) return;
            const uint32_t a = 100u - d;
            const uint32_t ab = a * (100u + t);
            if (mode == kModeRegisters) {
#pragma unroll
                for (int g = 0; g < 8; ++g) {
                    const bool hit = key == (uint32_t)g;
                    const uint32_t pg = hit ? p : 0u;
                    rc[g] += hit ? 1u : 0u;
                    rq[g] += hit ? q : 0u;
                    rd[g] += hit ? d : 0u;
                    rp[g] += pg;
                    rdp[g] = mad_wide(a, pg, rdp[g]);
                    rch[g] = mad_wide(ab, pg, rch[g]);
                }
            } else if (mode == kModeShared && key < kHotSlots) {
                atomicAdd(&t_cnt[key], 1u);
                atomicAdd(&t_q[key], (unsigned long long)q);
                atomicAdd(&t_d[key], (unsigned long long)d);
                atomicAdd(&t_p[key], (unsigned long long)p);
                const uint64_t ch = (uint64_t)ab * p;
                atomicAdd(&t_dp[key], (unsigned long long)((uint64_t)a * p));
                atomicAdd(&t_chl[key], (unsigned long long)(ch & 0xFFFFFFFFull));
                atomicAdd(&t_chh[key], (unsigned long long)(ch >> 32));
            } else {
                scratch_add(in.acc, key, 1, q, d, p, (uint64_t)a * p, (uint64_t)ab * p);
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
                in = prm.inst[cur];
                mode = in.mode;
            } else if ((mode == kModeRegisters && since >= (1ull << 19)) || (mode == kModeShared && since >= (1ull << 25))) {
                flush();
            }
            since += m.rows;
            if (m.kind == kKindFull) {
                const uint32_t base = ring + s * kStage;
#pragma unroll
                for (uint32_t itx = 0; itx < kSteps / (W * 32); ++itx) {
                    const uint32_t j = ctid + itx * (W * 32);
                    const uint2 sd = lds_v2(base + kOffShip + 8 * j);
                    const uint32_t Q = lds_u32(base + kOffQty + 4 * j);
                    const uint32_t D = lds_u32(base + kOffDisc + 4 * j);
                    const uint32_t X = lds_u32(base + kOffTax + 4 * j);
                    const uint4 Pv = lds_v4(base + kOffPrice + 16 * j);
                    const uint4 K = lds_v4(base + kOffKey + 16 * j);
                    if ((((D & 0x7F7F7F7Fu) + 0x1B1B1B1Bu) | D) & 0x80808080u) bad = 1;
                    const uint32_t sh[4] = {sd.x & 0xFFFFu, sd.x >> 16, sd.y & 0xFFFFu, sd.y >> 16};
                    const uint32_t pv[4] = {Pv.x, Pv.y, Pv.z, Pv.w};
                    const uint32_t kv[4] = {K.x, K.y, K.z, K.w};
#pragma unroll
                    for (int r = 0; r < 4; ++r)
                        row(kv[r], (int32_t)sh[r] <= in.cutoff, (Q >> (8 * r)) & 0xFFu, (D >> (8 * r)) & 0xFFu,
                            (X >> (8 * r)) & 0xFFu, pv[r]);
                }
            } else {
                for (uint32_t i = ctid; i < m.rows; i += W * 32) {
                    const uint64_t rr = m.row0 + i;
                    const uint32_t d = __ldg(in.col[2] + rr);
                    if (d > 100u) bad = 1;
                    row(__ldg(reinterpret_cast<const uint32_t*>(in.col[5]) + rr),
                        (int32_t)__ldg(reinterpret_cast<const uint16_t*>(in.col[0]) + rr) <= in.cutoff,
                        __ldg(in.col[1] + rr), d, __ldg(in.col[3] + rr),
                        __ldg(reinterpret_cast<const uint32_t*>(in.col[4]) + rr));
                }
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

uint32_t batch_smem_bytes() { return bk::S * bk::kStage + bk::kHotSlots * 52; }

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
