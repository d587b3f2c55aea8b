// Group-key aggregation for sm_100a: the Q1 predicate and aggregates, grouped by a synthetic
// uint32 key (up to 65,536 groups) instead of the (returnflag, linestatus) pair.
//
// The per-row arithmetic is the reference's (src/kernels/ht_in_global_mem.hpp:31-49); only the
// group index changes: group = key[i] (< num_groups) instead of (rf << 1) + ls.
//
// Input tile (R rows): ship u16 | qty u8 | disc u8 | tax u8 | price u32 | key u32  (13 B/row),
// streamed with one cp.async.bulk per column into an S-stage shared-memory ring exactly like the
// scan kernel (scan_kernels.cu).
//
// Placements:
//   in_registers_per_thread  num_groups <= 8: predicated per-thread registers over 8 groups
//   shared_mem_per_thread    hierarchical: keys < kHotSlots in a per-CTA shared-memory table
//                            (shared atomics), other keys spilled straight to the global
//                            accumulators
//   global                   every passing row updates the global accumulators directly
//
// Accumulators live in scratch memory (per launch, zeroed first): per group 8 x u64
//   count, qty (whole units), disc, price, disc_price low-32 sum, disc_price high-32 sum,
//   charge low-32 sum, charge high-32 sum
// Splitting the two wide products into 32-bit halves keeps every u64 sum exact for launches of
// up to 2^31 rows, so plain fire-and-forget reductions (red.global.add) suffice. A finalize
// kernel folds the scratch into the caller's int128 table [group][6] with 128-bit atomics
// (so, like the reference kernels, results accumulate into a caller-zeroed buffer).
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_common.cuh"
#include "q1_kernels.h"
#include "q1_ptx.cuh"

namespace q1 {

using namespace ptx;

namespace gk {

constexpr uint32_t R = 2048;          // rows per tile
constexpr uint32_t S = 4;             // ring stages
constexpr uint32_t W = 8;             // consumer warps
constexpr uint32_t kStage = R * 13;   // bytes per stage
// column offsets inside a stage (all multiples of 16)
constexpr uint32_t kOffShip = 0, kOffQty = 2 * R, kOffDisc = 3 * R, kOffTax = 4 * R, kOffPrice = 5 * R,
                   kOffKey = 9 * R;
__host__ __device__ constexpr uint32_t col_bytes(int c) { return c == 0 ? 2 * R : (c < 4 ? R : 4 * R); }
__host__ __device__ constexpr uint32_t col_off(int c) {
    return c == 0 ? kOffShip : (c == 1 ? kOffQty : (c == 2 ? kOffDisc : (c == 3 ? kOffTax : (c == 4 ? kOffPrice : kOffKey))));
}
constexpr uint32_t kSteps = R / 4;    // 4 rows per consumer step
static_assert(kSteps % (W * 32) == 0, "steps must divide evenly");
static_assert(kStage % 16 == 0, "stage alignment");

// Shared table of the hierarchical placement: SoA, 44 B per slot (count u32 + 5 x u64).
constexpr uint32_t kHotSlots = 2048;

__device__ __forceinline__ void red_add(unsigned long long* p, uint64_t v) {
    if (v) asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Adds one row (or a partial sum whose wide parts are given as full 64-bit values) into the
// global accumulators of group g.
__device__ __forceinline__ void global_add(unsigned long long* acc, uint32_t g, uint64_t cnt, uint64_t q, uint64_t d,
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

struct RegTable {   // 8 groups, predicated (same arithmetic as the scan kernel's per-thread table)
    uint64_t p[8], dp[8], ch[8];
    uint32_t q[8], d[8], cnt[8];   // per-thread rows stay below 2^31 / (148 * 256): no u32 overflow
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < 8; ++i) p[i] = dp[i] = ch[i] = q[i] = d[i] = cnt[i] = 0;
    }
    __device__ __forceinline__ void add(uint32_t key, bool pass, uint32_t q_, uint32_t d_, uint32_t a, uint32_t ab,
                                        uint32_t pr) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const bool hit = pass && key == (uint32_t)i;
            const uint32_t pg = hit ? pr : 0u;
            cnt[i] += hit ? 1u : 0u;
            q[i] += hit ? q_ : 0u;
            d[i] += hit ? d_ : 0u;
            p[i] += pg;
            dp[i] = mad_wide(a, pg, dp[i]);
            ch[i] = mad_wide(ab, pg, ch[i]);
        }
    }
};

}  // namespace gk

struct GroupKeyParams {
    const uint8_t* col[6];          // ship, qty, disc, tax, price, key (16-byte aligned)
    uint64_t rows;
    int32_t cutoff;                 // cutoff_day - 727563
    uint32_t num_groups;
    unsigned long long* acc;        // scratch: num_groups x 8 u64, zeroed
    uint32_t* status;
};

template <int P>
__global__ void __launch_bounds__((gk::W + 1) * 32, 1) q1_groupkey_kernel(const __grid_constant__ GroupKeyParams prm) {
    using namespace gk;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ __align__(16) unsigned long long red8[8 * 6];

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint64_t num_tiles = prm.rows / R;
    const uint32_t ring = smem_addr(smem);
    // shared table (hierarchical placement), after the ring
    uint32_t* t_cnt = reinterpret_cast<uint32_t*>(smem + S * kStage);
    unsigned long long* t_q = reinterpret_cast<unsigned long long*>(smem + S * kStage + 4 * kHotSlots);
    unsigned long long* t_d = t_q + kHotSlots;
    unsigned long long* t_p = t_d + kHotSlots;
    unsigned long long* t_dp = t_p + kHotSlots;
    unsigned long long* t_ch = t_dp + kHotSlots;   // 4 + 5*8 = 44 B per slot
    const uint32_t hot = prm.num_groups < kHotSlots ? prm.num_groups : kHotSlots;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        fence_mbar_init();
    }
    for (uint32_t i = threadIdx.x; i < 48; i += blockDim.x) red8[i] = 0;
    if (P == kPlaceSharedMemPerThread) {
        for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
            t_cnt[i] = 0;
            t_q[i] = t_d[i] = t_p[i] = t_dp[i] = t_ch[i] = 0;
        }
    }
    __syncthreads();

    if (warp == W) {
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            uint32_t k = 0;
            for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
                const uint32_t s = k % S;
                if (!mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) break;
                const uint32_t fb = smem_addr(&full_bar[s]);
                mbar_arrive_expect_tx(fb, kStage);
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    bulk_g2s(ring + s * kStage + col_off(c), prm.col[c] + t * (uint64_t)col_bytes(c), col_bytes(c), fb, pol);
            }
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
    } else {
        const uint32_t ctid = threadIdx.x;
        RegTable regs;
        if (P == kPlaceInRegistersPerThread) regs.zero();
        uint32_t bad = 0;
        auto row = [&](uint32_t key, bool pass, uint32_t q, uint32_t d, uint32_t t, uint32_t p) {
            const uint32_t a = 100u - d;
            const uint32_t ab = a * (100u + t);
            if (P == kPlaceInRegistersPerThread) {
                regs.add(key, pass && key < prm.num_groups, q, d, a, ab, p);
            } else if (pass && key < prm.num_groups) {
                const uint64_t dp = (uint64_t)a * p;
                const uint64_t ch = (uint64_t)ab * p;
                if (P == kPlaceSharedMemPerThread && key < hot) {
                    atomicAdd(&t_cnt[key], 1u);
                    atomicAdd(&t_q[key], (unsigned long long)q);
                    atomicAdd(&t_d[key], (unsigned long long)d);
                    atomicAdd(&t_p[key], (unsigned long long)p);
                    atomicAdd(&t_dp[key], (unsigned long long)dp);
                    atomicAdd(&t_ch[key], (unsigned long long)ch);
                } else {
                    global_add(prm.acc, key, 1, q, d, p, dp, ch);
                }
            }
            if (pass && key >= prm.num_groups) bad |= kStatusDomain;
        };
        bool ok = true;
        uint32_t k = 0;
        for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
            const uint32_t s = k % S;
            const bool landed = mbar_wait(smem_addr(&full_bar[s]), (k / S) & 1u, prm.status);
            if (!__all_sync(0xffffffffu, landed)) {
                ok = false;
                break;
            }
            const uint32_t base = ring + s * kStage;
#pragma unroll
            for (uint32_t it = 0; it < kSteps / (W * 32); ++it) {
                const uint32_t j = ctid + it * (W * 32);
                const uint2 sd = lds_v2(base + kOffShip + 8 * j);
                const uint32_t Q = lds_u32(base + kOffQty + 4 * j);
                const uint32_t D = lds_u32(base + kOffDisc + 4 * j);
                const uint32_t X = lds_u32(base + kOffTax + 4 * j);
                const uint4 Pv = lds_v4(base + kOffPrice + 16 * j);
                const uint4 K = lds_v4(base + kOffKey + 16 * j);
                bad |= ((((D & 0x7F7F7F7Fu) + 0x1B1B1B1Bu) | D) & 0x80808080u) ? kStatusDomain : 0u;
                const uint32_t sh[4] = {sd.x & 0xFFFFu, sd.x >> 16, sd.y & 0xFFFFu, sd.y >> 16};
                const uint32_t pv[4] = {Pv.x, Pv.y, Pv.z, Pv.w};
                const uint32_t kv[4] = {K.x, K.y, K.z, K.w};
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    row(kv[r], (int32_t)sh[r] <= prm.cutoff, (Q >> (8 * r)) & 0xFFu, (D >> (8 * r)) & 0xFFu,
                        (X >> (8 * r)) & 0xFFu, pv[r]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
        }
        if (ok && blockIdx.x == (uint32_t)(num_tiles % gridDim.x)) {
            for (uint64_t i = num_tiles * R + ctid; i < prm.rows; i += W * 32) {
                const uint32_t d = __ldg(prm.col[2] + i);
                bad |= d > 100u ? kStatusDomain : 0u;
                row(__ldg(reinterpret_cast<const uint32_t*>(prm.col[5]) + i),
                    (int32_t)__ldg(reinterpret_cast<const uint16_t*>(prm.col[0]) + i) <= prm.cutoff,
                    __ldg(prm.col[1] + i), d, __ldg(prm.col[3] + i), __ldg(reinterpret_cast<const uint32_t*>(prm.col[4]) + i));
            }
        }
        if (bad && prm.status) atomicOr(prm.status, bad);
        if (P == kPlaceInRegistersPerThread) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint64_t v[6] = {regs.cnt[i], regs.q[i], regs.d[i], regs.p[i], regs.dp[i], regs.ch[i]};
#pragma unroll
                for (int a = 0; a < 6; ++a) {
                    uint64_t lo = v[a], hi = 0;
                    warp_sum_u128(lo, hi);   // per-CTA sums stay below 2^64 (launches <= 2^31 rows)
                    if (lane == 0) atomicAdd(&red8[i * 6 + a], (unsigned long long)lo);
                }
            }
        }
    }
    __syncthreads();
    if (P == kPlaceInRegistersPerThread) {
        for (uint32_t g = threadIdx.x; g < 8 && g < prm.num_groups; g += blockDim.x)
            global_add(prm.acc, g, red8[g * 6 + 0], red8[g * 6 + 1], red8[g * 6 + 2], red8[g * 6 + 3],
                       red8[g * 6 + 4], red8[g * 6 + 5]);
    } else if (P == kPlaceSharedMemPerThread) {
        for (uint32_t g = threadIdx.x; g < hot; g += blockDim.x)
            if (t_cnt[g]) global_add(prm.acc, g, t_cnt[g], t_q[g], t_d[g], t_p[g], t_dp[g], t_ch[g]);
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

template <int P>
static cudaError_t launch_gk(const GroupKeyParams& prm, int sm_count, int max_blocks, cudaStream_t st) {
    using namespace gk;
    uint32_t dyn = S * kStage + (P == kPlaceSharedMemPerThread ? kHotSlots * 44 : 0);
    cudaError_t e = cudaFuncSetAttribute(q1_groupkey_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    const uint64_t tiles = prm.rows / R;
    uint64_t blocks = tiles ? tiles : 1;
    uint64_t cap = (uint64_t)sm_count;
    if (max_blocks > 0 && (uint64_t)max_blocks < cap) cap = (uint64_t)max_blocks;
    if (blocks > cap) blocks = cap;
    q1_groupkey_kernel<P><<<(unsigned)blocks, (W + 1) * 32, dyn, st>>>(prm);
    return cudaGetLastError();
}

cudaError_t launch_groupkey(int placement, const uint8_t* const cols[6], uint64_t rows, int32_t cutoff_rel,
                            uint32_t num_groups, unsigned long long* scratch, unsigned long long* out,
                            uint32_t* status, int sm_count, int max_blocks, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, groupkey_scratch_bytes(num_groups), stream);
    if (e != cudaSuccess) return e;
    const uint64_t kMaxRows = 1ull << 31;
    for (uint64_t off = 0; off < rows; off += kMaxRows) {
        GroupKeyParams prm{};
        const uint64_t n = rows - off < kMaxRows ? rows - off : kMaxRows;
        const uint32_t bytes[6] = {2, 1, 1, 1, 4, 4};
        for (int c = 0; c < 6; ++c) prm.col[c] = cols[c] + off * bytes[c];
        prm.rows = n;
        prm.cutoff = cutoff_rel;
        prm.num_groups = num_groups;
        prm.acc = scratch;
        prm.status = status;
        switch (placement) {
            case kPlaceInRegistersPerThread: e = launch_gk<kPlaceInRegistersPerThread>(prm, sm_count, max_blocks, stream); break;
            case kPlaceSharedMemPerThread: e = launch_gk<kPlaceSharedMemPerThread>(prm, sm_count, max_blocks, stream); break;
            case kPlaceGlobal: e = launch_gk<kPlaceGlobal>(prm, sm_count, max_blocks, stream); break;
            default: return cudaErrorInvalidValue;
        }
        if (e != cudaSuccess) return e;
        // fold after every 2^31-row launch so the scratch sums stay exact
        q1_groupkey_finalize<<<(num_groups + 255) / 256, 256, 0, stream>>>(scratch, num_groups, out);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (off + kMaxRows < rows) {
            e = cudaMemsetAsync(scratch, 0, groupkey_scratch_bytes(num_groups), stream);
            if (e != cudaSuccess) return e;
        }
    }
    if (rows == 0) return cudaSuccess;
    return cudaSuccess;
}

uint64_t groupkey_scratch_bytes(uint32_t num_groups) { return 64ull * num_groups; }

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
