// Kernels of the serving loop (q1_serve.cpp):
//   * generate_keyed_table: an ad-hoc group-key table (ship u16, qty u8, disc u8, tax u8,
//     price u32, key u32) from the seeded generator; key = the row's (returnflag, linestatus)
//     dictionary code (0..3 for AF, NF, NO, RF: "pair" keys, the Q1 groups) or a uniform key in
//     [0, G);
//   * cube_pass: partial aggregates per (ship day, group) for a window of days of the resident
//     table, reduced into split-limb scratch (one shared-memory table per CTA);
//   * cube_finalize / cube_prefix: scratch -> int128 cube, then prefix sums over days, so that the
//     answer for "ship <= c" is one row of the cumulative cube;
//   * cube_lookup: copies the answers of a round's resident requests into their response slots.
// All per-row arithmetic is the reference's (src/kernels/ht_in_global_mem.hpp:31-49).
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_common.cuh"
#include "q1_ptx.cuh"
#include "q1_serve.h"

namespace q1 {

using namespace ptx;

__global__ void __launch_bounds__(256) generate_keyed_table_kernel(uint64_t key, uint64_t rows, uint32_t pair_keys,
                                                                   uint32_t num_groups, KeyedTableOut out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const GenRow g = gen_row(key, i);
    out.shipdate[i] = (uint16_t)(g.shipdate - kShipDateFrame);
    out.quantity[i] = (uint8_t)g.quantity;
    out.discount[i] = (uint8_t)g.discount;
    out.tax[i] = (uint8_t)g.tax;
    out.extendedprice[i] = g.extprice;
    out.keys[i] = pair_keys ? gen_pair_code(group_of(encode_return_flag(g.returnflag), encode_line_status(g.linestatus)))
                            : gen_group_key_uniform(key, i, num_groups);
}

cudaError_t launch_generate_keyed_table(uint64_t seed, uint64_t rows, uint32_t pair_keys, uint32_t num_groups,
                                        const KeyedTableOut& out, cudaStream_t stream) {
    if (!rows) return cudaSuccess;
    generate_keyed_table_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(gen_key(seed), rows, pair_keys,
                                                                                  num_groups, out);
    return cudaGetLastError();
}

// One window of days [d0, d0 + days) x G groups; slot = (ship - d0) * G + group.
// Shared table per CTA: count u32 + 6 x u64 (qty, disc, price, disc_price, charge lo32 / hi),
// exact for up to 2^25 rows per CTA (the host caps the grid-stride share accordingly).
__global__ void __launch_bounds__(512) cube_pass_kernel(CubePassParams prm) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t slots = prm.days * prm.num_groups;
    uint32_t* t_cnt = reinterpret_cast<uint32_t*>(smem);
    unsigned long long* t = reinterpret_cast<unsigned long long*>(smem + ((4 * slots + 15) & ~15u));
    for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) {
        t_cnt[i] = 0;
        for (int k = 0; k < 6; ++k) t[k * slots + i] = 0;
    }
    __syncthreads();
    uint32_t bad = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < prm.rows; i += stride) {
        const uint32_t ship = prm.ship[i];
        if (ship >= prm.all_days) bad = 1;
        if (ship < prm.d0 || ship >= prm.d0 + prm.days) continue;
        const uint32_t g = prm.pair ? prm.pair_group[(prm.codes[i >> 4] >> (2 * (i & 15))) & 3u] : prm.keys[i];
        if (g >= prm.num_groups) {
            bad = 1;
            continue;
        }
        const uint32_t d = prm.disc[i], tx = prm.tax[i], p = prm.price[i], q = prm.qty[i];
        if (d > 100u) bad = 1;
        const uint32_t a = 100u - d, ab = a * (100u + tx);
        const uint64_t dp = (uint64_t)a * p, ch = (uint64_t)ab * p;
        const uint32_t s = (ship - prm.d0) * prm.num_groups + g;
        atomicAdd(&t_cnt[s], 1u);
        atomicAdd(&t[0 * slots + s], (unsigned long long)q);
        atomicAdd(&t[1 * slots + s], (unsigned long long)d);
        atomicAdd(&t[2 * slots + s], (unsigned long long)p);
        atomicAdd(&t[3 * slots + s], (unsigned long long)dp);
        atomicAdd(&t[4 * slots + s], (unsigned long long)(ch & 0xFFFFFFFFull));
        atomicAdd(&t[5 * slots + s], (unsigned long long)(ch >> 32));
    }
    if (bad && prm.status) atomicOr(prm.status, kStatusDomain);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) {
        if (!t_cnt[i]) continue;
        unsigned long long* a = prm.acc + 8ull * ((uint64_t)prm.d0 * prm.num_groups + i);
        atomicAdd(a + 0, (unsigned long long)t_cnt[i]);
        atomicAdd(a + 1, t[0 * slots + i]);
        atomicAdd(a + 2, t[1 * slots + i]);
        atomicAdd(a + 3, t[2 * slots + i]);
        atomicAdd(a + 4, t[3 * slots + i] & 0xFFFFFFFFull);
        atomicAdd(a + 5, t[3 * slots + i] >> 32);
        atomicAdd(a + 6, t[4 * slots + i]);
        atomicAdd(a + 7, t[5 * slots + i]);
    }
}

cudaError_t launch_cube_pass(const CubePassParams& prm, int sm_count, cudaStream_t stream) {
    const uint32_t slots = prm.days * prm.num_groups;
    const uint32_t dyn = ((4 * slots + 15) & ~15u) + 48 * slots;
    cudaError_t e = cudaFuncSetAttribute(cube_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    // enough CTAs that each handles at most 2^25 rows
    uint64_t grid = (uint64_t)sm_count * 2;
    while (prm.rows / grid > (1ull << 25)) grid *= 2;
    cube_pass_kernel<<<(unsigned)grid, 512, dyn, stream>>>(prm);
    return cudaGetLastError();
}

// scratch (days*G x 8 u64) -> int128 cube [days][G][6]
__global__ void cube_finalize_kernel(const unsigned long long* __restrict__ acc, uint64_t entries,
                                     unsigned long long* __restrict__ cube) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= entries) return;
    const unsigned long long* a = acc + 8 * e;
    unsigned long long* o = cube + 12 * e;
    const unsigned __int128 v[6] = {
        (unsigned __int128)a[0],
        (unsigned __int128)a[1] * 100u,
        (unsigned __int128)a[3],
        (unsigned __int128)a[2],
        (unsigned __int128)a[4] + ((unsigned __int128)a[5] << 32),
        (unsigned __int128)a[6] + ((unsigned __int128)a[7] << 32)};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        o[2 * k] = (uint64_t)v[k];
        o[2 * k + 1] = (uint64_t)(v[k] >> 64);
    }
}

// In-place prefix sums over days: cube[d][g][k] += cube[d-1][g][k]; one thread per (g, k).
__global__ void cube_prefix_kernel(unsigned long long* cube, uint32_t days, uint32_t num_groups) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_groups * 6) return;
    uint64_t lo = 0, hi = 0;
    for (uint32_t d = 0; d < days; ++d) {
        unsigned long long* o = cube + 12ull * ((uint64_t)d * num_groups) + 2 * t;
        const uint64_t nlo = lo + o[0];
        hi = hi + o[1] + (nlo < lo ? 1u : 0u);
        lo = nlo;
        o[0] = lo;
        o[1] = hi;
    }
}

cudaError_t launch_cube_finalize(const unsigned long long* acc, uint32_t days, uint32_t num_groups,
                                 unsigned long long* cube, cudaStream_t stream) {
    const uint64_t entries = (uint64_t)days * num_groups;
    cube_finalize_kernel<<<(unsigned)((entries + 255) / 256), 256, 0, stream>>>(acc, entries, cube);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cube_prefix_kernel<<<(num_groups * 6 + 255) / 256, 256, 0, stream>>>(cube, days, num_groups);
    return cudaGetLastError();
}

// For every resident request of a round: response[r] = cumulative cube row at its cutoff (zeros
// when nothing passes). One thread per (request, int128 word).
__global__ void cube_lookup_kernel(const CubeLookup* __restrict__ reqs, uint32_t n, uint32_t words_per_response,
                                   unsigned long long* __restrict__ responses) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = (uint32_t)(t / words_per_response), w = (uint32_t)(t % words_per_response);
    if (r >= n) return;
    const CubeLookup q = reqs[r];
    const uint32_t words = q.num_groups * 12;
    unsigned long long v = 0;
    if (w < words && q.day >= 0) v = q.cube[12ull * ((uint64_t)q.day * q.num_groups) + w];
    responses[(uint64_t)q.slot * words_per_response + w] = w < words ? v : 0;
}

cudaError_t launch_cube_lookup(const CubeLookup* reqs, uint32_t n, uint32_t words_per_response,
                               unsigned long long* responses, cudaStream_t stream) {
    if (!n) return cudaSuccess;
    const uint64_t threads = (uint64_t)n * words_per_response;
    cube_lookup_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(reqs, n, words_per_response, responses);
    return cudaGetLastError();
}

}  // namespace q1
