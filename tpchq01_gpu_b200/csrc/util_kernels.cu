// Utility kernels: the seeded generator fused with compression (device-side table creation) and
// the filter-bitmap precomputation (the GPU counterpart of src/main.cu:362-389).
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_common.cuh"
#include "q1_kernels.h"
#include "q1_ptx.cuh"

namespace q1 {

// Each thread produces a block of 32 consecutive rows, so that every packed container word
// (16 pair codes, 16 return flags, 32 line stati) is written by exactly one thread.
__global__ void __launch_bounds__(256) generate_compressed_kernel(uint64_t key, uint64_t first_row, uint64_t rows,
                                                                  GenCompressedOut out) {
    const uint64_t blk = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t r0 = blk * 32;
    if (r0 >= rows) return;
    const uint32_t n = (rows - r0 < 32) ? (uint32_t)(rows - r0) : 32u;
    uint32_t pair_w[2] = {0, 0}, rf_w[2] = {0, 0}, ls_w = 0;
    if (n == 32) {
        // Full block: vector stores (all outputs 16-byte aligned, r0 a multiple of 32).
        uint32_t ship_pk[16], q_pk[8], d_pk[8], t_pk[8], p_v[32];
#pragma unroll
        for (int i = 0; i < 16; ++i) ship_pk[i] = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) q_pk[i] = d_pk[i] = t_pk[i] = 0;
#pragma unroll
        for (uint32_t j = 0; j < 32; ++j) {
            const GenRow g = gen_row(key, first_row + r0 + j);
            ship_pk[j >> 1] |= (uint32_t)(g.shipdate - kShipDateFrame) << (16 * (j & 1));
            q_pk[j >> 2] |= g.quantity << (8 * (j & 3));
            d_pk[j >> 2] |= g.discount << (8 * (j & 3));
            t_pk[j >> 2] |= g.tax << (8 * (j & 3));
            p_v[j] = g.extprice;
            const uint32_t rf = encode_return_flag(g.returnflag), ls = encode_line_status(g.linestatus);
            pair_w[j >> 4] |= gen_pair_code(group_of(rf, ls)) << (2 * (j & 15));
            rf_w[j >> 4] |= rf << (2 * (j & 15));
            ls_w |= ls << j;
        }
        uint4* s4 = reinterpret_cast<uint4*>(out.shipdate + r0);
#pragma unroll
        for (int i = 0; i < 4; ++i) s4[i] = make_uint4(ship_pk[4 * i], ship_pk[4 * i + 1], ship_pk[4 * i + 2], ship_pk[4 * i + 3]);
        uint4* q4 = reinterpret_cast<uint4*>(out.quantity + r0);
        uint4* d4 = reinterpret_cast<uint4*>(out.discount + r0);
        uint4* t4 = reinterpret_cast<uint4*>(out.tax + r0);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            q4[i] = make_uint4(q_pk[4 * i], q_pk[4 * i + 1], q_pk[4 * i + 2], q_pk[4 * i + 3]);
            d4[i] = make_uint4(d_pk[4 * i], d_pk[4 * i + 1], d_pk[4 * i + 2], d_pk[4 * i + 3]);
            t4[i] = make_uint4(t_pk[4 * i], t_pk[4 * i + 1], t_pk[4 * i + 2], t_pk[4 * i + 3]);
        }
        uint4* p4 = reinterpret_cast<uint4*>(out.extendedprice + r0);
#pragma unroll
        for (int i = 0; i < 8; ++i) p4[i] = make_uint4(p_v[4 * i], p_v[4 * i + 1], p_v[4 * i + 2], p_v[4 * i + 3]);
    } else {
        for (uint32_t j = 0; j < n; ++j) {
            const GenRow g = gen_row(key, first_row + r0 + j);
            out.shipdate[r0 + j] = (uint16_t)(g.shipdate - kShipDateFrame);
            out.quantity[r0 + j] = (uint8_t)g.quantity;
            out.discount[r0 + j] = (uint8_t)g.discount;
            out.tax[r0 + j] = (uint8_t)g.tax;
            out.extendedprice[r0 + j] = g.extprice;
            const uint32_t rf = encode_return_flag(g.returnflag), ls = encode_line_status(g.linestatus);
            pair_w[j >> 4] |= gen_pair_code(group_of(rf, ls)) << (2 * (j & 15));
            rf_w[j >> 4] |= rf << (2 * (j & 15));
            ls_w |= ls << j;
        }
    }
    const uint64_t w16 = r0 / 16;
    const uint32_t nw16 = (n + 15) / 16;
    for (uint32_t i = 0; i < nw16; ++i) {
        if (out.flags) out.flags[w16 + i] = pair_w[i];
        if (out.returnflag) out.returnflag[w16 + i] = rf_w[i];
    }
    if (out.linestatus) out.linestatus[r0 / 32] = ls_w;
}

__global__ void wait_selftest_kernel(uint64_t limit_ns, uint32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t b = ptx::smem_addr(&bar);
    ptx::mbar_init(b, 1);
    ptx::fence_mbar_init();
    // nobody arrives: the phase never completes
    const uint64_t t0 = ptx::globaltimer();
    for (uint32_t i = 1;; ++i) {
        if (ptx::mbar_try_wait(b, 0)) return;
        if ((i & 63u) == 0 && ptx::globaltimer() - t0 > limit_ns) {
            atomicOr(status, ptx::kStatusWaitTimeout);
            return;
        }
    }
}

cudaError_t launch_wait_selftest(uint64_t limit_ns, uint32_t* status, cudaStream_t stream) {
    wait_selftest_kernel<<<1, 1, 0, stream>>>(limit_ns, status);
    return cudaGetLastError();
}

cudaError_t launch_generate_compressed(uint64_t seed, uint64_t first_row, uint64_t rows, const GenCompressedOut& out,
                                       cudaStream_t stream) {
    if (rows == 0) return cudaSuccess;
    const uint64_t blocks32 = (rows + 31) / 32;
    const uint64_t grid = (blocks32 + 255) / 256;
    generate_compressed_kernel<<<(unsigned)grid, 256, 0, stream>>>(gen_key(seed), first_row, rows, out);
    return cudaGetLastError();
}

// One thread per bitmap word: 32 ship dates (64 bytes, four 16-byte loads) -> 32 predicate bits.
__global__ void __launch_bounds__(256) precompute_filter_kernel(const uint16_t* __restrict__ ship, uint64_t rows,
                                                                int32_t cutoff_rel, uint32_t* __restrict__ bitmap) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t r0 = w * 32;
    if (r0 >= rows) return;
    uint32_t bits = 0;
    if (rows - r0 >= 32) {
        const uint4* s4 = reinterpret_cast<const uint4*>(ship + r0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint4 v = __ldg(s4 + i);
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                bits |= ((int32_t)(wv[k] & 0xFFFFu) <= cutoff_rel ? 1u : 0u) << (8 * i + 2 * k);
                bits |= ((int32_t)(wv[k] >> 16) <= cutoff_rel ? 1u : 0u) << (8 * i + 2 * k + 1);
            }
        }
    } else {
        for (uint32_t j = 0; r0 + j < rows; ++j) bits |= ((int32_t)ship[r0 + j] <= cutoff_rel ? 1u : 0u) << j;
    }
    bitmap[w] = bits;
}

cudaError_t launch_precompute_filter(const uint16_t* shipdate, uint64_t rows, int32_t cutoff_rel, uint32_t* bitmap,
                                     cudaStream_t stream) {
    if (rows == 0) return cudaSuccess;
    const uint64_t words = (rows + 31) / 32;
    precompute_filter_kernel<<<(unsigned)((words + 255) / 256), 256, 0, stream>>>(shipdate, rows, cutoff_rel, bitmap);
    return cudaGetLastError();
}

}  // namespace q1
