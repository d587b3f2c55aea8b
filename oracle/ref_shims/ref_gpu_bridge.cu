// Launchers for the reference's own compressed GPU kernels (src/kernels/*, K2-K3, K5-K6, K8-K9,
// K11-K12, K14-K15), compiled unmodified for sm_100a: the same-box GPU comparator. Test and
// measurement infrastructure only; the product never links it.
//
// Launch shape as the reference's execute_query_1_once (src/main.cu:627-650): in_registers uses
// a fixed 256 threads per block (src/kernels/ht_in_registers.cuh:26) and
// ceil(n / (5 tables per warp * warps * tuples_per_thread)) blocks; shared_mem_per_thread is
// capped at 160 threads per block (src/kernels/ht_in_shared_mem_per_thread.cuh:11-21); the
// others use ceil(n / (threads_per_block * tuples_per_thread)) blocks. Aggregates are the
// reference's: uint64 sums (quantity in whole units) and uint32 counts per group, accumulated
// with atomicAdd into caller-zeroed arrays.
#include "kernels/ht_in_global_mem.hpp"
#include "kernels/ht_in_registers.cuh"
#include "kernels/ht_in_registers_per_thread.cuh"
#include "kernels/ht_in_local_mem.cuh"
#include "kernels/ht_in_shared_mem_per_thread.cuh"

#include <cuda_runtime.h>

namespace {

using kernel_t = void (*)(sum_quantity_t*, sum_base_price_t*, sum_discounted_price_t*, sum_charge_t*, sum_discount_t*,
                          cardinality_t*, const compressed::ship_date_t*, const compressed::discount_t*,
                          const compressed::extended_price_t*, const compressed::tax_t*, const compressed::quantity_t*,
                          const bit_container_t*, const bit_container_t*, cardinality_t);
using pushdown_kernel_t = void (*)(sum_quantity_t*, sum_base_price_t*, sum_discounted_price_t*, sum_charge_t*,
                                   sum_discount_t*, cardinality_t*, const bit_container_t*, const compressed::discount_t*,
                                   const compressed::extended_price_t*, const compressed::tax_t*,
                                   const compressed::quantity_t*, const bit_container_t*, const bit_container_t*,
                                   cardinality_t);

}  // namespace

// placement: 0 in_registers, 1 in_registers_per_thread, 2 local_mem, 3 shared_mem_per_thread,
// 4 global. sums: 5 x 6 uint64 (quantity, base_price, discounted_price, charge, discount);
// counts: 6 uint32. ship_or_filter: uint16 ship offsets, or the 1-bit predicate bitmap when
// pushdown != 0. Returns the cudaError_t of the launch.
extern "C" int refgpu_launch_compressed(int placement, int pushdown, unsigned long long* sums, unsigned* counts,
                                        const void* ship_or_filter, const unsigned char* discount,
                                        const unsigned* price, const unsigned char* tax, const unsigned char* quantity,
                                        const unsigned* return_flag, const unsigned* line_status, unsigned num_tuples,
                                        int threads_per_block, int tuples_per_thread, void* stream) {
    if (num_tuples == 0) return 0;
    if (placement < 0 || placement > 4 || threads_per_block < 32 || threads_per_block % 32 || tuples_per_thread < 1)
        return (int)cudaErrorInvalidValue;
    static const kernel_t kernels[5] = {
        cuda::in_registers_ht_tpchQ01_compressed, cuda::in_registers_per_thread_ht_tpchQ01_compressed,
        cuda::in_local_mem_ht_tpchQ01_compressed, cuda::shared_mem_per_thread_ht_tpchQ01_compressed<>,
        cuda::global_ht_tpchQ01_compressed};
    static const pushdown_kernel_t pushdown_kernels[5] = {
        cuda::in_registers_ht_tpchQ01_filter_pushdown_compressed,
        cuda::in_registers_per_thread_ht_tpchQ01_filter_pushdown_compressed,
        cuda::in_local_mem_ht_tpchQ01_filter_pushdown_compressed,
        cuda::shared_mem_per_thread_ht_tpchQ01_pushdown_compressed<>,
        cuda::global_ht_tpchQ01_filter_pushdown_compressed};
    unsigned tpb = (unsigned)threads_per_block;
    unsigned long long blocks;
    if (placement == 0) {
        tpb = cuda::threads_per_block_for_in_registers_hash_table;
        const unsigned long long per_block =
            (unsigned long long)(cuda::warp_size / num_potential_groups) * (tpb / cuda::warp_size) * tuples_per_thread;
        blocks = (num_tuples + per_block - 1) / per_block;
    } else {
        if (placement == 3 && tpb > cuda::max_threads_per_block_for_per_thread_shared_mem)
            tpb = cuda::max_threads_per_block_for_per_thread_shared_mem;
        const unsigned long long per_block = (unsigned long long)tpb * tuples_per_thread;
        blocks = (num_tuples + per_block - 1) / per_block;
    }
    if (blocks > 0x7FFFFFFFull) return (int)cudaErrorInvalidValue;
    uint64_t* s = reinterpret_cast<uint64_t*>(sums);
    cudaStream_t st = (cudaStream_t)stream;
    if (pushdown) {
        pushdown_kernels[placement]<<<(unsigned)blocks, tpb, 0, st>>>(
            s, s + 6, s + 12, s + 18, s + 24, counts, (const bit_container_t*)ship_or_filter, discount, price, tax,
            quantity, return_flag, line_status, num_tuples);
    } else {
        kernels[placement]<<<(unsigned)blocks, tpb, 0, st>>>(
            s, s + 6, s + 12, s + 18, s + 24, counts, (const compressed::ship_date_t*)ship_or_filter, discount, price,
            tax, quantity, return_flag, line_status, num_tuples);
    }
    return (int)cudaGetLastError();
}
