// Internal interface of the serving loop's kernels (serve_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace q1 {

struct KeyedTableOut {
    uint16_t* shipdate;
    uint8_t* discount;
    uint32_t* extendedprice;
    uint8_t* tax;
    uint8_t* quantity;
    uint32_t* keys;
};

// pair_keys != 0: key = the dictionary code of the row's (rf, ls) pair (AF, NF, NO, RF = 0..3);
// otherwise uniform in [0, num_groups).
cudaError_t launch_generate_keyed_table(uint64_t seed, uint64_t rows, uint32_t pair_keys, uint32_t num_groups,
                                        const KeyedTableOut& out, cudaStream_t stream);

struct CubePassParams {
    const uint16_t* ship;
    const uint8_t* qty;
    const uint8_t* disc;
    const uint8_t* tax;
    const uint32_t* price;
    const uint32_t* codes;       // pair: 2-bit pair codes
    const uint32_t* keys;        // !pair: group keys
    uint8_t pair_group[4];
    uint32_t pair;
    uint32_t num_groups;
    uint32_t d0, days;           // window of ship-day offsets
    uint32_t all_days;           // every row must have ship < all_days (else: domain status)
    uint64_t rows;
    unsigned long long* acc;     // scratch [all days][num_groups][8]
    uint32_t* status;
};
cudaError_t launch_cube_pass(const CubePassParams& prm, int sm_count, cudaStream_t stream);
cudaError_t launch_cube_finalize(const unsigned long long* acc, uint32_t days, uint32_t num_groups,
                                 unsigned long long* cube, cudaStream_t stream);

struct CubeLookup {
    const unsigned long long* cube;   // cumulative cube [days][num_groups][6][lo, hi]
    int32_t day;                      // row to read, -1 = nothing passes
    uint32_t num_groups;
    uint32_t slot;                    // response slot of the request
    uint32_t pad;
};
cudaError_t launch_cube_lookup(const CubeLookup* reqs, uint32_t n, uint32_t words_per_response,
                               unsigned long long* responses, cudaStream_t stream);

}  // namespace q1
