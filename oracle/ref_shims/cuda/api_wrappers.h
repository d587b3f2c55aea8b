// Stand-in for the cuda-api-wrappers header the reference's kernel headers include; it supplies
// only the three names those headers use (the reference links the real library, absent here).
#pragma once
#include <cstdint>
namespace cuda {
using native_word_t = uint32_t;
enum : unsigned { warp_size = 32 };
using grid_block_dimension_t = unsigned;
}  // namespace cuda
