// Shared host/device definitions: constants, dictionary codes, the synthetic row generator.
//
// Everything here is usable from both nvcc device code and plain g++ host code.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define Q1_HD __host__ __device__ __forceinline__
#else
#define Q1_HD inline
#endif

namespace q1 {

// Frame of reference of the compressed ship date: 1992-01-01 (src/constants.hpp:50).
constexpr int32_t kShipDateFrame = 727563;
// Default predicate: l_shipdate <= 1998-12-01 - 90 days (cpu/common.cpp:60, src/constants.hpp:51).
constexpr int32_t kDefaultCutoffDay = 729999;
// 3 return flags x 2 line stati (src/constants.hpp:54-56).
constexpr int kNumGroups = 6;
constexpr int kNumAggs = 6;

enum AggIndex : int {
    kAggCount = 0,
    kAggQty = 1,
    kAggBasePrice = 2,
    kAggDisc = 3,
    kAggDiscPrice = 4,
    kAggCharge = 5,
};

// DICT encodings of the flags, release-build behaviour of src/data_types.h:52-116:
// A->0, N->1, R->2 (anything else -> 0); F->0, anything else -> 1.
Q1_HD uint32_t encode_return_flag(char c) { return ((c == 'R') ? 2u : 0u) + ((c == 'N') ? 1u : 0u); }
Q1_HD uint32_t encode_line_status(char c) { return (c == 'F') ? 0u : 1u; }
Q1_HD char decode_return_flag(uint32_t code) { return code == 0 ? 'A' : (code == 1 ? 'N' : 'R'); }
Q1_HD char decode_line_status(uint32_t code) { return code == 0 ? 'F' : 'O'; }
// Group index = (rf << 1) + ls (src/kernels/ht_in_global_mem.hpp:41-42).
Q1_HD uint32_t group_of(uint32_t rf_code, uint32_t ls_code) { return (rf_code << 1) + ls_code; }

// ---------------------------------------------------------------------------------------------
// Synthetic lineitem generator.
//
// Counter-based: every field of every row is a pure function of (seed, row, field), so any row
// range can be produced independently on the CPU or the GPU and the two agree bit for bit.
// Distribution (TPC-H-like lineitem restricted to the Q1 columns):
//   orderdate    uniform day in [1992-01-01, 1998-08-02]
//   shipdate     orderdate + U{1..121}
//   receiptdate  shipdate + U{1..30}
//   quantity     U{1..50}                       (stored x100 in the reference-typed column)
//   unit price   uniform cents in [90000, 209899]; extendedprice = quantity * unit price
//   discount     U{0..10} hundredths;  tax U{0..8} hundredths
//   returnflag   'R' or 'A' (p = 1/2 each) if receiptdate <= 1995-06-17, else 'N'
//   linestatus   'O' if shipdate > 1995-06-17, else 'F'
// ---------------------------------------------------------------------------------------------

constexpr int32_t kGenOrderDateFirst = 727563;  // 1992-01-01
constexpr int32_t kGenOrderDateLast = 729968;   // 1998-08-02
constexpr int32_t kGenCurrentDate = 728826;     // 1995-06-17

Q1_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Per-seed key, computed once.
Q1_HD uint64_t gen_key(uint64_t seed) { return mix64(seed ^ 0x5DEECE66DA3B9F21ull); }

// 32 uniform bits for (row, field); fields 0..15.
Q1_HD uint32_t gen_bits(uint64_t key, uint64_t row, uint32_t field) {
    return (uint32_t)(mix64(key + (row * 16u + field) * 0x9E3779B97F4A7C15ull) >> 32);
}

// Uniform integer in [lo, lo + span) from 32 random bits (multiply-shift).
Q1_HD uint32_t gen_uniform(uint32_t bits, uint32_t span) {
    return (uint32_t)(((uint64_t)bits * span) >> 32);
}

enum GenField : uint32_t {
    kFieldOrderDate = 0,
    kFieldShipDelta = 1,
    kFieldReceiptDelta = 2,
    kFieldQuantity = 3,
    kFieldUnitPrice = 4,
    kFieldDiscount = 5,
    kFieldTax = 6,
    kFieldReturnFlag = 7,
    kFieldGroupKey = 8,
};

struct GenRow {
    int32_t shipdate;      // day number
    uint32_t quantity;     // whole units
    uint32_t extprice;     // cents
    uint32_t discount;     // hundredths
    uint32_t tax;          // hundredths
    char returnflag;
    char linestatus;
};

Q1_HD GenRow gen_row(uint64_t key, uint64_t row) {
    GenRow r;
    const int32_t orderdate =
        kGenOrderDateFirst +
        (int32_t)gen_uniform(gen_bits(key, row, kFieldOrderDate), kGenOrderDateLast - kGenOrderDateFirst + 1);
    r.shipdate = orderdate + 1 + (int32_t)gen_uniform(gen_bits(key, row, kFieldShipDelta), 121);
    const int32_t receiptdate = r.shipdate + 1 + (int32_t)gen_uniform(gen_bits(key, row, kFieldReceiptDelta), 30);
    r.quantity = 1 + gen_uniform(gen_bits(key, row, kFieldQuantity), 50);
    const uint32_t unit_price = 90000u + gen_uniform(gen_bits(key, row, kFieldUnitPrice), 209899u - 90000u + 1u);
    r.extprice = r.quantity * unit_price;
    r.discount = gen_uniform(gen_bits(key, row, kFieldDiscount), 11);
    r.tax = gen_uniform(gen_bits(key, row, kFieldTax), 9);
    if (receiptdate <= kGenCurrentDate) {
        r.returnflag = (gen_bits(key, row, kFieldReturnFlag) >> 31) ? 'R' : 'A';
    } else {
        r.returnflag = 'N';
    }
    r.linestatus = (r.shipdate > kGenCurrentDate) ? 'O' : 'F';
    return r;
}

// Fixed pair dictionary of the generator: the four (rf, ls) combinations it can produce,
// in ascending group order: AF(0), NF(2), NO(3), RF(4).
constexpr uint32_t kGenPairCodes = 4;
Q1_HD uint32_t gen_pair_code(uint32_t group) {
    // group 0 -> 0, 2 -> 1, 3 -> 2, 4 -> 3
    return group == 0 ? 0u : (group == 2 ? 1u : (group == 3 ? 2u : 3u));
}
Q1_HD uint32_t gen_pair_group(uint32_t code) {
    return code == 0 ? 0u : (code == 1 ? 2u : (code == 2 ? 3u : 4u));
}

// Group key for the group-key aggregation: uniform over [0, G) or Zipf via an inverse-CDF table
// of G cumulative thresholds (uint32, non-decreasing, last == 0xFFFFFFFF). The key of a row is
// the smallest k with bits <= cdf[k].
Q1_HD uint32_t gen_group_key_uniform(uint64_t key, uint64_t row, uint32_t num_groups) {
    return gen_uniform(gen_bits(key, row, kFieldGroupKey), num_groups);
}
Q1_HD uint32_t gen_group_key_cdf(uint64_t key, uint64_t row, const uint32_t* cdf, uint32_t num_groups) {
    const uint32_t b = gen_bits(key, row, kFieldGroupKey);
    uint32_t lo = 0, hi = num_groups - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (b <= cdf[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

}  // namespace q1
