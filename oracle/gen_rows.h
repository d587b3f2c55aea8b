/*
 * gen_rows.h -- the seeded synthetic lineitem generator, restated in plain C for the oracle.
 *
 * TEST INFRASTRUCTURE. The product generates the same rows in CUDA/C++; this independent copy
 * (restated from the numpy version in tests/gen_np.py, which the CPU tests compare bit for bit
 * with the product's host and device generators) lets the oracle and the reference's own CPU
 * kernels build their inputs without loading the product library.
 *
 * Counter-based: each field of each row is a pure function of (seed, row, field):
 *   key  = mix64(seed ^ 0x5DEECE66DA3B9F21)
 *   bits = mix64(key + (row * 16 + field) * 0x9E3779B97F4A7C15) >> 32
 *   U(span) = (bits * span) >> 32
 * orderdate U[1992-01-01, 1998-08-02]; shipdate = orderdate + 1 + U(121);
 * receiptdate = shipdate + 1 + U(30); quantity 1 + U(50); unit price 90000 + U(119900) cents;
 * extendedprice = quantity * unit price; discount U(11); tax U(9) (hundredths);
 * returnflag R/A by the top bit of field 7 if receiptdate <= 1995-06-17, else N;
 * linestatus O if shipdate > 1995-06-17, else F. Group keys: field 8.
 */
#ifndef Q1_ORACLE_GEN_ROWS_H
#define Q1_ORACLE_GEN_ROWS_H

#include <stdint.h>

static inline uint64_t og_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t og_key(uint64_t seed) { return og_mix64(seed ^ 0x5DEECE66DA3B9F21ull); }

static inline uint32_t og_bits(uint64_t key, uint64_t row, uint32_t field) {
    return (uint32_t)(og_mix64(key + (row * 16u + field) * 0x9E3779B97F4A7C15ull) >> 32);
}

static inline uint32_t og_uniform(uint32_t bits, uint32_t span) { return (uint32_t)(((uint64_t)bits * span) >> 32); }

enum { OG_ORDER_FIRST = 727563, OG_ORDER_LAST = 729968, OG_CURRENT = 728826 };

/* One row in the reference's column types (cpu/tpch_kit.hpp lineitem): day number, hundredths
 * for quantity / discount / tax, cents for the extended price, one character per flag. */
static inline void og_row(uint64_t key, uint64_t row, int32_t* ship, int64_t* qty, int64_t* price, int64_t* disc,
                          int64_t* tax, char* rf, char* ls) {
    const int32_t order = OG_ORDER_FIRST + (int32_t)og_uniform(og_bits(key, row, 0), OG_ORDER_LAST - OG_ORDER_FIRST + 1);
    const int32_t s = order + 1 + (int32_t)og_uniform(og_bits(key, row, 1), 121);
    const int32_t receipt = s + 1 + (int32_t)og_uniform(og_bits(key, row, 2), 30);
    const int64_t q = 1 + (int64_t)og_uniform(og_bits(key, row, 3), 50);
    const int64_t unit = 90000 + (int64_t)og_uniform(og_bits(key, row, 4), 209899 - 90000 + 1);
    *ship = s;
    *qty = q * 100;
    *price = q * unit;
    *disc = (int64_t)og_uniform(og_bits(key, row, 5), 11);
    *tax = (int64_t)og_uniform(og_bits(key, row, 6), 9);
    *rf = receipt <= OG_CURRENT ? ((og_bits(key, row, 7) >> 31) ? 'R' : 'A') : 'N';
    *ls = s > OG_CURRENT ? 'O' : 'F';
}

#endif
