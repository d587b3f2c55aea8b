/*
 * q1_oracle.c -- CPU restatement of the reference's Q1 aggregation, used ONLY as a checker.
 *
 * TEST INFRASTRUCTURE: this file is the oracle. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it. The product (tpchq01_gpu_b200) never
 * links or calls it.
 *
 * Parity is pinned by tests/test_oracle_ref.py against the reference's own CPU kernels
 * (KernelHyPer<true>, KernelX100<kMagic,true,kNoAvx512>) built unmodified from the reference
 * sources into oracle/_ref/ (oracle/Makefile), on identical generated inputs, and against the
 * committed golden fixtures in tests/golden/.
 *
 * Algorithm followed (paths relative to the reference source tree):
 *   - predicate l_shipdate <= cutoff, tuple at a time:      cpu/kernel_hyper.hpp:66-69
 *   - disc_1 = 100 - disc; tax_1 = 100 + tax;
 *     disc_price = disc_1 * price; charge = disc_price * tax_1  (int64, overflow-checked):
 *                                                           cpu/kernel_hyper.hpp:70-75
 *   - sums: int64 quantity / base_price / disc / count, int128 disc_price / charge:
 *                                                           cpu/kernel_hyper.hpp:76-83, cpu/common.hpp:158-165
 *   - group index = (rf_code << 1) + ls_code with the release-build dictionaries
 *     A->0 N->1 R->2, F->0 else->1:                         src/data_types.h:52-80,
 *                                                           src/kernels/ht_in_global_mem.hpp:41-42
 *   - compressed inputs: shipdate - 727563 as uint16, quantity / 100 as uint8, flags
 *     bit-packed LSB first:                                 src/main.cu:773-803, src/bit_operations.hpp:60-154
 *   - filter bitmap: bit i%32 of word i/32 = (shipdate_u16[i] <= cutoff - 727563):
 *                                                           src/main.cu:362-389
 * All outputs are int128 in the product's conventions: sum_qty in hundredths (the compressed
 * inputs carry whole units, so their sums are multiplied by 100 exactly).
 */
#include <stdint.h>
#include <string.h>

typedef __int128 i128;

enum { NG = 6, NA = 6 };
enum { A_COUNT = 0, A_QTY = 1, A_PRICE = 2, A_DISC = 3, A_DISC_PRICE = 4, A_CHARGE = 5 };

static inline unsigned enc_rf(char c) { return ((c == 'R') ? 2u : 0u) + ((c == 'N') ? 1u : 0u); }
static inline unsigned enc_ls(char c) { return (c == 'F') ? 0u : 1u; }

/* One row's contribution, overflow-checked exactly like KernelHyPer<true>. Returns nonzero on
 * int64 overflow of a per-row product. */
static int row_add(i128* agg /* [NA] */, int64_t qty, int64_t price, int64_t disc, int64_t tax) {
    int64_t disc_1, tax_1, disc_price, charge;
    int flag = 0;
    flag |= __builtin_sub_overflow((int64_t)100, disc, &disc_1);
    flag |= __builtin_add_overflow((int64_t)100, tax, &tax_1);
    flag |= __builtin_mul_overflow(disc_1, price, &disc_price);
    flag |= __builtin_mul_overflow(disc_price, tax_1, &charge);
    agg[A_COUNT] += 1;
    agg[A_QTY] += qty;
    agg[A_PRICE] += price;
    agg[A_DISC] += disc;
    agg[A_DISC_PRICE] += disc_price;
    agg[A_CHARGE] += charge;
    return flag;
}

/* Uncompressed, reference-typed columns (src/data_types.h:19-25). out: [NG][NA] int128.
 * Returns nonzero if any per-row product overflowed int64 (HyPer's handle_overflow). */
int oracle_q1_uncompressed(const int32_t* shipdate, const int64_t* discount, const int64_t* extprice,
                           const int64_t* tax, const int64_t* quantity, const char* returnflag,
                           const char* linestatus, uint64_t rows, int32_t cutoff_day, i128* out) {
    memset(out, 0, sizeof(i128) * NG * NA);
    int flag = 0;
    for (uint64_t i = 0; i < rows; i++) {
        if (shipdate[i] <= cutoff_day) {
            const unsigned g = (enc_rf(returnflag[i]) << 1) + enc_ls(linestatus[i]);
            flag |= row_add(out + g * NA, quantity[i], extprice[i], discount[i], tax[i]);
        }
    }
    return flag;
}

static inline unsigned get_bits(const uint32_t* words, uint64_t i, unsigned bits) {
    const unsigned per = 32u / bits;
    return (words[i / per] >> (bits * (unsigned)(i % per))) & ((1u << bits) - 1u);
}

/* Compressed columns (src/main.cu:773-803). flag_packing 0 = 2-bit pair codes + dictionary
 * pair_group[code] -> group; 1 = separate 2-bit returnflag / 1-bit linestatus containers.
 * If filter != NULL the predicate is read from the bitmap (filter-pushdown kernels,
 * src/kernels/ht_in_registers_per_thread.cuh:150-218) instead of shipdate. */
int oracle_q1_compressed(const uint16_t* shipdate, const uint8_t* discount, const uint32_t* extprice,
                         const uint8_t* tax, const uint8_t* quantity, int flag_packing,
                         const uint32_t* flags, const uint8_t* pair_group, const uint32_t* returnflag,
                         const uint32_t* linestatus, const uint32_t* filter, uint64_t rows,
                         int32_t cutoff_day, i128* out) {
    memset(out, 0, sizeof(i128) * NG * NA);
    const int64_t cut = (int64_t)cutoff_day - 727563;
    int flag = 0;
    for (uint64_t i = 0; i < rows; i++) {
        int pass;
        if (filter) {
            pass = (int)get_bits(filter, i, 1);
        } else {
            pass = (int64_t)shipdate[i] <= cut;
        }
        if (!pass) continue;
        unsigned g;
        if (flag_packing == 0) {
            g = pair_group[get_bits(flags, i, 2)];
        } else {
            g = (get_bits(returnflag, i, 2) << 1) + get_bits(linestatus, i, 1);
        }
        if (g >= NG) continue; /* code 3 of the 2-bit return flag has no group */
        flag |= row_add(out + g * NA, (int64_t)quantity[i] * 100, (int64_t)extprice[i],
                        (int64_t)discount[i], (int64_t)tax[i]);
    }
    return flag;
}

/* Group-key aggregation over compressed columns: the group of a row is key[i] < num_groups
 * instead of the flags. out: [num_groups][NA]. */
int oracle_q1_groupkey(const uint16_t* shipdate, const uint8_t* discount, const uint32_t* extprice,
                       const uint8_t* tax, const uint8_t* quantity, const uint32_t* key,
                       uint32_t num_groups, uint64_t rows, int32_t cutoff_day, i128* out) {
    memset(out, 0, sizeof(i128) * (size_t)num_groups * NA);
    const int64_t cut = (int64_t)cutoff_day - 727563;
    int flag = 0;
    for (uint64_t i = 0; i < rows; i++) {
        if ((int64_t)shipdate[i] > cut) continue;
        const uint32_t g = key[i];
        if (g >= num_groups) { flag |= 2; continue; }
        flag |= row_add(out + (size_t)g * NA, (int64_t)quantity[i] * 100, (int64_t)extprice[i],
                        (int64_t)discount[i], (int64_t)tax[i]);
    }
    return flag;
}

/* Filter precomputation restated from src/main.cu:362-389 (chunk-aligned start). */
void oracle_precompute_filter(const uint16_t* shipdate, uint64_t rows, int32_t cutoff_day, uint32_t* bitmap) {
    const int64_t cut = (int64_t)cutoff_day - 727563;
    const uint64_t words = (rows + 31) / 32;
    for (uint64_t w = 0; w < words; w++) {
        uint32_t bits = 0;
        for (unsigned j = 0; j < 32 && w * 32 + j < rows; j++) {
            bits |= (uint32_t)((int64_t)shipdate[w * 32 + j] <= cut) << j;
        }
        bitmap[w] = bits;
    }
}

/* Compression restated from src/main.cu:773-803 for cross-checking the product compressor:
 * returns nonzero if a value would not round-trip. Separate-container packing only. */
int oracle_compress_separate(const int32_t* shipdate, const int64_t* discount, const int64_t* extprice,
                             const int64_t* tax, const int64_t* quantity, const char* returnflag,
                             const char* linestatus, uint64_t rows, uint16_t* c_ship, uint8_t* c_disc,
                             uint32_t* c_price, uint8_t* c_tax, uint8_t* c_qty, uint32_t* c_rf,
                             uint32_t* c_ls) {
    int bad = 0;
    memset(c_rf, 0, sizeof(uint32_t) * ((rows + 15) / 16));
    memset(c_ls, 0, sizeof(uint32_t) * ((rows + 31) / 32));
    for (uint64_t i = 0; i < rows; i++) {
        const int64_t s = (int64_t)shipdate[i] - 727563;
        c_ship[i] = (uint16_t)s;
        c_disc[i] = (uint8_t)discount[i];
        c_price[i] = (uint32_t)extprice[i];
        c_tax[i] = (uint8_t)tax[i];
        c_qty[i] = (uint8_t)(quantity[i] / 100);
        bad |= (int64_t)c_ship[i] != s;
        bad |= (int64_t)c_disc[i] != discount[i];
        bad |= (int64_t)c_price[i] != extprice[i];
        bad |= (int64_t)c_tax[i] != tax[i];
        bad |= (int64_t)c_qty[i] * 100 != quantity[i];
        c_rf[i / 16] |= enc_rf(returnflag[i]) << (2 * (i % 16));
        c_ls[i / 32] |= enc_ls(linestatus[i]) << (i % 32);
    }
    return bad;
}
