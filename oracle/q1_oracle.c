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
#include <pthread.h>
#include <stdint.h>
#include <string.h>

#include "gen_rows.h"

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

/* ---------------------------------------------------------------------------------------------
 * lineitem text (.tbl) parsing, restated from lineitem::FromFile (cpu/tpch_kit.cpp:155-172):
 *   - one row per line, fields split at '|' (TableReader::tokenize, cpu/tpch_kit.cpp:26-57);
 *     fields 5-11 (1-based) read, the rest skipped;
 *   - decimals "[+-]int[.frac]" -> 100 * int + frac, the fraction's digits read as an integer
 *     (BaseDecimal::parse + Decimal<15,2>::ToValue, cpu/tpch_kit.cpp:100-121, tpch_kit.hpp:52-80);
 *   - characters: exactly one byte (Char, cpu/tpch_kit.hpp:15-23);
 *   - dates "year-month-day" -> day number counted like MonetDB's todate (cpu/monetdb.cpp):
 *     365 * y + leap years before y (+1 for the year-0 convention) + days before the month
 *     (+1 after February of a leap year) + day - 1; 1992-01-01 -> 727563.
 * A line that does not match is malformed: its row is zeroed and counted in *bad, the byte
 * offset of the first one in *first_bad. Returns the number of rows (lines; a final '\n' starts
 * none); rows beyond `capacity` are counted as malformed and not written.
 * ------------------------------------------------------------------------------------------- */
static int tbl_int(const char* t, uint64_t n, uint64_t* p, int64_t* v) {
    int neg = 0;
    if (*p < n && (t[*p] == '+' || t[*p] == '-')) neg = t[(*p)++] == '-';
    int64_t x = 0;
    int nd = 0;
    while (*p < n && t[*p] >= '0' && t[*p] <= '9') {
        if (++nd > 18) return 0;
        x = x * 10 + (t[(*p)++] - '0');
    }
    *v = neg ? -x : x;
    return nd > 0;
}

static int tbl_dec(const char* t, uint64_t n, uint64_t* p, int64_t* v) {
    int64_t i = 0, f = 0;
    if (!tbl_int(t, n, p, &i)) return 0;
    if (*p < n && t[*p] == '.') {
        ++*p;
        if (!tbl_int(t, n, p, &f)) return 0;
    }
    *v = 100 * i + f;
    return 1;
}

static int tbl_sep(const char* t, uint64_t n, uint64_t* p) {
    if (*p >= n || t[*p] != '|') return 0;
    ++*p;
    return 1;
}

static int32_t tbl_day(int64_t y, int64_t m, int64_t d) {
    static const int mdays[13] = {0, 31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    static const int before[13] = {0, 0, 31, 59, 90, 120, 151, 181, 212, 243, 273, 304, 334};
    if (y < 1 || y > 999999 || m < 1 || m > 12 || d < 1) return -1;
    const int leap = (y % 4 == 0) && (y % 100 != 0 || y % 400 == 0);
    if (d > mdays[m] + ((m == 2 && leap) ? 1 : 0)) return -1;
    const int64_t q = y - 1;
    return (int32_t)(365 * y + (q / 4 - q / 100 + q / 400 + 1) + before[m] + ((m > 2 && leap) ? 1 : 0) + d - 1);
}

static int tbl_line(const char* t, uint64_t n, uint64_t p, int32_t* ship, int64_t* q, int64_t* pr, int64_t* di,
                    int64_t* tx, char* rf, char* ls) {
    for (int f = 0; f < 4; ++f) {
        while (p < n && t[p] != '|' && t[p] != '\n') ++p;
        if (!tbl_sep(t, n, &p)) return 0;
    }
    if (!tbl_dec(t, n, &p, q) || !tbl_sep(t, n, &p) || !tbl_dec(t, n, &p, pr) || !tbl_sep(t, n, &p) ||
        !tbl_dec(t, n, &p, di) || !tbl_sep(t, n, &p) || !tbl_dec(t, n, &p, tx) || !tbl_sep(t, n, &p))
        return 0;
    if (p >= n || t[p] == '|' || t[p] == '\n') return 0;
    *rf = t[p++];
    if (!tbl_sep(t, n, &p) || p >= n || t[p] == '|' || t[p] == '\n') return 0;
    *ls = t[p++];
    if (!tbl_sep(t, n, &p)) return 0;
    int64_t y, m, d;
    if (!tbl_int(t, n, &p, &y) || p >= n || t[p++] != '-' || !tbl_int(t, n, &p, &m) || p >= n || t[p++] != '-' ||
        !tbl_int(t, n, &p, &d))
        return 0;
    if (p < n && t[p] != '|' && t[p] != '\n') return 0;
    if (m > 31 || d > 31) return 0;
    *ship = tbl_day(y, m, d);
    return *ship >= 0;
}

uint64_t oracle_parse_tbl(const char* text, uint64_t bytes, int32_t* ship, int64_t* qty, int64_t* price,
                          int64_t* disc, int64_t* tax, char* rf, char* ls, uint64_t capacity, uint64_t* bad,
                          uint64_t* first_bad) {
    uint64_t row = 0, start = 0;
    *bad = 0;
    *first_bad = ~0ull;
    while (start < bytes) {
        uint64_t end = start;
        while (end < bytes && text[end] != '\n') ++end;
        int32_t s = 0;
        int64_t q = 0, pr = 0, di = 0, tx = 0;
        char a = 0, b = 0;
        const int ok = tbl_line(text, bytes, start, &s, &q, &pr, &di, &tx, &a, &b);
        if (row < capacity) {
            if (!ok) s = 0, q = pr = di = tx = 0, a = b = 0;
            ship[row] = s, qty[row] = q, price[row] = pr, disc[row] = di, tax[row] = tx, rf[row] = a, ls[row] = b;
        }
        if (!ok || row >= capacity) {
            ++*bad;
            if (start < *first_bad) *first_bad = start;
        }
        ++row;
        start = end + 1;
    }
    return row;
}

/* ---------------------------------------------------------------------------------------------
 * Reference-typed columns of rows [first_row, first_row + rows) of the seeded generator
 * (gen_rows.h), on `threads` host threads (contiguous row ranges per thread).
 * ------------------------------------------------------------------------------------------- */
struct gen_job {
    uint64_t key, first_row, begin, end;
    int32_t* ship;
    int64_t *qty, *price, *disc, *tax;
    char *rf, *ls;
};

static void* gen_range(void* arg) {
    const struct gen_job* j = (const struct gen_job*)arg;
    for (uint64_t i = j->begin; i < j->end; i++)
        og_row(j->key, j->first_row + i, j->ship + i, j->qty + i, j->price + i, j->disc + i, j->tax + i, j->rf + i,
               j->ls + i);
    return 0;
}

void oracle_generate(uint64_t seed, uint64_t first_row, uint64_t rows, int threads, int32_t* ship, int64_t* qty,
                     int64_t* price, int64_t* disc, int64_t* tax, char* rf, char* ls) {
    enum { MAX_THREADS = 64 };
    if (threads < 1) threads = 1;
    if (threads > MAX_THREADS) threads = MAX_THREADS;
    if ((uint64_t)threads > rows) threads = rows ? (int)rows : 1;
    struct gen_job jobs[MAX_THREADS];
    pthread_t tid[MAX_THREADS];
    int started[MAX_THREADS];
    const uint64_t per = (rows + (uint64_t)threads - 1) / (uint64_t)threads;
    for (int t = 0; t < threads; t++) {
        const uint64_t b = (uint64_t)t * per < rows ? (uint64_t)t * per : rows;
        const uint64_t e = b + per < rows ? b + per : rows;
        struct gen_job j = {og_key(seed), first_row, b, e, ship, qty, price, disc, tax, rf, ls};
        jobs[t] = j;
        started[t] = t > 0 && pthread_create(&tid[t], 0, gen_range, &jobs[t]) == 0;
        if (t > 0 && !started[t]) gen_range(&jobs[t]);
    }
    gen_range(&jobs[0]);
    for (int t = 1; t < threads; t++)
        if (started[t]) pthread_join(tid[t], 0);
}
