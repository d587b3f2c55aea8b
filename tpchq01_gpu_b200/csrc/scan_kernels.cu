// Q1 scan kernels for sm_100a: date predicate + (returnflag, linestatus) group-by with exact
// fixed-point sums, over HBM-resident columns.
//
// Replaces the 15 __global__ kernels of the reference (src/kernels/*: 5 table placements x
// {uncompressed, compressed, filter-pushdown compressed}); the per-row arithmetic is that of
// every reference kernel (e.g. src/kernels/ht_in_registers_per_thread.cuh:38-60):
//   disc_1 = 100 - disc, disc_price = disc_1 * price, charge = disc_price * (100 + tax),
//   group = (rf << 1) + ls; sums of quantity, price, disc_price, charge, disc and a count.
//
// Structure (one design for every layout and placement):
//   * persistent grid, one CTA per SM, each CTA = 1 producer warp + W consumer warps;
//   * the producer streams tiles of R rows, every column of the tile with one
//     cp.async.bulk (TMA bulk copy, evict-first L2 policy) into an S-stage shared-memory ring,
//     completion tracked on mbarriers; consumers release a stage with one arrive per warp;
//   * consumers decode the rows from shared memory in registers (predicate, group code,
//     quantity/discount/tax bytes, price) and accumulate according to the placement;
//   * one 128-bit atomic per CTA per (group, aggregate) into the caller's buffer.
// Every wait is bounded (q1_ptx.cuh, kWaitLimitNs); on expiry the kernel records
// kStatusWaitTimeout in the status word, drains its own copies and returns.
//
// Fast domain: discount <= 100 (so 100 - d >= 0), tax <= 255, extendedprice and quantity < 2^32.
// Then every per-row product fits 64 bits unsigned (charge < 2^47.2) and per-thread 64-bit
// partials cannot wrap for launches of up to 2^31 rows (the host splits longer launches).
// Compressed columns cannot leave it except by a discount above 100 or a ship offset above 32767,
// which set kStatusDomain (the host reports Q1_ERR_DOMAIN). The reference-typed (uncompressed)
// columns are int64: a passing row outside the fast domain is summed exactly by wide_row (signed
// 128-bit arithmetic, 128-bit atomics straight into the output), and only a row whose int64
// products overflow, which the reference's KernelHyPer reports through handle_overflow
// (cpu/kernel_hyper.hpp:65-91), sets kStatusDomain.
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_common.cuh"
#include "q1_kernels.h"
#include "q1_ptx.cuh"
#include "q1_quad.cuh"

namespace q1 {

using namespace ptx;

// ---------------------------------------------------------------------------------------------
// Layouts
// ---------------------------------------------------------------------------------------------

// Column order inside a tile: ship (or filter), qty, disc, tax, price, flags... (see q1_kernels.h)
template <int L>
struct LayoutTraits;

template <>
struct LayoutTraits<kLayPair> {
    static constexpr int kCols = 6;
    static constexpr uint64_t kBitsWord = 0x0000022008080810ull;  // bits per column, one byte each: {16, 8, 8, 8, 32, 2, 0}
    static constexpr int kRowsPerStep = 4;
    static constexpr int kCodes = 4;   // 2-bit pair dictionary
    static constexpr bool kFilter = false;
    static constexpr bool kWideQty = false;
};
template <>
struct LayoutTraits<kLayPairFilter> {
    static constexpr int kCols = 6;
    static constexpr uint64_t kBitsWord = 0x0000022008080801ull;  // bits per column, one byte each: {1, 8, 8, 8, 32, 2, 0}
    static constexpr int kRowsPerStep = 4;
    static constexpr int kCodes = 4;
    static constexpr bool kFilter = true;
    static constexpr bool kWideQty = false;
};
template <>
struct LayoutTraits<kLaySep> {
    static constexpr int kCols = 7;
    static constexpr uint64_t kBitsWord = 0x0001022008080810ull;  // bits per column, one byte each: {16, 8, 8, 8, 32, 2, 1}
    static constexpr int kRowsPerStep = 4;
    static constexpr int kCodes = 6;   // (rf << 1) + ls
    static constexpr bool kFilter = false;
    static constexpr bool kWideQty = false;
};
template <>
struct LayoutTraits<kLaySepFilter> {
    static constexpr int kCols = 7;
    static constexpr uint64_t kBitsWord = 0x0001022008080801ull;  // bits per column, one byte each: {1, 8, 8, 8, 32, 2, 1}
    static constexpr int kRowsPerStep = 4;
    static constexpr int kCodes = 6;
    static constexpr bool kFilter = true;
    static constexpr bool kWideQty = false;
};
template <>
struct LayoutTraits<kLayUncomp> {
    static constexpr int kCols = 7;
    static constexpr uint64_t kBitsWord = 0x0008084040404020ull;  // bits per column, one byte each: {32, 64, 64, 64, 64, 8, 8}
    static constexpr int kRowsPerStep = 2;
    static constexpr int kCodes = 6;
    static constexpr bool kFilter = false;
    static constexpr bool kWideQty = true;
};

template <int L>
__host__ __device__ constexpr uint32_t col_bits(int c) {
    return (uint32_t)((LayoutTraits<L>::kBitsWord >> (8 * c)) & 0xFFu);
}
template <int L>
__host__ __device__ constexpr uint32_t col_offset(int c, uint32_t R) {
    uint32_t off = 0;
    for (int i = 0; i < c; ++i) off += R * col_bits<L>(i) / 8u;
    return off;
}
template <int L>
__host__ __device__ constexpr uint32_t stage_bytes(uint32_t R) {
    return col_offset<L>(LayoutTraits<L>::kCols, R);
}

// ---------------------------------------------------------------------------------------------
// Accumulators (table placements)
// ---------------------------------------------------------------------------------------------

// Per-row decoded values handed to a placement:
//   c  group code (0..kCodes-1) of a passing row, or a value >= kCodes for a filtered row
//   q  quantity (whole units for compressed, hundredths for uncompressed)
//   d  discount, a = 100 - d, ab = a * (100 + tax), p = extendedprice

// Aggregates of one group, per thread, in registers.
template <bool kWideQty>
struct GroupRegs {
    uint64_t p, dp, ch;
    uint64_t qd64;      // packed: sum q (low 32) | sum d (high 32)   [!kWideQty]
    uint64_t q64;       // sum q                                      [kWideQty]
    uint32_t qd, d32, cnt;

    __device__ __forceinline__ void zero() {
        p = dp = ch = qd64 = q64 = 0;
        qd = d32 = cnt = 0;
    }
    __device__ __forceinline__ void add(bool hit, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t pr) {
        const uint32_t pg = hit ? pr : 0u;
        if (kWideQty) {
            q64 = mad_wide(hit ? q : 0u, 1u, q64);
            d32 += hit ? d : 0u;
        } else {
            qd += hit ? (q | (d << 16)) : 0u;
        }
        cnt += hit ? 1u : 0u;
        p += pg;
        dp = mad_wide(a, pg, dp);
        ch = mad_wide(ab, pg, ch);
    }
    // Move the 16-bit packed partials into 64 bits; needed at least every 256 rows.
    __device__ __forceinline__ void fold() {
        if (!kWideQty) {
            qd64 += (uint64_t)(qd & 0xFFFFu) | ((uint64_t)(qd >> 16) << 32);
            qd = 0;
        }
    }
    // Aggregate values in q1 order (count, qty, price, disc, disc_price, charge); after fold().
    __device__ __forceinline__ uint64_t value(int agg) const {
        switch (agg) {
            case kAggCount: return cnt;
            case kAggQty: return kWideQty ? q64 : (qd64 & 0xFFFFFFFFull);
            case kAggBasePrice: return p;
            case kAggDisc: return kWideQty ? (uint64_t)d32 : (qd64 >> 32);
            case kAggDiscPrice: return dp;
            default: return ch;
        }
    }
};

// Code of row r of a quad (0..7 = group code, 7 also = filtered out) for row-wise placements.
__device__ __forceinline__ uint32_t quad_code(const Quad& x, int r) {
    const uint32_t b = (x.OH >> (8 * r)) & 0xFFu;
    return b ? (uint32_t)(__ffs(b) - 1) : 7u;
}

// Aggregates of one group, per thread, fed a quad at a time. W1 (byte r = 1 iff row r is in the
// group) drives three byte dot products (count, quantity, discount of 4 rows in one dp4a each);
// the price products use the FMA pipe: pg = m * p (m in {0,1}), then wide multiply-adds.
// 32-bit count/quantity/discount partials stay exact: a thread adds at most 2^15 rows per launch
// (the host caps rows per launch at 2^15 per consumer thread), so quantity <= 255 * 2^15.
struct GroupQuadRegs {
    uint64_t p, dp, ch;
    uint32_t cnt, q, d;
    __device__ __forceinline__ void zero() {
        p = dp = ch = 0;
        cnt = q = d = 0;
    }
    __device__ __forceinline__ void add_quad(uint32_t W1, const Quad& x) {
        cnt = __dp4a(W1, 0x01010101u, cnt);
        q = __dp4a(W1, x.Q, q);
        d = __dp4a(W1, x.D, d);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t m = __byte_perm(W1, 0u, 0x4440u | (uint32_t)r);
            const uint32_t pg = m * x.p[r];
            p += pg;
            dp = mad_wide(x.a[r], pg, dp);
            ch = mad_wide(x.ab[r], pg, ch);
        }
    }
    __device__ __forceinline__ uint64_t value(int agg) const {
        switch (agg) {
            case kAggCount: return cnt;
            case kAggQty: return q;
            case kAggBasePrice: return p;
            case kAggDisc: return d;
            case kAggDiscPrice: return dp;
            default: return ch;
        }
    }
};

// Shared-memory reduction target of a CTA: [codes][6] x (lo, hi).
struct CtaRed {
    unsigned long long* v;
    __device__ __forceinline__ void add(int code, int agg, uint64_t lo, uint64_t hi) {
        atomic_add_u128_shared(v + 2 * (code * kNumAggs + agg), lo, hi);
    }
};

// --- in_registers_per_thread: every thread owns all groups in registers; a row updates the
// matching group through predicated (select) arithmetic over all groups
// (src/kernels/ht_in_registers_per_thread.cuh:11-79).
template <int G, bool kWideQty>
struct AccPerThread {
    // With the six (returnflag, linestatus) groups of the separate flag layout, A/O and R/O (codes
    // 1 and 5) need a receipt date before the ship date and do not occur in TPC-H data: their rows
    // go straight into the CTA's 128-bit shared table (red) behind one warp vote, so that only the
    // four other groups' planes take registers (a kernel of 128 registers a thread, 12 warps).
    static constexpr bool kCold = (G == 6) && !kWideQty;
    static constexpr int kPlanes = kWideQty ? 1 : (kCold ? 4 : G);
    GroupRegs<kWideQty> g[kWideQty ? G : 1];      // row-wise path (uncompressed layout)
    GroupPlanes gq[kPlanes];                      // quad path (compressed layouts)
    unsigned long long* red;                      // the CTA's [G][6][lo, hi] table (cold groups)
    // group of plane slot s: the codes themselves, or with cold groups AF, NF, NO, RF
    static __device__ __forceinline__ constexpr uint32_t group_of(int s) {
        return kCold ? (s == 0 ? 0u : (uint32_t)s + 1u) : (uint32_t)s;
    }
    static __device__ __forceinline__ constexpr bool cold(int grp) { return kCold && (grp == 1 || grp == 5); }
    __device__ __forceinline__ void init(uint32_t, uint32_t, uint8_t*, unsigned long long* cta_red) {
        red = cta_red;
#pragma unroll
        for (int i = 0; i < (kWideQty ? G : 1); ++i) g[i].zero();
#pragma unroll
        for (int i = 0; i < kPlanes; ++i) gq[i].zero();
    }
    // One passing row of a cold group, exactly, into the CTA's table.
    __device__ __forceinline__ void cold_row(uint32_t grp, uint32_t q, uint32_t d, uint32_t a, uint32_t ab,
                                             uint32_t p) {
        unsigned long long* v = red + 2 * (grp * kNumAggs);
        atomic_add_u128_shared(v + 2 * kAggCount, 1, 0);
        atomic_add_u128_shared(v + 2 * kAggQty, q, 0);
        atomic_add_u128_shared(v + 2 * kAggBasePrice, p, 0);
        atomic_add_u128_shared(v + 2 * kAggDisc, d, 0);
        atomic_add_u128_shared(v + 2 * kAggDiscPrice, (uint64_t)a * p, 0);
        atomic_add_u128_shared(v + 2 * kAggCharge, (uint64_t)ab * p, 0);
    }
    __device__ __forceinline__ void add(uint32_t c, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t p) {
        if constexpr (kWideQty) {
#pragma unroll
            for (int i = 0; i < G; ++i) g[i].add(c == (uint32_t)i, q, d, a, ab, p);
        } else {
            if (kCold && (c == 1u || c == 5u)) {
                cold_row(c, q, d, a, ab, p);
                return;
            }
            // one row through the quad path (tail rows)
            Quad x;
            x.OH = c < (uint32_t)G ? (1u << c) : 0u;
            x.Q = q;
            x.D = d;
            x.A = a;
            x.P[0] = p & 0xFFu;
            x.P[1] = (p >> 8) & 0xFFu;
            x.P[2] = (p >> 16) & 0xFFu;
            x.P[3] = p >> 24;
            x.ABL = ab & 0xFFu;
            x.ABH = ab >> 8;
#pragma unroll
            for (int i = 0; i < kPlanes; ++i) gq[i].add_quad(x.OH, group_of(i), x);   // no warp vote: lanes diverge here
        }
    }
    // Called by all lanes of the warp.
    template <bool kTop>
    __device__ __forceinline__ void add_quad_planes(const Quad& x) {
#pragma unroll
        for (int i = 0; i < kPlanes; ++i) gq[i].template add_quad<kTop>(x.OH, group_of(i), x);
        if constexpr (kCold) {
            if (__any_sync(0xffffffffu, x.OH & 0x22222222u)) {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const uint32_t b = (x.OH >> (8 * r)) & 0x22u;
                    if (b)
                        cold_row((b & 2u) ? 1u : 5u, (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu, x.a[r],
                                 x.ab[r], x.p[r]);
                }
            }
        }
    }
    __device__ __forceinline__ void add_quad(const Quad& x) {
        if constexpr (!kWideQty) {
            // the prices' top byte plane is zero for the whole warp unless a price is >= 2^24
            if (__any_sync(0xffffffffu, x.P[3])) add_quad_planes<true>(x);
            else add_quad_planes<false>(x);
        }
    }
    __device__ __forceinline__ void fold() {
        if constexpr (kWideQty) {
#pragma unroll
            for (int i = 0; i < G; ++i) g[i].fold();
        }
    }
    // plane slot of group i (not called for cold groups)
    static __device__ __forceinline__ constexpr int slot_of(int i) { return kCold ? (i == 0 ? 0 : i - 1) : i; }
    // The thread's partial of group i (0 for a cold group: its rows are in the CTA table already).
    __device__ __forceinline__ uint64_t value(int i, int a) const {
        if constexpr (kWideQty) return g[i].value(a);
        else return cold(i) ? 0ull : gq[slot_of(i)].value(a);
    }
    __device__ __forceinline__ void zero_group(int i) {
        if constexpr (kWideQty) g[i].zero();
        else if (!cold(i)) gq[slot_of(i)].zero();
    }
    // whether this thread sums the rows of group code c (every thread reads every row it is given)
    __device__ __forceinline__ bool owns(uint32_t) const { return true; }
    template <class P>
    __device__ __forceinline__ void tile_done(const P&, uint32_t) {}
    template <class P>
    __device__ __forceinline__ void finish(const P&, uint32_t) {}
    __device__ __forceinline__ void flush(CtaRed red, uint32_t lane) {
        fold();
#pragma unroll
        for (int i = 0; i < G; ++i) {
            if (cold(i)) continue;
#pragma unroll
            for (int a = 0; a < kNumAggs; ++a) {
                uint64_t lo = value(i, a), hi = 0;
                warp_sum_u128(lo, hi);
                if (lane == 0) red.add(i, a, lo, hi);
            }
        }
    }
};

// --- in_registers ("warp-lane tables", src/kernels/ht_in_registers.cuh:30-121): the lanes of a
// warp form floor(32/G) tables of G lanes; lane (table, g) keeps only group g in registers; all
// G lanes of a table read the same rows (a shared-memory broadcast, so unlike the reference no
// row is fetched from DRAM more than once) and each adds the rows of its own group.
template <int G, bool kWideQty>
struct AccWarpLane {
    GroupRegs<kWideQty> r;
    GroupQuadRegs rq;
    uint32_t my;
    __device__ __forceinline__ void init(uint32_t lane, uint32_t, uint8_t*, unsigned long long*) {
        r.zero();
        rq.zero();
        my = lane % G;
    }
    __device__ __forceinline__ void add(uint32_t c, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t p) {
        if constexpr (kWideQty) {
            r.add(c == my, q, d, a, ab, p);
        } else {
            Quad x;
            x.OH = c == my ? 1u << my : 0u;
            x.Q = q;
            x.D = d;
            x.a[0] = a;
            x.ab[0] = ab;
            x.p[0] = p;
            x.a[1] = x.a[2] = x.a[3] = x.ab[1] = x.ab[2] = x.ab[3] = x.p[1] = x.p[2] = x.p[3] = 0;
            add_quad(x);
        }
    }
    __device__ __forceinline__ void add_quad(const Quad& x) { rq.add_quad((x.OH >> my) & 0x01010101u, x); }
    __device__ __forceinline__ void fold() { r.fold(); }
    // all G lanes of a table read the same rows; the lane of group c sums them
    __device__ __forceinline__ bool owns(uint32_t c) const { return c == my; }
    template <class P>
    __device__ __forceinline__ void tile_done(const P&, uint32_t) {}
    template <class P>
    __device__ __forceinline__ void finish(const P&, uint32_t) {}
    __device__ __forceinline__ void flush(CtaRed red, uint32_t lane) {
        fold();
        if (lane < (32u / G) * G) {
#pragma unroll
            for (int a = 0; a < kNumAggs; ++a) red.add((int)my, a, kWideQty ? r.value(a) : rq.value(a), 0);
        }
    }
};

// Sums of the rows of one group in a quad (W1: byte r is 1 iff row r is in the group): the packed
// word count | quantity << 16 | discount << 39 (a thread adds at most 2^15 rows per launch, so
// count < 2^16, quantity <= 255 * 2^15 < 2^23, discount <= 100 * 2^15 < 2^22) and price,
// (100 - d) price and (100 - d)(100 + t) price.
struct QuadGroupSums {
    uint64_t w0, p, dp, ch;
};
__device__ __forceinline__ QuadGroupSums quad_group_sums(uint32_t W1, const Quad& x) {
    QuadGroupSums s{0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint32_t pg = __byte_perm(W1, 0u, 0x4440u | (uint32_t)r) * x.p[r];
        s.p += pg;
        s.dp = mad_wide(x.a[r], pg, s.dp);
        s.ch = mad_wide(x.ab[r], pg, s.ch);
    }
    s.w0 = (uint64_t)__popc(W1) | ((uint64_t)__dp4a(W1, x.Q, 0u) << 16) | ((uint64_t)__dp4a(W1, x.D, 0u) << 39);
    return s;
}

// --- local_mem (src/kernels/ht_in_local_mem.cuh:11-74): per-thread tables indexed by the row's
// group, which places them in (L1-cached) local memory. A group's entry is four 64-bit words
// (five for reference-typed columns, whose quantity needs a word of its own): the count, quantity
// and discount share one word (see quad_group_sums), then price, (100 - d) price and
// (100 - d)(100 + t) price. Compressed quads are added group by group, every lane of the warp at
// the same group at a time: the group's four rows are summed in registers and its entry is
// read and written once, by accesses that coalesce across the warp (a row-by-row update at each
// row's own group scatters the warp's accesses over the table: 2.8 sectors per row each way,
// L1-bound). Reference-typed rows come one at a time and update their group's entry.
template <int G, bool kWideQty>
struct AccLocal {
    static constexpr int kWords = kWideQty ? 5 : 4;
    static constexpr int kQtyShift = 16, kDiscShift = kWideQty ? 16 : 39;
    uint64_t t[G][kWords];   // [0] count | quantity << 16 | discount << 39 (or count | discount << 16), [1] p,
                             // [2] (100-d) p, [3] (100-d)(100+t) p, [4] quantity (reference-typed columns)
    __device__ __forceinline__ void init(uint32_t, uint32_t, uint8_t*, unsigned long long*) {
        for (int i = 0; i < G; ++i)
            for (int j = 0; j < kWords; ++j) t[i][j] = 0;
    }
    __device__ __forceinline__ void add(uint32_t c, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t p) {
        if (c < (uint32_t)G) {
            if constexpr (kWideQty) {
                t[c][0] += 1ull | ((uint64_t)d << kDiscShift);
                t[c][4] += q;
            } else {
                t[c][0] += 1ull | ((uint64_t)q << kQtyShift) | ((uint64_t)d << kDiscShift);
            }
            t[c][1] += p;
            t[c][2] = mad_wide(a, p, t[c][2]);
            t[c][3] = mad_wide(ab, p, t[c][3]);
        }
    }
    __device__ __forceinline__ void add_quad(const Quad& x) {
        // not unrolled, so that the table stays in local memory, indexed by the loop's group
#pragma unroll 1
        for (int g = 0; g < G; ++g) {
            const uint32_t W1 = (x.OH >> g) & 0x01010101u;
            if (W1) {
                const QuadGroupSums q = quad_group_sums(W1, x);
                t[g][0] += q.w0;
                t[g][1] += q.p;
                t[g][2] += q.dp;
                t[g][3] += q.ch;
            }
        }
    }
    __device__ __forceinline__ void fold() {}
    __device__ __forceinline__ bool owns(uint32_t) const { return true; }
    template <class P>
    __device__ __forceinline__ void tile_done(const P&, uint32_t) {}
    template <class P>
    __device__ __forceinline__ void finish(const P&, uint32_t) {}
    __device__ __forceinline__ void flush(CtaRed red, uint32_t lane) {
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const uint64_t w0 = t[i][0];
            const uint64_t qty = kWideQty ? t[i][kWords - 1] : (w0 >> kQtyShift) & ((1ull << 23) - 1);
            const uint64_t vals[kNumAggs] = {w0 & 0xFFFFull, qty, t[i][1], w0 >> kDiscShift, t[i][2], t[i][3]};
#pragma unroll
            for (int a = 0; a < kNumAggs; ++a) {
                uint64_t lo = vals[a], hi = 0;
                warp_sum_u128(lo, hi);
                if (lane == 0) red.add(i, a, lo, hi);
            }
        }
    }
};

// --- shared_mem_per_thread (src/kernels/ht_in_shared_mem_per_thread.cuh:23-118): per-thread
// tables in shared memory, laid out [word][group][thread] so a warp's accesses are bank-conflict
// free. A group's entry holds the same words as the local_mem table, and compressed quads are
// added group by group in the same way: every lane at the same group, one read-modify-write per
// word and group.
template <int G, bool kWideQty>
struct AccSharedPerThread {
    static constexpr int kWords = kWideQty ? 5 : 4;
    static constexpr int kDiscShift = kWideQty ? 16 : 39;
    uint64_t* tab;       // kWords * G * T entries: [w0, p, dp, ch, (quantity)][group][thread]
    uint32_t tid, nthreads;
    __device__ __forceinline__ void init(uint32_t, uint32_t consumer_tid, uint8_t* scratch, unsigned long long*) {
        tid = consumer_tid;
        nthreads = blockDim.x - 32;
        tab = reinterpret_cast<uint64_t*>(scratch);
        for (int i = 0; i < kWords * G; ++i) tab[i * nthreads + tid] = 0;
    }
    __device__ __forceinline__ void add(uint32_t c, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t p) {
        if (c < (uint32_t)G) {
            const uint32_t base = c * nthreads + tid;
            const uint32_t stride = G * nthreads;
            if constexpr (kWideQty) {
                tab[base] += 1ull | ((uint64_t)d << kDiscShift);
                tab[base + 4 * stride] += q;
            } else {
                tab[base] += 1ull | ((uint64_t)q << 16) | ((uint64_t)d << kDiscShift);
            }
            tab[base + stride] += p;
            tab[base + 2 * stride] = mad_wide(a, p, tab[base + 2 * stride]);
            tab[base + 3 * stride] = mad_wide(ab, p, tab[base + 3 * stride]);
        }
    }
    __device__ __forceinline__ void add_quad(const Quad& x) {
        const uint32_t stride = G * nthreads;
#pragma unroll 1
        for (int g = 0; g < G; ++g) {
            const uint32_t W1 = (x.OH >> g) & 0x01010101u;
            if (W1) {
                const QuadGroupSums q = quad_group_sums(W1, x);
                const uint32_t base = g * nthreads + tid;
                tab[base] += q.w0;
                tab[base + stride] += q.p;
                tab[base + 2 * stride] += q.dp;
                tab[base + 3 * stride] += q.ch;
            }
        }
    }
    __device__ __forceinline__ void fold() {}
    // whether this thread sums the rows of group code c (every thread reads every row it is given)
    __device__ __forceinline__ bool owns(uint32_t) const { return true; }
    template <class P>
    __device__ __forceinline__ void tile_done(const P&, uint32_t) {}
    template <class P>
    __device__ __forceinline__ void finish(const P&, uint32_t) {}
    __device__ __forceinline__ void flush(CtaRed red, uint32_t lane) {
        const uint32_t stride = G * nthreads;
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const uint32_t base = i * nthreads + tid;
            const uint64_t w0 = tab[base];
            const uint64_t qty = kWideQty ? tab[base + 4 * stride] : (w0 >> 16) & ((1ull << 23) - 1);
            const uint64_t vals[kNumAggs] = {w0 & 0xFFFFull, qty, tab[base + stride], w0 >> kDiscShift,
                                             tab[base + 2 * stride], tab[base + 3 * stride]};
#pragma unroll
            for (int a = 0; a < kNumAggs; ++a) {
                uint64_t lo = vals[a], hi = 0;
                warp_sum_u128(lo, hi);
                if (lane == 0) red.add(i, a, lo, hi);
            }
        }
    }
};

// --- global (src/kernels/ht_in_global_mem.hpp:11-52): no thread- or block-private table; the
// aggregates live only in the global output, updated by atomics all through the scan. The
// reference issues 6 atomics per row; here each warp write-combines its rows of
// kGlobalFlushTiles tiles in a register buffer, then issues one 128-bit atomic add per
// (group, aggregate) straight into the global table and empties the buffer.
template <int G, bool kWideQty>
struct AccGlobal {
    // A warp's flush of one sum is a 64-bit warp reduction; the kernel bounds the rows a lane
    // buffers between flushes so that it cannot wrap.
    static_assert(kGlobalFlushTiles >= 1, "flush cadence");
    AccPerThread<G, kWideQty> buf;
    uint32_t tiles;
    __device__ __forceinline__ void init(uint32_t a, uint32_t b, uint8_t* s, unsigned long long* r) {
        buf.init(a, b, s, r);
        tiles = 0;
    }
    __device__ __forceinline__ void add(uint32_t c, uint32_t q, uint32_t d, uint32_t a, uint32_t ab, uint32_t p) {
        buf.add(c, q, d, a, ab, p);
    }
    __device__ __forceinline__ void add_quad(const Quad& x) { buf.add_quad(x); }
    __device__ __forceinline__ void fold() { buf.fold(); }
    __device__ __forceinline__ bool owns(uint32_t) const { return true; }
    // Called by all lanes after each tile (warp-uniform count).
    template <class P>
    __device__ __forceinline__ void tile_done(const P& prm, uint32_t lane) {
        buf.fold();
        if (++tiles < kGlobalFlushTiles) return;
        to_global(prm, lane);
    }
    template <class P>
    __device__ __forceinline__ void finish(const P& prm, uint32_t lane) {
        buf.fold();
        if (tiles) to_global(prm, lane);
    }
    template <class P>
    __device__ __forceinline__ void to_global(const P& prm, uint32_t lane) {
        tiles = 0;
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const int grp = G == 4 ? prm.pair_group[i] : i;
#pragma unroll
            for (int a = 0; a < kNumAggs; ++a) {
                uint64_t v = warp_sum_u64(buf.value(i, a));
                if (a == kAggQty) v *= prm.qty_scale;
                if (lane == (uint32_t)((i * kNumAggs + a) & 31)) atomic_add_u128(prm.out + 2 * (grp * kNumAggs + a), v, 0);
            }
            buf.zero_group(i);
        }
    }
    __device__ __forceinline__ void flush(CtaRed, uint32_t) {}
};

template <int P, int G, bool W>
struct AccSel;
template <int G, bool W> struct AccSel<kPlaceInRegisters, G, W> { using T = AccWarpLane<G, W>; };
template <int G, bool W> struct AccSel<kPlaceInRegistersPerThread, G, W> { using T = AccPerThread<G, W>; };
template <int G, bool W> struct AccSel<kPlaceLocalMem, G, W> { using T = AccLocal<G, W>; };
template <int G, bool W> struct AccSel<kPlaceSharedMemPerThread, G, W> { using T = AccSharedPerThread<G, W>; };
template <int G, bool W> struct AccSel<kPlaceGlobal, G, W> { using T = AccGlobal<G, W>; };

// ---------------------------------------------------------------------------------------------
// Row decoding
// ---------------------------------------------------------------------------------------------


__device__ __forceinline__ uint32_t code_of_chars(uint32_t rf, uint32_t ls) {
    const uint32_t r = (rf == 'R' ? 2u : 0u) + (rf == 'N' ? 1u : 0u);
    return (r << 1) + (ls == 'F' ? 0u : 1u);
}

__device__ __forceinline__ bool fits_i64(__int128 v) { return v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX; }

__device__ __forceinline__ void atomic_add_i128(unsigned long long* p, __int128 v) {
    atomic_add_u128(p, (uint64_t)(unsigned __int128)v, (uint64_t)((unsigned __int128)v >> 64));
}

// One passing reference-typed row outside the fast domain, summed exactly with the reference's
// arithmetic (cpu/kernel_hyper.hpp:70-83): disc_1 = 100 - disc, tax_1 = 100 + tax,
// disc_price = disc_1 * price, charge = disc_price * tax_1, each an int64 in the reference and
// checked for overflow there; the six sums go straight into the output table as signed 128-bit
// values. A row whose int64 arithmetic would overflow is reported instead of summed.
__device__ __noinline__ void wide_row(const ScanParams& prm, uint32_t group, int64_t q, int64_t d, int64_t t,
                                      int64_t p) {
    const __int128 d1 = (__int128)100 - d, t1 = (__int128)100 + t;
    const __int128 dp = d1 * p;
    const __int128 ch = dp * t1;   // |dp| < 2^64 and |t1| < 2^64 here, so the product is exact
    if (!fits_i64(d1) || !fits_i64(t1) || !fits_i64(dp) || !fits_i64(ch)) {
        if (prm.status) atomicOr(prm.status, kStatusDomain);
        return;
    }
    unsigned long long* o = prm.out + 2 * (group * kNumAggs);
    atomic_add_i128(o + 2 * kAggCount, 1);
    atomic_add_i128(o + 2 * kAggQty, (__int128)q * prm.qty_scale);
    atomic_add_i128(o + 2 * kAggBasePrice, p);
    atomic_add_i128(o + 2 * kAggDisc, d);
    atomic_add_i128(o + 2 * kAggDiscPrice, dp);
    atomic_add_i128(o + 2 * kAggCharge, ch);
}

// One step of rows [kRowsPerStep * j, +kRowsPerStep) of the R-row tile held at shared address `base`.
template <int L, uint32_t R, class Acc>
__device__ __forceinline__ void process_step(const ScanParams& prm, uint32_t base, uint32_t j, int32_t cut,
                                             uint32_t lut, Acc& acc, uint32_t& bad) {
    using T = LayoutTraits<L>;
    if constexpr (L == kLayUncomp) {
        const uint2 sd = lds_v2(base + col_offset<L>(0, R) + 8 * j);
        const uint4 Q = lds_v4(base + col_offset<L>(1, R) + 16 * j);
        const uint4 D = lds_v4(base + col_offset<L>(2, R) + 16 * j);
        const uint4 X = lds_v4(base + col_offset<L>(3, R) + 16 * j);
        const uint4 P = lds_v4(base + col_offset<L>(4, R) + 16 * j);
        const uint32_t RF = lds_u16(base + col_offset<L>(5, R) + 2 * j);
        const uint32_t LS = lds_u16(base + col_offset<L>(6, R) + 2 * j);
        // Both rows in the fast domain (always, in TPC-H data): the placement's tables only. A
        // per-thread branch, not a warp vote: the warp-lane placement's lanes may diverge here.
        const bool fast = ((Q.y | Q.w | D.y | D.w | X.y | X.w | P.y | P.w) == 0u) & (D.x <= 100u) & (D.z <= 100u) &
                          (X.x <= 255u) & (X.z <= 255u);
        if (fast) {
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int32_t ship = (int32_t)(r ? sd.y : sd.x);
                const uint32_t code = code_of_chars((RF >> (8 * r)) & 0xFFu, (LS >> (8 * r)) & 0xFFu);
                const uint32_t c = ship <= cut ? code : 7u;
                const uint32_t q = r ? Q.z : Q.x;
                const uint32_t d = r ? D.z : D.x;
                const uint32_t t = r ? X.z : X.x;
                const uint32_t p = r ? P.z : P.x;
                const uint32_t a = 100u - d;
                acc.add(c, q, d, a, a * (100u + t), p);
            }
        } else {
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int32_t ship = (int32_t)(r ? sd.y : sd.x);
                const uint32_t code = code_of_chars((RF >> (8 * r)) & 0xFFu, (LS >> (8 * r)) & 0xFFu);
                const uint32_t q = r ? Q.z : Q.x;
                const uint32_t d = r ? D.z : D.x;
                const uint32_t t = r ? X.z : X.x;
                const uint32_t p = r ? P.z : P.x;
                const bool wide =
                    ((r ? (Q.w | D.w | X.w | P.w) : (Q.y | D.y | X.y | P.y)) != 0u) | (d > 100u) | (t > 255u);
                const bool pass = ship <= cut;
                if (wide && pass && acc.owns(code))
                    wide_row(prm, code, (int64_t)((uint64_t)(r ? Q.w : Q.y) << 32 | q),
                             (int64_t)((uint64_t)(r ? D.w : D.y) << 32 | d),
                             (int64_t)((uint64_t)(r ? X.w : X.y) << 32 | t),
                             (int64_t)((uint64_t)(r ? P.w : P.y) << 32 | p));
                const uint32_t c = (pass && !wide) ? code : 7u;
                const uint32_t a = 100u - d;
                acc.add(c, q, d, a, a * (100u + t), p);
            }
        }
    } else {
        constexpr bool kSep = (L == kLaySep || L == kLaySepFilter);
        // pass mask of the 4 rows: byte r = 0xFF iff row r passes
        uint32_t PM;
        if constexpr (T::kFilter) {
            const uint32_t bits = (lds_u8(base + col_offset<L>(0, R) + (j >> 1)) >> ((j & 1u) * 4u)) & 0xFu;
            PM = ((bits * 0x00204081u) & 0x01010101u) * 0xFFu;
        } else {
            PM = quad_pass_mask(lds_v2(base + col_offset<L>(0, R) + 8 * j), cut, bad);
        }
        Quad x;
        x.Q = lds_u32(base + col_offset<L>(1, R) + 4 * j);
        x.D = lds_u32(base + col_offset<L>(2, R) + 4 * j);
        const uint32_t X = lds_u32(base + col_offset<L>(3, R) + 4 * j);
        const uint4 P = lds_v4(base + col_offset<L>(4, R) + 16 * j);
        const uint32_t F = lds_u8(base + col_offset<L>(5, R) + j);
        bad |= disc_out_of_domain4(x.D);
        // one-hot group bit per row byte, from a 256-entry table indexed by the 4 codes' byte
        uint32_t OH = lds_u32(lut + 4 * F);
        if constexpr (kSep) {
            // the table gives bit 2*rf; a line status of 1 doubles it to bit 2*rf+1; rf 3 -> dropped
            const uint32_t LS = (lds_u8(base + col_offset<L>(6, R) + (j >> 1)) >> ((j & 1u) * 4u)) & 0xFu;
            const uint32_t lsm = ((LS * 0x00204081u) & 0x01010101u) * 0xFFu;   // byte r = 0xFF iff ls_r
            OH = (OH + (OH & lsm)) & 0x3F3F3F3Fu;
        }
        x.OH = OH & PM;
        x.p[0] = P.x;
        x.p[1] = P.y;
        x.p[2] = P.z;
        x.p[3] = P.w;
        quad_derive(x, X);
        acc.add_quad(x);
    }
}

// One row straight from global memory (tail rows that do not fill a tile).
template <int L, class Acc>
__device__ __forceinline__ void process_row_global(const ScanParams& prm, uint64_t i, Acc& acc, uint32_t& bad) {
    if constexpr (L == kLayUncomp) {
        const int32_t ship = __ldg(reinterpret_cast<const int32_t*>(prm.col[0]) + i);
        const uint64_t q = __ldg(reinterpret_cast<const unsigned long long*>(prm.col[1]) + i);
        const uint64_t d = __ldg(reinterpret_cast<const unsigned long long*>(prm.col[2]) + i);
        const uint64_t t = __ldg(reinterpret_cast<const unsigned long long*>(prm.col[3]) + i);
        const uint64_t p = __ldg(reinterpret_cast<const unsigned long long*>(prm.col[4]) + i);
        const uint32_t rf = (uint8_t)__ldg(reinterpret_cast<const char*>(prm.col[5]) + i);
        const uint32_t ls = (uint8_t)__ldg(reinterpret_cast<const char*>(prm.col[6]) + i);
        const bool wide = ((q | p) >> 32) != 0 || d > 100u || t > 255u;
        const bool pass = ship <= prm.cutoff;
        if (wide && pass && acc.owns(code_of_chars(rf, ls)))
            wide_row(prm, code_of_chars(rf, ls), (int64_t)q, (int64_t)d, (int64_t)t, (int64_t)p);
        const uint32_t c = (pass && !wide) ? code_of_chars(rf, ls) : 7u;
        const uint32_t a = 100u - (uint32_t)d;
        acc.add(c, (uint32_t)q, (uint32_t)d, a, a * (100u + (uint32_t)t), (uint32_t)p);
    } else {
        using T = LayoutTraits<L>;
        constexpr bool kSep = (L == kLaySep || L == kLaySepFilter);
        bool pass;
        if constexpr (T::kFilter) {
            pass = (__ldg(reinterpret_cast<const uint32_t*>(prm.col[0]) + (i >> 5)) >> (i & 31)) & 1u;
        } else {
            const uint32_t ship = __ldg(reinterpret_cast<const uint16_t*>(prm.col[0]) + i);
            bad |= ship > 32767u;
            pass = (int32_t)ship <= prm.cutoff;
        }
        const uint32_t q = __ldg(prm.col[1] + i);
        const uint32_t d = __ldg(prm.col[2] + i);
        const uint32_t t = __ldg(prm.col[3] + i);
        const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(prm.col[4]) + i);
        uint32_t code;
        const uint32_t rfw = __ldg(reinterpret_cast<const uint32_t*>(prm.col[5]) + (i >> 4));
        code = (rfw >> (2 * (i & 15))) & 3u;
        if constexpr (kSep) {
            const uint32_t lsw = __ldg(reinterpret_cast<const uint32_t*>(prm.col[6]) + (i >> 5));
            code = (code << 1) | ((lsw >> (i & 31)) & 1u);
        }
        bad |= d > 100u;
        const uint32_t c = pass ? code : 7u;
        const uint32_t a = 100u - d;
        acc.add(c, q, d, a, a * (100u + t), p);
    }
}

// ---------------------------------------------------------------------------------------------
// The kernel
// ---------------------------------------------------------------------------------------------

template <int L, int P>
__global__ void __launch_bounds__((kConsumerWarps<L, P> + 1) * 32, 1)
q1_scan_kernel(const __grid_constant__ ScanParams prm) {
    using T = LayoutTraits<L>;
    constexpr uint32_t R = kTileRows<L, P>;
    constexpr uint32_t S = kStages<L, P>;
    constexpr uint32_t W = kConsumerWarps<L, P>;
    constexpr uint32_t kStage = stage_bytes<L>(R);
    constexpr int G = T::kCodes;
    static_assert(kStage % 16 == 0, "stage must keep 16-byte alignment");

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ __align__(16) unsigned long long red[G * kNumAggs * 2];

    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t num_tiles = prm.rows / R;
    const uint32_t ring = ptx::smem_addr(smem);

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        fence_mbar_init();
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)(G * kNumAggs * 2); i += blockDim.x) red[i] = 0;
    // byte of four 2-bit codes -> one-hot bit per row byte (pair: bit code; separate: bit 2*rf)
    __shared__ uint32_t code_lut[256];
    for (uint32_t f = threadIdx.x; f < 256; f += blockDim.x) {
        uint32_t v = 0;
        for (uint32_t r = 0; r < 4; ++r) {
            const uint32_t code = (f >> (2 * r)) & 3u;
            v |= (1u << (G == 4 ? code : 2 * code)) << (8 * r);
        }
        code_lut[f] = v;
    }
    const uint32_t lut = smem_addr(code_lut);
    __syncthreads();

    if (warp == W) {
        // ----------------------------- producer warp ------------------------------------
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            uint32_t k = 0;
            for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
                const uint32_t s = k % S;
                if (!mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) break;
                const uint32_t fb = smem_addr(&full_bar[s]);
                mbar_arrive_expect_tx(fb, kStage);
                const uint32_t dst = ring + s * kStage;
#pragma unroll
                for (int c = 0; c < T::kCols; ++c) {
                    const uint32_t bytes = R * col_bits<L>(c) / 8u;
                    bulk_g2s(dst + col_offset<L>(c, R), prm.col[c] + t * (uint64_t)bytes, bytes, fb, pol);
                }
            }
            // Never leave with copies in flight: wait for the last tiles issued to land.
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
    } else {
        // ----------------------------- consumer warps -----------------------------------
        using Acc = typename AccSel<P, G, T::kWideQty>::T;
        const uint32_t ctid = threadIdx.x;  // 0 .. 32W-1
        Acc acc;
        acc.init(lane, ctid, smem + S * kStage, red);
        uint32_t bad = 0;
        constexpr uint32_t kSteps = R / T::kRowsPerStep;  // steps per tile
        // Rows one consumer thread adds per tile, and how often the 16-bit packed partials
        // (quantity <= 255 per row) must be folded into 64 bits: at most every 257 rows.
        constexpr uint32_t kTablesPerWarp = 32u / G;
        constexpr uint32_t kRowsPerThreadTile =
            (P == kPlaceInRegisters) ? (kSteps + W * kTablesPerWarp - 1) / (W * kTablesPerWarp) * T::kRowsPerStep
                                     : kSteps / (W * 32) * T::kRowsPerStep;
        constexpr uint32_t kFoldEvery = (257u / kRowsPerThreadTile) > 0 ? (257u / kRowsPerThreadTile) : 1u;
        static_assert(kRowsPerThreadTile <= 257u, "tile too large for the packed partials");
        static_assert(kSteps % (W * 32) == 0, "steps must divide evenly among consumer threads");
        // The global placement's warp flush is a 64-bit sum of 32 lanes' buffered rows: at most
        // 2048 rows a lane of charges below 100 (2^32 - 1) 355 < 2^47.2 stays below 2^64.
        static_assert(P != kPlaceGlobal || kRowsPerThreadTile * kGlobalFlushTiles <= 2048u,
                      "global flush sums must stay below 2^64");
        bool ok = true;
        uint32_t k = 0;
        for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
            const uint32_t s = k % S;
            // Every lane waits (acquiring the bulk-copy writes); the warp proceeds only together.
            const bool landed = mbar_wait(smem_addr(&full_bar[s]), (k / S) & 1u, prm.status);
            if (!__all_sync(0xffffffffu, landed)) {
                ok = false;
                break;
            }
            const uint32_t base = ring + s * kStage;
            if constexpr (P == kPlaceInRegisters) {
                const uint32_t tbl = lane / G;
                if (tbl < kTablesPerWarp) {
                    for (uint32_t j = warp * kTablesPerWarp + tbl; j < kSteps; j += W * kTablesPerWarp)
                        process_step<L, R>(prm, base, j, prm.cutoff, lut, acc, bad);
                }
            } else {
#pragma unroll
                for (uint32_t it = 0; it < kSteps / (W * 32); ++it)
                    process_step<L, R>(prm, base, ctid + it * (W * 32), prm.cutoff, lut, acc, bad);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
            acc.tile_done(prm, lane);
            if ((k + 1) % kFoldEvery == 0) acc.fold();
        }
        acc.fold();
        // Tail rows [num_tiles * R, rows): handled by the CTA next in the round robin.
        if (ok && blockIdx.x == (uint32_t)(num_tiles % gridDim.x)) {
            const uint64_t first = num_tiles * R;
            if constexpr (P == kPlaceInRegisters) {
                const uint32_t tbl = lane / G;
                if (tbl < kTablesPerWarp) {
                    for (uint64_t i = first + warp * kTablesPerWarp + tbl; i < prm.rows; i += W * kTablesPerWarp)
                        process_row_global<L>(prm, i, acc, bad);
                }
            } else {
                for (uint64_t i = first + ctid; i < prm.rows; i += W * 32) process_row_global<L>(prm, i, acc, bad);
            }
            acc.tile_done(prm, lane);
        }
        acc.finish(prm, lane);
        if (bad && prm.status) atomicOr(prm.status, kStatusDomain);
        acc.flush(CtaRed{red}, lane);
    }
    __syncthreads();
    if (prm.records) {
        // Per-CTA record instead of atomics: one thread per (group, aggregate), summing the codes
        // that map to the group.
        unsigned long long* rec = prm.records + (uint64_t)blockIdx.x * (kNumGroups * kNumAggs * 2);
        for (uint32_t i = threadIdx.x; i < (uint32_t)(kNumGroups * kNumAggs); i += blockDim.x) {
            const uint32_t grp = i / kNumAggs, agg = i % kNumAggs;
            uint64_t lo = 0, hi = 0;
            for (uint32_t code = 0; code < (uint32_t)G; ++code) {
                if (((G == 4) ? prm.pair_group[code] : code) != grp) continue;
                uint64_t clo = red[2 * (code * kNumAggs + agg)], chi = red[2 * (code * kNumAggs + agg) + 1];
                if (agg == kAggQty && prm.qty_scale != 1u) {
                    const unsigned __int128 v = ((unsigned __int128)chi << 64 | clo) * prm.qty_scale;
                    clo = (uint64_t)v;
                    chi = (uint64_t)(v >> 64);
                }
                const uint64_t nlo = lo + clo;
                hi += chi + (nlo < lo ? 1u : 0u);
                lo = nlo;
            }
            rec[2 * i] = lo;
            rec[2 * i + 1] = hi;
        }
        return;
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)(G * kNumAggs); i += blockDim.x) {
        const uint32_t code = i / kNumAggs, agg = i % kNumAggs;
        const uint32_t grp = (G == 4) ? prm.pair_group[code] : code;
        uint64_t lo = red[2 * i], hi = red[2 * i + 1];
        if (agg == kAggQty && prm.qty_scale != 1u) {
            // 128 x 32 -> 128 multiply (sum of quantity in whole units -> hundredths)
            const uint64_t l_lo = (lo & 0xFFFFFFFFull) * prm.qty_scale;
            const uint64_t l_hi = (lo >> 32) * prm.qty_scale;
            const uint64_t nlo = l_lo + (l_hi << 32);
            hi = hi * prm.qty_scale + (l_hi >> 32) + (nlo < l_lo ? 1u : 0u);
            lo = nlo;
        }
        atomic_add_u128(prm.out + 2 * (grp * kNumAggs + agg), lo, hi);
    }
}

// ---------------------------------------------------------------------------------------------
// Host launch table
// ---------------------------------------------------------------------------------------------

template <int L, int P>
static cudaError_t launch_one(const ScanParams& prm, int sm_count, int max_blocks, cudaStream_t stream) {
    constexpr uint32_t R = kTileRows<L, P>;
    constexpr uint32_t S = kStages<L, P>;
    constexpr uint32_t W = kConsumerWarps<L, P>;
    constexpr int G = LayoutTraits<L>::kCodes;
    uint32_t dyn = S * stage_bytes<L>(R);
    if (P == kPlaceSharedMemPerThread) dyn += (uint32_t)(8 * (L == kLayUncomp ? 5 : 4) * G * W * 32);
    cudaError_t e = cudaFuncSetAttribute(q1_scan_kernel<L, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = scan_grid_blocks(L, P, prm.rows, sm_count, max_blocks);
    q1_scan_kernel<L, P><<<blocks, (W + 1) * 32, dyn, stream>>>(prm);
    return cudaGetLastError();
}

template <int L>
static cudaError_t launch_layout(int placement, const ScanParams& prm, int sm_count, int max_blocks, cudaStream_t st) {
    switch (placement) {
        case kPlaceInRegisters: return launch_one<L, kPlaceInRegisters>(prm, sm_count, max_blocks, st);
        case kPlaceInRegistersPerThread: return launch_one<L, kPlaceInRegistersPerThread>(prm, sm_count, max_blocks, st);
        case kPlaceLocalMem: return launch_one<L, kPlaceLocalMem>(prm, sm_count, max_blocks, st);
        case kPlaceSharedMemPerThread: return launch_one<L, kPlaceSharedMemPerThread>(prm, sm_count, max_blocks, st);
        case kPlaceGlobal: return launch_one<L, kPlaceGlobal>(prm, sm_count, max_blocks, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_scan(int layout, int placement, const ScanParams& prm, int sm_count, int max_blocks,
                        cudaStream_t stream) {
    switch (layout) {
        case kLayPair: return launch_layout<kLayPair>(placement, prm, sm_count, max_blocks, stream);
        case kLayPairFilter: return launch_layout<kLayPairFilter>(placement, prm, sm_count, max_blocks, stream);
        case kLaySep: return launch_layout<kLaySep>(placement, prm, sm_count, max_blocks, stream);
        case kLaySepFilter: return launch_layout<kLaySepFilter>(placement, prm, sm_count, max_blocks, stream);
        case kLayUncomp: return launch_layout<kLayUncomp>(placement, prm, sm_count, max_blocks, stream);
        default: return cudaErrorInvalidValue;
    }
}

namespace {

struct Geometry {
    uint32_t warps, tile_rows;
};
template <int L>
Geometry geometry_of(int placement) {
    switch (placement) {
        case kPlaceInRegisters: return {kConsumerWarps<L, kPlaceInRegisters>, kTileRows<L, kPlaceInRegisters>};
        case kPlaceInRegistersPerThread:
            return {kConsumerWarps<L, kPlaceInRegistersPerThread>, kTileRows<L, kPlaceInRegistersPerThread>};
        case kPlaceLocalMem: return {kConsumerWarps<L, kPlaceLocalMem>, kTileRows<L, kPlaceLocalMem>};
        case kPlaceSharedMemPerThread:
            return {kConsumerWarps<L, kPlaceSharedMemPerThread>, kTileRows<L, kPlaceSharedMemPerThread>};
        default: return {kConsumerWarps<L, kPlaceGlobal>, kTileRows<L, kPlaceGlobal>};
    }
}
Geometry geometry(int layout, int placement) {
    switch (layout) {
        case kLayPair: return geometry_of<kLayPair>(placement);
        case kLayPairFilter: return geometry_of<kLayPairFilter>(placement);
        case kLaySep: return geometry_of<kLaySep>(placement);
        case kLaySepFilter: return geometry_of<kLaySepFilter>(placement);
        default: return geometry_of<kLayUncomp>(placement);
    }
}

}  // namespace

uint64_t scan_max_rows_per_launch(int layout, int placement, uint32_t grid) {
    // accumulating lanes per CTA: every consumer thread, or the lanes of one warp-lane table
    const uint64_t codes = (layout == kLayPair || layout == kLayPairFilter) ? 4 : 6;
    const Geometry g = geometry(layout, placement);
    const uint64_t lanes = placement == kPlaceInRegisters ? g.warps * (32 / codes) : g.warps * 32ull;
    uint64_t n = (uint64_t)grid * lanes * 32768ull;
    if (n > (1ull << 31)) n = 1ull << 31;
    return n / g.tile_rows * g.tile_rows;
}

uint32_t scan_grid_blocks(int layout, int placement, uint64_t rows, int sm_count, int max_blocks) {
    const uint64_t tiles = rows / scan_tile_rows(layout, placement);
    uint64_t blocks = tiles ? tiles : 1;
    uint64_t cap = (uint64_t)sm_count;  // one CTA per SM (shared-memory bound)
    if (max_blocks > 0 && (uint64_t)max_blocks < cap) cap = (uint64_t)max_blocks;
    if (blocks > cap) blocks = cap;
    return (uint32_t)blocks;
}

uint32_t scan_tile_rows(int layout, int placement) { return geometry(layout, placement).tile_rows; }

}  // namespace q1
