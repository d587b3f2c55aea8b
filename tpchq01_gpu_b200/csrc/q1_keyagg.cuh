// Group-key aggregation engines shared by the group-key kernel (groupkey_kernels.cu) and the
// batch kernel (batch_kernels.cu): the Q1 predicate and aggregates over a 13 B/row tile
// (ship u16 | qty u8 | disc u8 | tax u8 | price u32 | key u32), grouped by key < num_groups.
// The per-row arithmetic is the reference's (src/kernels/ht_in_global_mem.hpp:31-49) with
// group = key.
//
// Engines (one per placement):
//   PlaneRegs<NG>  num_groups <= NG (4 or 8): per-thread byte-plane dot products (dp4a), four
//                  rows per instruction, as in the scan kernel, over three price byte planes (a
//                  row with a price >= 2^24 goes to the global path); no atomics until a flush.
//   Cube3Table     num_groups <= 64: a shared-memory table per (group, discount, tax) cell; a
//                  row adds its count, its quantity and its price: three atomics.
//   CubeTableT     num_groups <= 1024: a shared-memory table per (group, discount) cell. A row
//                  adds its count, price and tax * price to its cell and its quantity to its
//                  group's word (the batch kernel's form: to one of four by discount & 3); the
//                  discounted sums follow exactly at the flush, because the
//                  discount of a cell is known there: sum (100-d) p = sum_d (100-d) P_d and
//                  sum (100-d)(100+t) p = sum_d (100-d) (100 P_d + TP_d).
//   SlotTable      one shared-memory slot per key below the table's size (2048 in the batch
//                  kernel, 4096 in the group-key kernel and the partitioned path): count,
//                  discount, quantity, price, discount x price, charge; disc_price follows at
//                  the flush as 100 sum p - sum d p.
//   global         every row reduces straight into the scratch accumulators.
// The shared tables use only 32-bit shared atomics (64-bit shared atomics are far slower).
// Counts and quantities cannot wrap a 32-bit word between two flushes (at most 2^23 rows per
// CTA: count < 2^24, quantity <= 255 * 2^23 < 2^32), so their atomics need no result and no carry
// check. (Packing a count and 2^24 x its quantity into one word saved an atomic but wrapped about
// every tenth row of a cell, so the warp-voted carry branch ran on nearly every quad: 11.7 shared
// atomic instructions per warp and quad where 8 were needed.) Price sums can wrap: the slot table
// and the (group, discount, tax) cube keep them as (low word, carry word) pairs: the low word's
// atomic returns the old value, and a wrap adds the carry to the high word. The
// (group, discount) cube keeps only the low words of its cells, so that 1024 groups fit: a wrap of
// a price or tax-price word (a few rows in a thousand) is counted in three words of its group
// (wraps, and the cells' 100 - d summed over price and over tax-price wraps), from which the
// flush adds what the wraps are worth. (Sending each wrap's 2^32 straight to the group's scratch
// sums in global memory serialised on the L2 when one key holds many rows: Zipf keys over 1024
// groups at full pass 2.98 ms per 600 M rows, 1.57 ms without those global atomics. The batch
// kernel, whose instances' keys are uniform, keeps that form: see CubeTableT.) Rows
// outside the tables' fast domain
// (discount > 10, tax > 8 or price >= 2^24; TPC-H data has none) take the global path, so every
// result is exact over the whole compressed domain.
//
// Scratch per group (8 x u64, zeroed before a launch): count, quantity (whole units), discount,
// price, disc_price = a4 + 2^32 a5, charge = a6 + 2^32 a7; folded into an int128 table later.
#pragma once

#include <stdint.h>

#include "q1_common.cuh"
#include "q1_ptx.cuh"
#include "q1_quad.cuh"

namespace q1 {
namespace ka {

using namespace ptx;

// ---------------------------------------------------------------------------------------------
// Tile layout (TR rows per tile, TR a multiple of 16, so every column offset is a multiple of 16
// bytes): ship u16 | qty u8 | disc u8 | tax u8 | price u32 | key u32
// ---------------------------------------------------------------------------------------------
template <uint32_t TR>
struct TileLayout {
    static_assert(TR % 16 == 0, "column offsets must stay 16-byte aligned");
    static constexpr uint32_t kOffShip = 0, kOffQty = 2 * TR, kOffDisc = 3 * TR, kOffTax = 4 * TR,
                              kOffPrice = 5 * TR, kOffKey = 9 * TR;
    static constexpr uint32_t kStageBytes = 13 * TR;
    static __host__ __device__ constexpr uint32_t col_bytes(int c) { return c == 0 ? 2 * TR : (c < 4 ? TR : 4 * TR); }
    static __host__ __device__ constexpr uint32_t col_off(int c) {
        return c == 0 ? kOffShip
                      : (c == 1 ? kOffQty : (c == 2 ? kOffDisc : (c == 3 ? kOffTax : (c == 4 ? kOffPrice : kOffKey))));
    }
};
// The 2048-row tile of the batch kernels, the partitioned path and the group-key kernel's table
// and global placements.
constexpr uint32_t R = 2048;
constexpr uint32_t kOffShip = TileLayout<R>::kOffShip, kOffQty = TileLayout<R>::kOffQty,
                   kOffDisc = TileLayout<R>::kOffDisc, kOffTax = TileLayout<R>::kOffTax,
                   kOffPrice = TileLayout<R>::kOffPrice, kOffKey = TileLayout<R>::kOffKey;
constexpr uint32_t kStageBytes = TileLayout<R>::kStageBytes;
__host__ __device__ constexpr uint32_t col_bytes(int c) { return TileLayout<R>::col_bytes(c); }
__host__ __device__ constexpr uint32_t col_off(int c) { return TileLayout<R>::col_off(c); }

// Flush cadences. Plane partials: at most 2^15 rows per thread; every consumer thread handles at
// most 8 rows of a tile (the kernels assert it), so 4032 tiles leave room for one more partial
// tile.
// Shared tables: at most 2^23 rows per CTA between flushes keeps every packed field and carry
// word below its limit (count < 2^24 per cell; carry words < 2^32).
constexpr uint32_t kPlaneFlushTiles = 4032;
constexpr uint64_t kTableFlushRows = 1ull << 23;

constexpr uint32_t kCubeMaxGroups = 1024;
constexpr uint32_t kCubeDisc = 11;          // discount 0..10
constexpr uint32_t kCubeWords = 3;          // count, price, tax * price (low words)
constexpr uint32_t kCube3MaxGroups = 64;
constexpr uint32_t kCubeTax = 9;            // tax 0..8
constexpr uint32_t kCube3Words = 4;         // count, quantity, price low, price carry
constexpr uint32_t kSlots = 2048;
constexpr uint32_t kSlotWords = 9;          // count, discount, quantity, price lo/hi, discount x price lo/hi, charge lo/hi

// cells, then (CubeTable) kCubeGroupWords words per group: quantity and three wrap counters
constexpr uint32_t kCubeGroupWords = 4;
__host__ __device__ constexpr uint32_t cube_bytes(uint32_t num_groups) {
    return num_groups * (kCubeDisc * kCubeWords + kCubeGroupWords) * 4;
}
__host__ __device__ constexpr uint32_t cube3_bytes(uint32_t num_groups) {
    return num_groups * kCubeDisc * kCubeTax * kCube3Words * 4;
}
__host__ __device__ constexpr uint32_t slot_bytes(uint32_t slots) { return slots * kSlotWords * 4; }

// ---------------------------------------------------------------------------------------------
// Scratch updates
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void red_add(unsigned long long* p, uint64_t v) {
    if (v) asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void scratch_add(unsigned long long* acc, uint32_t g, uint64_t cnt, uint64_t q, uint64_t d,
                                            uint64_t p, uint64_t dp_lo, uint64_t dp_hi, uint64_t ch_lo, uint64_t ch_hi) {
    unsigned long long* a = acc + 8ull * g;
    red_add(a + 0, cnt);
    red_add(a + 1, q);
    red_add(a + 2, d);
    red_add(a + 3, p);
    red_add(a + 4, dp_lo);
    red_add(a + 5, dp_hi);
    red_add(a + 6, ch_lo);
    red_add(a + 7, ch_hi);
}

// One passing row straight into the scratch (the global placement and the slow path).
__device__ __forceinline__ void scratch_row(unsigned long long* acc, uint32_t key, uint32_t q, uint32_t d, uint32_t t,
                                            uint32_t p) {
    const uint32_t a = 100u - d;
    const uint64_t dp = (uint64_t)a * p, ch = (uint64_t)(a * (100u + t)) * p;
    scratch_add(acc, key, 1, q, d, p, dp & 0xFFFFFFFFull, dp >> 32, ch & 0xFFFFFFFFull, ch >> 32);
}

__device__ __forceinline__ bool fast_domain(uint32_t d, uint32_t t, uint32_t p) {
    return d < kCubeDisc && t <= 8u && p < (1u << 24);
}

// 64-bit sum as (lo, hi) 32-bit shared words: lo += v, carry into hi.
__device__ __forceinline__ void add_carry(uint32_t* lo, uint32_t* hi, uint32_t v) {
    const uint32_t old = atomicAdd(lo, v);
    if (old + v < old) atomicAdd(hi, 1u);
}
__device__ __forceinline__ void add_wide(uint32_t* lo, uint32_t* hi, uint32_t vlo, uint32_t vhi) {
    const uint32_t old = atomicAdd(lo, vlo);
    const uint32_t h = vhi + (old + vlo < old ? 1u : 0u);
    if (h) atomicAdd(hi, h);
}

// ---------------------------------------------------------------------------------------------
// A quad: four consecutive rows of a tile
// ---------------------------------------------------------------------------------------------
struct KeyQuad {
    uint32_t PM;        // byte r = 0xFF iff row r passes the predicate
    uint32_t Q, D, X;   // bytes r: quantity, discount, tax
    uint32_t p[4];
    uint32_t k[4];
};

// Rows 4j..4j+3 of the TR-row tile at shared address `base`. `bad` becomes nonzero for a value
// outside the compressed domain (ship offset > 32767, discount > 100).
template <uint32_t TR = R>
__device__ __forceinline__ KeyQuad load_quad(uint32_t base, uint32_t j, int32_t cut, uint32_t& bad) {
    using TL = TileLayout<TR>;
    KeyQuad x;
    x.PM = quad_pass_mask(lds_v2(base + TL::kOffShip + 8 * j), cut, bad);
    x.Q = lds_u32(base + TL::kOffQty + 4 * j);
    x.D = lds_u32(base + TL::kOffDisc + 4 * j);
    x.X = lds_u32(base + TL::kOffTax + 4 * j);
    const uint4 P = lds_v4(base + TL::kOffPrice + 16 * j);
    const uint4 K = lds_v4(base + TL::kOffKey + 16 * j);
    bad |= disc_out_of_domain4(x.D);
    x.p[0] = P.x, x.p[1] = P.y, x.p[2] = P.z, x.p[3] = P.w;
    x.k[0] = K.x, x.k[1] = K.y, x.k[2] = K.z, x.k[3] = K.w;
    return x;
}

// A quad with no passing row (for lanes past the end of a partial tile, so that every lane of
// the warp takes part in the warp votes of the table engines).
__device__ __forceinline__ KeyQuad empty_quad() {
    KeyQuad x;
    x.PM = x.Q = x.D = x.X = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) x.p[r] = x.k[r] = 0;
    return x;
}

// One row read from global memory (tail rows of a partial tile), as a quad whose rows 1..3 fail.
__device__ __forceinline__ KeyQuad load_row(const uint8_t* const col[6], uint64_t i, int32_t cut, uint32_t& bad) {
    KeyQuad x;
    const uint32_t ship = __ldg(reinterpret_cast<const uint16_t*>(col[0]) + i);
    const uint32_t d = __ldg(col[2] + i);
    bad |= (ship > 32767u || d > 100u) ? 1u : 0u;
    x.PM = (int32_t)ship <= cut ? 0xFFu : 0u;
    x.Q = __ldg(col[1] + i);
    x.D = d;
    x.X = __ldg(col[3] + i);
    x.p[0] = __ldg(reinterpret_cast<const uint32_t*>(col[4]) + i);
    x.k[0] = __ldg(reinterpret_cast<const uint32_t*>(col[5]) + i);
    x.p[1] = x.p[2] = x.p[3] = 0;
    x.k[1] = x.k[2] = x.k[3] = 0;
    return x;
}

// ---------------------------------------------------------------------------------------------
// PlaneRegs: per-thread dp4a byte planes for num_groups <= NG
// ---------------------------------------------------------------------------------------------
template <int NG>
struct PlaneRegs {
    // Three price byte planes a group: a passing row with a price >= 2^24 (none in TPC-H data) is
    // added, exactly, straight into the scratch behind one warp vote, so that eight groups' planes
    // fit in registers (the fourth plane took 32 more a thread and made the 8-group kernel spill).
    GroupPlanesT<3> g[NG];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < NG; ++i) g[i].zero();
    }
    // Every lane of the warp calls it (warp vote).
    __device__ __forceinline__ void add(const KeyQuad& kq, uint32_t num_groups, unsigned long long* acc,
                                        uint32_t& bad) {
        uint32_t OH = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t key = kq.k[r];
            const bool in = key < num_groups;
            if (!in && ((kq.PM >> (8 * r)) & 1u)) bad = 1u;
            OH |= (in ? (1u << (key & 7u)) : 0u) << (8 * r);
        }
        Quad x;
        x.OH = OH & kq.PM;
        x.Q = kq.Q;
        x.D = kq.D;
#pragma unroll
        for (int r = 0; r < 4; ++r) x.p[r] = kq.p[r];
        quad_derive(x, kq.X);
        if (__any_sync(0xffffffffu, x.P[3])) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (((x.P[3] >> (8 * r)) & 0xFFu) && ((x.OH >> (8 * r)) & 0xFFu)) {
                    scratch_row(acc, kq.k[r], (kq.Q >> (8 * r)) & 0xFFu, (kq.D >> (8 * r)) & 0xFFu,
                                (kq.X >> (8 * r)) & 0xFFu, kq.p[r]);
                    x.OH &= ~(0xFFu << (8 * r));
                }
            }
        }
#pragma unroll
        for (int i = 0; i < NG; ++i) g[i].template add_quad<false>(x.OH, (uint32_t)i, x);
    }
    // Warp sums of the per-thread partials into the scratch; every lane of the warp calls it.
    __device__ __forceinline__ void flush(unsigned long long* acc, uint32_t num_groups, uint32_t lane) {
#pragma unroll
        for (int i = 0; i < NG; ++i) {
            if ((uint32_t)i < num_groups) {
                const uint64_t ch = g[i].value(kAggCharge), dp = g[i].value(kAggDiscPrice);
                const uint64_t cnt = warp_sum_u64(g[i].cnt);
                const uint64_t q = warp_sum_u64(g[i].q), d = warp_sum_u64(g[i].d);
                const uint64_t p = warp_sum_u64(g[i].value(kAggBasePrice));
                const uint64_t dpl = warp_sum_u64(dp & 0xFFFFFFFFull), dph = warp_sum_u64(dp >> 32);
                const uint64_t chl = warp_sum_u64(ch & 0xFFFFFFFFull), chh = warp_sum_u64(ch >> 32);
                if (lane == 0 && cnt) scratch_add(acc, (uint32_t)i, cnt, q, d, p, dpl, dph, chl, chh);
            }
            g[i].zero();
        }
    }
};

// ---------------------------------------------------------------------------------------------
// CubeTable: shared (group, discount) cells
// ---------------------------------------------------------------------------------------------
// kSharedCarries: wraps counted in the group's shared words (the group-key kernel); otherwise
// each wrap's worth goes straight to the group's scratch sums and the group's four words hold its
// quantity four ways, by discount & 3 (the batch kernel, whose combined engines measured 4-5% slower
// with the shared counters although its 1024-group instances do not contend: 256 instances 4.02
// -> 4.20 ms).
template <bool kSharedCarries>
struct CubeTableT {
    uint32_t* w;       // [kCubeWords][cells]: count, price, tax * price (low words)
    uint32_t* gw;      // kSharedCarries: [kCubeGroupWords][groups], word-major (consecutive groups'
                       // words in consecutive banks): quantity; wraps of the group's cells' price
                       // words; sum (100 - d) over those wraps; sum (100 - d) over wraps of tax *
                       // price words. Otherwise [groups][kCubeGroupWords]: quantity by discount & 3.
    uint32_t cells, groups;
    __device__ __forceinline__ void bind(uint8_t* base, uint32_t num_groups) {
        w = reinterpret_cast<uint32_t*>(base);
        cells = num_groups * kCubeDisc;
        groups = num_groups;
        gw = w + kCubeWords * cells;
    }
    __device__ __forceinline__ void zero(uint32_t tid, uint32_t nthreads) {
        for (uint32_t i = tid; i < kCubeWords * cells + kCubeGroupWords * groups; i += nthreads) w[i] = 0;
    }
    // Rows r of a quad with bit r of `m` set (passing, key < num_groups, fast domain). All
    // atomics of the quad are issued before any carry is checked, so their latencies overlap.
    static constexpr bool kPacked = true;
    // The quantity, discount and tax bytes of the four rows packed in Q, D, X; acc: the scratch. A
    // cell's count and a group's quantity cannot wrap between flushes (at most 2^23 rows per CTA:
    // count < 2^24, quantity <= 255 * 2^23 < 2^32), so their atomics need no result. A wrap of a
    // cell's price or tax * price word (a few rows in a thousand) is worth, with the cell's
    // discount d and a = 100 - d, 2^32 of price, 2^32 a of disc_price and 2^32 100 a of charge,
    // or 2^32 a of charge.
    __device__ __forceinline__ void add_quad_packed(uint32_t m, const uint32_t key[4], uint32_t Q, uint32_t D,
                                                    uint32_t X, const uint32_t p[4], unsigned long long* acc) {
        uint32_t c[4], vt[4], op[4], ot[4];
        if (!__any_sync(0xffffffffu, m)) return;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            c[r] = key[r] * kCubeDisc + ((D >> (8 * r)) & 0xFFu);
            vt[r] = ((X >> (8 * r)) & 0xFFu) * p[r];                     // t p < 2^28
            op[r] = ot[r] = 0;
            if ((m >> r) & 1u) {
                atomicAdd(w + c[r], 1u);
                if constexpr (kSharedCarries)
                    atomicAdd(gw + key[r], (Q >> (8 * r)) & 0xFFu);
                else
                    atomicAdd(gw + key[r] * kCubeGroupWords + ((D >> (8 * r)) & 3u), (Q >> (8 * r)) & 0xFFu);
                op[r] = atomicAdd(w + cells + c[r], p[r]);
                ot[r] = atomicAdd(w + 2 * cells + c[r], vt[r]);
            }
        }
        // a word wrapped iff old > ~added (rows not added have old == 0): one predicate, and
        // the rows only in the rare branch
        bool wrap = false;
#pragma unroll
        for (int r = 0; r < 4; ++r) wrap |= (op[r] > ~p[r]) | (ot[r] > ~vt[r]);
        if (__any_sync(0xffffffffu, wrap)) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const uint32_t a = 100u - ((D >> (8 * r)) & 0xFFu);
                if constexpr (kSharedCarries) {
                    uint32_t* g = gw + key[r];
                    if (op[r] > ~p[r]) {
                        atomicAdd(g + groups, 1u);
                        atomicAdd(g + 2 * groups, a);
                    }
                    if (ot[r] > ~vt[r]) atomicAdd(g + 3 * groups, a);
                } else {
                    unsigned long long* sg = acc + 8ull * key[r];
                    if (op[r] > ~p[r]) {
                        red_add(sg + 3, 1ull << 32);
                        red_add(sg + 5, a);
                        red_add(sg + 7, 100u * a);
                    }
                    if (ot[r] > ~vt[r]) red_add(sg + 7, a);
                }
            }
        }
    }
    // Cells -> per-group sums -> scratch; the caller synchronises the consumers around it.
    __device__ __forceinline__ void flush(unsigned long long* acc, uint32_t num_groups, uint32_t tid, uint32_t nthreads) {
        for (uint32_t g = tid; g < num_groups; g += nthreads) {
            uint64_t q = 0, pw = 0, aw = 0, tw = 0;
            if constexpr (kSharedCarries) {
                q = gw[g], pw = gw[groups + g], aw = gw[2 * groups + g], tw = gw[3 * groups + g];
#pragma unroll
                for (uint32_t j = 0; j < kCubeGroupWords; ++j) gw[j * groups + g] = 0;
            } else {
#pragma unroll
                for (uint32_t j = 0; j < kCubeGroupWords; ++j) {
                    q += gw[g * kCubeGroupWords + j];
                    gw[g * kCubeGroupWords + j] = 0;
                }
            }
            uint64_t cnt = 0, dsum = 0, P = pw << 32;
            unsigned __int128 DP = (unsigned __int128)aw << 32, CH = (unsigned __int128)(100u * aw + tw) << 32;
#pragma unroll
            for (uint32_t d = 0; d < kCubeDisc; ++d) {
                const uint32_t c = g * kCubeDisc + d;
                const uint32_t nd = w[c], Pd = w[cells + c], TPd = w[2 * cells + c];
                cnt += nd;
                dsum += (uint64_t)d * nd;
                P += Pd;
                DP += (uint64_t)(100u - d) * Pd;
                CH += (unsigned __int128)(100u - d) * ((uint64_t)Pd * 100u + TPd);
#pragma unroll
                for (uint32_t k = 0; k < kCubeWords; ++k) w[k * cells + c] = 0;
            }
            if (cnt)
                scratch_add(acc, g, cnt, q, dsum, P, (uint64_t)DP & 0xFFFFFFFFull, (uint64_t)(DP >> 32),
                            (uint64_t)CH & 0xFFFFFFFFull, (uint64_t)(CH >> 32));
        }
    }
};

// ---------------------------------------------------------------------------------------------
// Cube3Table: shared (group, discount, tax) cells, for num_groups <= 64. A row adds only its
// count, quantity and price: three atomics, of which only the price's can wrap (into the cell's
// carry word) between flushes. At the flush the cell's discount and tax give
// sum (100-d) p = (100-d) P and sum (100-d)(100+t) p = (100-d)(100+t) P.
// ---------------------------------------------------------------------------------------------
struct Cube3Table {
    uint32_t* w;       // [kCube3Words][cells]: count, quantity, price low word, price carry word
    uint32_t cells;
    __device__ __forceinline__ void bind(uint8_t* base, uint32_t num_groups) {
        w = reinterpret_cast<uint32_t*>(base);
        cells = num_groups * kCubeDisc * kCubeTax;
    }
    __device__ __forceinline__ void zero(uint32_t tid, uint32_t nthreads) {
        for (uint32_t i = tid; i < kCube3Words * cells; i += nthreads) w[i] = 0;
    }
    static constexpr bool kPacked = true;
    // Rows r of a quad with bit r of `m` set (fast domain), the quantity, discount and tax bytes
    // of the four rows packed in Q, D, X (D and X zero in rows outside the fast domain). There
    // 9 d + t < 99 fits a byte, so one shift-and-add gives the four (discount, tax) cell offsets.
    __device__ __forceinline__ void add_quad_packed(uint32_t m, const uint32_t key[4], uint32_t Q, uint32_t D,
                                                    uint32_t X, const uint32_t p[4], unsigned long long*) {
        uint32_t c[4], op[4];
        if (!__any_sync(0xffffffffu, m)) return;
        const uint32_t DT = (D << 3) + D + X;   // bytes r: 9 d + t (garbage outside the fast domain)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            c[r] = key[r] * (kCubeDisc * kCubeTax) + ((DT >> (8 * r)) & 0xFFu);
            op[r] = 0;
            if ((m >> r) & 1u) {
                atomicAdd(w + c[r], 1u);
                atomicAdd(w + cells + c[r], (Q >> (8 * r)) & 0xFFu);
                op[r] = atomicAdd(w + 2 * cells + c[r], p[r]);
            }
        }
        // a price word wrapped iff old > ~added (rows not added have old == 0): one predicate
        // and one vote, the rows only in the branch (a cell's price word wraps every thousand
        // rows or so; its count and quantity words cannot wrap between flushes)
        bool wrap = false;
#pragma unroll
        for (int r = 0; r < 4; ++r) wrap |= op[r] > ~p[r];
        if (__any_sync(0xffffffffu, wrap)) {
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (op[r] > ~p[r]) atomicAdd(w + 3 * cells + c[r], 1u);
        }
    }
    // Cells -> per-group sums -> scratch; the caller synchronises the consumers around it.
    __device__ __forceinline__ void flush(unsigned long long* acc, uint32_t num_groups, uint32_t tid, uint32_t nthreads) {
        for (uint32_t g = tid; g < num_groups; g += nthreads) {
            uint64_t cnt = 0, q = 0, dsum = 0, P = 0;
            unsigned __int128 DP = 0, CH = 0;
            for (uint32_t d = 0; d < kCubeDisc; ++d) {
                uint64_t Pd = 0, cd = 0;
                unsigned __int128 Td = 0;   // sum_t (100 + t) P_dt
#pragma unroll
                for (uint32_t t = 0; t < kCubeTax; ++t) {
                    const uint32_t c = (g * kCubeDisc + d) * kCubeTax + t;
                    const uint64_t Pt = ((uint64_t)w[3 * cells + c] << 32) | w[2 * cells + c];
                    cd += w[c];
                    q += w[cells + c];
                    Pd += Pt;
                    Td += (unsigned __int128)(100u + t) * Pt;
#pragma unroll
                    for (uint32_t k = 0; k < kCube3Words; ++k) w[k * cells + c] = 0;
                }
                cnt += cd;
                dsum += (uint64_t)d * cd;
                P += Pd;
                DP += (unsigned __int128)(100u - d) * Pd;
                CH += (unsigned __int128)(100u - d) * Td;
            }
            if (cnt)
                scratch_add(acc, g, cnt, q, dsum, P, (uint64_t)DP & 0xFFFFFFFFull, (uint64_t)(DP >> 32),
                            (uint64_t)CH & 0xFFFFFFFFull, (uint64_t)(CH >> 32));
        }
    }
};

// ---------------------------------------------------------------------------------------------
// SlotTable: shared per-group slots for keys < slots
// ---------------------------------------------------------------------------------------------
struct SlotTable {
    static constexpr bool kPacked = false;
    uint32_t* w;       // [kSlotWords][slots]
    uint32_t slots;
    __device__ __forceinline__ void bind(uint8_t* base, uint32_t n) {
        w = reinterpret_cast<uint32_t*>(base);
        slots = n;
    }
    __device__ __forceinline__ void zero(uint32_t tid, uint32_t nthreads) {
        for (uint32_t i = tid; i < kSlotWords * slots; i += nthreads) w[i] = 0;
    }
    // Rows r of a quad with bit r of `m` set (passing, key < slots, fast domain); atomics first,
    // carries after.
    __device__ __forceinline__ void add_quad(uint32_t m, const uint32_t key[4], const uint32_t q[4],
                                             const uint32_t d[4], const uint32_t t[4], const uint32_t p[4]) {
        const uint32_t S = slots;
        uint32_t vd[4], cl[4], ch[4], op[4], od[4], oc[4];
        if (!__any_sync(0xffffffffu, m)) return;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t a = 100u - d[r];
            vd[r] = d[r] * p[r];         // d p < 2^28 (the discounted price follows at the flush)
            const uint64_t c64 = (uint64_t)(a * (100u + t[r])) * p[r];
            cl[r] = (uint32_t)c64;
            ch[r] = (uint32_t)(c64 >> 32);
            op[r] = od[r] = oc[r] = 0;
            if ((m >> r) & 1u) {
                const uint32_t s = key[r];
                atomicAdd(w + s, 1u);
                atomicAdd(w + S + s, d[r]);
                atomicAdd(w + 2 * S + s, q[r]);
                op[r] = atomicAdd(w + 3 * S + s, p[r]);
                od[r] = atomicAdd(w + 5 * S + s, vd[r]);
                oc[r] = atomicAdd(w + 7 * S + s, cl[r]);
            }
        }
        // a word wrapped iff old > ~added (rows not added have old == 0): one predicate, and
        // the rows only in the rare branch
        bool wrap = false;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            wrap |= (op[r] > ~p[r]) | (od[r] > ~vd[r]);
            ch[r] = ((m >> r) & 1u) ? ch[r] + (oc[r] > ~cl[r] ? 1u : 0u) : 0u;
        }
        // the charge's high word is nonzero for most rows: added per row
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (ch[r]) atomicAdd(w + 8 * S + key[r], ch[r]);
        if (__any_sync(0xffffffffu, wrap)) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (op[r] > ~p[r]) atomicAdd(w + 4 * S + key[r], 1u);
                if (od[r] > ~vd[r]) atomicAdd(w + 6 * S + key[r], 1u);
            }
        }
    }
    __device__ __forceinline__ void flush(unsigned long long* acc, uint32_t tid, uint32_t nthreads) {
        const uint32_t S = slots;
        for (uint32_t s = tid; s < S; s += nthreads) {
            const uint64_t cnt = w[s];
            if (cnt) {
                const uint64_t P = ((uint64_t)w[4 * S + s] << 32) | w[3 * S + s];
                const uint64_t DP = 100u * P - (((uint64_t)w[6 * S + s] << 32) | w[5 * S + s]);   // sum (100 - d) p
                scratch_add(acc, s, cnt, w[2 * S + s], w[S + s], P, DP & 0xFFFFFFFFull, DP >> 32, w[7 * S + s],
                            w[8 * S + s]);
            }
#pragma unroll
            for (uint32_t k = 0; k < kSlotWords; ++k) w[k * S + s] = 0;
        }
    }
};

// One quad into a shared table (CubeTable or SlotTable): rows in the table's fast domain go to the
// table, other passing rows with key < num_groups straight to the scratch, passing rows with
// key >= num_groups make `bad` nonzero.
// All lanes of the warp call it (the slow path, the tables' early exit when no lane of the warp
// has a row to add, and the carries use warp votes).
template <class Table>
__device__ __forceinline__ void table_quad(Table& tab, const KeyQuad& x, uint32_t num_groups, uint32_t hot,
                                           unsigned long long* acc, uint32_t& bad) {
    // rows outside the tables' fast domain: bit 7 of byte r set when d > 10, t > 8 or p >= 2^24
    const uint32_t top = __byte_perm(__byte_perm(x.p[0], x.p[1], 0x0073u), __byte_perm(x.p[2], x.p[3], 0x0073u),
                                     0x5410u);   // bytes r: top byte of p[r]
    const uint32_t outside = (((top & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | top | ((x.D & 0x7F7F7F7Fu) + 0x75757575u) |
                              x.D | ((x.X & 0x7F7F7F7Fu) + 0x77777777u) | x.X) &
                             0x80808080u;
    uint32_t m = 0, slow = 0;
    const uint32_t kmax = max(max(x.k[0], x.k[1]), max(x.k[2], x.k[3]));
    if (kmax < hot) {
        // every key of the quad in the table (hot <= num_groups): byte-parallel masks, each
        // gathered to bits 0..3 by one multiply (byte r's bit 0 lands on bit 24 + r)
        const uint32_t ob = (outside >> 7) * 0xFFu;
        m = (((x.PM & ~ob) & 0x01010101u) * 0x01020408u) >> 24;
        slow = (((x.PM & ob) & 0x01010101u) * 0x01020408u) >> 24;
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t pass = (x.PM >> (8 * r)) & 1u;
            const uint32_t key = x.k[r];
            const uint32_t in = pass & (key < num_groups ? 1u : 0u);
            bad |= pass & (key >= num_groups ? 1u : 0u);
            const uint32_t fast = in & (key < hot ? 1u : 0u) & (((outside >> (8 * r + 7)) & 1u) ^ 1u);
            m |= fast << r;
            slow |= (in & (fast ^ 1u)) << r;
        }
    }
    // rows outside the tables' fast domain (none in TPC-H data): one vote skips the path
    if (__any_sync(0xffffffffu, slow)) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if ((slow >> r) & 1u)
                scratch_row(acc, x.k[r], (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu,
                            (x.X >> (8 * r)) & 0xFFu, x.p[r]);
    }
    if constexpr (Table::kPacked) {
        // discount and tax bytes of in-domain rows only (d <= 10, t <= 8), so that byte-wise
        // arithmetic on them cannot carry into a neighbouring row's byte
        const uint32_t inb = ((~outside & 0x80808080u) >> 7) * 0xFFu;
        tab.add_quad_packed(m, x.k, x.Q, x.D & inb, x.X & inb, x.p, acc);
    } else {
        uint32_t q[4], d[4], t[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            q[r] = (x.Q >> (8 * r)) & 0xFFu;
            d[r] = (x.D >> (8 * r)) & 0xFFu;
            t[r] = (x.X >> (8 * r)) & 0xFFu;
        }
        tab.add_quad(m, x.k, q, d, t, x.p);
    }
}

// Barrier of the consumer warps only (the producer keeps streaming): one arrive per warp on an
// mbarrier initialised with the warp count, bounded wait. Every consumer passes the same sequence
// of barriers, so a local phase counter tracks the parity.
struct ConsumerBarrier {
    uint32_t addr;
    uint32_t phase;
    __device__ __forceinline__ void sync(uint32_t lane, uint32_t* status) {
        __syncwarp();
        if (lane == 0) mbar_arrive(addr);
        mbar_wait(addr, phase & 1u, status);
        ++phase;
    }
};

}  // namespace ka
}  // namespace q1
