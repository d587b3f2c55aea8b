// Quad decode shared by the scan, group-key and batch kernels: four rows of a compressed tile
// at once, with byte-plane dot products (dp4a) for per-thread per-group sums.
#pragma once

#include <stdint.h>

#include "q1_common.cuh"
#include "q1_ptx.cuh"

namespace q1 {

// Four decoded rows of a compressed tile (a "quad"), handed to a placement at once.
struct Quad {
    uint32_t OH;      // byte r: bit g set iff row r passes the predicate and has group code g
    uint32_t Q, D;    // bytes r: quantity (units) and discount (hundredths) of row r
    uint32_t a[4];    // 100 - discount
    uint32_t ab[4];   // (100 - discount) * (100 + tax)
    uint32_t p[4];    // extendedprice
    uint32_t A;       // bytes r: 100 - discount
    uint32_t P[4];    // byte planes of the prices: byte r of P[k] = byte k of p[r]
    uint32_t ABL, ABH;  // bytes r: low / high byte of ab[r]
};

// Byte planes of four 32-bit words (a 4x4 byte transpose, eight byte permutes).
__device__ __forceinline__ void byte_planes(const uint32_t w[4], uint32_t out[4]) {
    const uint32_t t0 = __byte_perm(w[0], w[1], 0x5140u), t1 = __byte_perm(w[2], w[3], 0x5140u);
    const uint32_t t2 = __byte_perm(w[0], w[1], 0x7362u), t3 = __byte_perm(w[2], w[3], 0x7362u);
    out[0] = __byte_perm(t0, t1, 0x5410u);
    out[1] = __byte_perm(t0, t1, 0x7632u);
    out[2] = __byte_perm(t2, t3, 0x5410u);
    out[3] = __byte_perm(t2, t3, 0x7632u);
}

// Aggregates of one group, per thread, computed with byte dot products (dp4a: four rows per
// instruction). With W1 = 0/1 bytes of the group's rows and M = its 0x00/0xFF byte mask:
//   count, qty, disc      dp4a(W1, 1 | Q | D)
//   sum p                 sum_k 2^8k dp4a(W1, P_k)
//   sum (100-d) p         sum_k 2^8k dp4a(A & M, P_k)
//   sum (100-d)(100+t) p  sum_k 2^8k (dp4a(ABL & M, P_k) + 2^8 dp4a(ABH & M, P_k))
// Every 32-bit partial stays exact while a thread adds at most 2^15 rows per launch (the host
// caps launches accordingly): the largest, an ab-low plane, grows by <= 4*255*255 per quad.
// kPlanes = 4 covers every 32-bit price; with kPlanes = 3 the caller keeps rows with a price
// >= 2^24 out of the planes (they need the top byte plane).
template <int kPlanes>
struct GroupPlanesT {
    uint32_t cnt, q, d;
    uint32_t p[kPlanes], dp[kPlanes], chl[kPlanes], chh[kPlanes];
    __device__ __forceinline__ void zero() {
        cnt = q = d = 0;
#pragma unroll
        for (int k = 0; k < kPlanes; ++k) p[k] = dp[k] = chl[k] = chh[k] = 0;
    }
    // kTop: the prices' top byte plane may be nonzero. Callers pass false when no lane of the
    // warp has a price >= 2^24 in the quad (TPC-H prices stay below 2^24): 15 dp4a instead of 19.
    template <bool kTop = true>
    __device__ __forceinline__ void add_quad(uint32_t OH, uint32_t g, const Quad& x) {
        const uint32_t W1 = (OH >> g) & 0x01010101u;
        const uint32_t M = (W1 << 8) - W1;   // 0xFF in the group's row bytes
        const uint32_t MA = x.A & M, ML = x.ABL & M, MH = x.ABH & M;
        cnt = __dp4a(W1, 0x01010101u, cnt);
        q = __dp4a(W1, x.Q, q);
        d = __dp4a(W1, x.D, d);
#pragma unroll
        for (int k = 0; k < ((kTop && kPlanes == 4) ? 4 : 3); ++k) {
            p[k] = __dp4a(W1, x.P[k], p[k]);
            dp[k] = __dp4a(MA, x.P[k], dp[k]);
            chl[k] = __dp4a(ML, x.P[k], chl[k]);
            chh[k] = __dp4a(MH, x.P[k], chh[k]);
        }
    }
    __device__ __forceinline__ uint64_t value(int agg) const {
        uint64_t v = 0;
        switch (agg) {
            case kAggCount: return cnt;
            case kAggQty: return q;
            case kAggDisc: return d;
            case kAggBasePrice:
#pragma unroll
                for (int k = 0; k < kPlanes; ++k) v += (uint64_t)p[k] << (8 * k);
                return v;
            case kAggDiscPrice:
#pragma unroll
                for (int k = 0; k < kPlanes; ++k) v += (uint64_t)dp[k] << (8 * k);
                return v;
            default:
#pragma unroll
                for (int k = 0; k < kPlanes; ++k) v += ((uint64_t)chl[k] << (8 * k)) + ((uint64_t)chh[k] << (8 * k + 8));
                return v;
        }
    }
};
using GroupPlanes = GroupPlanesT<4>;


// Any byte of a discount word above 100 (top bit of (b & 0x7F) + 27, or b >= 128).
__device__ __forceinline__ uint32_t disc_out_of_domain4(uint32_t D) {
    return (((D & 0x7F7F7F7Fu) + 0x1B1B1B1Bu) | D) & 0x80808080u;
}

// Fills the derived fields of x (A, a, ab, price byte planes, ab byte planes) from x.D, x.p and
// the four tax bytes X.
__device__ __forceinline__ void quad_derive(Quad& x, uint32_t X) {
    const uint32_t A = 0x64646464u - x.D;   // 100 - d per byte (no borrow inside the domain)
    x.A = A;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        x.a[r] = __byte_perm(A, 0u, 0x4440u | (uint32_t)r);
        x.ab[r] = x.a[r] * (100u + __byte_perm(X, 0u, 0x4440u | (uint32_t)r));
    }
    byte_planes(x.p, x.P);
    const uint32_t u = __byte_perm(x.ab[0], x.ab[1], 0x5140u), v = __byte_perm(x.ab[2], x.ab[3], 0x5140u);
    x.ABL = __byte_perm(u, v, 0x5410u);
    x.ABH = __byte_perm(u, v, 0x7632u);
}

// Pass mask of four ship offsets (two u32 words of two u16 each): byte r = 0xFF iff ship_r <= cut.
// Two 16-bit lanes per subtraction: lane = (cut + 2^15) - ship has its top bit set iff
// ship <= cut; no borrow crosses lanes for ship <= 32767 and -1 <= cut <= 32767. A ship offset
// above 32767 is outside the compressed domain and makes `bad` nonzero.
__device__ __forceinline__ uint32_t quad_pass_mask(uint2 sd, int32_t cut, uint32_t& bad) {
    const uint32_t c2 = (uint32_t)(cut + 32768) * 0x00010001u;
    bad |= (sd.x | sd.y) & 0x80008000u;
    return ptx::prmt(c2 - sd.x, c2 - sd.y, 0xFDB9u);
}

}  // namespace q1
