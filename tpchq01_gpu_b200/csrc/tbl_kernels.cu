// lineitem text ingestion on the GPU: the reference's lineitem::FromFile (cpu/tpch_kit.cpp:155-172
// with the TableReader tokenizer at :10-99) as three kernels over a device copy of the text.
//
// Format (dbgen .tbl): one row per '\n'-terminated line (the last line may lack the '\n'), fields
// separated by '|'. Fields 5-11 (1-based) are read, the others skipped:
//   quantity, extendedprice, discount, tax   decimals "[+-]digits[.digits]" -> 100 * int + frac
//                                             (Decimal<15,2>::ToValue, cpu/tpch_kit.hpp:52-54;
//                                             the fraction's digits are read as an integer, as
//                                             the reference's parser does)
//   returnflag, linestatus                    exactly one character (Char, cpu/tpch_kit.hpp:15-23)
//   shipdate                                  "year-month-day" -> day number counted the MonetDB
//                                             way (Date, cpu/tpch_kit.cpp:142-153): 1992-01-01 is
//                                             727563
// A line that does not match is counted as malformed (its row is written as zeros) and the host
// reports the count and the first malformed line's byte offset.
//
// Kernels (64 KB text tiles, 256 threads, 256 bytes a thread):
//   tbl_count_kernel  newlines per tile (16-byte loads, byte compares on 32-bit words)
//   tbl_scan_kernel   exclusive prefix of the tile counts (one CTA)
//   tbl_parse_kernel  recounts its tile, ranks each thread's newlines with a block scan,
//                     gathers the line starts into shared memory in text order and parses them
//                     lane-parallel (row = newlines before the line); thread 0 of tile 0 also
//                     parses the line at byte 0.
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_kernels.h"

namespace q1 {

namespace tbl {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kPerThread = 256;                 // bytes
constexpr uint64_t kTile = (uint64_t)kThreads * kPerThread;

// Newlines in text[a, b) (a 16-byte aligned or b - a < 16 handled bytewise).
__device__ __forceinline__ uint32_t count_newlines(const char* __restrict__ text, uint64_t a, uint64_t b) {
    uint32_t n = 0;
    if (b - a == kPerThread && ((reinterpret_cast<uintptr_t>(text) + a) & 15u) == 0) {
        const uint4* p = reinterpret_cast<const uint4*>(text + a);
#pragma unroll 4
        for (uint32_t k = 0; k < kPerThread / 16; ++k) {
            const uint4 v = __ldg(p + k);
            n += __popc(__vcmpeq4(v.x, 0x0A0A0A0Au)) + __popc(__vcmpeq4(v.y, 0x0A0A0A0Au)) +
                 __popc(__vcmpeq4(v.z, 0x0A0A0A0Au)) + __popc(__vcmpeq4(v.w, 0x0A0A0A0Au));
        }
        return n / 8;   // __vcmpeq4 sets all 8 bits of an equal byte
    }
    for (uint64_t i = a; i < b; ++i) n += text[i] == '\n' ? 1u : 0u;
    return n;
}

// Day number of a civil date counted the MonetDB way (days since a year 0, years >= 1 here);
// -1 for a date that does not exist.
__device__ __forceinline__ int32_t days_before_month(int32_t m) {   // non-leap year, m in 1..13
    return (367 * m - 362) / 12 - (m > 2 ? 2 : 0);
}
__device__ __forceinline__ int32_t day_number(int32_t y, int32_t m, int32_t d) {
    const bool leap = (y % 4 == 0) && (y % 100 != 0 || y % 400 == 0);
    if (y < 1 || y > 999999 || m < 1 || m > 12 || d < 1) return -1;
    const int32_t len = (m == 12 ? 31 : days_before_month(m + 1) - days_before_month(m)) + ((m == 2 && leap) ? 1 : 0);
    if (d > len) return -1;
    const int32_t p = y - 1;
    return 365 * y + (p / 4 - p / 100 + p / 400 + 1) + days_before_month(m) + ((m > 2 && leap) ? 1 : 0) + d - 1;
}

// Reads a line through a 16-byte window: one aligned 16-byte load per 16 bytes of the line
// (lanes of a warp read different lines, so every load touches a different cache line; byte
// loads would cost one L1 wavefront per byte). Offsets are 32-bit and relative to the line's
// start (a line whose first eleven fields span more than 2^31 bytes reads as malformed). The
// last, partial 16-byte block of the buffer is read bytewise so that no load goes past its end.
struct Cursor {
    const char* __restrict__ line;   // the line's first byte
    const uint4* __restrict__ blk;   // 16-byte blocks from the one holding line[0]
    uint32_t off;                    // line's offset inside its first block
    uint32_t p, end;                 // cursor and end of the buffer, relative to line
    uint32_t full;                   // blocks [0, full) lie wholly inside the buffer
    uint32_t wi = 0xFFFFFFFFu;       // block in the window
    uint4 win;
    __device__ __forceinline__ Cursor(const char* __restrict__ text, uint64_t s, uint64_t bytes) {
        line = text + s;
        const uintptr_t a = reinterpret_cast<uintptr_t>(line);
        off = (uint32_t)(a & 15u);
        blk = reinterpret_cast<const uint4*>(a - off);
        const uint64_t rest = bytes - s;
        end = rest < 0x7FFFFFFFull ? (uint32_t)rest : 0x7FFFFFFFu;
        full = (uint32_t)(((uint64_t)off + end) >> 4);
        p = 0;
    }
    __device__ __forceinline__ int peek() {
        if (p >= end) return -1;
        const uint32_t a = off + p, bi = a >> 4;
        if (bi >= full) return (int)(unsigned char)line[p];
        if (bi != wi) {
            win = __ldg(blk + bi);
            wi = bi;
        }
        const uint32_t o = a & 15u;
        const uint32_t w = o < 8 ? (o < 4 ? win.x : win.y) : (o < 12 ? win.z : win.w);
        return (int)((w >> (8 * (o & 3u))) & 0xFFu);
    }
    // skips to just after the next '|' of this line; false at '\n' or the end
    __device__ __forceinline__ bool skip_field() {
        for (;;) {
            const int c = peek();
            if (c < 0 || c == '\n') return false;
            ++p;
            if (c == '|') return true;
        }
    }
    __device__ __forceinline__ bool sep() {
        if (peek() != '|') return false;
        ++p;
        return true;
    }
    // "[+-]digits" (at most 18 digits)
    __device__ __forceinline__ bool integer(int64_t& v) {
        bool neg = false;
        int c = peek();
        if (c == '+' || c == '-') {
            neg = c == '-';
            ++p;
        }
        int64_t x = 0;
        uint32_t nd = 0;
        while ((c = peek()) >= '0' && c <= '9') {
            if (++nd > 18) return false;
            x = x * 10 + (c - '0');
            ++p;
        }
        if (!nd) return false;
        v = neg ? -x : x;
        return true;
    }
    // "[+-]digits[.digits]" -> 100 * int + frac
    __device__ __forceinline__ bool decimal(int64_t& v) {
        int64_t i = 0, f = 0;
        if (!integer(i)) return false;
        if (peek() == '.') {
            ++p;
            if (!integer(f)) return false;
        }
        v = 100 * i + f;
        return true;
    }
    __device__ __forceinline__ bool chr(char& c) {
        const int x = peek();
        if (x < 0 || x == '|' || x == '\n') return false;
        ++p;
        c = (char)x;
        return true;
    }
    __device__ __forceinline__ bool date(int32_t& day) {
        int64_t y, m, d;
        if (!integer(y) || peek() != '-') return false;
        ++p;
        if (!integer(m) || peek() != '-') return false;
        ++p;
        if (!integer(d)) return false;
        const int c = peek();
        if (!(c < 0 || c == '|' || c == '\n')) return false;
        if (y < 1 || y > 999999 || m < 1 || m > 12 || d < 1 || d > 31) return false;
        day = day_number((int32_t)y, (int32_t)m, (int32_t)d);
        return day >= 0;
    }
};

struct Out {
    int32_t* ship;
    int64_t *qty, *price, *disc, *tax;
    char *rf, *ls;
};

// Parses the line starting at byte s into row `row`; false (row zeroed) if malformed.
__device__ bool parse_line(const char* __restrict__ text, uint64_t bytes, uint64_t s, uint64_t row, const Out& o) {
    Cursor c(text, s, bytes);
    int64_t q = 0, pr = 0, di = 0, tx = 0;
    char rf = 0, ls = 0;
    int32_t ship = 0;
    bool ok = c.skip_field() && c.skip_field() && c.skip_field() && c.skip_field();
    ok = ok && c.decimal(q) && c.sep() && c.decimal(pr) && c.sep() && c.decimal(di) && c.sep() && c.decimal(tx) &&
         c.sep();
    ok = ok && c.chr(rf) && c.sep() && c.chr(ls) && c.sep() && c.date(ship);
    if (!ok) q = pr = di = tx = 0, rf = ls = 0, ship = 0;
    o.ship[row] = ship;
    o.qty[row] = q;
    o.price[row] = pr;
    o.disc[row] = di;
    o.tax[row] = tx;
    o.rf[row] = rf;
    o.ls[row] = ls;
    return ok;
}

}  // namespace tbl

__global__ void __launch_bounds__(tbl::kThreads) tbl_count_kernel(const char* __restrict__ text, uint64_t bytes,
                                                                  unsigned long long* __restrict__ tile_lines) {
    using namespace tbl;
    __shared__ uint32_t sum;
    if (threadIdx.x == 0) sum = 0;
    __syncthreads();
    const uint64_t a = blockIdx.x * kTile + (uint64_t)threadIdx.x * kPerThread;
    const uint64_t b = a + kPerThread < bytes ? a + kPerThread : bytes;
    uint32_t n = a < bytes ? count_newlines(text, a, b) : 0u;
    n += __shfl_xor_sync(0xffffffffu, n, 16);
    n += __shfl_xor_sync(0xffffffffu, n, 8);
    n += __shfl_xor_sync(0xffffffffu, n, 4);
    n += __shfl_xor_sync(0xffffffffu, n, 2);
    n += __shfl_xor_sync(0xffffffffu, n, 1);
    if ((threadIdx.x & 31u) == 0) atomicAdd(&sum, n);
    __syncthreads();
    if (threadIdx.x == 0) tile_lines[blockIdx.x] = sum;
}

// In-place exclusive prefix over `tiles` counts; element `tiles` receives the total.
__global__ void __launch_bounds__(1024) tbl_scan_kernel(unsigned long long* v, uint64_t tiles) {
    __shared__ unsigned long long part[1024];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < tiles; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        const unsigned long long x = i < tiles ? v[i] : 0ull;
        part[threadIdx.x] = x;
        __syncthreads();
        for (uint32_t off = 1; off < 1024; off <<= 1) {
            const unsigned long long y = threadIdx.x >= off ? part[threadIdx.x - off] : 0ull;
            __syncthreads();
            part[threadIdx.x] += y;
            __syncthreads();
        }
        if (i < tiles) v[i] = carry + part[threadIdx.x] - x;
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) v[tiles] = carry;
}

// Parses the lines that start in this block's tile. The line starts are first gathered into
// shared memory in text order (each thread's newlines at its block-scan rank), then every thread
// parses lines tid, tid + 256, ...: the lanes of a warp parse different lines side by side instead
// of one lane at a time. Tiles with more than kList lines take several rounds.
__global__ void __launch_bounds__(tbl::kThreads) tbl_parse_kernel(const char* __restrict__ text, uint64_t bytes,
                                                                  const unsigned long long* __restrict__ tile_first,
                                                                  tbl::Out o, uint64_t capacity,
                                                                  unsigned long long* __restrict__ bad) {
    using namespace tbl;
    constexpr uint32_t kList = 4096;
    __shared__ uint32_t warp_sum[kThreads / 32];
    __shared__ uint32_t total;
    __shared__ uint32_t starts[kList];   // newline offsets within the tile, in text order
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint64_t tile = blockIdx.x * kTile;
    const uint64_t a = tile + (uint64_t)tid * kPerThread;
    const uint64_t b = a + kPerThread < bytes ? a + kPerThread : bytes;
    const uint32_t n = a < bytes ? count_newlines(text, a, b) : 0u;
    // block-wide exclusive prefix of n
    uint32_t inc = n;
#pragma unroll
    for (uint32_t off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t w = 0; w < warp; ++w) before += warp_sum[w];
    before += inc - n;
    if (tid == kThreads - 1) total = before + n;
    __syncthreads();
    const uint32_t T = total;
    const unsigned long long first = tile_first[blockIdx.x];   // newlines before this tile
    unsigned long long nbad = 0, first_bad = ~0ull;
    auto one = [&](uint64_t s, uint64_t row) {
        if (row >= capacity || !parse_line(text, bytes, s, row, o)) {
            ++nbad;
            if (s < first_bad) first_bad = s;
        }
    };
    if (blockIdx.x == 0 && tid == 0 && bytes > 0) one(0, 0);
    const bool vec = b - a == kPerThread && ((reinterpret_cast<uintptr_t>(text) + a) & 15u) == 0;
    for (uint32_t r0 = 0; r0 < T; r0 += kList) {
        // gather: this thread's newlines whose block rank falls in [r0, r0 + kList)
        if (n && before + n > r0 && before < r0 + kList) {
            uint32_t k = before;
            if (vec) {
                const uint4* p = reinterpret_cast<const uint4*>(text + a);
                for (uint32_t q = 0; q < kPerThread / 16; ++q) {
                    const uint4 v = __ldg(p + q);
                    const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                    for (uint32_t h = 0; h < 4; ++h) {
                        uint32_t m = __vcmpeq4(w4[h], 0x0A0A0A0Au) & 0x80808080u;
                        while (m) {
                            const uint32_t byte = (uint32_t)(__ffs(m) - 1) >> 3;
                            m &= m - 1;
                            if (k >= r0 && k < r0 + kList) starts[k - r0] = (uint32_t)(a - tile) + q * 16 + h * 4 + byte;
                            ++k;
                        }
                    }
                }
            } else {
                for (uint64_t i = a; i < b; ++i) {
                    if (text[i] != '\n') continue;
                    if (k >= r0 && k < r0 + kList) starts[k - r0] = (uint32_t)(i - tile);
                    ++k;
                }
            }
        }
        __syncthreads();
        const uint32_t cnt = T - r0 < kList ? T - r0 : kList;
        for (uint32_t j = tid; j < cnt; j += kThreads) {
            const uint64_t i = tile + starts[j];            // a newline; the next line is row first + rank + 1
            if (i + 1 < bytes) one(i + 1, first + r0 + j + 1);
        }
        __syncthreads();
    }
    if (nbad) {
        atomicAdd(&bad[0], nbad);
        atomicMin(&bad[1], first_bad);
    }
}

uint64_t tbl_tiles(uint64_t bytes) { return (bytes + tbl::kTile - 1) / tbl::kTile; }

cudaError_t launch_tbl_count(const char* text, uint64_t bytes, unsigned long long* tile_lines, cudaStream_t stream) {
    const uint64_t tiles = tbl_tiles(bytes);
    if (tiles) {
        tbl_count_kernel<<<(unsigned)tiles, tbl::kThreads, 0, stream>>>(text, bytes, tile_lines);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    tbl_scan_kernel<<<1, 1024, 0, stream>>>(tile_lines, tiles);
    return cudaGetLastError();
}

cudaError_t launch_tbl_parse(const char* text, uint64_t bytes, const unsigned long long* tile_first,
                             int32_t* ship, int64_t* qty, int64_t* price, int64_t* disc, int64_t* tax, char* rf,
                             char* ls, uint64_t capacity, unsigned long long* bad, cudaStream_t stream) {
    const uint64_t tiles = tbl_tiles(bytes);
    if (!tiles) return cudaSuccess;
    tbl::Out o{ship, qty, price, disc, tax, rf, ls};
    tbl_parse_kernel<<<(unsigned)tiles, tbl::kThreads, 0, stream>>>(text, bytes, tile_first, o, capacity, bad);
    return cudaGetLastError();
}

}  // namespace q1
