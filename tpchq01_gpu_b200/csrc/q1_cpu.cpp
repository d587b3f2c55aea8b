// CPU share of the coprocessing mode, the worker pool that runs it, and the filter-chunk queue.
//
// The reference runs its CPU share with Morsel<KernelX100<...>> (cpu/kernel_x100.hpp:423-665)
// behind CoProc (src/cpu.cpp:13-69) and hands filter chunks to the GPU loop through a moodycamel
// queue (src/cpu.h:12-21). This file is this project's own equivalent: a fixed thread pool with
// an atomic morsel cursor supplied by the caller, an exact 128-bit merge, and a blocking queue.
#include <immintrin.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <thread>
#include <vector>

#include "q1_common.cuh"
#include "q1_internal.h"

namespace q1 {

// ---------------------------------------------------------------------------------------------
// Host memory read rate (q1_measure_host_read)
// ---------------------------------------------------------------------------------------------

// XOR of every 64-byte line of [p, p + 64 * lines) (p 64-byte aligned), eight independent
// accumulators so that loads, not the reduction, set the pace; AVX-512 where the host has it.
__attribute__((target("avx512f"))) static uint64_t xor_lines_avx512(const uint8_t* p, uint64_t lines) {
    __m512i a[8];
    for (int k = 0; k < 8; ++k) a[k] = _mm512_setzero_si512();
    uint64_t i = 0;
    for (; i + 8 <= lines; i += 8)
        for (int k = 0; k < 8; ++k) a[k] = _mm512_xor_si512(a[k], _mm512_load_si512(p + 64 * (i + k)));
    for (; i < lines; ++i) a[0] = _mm512_xor_si512(a[0], _mm512_load_si512(p + 64 * i));
    for (int k = 1; k < 8; ++k) a[0] = _mm512_xor_si512(a[0], a[k]);
    return (uint64_t)_mm512_reduce_or_epi64(a[0]);
}

__attribute__((target("avx2"))) static uint64_t xor_lines_avx2(const uint8_t* p, uint64_t lines) {
    __m256i a[8];
    for (int k = 0; k < 8; ++k) a[k] = _mm256_setzero_si256();
    uint64_t i = 0;
    for (; i + 4 <= lines; i += 4)
        for (int k = 0; k < 8; ++k)
            a[k] = _mm256_xor_si256(a[k], _mm256_load_si256(reinterpret_cast<const __m256i*>(p + 64 * i + 32 * k)));
    for (; i < lines; ++i) {
        a[0] = _mm256_xor_si256(a[0], _mm256_load_si256(reinterpret_cast<const __m256i*>(p + 64 * i)));
        a[1] = _mm256_xor_si256(a[1], _mm256_load_si256(reinterpret_cast<const __m256i*>(p + 64 * i + 32)));
    }
    for (int k = 1; k < 8; ++k) a[0] = _mm256_xor_si256(a[0], a[k]);
    return (uint64_t)_mm256_extract_epi64(a[0], 0) ^ (uint64_t)_mm256_extract_epi64(a[0], 3);
}

double host_read_gbs(const void* buf, uint64_t bytes, int threads) {
    static const bool avx512 = __builtin_cpu_supports("avx512f");
    const uint64_t skip = (64 - (reinterpret_cast<uintptr_t>(buf) & 63)) & 63;
    if (bytes <= skip + 64) return 0.0;
    const uint8_t* base = static_cast<const uint8_t*>(buf) + skip;
    const uint64_t lines = (bytes - skip) / 64;
    if (threads < 1) threads = 1;
    std::vector<std::thread> ts;
    std::vector<uint64_t> out((size_t)threads);
    const uint64_t per = (lines + (uint64_t)threads - 1) / (uint64_t)threads;
    const auto t0 = std::chrono::steady_clock::now();
    for (int t = 0; t < threads; ++t) {
        const uint64_t b = std::min<uint64_t>(lines, (uint64_t)t * per), e = std::min<uint64_t>(lines, b + per);
        ts.emplace_back([&out, base, b, e, t] {
            out[(size_t)t] = avx512 ? xor_lines_avx512(base + 64 * b, e - b) : xor_lines_avx2(base + 64 * b, e - b);
        });
    }
    for (auto& t : ts) t.join();
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    volatile uint64_t sink = 0;
    for (const uint64_t v : out) sink = sink ^ v;
    (void)sink;
    return s > 0 ? (double)(lines * 64) / s / 1e9 : 0.0;
}

// ---------------------------------------------------------------------------------------------
// Pool
// ---------------------------------------------------------------------------------------------

CpuPool::CpuPool(int threads) {
    if (threads < 1) threads = 1;
    for (int i = 0; i < threads; ++i) workers_.emplace_back(&CpuPool::loop, this, i);
}

CpuPool::~CpuPool() {
    {
        std::lock_guard<std::mutex> lk(m_);
        stop_ = true;
    }
    cv_start_.notify_all();
    for (auto& w : workers_) w.join();
}

void CpuPool::start(std::function<void(int)> fn) {
    std::lock_guard<std::mutex> lk(m_);
    job_ = std::move(fn);
    running_ = (int)workers_.size();
    failed_ = false;
    error_.clear();
    ++generation_;
    cv_start_.notify_all();
}

bool CpuPool::failed() {
    std::lock_guard<std::mutex> lk(m_);
    return failed_;
}

bool CpuPool::wait() {
    std::unique_lock<std::mutex> lk(m_);
    cv_done_.wait(lk, [&] { return running_ == 0; });
    return !failed_;
}

void CpuPool::loop(int id) {
    uint64_t seen = 0;
    for (;;) {
        std::function<void(int)> job;
        {
            std::unique_lock<std::mutex> lk(m_);
            cv_start_.wait(lk, [&] { return stop_ || generation_ != seen; });
            if (stop_) return;
            seen = generation_;
            job = job_;
        }
        std::string err;
        try {
            if (take_fault(kFaultCpuWorker)) throw std::runtime_error("injected CPU worker fault");
            job(id);
        } catch (const std::exception& e) {
            err = e.what();
            if (err.empty()) err = "CPU worker exception";
        } catch (...) {
            err = "CPU worker exception";
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            if (!err.empty() && !failed_) {
                failed_ = true;
                error_ = err;
            }
            if (--running_ == 0) cv_done_.notify_all();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Queue
// ---------------------------------------------------------------------------------------------

void ChunkQueue::push(FilterChunk c) {
    {
        std::lock_guard<std::mutex> lk(m_);
        q_.push_back(c);
    }
    cv_.notify_one();
}

bool ChunkQueue::pop(FilterChunk* c, int timeout_ms) {
    std::unique_lock<std::mutex> lk(m_);
    if (!cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return closed_ || !q_.empty(); })) return false;
    if (q_.empty()) return false;
    *c = q_.front();
    q_.pop_front();
    return true;
}

void ChunkQueue::close() {
    {
        std::lock_guard<std::mutex> lk(m_);
        closed_ = true;
    }
    cv_.notify_all();
}

void ChunkQueue::reset() {
    std::lock_guard<std::mutex> lk(m_);
    q_.clear();
    closed_ = false;
}

// ---------------------------------------------------------------------------------------------
// CPU aggregation (same arithmetic and domain as the GPU kernels)
// ---------------------------------------------------------------------------------------------

namespace {

// 64-bit partials of one block of at most kBlock rows; charge < 2^47.2 per row keeps them exact.
constexpr uint64_t kBlock = 1u << 15;

struct Partial {
    uint64_t v[6][6];
    void clear() { memset(v, 0, sizeof(v)); }
    void into(Agg128* a) const {
        for (int g = 0; g < 6; ++g)
            for (int k = 0; k < 6; ++k) a->v[g][k] += v[g][k];
    }
};

// A passing reference-typed row outside the fast domain (any int64 values), with the reference's
// arithmetic (cpu/kernel_hyper.hpp:70-83) in exact signed 128-bit sums, as the GPU kernels' wide
// path does. Returns false, adding nothing, when an int64 product or difference of the reference
// would overflow (its handle_overflow).
inline bool wide_row(Agg128* out, uint32_t g, int64_t q, int64_t d, int64_t t, int64_t pr) {
    const __int128 d1 = (__int128)100 - d, t1 = (__int128)100 + t;
    const __int128 dp = d1 * pr;
    const __int128 ch = dp * t1;
    const auto fits = [](__int128 v) { return v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX; };
    if (!fits(d1) || !fits(t1) || !fits(dp) || !fits(ch)) return false;
    u128* o = out->v[g];
    o[kAggCount] += 1;
    o[kAggQty] += (u128)(__int128)q;
    o[kAggBasePrice] += (u128)(__int128)pr;
    o[kAggDisc] += (u128)(__int128)d;
    o[kAggDiscPrice] += (u128)dp;
    o[kAggCharge] += (u128)ch;
    return true;
}

inline void add_row(Partial& p, uint32_t g, uint64_t q, uint64_t d, uint64_t t, uint64_t pr) {
    const uint64_t a = 100 - d;
    const uint64_t dp = a * pr;
    uint64_t* r = p.v[g];
    r[kAggCount] += 1;
    r[kAggQty] += q;
    r[kAggBasePrice] += pr;
    r[kAggDisc] += d;
    r[kAggDiscPrice] += dp;
    r[kAggCharge] += dp * (100 + t);
}

}  // namespace

namespace {

// Pair layout, 16 rows per step with AVX-512: the 2-bit codes of a 16-row word become per-code
// lane masks; count, quantity and discount add in 32-bit lanes, price, (100-d) p and
// (100-d)(100+t) p in 64-bit lanes (products of 32-bit lanes, exact). Every lane sum stays
// exact within a block of kBlock rows. Rows [begin, end) with begin and end multiples of 16.
__attribute__((target("avx512f,avx512bw,avx512dq"))) bool aggregate_pair_avx512(const HostCompressed& t,
                                                                                 uint64_t begin, uint64_t end,
                                                                                 int32_t cutoff_rel, Agg128* out) {
    const __m512i shifts = _mm512_setr_epi32(0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24, 26, 28, 30);
    const __m512i three = _mm512_set1_epi32(3), one = _mm512_set1_epi32(1), hundred = _mm512_set1_epi32(100);
    const __m512i cut = _mm512_set1_epi32(cutoff_rel);
    bool ok = true;
    for (uint64_t b0 = begin; b0 < end; b0 += kBlock) {
        const uint64_t b1 = std::min(end, b0 + kBlock);
        __m512i cnt[4], q[4], d[4], p[4][2], dp[4][2], ch[4][2];
        for (int k = 0; k < 4; ++k) {
            cnt[k] = q[k] = d[k] = _mm512_setzero_si512();
            for (int h = 0; h < 2; ++h) p[k][h] = dp[k][h] = ch[k][h] = _mm512_setzero_si512();
        }
        __mmask16 bad = 0;
        for (uint64_t i = b0; i < b1; i += 16) {
            const __m512i ship = _mm512_cvtepu16_epi32(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(t.ship + i)));
            const __mmask16 pass = _mm512_cmple_epi32_mask(ship, cut);
            const __m512i code = _mm512_and_si512(_mm512_srlv_epi32(_mm512_set1_epi32((int)t.flags[i >> 4]), shifts), three);
            const __m512i vq = _mm512_cvtepu8_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(t.qty + i)));
            const __m512i vd = _mm512_cvtepu8_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(t.disc + i)));
            const __m512i vt = _mm512_cvtepu8_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(t.tax + i)));
            const __m512i vp = _mm512_loadu_si512(t.price + i);
            bad |= _mm512_mask_cmpgt_epu32_mask(pass, vd, hundred);
            const __m512i a = _mm512_sub_epi32(hundred, vd);
            const __m512i ab = _mm512_mullo_epi32(a, _mm512_add_epi32(hundred, vt));
            // 64-bit lanes: rows 0-7 (h = 0) and 8-15 (h = 1)
            __m512i p64[2], a64[2], ab64[2];
            p64[0] = _mm512_cvtepu32_epi64(_mm512_castsi512_si256(vp));
            p64[1] = _mm512_cvtepu32_epi64(_mm512_extracti64x4_epi64(vp, 1));
            a64[0] = _mm512_cvtepu32_epi64(_mm512_castsi512_si256(a));
            a64[1] = _mm512_cvtepu32_epi64(_mm512_extracti64x4_epi64(a, 1));
            ab64[0] = _mm512_cvtepu32_epi64(_mm512_castsi512_si256(ab));
            ab64[1] = _mm512_cvtepu32_epi64(_mm512_extracti64x4_epi64(ab, 1));
            __m512i dp64[2], ch64[2];
            for (int h = 0; h < 2; ++h) {
                dp64[h] = _mm512_mul_epu32(a64[h], p64[h]);
                ch64[h] = _mm512_mul_epu32(ab64[h], p64[h]);
            }
            for (int k = 0; k < 4; ++k) {
                const __mmask16 m = pass & _mm512_cmpeq_epi32_mask(code, _mm512_set1_epi32(k));
                cnt[k] = _mm512_mask_add_epi32(cnt[k], m, cnt[k], one);
                q[k] = _mm512_mask_add_epi32(q[k], m, q[k], vq);
                d[k] = _mm512_mask_add_epi32(d[k], m, d[k], vd);
                const __mmask8 m0 = (__mmask8)(m & 0xFF), m1 = (__mmask8)(m >> 8);
                p[k][0] = _mm512_mask_add_epi64(p[k][0], m0, p[k][0], p64[0]);
                p[k][1] = _mm512_mask_add_epi64(p[k][1], m1, p[k][1], p64[1]);
                dp[k][0] = _mm512_mask_add_epi64(dp[k][0], m0, dp[k][0], dp64[0]);
                dp[k][1] = _mm512_mask_add_epi64(dp[k][1], m1, dp[k][1], dp64[1]);
                ch[k][0] = _mm512_mask_add_epi64(ch[k][0], m0, ch[k][0], ch64[0]);
                ch[k][1] = _mm512_mask_add_epi64(ch[k][1], m1, ch[k][1], ch64[1]);
            }
        }
        ok &= bad == 0;
        for (int k = 0; k < 4; ++k) {
            const uint32_t g = t.pair_group[k];
            if (g >= 6) continue;
            u128* r = out->v[g];
            r[kAggCount] += (uint64_t)_mm512_reduce_add_epi32(cnt[k]);
            r[kAggQty] += (uint64_t)(uint32_t)_mm512_reduce_add_epi32(q[k]) * 100u;
            r[kAggDisc] += (uint64_t)(uint32_t)_mm512_reduce_add_epi32(d[k]);
            r[kAggBasePrice] += (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(p[k][0], p[k][1]));
            r[kAggDiscPrice] += (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(dp[k][0], dp[k][1]));
            r[kAggCharge] += (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(ch[k][0], ch[k][1]));
        }
    }
    return ok;
}

// 64 rows per step with AVX-512 VNNI and VBMI: the host form of the GPU kernels' byte-plane dot
// products. Per step the rows' group masks come from the flag bits by bit extracts (pair layout:
// the 2-bit pair codes; separate layout: the 2-bit return flags and the 1-bit line stati), the
// prices become three byte planes (byte k of rows 0..63, by byte permutes), and
// (100 - d)(100 + t) two 7-bit planes from a 128-entry byte table indexed by 9 d + t. Then, per
// group, vpdpbusd adds four rows' byte products into each 32-bit lane: quantity and discount
// against the group's 0/1 bytes, and every price plane against the 0/1 bytes, 100 - d and the two
// charge planes: 14 instructions per group for 64 rows. A step with a passing row outside that
// fast domain (discount > 10, tax > 8 or a price >= 2^24; TPC-H data has none) goes to the 16-row
// kernel above (pair layout) or the row loop (separate layout), so every result stays exact.
// Steps are staged 64 at a time and the groups visit them in turn, so that one group's 14
// accumulators fit in the registers; a lane adds at most 64 x 4 x 255 x 127 < 2^31 before it is
// folded into 64 bits. Rows [begin, end) with begin and end multiples of 64.
constexpr uint32_t kVSteps = 64;

struct VnniTables {
    alignas(64) uint8_t abl[128], abh[128];   // 9 d + t -> low / high 7 bits of (100 - d)(100 + t)
    alignas(64) uint8_t plane[3][64];         // permute indices: byte k of the price of row j
    VnniTables() {
        for (int i = 0; i < 128; ++i) {
            const int d = i / 9, x = i % 9;
            const int ab = d <= 10 ? (100 - d) * (100 + x) : 0;
            abl[i] = (uint8_t)(ab & 127);
            abh[i] = (uint8_t)(ab >> 7);
        }
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 64; ++j) plane[k][j] = (uint8_t)((4 * j + k) & 127);
    }
};

__attribute__((target("avx512f,avx512bw,avx512dq"))) inline uint64_t lane_sum(__m512i v) {
    const __m512i lo = _mm512_cvtepu32_epi64(_mm512_castsi512_si256(v));
    const __m512i hi = _mm512_cvtepu32_epi64(_mm512_extracti64x4_epi64(v, 1));
    return (uint64_t)_mm512_reduce_add_epi64(_mm512_add_epi64(lo, hi));
}

bool aggregate_rows(const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out);

// kPair: pair codes, 4 masks (code k -> group t.pair_group[k]); else 6 masks, one per group.
template <bool kPair>
__attribute__((target("avx512f,avx512bw,avx512dq,avx512vnni,avx512vbmi,bmi2,popcnt"))) bool aggregate_vnni(
    const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out) {
    constexpr int NG = kPair ? 4 : 6;
    if (cutoff_rel < 0) return true;   // no row passes
    static const VnniTables tab;
    const __m512i cut = _mm512_set1_epi16((short)(uint16_t)std::min<int32_t>(cutoff_rel, 65535));
    const __m512i ones = _mm512_set1_epi8(1), hundred = _mm512_set1_epi8(100), low4 = _mm512_set1_epi8(15);
    const __m512i ten = _mm512_set1_epi8(10), eight = _mm512_set1_epi8(8), top = _mm512_set1_epi32((int)0xFF000000u);
    const __m512i abl0 = _mm512_load_si512(tab.abl), abl1 = _mm512_load_si512(tab.abl + 64);
    const __m512i abh0 = _mm512_load_si512(tab.abh), abh1 = _mm512_load_si512(tab.abh + 64);
    __m512i pidx[3];
    for (int k = 0; k < 3; ++k) pidx[k] = _mm512_load_si512(tab.plane[k]);
    constexpr uint64_t kEven = 0x5555555555555555ull, kOdd = 0xAAAAAAAAAAAAAAAAull;
    __m512i st[kVSteps][6];   // per step: price planes 0..2, 100 - d, charge planes low, high
    uint64_t gm[kVSteps][NG]; // per step: rows of each code (pair) or group (separate) that pass
    bool ok = true;
    for (uint64_t s0 = begin; s0 < end; s0 += (uint64_t)kVSteps * 64) {
        const uint32_t ns = (uint32_t)std::min<uint64_t>(kVSteps, (end - s0) / 64);
        for (uint32_t j = 0; j < ns; ++j) {
            const uint64_t i = s0 + 64ull * j;
            const __m512i sh0 = _mm512_loadu_si512(t.ship + i), sh1 = _mm512_loadu_si512(t.ship + i + 32);
            const uint64_t pass = (uint64_t)_mm512_cmple_epu16_mask(sh0, cut) |
                                  ((uint64_t)_mm512_cmple_epu16_mask(sh1, cut) << 32);
            const __m512i D = _mm512_loadu_si512(t.disc + i), X = _mm512_loadu_si512(t.tax + i);
            const __m512i p0 = _mm512_loadu_si512(t.price + i), p1 = _mm512_loadu_si512(t.price + i + 16);
            const __m512i p2 = _mm512_loadu_si512(t.price + i + 32), p3 = _mm512_loadu_si512(t.price + i + 48);
            const uint64_t outside = _mm512_mask_cmpgt_epu8_mask(pass, D, ten) | _mm512_mask_cmpgt_epu8_mask(pass, X, eight);
            const __m512i por = _mm512_or_si512(_mm512_or_si512(p0, p1), _mm512_or_si512(p2, p3));
            if (outside || _mm512_test_epi32_mask(por, top)) {
                ok &= kPair ? aggregate_pair_avx512(t, i, i + 64, cutoff_rel, out)
                            : aggregate_rows(t, i, i + 64, cutoff_rel, out);
                for (int k = 0; k < NG; ++k) gm[j][k] = 0;
                for (int k = 0; k < 6; ++k) st[j][k] = _mm512_setzero_si512();
                continue;
            }
            uint64_t w0, w1;
            memcpy(&w0, (kPair ? t.flags : t.rf) + i / 16, 8);
            memcpy(&w1, (kPair ? t.flags : t.rf) + i / 16 + 2, 8);
            const uint64_t lo = _pext_u64(w0, kEven) | (_pext_u64(w1, kEven) << 32);
            const uint64_t hi = _pext_u64(w0, kOdd) | (_pext_u64(w1, kOdd) << 32);
            if constexpr (kPair) {
                gm[j][0] = pass & ~lo & ~hi;
                gm[j][1] = pass & lo & ~hi;
                gm[j][2] = pass & ~lo & hi;
                gm[j][3] = pass & lo & hi;
            } else {
                // return flag codes A=0 N=1 R=2 (3 is no group), line status F=0 O=1:
                // group 2 rf + ls
                uint64_t ls;
                memcpy(&ls, t.ls + i / 32, 8);
                const uint64_t a = pass & ~lo & ~hi, n = pass & lo & ~hi, r = pass & ~lo & hi;
                gm[j][0] = a & ~ls;
                gm[j][1] = a & ls;
                gm[j][2] = n & ~ls;
                gm[j][3] = n & ls;
                gm[j][4] = r & ~ls;
                gm[j][5] = r & ls;
            }
            for (int k = 0; k < 3; ++k)
                st[j][k] = _mm512_mask_blend_epi8(0xFFFFFFFF00000000ull, _mm512_permutex2var_epi8(p0, pidx[k], p1),
                                                  _mm512_permutex2var_epi8(p2, pidx[k], p3));
            // 9 d + t on 4-bit fields (no carry between bytes; rows outside the domain do not pass)
            const __m512i d4 = _mm512_and_si512(D, low4), t4 = _mm512_and_si512(X, low4);
            const __m512i idx = _mm512_add_epi8(_mm512_add_epi8(_mm512_slli_epi16(d4, 3), d4), t4);
            st[j][3] = _mm512_sub_epi8(hundred, D);
            st[j][4] = _mm512_permutex2var_epi8(abl0, idx, abl1);
            st[j][5] = _mm512_permutex2var_epi8(abh0, idx, abh1);
        }
        for (int k = 0; k < NG; ++k) {
            const uint32_t g = kPair ? t.pair_group[k] : (uint32_t)k;
            if (g >= 6) continue;
            __m512i aq = _mm512_setzero_si512(), ad = aq, ap[3] = {aq, aq, aq}, aa[3] = {aq, aq, aq},
                    al[3] = {aq, aq, aq}, ah[3] = {aq, aq, aq};
            uint64_t cnt = 0;
            for (uint32_t j = 0; j < ns; ++j) {
                const uint64_t m = gm[j][k];
                cnt += (uint64_t)_mm_popcnt_u64(m);
                const uint64_t i = s0 + 64ull * j;
                const __m512i w = _mm512_maskz_mov_epi8(m, ones);
                const __m512i ak = _mm512_maskz_mov_epi8(m, st[j][3]);
                const __m512i lk = _mm512_maskz_mov_epi8(m, st[j][4]);
                const __m512i hk = _mm512_maskz_mov_epi8(m, st[j][5]);
                aq = _mm512_dpbusd_epi32(aq, _mm512_loadu_si512(t.qty + i), w);
                ad = _mm512_dpbusd_epi32(ad, _mm512_loadu_si512(t.disc + i), w);
                for (int b = 0; b < 3; ++b) {
                    ap[b] = _mm512_dpbusd_epi32(ap[b], st[j][b], w);
                    aa[b] = _mm512_dpbusd_epi32(aa[b], st[j][b], ak);
                    al[b] = _mm512_dpbusd_epi32(al[b], st[j][b], lk);
                    ah[b] = _mm512_dpbusd_epi32(ah[b], st[j][b], hk);
                }
            }
            uint64_t P = 0, DP = 0, CH = 0;
            for (int b = 0; b < 3; ++b) {
                P += lane_sum(ap[b]) << (8 * b);
                DP += lane_sum(aa[b]) << (8 * b);
                CH += (lane_sum(al[b]) + (lane_sum(ah[b]) << 7)) << (8 * b);
            }
            u128* r = out->v[g];
            r[kAggCount] += cnt;
            r[kAggQty] += lane_sum(aq) * 100u;
            r[kAggDisc] += lane_sum(ad);
            r[kAggBasePrice] += P;
            r[kAggDiscPrice] += DP;
            r[kAggCharge] += CH;
        }
    }
    return ok;
}

}  // namespace

bool cpu_aggregate_compressed(const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out) {
    static const bool avx512 = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
                               __builtin_cpu_supports("avx512dq");
    static const bool vnni = avx512 && __builtin_cpu_supports("avx512vnni") && __builtin_cpu_supports("avx512vbmi") &&
                             __builtin_cpu_supports("bmi2") && __builtin_cpu_supports("popcnt");
    if (vnni && end - begin >= 128) {
        // head and tail around a 64-aligned body
        const uint64_t b = std::min<uint64_t>(end, (begin + 63) & ~(uint64_t)63);
        const uint64_t e = std::max<uint64_t>(b, end & ~(uint64_t)63);
        bool ok = true;
        if (begin < b) ok &= cpu_aggregate_compressed(t, begin, b, cutoff_rel, out);
        if (b < e) ok &= t.pair ? aggregate_vnni<true>(t, b, e, cutoff_rel, out) : aggregate_vnni<false>(t, b, e, cutoff_rel, out);
        if (e < end) ok &= cpu_aggregate_compressed(t, e, end, cutoff_rel, out);
        return ok;
    }
    if (avx512 && t.pair && end - begin >= 64) {
        // scalar head and tail around a 16-aligned body
        const uint64_t b = std::min<uint64_t>(end, (begin + 15) & ~(uint64_t)15);
        const uint64_t e = std::max<uint64_t>(b, end & ~(uint64_t)15);
        bool ok = true;
        if (begin < b) ok &= cpu_aggregate_compressed(t, begin, b, cutoff_rel, out);
        if (b < e) ok &= aggregate_pair_avx512(t, b, e, cutoff_rel, out);
        if (e < end) ok &= cpu_aggregate_compressed(t, e, end, cutoff_rel, out);
        return ok;
    }
    return aggregate_rows(t, begin, end, cutoff_rel, out);
}

namespace {

// One row at a time (heads and tails of the vector kernels, the separate layout without them).
bool aggregate_rows(const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out) {
    Partial part;
    bool ok = true;
    for (uint64_t b0 = begin; b0 < end; b0 += kBlock) {
        const uint64_t b1 = std::min(end, b0 + kBlock);
        part.clear();
        for (uint64_t i = b0; i < b1; ++i) {
            if ((int32_t)t.ship[i] > cutoff_rel) continue;
            uint32_t g;
            if (t.pair) {
                g = t.pair_group[(t.flags[i >> 4] >> (2 * (i & 15))) & 3u];
            } else {
                const uint32_t rf = (t.rf[i >> 4] >> (2 * (i & 15))) & 3u;
                const uint32_t ls = (t.ls[i >> 5] >> (i & 31)) & 1u;
                g = (rf << 1) + ls;
                if (g >= 6) continue;
            }
            const uint32_t d = t.disc[i];
            ok &= d <= 100;
            add_row(part, g, (uint64_t)t.qty[i] * 100u, d, t.tax[i], t.price[i]);
        }
        part.into(out);
    }
    return ok;
}

}  // namespace

namespace {

// Reference-typed columns, 8 rows per step with AVX-512: the passing rows' group masks from byte
// compares on the flag characters, the domain test as four unsigned compares, disc_price and
// charge by 64-bit multiplies, then per group four masked 64-bit adds, count packed above the
// quantity (bit 48) and the discount above the price (bit 45). Within a block of kBlock rows a
// lane adds at most 2^12 in-domain rows: quantity and price sums < 2^44, discount sum < 2^19,
// count <= 2^12, charge < 2^59.2, so every packed field stays exact (out-of-domain rows clear
// `ok`, and their sums are not used). Rows [begin, end) with begin and end multiples of 8.
__attribute__((target("avx512f,avx512bw,avx512dq,avx512vl"))) bool aggregate_unc_avx512(const HostUncompressed& t,
                                                                                       uint64_t begin, uint64_t end,
                                                                                       int32_t cutoff_day, Agg128* out) {
    const __m256i cut = _mm256_set1_epi32(cutoff_day);
    const __m512i hundred = _mm512_set1_epi64(100), cnt1 = _mm512_set1_epi64(1ll << 48);
    const __m512i max32 = _mm512_set1_epi64(0xFFFFFFFFll), max8 = _mm512_set1_epi64(255);
    const __m512i low45 = _mm512_set1_epi64((1ll << 45) - 1);
    const __m128i cR = _mm_set1_epi8('R'), cN = _mm_set1_epi8('N'), cF = _mm_set1_epi8('F');
    bool ok = true;
    for (uint64_t b0 = begin; b0 < end; b0 += kBlock) {
        const uint64_t b1 = std::min(end, b0 + kBlock);
        __m512i acc[6][4];
        for (int g = 0; g < 6; ++g)
            for (int k = 0; k < 4; ++k) acc[g][k] = _mm512_setzero_si512();
        __mmask8 bad = 0;
        for (uint64_t i = b0; i < b1; i += 8) {
            const __mmask8 pass_all =
                _mm256_cmple_epi32_mask(_mm256_loadu_si256(reinterpret_cast<const __m256i*>(t.ship + i)), cut);
            const __m512i Q = _mm512_loadu_si512(t.qty + i), D = _mm512_loadu_si512(t.disc + i);
            const __m512i X = _mm512_loadu_si512(t.tax + i), P = _mm512_loadu_si512(t.price + i);
            // passing rows outside the fast domain (unsigned compares also catch negative values)
            const __mmask8 wide = _mm512_mask_cmpgt_epu64_mask(pass_all, Q, max32) |
                                  _mm512_mask_cmpgt_epu64_mask(pass_all, D, hundred) |
                                  _mm512_mask_cmpgt_epu64_mask(pass_all, X, max8) |
                                  _mm512_mask_cmpgt_epu64_mask(pass_all, P, max32);
            for (uint32_t w = wide; w; w &= w - 1) {
                const uint64_t j = i + (uint64_t)__builtin_ctz(w);
                bad |= !wide_row(out, group_of(encode_return_flag(t.rf[j]), encode_line_status(t.ls[j])), t.qty[j],
                                 t.disc[j], t.tax[j], t.price[j]);
            }
            const __mmask8 pass = (__mmask8)(pass_all & ~wide);
            const __m512i DP = _mm512_mullo_epi64(_mm512_sub_epi64(hundred, D), P);
            const __m512i CH = _mm512_mullo_epi64(DP, _mm512_add_epi64(hundred, X));
            const __m512i QC = _mm512_add_epi64(Q, cnt1);
            const __m512i PD = _mm512_add_epi64(P, _mm512_slli_epi64(D, 45));
            uint64_t rfw, lsw;
            memcpy(&rfw, t.rf + i, 8);
            memcpy(&lsw, t.ls + i, 8);
            const __m128i rf = _mm_cvtsi64_si128((long long)rfw), ls = _mm_cvtsi64_si128((long long)lsw);
            // return flag R -> 2, N -> 1, anything else -> 0; line status F -> 0, anything else -> 1
            const __mmask8 r = (__mmask8)_mm_cmpeq_epi8_mask(rf, cR), n = (__mmask8)_mm_cmpeq_epi8_mask(rf, cN) & ~r;
            const __mmask8 a = (__mmask8)~(r | n), f = (__mmask8)_mm_cmpeq_epi8_mask(ls, cF), o = (__mmask8)~f;
            const __mmask8 gm[6] = {(__mmask8)(pass & a & f), (__mmask8)(pass & a & o), (__mmask8)(pass & n & f),
                                    (__mmask8)(pass & n & o), (__mmask8)(pass & r & f), (__mmask8)(pass & r & o)};
            for (int g = 0; g < 6; ++g) {
                acc[g][0] = _mm512_mask_add_epi64(acc[g][0], gm[g], acc[g][0], QC);
                acc[g][1] = _mm512_mask_add_epi64(acc[g][1], gm[g], acc[g][1], PD);
                acc[g][2] = _mm512_mask_add_epi64(acc[g][2], gm[g], acc[g][2], DP);
                acc[g][3] = _mm512_mask_add_epi64(acc[g][3], gm[g], acc[g][3], CH);
            }
        }
        ok &= bad == 0;
        for (int g = 0; g < 6; ++g) {
            const uint64_t qc = (uint64_t)_mm512_reduce_add_epi64(acc[g][0]);
            const uint64_t pr = (uint64_t)_mm512_reduce_add_epi64(_mm512_and_si512(acc[g][1], low45));
            const uint64_t d = (uint64_t)_mm512_reduce_add_epi64(_mm512_srli_epi64(acc[g][1], 45));
            u128* o = out->v[g];
            o[kAggCount] += qc >> 48;
            o[kAggQty] += qc & ((1ull << 48) - 1);
            o[kAggBasePrice] += pr;
            o[kAggDisc] += d;
            o[kAggDiscPrice] += (uint64_t)_mm512_reduce_add_epi64(acc[g][2]);
            o[kAggCharge] += (uint64_t)_mm512_reduce_add_epi64(acc[g][3]);
        }
    }
    return ok;
}

}  // namespace

bool cpu_aggregate_uncompressed(const HostUncompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_day,
                                Agg128* out) {
    static const bool avx512 = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
                               __builtin_cpu_supports("avx512dq") && __builtin_cpu_supports("avx512vl");
    if (avx512 && end - begin >= 64) {
        // row loop for the head and tail around an 8-aligned body
        const uint64_t b = std::min<uint64_t>(end, (begin + 7) & ~(uint64_t)7);
        const uint64_t e = std::max<uint64_t>(b, end & ~(uint64_t)7);
        bool ok = true;
        if (begin < b) ok &= cpu_aggregate_uncompressed(t, begin, b, cutoff_day, out);
        if (b < e) ok &= aggregate_unc_avx512(t, b, e, cutoff_day, out);
        if (e < end) ok &= cpu_aggregate_uncompressed(t, e, end, cutoff_day, out);
        return ok;
    }
    Partial part;
    bool ok = true;
    for (uint64_t b0 = begin; b0 < end; b0 += kBlock) {
        const uint64_t b1 = std::min(end, b0 + kBlock);
        part.clear();
        for (uint64_t i = b0; i < b1; ++i) {
            if (t.ship[i] > cutoff_day) continue;
            const int64_t q = t.qty[i], d = t.disc[i], x = t.tax[i], p = t.price[i];
            const uint32_t g = group_of(encode_return_flag(t.rf[i]), encode_line_status(t.ls[i]));
            if (q >= 0 && q < (1ll << 32) && d >= 0 && d <= 100 && x >= 0 && x <= 255 && p >= 0 && p < (1ll << 32))
                add_row(part, g, (uint64_t)q, (uint64_t)d, (uint64_t)x, (uint64_t)p);
            else
                ok &= wide_row(out, g, q, d, x, p);
        }
        part.into(out);
    }
    return ok;
}

namespace {

uint32_t filter_word_scalar(const uint16_t* ship, uint64_t n, int32_t cutoff_rel) {
    uint32_t bits = 0;
    for (uint64_t j = 0; j < n; ++j) bits |= (uint32_t)((int32_t)ship[j] <= cutoff_rel) << j;
    return bits;
}

// 32 ship offsets per step with AVX2: two signed 16-bit compares against the cutoff, a pack and a
// byte movemask. Offsets above 32767 (outside the compressed domain) read as negative int16, so
// such a word is redone by the scalar loop.
__attribute__((target("avx2"))) void filter_avx2(const uint16_t* ship, uint64_t begin, uint64_t end,
                                                  int32_t cutoff_rel, uint32_t* bitmap) {
    const int16_t cut = (int16_t)std::max(-1, std::min(32767, cutoff_rel));
    const __m256i vcut = _mm256_set1_epi16(cut);
    const __m256i zero = _mm256_setzero_si256();
    uint64_t w0 = begin;
    for (; w0 + 32 <= end; w0 += 32) {
        const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(ship + w0));
        const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(ship + w0 + 16));
        const __m256i gt = _mm256_permute4x64_epi64(
            _mm256_packs_epi16(_mm256_cmpgt_epi16(a, vcut), _mm256_cmpgt_epi16(b, vcut)), 0xD8);
        const __m256i neg = _mm256_packs_epi16(_mm256_cmpgt_epi16(zero, a), _mm256_cmpgt_epi16(zero, b));
        if (_mm256_movemask_epi8(neg)) bitmap[w0 / 32] = filter_word_scalar(ship + w0, 32, cutoff_rel);
        else bitmap[w0 / 32] = ~(uint32_t)_mm256_movemask_epi8(gt);
    }
    if (w0 < end) bitmap[w0 / 32] = filter_word_scalar(ship + w0, end - w0, cutoff_rel);
}

}  // namespace

void cpu_precompute_filter(const uint16_t* ship, uint64_t begin, uint64_t end, int32_t cutoff_rel, uint32_t* bitmap) {
    static const bool avx2 = __builtin_cpu_supports("avx2");
    if (avx2) {
        filter_avx2(ship, begin, end, cutoff_rel, bitmap);
        return;
    }
    for (uint64_t w0 = begin; w0 < end; w0 += 32)
        bitmap[w0 / 32] = filter_word_scalar(ship + w0, std::min<uint64_t>(32, end - w0), cutoff_rel);
}

}  // namespace q1
