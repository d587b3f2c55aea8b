// CPU share of the coprocessing mode, the worker pool that runs it, and the filter-chunk queue.
//
// The reference runs its CPU share with Morsel<KernelX100<...>> (cpu/kernel_x100.hpp:423-665)
// behind CoProc (src/cpu.cpp:13-69) and hands filter chunks to the GPU loop through a moodycamel
// queue (src/cpu.h:12-21). This file is this project's own equivalent: a fixed thread pool with
// an atomic morsel cursor supplied by the caller, an exact 128-bit merge, and a blocking queue.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>

#include "q1_common.cuh"
#include "q1_internal.h"

namespace q1 {

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

bool cpu_aggregate_compressed(const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out) {
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

bool cpu_aggregate_uncompressed(const HostUncompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_day,
                                Agg128* out) {
    Partial part;
    bool ok = true;
    for (uint64_t b0 = begin; b0 < end; b0 += kBlock) {
        const uint64_t b1 = std::min(end, b0 + kBlock);
        part.clear();
        for (uint64_t i = b0; i < b1; ++i) {
            if (t.ship[i] > cutoff_day) continue;
            const int64_t q = t.qty[i], d = t.disc[i], x = t.tax[i], p = t.price[i];
            ok &= (q >= 0 && q < (1ll << 32) && d >= 0 && d <= 100 && x >= 0 && x <= 255 && p >= 0 && p < (1ll << 32));
            const uint32_t g = group_of(encode_return_flag(t.rf[i]), encode_line_status(t.ls[i]));
            add_row(part, g, (uint64_t)q, (uint64_t)d, (uint64_t)x, (uint64_t)p);
        }
        part.into(out);
    }
    return ok;
}

void cpu_precompute_filter(const uint16_t* ship, uint64_t begin, uint64_t end, int32_t cutoff_rel, uint32_t* bitmap) {
    for (uint64_t w0 = begin; w0 < end; w0 += 32) {
        uint32_t bits = 0;
        const uint64_t n = std::min<uint64_t>(32, end - w0);
        for (uint64_t j = 0; j < n; ++j) bits |= (uint32_t)((int32_t)ship[w0 + j] <= cutoff_rel) << j;
        bitmap[w0 / 32] = bits;
    }
}

}  // namespace q1
