// Host-side internal declarations shared by the runtime translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "q1.h"

namespace q1 {

typedef unsigned __int128 u128;
typedef __int128 i128;

// Error text of the calling thread (q1_last_error).
q1_status set_error(q1_status s, const std::string& msg);
q1_status cuda_error(cudaError_t e, const char* what);

#define Q1_CUDA(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return ::q1::cuda_error(e_, #call); \
    } while (0)

// Per-device facts and the device status word used by the kernels (kStatus* bits).
struct DeviceInfo {
    int sm_count = 0;
    uint32_t* status = nullptr;   // one device word, allocated on first use
};
q1_status device_info(int device, DeviceInfo** out);
// Reads (and clears) the status word of the current device after synchronising `stream`.
q1_status check_device_status(cudaStream_t stream, uint32_t* status_word);

// Aggregates of up to 6 groups in 128 bits: [group][aggregate].
struct Agg128 {
    u128 v[6][6];
    void clear();
    void add(const Agg128& o);
};
void agg_from_device_words(const unsigned long long* words, Agg128* out);   // [6][6][lo,hi]
void agg_to_i128(const Agg128& a, q1_i128* out);                              // 36 entries

// Column byte sizes.
uint64_t words16(uint64_t rows);   // 2-bit containers
uint64_t words32(uint64_t rows);   // 1-bit containers

// ------------------------------------------------------------------------------------------
// CPU coprocessing share (the reference's CoProc / Morsel<KernelX100>, src/cpu.h:23-38)
// ------------------------------------------------------------------------------------------

// Host-side fault injection (q1_inject_fault): the next `count` events of a kind fail.
enum FaultKind : int { kFaultCpuWorker = 1, kFaultDeviceAlloc = 2, kFaultPinnedAlloc = 3, kFaultServeRound = 4,
                       kFaultKinds = 5 };
bool take_fault(FaultKind kind);   // consumes one pending fault of `kind`, if any
void set_faults(int kind, uint32_t count);

// A fixed pool of worker threads executing morsel-driven jobs.
class CpuPool {
public:
    explicit CpuPool(int threads);
    ~CpuPool();
    int threads() const { return (int)workers_.size(); }
    // Runs fn(worker_id) on every worker; returns immediately. wait() joins the job.
    void start(std::function<void(int)> fn);
    // Returns false if a worker raised an exception (message in error()).
    bool wait();
    // True once a worker of the current job has raised an exception.
    bool failed();
    const std::string& error() const { return error_; }

private:
    void loop(int id);
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_start_, cv_done_;
    std::function<void(int)> job_;
    uint64_t generation_ = 0;
    int running_ = 0;
    bool stop_ = false;
    bool failed_ = false;
    std::string error_;
};

// Bounded blocking queue of filter chunks (the reference's moodycamel queue, src/cpu.h:12-21).
struct FilterChunk {
    uint64_t offset;
    uint64_t num;
};
class ChunkQueue {
public:
    void push(FilterChunk c);
    // Waits up to timeout_ms; returns false on timeout or when closed and empty.
    bool pop(FilterChunk* c, int timeout_ms);
    void close();
    void reset();

private:
    std::mutex m_;
    std::condition_variable cv_;
    std::deque<FilterChunk> q_;
    bool closed_ = false;
};

// Host views of a table's columns.
struct HostCompressed {
    const uint16_t* ship = nullptr;
    const uint8_t* disc = nullptr;
    const uint32_t* price = nullptr;
    const uint8_t* tax = nullptr;
    const uint8_t* qty = nullptr;
    const uint32_t* flags = nullptr;   // pair codes
    const uint32_t* rf = nullptr;      // separate
    const uint32_t* ls = nullptr;
    bool pair = true;
    uint8_t pair_group[4] = {0, 0, 0, 0};
};
struct HostUncompressed {
    const int32_t* ship = nullptr;
    const int64_t* disc = nullptr;
    const int64_t* price = nullptr;
    const int64_t* tax = nullptr;
    const int64_t* qty = nullptr;
    const char* rf = nullptr;
    const char* ls = nullptr;
};

// Exact aggregation of rows [begin, end) on the calling thread. Returns false if a row is
// outside the kernels' domain (same rule as the GPU: discount <= 100 etc.).
bool cpu_aggregate_compressed(const HostCompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_rel, Agg128* out);
bool cpu_aggregate_uncompressed(const HostUncompressed& t, uint64_t begin, uint64_t end, int32_t cutoff_day,
                                Agg128* out);
// Bitmap words for rows [begin, end); begin must be a multiple of 32 (src/main.cu:367-368).
void cpu_precompute_filter(const uint16_t* ship, uint64_t begin, uint64_t end, int32_t cutoff_rel, uint32_t* bitmap);
// Rate at which `threads` host threads read [buf, buf + bytes), GB/s (q1_measure_host_read).
double host_read_gbs(const void* buf, uint64_t bytes, int threads);

}  // namespace q1
