// Allocation-free variant of the compressed scan launch (q1_launch_compressed_noalloc).
//
// Who needs it: a host program that owns all device memory itself (a database engine or plugin
// host with its own pool, a process under a hard device-memory cap) or a latency-critical loop
// in which cudaMalloc/cudaFree must never run (cudaFree, for one, synchronises the device).
// q1_launch_compressed allocates once, on first use of a device: the word in which the kernels
// report expired waits and out-of-domain rows. This entry point allocates nothing. Its scratch
// memory is the file-scope array below, which every GPU that loads the library holds until the
// process exits:
//   words [0, 32)                 status block (word 0 = the kernel status bits)
//   words [32, 32 + 256 * 72)     one record per CTA: 6 groups x 6 aggregates x (lo, hi)
// In the placements with per-thread or per-lane tables (in_registers, in_registers_per_thread,
// local_mem, shared_mem_per_thread) the scan kernel writes its CTA's partial sums into its record
// instead of one 128-bit atomic per (group, aggregate) into the caller's table, and a one-block
// reduction kernel adds the records into the caller's table. The global placement keeps no CTA
// partials: its warps add every tile's sums straight into the caller's table, as they do under
// q1_launch_compressed, so its records stay zero and the reduction adds nothing.
// Limit: at most kNoAllocMaxCtas CTAs per launch (the library uses one per SM, 148 on a B200).
//
// The array is shared by every call and keeps the last call's contents: each call clears the
// status word before launching, and every CTA overwrites its whole record. Calls whose GPU work
// overlaps (two host threads, or two streams of one device) race on this array.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "q1.h"
#include "q1_common.cuh"
#include "q1_internal.h"
#include "q1_kernels.h"
#include "q1_ptx.cuh"

namespace q1 {

constexpr uint32_t kNoAllocMaxCtas = 256;
constexpr uint32_t kNoAllocStatusWords = 32;
constexpr uint32_t kRecordWords = kNumGroups * kNumAggs * 2;   // 72
constexpr uint32_t kNoAllocWords = kNoAllocStatusWords + kNoAllocMaxCtas * kRecordWords;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];   // 147,712 bytes

// Device address of g_noalloc_scratch per device, resolved with that device current by the
// first call on the device, and again by the first call after the device's context was replaced
// (cudaDeviceReset destroys the context and the module with the array; the next context loads it
// again, possibly at another address). A context is told apart by the unique id the driver gives
// every context (cuCtxGetId), reached through the runtime's driver entry points so that the
// library needs no link against the driver library.
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

struct NoAllocSlot {
    unsigned long long ctx_id = 0;
    unsigned long long* ptr = nullptr;
};

static std::mutex g_noalloc_mutex;
static NoAllocSlot g_noalloc_slot[64];
static CtxGetCurrentFn g_ctx_get_current = nullptr;
static CtxGetIdFn g_ctx_get_id = nullptr;

static q1_status current_context_id(unsigned long long* id) {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult found;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &found);
        if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !f)
            return set_error(Q1_ERR_CUDA, "driver entry point cuCtxGetCurrent not found");
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &found);
        if (e != cudaSuccess || found != cudaDriverEntryPointSuccess || !f)
            return set_error(Q1_ERR_CUDA, "driver entry point cuCtxGetId not found");
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return set_error(Q1_ERR_CUDA, "no current CUDA context");
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return set_error(Q1_ERR_CUDA, "cuCtxGetId failed");
    return Q1_OK;
}

static q1_status noalloc_scratch(int device, unsigned long long** out) {
    if (device < 0 || device >= 64) return set_error(Q1_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    // Makes the device's primary context current, creating it if a reset destroyed it.
    Q1_CUDA(cudaSetDevice(device));
    unsigned long long id = 0;
    q1_status st = current_context_id(&id);
    if (st != Q1_OK) return st;
    NoAllocSlot& slot = g_noalloc_slot[device];
    if (!slot.ptr || slot.ctx_id != id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        slot.ptr = static_cast<unsigned long long*>(p);
        slot.ctx_id = id;
    }
    *out = slot.ptr;
    return Q1_OK;
}

// Sums the first `nrec` CTA records into the caller's table (one thread per entry, fixed order).
__global__ void __launch_bounds__(64) noalloc_reduce_records(const unsigned long long* __restrict__ records,
                                                            uint32_t nrec, unsigned long long* out) {
    const uint32_t i = threadIdx.x;
    if (i >= kNumGroups * kNumAggs) return;
    uint64_t lo = 0, hi = 0;
    for (uint32_t r = 0; r < nrec; ++r) {
        const uint64_t a = records[(uint64_t)r * kRecordWords + 2 * i];
        const uint64_t b = records[(uint64_t)r * kRecordWords + 2 * i + 1];
        const uint64_t nlo = lo + a;
        hi += b + (nlo < lo ? 1u : 0u);
        lo = nlo;
    }
    ptx::atomic_add_u128(out + 2 * i, lo, hi);
}

}  // namespace q1

using namespace q1;

extern "C" q1_status q1_launch_compressed_noalloc(q1_placement placement, const q1_compressed_columns* c,
                                                  uint64_t rows, int32_t cutoff_day, int32_t use_filter,
                                                  const q1_launch_config* cfg, q1_i128* dev_aggregates,
                                                  void* cuda_stream) {
    if (!c || !dev_aggregates) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if ((int)placement < 0 || (int)placement >= Q1_NUM_PLACEMENTS) return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown placement");
    const bool pair = c->flag_packing == Q1_FLAGS_PAIR_2BIT;
    if (!pair && c->flag_packing != Q1_FLAGS_SEPARATE) return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");
    if (pair && (c->num_pair_codes < 1 || c->num_pair_codes > 4))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "pair dictionary must have 1..4 entries");
    uint8_t pg[4] = {0, 0, 0, 0};
    if (pair) {
        for (uint32_t i = 0; i < 4; ++i) {
            pg[i] = i < c->num_pair_codes ? c->pair_group[i] : c->pair_group[0];
            if (pg[i] >= 6) return set_error(Q1_ERR_INVALID_ARGUMENT, "pair dictionary entry is not a group 0..5");
        }
    }
    const int layout = pair ? (use_filter ? kLayPairFilter : kLayPair) : (use_filter ? kLaySepFilter : kLaySep);
    const uint8_t* cols[7] = {
        reinterpret_cast<const uint8_t*>(use_filter ? (const void*)c->filter : (const void*)c->shipdate),
        c->quantity, c->discount, c->tax, reinterpret_cast<const uint8_t*>(c->extendedprice),
        reinterpret_cast<const uint8_t*>(pair ? c->flags : c->returnflag), reinterpret_cast<const uint8_t*>(c->linestatus)};
    const int ncols = pair ? 6 : 7;
    if (((uintptr_t)dev_aggregates & 15u) != 0) return set_error(Q1_ERR_INVALID_ARGUMENT, "aggregate buffer must be 16-byte aligned");
    for (int k = 0; k < ncols; ++k) {
        if (!cols[k] && rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
        if (((uintptr_t)cols[k] & 15u) != 0)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "device columns must start on a 16-byte boundary");
    }
    if (rows == 0) return Q1_OK;

    int dev = 0;
    Q1_CUDA(cudaGetDevice(&dev));
    int sms = 0;
    Q1_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int max_blocks = 0;
    if (cfg) {
        if (cfg->threads_per_block < 0 || cfg->threads_per_block % 32 != 0)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "threads per block must be a multiple of 32");
        if (cfg->blocks > 0) max_blocks = cfg->blocks;
        else if (cfg->threads_per_block > 0 && cfg->tuples_per_thread > 0) {
            const uint64_t per = (uint64_t)cfg->threads_per_block * (uint64_t)cfg->tuples_per_thread;
            max_blocks = (int)std::min<uint64_t>((rows + per - 1) / per, (uint64_t)sms);
        }
    }
    const uint32_t grid = scan_grid_blocks(layout, placement, rows, sms, max_blocks);
    const uint64_t kMaxRows = scan_max_rows_per_launch(layout, placement, grid);
    if (grid > kNoAllocMaxCtas)
        return set_error(Q1_ERR_INVALID_ARGUMENT,
                         "q1_launch_compressed_noalloc: the launch needs " + std::to_string(grid) +
                             " CTAs but the static scratch holds records for at most " +
                             std::to_string(kNoAllocMaxCtas) + "; pass cfg->blocks <= " +
                             std::to_string(kNoAllocMaxCtas));

    unsigned long long* scratch = nullptr;
    q1_status st = noalloc_scratch(dev, &scratch);
    if (st != Q1_OK) return st;
    uint32_t* status = reinterpret_cast<uint32_t*>(scratch);
    unsigned long long* records = scratch + kNoAllocStatusWords;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    Q1_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), stream));

    for (uint64_t off = 0; off < rows; off += kMaxRows) {
        const uint64_t n = std::min(kMaxRows, rows - off);
        ScanParams prm{};
        const int bits[7] = {(layout == kLayPairFilter || layout == kLaySepFilter) ? 1 : 16, 8, 8, 8, 32, 2, 1};
        for (int k = 0; k < ncols; ++k) prm.col[k] = cols[k] + off * (uint64_t)bits[k] / 8;
        prm.rows = n;
        const int64_t rel = (int64_t)cutoff_day - kShipDateFrame;
        prm.cutoff = rel < -1 ? -1 : (rel > 32767 ? 32767 : (int32_t)rel);
        prm.qty_scale = 100u;
        for (int i = 0; i < 4; ++i) prm.pair_group[i] = pg[i];
        prm.out = reinterpret_cast<unsigned long long*>(dev_aggregates);
        prm.status = status;
        prm.records = records;
        const uint32_t nrec = scan_grid_blocks(layout, placement, n, sms, max_blocks);
        cudaError_t e = launch_scan(layout, placement, prm, sms, max_blocks, stream);
        if (e != cudaSuccess) return cuda_error(e, "scan kernel launch");
        noalloc_reduce_records<<<1, 64, 0, stream>>>(records, nrec, reinterpret_cast<unsigned long long*>(dev_aggregates));
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_error(e, "record reduction launch");
    }
    // Synchronous: report expired waits / out-of-domain rows through the returned status.
    Q1_CUDA(cudaStreamSynchronize(stream));
    uint32_t bits = 0;
    Q1_CUDA(cudaMemcpy(&bits, status, sizeof(bits), cudaMemcpyDeviceToHost));
    if (bits & 1u) return set_error(Q1_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
    if (bits) return set_error(Q1_ERR_DOMAIN, "a row is outside the kernel domain (discount > 100)");
    return Q1_OK;
}
