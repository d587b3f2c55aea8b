// Query context: the reference's tpch_01 driver (src/main.cu:738-916) as a library.
//
//   load    -> compression (src/main.cu:773-803) and placement of the columns: HBM-resident
//              (copied once) or pinned host memory (streamed every run, src/main.cu:567-719)
//   run     -> execute_query_1_once (src/main.cu:498-736): aggregate zeroing, CPU/GPU split
//              (:517-550), chunked H2D + kernel per stream round robin, filter pushdown chunks
//              from CPU workers (:575-580), join, D2H, exact merge of the CPU share
//              (the reference merges only inside print_results, :136-148).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "q1.h"
#include "q1_common.cuh"
#include "q1_internal.h"
#include "q1_kernels.h"

using namespace q1;

namespace {

constexpr int kMaxStreams = 64;
constexpr uint64_t kAlign = 256;

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Byte sizes of the 7 column slots (tile order: ship, qty, disc, tax, price, flags|rf, ls) of
// a table of `rows` rows, and of its filter bitmap.
struct Plan {
    uint64_t bytes[7] = {0, 0, 0, 0, 0, 0, 0};
    uint64_t offset[7] = {0, 0, 0, 0, 0, 0, 0};
    uint64_t filter_bytes = 0, filter_offset = 0;
    uint64_t total = 0;
};

Plan make_plan(uint64_t rows, q1_layout layout, q1_flag_packing packing, bool with_filter) {
    Plan p;
    if (layout == Q1_LAYOUT_COMPRESSED) {
        p.bytes[0] = 2 * rows;
        p.bytes[1] = rows;
        p.bytes[2] = rows;
        p.bytes[3] = rows;
        p.bytes[4] = 4 * rows;
        p.bytes[5] = 4 * words16(rows);
        p.bytes[6] = packing == Q1_FLAGS_SEPARATE ? 4 * words32(rows) : 0;
    } else {
        p.bytes[0] = 4 * rows;
        p.bytes[1] = p.bytes[2] = p.bytes[3] = p.bytes[4] = 8 * rows;
        p.bytes[5] = p.bytes[6] = rows;
    }
    uint64_t off = 0;
    for (int c = 0; c < 7; ++c) {
        p.offset[c] = off;
        off += align_up(p.bytes[c] + 16, kAlign);   // +16: slack past the last full word
    }
    if (with_filter) {
        p.filter_bytes = 4 * words32(rows);
        p.filter_offset = off;
        off += align_up(p.filter_bytes + 16, kAlign);
    }
    p.total = off;
    return p;
}

struct PinnedBuf {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    ~PinnedBuf() { reset(); }
    void reset() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
    q1_status alloc(uint64_t bytes) {
        reset();
        if (!bytes) return Q1_OK;
        if (take_fault(kFaultPinnedAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected pinned allocation failure");
        cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaHostAlloc");
        }
        n = bytes;
        return Q1_OK;
    }
};

struct DevBuf {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    ~DevBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    q1_status alloc(uint64_t bytes) {
        reset();
        if (!bytes) return Q1_OK;
        if (take_fault(kFaultDeviceAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected device allocation failure");
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaMalloc");
        }
        n = bytes;
        return Q1_OK;
    }
};

}  // namespace

struct q1_ctx {
    int device = 0;
    DeviceInfo* di = nullptr;
    cudaStream_t streams[kMaxStreams] = {};
    int nstreams = 0;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_zeroed = nullptr;
    cudaEvent_t ev_join[kMaxStreams] = {};

    // Loaded table.
    bool loaded = false;
    uint64_t rows = 0;
    q1_layout layout = Q1_LAYOUT_COMPRESSED;
    q1_flag_packing packing = Q1_FLAGS_PAIR_2BIT;
    q1_residency residency = Q1_RESIDENCY_HBM;
    q1_column_stats stats{};
    Plan plan;
    DevBuf dtable;          // HBM residency: all columns + filter bitmap
    PinnedBuf htable;       // PINNED_HOST: all columns + filter bitmap
    std::vector<uint8_t> hcopy;   // HBM residency: host copy for the coprocessing CPU share
    bool hcopy_valid = false;
    int32_t filter_cutoff = INT32_MIN;   // cutoff the HBM bitmap was computed for (HBM)

    // Aggregates.
    DevBuf daggs;
    PinnedBuf haggs;

    // Streamed mode: per-stream chunk buffers.
    DevBuf dchunks;
    uint64_t chunk_rows = 0;
    int chunk_streams = 0;
    Plan chunk_plan;

    std::unique_ptr<CpuPool> pool;
    int cpu_threads = 1;
    ChunkQueue queue;

    std::vector<double> wall_ms, gpu_ms;

    const uint8_t* col(const uint8_t* base, int c) const { return base + plan.offset[c]; }
    uint8_t* host_base() {
        if (residency == Q1_RESIDENCY_PINNED_HOST) return htable.p;
        return hcopy_valid ? hcopy.data() : nullptr;
    }
};

static q1_status select_device(q1_ctx* ctx) {
    Q1_CUDA(cudaSetDevice(ctx->device));
    return Q1_OK;
}

extern "C" {

q1_status q1_sync_check(void* cuda_stream) {
    int dev = 0;
    Q1_CUDA(cudaGetDevice(&dev));
    DeviceInfo* di = nullptr;
    q1_status st = device_info(dev, &di);
    if (st != Q1_OK) return st;
    return check_device_status((cudaStream_t)cuda_stream, di->status);
}

void q1_params_default(q1_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->placement = Q1_PLACEMENT_IN_REGISTERS_PER_THREAD;   // src/constants.hpp:21
    p->apply_compression = 0;
    p->use_filter_pushdown = 0;
    p->use_coprocessing = 0;
    p->cpu_fraction = 0.5;                                  // src/constants.hpp:22-23
    p->streams = 4;                                         // src/constants.hpp:12
    p->threads_per_block = 0;
    p->tuples_per_thread = 0;
    p->tuples_per_launch = 1 << 21;                         // src/constants.hpp:13
    p->runs = 5;                                            // src/constants.hpp:17
    p->cutoff_day = Q1_DEFAULT_CUTOFF_DAY;
}

q1_status q1_params_validate(const q1_params* p) {
    if (!p) return set_error(Q1_ERR_INVALID_ARGUMENT, "null params");
    if (p->placement < 0 || p->placement >= Q1_NUM_PLACEMENTS) return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown placement");
    if (p->use_filter_pushdown && !p->apply_compression)
        return set_error(Q1_ERR_INVALID_ARGUMENT,
                         "Filter precomputation is only currently supported when compression is applied; "
                         "invoke with \"--apply-compression\".");
    if (p->threads_per_block < 0 || p->threads_per_block % 32 != 0 || p->threads_per_block > 1024)
        return set_error(Q1_ERR_INVALID_ARGUMENT,
                         "All kernels only support numbers of threads per grid block which are multiples of the warp size (32)");
    if (p->tuples_per_thread < 0) return set_error(Q1_ERR_INVALID_ARGUMENT, "tuples per thread must be >= 0");
    if (p->tuples_per_launch <= 0 || p->tuples_per_launch % 128 != 0)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "tuples per kernel launch must be a positive multiple of 128");
    if (p->runs <= 0) return set_error(Q1_ERR_INVALID_ARGUMENT, "Number of runs must be positive");
    if (!(p->cpu_fraction >= 0.0 && p->cpu_fraction <= 1.0))
        return set_error(Q1_ERR_INVALID_ARGUMENT,
                         "The fraction of aggregation work be performed by the CPU must be in the range 0.0 - 1.0");
    if (p->streams < 1 || p->streams > kMaxStreams) return set_error(Q1_ERR_INVALID_ARGUMENT, "streams must be 1..64");
    return Q1_OK;
}

q1_status q1_open(q1_ctx** out, const q1_device_opts* opts) {
    if (!out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<q1_ctx> ctx(new q1_ctx());
    ctx->device = opts ? opts->device : 0;
    int ndev = 0;
    Q1_CUDA(cudaGetDeviceCount(&ndev));
    if (ctx->device < 0 || ctx->device >= ndev) return set_error(Q1_ERR_INVALID_ARGUMENT, "no such CUDA device");
    q1_status st = select_device(ctx.get());
    if (st != Q1_OK) return st;
    st = device_info(ctx->device, &ctx->di);
    if (st != Q1_OK) return st;
    for (int i = 0; i < kMaxStreams; ++i) ctx->streams[i] = nullptr;
    Q1_CUDA(cudaStreamCreateWithFlags(&ctx->streams[0], cudaStreamNonBlocking));
    ctx->nstreams = 1;
    Q1_CUDA(cudaEventCreate(&ctx->ev_start));
    Q1_CUDA(cudaEventCreate(&ctx->ev_stop));
    Q1_CUDA(cudaEventCreateWithFlags(&ctx->ev_zeroed, cudaEventDisableTiming));
    st = ctx->daggs.alloc(Q1_NUM_POTENTIAL_GROUPS * Q1_NUM_AGGREGATES * 16);
    if (st != Q1_OK) return st;
    st = ctx->haggs.alloc(Q1_NUM_POTENTIAL_GROUPS * Q1_NUM_AGGREGATES * 16);
    if (st != Q1_OK) return st;
    int threads = opts ? opts->cpu_threads : 0;
    if (threads <= 0) {
        // hardware_concurrency/2, minus core 0 (cpu/kernel_x100.hpp:535-548, wo_core0 = true)
        threads = (int)std::thread::hardware_concurrency() / 2 - 1;
        if (threads < 1) threads = 1;
    }
    ctx->cpu_threads = threads;
    *out = ctx.release();
    return Q1_OK;
}

q1_status q1_close(q1_ctx* ctx) {
    if (!ctx) return Q1_OK;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < ctx->nstreams; ++i) {
        if (ctx->streams[i]) {
            cudaStreamSynchronize(ctx->streams[i]);
            cudaStreamDestroy(ctx->streams[i]);
        }
        if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
    if (ctx->ev_zeroed) cudaEventDestroy(ctx->ev_zeroed);
    delete ctx;
    return Q1_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Loading
// ---------------------------------------------------------------------------------------------

static void unload(q1_ctx* ctx) {
    ctx->loaded = false;
    ctx->dtable.reset();
    ctx->htable.reset();
    ctx->hcopy.clear();
    ctx->hcopy.shrink_to_fit();
    ctx->hcopy_valid = false;
    ctx->filter_cutoff = INT32_MIN;
    ctx->rows = 0;
}

// Places host columns (already in the plan's layout, contiguous at `src`) per residency.
static q1_status place_table(q1_ctx* ctx, const uint8_t* src, bool src_is_pinned_table) {
    const Plan& p = ctx->plan;
    if (ctx->residency == Q1_RESIDENCY_HBM) {
        q1_status st = ctx->dtable.alloc(p.total);
        if (st != Q1_OK) return st;
        Q1_CUDA(cudaMemset(ctx->dtable.p, 0, p.total));
        Q1_CUDA(cudaMemcpy(ctx->dtable.p, src, p.total, cudaMemcpyHostToDevice));
    } else if (!src_is_pinned_table) {
        q1_status st = ctx->htable.alloc(p.total);
        if (st != Q1_OK) return st;
        memcpy(ctx->htable.p, src, p.total);
    }
    return Q1_OK;
}

extern "C" {

q1_status q1_load_columns(q1_ctx* ctx, const q1_columns* in, uint64_t rows, q1_layout layout, q1_flag_packing packing,
                          q1_residency residency) {
    if (!ctx || !in) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (layout != Q1_LAYOUT_COMPRESSED && layout != Q1_LAYOUT_UNCOMPRESSED)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown layout");
    if (residency != Q1_RESIDENCY_HBM && residency != Q1_RESIDENCY_PINNED_HOST)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown residency");
    if (layout == Q1_LAYOUT_COMPRESSED && packing != Q1_FLAGS_PAIR_2BIT && packing != Q1_FLAGS_SEPARATE)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");
    q1_status st = select_device(ctx);
    if (st != Q1_OK) return st;
    unload(ctx);
    ctx->rows = rows;
    ctx->layout = layout;
    ctx->packing = layout == Q1_LAYOUT_COMPRESSED ? packing : Q1_FLAGS_SEPARATE;
    ctx->residency = residency;
    ctx->plan = make_plan(rows, layout, packing, true);
    const Plan& p = ctx->plan;

    // Stage the table in host memory: pinned when it stays there, pageable otherwise (the
    // pageable copy is kept as the coprocessing CPU share's source).
    uint8_t* host = nullptr;
    if (residency == Q1_RESIDENCY_PINNED_HOST) {
        st = ctx->htable.alloc(p.total);
        if (st != Q1_OK) return st;
        host = ctx->htable.p;
    } else {
        ctx->hcopy.assign(p.total, 0);
        host = ctx->hcopy.data();
    }
    memset(host, 0, p.total);
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    if (layout == Q1_LAYOUT_COMPRESSED) {
        q1_compressed_host_out o{};
        o.shipdate = reinterpret_cast<uint16_t*>(host + p.offset[0]);
        o.quantity = host + p.offset[1];
        o.discount = host + p.offset[2];
        o.tax = host + p.offset[3];
        o.extendedprice = reinterpret_cast<uint32_t*>(host + p.offset[4]);
        if (packing == Q1_FLAGS_PAIR_2BIT) o.flags = reinterpret_cast<uint32_t*>(host + p.offset[5]);
        else {
            o.returnflag = reinterpret_cast<uint32_t*>(host + p.offset[5]);
            o.linestatus = reinterpret_cast<uint32_t*>(host + p.offset[6]);
        }
        st = q1_compress_host(in, rows, packing, &o, &ctx->stats);
        if (st != Q1_OK) {
            unload(ctx);
            return st;
        }
    } else {
        if (rows && (!in->shipdate || !in->quantity || !in->discount || !in->tax || !in->extendedprice ||
                     !in->returnflag || !in->linestatus)) {
            unload(ctx);
            return set_error(Q1_ERR_INVALID_ARGUMENT, "missing input column");
        }
        const void* srcs[7] = {in->shipdate, in->quantity, in->discount, in->tax, in->extendedprice, in->returnflag,
                               in->linestatus};
        for (int c = 0; c < 7; ++c)
            if (rows) memcpy(host + p.offset[c], srcs[c], p.bytes[c]);
        ctx->stats.rows = rows;
    }
    st = place_table(ctx, host, residency == Q1_RESIDENCY_PINNED_HOST);
    if (st != Q1_OK) {
        unload(ctx);
        return st;
    }
    ctx->hcopy_valid = residency == Q1_RESIDENCY_HBM;
    ctx->loaded = true;
    return Q1_OK;
}

q1_status q1_load_compressed(q1_ctx* ctx, const q1_compressed_columns* c, uint64_t rows, q1_residency residency) {
    if (!ctx || !c) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    const bool pair = c->flag_packing == Q1_FLAGS_PAIR_2BIT;
    if (!pair && c->flag_packing != Q1_FLAGS_SEPARATE) return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");
    if (pair && (c->num_pair_codes < 1 || c->num_pair_codes > 4))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "pair dictionary must have 1..4 entries");
    if (rows && (!c->shipdate || !c->quantity || !c->discount || !c->tax || !c->extendedprice ||
                 (pair ? !c->flags : (!c->returnflag || !c->linestatus))))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
    q1_status st = select_device(ctx);
    if (st != Q1_OK) return st;
    unload(ctx);
    ctx->rows = rows;
    ctx->layout = Q1_LAYOUT_COMPRESSED;
    ctx->packing = (q1_flag_packing)c->flag_packing;
    ctx->residency = residency;
    ctx->plan = make_plan(rows, ctx->layout, ctx->packing, true);
    const Plan& p = ctx->plan;
    uint8_t* host = nullptr;
    if (residency == Q1_RESIDENCY_PINNED_HOST) {
        st = ctx->htable.alloc(p.total);
        if (st != Q1_OK) return st;
        host = ctx->htable.p;
    } else {
        ctx->hcopy.assign(p.total, 0);
        host = ctx->hcopy.data();
    }
    memset(host, 0, p.total);
    const void* srcs[7] = {c->shipdate, c->quantity, c->discount, c->tax, c->extendedprice,
                           pair ? (const void*)c->flags : (const void*)c->returnflag, c->linestatus};
    for (int k = 0; k < 7; ++k)
        if (rows && p.bytes[k]) memcpy(host + p.offset[k], srcs[k], p.bytes[k]);
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.rows = rows;
    if (pair) {
        ctx->stats.num_pair_codes = c->num_pair_codes;
        memcpy(ctx->stats.pair_group, c->pair_group, 4);
        for (uint32_t i = 0; i < c->num_pair_codes; ++i) ctx->stats.group_present_mask |= 1u << c->pair_group[i];
    }
    st = place_table(ctx, host, residency == Q1_RESIDENCY_PINNED_HOST);
    if (st != Q1_OK) {
        unload(ctx);
        return st;
    }
    ctx->hcopy_valid = residency == Q1_RESIDENCY_HBM;
    ctx->loaded = true;
    return Q1_OK;
}

q1_status q1_generate_table(q1_ctx* ctx, uint64_t seed, uint64_t first_row, uint64_t rows, q1_layout layout,
                            q1_flag_packing packing, q1_residency residency) {
    if (residency != Q1_RESIDENCY_HBM && residency != Q1_RESIDENCY_PINNED_HOST)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown residency");
    if (!ctx) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (layout == Q1_LAYOUT_UNCOMPRESSED) {
        // Host generation of reference-typed columns, then the normal load path.
        std::vector<int32_t> ship(rows);
        std::vector<int64_t> disc(rows), price(rows), tax(rows), qty(rows);
        std::vector<char> rf(rows), ls(rows);
        q1_columns c{ship.data(), disc.data(), price.data(), tax.data(), qty.data(), rf.data(), ls.data()};
        q1_status st = q1_generate_host(seed, first_row, rows, &c);
        if (st != Q1_OK) return st;
        return q1_load_columns(ctx, &c, rows, layout, packing, residency);
    }
    if (packing != Q1_FLAGS_PAIR_2BIT && packing != Q1_FLAGS_SEPARATE)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");
    if (first_row % 32) return set_error(Q1_ERR_INVALID_ARGUMENT, "first_row must be a multiple of 32");
    q1_status st = select_device(ctx);
    if (st != Q1_OK) return st;
    unload(ctx);
    ctx->rows = rows;
    ctx->layout = layout;
    ctx->packing = packing;
    ctx->residency = residency;
    ctx->plan = make_plan(rows, layout, packing, true);
    const Plan& p = ctx->plan;
    auto outputs = [&](uint8_t* d, const Plan& pl) {
        q1_compressed_host_out o{};
        o.shipdate = reinterpret_cast<uint16_t*>(d + pl.offset[0]);
        o.quantity = d + pl.offset[1];
        o.discount = d + pl.offset[2];
        o.tax = d + pl.offset[3];
        o.extendedprice = reinterpret_cast<uint32_t*>(d + pl.offset[4]);
        if (packing == Q1_FLAGS_PAIR_2BIT) o.flags = reinterpret_cast<uint32_t*>(d + pl.offset[5]);
        else {
            o.returnflag = reinterpret_cast<uint32_t*>(d + pl.offset[5]);
            o.linestatus = reinterpret_cast<uint32_t*>(d + pl.offset[6]);
        }
        return o;
    };
    if (residency == Q1_RESIDENCY_HBM) {
        st = ctx->dtable.alloc(p.total);
        if (st != Q1_OK) return st;
        Q1_CUDA(cudaMemsetAsync(ctx->dtable.p, 0, p.total, ctx->streams[0]));
        q1_compressed_host_out o = outputs(ctx->dtable.p, p);
        st = q1_generate_compressed_device(seed, first_row, rows, packing, &o, ctx->streams[0]);
        if (st != Q1_OK) return st;
        Q1_CUDA(cudaStreamSynchronize(ctx->streams[0]));
    } else {
        st = ctx->htable.alloc(p.total);
        if (st != Q1_OK) return st;
        memset(ctx->htable.p, 0, p.total);
        const uint64_t chunk = std::min<uint64_t>(rows ? rows : 1, 1ull << 26);   // multiple of 32
        const Plan cp = make_plan(chunk, layout, packing, false);
        DevBuf tmp;
        st = tmp.alloc(cp.total);
        if (st != Q1_OK) return st;
        for (uint64_t off = 0; off < rows; off += chunk) {
            const uint64_t n = std::min(chunk, rows - off);
            q1_compressed_host_out o = outputs(tmp.p, cp);
            st = q1_generate_compressed_device(seed, first_row + off, n, packing, &o, ctx->streams[0]);
            if (st != Q1_OK) return st;
            const uint64_t src_off[7] = {0, 0, 0, 0, 0, 0, 0};
            (void)src_off;
            const uint64_t dst_off[7] = {2 * off, off, off, off, 4 * off, 4 * (off / 16), 4 * (off / 32)};
            const uint64_t bytes[7] = {2 * n, n, n, n, 4 * n, 4 * words16(n),
                                       packing == Q1_FLAGS_SEPARATE ? 4 * words32(n) : 0};
            for (int c = 0; c < 7; ++c) {
                if (!bytes[c]) continue;
                Q1_CUDA(cudaMemcpyAsync(ctx->htable.p + p.offset[c] + dst_off[c], tmp.p + cp.offset[c], bytes[c],
                                        cudaMemcpyDeviceToHost, ctx->streams[0]));
            }
            Q1_CUDA(cudaStreamSynchronize(ctx->streams[0]));
        }
    }
    // Statistics known by construction of the generator.
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    ctx->stats.rows = rows;
    ctx->stats.min_shipdate = kGenOrderDateFirst + 1;
    ctx->stats.max_shipdate = kGenOrderDateLast + 121;
    ctx->stats.max_quantity = 50;
    ctx->stats.max_discount = 10;
    ctx->stats.max_tax = 8;
    ctx->stats.max_extendedprice = 50u * 209899u;
    ctx->stats.num_pair_codes = packing == Q1_FLAGS_PAIR_2BIT ? kGenPairCodes : 0;
    for (uint32_t i = 0; i < 4; ++i) ctx->stats.pair_group[i] = (uint8_t)gen_pair_group(i);
    ctx->stats.group_present_mask = (1u << 0) | (1u << 2) | (1u << 3) | (1u << 4);
    ctx->hcopy_valid = false;   // made on demand (coprocessing) from device memory
    ctx->loaded = true;
    return Q1_OK;
}

q1_status q1_table_columns(q1_ctx* ctx, q1_compressed_columns* comp, q1_columns* unc, uint64_t* rows,
                           q1_layout* layout, q1_residency* residency) {
    if (!ctx) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->loaded) return set_error(Q1_ERR_NOT_LOADED, "no table loaded");
    const uint8_t* base = ctx->residency == Q1_RESIDENCY_HBM ? ctx->dtable.p : ctx->htable.p;
    const Plan& p = ctx->plan;
    if (rows) *rows = ctx->rows;
    if (layout) *layout = ctx->layout;
    if (residency) *residency = ctx->residency;
    if (ctx->layout == Q1_LAYOUT_COMPRESSED && comp) {
        memset(comp, 0, sizeof(*comp));
        comp->shipdate = reinterpret_cast<const uint16_t*>(base + p.offset[0]);
        comp->quantity = base + p.offset[1];
        comp->discount = base + p.offset[2];
        comp->tax = base + p.offset[3];
        comp->extendedprice = reinterpret_cast<const uint32_t*>(base + p.offset[4]);
        if (ctx->packing == Q1_FLAGS_PAIR_2BIT) comp->flags = reinterpret_cast<const uint32_t*>(base + p.offset[5]);
        else {
            comp->returnflag = reinterpret_cast<const uint32_t*>(base + p.offset[5]);
            comp->linestatus = reinterpret_cast<const uint32_t*>(base + p.offset[6]);
        }
        comp->filter = reinterpret_cast<const uint32_t*>(base + p.filter_offset);
        comp->flag_packing = ctx->packing;
        comp->num_pair_codes = ctx->stats.num_pair_codes ? ctx->stats.num_pair_codes : 1;
        memcpy(comp->pair_group, ctx->stats.pair_group, 4);
    }
    if (ctx->layout == Q1_LAYOUT_UNCOMPRESSED && unc) {
        unc->shipdate = reinterpret_cast<const int32_t*>(base + p.offset[0]);
        unc->quantity = reinterpret_cast<const int64_t*>(base + p.offset[1]);
        unc->discount = reinterpret_cast<const int64_t*>(base + p.offset[2]);
        unc->tax = reinterpret_cast<const int64_t*>(base + p.offset[3]);
        unc->extendedprice = reinterpret_cast<const int64_t*>(base + p.offset[4]);
        unc->returnflag = reinterpret_cast<const char*>(base + p.offset[5]);
        unc->linestatus = reinterpret_cast<const char*>(base + p.offset[6]);
    }
    return Q1_OK;
}

q1_status q1_table_stats(q1_ctx* ctx, q1_column_stats* stats) {
    if (!ctx || !stats) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (!ctx->loaded) return set_error(Q1_ERR_NOT_LOADED, "no table loaded");
    *stats = ctx->stats;
    return Q1_OK;
}

q1_status q1_run_times(q1_ctx* ctx, double* wall_ms, double* gpu_ms, int32_t capacity, int32_t* count) {
    if (!ctx) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    const int32_t n = (int32_t)ctx->wall_ms.size();
    if (count) *count = n;
    for (int32_t i = 0; i < n && i < capacity; ++i) {
        if (wall_ms) wall_ms[i] = ctx->wall_ms[i];
        if (gpu_ms) gpu_ms[i] = ctx->gpu_ms[i];
    }
    return Q1_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Running
// ---------------------------------------------------------------------------------------------

static q1_status ensure_streams(q1_ctx* ctx, int n) {
    for (int i = ctx->nstreams; i < n; ++i) {
        Q1_CUDA(cudaStreamCreateWithFlags(&ctx->streams[i], cudaStreamNonBlocking));
        ctx->nstreams = i + 1;
    }
    for (int i = 0; i < n; ++i) {
        if (!ctx->ev_join[i]) Q1_CUDA(cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming));
    }
    return Q1_OK;
}

static q1_status ensure_pool(q1_ctx* ctx) {
    if (!ctx->pool) ctx->pool.reset(new CpuPool(ctx->cpu_threads));
    return Q1_OK;
}

// Host copy of a device-generated table for the CPU share (one-time, outside any timing).
static q1_status ensure_host_copy(q1_ctx* ctx) {
    if (ctx->residency == Q1_RESIDENCY_PINNED_HOST || ctx->hcopy_valid) return Q1_OK;
    ctx->hcopy.assign(ctx->plan.total, 0);
    Q1_CUDA(cudaMemcpy(ctx->hcopy.data(), ctx->dtable.p, ctx->plan.total, cudaMemcpyDeviceToHost));
    ctx->hcopy_valid = true;
    return Q1_OK;
}

static HostCompressed host_compressed_view(q1_ctx* ctx, const uint8_t* base) {
    const Plan& p = ctx->plan;
    HostCompressed h;
    h.ship = reinterpret_cast<const uint16_t*>(base + p.offset[0]);
    h.qty = base + p.offset[1];
    h.disc = base + p.offset[2];
    h.tax = base + p.offset[3];
    h.price = reinterpret_cast<const uint32_t*>(base + p.offset[4]);
    h.pair = ctx->packing == Q1_FLAGS_PAIR_2BIT;
    if (h.pair) h.flags = reinterpret_cast<const uint32_t*>(base + p.offset[5]);
    else {
        h.rf = reinterpret_cast<const uint32_t*>(base + p.offset[5]);
        h.ls = reinterpret_cast<const uint32_t*>(base + p.offset[6]);
    }
    memcpy(h.pair_group, ctx->stats.pair_group, 4);
    if (h.pair)
        for (uint32_t i = ctx->stats.num_pair_codes; i < 4; ++i) h.pair_group[i] = h.pair_group[0];
    return h;
}

static HostUncompressed host_uncompressed_view(q1_ctx* ctx, const uint8_t* base) {
    const Plan& p = ctx->plan;
    HostUncompressed h;
    h.ship = reinterpret_cast<const int32_t*>(base + p.offset[0]);
    h.qty = reinterpret_cast<const int64_t*>(base + p.offset[1]);
    h.disc = reinterpret_cast<const int64_t*>(base + p.offset[2]);
    h.tax = reinterpret_cast<const int64_t*>(base + p.offset[3]);
    h.price = reinterpret_cast<const int64_t*>(base + p.offset[4]);
    h.rf = reinterpret_cast<const char*>(base + p.offset[5]);
    h.ls = reinterpret_cast<const char*>(base + p.offset[6]);
    return h;
}

// Launch the scan over rows [0, n) of a column set laid out per `plan` at `base` (device).
static q1_status launch_on(q1_ctx* ctx, const q1_params* prm, const uint8_t* base, const Plan& plan, uint64_t n,
                           bool use_filter, cudaStream_t stream) {
    q1_launch_config cfg{prm->threads_per_block, prm->tuples_per_thread, 0};
    if (ctx->layout == Q1_LAYOUT_COMPRESSED) {
        q1_compressed_columns c{};
        c.shipdate = reinterpret_cast<const uint16_t*>(base + plan.offset[0]);
        c.quantity = base + plan.offset[1];
        c.discount = base + plan.offset[2];
        c.tax = base + plan.offset[3];
        c.extendedprice = reinterpret_cast<const uint32_t*>(base + plan.offset[4]);
        if (ctx->packing == Q1_FLAGS_PAIR_2BIT) c.flags = reinterpret_cast<const uint32_t*>(base + plan.offset[5]);
        else {
            c.returnflag = reinterpret_cast<const uint32_t*>(base + plan.offset[5]);
            c.linestatus = reinterpret_cast<const uint32_t*>(base + plan.offset[6]);
        }
        c.filter = reinterpret_cast<const uint32_t*>(base + plan.filter_offset);
        c.flag_packing = ctx->packing;
        c.num_pair_codes = ctx->stats.num_pair_codes ? ctx->stats.num_pair_codes : 1;
        memcpy(c.pair_group, ctx->stats.pair_group, 4);
        return q1_launch_compressed((q1_placement)prm->placement, &c, n, prm->cutoff_day, use_filter ? 1 : 0, &cfg,
                                    reinterpret_cast<q1_i128*>(ctx->daggs.p), stream);
    }
    q1_columns c{};
    c.shipdate = reinterpret_cast<const int32_t*>(base + plan.offset[0]);
    c.quantity = reinterpret_cast<const int64_t*>(base + plan.offset[1]);
    c.discount = reinterpret_cast<const int64_t*>(base + plan.offset[2]);
    c.tax = reinterpret_cast<const int64_t*>(base + plan.offset[3]);
    c.extendedprice = reinterpret_cast<const int64_t*>(base + plan.offset[4]);
    c.returnflag = reinterpret_cast<const char*>(base + plan.offset[5]);
    c.linestatus = reinterpret_cast<const char*>(base + plan.offset[6]);
    return q1_launch_uncompressed((q1_placement)prm->placement, &c, n, prm->cutoff_day, &cfg,
                                  reinterpret_cast<q1_i128*>(ctx->daggs.p), stream);
}

// Copy rows [off, off+n) of every column from the pinned table into a chunk buffer.
static q1_status copy_chunk(q1_ctx* ctx, uint8_t* dst, uint64_t off, uint64_t n, bool with_filter, bool skip_ship,
                            cudaStream_t stream) {
    const Plan& p = ctx->plan;
    const Plan& cp = ctx->chunk_plan;
    const uint8_t* src = ctx->htable.p;
    auto copy = [&](int c, uint64_t src_off, uint64_t bytes) -> q1_status {
        if (!bytes) return Q1_OK;
        Q1_CUDA(cudaMemcpyAsync(dst + cp.offset[c], src + p.offset[c] + src_off, bytes, cudaMemcpyHostToDevice, stream));
        return Q1_OK;
    };
    q1_status st;
    if (ctx->layout == Q1_LAYOUT_COMPRESSED) {
        if (!skip_ship && (st = copy(0, 2 * off, 2 * n)) != Q1_OK) return st;
        if ((st = copy(1, off, n)) != Q1_OK) return st;
        if ((st = copy(2, off, n)) != Q1_OK) return st;
        if ((st = copy(3, off, n)) != Q1_OK) return st;
        if ((st = copy(4, 4 * off, 4 * n)) != Q1_OK) return st;
        if ((st = copy(5, 4 * (off / 16), 4 * words16(n))) != Q1_OK) return st;
        if (ctx->packing == Q1_FLAGS_SEPARATE && (st = copy(6, 4 * (off / 32), 4 * words32(n))) != Q1_OK) return st;
        if (with_filter) {
            Q1_CUDA(cudaMemcpyAsync(dst + cp.filter_offset, src + p.filter_offset + 4 * (off / 32), 4 * words32(n),
                                    cudaMemcpyHostToDevice, stream));
        }
    } else {
        if ((st = copy(0, 4 * off, 4 * n)) != Q1_OK) return st;
        for (int c = 1; c <= 4; ++c)
            if ((st = copy(c, 8 * off, 8 * n)) != Q1_OK) return st;
        if ((st = copy(5, off, n)) != Q1_OK) return st;
        if ((st = copy(6, off, n)) != Q1_OK) return st;
    }
    return Q1_OK;
}

static q1_status run_once(q1_ctx* ctx, const q1_params* prm, Agg128* total, double* gpu_ms, uint64_t* rows_gpu,
                          uint64_t* rows_cpu) {
    const uint64_t N = ctx->rows;
    const bool streamed = ctx->residency == Q1_RESIDENCY_PINNED_HOST;
    const bool pushdown = prm->use_filter_pushdown != 0;
    const bool coproc = prm->use_coprocessing != 0;
    cudaStream_t s0 = ctx->streams[0];
    const int32_t cutoff_rel = (int32_t)std::max<int64_t>(-1, std::min<int64_t>(32767, (int64_t)prm->cutoff_day - kShipDateFrame));

    // CPU/GPU split (src/main.cu:517-550): the CPU share starts at a chunk boundary.
    uint64_t cpu_start = N;
    if (coproc) {
        cpu_start = N - (uint64_t)((double)N * prm->cpu_fraction);
        const uint64_t unit = streamed ? (uint64_t)prm->tuples_per_launch : (uint64_t)scan_tile_rows(kLayPair, kPlaceInRegistersPerThread);
        cpu_start -= cpu_start % unit;
    }
    const uint64_t gpu_end = cpu_start;
    *rows_gpu = gpu_end;
    *rows_cpu = N - cpu_start;

    Q1_CUDA(cudaMemsetAsync(ctx->daggs.p, 0, ctx->daggs.n, s0));
    Q1_CUDA(cudaEventRecord(ctx->ev_start, s0));

    // ---- CPU side: the coprocessing share and/or the filter producer -----------------------
    const bool cpu_job = coproc || (pushdown && streamed);
    std::vector<Agg128> cpu_parts;
    std::atomic<uint64_t> cursor{0};
    std::atomic<int> cpu_domain_bad{0};
    const uint64_t morsel = streamed ? (uint64_t)prm->tuples_per_launch : (uint64_t)(1u << 21);
    if (cpu_job) {
        ensure_pool(ctx);
        q1_status st = ensure_host_copy(ctx);
        if (st != Q1_OK) return st;
        uint8_t* hb = ctx->host_base();
        cpu_parts.assign(ctx->pool->threads(), Agg128{});
        for (auto& a : cpu_parts) a.clear();
        ctx->queue.reset();
        // Morsels below cpu_start only produce filter chunks (streamed pushdown); morsels at or
        // above cpu_start are aggregated (cpu/kernel_x100.hpp:456-483).
        const uint64_t filter_end = (pushdown && streamed) ? gpu_end : 0;
        const uint64_t first = filter_end ? 0 : cpu_start;
        cursor.store(first);
        const bool comp = ctx->layout == Q1_LAYOUT_COMPRESSED;
        HostCompressed hc;
        HostUncompressed hu;
        if (comp) hc = host_compressed_view(ctx, hb);
        else hu = host_uncompressed_view(ctx, hb);
        uint32_t* hfilter = reinterpret_cast<uint32_t*>(hb + ctx->plan.filter_offset);
        const int32_t cut_day = prm->cutoff_day;
        ctx->pool->start([&, hc, hu, hfilter, filter_end, first, comp, cut_day](int id) {
            for (;;) {
                uint64_t off = cursor.fetch_add(morsel);
                if (off >= N) break;
                if (off < filter_end) {
                    const uint64_t n = std::min(morsel, filter_end - off);
                    cpu_precompute_filter(hc.ship, off, off + n, cutoff_rel, hfilter);
                    ctx->queue.push(FilterChunk{off, n});
                    continue;
                }
                if (off < cpu_start) continue;   // (only when filter_end < cpu_start, never)
                const uint64_t n = std::min(morsel, N - off);
                bool ok = comp ? cpu_aggregate_compressed(hc, off, off + n, cutoff_rel, &cpu_parts[id])
                               : cpu_aggregate_uncompressed(hu, off, off + n, cut_day, &cpu_parts[id]);
                if (!ok) cpu_domain_bad.store(1);
            }
        });
    }

    // ---- GPU side ------------------------------------------------------------------------
    q1_status st = Q1_OK;
    if (!streamed) {
        const uint8_t* base = ctx->dtable.p;
        if (pushdown && gpu_end) {
            st = q1_precompute_filter(reinterpret_cast<const uint16_t*>(base + ctx->plan.offset[0]), gpu_end,
                                      prm->cutoff_day, reinterpret_cast<uint32_t*>(ctx->dtable.p + ctx->plan.filter_offset),
                                      s0);
        }
        if (st == Q1_OK) st = launch_on(ctx, prm, base, ctx->plan, gpu_end, pushdown, s0);
    } else {
        const int ns = prm->streams;
        st = ensure_streams(ctx, ns);
        const uint64_t chunk = (uint64_t)prm->tuples_per_launch;
        if (st == Q1_OK && (ctx->chunk_rows != chunk || ctx->chunk_streams != ns || !ctx->dchunks.p)) {
            ctx->chunk_plan = make_plan(chunk, ctx->layout, ctx->packing, true);
            st = ctx->dchunks.alloc(ctx->chunk_plan.total * ns);
            if (st == Q1_OK) {
                ctx->chunk_rows = chunk;
                ctx->chunk_streams = ns;
            }
        }
        if (st == Q1_OK) {
            cudaError_t e = cudaEventRecord(ctx->ev_zeroed, s0);
            for (int i = 1; i < ns && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(ctx->streams[i], ctx->ev_zeroed, 0);
            if (e != cudaSuccess) st = cuda_error(e, "stream fan-out");
        }
        const uint64_t nchunks = (gpu_end + chunk - 1) / chunk;
        for (uint64_t k = 0; k < nchunks && st == Q1_OK; ++k) {
            const int si = (int)(k % ns);
            cudaStream_t s = ctx->streams[si];
            uint64_t off = k * chunk, n = std::min(chunk, gpu_end - off);
            if (pushdown) {
                FilterChunk fc;
                bool got = false;
                for (int waited = 0; waited < 120000 && !(got = ctx->queue.pop(&fc, 50)); waited += 50)
                    if (ctx->pool->failed()) break;   // a producer died: no chunk will come
                if (!got) {
                    st = set_error(Q1_ERR_CPU_WORKER, ctx->pool->failed()
                                                          ? "CPU worker failed: " + ctx->pool->error()
                                                          : std::string("filter producer delivered no chunk within 120 s"));
                    break;
                }
                off = fc.offset;
                n = fc.num;
            }
            uint8_t* dst = ctx->dchunks.p + (uint64_t)si * ctx->chunk_plan.total;
            st = copy_chunk(ctx, dst, off, n, pushdown, pushdown, s);
            if (st == Q1_OK) st = launch_on(ctx, prm, dst, ctx->chunk_plan, n, pushdown, s);
        }
        for (int i = 1; i < ns && st == Q1_OK; ++i) {
            cudaError_t e = cudaEventRecord(ctx->ev_join[i], ctx->streams[i]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s0, ctx->ev_join[i], 0);
            if (e != cudaSuccess) st = cuda_error(e, "stream join");
        }
    }
    if (st == Q1_OK) {
        cudaError_t e = cudaEventRecord(ctx->ev_stop, s0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->haggs.p, ctx->daggs.p, ctx->daggs.n, cudaMemcpyDeviceToHost, s0);
        if (e != cudaSuccess) st = cuda_error(e, "aggregate read-back");
    }
    q1_status dev_st = q1_sync_check(s0);
    if (st == Q1_OK) st = dev_st;
    if (cpu_job) {
        ctx->queue.close();
        if (!ctx->pool->wait() && st == Q1_OK) st = set_error(Q1_ERR_CPU_WORKER, "CPU worker failed: " + ctx->pool->error());
        if (cpu_domain_bad.load() && st == Q1_OK)
            st = set_error(Q1_ERR_DOMAIN, "a row of the CPU share is outside the kernels' domain (compressed) or "
                                          "its int64 products overflow (reference-typed)");
    }
    if (st != Q1_OK) {
        // leave every stream idle before reporting
        for (int i = 0; i < ctx->nstreams; ++i) cudaStreamSynchronize(ctx->streams[i]);
        return st;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    *gpu_ms = ms;
    agg_from_device_words(reinterpret_cast<const unsigned long long*>(ctx->haggs.p), total);
    for (auto& a : cpu_parts) total->add(a);   // exact 128-bit merge of the CPU share
    return Q1_OK;
}

extern "C" q1_status q1_run(q1_ctx* ctx, const q1_params* prm, q1_result* out) {
    if (!ctx || !prm) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    q1_status st = q1_params_validate(prm);
    if (st != Q1_OK) return st;
    if (!ctx->loaded) return set_error(Q1_ERR_NOT_LOADED, "no table loaded (q1_load_columns)");
    if ((prm->apply_compression != 0) != (ctx->layout == Q1_LAYOUT_COMPRESSED))
        return set_error(Q1_ERR_INVALID_ARGUMENT, prm->apply_compression
                                                      ? "apply_compression set but the loaded table is uncompressed"
                                                      : "the loaded table is compressed; set apply_compression");
    st = select_device(ctx);
    if (st != Q1_OK) return st;
    ctx->wall_ms.clear();
    ctx->gpu_ms.clear();
    Agg128 agg;
    uint64_t rg = 0, rc = 0;
    for (int run = 0; run < prm->runs; ++run) {
        const auto t0 = std::chrono::steady_clock::now();
        agg.clear();
        double gms = 0;
        st = run_once(ctx, prm, &agg, &gms, &rg, &rc);
        if (st != Q1_OK) return st;
        const auto t1 = std::chrono::steady_clock::now();
        ctx->wall_ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        ctx->gpu_ms.push_back(gms);
    }
    if (out) {
        memset(out, 0, sizeof(*out));
        q1_i128 flat[36];
        agg_to_i128(agg, flat);
        out->num_groups = Q1_NUM_POTENTIAL_GROUPS;
        q1_finalize_groups(flat, Q1_NUM_POTENTIAL_GROUPS, out->groups);
        out->rows_total = ctx->rows;
        out->rows_gpu = rg;
        out->rows_cpu = rc;
        out->ms_last_run = ctx->wall_ms.back();
        out->ms_gpu_last_run = ctx->gpu_ms.back();
    }
    return Q1_OK;
}
