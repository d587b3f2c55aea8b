// C ABI: errors, names, compressor, filter precomputation, result finalisation, the
// kernel-level launch entry points and the generators.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "q1.h"
#include "q1_common.cuh"
#include "q1_internal.h"
#include "q1_kernels.h"

namespace q1 {

static thread_local std::string t_error;

q1_status set_error(q1_status s, const std::string& msg) {
    t_error = msg;
    return s;
}

q1_status cuda_error(cudaError_t e, const char* what) {
    return set_error(e == cudaErrorMemoryAllocation ? Q1_ERR_OUT_OF_MEMORY : Q1_ERR_CUDA,
                     std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

uint64_t words16(uint64_t rows) { return (rows + 15) / 16; }
uint64_t words32(uint64_t rows) { return (rows + 31) / 32; }

void Agg128::clear() { memset(v, 0, sizeof(v)); }
void Agg128::add(const Agg128& o) {
    for (int g = 0; g < 6; ++g)
        for (int k = 0; k < 6; ++k) v[g][k] += o.v[g][k];
}
void agg_from_device_words(const unsigned long long* w, Agg128* out) {
    for (int g = 0; g < 6; ++g)
        for (int k = 0; k < 6; ++k) out->v[g][k] = ((u128)w[2 * (g * 6 + k) + 1] << 64) | (u128)w[2 * (g * 6 + k)];
}
void agg_to_i128(const Agg128& a, q1_i128* out) {
    for (int g = 0; g < 6; ++g)
        for (int k = 0; k < 6; ++k) {
            out[g * 6 + k].lo = (uint64_t)a.v[g][k];
            out[g * 6 + k].hi = (uint64_t)(a.v[g][k] >> 64);
        }
}

static std::mutex g_dev_mutex;
static DeviceInfo g_devices[64];

q1_status device_info(int device, DeviceInfo** out) {
    if (device < 0 || device >= 64) return set_error(Q1_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_dev_mutex);
    DeviceInfo& d = g_devices[device];
    if (!d.sm_count) {
        int sms = 0;
        Q1_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        int cur = 0;
        Q1_CUDA(cudaGetDevice(&cur));
        if (cur != device) Q1_CUDA(cudaSetDevice(device));
        uint32_t* st = nullptr;
        cudaError_t e = cudaMalloc(&st, 256);
        if (e == cudaSuccess) e = cudaMemset(st, 0, 256);
        if (cur != device) cudaSetDevice(cur);
        if (e != cudaSuccess) return cuda_error(e, "allocating the device status word");
        d.status = st;
        d.sm_count = sms;
    }
    *out = &d;
    return Q1_OK;
}

q1_status check_device_status(cudaStream_t stream, uint32_t* status_word) {
    Q1_CUDA(cudaStreamSynchronize(stream));
    if (!status_word) return Q1_OK;
    uint32_t bits = 0;
    Q1_CUDA(cudaMemcpy(&bits, status_word, sizeof(bits), cudaMemcpyDeviceToHost));
    if (bits) {
        Q1_CUDA(cudaMemset(status_word, 0, sizeof(bits)));
        if (bits & 1u) return set_error(Q1_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
        if (bits & 4u) return set_error(Q1_ERR_INTERNAL, "a device work buffer would have overflowed");
        return set_error(Q1_ERR_DOMAIN, "a row is outside the kernels' domain: a compressed row with a discount "
                                        "above 100 or a ship offset above 32767, or a reference-typed row whose "
                                        "int64 products overflow");
    }
    return Q1_OK;
}

}  // namespace q1

using namespace q1;

// =============================================================================================
// extern "C"
// =============================================================================================

extern "C" {

const char* q1_last_error(void) { return t_error.c_str(); }

const char* q1_status_string(q1_status s) {
    switch (s) {
        case Q1_OK: return "Q1_OK";
        case Q1_ERR_INVALID_ARGUMENT: return "Q1_ERR_INVALID_ARGUMENT";
        case Q1_ERR_CUDA: return "Q1_ERR_CUDA";
        case Q1_ERR_OUT_OF_MEMORY: return "Q1_ERR_OUT_OF_MEMORY";
        case Q1_ERR_NOT_LOADED: return "Q1_ERR_NOT_LOADED";
        case Q1_ERR_UNSUPPORTED: return "Q1_ERR_UNSUPPORTED";
        case Q1_ERR_DOMAIN: return "Q1_ERR_DOMAIN";
        case Q1_ERR_DEVICE_TIMEOUT: return "Q1_ERR_DEVICE_TIMEOUT";
        case Q1_ERR_BUSY: return "Q1_ERR_BUSY";
        case Q1_ERR_CPU_WORKER: return "Q1_ERR_CPU_WORKER";
        case Q1_ERR_INTERNAL: return "Q1_ERR_INTERNAL";
    }
    return "Q1_ERR_UNKNOWN";
}

const char* q1_version(void) { return "q1-b200 1.0 (sm_100a)"; }

q1_status q1_measure_host_read(const void* host_buf, uint64_t bytes, int32_t threads, double* gb_per_s) {
    if (!host_buf || !gb_per_s) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (bytes < 4096 || threads < 1 || threads > 1024)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "bytes must be >= 4096 and threads 1..1024");
    *gb_per_s = host_read_gbs(host_buf, bytes, threads);
    return Q1_OK;
}

q1_status q1_device_describe(int32_t device, char* buf, size_t buf_len) {
    if (!buf || !buf_len) return set_error(Q1_ERR_INVALID_ARGUMENT, "null buffer");
    cudaDeviceProp p;
    Q1_CUDA(cudaGetDeviceProperties(&p, device));
    snprintf(buf, buf_len, "Device %d: %s, compute capability %d.%d, %d SMs, %.1f GiB, L2 %d MiB, %d KiB smem/block opt-in",
             device, p.name, p.major, p.minor, p.multiProcessorCount, p.totalGlobalMem / 1073741824.0,
             p.l2CacheSize >> 20, (int)(p.sharedMemPerBlockOptin >> 10));
    return Q1_OK;
}

static const char* kPlacementNames[Q1_NUM_PLACEMENTS] = {"in_registers", "in_registers_per_thread", "local_mem",
                                                           "shared_mem_per_thread", "global"};

q1_status q1_placement_from_name(const char* name, q1_placement* out) {
    if (!name || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    std::string n(name);
    std::replace(n.begin(), n.end(), '-', '_');
    if (n == "per_thread_shared_mem") n = "shared_mem_per_thread";   // README spelling
    if (n == "in_registers_per_thread_shared_mem") n = "shared_mem_per_thread";
    for (int i = 0; i < Q1_NUM_PLACEMENTS; ++i) {
        if (n == kPlacementNames[i]) {
            *out = (q1_placement)i;
            return Q1_OK;
        }
    }
    return set_error(Q1_ERR_INVALID_ARGUMENT, std::string("No kernel variant named \"") + name + "\" is available");
}

const char* q1_placement_name(q1_placement p) {
    if ((int)p < 0 || (int)p >= Q1_NUM_PLACEMENTS) return "unknown";
    return kPlacementNames[p];
}

// ---------------------------------------------------------------------------------------------
// Compressor (src/main.cu:773-803), multi-threaded over blocks of 4096 rows.
// ---------------------------------------------------------------------------------------------

q1_status q1_compress_host(const q1_columns* in, uint64_t rows, q1_flag_packing packing,
                           const q1_compressed_host_out* out, q1_column_stats* stats) {
    if (!in || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (rows && (!in->shipdate || !in->discount || !in->extendedprice || !in->tax || !in->quantity ||
                 !in->returnflag || !in->linestatus))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing input column");
    if (rows && (!out->shipdate || !out->discount || !out->extendedprice || !out->tax || !out->quantity))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output column");
    if (packing == Q1_FLAGS_PAIR_2BIT && rows && !out->flags)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output flags column");
    if (packing == Q1_FLAGS_SEPARATE && rows && (!out->returnflag || !out->linestatus))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output returnflag/linestatus columns");
    if (packing != Q1_FLAGS_PAIR_2BIT && packing != Q1_FLAGS_SEPARATE)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");

    constexpr uint64_t kBlock = 4096;   // multiple of 32: every container word has one writer
    const uint64_t nblocks = (rows + kBlock - 1) / kBlock;
    unsigned nthreads = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
    if (nblocks < 8 * (uint64_t)nthreads) nthreads = std::max<uint64_t>(1, nblocks / 8);

    struct Local {
        int32_t min_ship = INT32_MAX, max_ship = INT32_MIN;
        uint32_t max_q = 0, max_d = 0, max_t = 0, max_p = 0, present = 0;
        uint64_t bad_row = UINT64_MAX;
        const char* why = nullptr;
    };
    std::vector<Local> loc(nthreads);

    // Pass 1: validate, fill the byte columns, find the (rf, ls) combinations present.
    auto pass1 = [&](unsigned tid) {
        Local& L = loc[tid];
        for (uint64_t b = tid; b < nblocks; b += nthreads) {
            const uint64_t r0 = b * kBlock, r1 = std::min(rows, r0 + kBlock);
            for (uint64_t i = r0; i < r1; ++i) {
                const int64_t s = (int64_t)in->shipdate[i] - kShipDateFrame;
                const int64_t d = in->discount[i], x = in->tax[i], p = in->extendedprice[i], q = in->quantity[i];
                const char rf = in->returnflag[i], ls = in->linestatus[i];
                const char* why = nullptr;
                if (s < 0 || s > 32767) why = "shipdate outside [1992-01-01, 1992-01-01 + 32767 days]";
                else if (d < 0 || d > 100) why = "discount outside [0, 1.00]";
                else if (x < 0 || x > 255) why = "tax outside [0, 2.55]";
                else if (p < 0 || p > 0xFFFFFFFFll) why = "extendedprice outside uint32 cents";
                else if (q < 0 || q % 100 != 0 || q / 100 > 255) why = "quantity not a whole number of units in [0, 255]";
                else if (rf != 'A' && rf != 'N' && rf != 'R') why = "returnflag not one of A, N, R";
                else if (ls != 'F' && ls != 'O') why = "linestatus not one of F, O";
                if (why) {
                    if (i < L.bad_row) {
                        L.bad_row = i;
                        L.why = why;
                    }
                    continue;
                }
                out->shipdate[i] = (uint16_t)s;
                out->discount[i] = (uint8_t)d;
                out->tax[i] = (uint8_t)x;
                out->extendedprice[i] = (uint32_t)p;
                out->quantity[i] = (uint8_t)(q / 100);
                L.min_ship = std::min<int32_t>(L.min_ship, in->shipdate[i]);
                L.max_ship = std::max<int32_t>(L.max_ship, in->shipdate[i]);
                L.max_q = std::max<uint32_t>(L.max_q, (uint32_t)(q / 100));
                L.max_d = std::max<uint32_t>(L.max_d, (uint32_t)d);
                L.max_t = std::max<uint32_t>(L.max_t, (uint32_t)x);
                L.max_p = std::max<uint32_t>(L.max_p, (uint32_t)p);
                L.present |= 1u << group_of(encode_return_flag(rf), encode_line_status(ls));
            }
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nthreads; ++t) th.emplace_back(pass1, t);
    pass1(0);
    for (auto& t : th) t.join();
    th.clear();

    Local all;
    for (auto& L : loc) {
        all.min_ship = std::min(all.min_ship, L.min_ship);
        all.max_ship = std::max(all.max_ship, L.max_ship);
        all.max_q = std::max(all.max_q, L.max_q);
        all.max_d = std::max(all.max_d, L.max_d);
        all.max_t = std::max(all.max_t, L.max_t);
        all.max_p = std::max(all.max_p, L.max_p);
        all.present |= L.present;
        if (L.bad_row < all.bad_row) {
            all.bad_row = L.bad_row;
            all.why = L.why;
        }
    }
    if (all.why)
        return set_error(Q1_ERR_DOMAIN, "row " + std::to_string(all.bad_row) + ": " + all.why);

    // Pair dictionary: the groups present, ascending.
    uint8_t code_of[6] = {0, 0, 0, 0, 0, 0};
    uint8_t dict[4] = {0, 0, 0, 0};
    uint32_t ncodes = 0;
    for (uint32_t g = 0; g < 6; ++g) {
        if (all.present >> g & 1u) {
            if (ncodes < 4) dict[ncodes] = (uint8_t)g;
            code_of[g] = (uint8_t)ncodes;
            ++ncodes;
        }
    }
    if (packing == Q1_FLAGS_PAIR_2BIT && ncodes > 4)
        return set_error(Q1_ERR_DOMAIN, "more than 4 (returnflag, linestatus) combinations: use Q1_FLAGS_SEPARATE");
    if (ncodes == 0) ncodes = 1;   // empty or filtered-out table: a one-entry dictionary

    // Pass 2: bit containers (src/bit_operations.hpp:60-154, LSB first).
    auto pass2 = [&](unsigned tid) {
        for (uint64_t b = tid; b < nblocks; b += nthreads) {
            const uint64_t r0 = b * kBlock, r1 = std::min(rows, r0 + kBlock);
            for (uint64_t w0 = r0; w0 < r1; w0 += 16) {
                uint32_t pw = 0, rw = 0;
                for (uint64_t i = w0; i < std::min(r1, w0 + 16); ++i) {
                    const uint32_t rf = encode_return_flag(in->returnflag[i]);
                    const uint32_t ls = encode_line_status(in->linestatus[i]);
                    pw |= (uint32_t)code_of[group_of(rf, ls)] << (2 * (i - w0));
                    rw |= rf << (2 * (i - w0));
                }
                if (packing == Q1_FLAGS_PAIR_2BIT) out->flags[w0 / 16] = pw;
                else out->returnflag[w0 / 16] = rw;
            }
            if (packing == Q1_FLAGS_SEPARATE) {
                for (uint64_t w0 = r0; w0 < r1; w0 += 32) {
                    uint32_t lw = 0;
                    for (uint64_t i = w0; i < std::min(r1, w0 + 32); ++i)
                        lw |= encode_line_status(in->linestatus[i]) << (i - w0);
                    out->linestatus[w0 / 32] = lw;
                }
            }
        }
    };
    for (unsigned t = 1; t < nthreads; ++t) th.emplace_back(pass2, t);
    pass2(0);
    for (auto& t : th) t.join();

    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->rows = rows;
        stats->min_shipdate = rows ? all.min_ship : 0;
        stats->max_shipdate = rows ? all.max_ship : 0;
        stats->max_quantity = all.max_q;
        stats->max_discount = all.max_d;
        stats->max_tax = all.max_t;
        stats->max_extendedprice = all.max_p;
        stats->num_pair_codes = packing == Q1_FLAGS_PAIR_2BIT ? ncodes : 0;
        memcpy(stats->pair_group, dict, 4);
        stats->group_present_mask = all.present;
    }
    return Q1_OK;
}

q1_status q1_precompute_filter_host(const uint16_t* shipdate, uint64_t rows, int32_t cutoff_day, uint32_t* bitmap) {
    if (rows && (!shipdate || !bitmap)) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    cpu_precompute_filter(shipdate, 0, rows, cutoff_day - kShipDateFrame, bitmap);
    return Q1_OK;
}

// ---------------------------------------------------------------------------------------------
// Results
// ---------------------------------------------------------------------------------------------

static int64_t avg_e4(u128 sum_u, uint64_t count) {
    if (!count) return 0;
    const i128 sum = (i128)sum_u;
    const i128 q = (sum * 100) / (i128)count;   // C division: truncation toward zero
    if (q > (i128)INT64_MAX) return INT64_MAX;
    if (q < (i128)INT64_MIN) return INT64_MIN;
    return (int64_t)q;
}

q1_status q1_finalize_groups(const q1_i128* aggregates, uint32_t num_groups, q1_group_result* out) {
    if (!aggregates || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    for (uint32_t g = 0; g < num_groups; ++g) {
        const q1_i128* a = aggregates + (size_t)g * Q1_NUM_AGGREGATES;
        q1_group_result& r = out[g];
        memset(&r, 0, sizeof(r));
        r.group = (int32_t)g;
        r.returnflag = g < 6 ? decode_return_flag(g >> 1) : '?';
        r.linestatus = g < 6 ? decode_line_status(g & 1) : '?';
        r.count = a[Q1_AGG_COUNT].lo;
        r.sum_qty = a[Q1_AGG_SUM_QTY];
        r.sum_base_price = a[Q1_AGG_SUM_BASE_PRICE];
        r.sum_disc = a[Q1_AGG_SUM_DISC];
        r.sum_disc_price = a[Q1_AGG_SUM_DISC_PRICE];
        r.sum_charge = a[Q1_AGG_SUM_CHARGE];
        auto u = [](const q1_i128& x) { return ((u128)x.hi << 64) | x.lo; };
        r.avg_qty_e4 = avg_e4(u(r.sum_qty), r.count);
        r.avg_price_e4 = avg_e4(u(r.sum_base_price), r.count);
        r.avg_disc_e4 = avg_e4(u(r.sum_disc), r.count);
    }
    return Q1_OK;
}

// ---------------------------------------------------------------------------------------------
// Kernel-level ABI
// ---------------------------------------------------------------------------------------------

static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

static q1_status scan_launch(int layout, q1_placement placement, const uint8_t* const cols[7], int ncols,
                             uint64_t rows, int32_t cutoff, uint32_t qty_scale, const uint8_t pair_group[4],
                             const q1_launch_config* cfg, q1_i128* dev_aggregates, cudaStream_t stream) {
    if ((int)placement < 0 || (int)placement >= Q1_NUM_PLACEMENTS)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown placement");
    if (!dev_aggregates) return set_error(Q1_ERR_INVALID_ARGUMENT, "null aggregate buffer");
    if (!aligned16(dev_aggregates)) return set_error(Q1_ERR_INVALID_ARGUMENT, "aggregate buffer must be 16-byte aligned");
    for (int c = 0; c < ncols; ++c) {
        if (!cols[c] && rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
        if (!aligned16(cols[c]))
            return set_error(Q1_ERR_INVALID_ARGUMENT, "device columns must start on a 16-byte boundary");
    }
    if (rows == 0) return Q1_OK;
    int dev = 0;
    Q1_CUDA(cudaGetDevice(&dev));
    DeviceInfo* di = nullptr;
    q1_status st = device_info(dev, &di);
    if (st != Q1_OK) return st;

    int max_blocks = 0;
    if (cfg) {
        if (cfg->threads_per_block < 0 || cfg->threads_per_block % 32 != 0)
            return set_error(Q1_ERR_INVALID_ARGUMENT,
                             "All kernels only support numbers of threads per grid block which are multiples of the warp size (32)");
        if (cfg->blocks > 0) max_blocks = cfg->blocks;
        else if (cfg->threads_per_block > 0 && cfg->tuples_per_thread > 0) {
            const uint64_t per_block = (uint64_t)cfg->threads_per_block * (uint64_t)cfg->tuples_per_thread;
            max_blocks = (int)std::min<uint64_t>((rows + per_block - 1) / per_block, (uint64_t)di->sm_count);
        }
    }

    // Launch size bound that keeps every per-thread partial exact (scan_max_rows_per_launch).
    const uint64_t kMaxRows =
        scan_max_rows_per_launch(layout, placement, scan_grid_blocks(layout, placement, rows, di->sm_count, max_blocks));
    for (uint64_t off = 0; off < rows; off += kMaxRows) {
        const uint64_t n = std::min(kMaxRows, rows - off);
        ScanParams prm{};
        for (int c = 0; c < ncols; ++c) {
            // byte offset of row `off` in column c (kMaxRows is a multiple of every packing)
            uint64_t bits = 0;
            switch (layout) {
                case kLayUncomp: {
                    static const int b[7] = {32, 64, 64, 64, 64, 8, 8};
                    bits = b[c];
                    break;
                }
                default: {
                    static const int b[7] = {16, 8, 8, 8, 32, 2, 1};
                    bits = b[c];
                    if (c == 0 && (layout == kLayPairFilter || layout == kLaySepFilter)) bits = 1;
                    break;
                }
            }
            prm.col[c] = cols[c] + off * bits / 8;
        }
        prm.rows = n;
        prm.cutoff = cutoff;
        prm.qty_scale = qty_scale;
        if (pair_group) memcpy(prm.pair_group, pair_group, 4);
        prm.out = reinterpret_cast<unsigned long long*>(dev_aggregates);
        prm.status = di->status;
        cudaError_t e = launch_scan(layout, placement, prm, di->sm_count, max_blocks, stream);
        if (e != cudaSuccess) return cuda_error(e, "scan kernel launch");
    }
    return Q1_OK;
}

// Cutoff relative to 1992-01-01, clamped to [-1, 32767]: compressed ship offsets are at most
// 32767, so -1 lets no row pass and 32767 lets every row pass.
static int32_t clamp_rel(int32_t cutoff_day) {
    const int64_t r = (int64_t)cutoff_day - kShipDateFrame;
    if (r < -1) return -1;
    if (r > 32767) return 32767;
    return (int32_t)r;
}

q1_status q1_launch_compressed(q1_placement placement, const q1_compressed_columns* c, uint64_t rows,
                               int32_t cutoff_day, int32_t use_filter, const q1_launch_config* cfg,
                               q1_i128* dev_aggregates, void* cuda_stream) {
    if (!c) return set_error(Q1_ERR_INVALID_ARGUMENT, "null columns");
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
    const uint8_t* cols[7] = {
        reinterpret_cast<const uint8_t*>(use_filter ? (const void*)c->filter : (const void*)c->shipdate),
        c->quantity, c->discount, c->tax, reinterpret_cast<const uint8_t*>(c->extendedprice),
        reinterpret_cast<const uint8_t*>(pair ? c->flags : c->returnflag),
        reinterpret_cast<const uint8_t*>(c->linestatus)};
    const int layout = pair ? (use_filter ? kLayPairFilter : kLayPair) : (use_filter ? kLaySepFilter : kLaySep);
    return scan_launch(layout, placement, cols, pair ? 6 : 7, rows, clamp_rel(cutoff_day), 100u, pg, cfg,
                       dev_aggregates, (cudaStream_t)cuda_stream);
}

q1_status q1_launch_uncompressed(q1_placement placement, const q1_columns* c, uint64_t rows, int32_t cutoff_day,
                                 const q1_launch_config* cfg, q1_i128* dev_aggregates, void* cuda_stream) {
    if (!c) return set_error(Q1_ERR_INVALID_ARGUMENT, "null columns");
    const uint8_t* cols[7] = {reinterpret_cast<const uint8_t*>(c->shipdate), reinterpret_cast<const uint8_t*>(c->quantity),
                              reinterpret_cast<const uint8_t*>(c->discount), reinterpret_cast<const uint8_t*>(c->tax),
                              reinterpret_cast<const uint8_t*>(c->extendedprice),
                              reinterpret_cast<const uint8_t*>(c->returnflag),
                              reinterpret_cast<const uint8_t*>(c->linestatus)};
    return scan_launch(kLayUncomp, placement, cols, 7, rows, cutoff_day, 1u, nullptr, cfg, dev_aggregates,
                       (cudaStream_t)cuda_stream);
}

q1_status q1_precompute_filter(const uint16_t* dev_shipdate, uint64_t rows, int32_t cutoff_day, uint32_t* dev_bitmap,
                               void* cuda_stream) {
    if (rows == 0) return Q1_OK;
    if (!dev_shipdate || !dev_bitmap) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (!aligned16(dev_shipdate)) return set_error(Q1_ERR_INVALID_ARGUMENT, "shipdate must be 16-byte aligned");
    cudaError_t e = launch_precompute_filter(dev_shipdate, rows, clamp_rel(cutoff_day), dev_bitmap, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return cuda_error(e, "filter kernel launch");
    return Q1_OK;
}

// ---------------------------------------------------------------------------------------------
// Group-key aggregation
// ---------------------------------------------------------------------------------------------

uint64_t q1_groupkey_scratch_bytes(uint32_t num_groups) { return groupkey_scratch_bytes(num_groups); }

q1_status q1_launch_groupkey(q1_placement placement, const q1_compressed_columns* c, const uint32_t* dev_keys,
                             uint32_t num_groups, uint64_t rows, int32_t cutoff_day, const q1_launch_config* cfg,
                             void* dev_scratch, q1_i128* dev_aggregates, void* cuda_stream) {
    if (!c || !dev_aggregates || !dev_scratch) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (num_groups < 1 || num_groups > Q1_MAX_KEY_GROUPS)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "num_groups must be 1..65536");
    if (placement == Q1_PLACEMENT_IN_REGISTERS_PER_THREAD && num_groups > 8)
        return set_error(Q1_ERR_UNSUPPORTED, "in_registers_per_thread holds at most 8 groups per thread; use "
                                             "shared_mem_per_thread or global");
    if (placement != Q1_PLACEMENT_IN_REGISTERS_PER_THREAD && placement != Q1_PLACEMENT_SHARED_MEM_PER_THREAD &&
        placement != Q1_PLACEMENT_GLOBAL)
        return set_error(Q1_ERR_UNSUPPORTED, "group-key aggregation offers in_registers_per_thread, "
                                             "shared_mem_per_thread and global placements");
    const uint8_t* cols[6] = {reinterpret_cast<const uint8_t*>(c->shipdate), c->quantity, c->discount, c->tax,
                              reinterpret_cast<const uint8_t*>(c->extendedprice),
                              reinterpret_cast<const uint8_t*>(dev_keys)};
    for (int k = 0; k < 6; ++k) {
        if (!cols[k] && rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
        if (!aligned16(cols[k])) return set_error(Q1_ERR_INVALID_ARGUMENT, "device columns must start on a 16-byte boundary");
    }
    if (!aligned16(dev_aggregates) || !aligned16(dev_scratch))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "aggregates and scratch must be 16-byte aligned");
    if (rows == 0) return Q1_OK;
    int dev = 0;
    Q1_CUDA(cudaGetDevice(&dev));
    DeviceInfo* di = nullptr;
    q1_status st = device_info(dev, &di);
    if (st != Q1_OK) return st;
    const int max_blocks = (cfg && cfg->blocks > 0) ? cfg->blocks : 0;
    cudaError_t e = launch_groupkey(placement, cols, rows, clamp_rel(cutoff_day), num_groups,
                                    reinterpret_cast<unsigned long long*>(dev_scratch),
                                    reinterpret_cast<unsigned long long*>(dev_aggregates), di->status, di->sm_count,
                                    max_blocks, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return cuda_error(e, "group-key kernel launch");
    return Q1_OK;
}

q1_status q1_zipf_cdf(uint32_t num_groups, double s, uint32_t* cdf) {
    if (!cdf || num_groups < 1) return set_error(Q1_ERR_INVALID_ARGUMENT, "bad argument");
    std::vector<double> c(num_groups);
    double acc = 0;
    for (uint32_t k = 0; k < num_groups; ++k) {
        acc += 1.0 / std::pow((double)(k + 1), s);
        c[k] = acc;
    }
    for (uint32_t k = 0; k < num_groups; ++k) {
        double t = std::floor(c[k] / acc * 4294967296.0);
        cdf[k] = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
    }
    cdf[num_groups - 1] = 0xFFFFFFFFu;
    return Q1_OK;
}

q1_status q1_generate_group_keys_device(uint64_t seed, uint64_t first_row, uint64_t rows, uint32_t num_groups,
                                        const uint32_t* dev_cdf, uint32_t* dev_keys, void* cuda_stream) {
    if (!dev_keys || num_groups < 1) return set_error(Q1_ERR_INVALID_ARGUMENT, "bad argument");
    cudaError_t e = launch_generate_keys(seed, first_row, rows, num_groups, dev_cdf, dev_keys, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return cuda_error(e, "key generator launch");
    return Q1_OK;
}

// ---------------------------------------------------------------------------------------------
// Generators
// ---------------------------------------------------------------------------------------------

q1_status q1_generate_host(uint64_t seed, uint64_t first_row, uint64_t rows, q1_columns* out) {
    if (!out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    const uint64_t key = gen_key(seed);
    auto work = [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; ++i) {
            const GenRow g = gen_row(key, first_row + i);
            if (out->shipdate) const_cast<int32_t*>(out->shipdate)[i] = g.shipdate;
            if (out->quantity) const_cast<int64_t*>(out->quantity)[i] = (int64_t)g.quantity * 100;
            if (out->extendedprice) const_cast<int64_t*>(out->extendedprice)[i] = g.extprice;
            if (out->discount) const_cast<int64_t*>(out->discount)[i] = g.discount;
            if (out->tax) const_cast<int64_t*>(out->tax)[i] = g.tax;
            if (out->returnflag) const_cast<char*>(out->returnflag)[i] = g.returnflag;
            if (out->linestatus) const_cast<char*>(out->linestatus)[i] = g.linestatus;
        }
    };
    unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
    if (rows < (1u << 20)) nt = 1;
    std::vector<std::thread> th;
    const uint64_t per = (rows + nt - 1) / nt;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, std::min(rows, t * per), std::min(rows, (t + 1) * per));
    work(0, std::min(rows, per));
    for (auto& t : th) t.join();
    return Q1_OK;
}

q1_status q1_generate_compressed_device(uint64_t seed, uint64_t first_row, uint64_t rows, q1_flag_packing packing,
                                        const q1_compressed_host_out* o, void* cuda_stream) {
    if (!o) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (rows == 0) return Q1_OK;
    if (!o->shipdate || !o->discount || !o->extendedprice || !o->tax || !o->quantity)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output column");
    if (!aligned16(o->shipdate) || !aligned16(o->discount) || !aligned16(o->extendedprice) || !aligned16(o->tax) ||
        !aligned16(o->quantity))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "device columns must start on a 16-byte boundary");
    if (first_row % 32) return set_error(Q1_ERR_INVALID_ARGUMENT, "first_row must be a multiple of 32");
    GenCompressedOut g{o->shipdate, o->discount, o->extendedprice, o->tax, o->quantity, nullptr, nullptr, nullptr};
    if (packing == Q1_FLAGS_PAIR_2BIT) {
        if (!o->flags) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing flags column");
        g.flags = o->flags;
    } else if (packing == Q1_FLAGS_SEPARATE) {
        if (!o->returnflag || !o->linestatus) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing flag columns");
        g.returnflag = o->returnflag;
        g.linestatus = o->linestatus;
    } else {
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown flag packing");
    }
    cudaError_t e = launch_generate_compressed(seed, first_row, rows, g, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return cuda_error(e, "generator kernel launch");
    return Q1_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Fault injection and the bounded-wait self-test
// ---------------------------------------------------------------------------------------------

namespace q1 {
namespace {
std::atomic<uint32_t> g_faults[kFaultKinds];
}
bool take_fault(FaultKind kind) {
    uint32_t v = g_faults[kind].load(std::memory_order_relaxed);
    while (v) {
        if (g_faults[kind].compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return true;
    }
    return false;
}
void set_faults(int kind, uint32_t count) { g_faults[kind].store(count, std::memory_order_relaxed); }
}  // namespace q1

extern "C" {

q1_status q1_inject_fault(q1_fault kind, uint32_t count) {
    if (kind == Q1_FAULT_NONE) {
        for (int k = 1; k < kFaultKinds; ++k) set_faults(k, 0);
        return Q1_OK;
    }
    if (kind < Q1_FAULT_CPU_WORKER || kind > Q1_FAULT_SERVE_ROUND)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown fault kind");
    set_faults((int)kind, count);
    return Q1_OK;
}

q1_status q1_selftest_cpu_share(const q1_compressed_columns* cols, uint64_t begin, uint64_t end, int32_t cutoff_day,
                                void* aggregates) {
    if (!cols || !aggregates || begin > end) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument or begin > end");
    if (begin == end) return Q1_OK;
    HostCompressed h;
    h.ship = cols->shipdate;
    h.disc = cols->discount;
    h.price = cols->extendedprice;
    h.tax = cols->tax;
    h.qty = cols->quantity;
    h.pair = cols->flag_packing == Q1_FLAGS_PAIR_2BIT;
    if (h.pair) {
        if (cols->num_pair_codes < 1 || cols->num_pair_codes > 4)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "num_pair_codes must be 1..4");
        h.flags = cols->flags;
        memcpy(h.pair_group, cols->pair_group, 4);
        for (uint32_t i = 0; i < 4; ++i) {
            if (i >= cols->num_pair_codes) h.pair_group[i] = h.pair_group[0];
            if (h.pair_group[i] >= 6) return set_error(Q1_ERR_INVALID_ARGUMENT, "pair_group entries must be < 6");
        }
    } else {
        h.rf = cols->returnflag;
        h.ls = cols->linestatus;
    }
    if (!h.ship || !h.disc || !h.price || !h.tax || !h.qty || (h.pair ? !h.flags : (!h.rf || !h.ls)))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
    Agg128 a;
    memcpy(&a, aggregates, sizeof(a));
    const bool ok = cpu_aggregate_compressed(h, begin, end, cutoff_day - kShipDateFrame, &a);
    memcpy(aggregates, &a, sizeof(a));
    return ok ? Q1_OK : set_error(Q1_ERR_DOMAIN, "a passing row is outside the kernels' domain");
}

q1_status q1_selftest_cpu_share_uncompressed(const q1_columns* cols, uint64_t begin, uint64_t end, int32_t cutoff_day,
                                             void* aggregates) {
    if (!cols || !aggregates || begin > end) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument or begin > end");
    if (begin == end) return Q1_OK;
    HostUncompressed h;
    h.ship = cols->shipdate;
    h.disc = cols->discount;
    h.price = cols->extendedprice;
    h.tax = cols->tax;
    h.qty = cols->quantity;
    h.rf = cols->returnflag;
    h.ls = cols->linestatus;
    if (!h.ship || !h.disc || !h.price || !h.tax || !h.qty || !h.rf || !h.ls)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
    Agg128 a;
    memcpy(&a, aggregates, sizeof(a));
    const bool ok = cpu_aggregate_uncompressed(h, begin, end, cutoff_day, &a);
    memcpy(aggregates, &a, sizeof(a));
    return ok ? Q1_OK : set_error(Q1_ERR_DOMAIN, "a passing row's int64 products overflow");
}

q1_status q1_selftest_wait_timeout(uint32_t limit_us, void* cuda_stream) {
    if (limit_us == 0 || limit_us > 2000000) return set_error(Q1_ERR_INVALID_ARGUMENT, "limit must be 1 us .. 2 s");
    int dev = 0;
    Q1_CUDA(cudaGetDevice(&dev));
    DeviceInfo* di = nullptr;
    q1_status st = device_info(dev, &di);
    if (st != Q1_OK) return st;
    cudaError_t e = launch_wait_selftest((uint64_t)limit_us * 1000ull, di->status, (cudaStream_t)cuda_stream);
    if (e != cudaSuccess) return cuda_error(e, "self-test launch");
    return Q1_OK;
}

}  // extern "C"
