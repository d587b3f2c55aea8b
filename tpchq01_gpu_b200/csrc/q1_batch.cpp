// Batched aggregation host runtime: instance descriptors, the device work queue, the autotuner
// and CUDA-graph capture of one batch execution.
//
// One execution = [zero the instances' result tables] + zero the scratch + reset the queue
// cursor + the persistent batch kernel + the finalize kernel, captured once into a CUDA graph and
// replayed by every q1_batch_run.
//
// Autotuner: an instance's class is (floor(log2 rows), num_groups, selectivity decile), the
// selectivity being measured on a strided sample of its ship dates. For every class the tuner
// times the batch kernel on the class's largest instance alone under each applicable placement
// (registers when num_groups <= 4, shared table, global) and keeps the fastest; the work-item
// size (tiles per item) is then chosen by timing the whole batch with a few candidates. Results
// are cached in a text file ("mode <log2rows> <groups> <decile> <mode>", "chunk <signature>
// <tiles>") so later batches with the same classes skip the measurements.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "q1.h"
#include "q1_batch.h"
#include "q1_common.cuh"
#include "q1_internal.h"

using namespace q1;

namespace {

struct DevMem {
    void* p = nullptr;
    ~DevMem() {
        if (p) cudaFree(p);
    }
    q1_status alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        if (!n) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaMalloc (batch)");
        }
        return Q1_OK;
    }
};

using ClassKey = std::tuple<int, uint32_t, int>;   // log2 rows, groups, selectivity decile

std::mutex g_cache_mutex;
std::map<std::string, std::map<ClassKey, uint32_t>> g_mode_cache;     // per cache file
std::map<std::string, std::map<std::string, uint32_t>> g_chunk_cache;

void load_cache(const std::string& path) {
    if (path.empty() || g_mode_cache.count(path)) return;
    auto& modes = g_mode_cache[path];
    auto& chunks = g_chunk_cache[path];
    std::ifstream f(path);
    std::string kind;
    while (f >> kind) {
        if (kind == "mode") {
            int lr, dec;
            uint32_t g, m;
            if (f >> lr >> g >> dec >> m) modes[ClassKey(lr, g, dec)] = m;
        } else if (kind == "chunk") {
            std::string sig;
            uint32_t t;
            if (f >> sig >> t) chunks[sig] = t;
        } else {
            std::string rest;
            std::getline(f, rest);
        }
    }
}

void save_cache(const std::string& path) {
    if (path.empty()) return;
    std::ofstream f(path, std::ios::trunc);
    f << "# q1 batch autotuner cache: mode <log2rows> <groups> <selectivity decile> <0 registers|1 shared|2 global>;"
         " chunk <signature> <tiles per work item>\n";
    for (auto& kv : g_mode_cache[path])
        f << "mode " << std::get<0>(kv.first) << ' ' << std::get<1>(kv.first) << ' ' << std::get<2>(kv.first) << ' '
          << kv.second << '\n';
    for (auto& kv : g_chunk_cache[path]) f << "chunk " << kv.first << ' ' << kv.second << '\n';
}

}  // namespace

uint32_t q1::batch_engine(uint32_t mode, uint32_t num_groups) {
    if (mode == kModeRegisters && num_groups <= 4) return kEngRegisters;
    if (mode == kModeGlobal) return kEngGlobal;
    if (num_groups <= 64) return kEngCube3;     // ka::kCube3MaxGroups
    if (num_groups <= 1024) return kEngCube;    // ka::kCubeMaxGroups
    return kEngSlots;
}

namespace {

// Relative cost of a row per engine (time per row of the group-key kernel on a B200 at 100% pass,
// uniform keys, register planes = 1: 4 groups 1.57 ms per 600 M rows, 64 groups 1.87 ms, 1024
// groups 2.26 ms, 4096 groups 2.79 ms): used only to split the grid.
constexpr double kEngineCost[kEngines] = {1.0, 1.19, 1.44, 1.78, 10.0};

void plan_items(const BatchInstanceDev* inst, uint32_t n, uint32_t chunk, int only, std::vector<BatchItem>& items,
                uint32_t begin[kEngines + 1]) {
    std::vector<BatchItem> per[kEngines];
    for (uint32_t i = 0; i < n; ++i) {
        if (only >= 0 && i != (uint32_t)only) continue;
        const uint32_t e = batch_engine(inst[i].mode, inst[i].num_groups);
        const uint64_t tiles = (inst[i].rows + kBatchTileRows - 1) / kBatchTileRows;
        for (uint64_t t = 0; t < tiles; t += chunk) {
            BatchItem it{};
            it.instance = i;
            it.first_tile = (uint32_t)t;
            it.num_tiles = (uint32_t)std::min<uint64_t>(chunk, tiles - t);
            per[e].push_back(it);
        }
    }
    items.clear();
    for (uint32_t e = 0; e < kEngines; ++e) {
        // largest items first: the atomic cursor then hands out an engine's work in LPT order
        std::stable_sort(per[e].begin(), per[e].end(),
                         [](const BatchItem& a, const BatchItem& c) { return a.num_tiles > c.num_tiles; });
        begin[e] = (uint32_t)items.size();
        items.insert(items.end(), per[e].begin(), per[e].end());
    }
    begin[kEngines] = (uint32_t)items.size();
}

// Splits `grid` CTAs: the register-planes kernel gets its cost share (a little under, since the
// table kernel also drains queue 0 once its own queues are empty), the table kernel the rest,
// divided among queues 1..4 by cost.
void plan_roles(const std::vector<BatchItem>& items, const uint32_t begin[kEngines + 1], uint32_t grid,
                BatchParams& prm) {
    double cost[kEngines] = {0, 0, 0, 0, 0}, total = 0, tables = 0;
    for (uint32_t e = 0; e < kEngines; ++e) {
        for (uint32_t j = begin[e]; j < begin[e + 1]; ++j) cost[e] += (double)items[j].num_tiles * kEngineCost[e];
        total += cost[e];
        if (e) tables += cost[e];
    }
    uint32_t regs = 0;
    if (cost[0] > 0) {
        regs = tables > 0 ? (uint32_t)(0.9 * grid * cost[0] / total) : grid;
        regs = std::max<uint32_t>(1, std::min<uint32_t>(regs, grid - (tables > 0 ? 1 : 0)));
        regs = std::min<uint32_t>(regs, begin[1] - begin[0]);
    }
    const uint32_t tgrid = tables > 0 ? std::max<uint32_t>(1, std::min<uint32_t>(grid - regs, begin[kEngines] - begin[1]))
                                      : 0;
    prm.grid_regs = regs;
    prm.grid_tables = tgrid;
    // queue shares of the table kernel
    uint32_t share[kEngines] = {0, 0, 0, 0, 0}, used = 0, big = 1;
    for (uint32_t e = 1; e < kEngines; ++e) {
        if (cost[e] <= 0) continue;
        share[e] = std::max<uint32_t>(1, (uint32_t)(tgrid * cost[e] / (tables > 0 ? tables : 1)));
        used += share[e];
        if (share[e] > share[big]) big = e;
    }
    if (tgrid) {
        if (used > tgrid) share[big] -= std::min(share[big] - 1, used - tgrid);
        else share[big] += tgrid - used;
    }
    prm.role_end[0] = 0;
    uint32_t acc = 0;
    for (uint32_t e = 1; e < kEngines; ++e) prm.role_end[e] = (acc += share[e]);
}

}  // namespace

void q1::batch_plan(const BatchInstanceDev* inst, uint32_t n, uint32_t chunk, uint32_t grid, std::vector<BatchItem>& items,
                    BatchParams& prm) {
    plan_items(inst, n, std::max<uint32_t>(1, chunk), -1, items, prm.item_begin);
    plan_roles(items, prm.item_begin, grid, prm);
}

struct q1_batch {
    int device = 0;
    DeviceInfo* di = nullptr;
    uint32_t n = 0;
    std::vector<BatchInstanceDev> inst;      // host copy of the device descriptors
    std::vector<uint64_t> group_base;        // n + 1 prefix sums of num_groups
    std::vector<ClassKey> cls;
    std::vector<uint32_t> modes;
    std::vector<BatchItem> items;
    BatchParams roles{};                     // item_begin / role_end of `items`
    uint32_t launch_grid = 0;
    uint64_t total_groups = 0;
    uint64_t total_rows = 0;
    uint32_t chunk = 0;
    uint32_t grid = 0;
    bool use_graph = true;
    bool zero_outputs = true;
    std::string cache;
    DevMem d_inst, d_items, d_base, d_scratch, d_cursor;
    cudaStream_t aux = nullptr;              // the register-planes kernel runs beside the table kernel
    cudaEvent_t fork = nullptr, join = nullptr;
    ~q1_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (aux) cudaStreamDestroy(aux);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t tuned_classes = 0;
};

// Items of every instance (only < 0) or of one instance, grouped by engine, and the grid roles.
static void build_items(q1_batch* b, uint32_t chunk, int only = -1) {
    for (uint32_t i = 0; i < b->n; ++i) b->inst[i].mode = b->modes[i];
    plan_items(b->inst.data(), b->n, std::max<uint32_t>(1, chunk), only, b->items, b->roles.item_begin);
    plan_roles(b->items, b->roles.item_begin, b->grid, b->roles);
    b->launch_grid = b->roles.grid_regs + b->roles.grid_tables;
}

static q1_status upload(q1_batch* b) {
    for (uint32_t i = 0; i < b->n; ++i) b->inst[i].mode = b->modes[i];
    Q1_CUDA(cudaMemcpy(b->d_inst.p, b->inst.data(), sizeof(BatchInstanceDev) * b->n, cudaMemcpyHostToDevice));
    q1_status st = b->d_items.alloc(sizeof(BatchItem) * std::max<size_t>(1, b->items.size()));
    if (st != Q1_OK) return st;
    if (!b->items.empty())
        Q1_CUDA(cudaMemcpy(b->d_items.p, b->items.data(), sizeof(BatchItem) * b->items.size(), cudaMemcpyHostToDevice));
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return Q1_OK;
}

// The launches of one execution (graph body).
static q1_status enqueue(q1_batch* b, cudaStream_t s) {
    if (b->zero_outputs && b->total_groups) {
        Q1_CUDA(launch_batch_zero_outputs(static_cast<const BatchInstanceDev*>(b->d_inst.p),
                                          static_cast<const uint64_t*>(b->d_base.p), b->n, b->total_groups, s));
    }
    Q1_CUDA(cudaMemsetAsync(b->d_scratch.p, 0, b->total_groups * 64ull, s));
    Q1_CUDA(cudaMemsetAsync(b->d_cursor.p, 0, 4 * kEngines, s));
    if (!b->items.empty()) {
        BatchParams prm = b->roles;
        prm.inst = static_cast<const BatchInstanceDev*>(b->d_inst.p);
        prm.items = static_cast<const BatchItem*>(b->d_items.p);
        prm.cursor = static_cast<uint32_t*>(b->d_cursor.p);
        prm.status = b->di->status;
        Q1_CUDA(launch_batch(prm, prm.grid_regs, prm.grid_tables, s, b->aux, b->fork, b->join));
    }
    Q1_CUDA(launch_batch_finalize(static_cast<const BatchInstanceDev*>(b->d_inst.p),
                                  static_cast<const uint64_t*>(b->d_base.p), b->n, b->total_groups, s));
    return Q1_OK;
}

static q1_status time_batch(q1_batch* b, cudaStream_t s, int reps, float* best_ms) {
    cudaEvent_t e0, e1;
    Q1_CUDA(cudaEventCreate(&e0));
    Q1_CUDA(cudaEventCreate(&e1));
    *best_ms = 1e30f;
    for (int r = 0; r < reps; ++r) {
        Q1_CUDA(cudaEventRecord(e0, s));
        q1_status st = enqueue(b, s);
        if (st != Q1_OK) return st;
        Q1_CUDA(cudaEventRecord(e1, s));
        Q1_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        Q1_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *best_ms = std::min(*best_ms, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return check_device_status(s, b->di->status);
}

// Work-item size: about 16 items per CTA. Smaller items keep the CTAs reading neighbouring tiles
// of the same instance at the same time; on 256 instances of 1.49 G rows, 64-tile items ran
// 5.14 ms against 5.25 ms for 256-tile items.
static uint32_t default_chunk(const q1_batch* b) {
    const uint64_t tiles = (b->total_rows + kBatchTileRows - 1) / kBatchTileRows;
    uint64_t c = tiles / (uint64_t)(b->grid ? b->grid * 16 : 1);
    return (uint32_t)std::max<uint64_t>(4, std::min<uint64_t>(1024, c));
}

static std::string chunk_signature(const q1_batch* b) {
    std::ostringstream o;
    double lg = 0;
    for (uint32_t i = 0; i < b->n; ++i) lg += std::log2((double)std::max<uint32_t>(1, b->inst[i].num_groups));
    o << b->n << 'x' << (int)std::log2((double)std::max<uint64_t>(1, b->total_rows)) << 'g'
      << (int)std::lround(lg / std::max<uint32_t>(1, b->n));
    return o.str();
}

extern "C" {

q1_status q1_batch_create(const q1_batch_instance* in, uint32_t n, const q1_batch_opts* opts, void* cuda_stream,
                          q1_batch** out) {
    if (!out || (n && !in)) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<q1_batch> b(new q1_batch());
    cudaStream_t s = (cudaStream_t)cuda_stream;
    Q1_CUDA(cudaGetDevice(&b->device));
    q1_status st = device_info(b->device, &b->di);
    if (st == Q1_OK) {
        Q1_CUDA(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
        Q1_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        Q1_CUDA(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
    }
    if (st != Q1_OK) return st;
    b->n = n;
    b->use_graph = opts ? opts->use_graph != 0 : true;
    b->zero_outputs = opts ? opts->accumulate == 0 : true;
    b->cache = (opts && opts->tune_cache) ? opts->tune_cache : "";
    const int tune = opts ? opts->tune : 0;
    b->grid = (uint32_t)b->di->sm_count;
    b->inst.resize(n);
    b->group_base.assign(n + 1, 0);
    b->modes.assign(n, kModeShared);
    b->cls.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const q1_batch_instance& x = in[i];
        if (x.num_groups < 1 || x.num_groups > Q1_MAX_KEY_GROUPS)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + ": num_groups must be 1..65536");
        if (!x.aggregates) return set_error(Q1_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + ": null aggregates");
        const uint8_t* cols[6] = {reinterpret_cast<const uint8_t*>(x.cols.shipdate), x.cols.quantity, x.cols.discount,
                                  x.cols.tax, reinterpret_cast<const uint8_t*>(x.cols.extendedprice),
                                  reinterpret_cast<const uint8_t*>(x.keys)};
        for (int c = 0; c < 6; ++c) {
            if (x.rows && !cols[c]) return set_error(Q1_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + ": missing column");
            if (((uintptr_t)cols[c] & 15u) != 0)
                return set_error(Q1_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + ": columns must be 16-byte aligned");
        }
        if (x.rows > (uint64_t)UINT32_MAX * kBatchTileRows)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "instance " + std::to_string(i) + ": too many rows");
        BatchInstanceDev& d = b->inst[i];
        memset(&d, 0, sizeof(d));
        for (int c = 0; c < 6; ++c) d.col[c] = cols[c];
        d.rows = x.rows;
        const int64_t rel = (int64_t)x.cutoff_day - kShipDateFrame;
        d.cutoff = rel < -1 ? -1 : (rel > 32767 ? 32767 : (int32_t)rel);
        d.num_groups = x.num_groups;
        d.out = reinterpret_cast<unsigned long long*>(x.aggregates);
        b->group_base[i + 1] = b->group_base[i] + x.num_groups;
        b->total_rows += x.rows;
        b->modes[i] = x.num_groups <= 4 ? kModeRegisters : kModeShared;   // heuristic default
    }
    b->total_groups = b->group_base[n];
    if ((st = b->d_inst.alloc(sizeof(BatchInstanceDev) * std::max<uint32_t>(1, n))) != Q1_OK) return st;
    if ((st = b->d_base.alloc(sizeof(uint64_t) * (n + 1))) != Q1_OK) return st;
    if ((st = b->d_scratch.alloc(b->total_groups * 64ull)) != Q1_OK) return st;
    if ((st = b->d_cursor.alloc(4 * kEngines)) != Q1_OK) return st;
    unsigned long long* scratch = static_cast<unsigned long long*>(b->d_scratch.p);
    for (uint32_t i = 0; i < n; ++i) b->inst[i].acc = scratch + 8ull * b->group_base[i];
    Q1_CUDA(cudaMemcpy(b->d_base.p, b->group_base.data(), sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice));
    Q1_CUDA(batch_prepare_launch());

    // classes: log2 rows, groups, selectivity decile of a strided sample of ship dates
    for (uint32_t i = 0; i < n; ++i) {
        const BatchInstanceDev& d = b->inst[i];
        int dec = 10;
        if (d.rows) {
            const uint64_t k = std::min<uint64_t>(d.rows, 64);
            std::vector<uint16_t> sample(k);
            const uint64_t stride = d.rows / k;
            Q1_CUDA(cudaMemcpy2D(sample.data(), sizeof(uint16_t), d.col[0], stride * sizeof(uint16_t), sizeof(uint16_t), k,
                                 cudaMemcpyDeviceToHost));
            uint64_t pass = 0;
            for (uint16_t v : sample) pass += (int32_t)v <= d.cutoff;
            dec = (int)(pass * 10 / k);
        }
        b->cls[i] = ClassKey((int)std::log2((double)std::max<uint64_t>(1, d.rows)), d.num_groups, dec);
    }

    b->chunk = (opts && opts->chunk_tiles > 0) ? (uint32_t)opts->chunk_tiles : default_chunk(b.get());
    if (tune > 0) {
        std::lock_guard<std::mutex> lk(g_cache_mutex);
        load_cache(b->cache);
        auto& modes = g_mode_cache[b->cache];
        // per class: time the candidate placements on the class's largest instance alone
        std::map<ClassKey, uint32_t> rep;
        for (uint32_t i = 0; i < n; ++i)
            if (!rep.count(b->cls[i]) || b->inst[i].rows > b->inst[rep[b->cls[i]]].rows) rep[b->cls[i]] = i;
        const std::vector<uint32_t> saved_modes = b->modes;
        for (auto& kv : rep) {
            if (tune == 1 && modes.count(kv.first)) continue;
            const uint32_t i = kv.second;
            // Below 256 tiles a class's time is launch overhead, not placement: keep the heuristic.
            if ((b->inst[i].rows + kBatchTileRows - 1) / kBatchTileRows < 256) {
                modes[kv.first] = b->modes[i];
                continue;
            }
            std::vector<uint32_t> cands;
            if (b->inst[i].num_groups <= 4) cands.push_back(kModeRegisters);
            cands.push_back(kModeShared);
            cands.push_back(kModeGlobal);
            // the heuristic placement keeps the class unless another is faster by more than 3%
            uint32_t best = saved_modes[i];
            float best_ms = 1e30f;
            std::stable_sort(cands.begin(), cands.end(), [&](uint32_t a, uint32_t c) {
                return (a == saved_modes[i]) > (c == saved_modes[i]);
            });
            for (uint32_t m : cands) {
                b->modes = saved_modes;
                b->modes[i] = m;
                const uint64_t tiles = (b->inst[i].rows + kBatchTileRows - 1) / kBatchTileRows;
                const uint32_t c = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(1024, tiles / (b->grid * 4ull) + 1));
                build_items(b.get(), c, (int)i);
                if ((st = upload(b.get())) != Q1_OK) return st;
                float ms = 0;
                if ((st = time_batch(b.get(), s, 3, &ms)) != Q1_OK) return st;
                if (m != saved_modes[i]) ms *= 1.03f;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = m;
                }
            }
            modes[kv.first] = best;
            b->modes = saved_modes;
            ++b->tuned_classes;
        }
        for (uint32_t i = 0; i < n; ++i)
            if (modes.count(b->cls[i])) b->modes[i] = modes[b->cls[i]];
        // work-item size for the whole batch
        auto& chunks = g_chunk_cache[b->cache];
        const std::string sig = chunk_signature(b.get());
        if (!(opts && opts->chunk_tiles > 0)) {
            if (tune == 1 && chunks.count(sig)) {
                b->chunk = chunks[sig];
            } else {
                const uint32_t base = default_chunk(b.get());
                std::vector<uint32_t> cands = {std::max<uint32_t>(2, base / 4), base, std::min<uint32_t>(4096, base * 4)};
                float best_ms = 1e30f;
                for (uint32_t c : cands) {
                    build_items(b.get(), c);
                    if ((st = upload(b.get())) != Q1_OK) return st;
                    float ms = 0;
                    if ((st = time_batch(b.get(), s, 2, &ms)) != Q1_OK) return st;
                    if (ms < best_ms) {
                        best_ms = ms;
                        b->chunk = c;
                    }
                }
                chunks[sig] = b->chunk;
            }
        }
        save_cache(b->cache);
    }
    build_items(b.get(), b->chunk);
    if ((st = upload(b.get())) != Q1_OK) return st;
    *out = b.release();
    return Q1_OK;
}

q1_status q1_batch_run(q1_batch* b, void* cuda_stream) {
    if (!b) return set_error(Q1_ERR_INVALID_ARGUMENT, "null batch");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    if (!b->use_graph) return enqueue(b, s);
    if (!b->exec) {
        // capture on a private stream so that the caller's stream may be the legacy default one
        cudaStream_t cap;
        Q1_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        q1_status st = Q1_OK;
        if (e == cudaSuccess) st = enqueue(b, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamBeginCapture");
        if (st != Q1_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e2 != cudaSuccess) return cuda_error(e2, "cudaStreamEndCapture");
        b->graph = g;
        Q1_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    Q1_CUDA(cudaGraphLaunch(b->exec, s));
    return Q1_OK;
}

q1_status q1_batch_describe(q1_batch* b, q1_batch_desc* d) {
    if (!b || !d) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    memset(d, 0, sizeof(*d));
    d->instances = b->n;
    d->items = (uint32_t)b->items.size();
    d->chunk_tiles = b->chunk;
    d->tile_rows = kBatchTileRows;
    d->grid = b->launch_grid;
    d->total_rows = b->total_rows;
    d->total_groups = b->total_groups;
    d->uses_graph = b->use_graph ? 1 : 0;
    d->tuned_classes = b->tuned_classes;
    for (uint32_t i = 0; i < b->n; ++i) d->mode_count[std::min<uint32_t>(2, b->modes[i])]++;
    return Q1_OK;
}

q1_status q1_batch_instance_mode(q1_batch* b, uint32_t i, int32_t* mode) {
    if (!b || !mode || i >= b->n) return set_error(Q1_ERR_INVALID_ARGUMENT, "bad argument");
    *mode = (int32_t)b->modes[i];
    return Q1_OK;
}

q1_status q1_batch_destroy(q1_batch* b) {
    if (!b) return Q1_OK;
    delete b;
    return Q1_OK;
}

}  // extern "C"
