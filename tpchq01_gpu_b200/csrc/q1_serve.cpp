// Serving loop: queries arrive one by one and are answered in rounds (continuous batching).
//
// Resident table: `resident_rows` rows of the seeded generator, compressed (pair codes) plus a
// uint32 key column uniform over [0, 64), held in HBM. At open the server builds, for both
// groupings (the 6 (returnflag, linestatus) groups and the 64 keys), the partial aggregates per
// ship day and turns them into prefix sums over days: the exact answer for "l_shipdate <= c" is
// then the row of day c. These partial aggregates stay resident in HBM.
//
// Ad-hoc requests name a table of their own (seed, rows, grouping, groups). It is generated on
// the device into an arena whose size is the HBM budget the first time it is named and stays
// resident; when a new table does not fit, least recently used tables that no admitted request
// reads are evicted.
//
// Continuous batching over round lanes. A lane is one round's worth of streams, device and pinned
// buffers and a status word (opts.max_rounds_in_flight lanes, 2 by default). A dispatcher thread
// forms a round from the queue head (FIFO) whenever a lane is free, as long as a response slot is
// free and, for an ad-hoc request, its table is or can be made resident, and enqueues it on the
// lane's streams without waiting: requests that arrive while a round is on the GPU form the next
// round at once, and its copies, generation and kernels queue behind and overlap the running
// round on the device (the persistent kernels of the next round take SMs as the running round's
// CTAs finish). A completer thread retires rounds in order: it waits for the oldest lane's
// streams, reads the lane's status word and the responses, completes the tickets and frees the
// lane. A round = generate the missing tables, one launch of the persistent batch kernel over all
// ad-hoc requests (batch_kernels.cu), one lookup kernel for the resident requests, one copy of
// every response back to the host. A table generated by one lane and read by another is ordered
// by an event. Latency is measured per request from submission to completion. Q1_SERVE_PLAIN
// runs the same loop with one lane, one request per round and one plain scan launch per request:
// the comparison point.
//
// q1_server_plain answers one request from scratch (fresh table, plain scan launch) on its own
// stream and is the arbiter every served response must equal bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "q1.h"
#include "q1_batch.h"
#include "q1_common.cuh"
#include "q1_internal.h"
#include "q1_kernels.h"
#include "q1_serve.h"

using namespace q1;

namespace {

constexpr uint32_t kMaxGroups = Q1_SERVE_MAX_GROUPS;
constexpr uint32_t kRespWords = kMaxGroups * 12;   // u64 words per response slot
constexpr uint64_t kAlign = 256;

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }
double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Dev {
    void* p = nullptr;
    uint64_t n = 0;
    Dev() = default;
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
    ~Dev() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    q1_status alloc(uint64_t bytes) {
        release();
        if (take_fault(kFaultDeviceAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected device allocation failure");
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaMalloc (server)");
        }
        n = bytes;
        return Q1_OK;
    }
    template <class T>
    T* as(uint64_t byte_off = 0) const { return reinterpret_cast<T*>(static_cast<uint8_t*>(p) + byte_off); }
};

struct Pinned {
    void* p = nullptr;
    Pinned() = default;
    Pinned(const Pinned&) = delete;
    Pinned& operator=(const Pinned&) = delete;
    ~Pinned() { release(); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
    }
    q1_status alloc(uint64_t bytes) {
        release();
        if (take_fault(kFaultPinnedAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected pinned allocation failure");
        cudaError_t e = cudaHostAlloc(&p, bytes ? bytes : 16, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_error(e, "cudaHostAlloc (server)");
        }
        return Q1_OK;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

// First-fit free list over the ad-hoc arena (offsets and lengths in bytes).
struct Arena {
    std::map<uint64_t, uint64_t> free_;   // offset -> length
    void reset(uint64_t n) {
        free_.clear();
        if (n) free_[0] = n;
    }
    bool alloc(uint64_t n, uint64_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                const uint64_t rest = it->second - n, at = it->first + n;
                free_.erase(it);
                if (rest) free_[at] = rest;
                return true;
            }
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

// Byte layout of one table of `rows` rows: ship u16 | qty u8 | disc u8 | tax u8 | price u32 |
// keys u32 (or, for the plain path's pair layout, 2-bit pair codes in the key slot).
struct TableLayout {
    uint64_t off[6];
    uint64_t total;
    explicit TableLayout(uint64_t rows) {
        const uint64_t b[6] = {2 * rows, rows, rows, rows, 4 * rows, 4 * rows};
        uint64_t o = 0;
        for (int c = 0; c < 6; ++c) {
            off[c] = o;
            o += align_up(b[c] + 16, kAlign);
        }
        total = o;
    }
};

// An ad-hoc table is named by (seed, rows, grouping, groups): its key column depends on both.
struct TableKey {
    uint64_t seed, rows;
    uint32_t grouping, groups;
    bool operator<(const TableKey& o) const {
        if (seed != o.seed) return seed < o.seed;
        if (rows != o.rows) return rows < o.rows;
        if (grouping != o.grouping) return grouping < o.grouping;
        return groups < o.groups;
    }
};

struct CachedTable {
    uint64_t off = 0, len = 0;
    uint32_t pins = 0;        // requests of the forming or running round that read it
    uint64_t last_use = 0;
    bool ready = false;       // generation enqueued (readers on other lanes wait for gen_ev)
    cudaEvent_t gen_ev = nullptr;   // recorded after the generation on gen_stream
    cudaStream_t gen_stream = nullptr;
};

struct Ticket {
    uint64_t id = 0;
    q1_request req{};
    double t_submit = 0, t_admit = 0, t_done = 0;
    bool done = false;
    q1_status status = Q1_OK;
    uint32_t groups = 0;
    std::vector<q1_i128> aggs;   // [groups][6]
    CachedTable* table = nullptr;
};

inline TableKey key_of(const q1_request& r) {
    return TableKey{r.adhoc_seed, r.adhoc_rows, (uint32_t)r.grouping,
                    r.grouping == Q1_GROUP_FLAGS ? 6u : r.num_groups};
}

q1_status validate_request(const q1_request* r, uint64_t max_adhoc_rows, uint64_t budget) {
    if (r->kind != Q1_REQ_RESIDENT && r->kind != Q1_REQ_ADHOC)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown request kind");
    if (r->grouping != Q1_GROUP_FLAGS && r->grouping != Q1_GROUP_KEYS)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown grouping");
    if (r->grouping == Q1_GROUP_KEYS) {
        if (r->num_groups < 1 || r->num_groups > kMaxGroups)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "num_groups must be in 1..64");
        if (r->kind == Q1_REQ_RESIDENT && r->num_groups != Q1_SERVE_RESIDENT_KEY_GROUPS)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "the resident key column has 64 groups");
    }
    if (r->kind == Q1_REQ_ADHOC) {
        if (r->adhoc_rows > max_adhoc_rows)
            return set_error(Q1_ERR_INVALID_ARGUMENT, "ad-hoc table larger than max_adhoc_rows");
        if (TableLayout(r->adhoc_rows).total > budget)
            return set_error(Q1_ERR_BUSY, "ad-hoc table larger than the HBM budget");
    }
    return Q1_OK;
}

// Group slots of a response: the 6 (returnflag, linestatus) groups or the request's key groups.
inline uint32_t groups_of(const q1_request& r) { return r.grouping == Q1_GROUP_FLAGS ? 6u : r.num_groups; }

// Key values of an ad-hoc table: its (returnflag, linestatus) dictionary codes (AF, NF, NO, RF)
// or the request's key groups. Code c belongs to group kPairGroup[c].
constexpr uint32_t kPairGroup[4] = {0, 2, 3, 4};
inline bool coded(const q1_request& r) { return r.kind == Q1_REQ_ADHOC && r.grouping == Q1_GROUP_FLAGS; }
inline uint32_t key_groups(const q1_request& r) { return coded(r) ? 4u : groups_of(r); }

inline int32_t cutoff_rel(int32_t cutoff_day) {
    const int64_t rel = (int64_t)cutoff_day - kShipDateFrame;
    return rel < -1 ? -1 : (rel > 32767 ? 32767 : (int32_t)rel);
}

}  // namespace

namespace {

// One round in flight: its streams (the round; the batch's register-planes kernel), device and
// pinned buffers and status word, and the tickets it answers.
struct Lane {
    cudaStream_t stream = nullptr, aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    Dev d_resp, d_inst, d_items, d_base, d_scratch, d_cursor, d_lookup, d_status;
    Pinned h_resp, h_inst, h_items, h_base, h_lookup, h_status;
    uint64_t items_cap = 0;
    std::vector<Ticket*> batch;
    q1_status enq = Q1_OK;   // status of enqueueing the round
    std::string err;
    Lane() = default;
    Lane(const Lane&) = delete;
    Lane& operator=(const Lane&) = delete;
    ~Lane() {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (aux) {
            cudaStreamSynchronize(aux);
            cudaStreamDestroy(aux);
        }
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

}  // namespace

struct q1_server {
    int device = 0;
    DeviceInfo* di = nullptr;
    cudaStream_t stream = nullptr;         // building the resident table at open
    cudaStream_t plain_stream = nullptr;   // q1_server_plain
    q1_server_opts opts{};

    // resident table: ship | qty | disc | tax | price | codes | keys
    uint64_t res_rows = 0;
    Dev res;
    uint64_t res_off[7] = {};
    uint8_t pair_group[4] = {0, 2, 3, 4};   // the generator's dictionary AF, NF, NO, RF
    uint32_t days = 0;
    Dev cube_pair, cube_key;   // cumulative [days][groups][6] int128

    // ad-hoc tables resident in the arena (dispatcher thread only)
    Arena arena;
    Dev arena_mem;
    std::map<TableKey, CachedTable> cache;
    uint64_t lru_clock = 0;

    // round lanes: free ones, and the ones whose round is on the GPU in submission order
    std::vector<std::unique_ptr<Lane>> lanes;
    std::deque<Lane*> free_lanes, inflight;

    // plain launches: plain_scratch for Q1_SERVE_PLAIN rounds (dispatcher thread); the arbiter
    // (q1_server_plain) has buffers of its own, serialised by arbiter_m
    Dev plain_scratch;
    std::mutex arbiter_m;
    Dev arbiter_table, arbiter_scratch, arbiter_out;

    // queue
    std::mutex m;
    std::condition_variable cv_work, cv_done, cv_retire;
    std::deque<Ticket*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Ticket>> tickets;
    uint64_t next_id = 1;
    bool stop = false;
    bool dispatcher_done = false;
    std::thread dispatcher, completer;
    q1_status fatal = Q1_OK;
    std::string fatal_msg;

    // statistics
    std::vector<double> latencies;
    uint64_t rounds = 0, completed = 0, failed = 0, logical_rows = 0, scanned_rows = 0, admitted_total = 0;
    uint64_t generated_rows = 0, cache_hits = 0, cache_misses = 0, evictions = 0;
    uint64_t overlapped_rounds = 0;   // rounds enqueued while another round was on the GPU
    uint32_t max_in_flight = 0;       // most rounds on the GPU at once
    double t_first = 0, t_last = 0;
};

namespace {

q1_status build_resident(q1_server* s) {
    const uint64_t n = s->res_rows;
    const uint64_t b[7] = {2 * n, n, n, n, 4 * n, 4 * words16(n), 4 * n};
    uint64_t o = 0;
    for (int c = 0; c < 7; ++c) {
        s->res_off[c] = o;
        o += align_up(b[c] + 16, kAlign);
    }
    q1_status st = s->res.alloc(o);
    if (st != Q1_OK) return st;
    Q1_CUDA(cudaMemsetAsync(s->res.p, 0, o, s->stream));
    GenCompressedOut g{s->res.as<uint16_t>(s->res_off[0]), s->res.as<uint8_t>(s->res_off[2]),
                       s->res.as<uint32_t>(s->res_off[4]), s->res.as<uint8_t>(s->res_off[3]),
                       s->res.as<uint8_t>(s->res_off[1]), s->res.as<uint32_t>(s->res_off[5]), nullptr, nullptr};
    Q1_CUDA(launch_generate_compressed(s->opts.seed, 0, n, g, s->stream));
    Q1_CUDA(launch_generate_keys(s->opts.seed, 0, n, Q1_SERVE_RESIDENT_KEY_GROUPS, nullptr,
                                 s->res.as<uint32_t>(s->res_off[6]), s->stream));
    // ship offsets of the generator lie in [1, last order date + 121 - 727563]
    s->days = (uint32_t)(kGenOrderDateLast + 121 - kShipDateFrame + 1);

    // per (day, group) partial aggregates, in windows of days whose table fits shared memory
    Dev acc;
    for (int which = 0; which < 2; ++which) {
        const uint32_t G = which == 0 ? 6u : Q1_SERVE_RESIDENT_KEY_GROUPS;
        const uint64_t acc_bytes = (uint64_t)s->days * G * 64;
        if ((st = acc.alloc(acc_bytes)) != Q1_OK) return st;
        Q1_CUDA(cudaMemsetAsync(acc.p, 0, acc_bytes, s->stream));
        const uint32_t max_slots = 200u * 1024u / 52u;
        const uint32_t window = std::max<uint32_t>(1, max_slots / G);
        for (uint32_t d0 = 0; d0 < s->days; d0 += window) {
            CubePassParams p{};
            p.ship = s->res.as<uint16_t>(s->res_off[0]);
            p.qty = s->res.as<uint8_t>(s->res_off[1]);
            p.disc = s->res.as<uint8_t>(s->res_off[2]);
            p.tax = s->res.as<uint8_t>(s->res_off[3]);
            p.price = s->res.as<uint32_t>(s->res_off[4]);
            p.codes = s->res.as<uint32_t>(s->res_off[5]);
            p.keys = s->res.as<uint32_t>(s->res_off[6]);
            memcpy(p.pair_group, s->pair_group, 4);
            p.pair = which == 0;
            p.num_groups = G;
            p.d0 = d0;
            p.days = std::min(window, s->days - d0);
            p.all_days = s->days;
            p.rows = n;
            p.acc = acc.as<unsigned long long>();
            p.status = s->di->status;
            Q1_CUDA(launch_cube_pass(p, s->di->sm_count, s->stream));
        }
        Dev& cube = which == 0 ? s->cube_pair : s->cube_key;
        if ((st = cube.alloc((uint64_t)s->days * G * 96)) != Q1_OK) return st;
        Q1_CUDA(launch_cube_finalize(acc.as<unsigned long long>(), s->days, G, cube.as<unsigned long long>(), s->stream));
        if ((st = check_device_status(s->stream, s->di->status)) != Q1_OK) return st;
    }
    return Q1_OK;
}

// Called with the lock held.
void complete(q1_server* s, Ticket* t, q1_status st, double when) {
    t->status = st;
    t->done = true;
    t->t_done = when;
    if (st != Q1_OK) {
        s->failed++;
        return;
    }
    s->completed++;
    s->latencies.push_back(t->t_done - t->t_submit);
    const uint64_t rows = t->req.kind == Q1_REQ_RESIDENT ? s->res_rows : t->req.adhoc_rows;
    s->logical_rows += rows;
    if (t->req.kind == Q1_REQ_ADHOC) s->scanned_rows += rows;
    if (s->t_first == 0 || t->t_submit < s->t_first) s->t_first = t->t_submit;
    s->t_last = std::max(s->t_last, when);
}

q1_status grow_items(Lane* L, uint64_t n) {
    if (n <= L->items_cap) return Q1_OK;
    q1_status st;
    if ((st = L->d_items.alloc(sizeof(BatchItem) * n)) != Q1_OK) return st;
    if ((st = L->h_items.alloc(sizeof(BatchItem) * n)) != Q1_OK) return st;
    L->items_cap = n;
    return Q1_OK;
}

q1_status lane_open(Lane* L, uint64_t m) {
    Q1_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
    Q1_CUDA(cudaStreamCreateWithFlags(&L->aux, cudaStreamNonBlocking));
    Q1_CUDA(cudaEventCreateWithFlags(&L->fork, cudaEventDisableTiming));
    Q1_CUDA(cudaEventCreateWithFlags(&L->join, cudaEventDisableTiming));
    q1_status st;
    if ((st = L->d_resp.alloc(m * kRespWords * 8)) != Q1_OK) return st;
    if ((st = L->h_resp.alloc(m * kRespWords * 8)) != Q1_OK) return st;
    if ((st = L->d_inst.alloc(sizeof(BatchInstanceDev) * m)) != Q1_OK) return st;
    if ((st = L->h_inst.alloc(sizeof(BatchInstanceDev) * m)) != Q1_OK) return st;
    if ((st = L->d_base.alloc(sizeof(uint64_t) * (m + 1))) != Q1_OK) return st;
    if ((st = L->h_base.alloc(sizeof(uint64_t) * (m + 1))) != Q1_OK) return st;
    if ((st = L->d_scratch.alloc(m * kMaxGroups * 64)) != Q1_OK) return st;
    if ((st = L->d_cursor.alloc(4 * kEngines)) != Q1_OK) return st;
    if ((st = L->d_lookup.alloc(sizeof(CubeLookup) * m)) != Q1_OK) return st;
    if ((st = L->h_lookup.alloc(sizeof(CubeLookup) * m)) != Q1_OK) return st;
    if ((st = L->d_status.alloc(16)) != Q1_OK) return st;
    if ((st = L->h_status.alloc(16)) != Q1_OK) return st;
    Q1_CUDA(cudaMemset(L->d_status.p, 0, 16));
    *L->h_status.as<uint32_t>() = 0;
    return grow_items(L, 4096);
}

// Makes the request's table resident (or finds it) and pins it; false if it cannot be placed
// now because pinned tables hold the space. Dispatcher thread, lock held.
bool admit_table(q1_server* s, Ticket* t) {
    const TableKey k = key_of(t->req);
    auto it = s->cache.find(k);
    if (it != s->cache.end()) {
        it->second.pins++;
        it->second.last_use = ++s->lru_clock;
        t->table = &it->second;
        s->cache_hits++;
        return true;
    }
    const uint64_t need = TableLayout(k.rows).total;
    uint64_t off = 0;
    while (!s->arena.alloc(need, &off)) {
        // evict the least recently used table nobody reads
        auto victim = s->cache.end();
        for (auto c = s->cache.begin(); c != s->cache.end(); ++c)
            if (c->second.pins == 0 && (victim == s->cache.end() || c->second.last_use < victim->second.last_use))
                victim = c;
        if (victim == s->cache.end()) return false;
        s->arena.release(victim->second.off, victim->second.len);
        if (victim->second.gen_ev) cudaEventDestroy(victim->second.gen_ev);   // released once it completes
        s->cache.erase(victim);
        s->evictions++;
    }
    CachedTable& e = s->cache[k];
    e.off = off;
    e.len = need;
    e.pins = 1;
    e.last_use = ++s->lru_clock;
    e.ready = false;
    t->table = &e;
    s->cache_misses++;
    return true;
}

struct TablePtrs {
    uint8_t* base;
    TableLayout L;
};

TablePtrs table_ptrs(q1_server* s, const Ticket* t) {
    return TablePtrs{s->arena_mem.as<uint8_t>(t->table->off), TableLayout(t->req.adhoc_rows)};
}

// Generates the ticket's table on the lane's stream if it is not resident yet; a table that another
// lane generated is waited for through its event (a no-op once that generation has finished).
q1_status ensure_generated(q1_server* s, Ticket* t, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(s->m);
    CachedTable* tab = t->table;
    if (tab->ready) {
        if (tab->gen_ev && tab->gen_stream != st) Q1_CUDA(cudaStreamWaitEvent(st, tab->gen_ev, 0));
        return Q1_OK;
    }
    const TablePtrs tp = table_ptrs(s, t);
    uint8_t* tb = tp.base;
    const TableLayout& L = tp.L;
    KeyedTableOut o{reinterpret_cast<uint16_t*>(tb + L.off[0]), tb + L.off[2], reinterpret_cast<uint32_t*>(tb + L.off[4]),
                    tb + L.off[3], tb + L.off[1], reinterpret_cast<uint32_t*>(tb + L.off[5])};
    const bool flags = t->req.grouping == Q1_GROUP_FLAGS;
    Q1_CUDA(launch_generate_keyed_table(t->req.adhoc_seed, t->req.adhoc_rows, flags ? 1u : 0u, groups_of(t->req), o, st));
    if (!tab->gen_ev) Q1_CUDA(cudaEventCreateWithFlags(&tab->gen_ev, cudaEventDisableTiming));
    Q1_CUDA(cudaEventRecord(tab->gen_ev, st));
    tab->gen_stream = st;
    tab->ready = true;
    s->generated_rows += t->req.adhoc_rows;
    return Q1_OK;
}

// Enqueues one batched round for the lane's tickets on the lane's streams.
q1_status enqueue_round(q1_server* s, Lane* Ln) {
    const std::vector<Ticket*>& batch = Ln->batch;
    const uint32_t n = (uint32_t)batch.size();
    cudaStream_t st = Ln->stream;
    BatchInstanceDev* inst = Ln->h_inst.as<BatchInstanceDev>();
    uint64_t* base = Ln->h_base.as<uint64_t>();
    CubeLookup* look = Ln->h_lookup.as<CubeLookup>();
    uint32_t ninst = 0, nlook = 0;
    uint64_t groups = 0, tiles = 0;
    base[0] = 0;
    q1_status r;
    Q1_CUDA(cudaMemsetAsync(Ln->d_status.p, 0, 4, st));
    Q1_CUDA(cudaMemsetAsync(Ln->d_resp.p, 0, (uint64_t)n * kRespWords * 8, st));
    for (uint32_t i = 0; i < n; ++i) {
        Ticket* t = batch[i];
        const bool flags = t->req.grouping == Q1_GROUP_FLAGS;
        t->groups = groups_of(t->req);
        const int32_t cut = cutoff_rel(t->req.cutoff_day);
        if (t->req.kind == Q1_REQ_RESIDENT) {
            CubeLookup& l = look[nlook++];
            l.cube = (flags ? s->cube_pair : s->cube_key).as<unsigned long long>();
            l.day = cut < 0 ? -1 : std::min<int32_t>(cut, (int32_t)s->days - 1);
            l.num_groups = t->groups;
            l.slot = i;
            l.pad = 0;
            continue;
        }
        if ((r = ensure_generated(s, t, st)) != Q1_OK) return r;
        const TablePtrs tp = table_ptrs(s, t);
        BatchInstanceDev& d = inst[ninst];
        memset(&d, 0, sizeof(d));
        for (int c = 0; c < 6; ++c) d.col[c] = tp.base + tp.L.off[c];
        const uint32_t kg = key_groups(t->req);
        d.rows = t->req.adhoc_rows;
        d.cutoff = cut;
        d.num_groups = kg;
        d.mode = kg <= 4 ? kModeRegisters : kModeShared;
        d.acc = Ln->d_scratch.as<unsigned long long>() + 8 * groups;
        d.out = Ln->d_resp.as<unsigned long long>() + (uint64_t)i * kRespWords;
        groups += kg;
        base[ninst + 1] = groups;
        tiles += (d.rows + kBatchTileRows - 1) / kBatchTileRows;
        ++ninst;
    }
    if (ninst) {
        // work items: chunks of tiles grouped by engine, largest first; grid roles by engine cost
        const uint64_t chunk = std::max<uint64_t>(4, std::min<uint64_t>(1024, tiles / ((uint64_t)s->di->sm_count * 4)));
        std::vector<BatchItem> items;
        BatchParams prm{};
        batch_plan(inst, ninst, (uint32_t)chunk, (uint32_t)s->di->sm_count, items, prm);
        if ((r = grow_items(Ln, items.size())) != Q1_OK) return r;
        if (!items.empty()) {
            memcpy(Ln->h_items.p, items.data(), sizeof(BatchItem) * items.size());
            Q1_CUDA(cudaMemcpyAsync(Ln->d_items.p, Ln->h_items.p, sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice, st));
        }
        Q1_CUDA(cudaMemcpyAsync(Ln->d_inst.p, inst, sizeof(BatchInstanceDev) * ninst, cudaMemcpyHostToDevice, st));
        Q1_CUDA(cudaMemcpyAsync(Ln->d_base.p, base, sizeof(uint64_t) * (ninst + 1), cudaMemcpyHostToDevice, st));
        Q1_CUDA(cudaMemsetAsync(Ln->d_scratch.p, 0, groups * 64, st));
        if (!items.empty()) {
            Q1_CUDA(cudaMemsetAsync(Ln->d_cursor.p, 0, 4 * kEngines, st));
            prm.inst = Ln->d_inst.as<BatchInstanceDev>();
            prm.items = Ln->d_items.as<BatchItem>();
            prm.cursor = Ln->d_cursor.as<uint32_t>();
            prm.status = Ln->d_status.as<uint32_t>();
            Q1_CUDA(launch_batch(prm, prm.grid_regs, prm.grid_tables, st, Ln->aux, Ln->fork, Ln->join));
        }
        Q1_CUDA(launch_batch_finalize(Ln->d_inst.as<BatchInstanceDev>(), Ln->d_base.as<uint64_t>(), ninst, groups, st));
    }
    if (nlook) {
        Q1_CUDA(cudaMemcpyAsync(Ln->d_lookup.p, look, sizeof(CubeLookup) * nlook, cudaMemcpyHostToDevice, st));
        Q1_CUDA(launch_cube_lookup(Ln->d_lookup.as<CubeLookup>(), nlook, kRespWords, Ln->d_resp.as<unsigned long long>(), st));
    }
    Q1_CUDA(cudaMemcpyAsync(Ln->h_resp.p, Ln->d_resp.p, (uint64_t)n * kRespWords * 8, cudaMemcpyDeviceToHost, st));
    Q1_CUDA(cudaMemcpyAsync(Ln->h_status.p, Ln->d_status.p, 4, cudaMemcpyDeviceToHost, st));
    return Q1_OK;
}

// The plain launch of one request over device columns: the drop-in Q1 scan for the
// (returnflag, linestatus) grouping of pair-coded columns, else the group-key scan. Accumulates
// into `out` (caller-zeroed int128 [groups][6]).
q1_status plain_launch(const q1_request& req, const q1_compressed_columns& c, const uint32_t* keys, uint32_t G,
                       uint64_t rows, void* scratch, q1_i128* out, cudaStream_t sm) {
    if (c.flags && !keys)
        return q1_launch_compressed(Q1_PLACEMENT_IN_REGISTERS_PER_THREAD, &c, rows, req.cutoff_day, 0, nullptr, out, sm);
    return q1_launch_groupkey(G <= 8 ? Q1_PLACEMENT_IN_REGISTERS_PER_THREAD : Q1_PLACEMENT_SHARED_MEM_PER_THREAD, &c,
                              keys, G, rows, req.cutoff_day, nullptr, scratch, out, sm);
}

// Q1_SERVE_PLAIN: one request, one plain launch over the resident or cached table.
q1_status enqueue_plain(q1_server* s, Lane* Ln) {
    Ticket* t = Ln->batch[0];
    cudaStream_t st = Ln->stream;
    t->groups = groups_of(t->req);
    Q1_CUDA(cudaMemsetAsync(Ln->d_resp.p, 0, kRespWords * 8, st));
    q1_compressed_columns c{};
    const uint32_t* keys = nullptr;
    uint64_t rows = 0;
    q1_status r;
    if (t->req.kind == Q1_REQ_RESIDENT) {
        q1_server_resident_columns(s, &c, &keys, &rows);
        if (t->req.grouping == Q1_GROUP_FLAGS) keys = nullptr;
    } else {
        if ((r = ensure_generated(s, t, st)) != Q1_OK) return r;
        const TablePtrs tp = table_ptrs(s, t);
        c.shipdate = reinterpret_cast<const uint16_t*>(tp.base + tp.L.off[0]);
        c.quantity = tp.base + tp.L.off[1];
        c.discount = tp.base + tp.L.off[2];
        c.tax = tp.base + tp.L.off[3];
        c.extendedprice = reinterpret_cast<const uint32_t*>(tp.base + tp.L.off[4]);
        keys = reinterpret_cast<const uint32_t*>(tp.base + tp.L.off[5]);
        rows = t->req.adhoc_rows;
    }
    const uint32_t G = t->req.kind == Q1_REQ_RESIDENT ? t->groups : key_groups(t->req);
    if ((r = plain_launch(t->req, c, keys, G, rows, s->plain_scratch.p, Ln->d_resp.as<q1_i128>(), st)) != Q1_OK) return r;
    Q1_CUDA(cudaMemcpyAsync(Ln->h_resp.p, Ln->d_resp.p, (uint64_t)G * 12 * 8, cudaMemcpyDeviceToHost, st));
    return Q1_OK;
}

// Completer thread: waits for the lane's round, then answers its tickets. Rounds retire in the
// order they were enqueued; a round behind a failed one fails too (the device state is suspect).
void retire_round(q1_server* s, Lane* Ln) {
    const std::vector<Ticket*>& batch = Ln->batch;
    q1_status r = Ln->enq;
    std::string err = Ln->err;
    // drain the lane even after a failed enqueue, before any of its buffers is reused
    const cudaError_t se = cudaStreamSynchronize(Ln->stream);
    const cudaError_t sa = cudaStreamSynchronize(Ln->aux);
    if (r == Q1_OK && (se != cudaSuccess || sa != cudaSuccess)) {
        r = cuda_error(se != cudaSuccess ? se : sa, "serving round");
        err = q1_last_error();
    }
    if (r == Q1_OK) {
        if (s->opts.mode == Q1_SERVE_PLAIN) {
            // the plain launch reports through the device's status word (one lane in this mode)
            r = check_device_status(Ln->stream, s->di->status);
        } else {
            const uint32_t bits = *Ln->h_status.as<volatile uint32_t>();
            if (bits & 1u) r = set_error(Q1_ERR_DEVICE_TIMEOUT, "a bounded device-side wait expired");
            else if (bits & 4u) r = set_error(Q1_ERR_INTERNAL, "a device work buffer would have overflowed");
            else if (bits) r = set_error(Q1_ERR_DOMAIN, "a row is outside the kernels' domain");
        }
        if (r != Q1_OK) err = q1_last_error();
    }
    const double when = now_ms();
    const unsigned long long* words = Ln->h_resp.as<unsigned long long>();
    std::lock_guard<std::mutex> lk(s->m);
    if (r == Q1_OK && s->fatal != Q1_OK) {
        r = s->fatal;
        err = s->fatal_msg;
    }
    for (size_t i = 0; i < batch.size(); ++i) {
        Ticket* t = batch[i];
        if (r == Q1_OK) {
            const unsigned long long* src = words + i * kRespWords;
            t->aggs.assign((size_t)t->groups * 6, q1_i128{0, 0});
            if (coded(t->req)) {
                // table keys are dictionary codes: code c holds group kPairGroup[c]
                for (uint32_t c = 0; c < 4; ++c)
                    for (uint32_t a = 0; a < 6; ++a) {
                        t->aggs[kPairGroup[c] * 6 + a].lo = src[12 * c + 2 * a];
                        t->aggs[kPairGroup[c] * 6 + a].hi = src[12 * c + 2 * a + 1];
                    }
            } else {
                for (uint32_t w = 0; w < t->groups * 6; ++w) {
                    t->aggs[w].lo = src[2 * w];
                    t->aggs[w].hi = src[2 * w + 1];
                }
            }
        }
        if (t->table) {
            t->table->pins--;
            if (r != Q1_OK) t->table->ready = false;   // contents unknown after a failed round
            t->table = nullptr;
        }
        complete(s, t, r, when);
    }
    s->rounds++;
    if (r != Q1_OK && s->fatal == Q1_OK) {
        s->fatal = r;
        s->fatal_msg = err;
    }
    Ln->batch.clear();
    s->inflight.pop_front();
    s->free_lanes.push_back(Ln);
    s->cv_work.notify_all();
    s->cv_done.notify_all();
}

void completer_loop(q1_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        Lane* Ln;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_retire.wait(lk, [&] { return !s->inflight.empty() || s->dispatcher_done; });
            if (s->inflight.empty()) return;   // the dispatcher has stopped and every round retired
            Ln = s->inflight.front();
        }
        retire_round(s, Ln);
    }
}

void dispatcher_loop(q1_server* s) {
    cudaSetDevice(s->device);
    const uint32_t slots = s->opts.mode == Q1_SERVE_PLAIN ? 1u : s->opts.max_inflight;
    for (;;) {
        Lane* Ln = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return (s->stop && s->pending.empty()) || (!s->pending.empty() && !s->free_lanes.empty()); });
            if (s->pending.empty()) break;   // stop requested and the queue is drained
            if (s->fatal != Q1_OK) {
                // after a failed round the device state is suspect: fail what is queued
                const double when = now_ms();
                for (Ticket* t : s->pending) complete(s, t, s->fatal, when);
                s->pending.clear();
                s->cv_done.notify_all();
                continue;
            }
            Ln = s->free_lanes.front();
            // admit from the head while a slot is free and the next table is or can be resident
            while (!s->pending.empty() && Ln->batch.size() < slots) {
                Ticket* t = s->pending.front();
                if (t->req.kind == Q1_REQ_ADHOC && !admit_table(s, t)) break;   // with a later round
                t->t_admit = now_ms();
                Ln->batch.push_back(t);
                s->pending.pop_front();
            }
            if (Ln->batch.empty()) {
                // The head's table cannot be placed while running rounds pin the arena; with no
                // round running nothing is pinned and any table that submission accepted fits.
                if (s->inflight.empty()) {
                    Ticket* t = s->pending.front();
                    s->pending.pop_front();
                    complete(s, t, set_error(Q1_ERR_BUSY, "ad-hoc table does not fit the arena"), now_ms());
                    s->cv_done.notify_all();
                } else {
                    s->cv_work.wait(lk);   // until a round retires and unpins its tables
                }
                continue;
            }
            s->free_lanes.pop_front();
            s->admitted_total += Ln->batch.size();
            if (!s->inflight.empty()) s->overlapped_rounds++;
            s->max_in_flight = std::max<uint32_t>(s->max_in_flight, (uint32_t)s->inflight.size() + 1);
        }
        if (take_fault(kFaultServeRound))
            Ln->enq = set_error(Q1_ERR_INTERNAL, "injected serving round failure");
        else
            Ln->enq = s->opts.mode == Q1_SERVE_PLAIN ? enqueue_plain(s, Ln) : enqueue_round(s, Ln);
        Ln->err = Ln->enq == Q1_OK ? std::string() : std::string(q1_last_error());
        std::lock_guard<std::mutex> lk(s->m);
        s->inflight.push_back(Ln);
        s->cv_retire.notify_one();
    }
    std::lock_guard<std::mutex> lk(s->m);
    s->dispatcher_done = true;
    s->cv_retire.notify_one();
}

}  // namespace

extern "C" {

void q1_server_opts_default(q1_server_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->device = 0;
    o->max_inflight = 256;
    o->max_rounds_in_flight = 2;
    o->seed = 20260104;
    o->resident_rows = 600000000ull;
    o->hbm_budget_bytes = 120ull << 30;
    o->max_adhoc_rows = 100000000ull;
}

namespace {

// Device state of a server whose options are valid: streams, resident table and cubes, arena,
// lanes. On failure the caller closes the server, which releases whatever was made.
q1_status server_setup(q1_server* s) {
    s->device = s->opts.device;
    Q1_CUDA(cudaSetDevice(s->device));
    q1_status st = device_info(s->device, &s->di);
    if (st != Q1_OK) return st;
    Q1_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    Q1_CUDA(cudaStreamCreateWithFlags(&s->plain_stream, cudaStreamNonBlocking));
    Q1_CUDA(batch_prepare_launch());
    s->res_rows = s->opts.resident_rows;
    if ((st = build_resident(s)) != Q1_OK) return st;
    if ((st = s->arena_mem.alloc(s->opts.hbm_budget_bytes)) != Q1_OK) return st;
    s->arena.reset(s->opts.hbm_budget_bytes);
    const uint32_t nlanes = s->opts.mode == Q1_SERVE_PLAIN ? 1u : s->opts.max_rounds_in_flight;
    for (uint32_t i = 0; i < nlanes; ++i) {
        s->lanes.emplace_back(new Lane());
        if ((st = lane_open(s->lanes.back().get(), s->opts.max_inflight)) != Q1_OK) return st;
        s->free_lanes.push_back(s->lanes.back().get());
    }
    return s->plain_scratch.alloc(q1_groupkey_scratch_bytes(kMaxGroups));
}

}  // namespace

q1_status q1_server_open(const q1_server_opts* opts, q1_server** out) {
    if (!out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<q1_server> s(new q1_server());
    q1_server_opts_default(&s->opts);
    if (opts) s->opts = *opts;
    if (s->opts.max_inflight < 1 || s->opts.max_inflight > 65536)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "max_inflight must be in 1..65536");
    if (s->opts.max_rounds_in_flight == 0) s->opts.max_rounds_in_flight = 2;
    if (s->opts.max_rounds_in_flight > 8)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "max_rounds_in_flight must be in 0..8 (0 = 2)");
    if (s->opts.resident_rows > (1ull << 40)) return set_error(Q1_ERR_INVALID_ARGUMENT, "resident table too large");
    if (s->opts.max_adhoc_rows > (uint64_t)UINT32_MAX * kBatchTileRows)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "max_adhoc_rows too large");
    const q1_status st = server_setup(s.get());
    if (st != Q1_OK) {
        const std::string msg = q1_last_error();
        q1_server_close(s.release());   // streams, events and lanes made so far
        return set_error(st, msg);
    }
    s->completer = std::thread(completer_loop, s.get());
    s->dispatcher = std::thread(dispatcher_loop, s.get());
    *out = s.release();
    return Q1_OK;
}

q1_status q1_server_submit(q1_server* s, const q1_request* req, uint64_t* ticket) {
    if (!s || !req || !ticket) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    q1_status st = validate_request(req, s->opts.max_adhoc_rows, s->opts.hbm_budget_bytes);
    if (st != Q1_OK) return st;
    std::lock_guard<std::mutex> lk(s->m);
    if (s->fatal != Q1_OK) return set_error(s->fatal, "server stopped after an error: " + s->fatal_msg);
    if (s->stop) return set_error(Q1_ERR_BUSY, "server is closing");
    std::unique_ptr<Ticket> t(new Ticket());
    t->id = s->next_id++;
    t->req = *req;
    t->t_submit = now_ms();
    *ticket = t->id;
    s->pending.push_back(t.get());
    s->tickets[t->id] = std::move(t);
    s->cv_work.notify_one();
    return Q1_OK;
}

q1_status q1_server_wait(q1_server* s, uint64_t ticket, int32_t timeout_ms, q1_response* out) {
    if (!s || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return set_error(Q1_ERR_INVALID_ARGUMENT, "unknown ticket");
    Ticket* t = it->second.get();
    const auto pred = [&] { return t->done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, pred);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        return set_error(Q1_ERR_BUSY, "request not finished within the timeout");
    }
    memset(out, 0, sizeof(*out));
    out->ticket = t->id;
    out->status = t->status;
    out->num_groups = t->groups;
    out->latency_ms = t->t_done - t->t_submit;
    out->queue_ms = t->t_admit - t->t_submit;
    for (size_t w = 0; w < t->aggs.size() && w < (size_t)kMaxGroups * 6; ++w) out->aggregates[w] = t->aggs[w];
    const q1_status result = t->status;
    const std::string msg = s->fatal_msg;
    s->tickets.erase(it);
    if (result != Q1_OK) return set_error(result, "request failed: " + msg);
    return Q1_OK;
}

q1_status q1_server_stats_get(q1_server* s, q1_server_stats* out) {
    if (!s || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->m);
    memset(out, 0, sizeof(*out));
    out->completed = s->completed;
    out->failed = s->failed;
    out->rounds = s->rounds;
    out->pending = s->pending.size();
    out->logical_rows = s->logical_rows;
    out->scanned_rows = s->scanned_rows;
    out->generated_rows = s->generated_rows;
    out->cache_hits = s->cache_hits;
    out->cache_misses = s->cache_misses;
    out->evictions = s->evictions;
    out->cached_tables = s->cache.size();
    for (const auto& e : s->cache) out->cached_bytes += e.second.len;
    out->wall_ms = s->t_last > s->t_first ? s->t_last - s->t_first : 0;
    out->mean_round_size = s->rounds ? (double)s->admitted_total / (double)s->rounds : 0;
    out->overlapped_rounds = s->overlapped_rounds;
    out->max_rounds_in_flight = s->max_in_flight;
    std::vector<double> l = s->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        const auto pct = [&](double p) {
            return l[std::min<size_t>(l.size() - 1, (size_t)(p * (double)(l.size() - 1) + 0.5))];
        };
        out->p50_ms = pct(0.50);
        out->p90_ms = pct(0.90);
        out->p99_ms = pct(0.99);
        out->max_ms = l.back();
        double sum = 0;
        for (double v : l) sum += v;
        out->mean_ms = sum / (double)l.size();
    }
    return Q1_OK;
}

q1_status q1_server_reset_stats(q1_server* s) {
    if (!s) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->m);
    s->latencies.clear();
    s->rounds = s->completed = s->failed = s->logical_rows = s->scanned_rows = s->admitted_total = 0;
    s->generated_rows = s->cache_hits = s->cache_misses = s->evictions = 0;
    s->overlapped_rounds = 0;
    s->max_in_flight = 0;
    s->t_first = s->t_last = 0;
    return Q1_OK;
}

q1_status q1_server_plain(q1_server* s, const q1_request* req, q1_response* out) {
    if (!s || !req || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    q1_status st = validate_request(req, s->opts.max_adhoc_rows, UINT64_MAX);
    if (st != Q1_OK) return st;
    Q1_CUDA(cudaSetDevice(s->device));
    const bool flags = req->grouping == Q1_GROUP_FLAGS;
    const uint32_t G = groups_of(*req);
    std::lock_guard<std::mutex> jl(s->arbiter_m);
    if (!s->arbiter_out.p && (st = s->arbiter_out.alloc(kRespWords * 8)) != Q1_OK) return st;
    if (!s->arbiter_scratch.p && (st = s->arbiter_scratch.alloc(q1_groupkey_scratch_bytes(kMaxGroups))) != Q1_OK) return st;
    cudaStream_t sm = s->plain_stream;
    const double t0 = now_ms();
    Q1_CUDA(cudaMemsetAsync(s->arbiter_out.p, 0, kRespWords * 8, sm));
    q1_compressed_columns c{};
    const uint32_t* keys = nullptr;
    uint64_t rows = 0;
    if (req->kind == Q1_REQ_RESIDENT) {
        q1_server_resident_columns(s, &c, &keys, &rows);
        if (flags) keys = nullptr;
    } else {
        // a fresh table, independent of the served copy: pair-coded columns (the drop-in layout)
        // for the (returnflag, linestatus) grouping, else a keyed table
        rows = req->adhoc_rows;
        const TableLayout L(rows);
        if (L.total > s->arbiter_table.n) {
            if ((st = s->arbiter_table.alloc(TableLayout(s->opts.max_adhoc_rows).total)) != Q1_OK) return st;
        }
        uint8_t* tb = s->arbiter_table.as<uint8_t>();
        c.shipdate = reinterpret_cast<const uint16_t*>(tb + L.off[0]);
        c.quantity = tb + L.off[1];
        c.discount = tb + L.off[2];
        c.tax = tb + L.off[3];
        c.extendedprice = reinterpret_cast<const uint32_t*>(tb + L.off[4]);
        if (flags) {
            GenCompressedOut g{reinterpret_cast<uint16_t*>(tb + L.off[0]), tb + L.off[2],
                               reinterpret_cast<uint32_t*>(tb + L.off[4]), tb + L.off[3], tb + L.off[1],
                               reinterpret_cast<uint32_t*>(tb + L.off[5]), nullptr, nullptr};
            Q1_CUDA(launch_generate_compressed(req->adhoc_seed, 0, rows, g, sm));
            c.flags = reinterpret_cast<const uint32_t*>(tb + L.off[5]);
            c.flag_packing = Q1_FLAGS_PAIR_2BIT;
            c.num_pair_codes = 4;
            memcpy(c.pair_group, s->pair_group, 4);
        } else {
            KeyedTableOut o{reinterpret_cast<uint16_t*>(tb + L.off[0]), tb + L.off[2],
                            reinterpret_cast<uint32_t*>(tb + L.off[4]), tb + L.off[3], tb + L.off[1],
                            reinterpret_cast<uint32_t*>(tb + L.off[5])};
            Q1_CUDA(launch_generate_keyed_table(req->adhoc_seed, rows, 0u, G, o, sm));
            keys = reinterpret_cast<const uint32_t*>(tb + L.off[5]);
        }
    }
    if ((st = plain_launch(*req, c, keys, G, rows, s->arbiter_scratch.p, s->arbiter_out.as<q1_i128>(), sm)) != Q1_OK)
        return st;
    std::vector<unsigned long long> words((size_t)G * 12);
    Q1_CUDA(cudaMemcpyAsync(words.data(), s->arbiter_out.p, (size_t)G * 12 * 8, cudaMemcpyDeviceToHost, sm));
    if ((st = check_device_status(sm, s->di->status)) != Q1_OK) return st;
    memset(out, 0, sizeof(*out));
    out->status = Q1_OK;
    out->num_groups = G;
    out->latency_ms = now_ms() - t0;
    for (uint32_t w = 0; w < G * 6; ++w) {
        out->aggregates[w].lo = words[2 * w];
        out->aggregates[w].hi = words[2 * w + 1];
    }
    return Q1_OK;
}

q1_status q1_server_resident_columns(q1_server* s, q1_compressed_columns* cols, const uint32_t** keys, uint64_t* rows) {
    if (!s || !cols) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    memset(cols, 0, sizeof(*cols));
    cols->shipdate = s->res.as<uint16_t>(s->res_off[0]);
    cols->quantity = s->res.as<uint8_t>(s->res_off[1]);
    cols->discount = s->res.as<uint8_t>(s->res_off[2]);
    cols->tax = s->res.as<uint8_t>(s->res_off[3]);
    cols->extendedprice = s->res.as<uint32_t>(s->res_off[4]);
    cols->flags = s->res.as<uint32_t>(s->res_off[5]);
    cols->flag_packing = Q1_FLAGS_PAIR_2BIT;
    cols->num_pair_codes = 4;
    memcpy(cols->pair_group, s->pair_group, 4);
    if (keys) *keys = s->res.as<uint32_t>(s->res_off[6]);
    if (rows) *rows = s->res_rows;
    return Q1_OK;
}

q1_status q1_server_close(q1_server* s) {
    if (!s) return Q1_OK;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    else {
        std::lock_guard<std::mutex> lk(s->m);   // open failed before the dispatcher started
        s->dispatcher_done = true;
    }
    s->cv_retire.notify_all();
    if (s->completer.joinable()) s->completer.join();
    cudaSetDevice(s->device);
    s->lanes.clear();
    for (auto& e : s->cache)
        if (e.second.gen_ev) cudaEventDestroy(e.second.gen_ev);
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    if (s->plain_stream) {
        cudaStreamSynchronize(s->plain_stream);
        cudaStreamDestroy(s->plain_stream);
    }
    delete s;
    return Q1_OK;
}

}  // extern "C"
