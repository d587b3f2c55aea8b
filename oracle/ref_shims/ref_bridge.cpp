// ref_bridge.cpp -- extern "C" access to the reference's own CPU kernels, built unmodified from
// the reference sources (cpu/common.cpp, cpu/monetdb.cpp, cpu/vectorized.cpp,
// cpu/kernel_hyper.hpp, cpu/kernel_x100.hpp). TEST INFRASTRUCTURE ONLY (the oracle's pin and
// the timed CPU baseline); the product never loads this library.
//
// Kernels exposed:
//   KernelHyPer<true>                    cpu/kernel_hyper.hpp:6-96 (tuple at a time, int128 sums)
//   KernelHyPerCompact<true>             cpu/kernel_hyper_compact.hpp (same loop, compact columns)
//   lineitem text values                 Decimal<15,2> / Char / Date (cpu/tpch_kit.hpp, .cpp)
//   KernelX100<kMagic,true,kNoAvx512>    cpu/kernel_x100.hpp:16-405 (vectorised, partial shuffle)
// The reference's own multi-threaded driver, Morsel<> (cpu/kernel_x100.hpp:423-665), returns
// from wait() before the last morsel and the per-thread merges have finished (it compares a
// floor-rounded morsel count, :586-590 / :479-483, and notifies only on the (n+1)-th
// completion), and can block forever when the row count is an exact multiple of the morsel
// size. The parallel entry point below therefore runs the same per-thread KernelX100::task()
// calls under a race-free pool of its own: an atomic morsel cursor, one kernel instance per
// thread, a join, then the per-thread tables summed (what Morsel::Query does at :456-500).
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include <sys/mman.h>

#include "../gen_rows.h"
#include "common.hpp"
#include "kernel_hyper.hpp"
#include "kernel_hyper_compact.hpp"
#include "vectorized.hpp"
#include "kernel_x100.hpp"

// Globals declared by src/cpu.h (defined in src/cpu.cpp, which also pulls in the GPU driver).
uint32_t* precomp_filter = nullptr;
uint16_t* compr_shipdate = nullptr;
moodycamel::BlockingConcurrentQueue<FilterChunk> precomp_filter_queue;
size_t morsel_size = 10 * 1024;

// Per-NUMA-node compact copy cache of cpu/common.cpp:142-172 (built from the first lineitem
// it sees); reset when the oracle switches to another table.
extern ComprData** numa_data;

// Same behaviour as cpu/vectorized.cpp:649-656, with the missing return added.
int Primitives::ordaggr_count(AggrHashTable* RESTRICT aggr0, idx_t* RESTRICT pos, idx_t* RESTRICT lim,
                              idx_t* RESTRICT grp, idx_t num_groups) {
    (void)pos;
    idx_t prev = 0;
    for (idx_t g = 0; g < num_groups; g++) {
        aggr0[grp[g]].count += lim[g] - prev;
        prev = lim[g];
    }
    return 0;
}

// handle_overflow() (cpu/common.cpp:7-11) asserts; calls from the kernels instantiated in this
// file are redirected here at link time (-Wl,--wrap=handle_overflow) and recorded instead.
static std::atomic<int> g_overflow{0};
extern "C" void __wrap_handle_overflow() { g_overflow.store(1); }

typedef __int128 i128;
enum { NG = 6, NA = 6 };

static const char kRf[3] = {'A', 'N', 'R'};
static const char kLs[2] = {'F', 'O'};

static void table_to_groups_hyper(const AggrHashTable* t, i128* out) {
    memset(out, 0, sizeof(i128) * NG * NA);
    for (int g = 0; g < NG; g++) {
        const char rf = kRf[g >> 1], ls = kLs[g & 1];
        const AggrHashTable& e = t[((idx_t)rf) << 8 | (idx_t)ls];  // cpu/kernel_hyper.hpp:76
        i128* o = out + g * NA;
        o[0] = e.count;
        o[1] = e.sum_quantity;
        o[2] = e.sum_base_price;
        o[3] = e.sum_disc;
        o[4] = e.sum_disc_price;
        o[5] = e.sum_charge;
    }
}

// Group id of map_gid2_dom_restrict (cpu/vectorized.cpp:512-535) for one (rf, ls) pair.
static idx_t x100_gid(const lineitem& li, char rf, char ls) {
    const int8_t min_a = (int8_t)li.l_returnflag.minmax.min;
    const int8_t max_b = (int8_t)li.l_linestatus.minmax.max;
    const int8_t min_b = (int8_t)li.l_linestatus.minmax.min;
    const uint8_t d = max_b - min_b;
    const int8_t a = (int8_t)rf, b = (int8_t)ls;
    if (min_a) {
        if (min_b) return ((uint8_t)(a - (uint8_t)min_a)) * d + ((uint8_t)(b - (uint8_t)min_b));
        return ((uint8_t)(a - (uint8_t)min_a)) * d + (uint8_t)b;
    }
    if (min_b) return a * d + (uint8_t)(b - (uint8_t)min_b);
    return a * d + b;
}

// x100 sums disc_1 = 100 - disc (cpu/kernel_x100.hpp:302), HyPer sums disc; map to sum(disc).
// present_mask selects the groups that occur; returns -1 if two present groups share a gid.
static int table_to_groups_x100(const lineitem& li, const AggrHashTable* t, unsigned present_mask, i128* out) {
    memset(out, 0, sizeof(i128) * NG * NA);
    idx_t gids[NG];
    for (int g = 0; g < NG; g++) gids[g] = x100_gid(li, kRf[g >> 1], kLs[g & 1]);
    for (int g = 0; g < NG; g++) {
        if (!(present_mask >> g & 1)) continue;
        for (int h = g + 1; h < NG; h++)
            if ((present_mask >> h & 1) && gids[g] == gids[h]) return -1;
        const AggrHashTable& e = t[gids[g]];
        i128* o = out + g * NA;
        o[0] = e.count;
        o[1] = e.sum_quantity;
        o[2] = e.sum_base_price;
        o[3] = (i128)100 * e.count - e.sum_disc;
        o[4] = e.sum_disc_price;
        o[5] = e.sum_charge;
    }
    return 0;
}

struct RefTable {
    lineitem li;
    unsigned present_mask = 0;
    explicit RefTable(size_t cap) : li(cap) {}
};

static std::mutex g_compact_mutex;
static const lineitem* g_compact_owner = nullptr;

static void use_compact_copy_of(const lineitem& li) {
    std::lock_guard<std::mutex> lk(g_compact_mutex);
    if (g_compact_owner != &li) {
        if (numa_data) numa_data[0] = nullptr;  // the old copy is leaked (IKernel never frees)
        g_compact_owner = &li;
    }
}

using X100 = KernelX100<kMagic, true, kNoAvx512>;

extern "C" {

void* q1ref_table_new(uint64_t capacity) { return new RefTable(capacity ? capacity : 1); }

void q1ref_table_free(void* t) {
    RefTable* r = (RefTable*)t;
    {
        std::lock_guard<std::mutex> lk(g_compact_mutex);
        if (g_compact_owner == &r->li) {
            if (numa_data) numa_data[0] = nullptr;
            g_compact_owner = nullptr;
        }
    }
    delete r;
}

// Appends rows. The reference kernels have the cutoff fixed at 1998-09-02 (cpu/common.cpp:60);
// a different cutoff c is applied by shifting every ship date by (729999 - c), which leaves
// the predicate's outcome unchanged.
int q1ref_table_push(void* t, const int32_t* shipdate, const int64_t* discount, const int64_t* extprice,
                     const int64_t* tax, const int64_t* quantity, const char* returnflag, const char* linestatus,
                     uint64_t n, int32_t cutoff_day) {
    RefTable* r = (RefTable*)t;
    const int32_t shift = 729999 - cutoff_day;
    for (uint64_t i = 0; i < n; i++) {
        r->li.l_shipdate.Push(shipdate[i] + shift);
        r->li.l_discount.Push(discount[i]);
        r->li.l_extendedprice.Push(extprice[i]);
        r->li.l_tax.Push(tax[i]);
        r->li.l_quantity.Push(quantity[i]);
        r->li.l_returnflag.Push(returnflag[i]);
        r->li.l_linestatus.Push(linestatus[i]);
        const unsigned rf = ((returnflag[i] == 'R') ? 2u : 0u) + ((returnflag[i] == 'N') ? 1u : 0u);
        const unsigned ls = (linestatus[i] == 'F') ? 0u : 1u;
        r->present_mask |= 1u << ((rf << 1) + ls);
    }
    return 0;
}

uint64_t q1ref_table_rows(void* t) { return ((RefTable*)t)->li.l_extendedprice.cardinality; }

// Appends rows [first_row, first_row + n) of the seeded generator (oracle/gen_rows.h), pushed one
// value at a time like q1ref_table_push, with the same cutoff shift. No product code is involved.
int q1ref_table_generate(void* t, uint64_t seed, uint64_t first_row, uint64_t n, int32_t cutoff_day) {
    RefTable* r = (RefTable*)t;
    const int32_t shift = 729999 - cutoff_day;
    const uint64_t key = og_key(seed);
    for (uint64_t i = 0; i < n; i++) {
        int32_t ship;
        int64_t qty, price, disc, tax;
        char rf, ls;
        og_row(key, first_row + i, &ship, &qty, &price, &disc, &tax, &rf, &ls);
        r->li.l_shipdate.Push(ship + shift);
        r->li.l_discount.Push(disc);
        r->li.l_extendedprice.Push(price);
        r->li.l_tax.Push(tax);
        r->li.l_quantity.Push(qty);
        r->li.l_returnflag.Push(rf);
        r->li.l_linestatus.Push(ls);
        const unsigned rfc = ((rf == 'R') ? 2u : 0u) + ((rf == 'N') ? 1u : 0u);
        r->present_mask |= 1u << ((rfc << 1) + (ls == 'F' ? 0u : 1u));
    }
    return 0;
}

// KernelHyPer<true> over the whole table. out: [6][6] int128. Returns 1 on int64 overflow.
int q1ref_hyper(void* t, i128* out) {
    RefTable* r = (RefTable*)t;
    g_overflow.store(0);
    KernelHyPer<true> k(r->li);
    k.Clear();
    k();
    table_to_groups_hyper(k.aggrs0, out);
    return g_overflow.load();
}

// KernelHyPerCompact<true> (cpu/kernel_hyper_compact.hpp): HyPer's tuple-at-a-time loop over the
// int8/int16/int32 compact copy (ComprData, cpu/common.cpp:113-137). Built with -DGPU (as the
// reference's GPU binary is), the compact ship date is ship - 727563 while this kernel compares it
// with the int16 truncation of the cutoff day (729999 -> 9103), so the table must be pushed with
// cutoff_day - 6667 to evaluate Q1's predicate. out: [6][6] int128. Returns 1 on overflow.
int q1ref_hyper_compact(void* t, i128* out) {
    RefTable* r = (RefTable*)t;
    use_compact_copy_of(r->li);
    g_overflow.store(0);
    KernelHyPerCompact<true> k(r->li, 0);
    k.Clear();
    k();
    table_to_groups_hyper(k.aggrs0, out);
    return g_overflow.load();
}

// KernelX100<kMagic,true,kNoAvx512>::task(offset, num) on one thread. Returns -1 if the x100
// group-id map cannot tell two present groups apart.
int q1ref_x100(void* t, uint64_t offset, uint64_t num, i128* out) {
    RefTable* r = (RefTable*)t;
    use_compact_copy_of(r->li);
    X100 k(r->li, 0);
    k.Clear();
    if (num) k.task(offset, num);
    return table_to_groups_x100(r->li, k.aggrs0, r->present_mask, out);
}

// Persistent pool of KernelX100 instances (one per thread), morsel-driven.
struct X100Pool {
    RefTable* table;
    std::vector<std::thread> workers;
    std::vector<X100*> kernels;
    std::mutex m;
    std::condition_variable cv_start, cv_done;
    uint64_t generation = 0;
    int running = 0;
    bool stop = false;
    uint64_t begin = 0, end = 0, morsel = 1 << 16;
    std::atomic<uint64_t> cursor{0};

    void work(int id) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m);
                cv_start.wait(lk, [&] { return stop || generation != seen; });
                if (stop) return;
                seen = generation;
            }
            X100* k = kernels[id];
            for (;;) {
                const uint64_t off = cursor.fetch_add(morsel);
                if (off >= end) break;
                const uint64_t n = (end - off < morsel) ? end - off : morsel;
                k->task(off, n);
            }
            {
                std::lock_guard<std::mutex> lk(m);
                if (--running == 0) cv_done.notify_all();
            }
        }
    }
};

void* q1ref_pool_new(void* t, int threads) {
    RefTable* r = (RefTable*)t;
    use_compact_copy_of(r->li);
    if (threads < 1) threads = 1;
    X100Pool* p = new X100Pool();
    p->table = r;
    for (int i = 0; i < threads; i++) p->kernels.push_back(new X100(r->li, 0));
    for (int i = 0; i < threads; i++) p->workers.emplace_back(&X100Pool::work, p, i);
    return p;
}

// Aggregates rows [offset, offset+num) on all pool threads. out: [6][6] int128.
int q1ref_pool_run(void* pool, uint64_t offset, uint64_t num, uint64_t morsel, i128* out) {
    X100Pool* p = (X100Pool*)pool;
    for (X100* k : p->kernels) k->Clear();
    {
        std::unique_lock<std::mutex> lk(p->m);
        p->begin = offset;
        p->end = offset + num;
        p->morsel = morsel ? morsel : (1 << 16);
        p->cursor.store(offset);
        p->running = (int)p->workers.size();
        p->generation++;
        p->cv_start.notify_all();
        p->cv_done.wait(lk, [&] { return p->running == 0; });
    }
    // Sum the per-thread tables (Morsel::Query's merge, cpu/kernel_x100.hpp:485-496).
    std::vector<AggrHashTable> sum(MAX_GROUPS);
    memset(sum.data(), 0, sizeof(AggrHashTable) * MAX_GROUPS);
    for (X100* k : p->kernels) {
        for (size_t g = 0; g < MAX_GROUPS; g++) {
            const AggrHashTable& e = k->aggrs0[g];
            if (!e.count) continue;
            sum[g].sum_quantity += e.sum_quantity;
            sum[g].count += e.count;
            sum[g].sum_base_price += e.sum_base_price;
            sum[g].sum_disc += e.sum_disc;
            sum[g].sum_disc_price += e.sum_disc_price;
            sum[g].sum_charge += e.sum_charge;
        }
    }
    return table_to_groups_x100(p->table->li, sum.data(), p->table->present_mask, out);
}

int q1ref_pool_threads(void* pool) { return (int)((X100Pool*)pool)->workers.size(); }

// lineitem text through the reference's own value types: each line is split at '|' the way
// TableReader::tokenize does (cpu/tpch_kit.cpp:26-57; restated here because tpch_kit.cpp also
// holds the boost-based parsers), and fields 5-11 are converted by the reference's
// Decimal<15,2>, Char and Date constructors (cpu/tpch_kit.hpp:15-80, cpu/tpch_kit.cpp:142-153)
// exactly as lineitem::FromFile pushes them (cpu/tpch_kit.cpp:155-172). Only for well-formed
// text: the reference asserts on anything else. Returns the rows parsed.
uint64_t q1ref_parse_tbl(const char* text, uint64_t bytes, int32_t* ship, int64_t* qty, int64_t* price,
                         int64_t* disc, int64_t* tax, char* rf, char* ls, uint64_t capacity) {
    std::vector<char> line;
    uint64_t row = 0, start = 0;
    while (start < bytes && row < capacity) {
        uint64_t end = start;
        while (end < bytes && text[end] != '\n') ++end;
        line.assign(text + start, text + end);
        line.push_back('\0');
        const char* w[11];
        int64_t len[11];
        int nw = 0;
        int64_t ws = 0;
        for (int64_t i = 0; nw < 11; ++i) {
            const char c = line[i];
            if (c == '|' || c == '\0') {
                w[nw] = &line[ws];
                len[nw] = i - ws;
                line[i] = '\0';
                ws = i + 1;
                ++nw;
                if (c == '\0') break;
            }
        }
        if (nw < 11) break;
        qty[row] = Decimal<15, 2>(w[4], len[4]).dec_val;
        price[row] = Decimal<15, 2>(w[5], len[5]).dec_val;
        disc[row] = Decimal<15, 2>(w[6], len[6]).dec_val;
        tax[row] = Decimal<15, 2>(w[7], len[7]).dec_val;
        rf[row] = Char(w[8], len[8]).chr_val;
        ls[row] = Char(w[9], len[9]).chr_val;
        ship[row] = Date(w[10], len[10]).dte_val;
        ++row;
        start = end + 1;
    }
    return row;
}

void q1ref_pool_free(void* pool) {
    X100Pool* p = (X100Pool*)pool;
    {
        std::lock_guard<std::mutex> lk(p->m);
        p->stop = true;
        p->cv_start.notify_all();
    }
    for (auto& w : p->workers) w.join();
    for (X100* k : p->kernels) delete k;
    delete p;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// KernelX100 over a table too large for the reference's int64 lineitem in one piece (600 M rows
// take 23 GB there). The rows are generated in chunks, each into its own lineitem, and
// ComprData::Get (cpu/common.cpp:155-174) builds that chunk's compact int8/int16/int32 copy: the
// only column data KernelX100::task reads (its scan() pointers are the l_* members that
// kernel_compact_init sets, cpu/kernel_x100.hpp:44, :154-173; the lineitem itself supplies only
// the flags' MinMax for the group-id map, :223-224). The chunk's wide pages are then handed back
// to the OS (madvise; the mapping stays valid), so the whole table costs 12 B/row. A run clears
// one KernelX100 per thread once, points every kernel's seven compact-column pointers at chunk c,
// runs chunk c's morsels on all threads, and so on over the chunks; the per-thread tables are
// then summed as in q1ref_pool_run. Every kernel keeps chunk 0's lineitem for the group-id map,
// after its flag MinMax are widened to the whole table's (the union of the chunks'), which is
// what one lineitem holding every row would carry.
// ---------------------------------------------------------------------------------------------

// IKernel never frees what new_array allocated (cpu/common.cpp:104-111: `m_clean && false`);
// these release the arrays the bridge knows by name (all aligned_alloc'ed).
static void free_base_arrays(BaseKernel* k) {
    void* arrays[] = {k->aggrs0, k->aggr_dsm0_sum_quantity, k->aggr_dsm0_count, k->aggr_dsm0_sum_base_price,
                      k->aggr_dsm0_sum_disc_price, k->aggr_dsm0_sum_charge, k->aggr_dsm0_sum_disc,
                      k->aggr_avx0_count, k->aggr_avx0_sum_quantity, k->aggr_avx0_sum_base_price,
                      k->aggr_avx0_sum_disc_price_lo, k->aggr_avx0_sum_disc_price_hi, k->aggr_avx0_sum_charge_lo,
                      k->aggr_avx0_sum_charge_hi, k->aggr_avx0_sum_disc};
    for (void* a : arrays) free(a);
}

static void free_compact(ComprData* d) {
    void* arrays[] = {d->l_shipdate, d->l_returnflag, d->l_linestatus, d->l_discount, d->l_tax, d->l_extendedprice,
                      d->l_quantity};
    for (void* a : arrays) free(a);
    free_base_arrays(d);
    delete d;
}

template <typename T>
static void drop_pages(Column<T>& c) {
    madvise(c.m_ptr, c.m_alloc_size, MADV_DONTNEED);
}

static void point_at(X100* k, const ComprData* d) {
    k->l_shipdate = d->l_shipdate;
    k->l_returnflag = d->l_returnflag;
    k->l_linestatus = d->l_linestatus;
    k->l_discount = d->l_discount;
    k->l_tax = d->l_tax;
    k->l_extendedprice = d->l_extendedprice;
    k->l_quantity = d->l_quantity;
}

struct RefChunks {
    std::vector<RefTable*> chunks;
    std::vector<ComprData*> comp;
    std::vector<X100*> kernels;
    std::vector<std::thread> workers;
    std::mutex m;
    std::condition_variable cv_start, cv_done;
    uint64_t generation = 0;
    int running = 0;
    bool stop = false;
    uint64_t end = 0, morsel = 1 << 16;
    std::atomic<uint64_t> cursor{0};
    unsigned present_mask = 0;

    void work(int id) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m);
                cv_start.wait(lk, [&] { return stop || generation != seen; });
                if (stop) return;
                seen = generation;
            }
            X100* k = kernels[id];
            for (;;) {
                const uint64_t off = cursor.fetch_add(morsel);
                if (off >= end) break;
                k->task(off, (end - off < morsel) ? end - off : morsel);
            }
            {
                std::lock_guard<std::mutex> lk(m);
                if (--running == 0) cv_done.notify_all();
            }
        }
    }
};

extern "C" {

// Rows [first_row, first_row + rows) of the seeded generator in chunks of chunk_rows, the
// predicate's cutoff applied by the ship-date shift of q1ref_table_push, `threads` workers.
// Returns NULL when rows is 0.
void* q1ref_chunks_new(uint64_t seed, uint64_t first_row, uint64_t rows, uint64_t chunk_rows, int32_t cutoff_day,
                       int threads) {
    if (!rows) return nullptr;
    if (threads < 1) threads = 1;
    if (!chunk_rows) chunk_rows = 1ull << 24;
    RefChunks* h = new RefChunks();
    const uint64_t nchunks = (rows + chunk_rows - 1) / chunk_rows;
    h->chunks.assign(nchunks, nullptr);
    h->comp.assign(nchunks, nullptr);
    std::atomic<uint64_t> next{0};
    auto build = [&]() {
        for (;;) {
            const uint64_t c = next.fetch_add(1);
            if (c >= nchunks) return;
            const uint64_t first = c * chunk_rows;
            const uint64_t n = (rows - first < chunk_rows) ? rows - first : chunk_rows;
            RefTable* t = new RefTable(n + 1);
            q1ref_table_generate(t, seed, first_row + first, n, cutoff_day);
            {
                std::lock_guard<std::mutex> lk(g_compact_mutex);
                if (numa_data) numa_data[0] = nullptr;
                h->comp[c] = ComprData::Get(t->li, 0);
                numa_data[0] = nullptr;
                g_compact_owner = nullptr;
            }
            drop_pages(t->li.l_shipdate);
            drop_pages(t->li.l_discount);
            drop_pages(t->li.l_extendedprice);
            drop_pages(t->li.l_tax);
            drop_pages(t->li.l_quantity);
            drop_pages(t->li.l_returnflag);
            drop_pages(t->li.l_linestatus);
            h->chunks[c] = t;
        }
    };
    // at most 8 chunks in their wide form at once
    const int builders = (int)std::min<uint64_t>(std::min(threads, 8), nchunks);
    std::vector<std::thread> bt;
    for (int i = 0; i < builders; i++) bt.emplace_back(build);
    for (auto& t : bt) t.join();
    // chunk 0's lineitem, which the kernels keep, takes the flags' MinMax of the whole table
    lineitem& li0 = h->chunks[0]->li;
    for (RefTable* t : h->chunks) {
        h->present_mask |= t->present_mask;
        const lineitem& li = t->li;
        li0.l_returnflag.minmax.min = std::min(li0.l_returnflag.minmax.min, li.l_returnflag.minmax.min);
        li0.l_returnflag.minmax.max = std::max(li0.l_returnflag.minmax.max, li.l_returnflag.minmax.max);
        li0.l_linestatus.minmax.min = std::min(li0.l_linestatus.minmax.min, li.l_linestatus.minmax.min);
        li0.l_linestatus.minmax.max = std::max(li0.l_linestatus.minmax.max, li.l_linestatus.minmax.max);
    }
    {
        std::lock_guard<std::mutex> lk(g_compact_mutex);
        ComprData* saved = numa_data[0];   // numa_data exists: ComprData::Get created it above
        numa_data[0] = h->comp[0];   // the kernels' constructors take this copy (kernel_compact_init)
        for (int i = 0; i < threads; i++) h->kernels.push_back(new X100(li0, 0));
        numa_data[0] = saved;
    }
    for (int i = 0; i < threads; i++) h->workers.emplace_back(&RefChunks::work, h, i);
    return h;
}

// KernelX100 over every chunk on all threads. out: [6][6] int128. Returns -1 if the x100 group-id
// map cannot tell two present groups apart.
int q1ref_chunks_run(void* hh, uint64_t morsel, i128* out) {
    RefChunks* h = (RefChunks*)hh;
    for (X100* k : h->kernels) k->Clear();
    for (size_t c = 0; c < h->chunks.size(); c++) {
        for (X100* k : h->kernels) point_at(k, h->comp[c]);
        std::unique_lock<std::mutex> lk(h->m);
        h->end = h->chunks[c]->li.l_extendedprice.cardinality;
        h->morsel = morsel ? morsel : (1 << 16);
        h->cursor.store(0);
        h->running = (int)h->workers.size();
        h->generation++;
        h->cv_start.notify_all();
        h->cv_done.wait(lk, [&] { return h->running == 0; });
    }
    std::vector<AggrHashTable> sum(MAX_GROUPS);
    memset(sum.data(), 0, sizeof(AggrHashTable) * MAX_GROUPS);
    for (X100* k : h->kernels) {
        for (size_t g = 0; g < MAX_GROUPS; g++) {
            const AggrHashTable& e = k->aggrs0[g];
            if (!e.count) continue;
            sum[g].sum_quantity += e.sum_quantity;
            sum[g].count += e.count;
            sum[g].sum_base_price += e.sum_base_price;
            sum[g].sum_disc += e.sum_disc;
            sum[g].sum_disc_price += e.sum_disc_price;
            sum[g].sum_charge += e.sum_charge;
        }
    }
    return table_to_groups_x100(h->chunks[0]->li, sum.data(), h->present_mask, out);
}

int q1ref_chunks_threads(void* hh) { return (int)((RefChunks*)hh)->workers.size(); }

uint64_t q1ref_chunks_count(void* hh) { return ((RefChunks*)hh)->chunks.size(); }

void q1ref_chunks_free(void* hh) {
    RefChunks* h = (RefChunks*)hh;
    {
        std::lock_guard<std::mutex> lk(h->m);
        h->stop = true;
        h->cv_start.notify_all();
    }
    for (auto& w : h->workers) w.join();
    for (X100* k : h->kernels) {
        free_base_arrays(k);
        delete k;
    }
    for (ComprData* d : h->comp) free_compact(d);
    for (RefTable* t : h->chunks) delete t;
    delete h;
}

}  // extern "C"
