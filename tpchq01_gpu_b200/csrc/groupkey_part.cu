// High-cardinality group-key aggregation for sm_100a (shared_mem_per_thread placement,
// num_groups > 4096, when the sample-based choice in groupkey_kernels.cu picks it): a radix
// partition of the passing rows by key, then one shared-memory slot table per partition.
//
// A shared-memory table holds at most a few thousand groups (9 words a group), and sending the
// other rows straight to global accumulators is bound by L2 atomic throughput (at G = 65,536 with
// uniform keys, 97% of the rows). Instead, per segment of at most 2^27 rows:
//
//   pass 1  q1_gk_partition_kernel: the 13 B/row tiles stream in exactly as in the group-key
//           kernel (cp.async.bulk into a 3-stage ring; 16 consumer warps). Every passing row in the tables' fast
//           domain becomes one 8-byte record (price 24 bits, quantity 8 | discount 4, tax 4,
//           key mod 4096 in 16 bits, valid bit) appended to the shared-memory ring of its
//           partition (key / 4096) owned by the consumer warp; each full run of 32 records
//           (256 B) is written to a chunk of a global pool, and the chunk's partition to a
//           directory. Chunks are reserved 16 at a time with one atomic whose result is consumed
//           only when the previous 16 are used up, so its latency is hidden. Rows outside the
//           fast domain reduce straight into the scratch accumulators, as in the group-key kernel.
//   lists   q1_gk_lists_kernel: directory -> chunk list per partition (counting sort; block-level
//           histograms, one global atomic per block and partition).
//   pass 2  q1_gk_partagg_kernel: the concatenated lists (partition by partition) are split
//           evenly over the CTAs and walked in stages of 128 chunks within one partition; every
//           thread loads its two quads of records (2 x 32 B) straight from the pool, one stage
//           ahead of the stage it adds into a 4096-slot table (ka::SlotTable) of the stage's
//           partition; the table is flushed into the scratch accumulators whenever the
//           partition changes. (256-byte chunks are too small for one bulk copy each: a TMA
//           producer left this pass short of data.)
//
// The arithmetic per row is the reference's (src/kernels/ht_in_global_mem.hpp:31-49), grouped
// by key; results are bit-identical to the single-pass placements.
#include <cuda_runtime.h>
#include <stdint.h>

#include "q1_common.cuh"
#include "q1_keyagg.cuh"
#include "q1_kernels.h"
#include "q1_ptx.cuh"

namespace q1 {

using namespace ptx;

namespace gp {

constexpr uint32_t kWidthLog = 12;
constexpr uint32_t kWidth = 1u << kWidthLog;     // keys per partition = pass-2 table slots
constexpr uint32_t kMaxParts = 16;               // 65,536 / 4096
constexpr uint32_t kChunk = 32;                  // records per chunk (256 B)
constexpr uint32_t kStageCap = 64;               // staged records per (warp, partition)
constexpr uint32_t kBatch = 16;                  // chunks reserved per pool atomic
constexpr uint32_t kNoPart = 0xFFFFFFFFu;
constexpr uint8_t kNoPartByte = 0xFF;
constexpr uint64_t kSegRows = 1ull << 27;        // rows per segment (bounds the pool)
constexpr uint32_t kMaxGrid = 256;               // CTAs per pass (bounds the pool's slack)

// pass 1
constexpr uint32_t kP1Warps = 16;
constexpr uint32_t kP1Stages = 3;
constexpr uint32_t kStagingBytes = kP1Warps * kMaxParts * kStageCap * 8;   // 128 KB
constexpr uint32_t kP1Smem = kP1Stages * ka::kStageBytes + kStagingBytes;
// pass 2
constexpr uint32_t kP2Warps = 16;
constexpr uint32_t kStageChunks = 128;                                     // 4096 records a stage
constexpr uint32_t kP2Smem = ka::kSlotWords * kWidth * 4;
static_assert(kP2Smem <= 227 * 1024, "pass-2 shared memory");
static_assert(kP1Smem <= 227 * 1024, "pass-1 shared memory");
static_assert(kStageChunks * kChunk / 4 % (kP2Warps * 32) == 0, "whole quads per thread per stage");

// Chunks a segment may reserve: full chunks, plus per warp one partial chunk per partition and
// at most two unused batches (the current one and the prefetched one).
constexpr uint64_t kPoolChunks = kSegRows / kChunk + (uint64_t)kMaxGrid * kP1Warps * (kMaxParts + 2 * kBatch);

struct Ctl {
    uint32_t pool_next;                // chunks reserved
    uint32_t part_chunks[kMaxParts];   // chunks written per partition
    uint32_t list_cursor[kMaxParts];   // list entries placed per partition
};

__host__ __device__ constexpr uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

// Workspace after the accumulators: ctl | dir (1 B a chunk) | lists (4 B a chunk) | pool.
constexpr uint64_t kOffDir = 256;
constexpr uint64_t kOffLists = kOffDir + align256(kPoolChunks);
constexpr uint64_t kOffPool = kOffLists + align256(4 * kPoolChunks);
constexpr uint64_t kWorkspaceBytes = kOffPool + kPoolChunks * kChunk * 8;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace gp

struct PartParams {
    const uint8_t* col[6];          // ship, qty, disc, tax, price, key (16-byte aligned)
    uint64_t rows;                  // rows of this segment (<= kSegRows)
    int32_t cutoff;                 // cutoff_day - 727563
    uint32_t num_groups;
    uint32_t parts;                 // ceil(num_groups / kWidth)
    uint32_t pool_cap;              // chunks
    unsigned long long* acc;        // scratch accumulators: num_groups x 8 u64
    uint32_t* status;
    const uint32_t* mode;           // when set, the kernels run only if *mode == kModePartitioned
    gp::Ctl* ctl;
    uint8_t* dir;
    uint32_t* lists;
    unsigned long long* pool;
};

// ---------------------------------------------------------------------------------------------
// Pass 1: partition
// ---------------------------------------------------------------------------------------------

// The consumer warp's staging state: per partition a 64-record ring in warp-private shared
// memory, filled at positions handed out by a shared atomic on the partition's tail counter
// (cheaper than a warp match plus one atomic per partition, even when skewed keys put most
// lanes in one partition). The lane whose record takes position 32j + 31 of a partition
// completes chunk j and has the warp write it out at once, so a ring never holds more than 31
// unwritten records between calls. Lane f (< kMaxParts) counts partition f's chunks.
struct Stager {
    unsigned long long* stage;      // [kMaxParts][kStageCap]
    uint32_t* tail;                 // [kMaxParts] records staged so far (shared)
    uint32_t chunks;                // lane f: chunks of partition f written
    uint32_t cur, end;              // current reserved batch [cur, end)
    uint32_t pre;                   // lane 0: first chunk of the prefetched batch
    uint32_t lane;

    // Writes the n <= 32 staged records of partition f from position h on (zero-padded) as one
    // chunk. All lanes call it with the same f, h, n.
    __device__ __forceinline__ void flush(uint32_t f, uint32_t h, uint32_t n, const PartParams& prm) {
        using namespace gp;
        if (cur == end) {
            cur = __shfl_sync(0xffffffffu, pre, 0);
            end = cur + kBatch;
            if (lane == 0) pre = atomicAdd(&prm.ctl->pool_next, kBatch);
        }
        const uint32_t c = cur++;
        const unsigned long long a = stage[f * kStageCap + ((h + lane) & (kStageCap - 1))];
        if (c < prm.pool_cap) {
            prm.pool[(uint64_t)c * kChunk + lane] = lane < n ? a : 0ull;
            if (lane == 0) prm.dir[c] = (uint8_t)f;
            if (lane == f) ++chunks;
        } else if (lane == 0 && prm.status) {
            atomicOr(prm.status, kStatusInternal);
        }
    }

    // One record per lane (part == kNoPart: none) into the rings; chunks completed are written
    // out. A call adds at most 32 records to a ring that held at most 31, so they fit in 64.
    __device__ __forceinline__ void add(uint32_t part, unsigned long long rec, const PartParams& prm) {
        using namespace gp;
        const bool v = part != kNoPart;
        uint32_t pos = 0;
        if (v) {
            pos = atomicAdd(&tail[part], 1u);
            stage[part * kStageCap + (pos & (kStageCap - 1))] = rec;
        }
        // positions of one partition in one call are consecutive: at most one completes a chunk
        uint32_t full = __ballot_sync(0xffffffffu, v && (pos & (kChunk - 1)) == kChunk - 1);
        if (full) {
            __syncwarp();
            do {
                const uint32_t l = __ffs(full) - 1;
                full &= full - 1;
                const uint32_t f = __shfl_sync(0xffffffffu, part, l);
                const uint32_t h = __shfl_sync(0xffffffffu, pos, l) - (kChunk - 1);
                flush(f, h, kChunk, prm);
            } while (full);
            __syncwarp();   // the ring slots just read are reused by later calls
        }
    }
};

// One quad: fast-domain rows become records; other passing rows with key < num_groups reduce
// into the scratch; passing rows with key >= num_groups set `bad`. All lanes call it.
__device__ __forceinline__ void partition_quad(Stager& sg, const ka::KeyQuad& x, const PartParams& prm,
                                               uint32_t& bad) {
    using namespace gp;
    const uint32_t G = prm.num_groups;
    // rows outside the fast domain: bit 7 of byte r set when d > 10, t > 8 or p >= 2^24
    const uint32_t top = __byte_perm(__byte_perm(x.p[0], x.p[1], 0x0073u), __byte_perm(x.p[2], x.p[3], 0x0073u),
                                     0x5410u);
    const uint32_t outside = (((top & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | top | ((x.D & 0x7F7F7F7Fu) + 0x75757575u) |
                              x.D | ((x.X & 0x7F7F7F7Fu) + 0x77777777u) | x.X) &
                             0x80808080u;
    const uint32_t inb = ((~outside & 0x80808080u) >> 7) * 0xFFu;
    const uint32_t DT = (x.D & inb) | ((x.X & inb) << 4);   // bytes r: d | t << 4 (in-domain rows)
    uint32_t part[4], slow = 0;
    unsigned long long rec[4];
    uint32_t fastb;   // byte r = 0xFF: row r becomes a record
    if (max(max(x.k[0], x.k[1]), max(x.k[2], x.k[3])) < G) {
        // every key of the quad in range: byte-parallel masks, the slow rows gathered to bits
        // 0..3 by one multiply (byte r's bit 0 lands on bit 24 + r)
        const uint32_t ob = (outside >> 7) * 0xFFu;
        fastb = x.PM & ~ob;
        slow = (((x.PM & ob) & 0x01010101u) * 0x01020408u) >> 24;
    } else {
        fastb = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t pass = (x.PM >> (8 * r)) & 1u;
            const uint32_t key = x.k[r];
            const uint32_t in = pass & (key < G ? 1u : 0u);
            bad |= pass & (key >= G ? 1u : 0u);
            const uint32_t fast = in & (((outside >> (8 * r + 7)) & 1u) ^ 1u);
            slow |= (in & (fast ^ 1u)) << r;
            fastb |= (fast * 0xFFu) << (8 * r);
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint32_t key = x.k[r];
        part[r] = (fastb >> (8 * r)) & 1u ? key >> kWidthLog : kNoPart;
        const uint32_t lo = __byte_perm(x.p[r], x.Q, 0x0210u | ((4u + (uint32_t)r) << 12));   // p | q << 24
        const uint32_t hi = ((DT >> (8 * r)) & 0xFFu) | ((key & (kWidth - 1)) << 8) | 0x80000000u;
        rec[r] = ((unsigned long long)hi << 32) | lo;
    }
    if (__any_sync(0xffffffffu, slow)) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if ((slow >> r) & 1u)
                ka::scratch_row(prm.acc, x.k[r], (x.Q >> (8 * r)) & 0xFFu, (x.D >> (8 * r)) & 0xFFu,
                                (x.X >> (8 * r)) & 0xFFu, x.p[r]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) sg.add(part[r], rec[r], prm);
}

__global__ void __launch_bounds__((gp::kP1Warps + 1) * 32, 1)
    q1_gk_partition_kernel(const __grid_constant__ PartParams prm) {
    using namespace gp;
    constexpr uint32_t W = kP1Warps, S = kP1Stages, R = ka::R, kStage = ka::kStageBytes;
    constexpr uint32_t kSteps = R / 4;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ uint32_t tail_s[W][kMaxParts];
    if (prm.mode && *prm.mode != kModePartitioned) return;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint64_t num_tiles = prm.rows / R;
    const uint32_t ring = smem_addr(smem);

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(smem_addr(&full_bar[s]), 1);
            mbar_init(smem_addr(&empty_bar[s]), W);
        }
        fence_mbar_init();
    }
    for (uint32_t i = threadIdx.x; i < W * kMaxParts; i += blockDim.x) (&tail_s[0][0])[i] = 0;
    __syncthreads();

    if (warp == W) {
        if (lane == 0) {
            const uint64_t pol = policy_evict_first();
            uint32_t k = 0;
            for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
                const uint32_t s = k % S;
                if (!mbar_wait(smem_addr(&empty_bar[s]), ((k / S) & 1u) ^ 1u, prm.status)) break;
                const uint32_t fb = smem_addr(&full_bar[s]);
                mbar_arrive_expect_tx(fb, kStage);
#pragma unroll
                for (int c = 0; c < 6; ++c)
                    bulk_g2s(ring + s * kStage + ka::col_off(c), prm.col[c] + t * (uint64_t)ka::col_bytes(c),
                             ka::col_bytes(c), fb, pol);
            }
            for (uint32_t i = (k > S ? k - S : 0u); i < k; ++i) mbar_wait(smem_addr(&full_bar[i % S]), (i / S) & 1u, prm.status);
        }
        return;
    }

    Stager sg;
    sg.stage = reinterpret_cast<unsigned long long*>(smem + S * kStage) + (uint64_t)warp * kMaxParts * kStageCap;
    sg.tail = tail_s[warp];
    sg.chunks = 0;
    sg.cur = sg.end = 0;
    sg.pre = 0;
    sg.lane = lane;
    if (lane == 0) sg.pre = atomicAdd(&prm.ctl->pool_next, kBatch);

    const uint32_t ctid = threadIdx.x;
    uint32_t bad = 0;
    bool ok = true;
    uint32_t k = 0;
    for (uint64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {
        const uint32_t s = k % S;
        const bool landed = mbar_wait(smem_addr(&full_bar[s]), (k / S) & 1u, prm.status);
        if (!__all_sync(0xffffffffu, landed)) {
            ok = false;
            break;
        }
        const uint32_t base = ring + s * kStage;
#pragma unroll
        for (uint32_t it = 0; it < kSteps / (W * 32); ++it)
            partition_quad(sg, ka::load_quad(base, ctid + it * (W * 32), prm.cutoff, bad), prm, bad);
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_addr(&empty_bar[s]));
    }
    // the rows after the last full tile, by one CTA straight from global memory
    if (ok && blockIdx.x == (uint32_t)(num_tiles % gridDim.x) && num_tiles * R < prm.rows) {
        for (uint64_t i0 = num_tiles * R; i0 < prm.rows; i0 += W * 32) {
            const uint64_t i = i0 + ctid;
            partition_quad(sg, i < prm.rows ? ka::load_row(prm.col, i, prm.cutoff, bad) : ka::empty_quad(), prm, bad);
        }
    }
    // partial chunks (full ones are written as they complete), then the reserved chunks left
    // unused
    __syncwarp();
    const uint32_t tl = lane < kMaxParts ? sg.tail[lane] : 0u;
    uint32_t left = __ballot_sync(0xffffffffu, lane < kMaxParts && (tl & (kChunk - 1)) != 0u);
    while (left) {
        const uint32_t f = __ffs(left) - 1;
        left &= left - 1;
        const uint32_t t = __shfl_sync(0xffffffffu, tl, f);
        sg.flush(f, t & ~(kChunk - 1), t & (kChunk - 1), prm);
    }
    const uint32_t p0 = __shfl_sync(0xffffffffu, sg.pre, 0);
    for (uint32_t c = sg.cur + lane; c < sg.end; c += 32)
        if (c < prm.pool_cap) prm.dir[c] = kNoPartByte;
    for (uint32_t c = p0 + lane; c < p0 + kBatch; c += 32)
        if (c < prm.pool_cap) prm.dir[c] = kNoPartByte;
    if (lane < kMaxParts && sg.chunks) atomicAdd(&prm.ctl->part_chunks[lane], sg.chunks);
    if (bad && prm.status) atomicOr(prm.status, kStatusDomain);
}

// ---------------------------------------------------------------------------------------------
// Lists: directory -> per-partition chunk lists, laid out partition after partition
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) q1_gk_lists_kernel(const __grid_constant__ PartParams prm) {
    using namespace gp;
    constexpr uint32_t kPer = 8, kTile = 256 * kPer;
    __shared__ uint32_t hist[kMaxParts], base[kMaxParts], off[kMaxParts];
    if (prm.mode && *prm.mode != kModePartitioned) return;
    const uint32_t tid = threadIdx.x;
    const uint32_t n = min(prm.ctl->pool_next, prm.pool_cap);
    if (tid == 0) {
        uint32_t o = 0;
        for (uint32_t p = 0; p < kMaxParts; ++p) {
            off[p] = o;
            o += p < prm.parts ? prm.ctl->part_chunks[p] : 0u;
        }
    }
    for (uint64_t t0 = (uint64_t)blockIdx.x * kTile; t0 < n; t0 += (uint64_t)gridDim.x * kTile) {
        if (tid < kMaxParts) hist[tid] = 0;
        __syncthreads();
        uint32_t f[kPer], rk[kPer];
#pragma unroll
        for (uint32_t j = 0; j < kPer; ++j) {
            const uint64_t i = t0 + j * 256 + tid;
            f[j] = i < n ? prm.dir[i] : kNoPart;
            rk[j] = 0;
            if (f[j] < prm.parts) rk[j] = atomicAdd(&hist[f[j]], 1u);
        }
        __syncthreads();
        if (tid < prm.parts && hist[tid]) base[tid] = off[tid] + atomicAdd(&prm.ctl->list_cursor[tid], hist[tid]);
        __syncthreads();
#pragma unroll
        for (uint32_t j = 0; j < kPer; ++j) {
            if (f[j] < prm.parts) {
                const uint32_t at = base[f[j]] + rk[j];
                if (at < prm.pool_cap) prm.lists[at] = (uint32_t)(t0 + j * 256 + tid);
                else if (prm.status) atomicOr(prm.status, kStatusInternal);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Pass 2: per-partition slot tables
// ---------------------------------------------------------------------------------------------

// The stage sequence of one CTA: [lo, hi) of the concatenated lists in runs of at most
// kStageChunks chunks that never cross a partition boundary. Producer and consumers walk it alike.
struct StageWalk {
    const uint32_t* off;            // [kMaxParts + 1] list offsets of the partitions (shared)
    uint32_t pos, hi, part;
    __device__ __forceinline__ void init(const uint32_t* off_s) {
        using namespace gp;
        off = off_s;
        const uint64_t T = off[kMaxParts];
        pos = (uint32_t)(T * blockIdx.x / gridDim.x);
        hi = (uint32_t)(T * (blockIdx.x + 1) / gridDim.x);
        part = 0;
    }
    // Next stage: partition and chunk count; false at the end.
    __device__ __forceinline__ bool next(uint32_t& p, uint32_t& first, uint32_t& n) {
        using namespace gp;
        if (pos >= hi) return false;
        while (part + 1 < kMaxParts && off[part + 1] <= pos) ++part;
        const uint32_t lim = min(hi, off[part + 1]);
        p = part;
        first = pos;
        n = min(kStageChunks, lim - pos);
        pos += n;
        return true;
    }
};

// 16 bytes of a chunk the previous kernel wrote (read-only here).
__device__ __forceinline__ uint4 ldg_nc_v4(const void* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// One stage of a CTA's walk and the thread's share of it: kQuads quads (4 records, 32 B each).
struct P2Stage {
    uint32_t p, first, n;
    bool ok;
};

__global__ void __launch_bounds__(gp::kP2Warps * 32, 1) q1_gk_partagg_kernel(const __grid_constant__ PartParams prm) {
    using namespace gp;
    constexpr uint32_t T = kP2Warps * 32;
    constexpr uint32_t kQuads = kStageChunks * (kChunk / 4) / T;   // quads per thread per stage
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint32_t off_s[kMaxParts + 1];
    if (prm.mode && *prm.mode != kModePartitioned) return;

    const uint32_t tid = threadIdx.x;
    ka::SlotTable slots;
    slots.bind(smem, kWidth);
    if (tid == 0) {
        uint32_t o = 0;
        for (uint32_t q = 0; q < kMaxParts; ++q) {
            off_s[q] = o;
            o += q < prm.parts ? prm.ctl->part_chunks[q] : 0u;
        }
        off_s[kMaxParts] = o;
    }
    slots.zero(tid, T);
    __syncthreads();

    StageWalk walk;
    walk.init(off_s);
    auto next = [&](P2Stage& st) { st.ok = walk.next(st.p, st.first, st.n); };
    // the chunk of quad h of this thread in stage st (kNoPart: none)
    auto chunk_of = [&](const P2Stage& st, uint32_t h) -> uint32_t {
        const uint32_t i = (tid + h * T) / (kChunk / 4);
        return (st.ok && i < st.n) ? prm.lists[st.first + i] : kNoPart;
    };
    auto load = [&](uint32_t c, uint32_t h, uint4& a, uint4& b) {
        a = make_uint4(0, 0, 0, 0);
        b = a;
        if (c < prm.pool_cap) {
            const unsigned long long* src = prm.pool + (uint64_t)c * kChunk + ((tid + h * T) % (kChunk / 4)) * 4;
            a = ldg_nc_v4(src);
            b = ldg_nc_v4(src + 2);
        } else if (c != kNoPart && prm.status) {
            atomicOr(prm.status, kStatusInternal);
        }
    };

    // software pipeline: records of stage k+1 and chunk ids of stage k+2 load while stage k adds
    P2Stage s0, s1, s2;
    next(s0);
    next(s1);
    next(s2);
    uint4 a0[kQuads], b0[kQuads], a1[kQuads], b1[kQuads];
    uint32_t c1[kQuads], c2[kQuads];
#pragma unroll
    for (uint32_t h = 0; h < kQuads; ++h) {
        load(chunk_of(s0, h), h, a0[h], b0[h]);
        c1[h] = chunk_of(s1, h);
    }
    uint32_t cur = kNoPart;
    uint64_t rows_since = 0;
    while (s0.ok) {
#pragma unroll
        for (uint32_t h = 0; h < kQuads; ++h) {
            load(c1[h], h, a1[h], b1[h]);
            c2[h] = chunk_of(s2, h);
        }
        if (s0.p != cur || rows_since + s0.n * kChunk > ka::kTableFlushRows) {
            if (cur != kNoPart) {
                __syncthreads();
                slots.flush(prm.acc + 8ull * cur * kWidth, tid, T);
                __syncthreads();
            }
            cur = s0.p;
            rows_since = 0;
        }
        rows_since += s0.n * kChunk;
#pragma unroll
        for (uint32_t h = 0; h < kQuads; ++h) {
            uint32_t m = 0, key[4], q[4], d[4], t[4], pr[4];
            const uint32_t lo[4] = {a0[h].x, a0[h].z, b0[h].x, b0[h].z};
            const uint32_t hw[4] = {a0[h].y, a0[h].w, b0[h].y, b0[h].w};
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                m |= (hw[r] >> 31) << r;
                pr[r] = lo[r] & 0xFFFFFFu;
                q[r] = lo[r] >> 24;
                d[r] = hw[r] & 0xFu;
                t[r] = (hw[r] >> 4) & 0xFu;
                key[r] = (hw[r] >> 8) & (kWidth - 1);
            }
            slots.add_quad(m, key, q, d, t, pr);
        }
        s0 = s1;
        s1 = s2;
        next(s2);
#pragma unroll
        for (uint32_t h = 0; h < kQuads; ++h) {
            a0[h] = a1[h];
            b0[h] = b1[h];
            c1[h] = c2[h];
        }
    }
    __syncthreads();
    if (cur != kNoPart) slots.flush(prm.acc + 8ull * cur * kWidth, tid, T);
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
uint64_t groupkey_part_workspace_bytes() { return gp::kWorkspaceBytes; }

uint32_t groupkey_part_min_groups() { return gp::kWidth + 1; }

uint64_t groupkey_part_mode_offset() { return 192; }
static_assert(sizeof(gp::Ctl) <= 192, "the mode word follows the control block");

cudaError_t launch_groupkey_part(const uint8_t* const cols[6], uint64_t rows, int32_t cutoff_rel,
                                 uint32_t num_groups, unsigned long long* acc, uint8_t* workspace,
                                 const uint32_t* mode, uint32_t* status, int sm_count, int max_blocks,
                                 cudaStream_t stream) {
    using namespace gp;
    if (num_groups > kWidth * kMaxParts) return cudaErrorInvalidValue;
    cudaError_t e =
        cudaFuncSetAttribute(q1_gk_partition_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP1Smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(q1_gk_partagg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2Smem);
    if (e != cudaSuccess) return e;
    uint32_t grid = (uint32_t)sm_count;
    if (max_blocks > 0 && (uint32_t)max_blocks < grid) grid = (uint32_t)max_blocks;
    if (grid > kMaxGrid) grid = kMaxGrid;
    if (grid < 1) grid = 1;
    PartParams prm{};
    prm.cutoff = cutoff_rel;
    prm.num_groups = num_groups;
    prm.parts = (num_groups + kWidth - 1) / kWidth;
    prm.pool_cap = (uint32_t)kPoolChunks;
    prm.acc = acc;
    prm.status = status;
    prm.mode = mode;
    prm.ctl = reinterpret_cast<Ctl*>(workspace);
    prm.dir = workspace + kOffDir;
    prm.lists = reinterpret_cast<uint32_t*>(workspace + kOffLists);
    prm.pool = reinterpret_cast<unsigned long long*>(workspace + kOffPool);
    const uint32_t bytes[6] = {2, 1, 1, 1, 4, 4};
    for (uint64_t off = 0; off < rows; off += kSegRows) {
        const uint64_t n = rows - off < kSegRows ? rows - off : kSegRows;
        for (int c = 0; c < 6; ++c) prm.col[c] = cols[c] + off * bytes[c];
        prm.rows = n;
        e = cudaMemsetAsync(prm.ctl, 0, sizeof(Ctl), stream);
        if (e != cudaSuccess) return e;
        const uint64_t tiles = n / ka::R;
        const uint32_t g1 = (uint32_t)(tiles == 0 ? 1 : (tiles < grid ? tiles : grid));
        q1_gk_partition_kernel<<<g1, (kP1Warps + 1) * 32, kP1Smem, stream>>>(prm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const uint64_t max_chunks = n / kChunk + (uint64_t)g1 * kP1Warps * (kMaxParts + 2 * kBatch);
        uint64_t gl = (max_chunks + 2047) / 2048;
        if (gl > 4ull * (uint64_t)sm_count) gl = 4ull * (uint64_t)sm_count;
        if (gl < 1) gl = 1;
        q1_gk_lists_kernel<<<(unsigned)gl, 256, 0, stream>>>(prm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        q1_gk_partagg_kernel<<<grid, kP2Warps * 32, kP2Smem, stream>>>(prm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace q1
