// lineitem text (dbgen .tbl) ingestion: the reference's load path when no column cache exists
// (src/main.cu:441-475: lineitem::FromFile, cpu/tpch_kit.cpp:155-172), with the parse on the GPU
// (tbl_kernels.cu), and the inverse, writing host columns as .tbl text.
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "q1.h"
#include "q1_internal.h"
#include "q1_kernels.h"

using namespace q1;

namespace {

// A stream-ordered memory pool per device that keeps what it frees (the default pool hands freed
// memory back at every synchronisation, so each call would map its scratch afresh).
cudaError_t scratch_pool(cudaMemPool_t* pool) {
    static std::mutex m;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(m);
    if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return e;
        uint64_t keep = ~0ull;
        if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
        pools[dev] = p;
    }
    *pool = pools[dev];
    return cudaSuccess;
}

struct DeviceMem {
    void* p = nullptr;
    cudaStream_t st = nullptr;   // set: stream-ordered allocation (no device-wide sync on free)
    ~DeviceMem() {
        if (p) {
            if (st) cudaFreeAsync(p, st);
            else cudaFree(p);
        }
    }
    q1_status alloc_async(uint64_t bytes, cudaStream_t stream) {
        if (take_fault(kFaultDeviceAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected device allocation failure");
        cudaMemPool_t pool = nullptr;
        if (scratch_pool(&pool) != cudaSuccess || cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, pool, stream) != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return set_error(Q1_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
        st = stream;
        return Q1_OK;
    }
    q1_status alloc(uint64_t bytes) {
        if (take_fault(kFaultDeviceAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected device allocation failure");
        if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return set_error(Q1_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
        return Q1_OK;
    }
};

struct PinnedMem {
    void* p = nullptr;
    ~PinnedMem() {
        if (p) cudaFreeHost(p);
    }
    q1_status alloc(uint64_t bytes) {
        if (take_fault(kFaultPinnedAlloc)) return set_error(Q1_ERR_OUT_OF_MEMORY, "injected pinned allocation failure");
        if (cudaHostAlloc(&p, bytes ? bytes : 16, cudaHostAllocDefault) != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return set_error(Q1_ERR_OUT_OF_MEMORY, "pinned allocation of " + std::to_string(bytes) + " bytes failed");
        }
        return Q1_OK;
    }
};

// Civil date of a MonetDB day number (inverse of the parser's day_number), years >= 1.
void civil_from_day(int32_t n, int* y, int* m, int* d) {
    auto first = [](int yy) {
        const int p = yy - 1;
        return 365 * yy + (p / 4 - p / 100 + p / 400 + 1);
    };
    int yy = (int)((double)n / 365.2425);
    if (yy < 1) yy = 1;
    while (yy > 1 && first(yy) > n) --yy;
    while (first(yy + 1) <= n) ++yy;
    const bool leap = (yy % 4 == 0) && (yy % 100 != 0 || yy % 400 == 0);
    static const int kDays[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    int doy = n - first(yy), mm = 0;
    for (; mm < 12; ++mm) {
        const int len = kDays[mm] + ((mm == 1 && leap) ? 1 : 0);
        if (doy < len) break;
        doy -= len;
    }
    *y = yy, *m = mm + 1, *d = doy + 1;
}

uint64_t mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void put_decimal(std::string& s, int64_t v) {
    char b[32];
    const uint64_t a = v < 0 ? (uint64_t)(-(v + 1)) + 1 : (uint64_t)v;
    snprintf(b, sizeof(b), "%s%llu.%02llu|", v < 0 ? "-" : "", (unsigned long long)(a / 100),
             (unsigned long long)(a % 100));
    s += b;
}

void put_date(std::string& s, int32_t day, char end) {
    int y, m, d;
    civil_from_day(day, &y, &m, &d);
    char b[32];
    snprintf(b, sizeof(b), "%04d-%02d-%02d%c", y, m, d, end);
    s += b;
}

// One row in the dbgen lineitem layout. Fields Q1 does not read (keys, line number, commit and
// receipt dates, instruction, mode, comment) get deterministic placeholder values.
void format_row(std::string& s, const q1_columns& c, uint64_t i, uint64_t row) {
    const uint64_t h = mix(row);
    char b[96];
    snprintf(b, sizeof(b), "%llu|%llu|%llu|%llu|", (unsigned long long)(row / 4 + 1),
             (unsigned long long)(1 + h % 200000), (unsigned long long)(1 + (h >> 20) % 10000),
             (unsigned long long)(row % 4 + 1));
    s += b;
    put_decimal(s, c.quantity[i]);
    put_decimal(s, c.extendedprice[i]);
    put_decimal(s, c.discount[i]);
    put_decimal(s, c.tax[i]);
    s += c.returnflag[i];
    s += '|';
    s += c.linestatus[i];
    s += '|';
    put_date(s, c.shipdate[i], '|');
    put_date(s, c.shipdate[i] + 1 + (int32_t)((h >> 40) % 60), '|');
    put_date(s, c.shipdate[i] + 1 + (int32_t)((h >> 46) % 30), '|');
    snprintf(b, sizeof(b), "INSTRUCTION %u|MODE %u|", (unsigned)((h >> 52) % 4), (unsigned)((h >> 54) % 7));
    s += b;
    const uint32_t len = 10 + (uint32_t)((h >> 57) % 34);
    uint64_t w = mix(h);
    for (uint32_t k = 0; k < len; ++k) {
        if ((k & 7) == 0) w = mix(w);
        const uint32_t x = (uint32_t)(w >> (8 * (k & 7))) & 0xFFu;
        s += (x % 6 == 0 && k && k + 1 < len) ? ' ' : (char)('a' + x % 26);
    }
    s += "|\n";
}

q1_status file_size(const char* path, uint64_t* size) {
    struct stat sb;
    if (stat(path, &sb) != 0) return set_error(Q1_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path + ": " + strerror(errno));
    *size = (uint64_t)sb.st_size;
    return Q1_OK;
}

}  // namespace

extern "C" {

q1_status q1_tbl_count_device(const char* dev_text, uint64_t bytes, uint64_t* rows, void* cuda_stream) {
    if (!rows || (!dev_text && bytes)) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *rows = 0;
    if (!bytes) return Q1_OK;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const uint64_t tiles = tbl_tiles(bytes);
    DeviceMem lines;
    q1_status s = lines.alloc_async((tiles + 1) * 8, st);
    if (s != Q1_OK) return s;
    auto* v = static_cast<unsigned long long*>(lines.p);
    Q1_CUDA(launch_tbl_count(dev_text, bytes, v, st));
    unsigned long long total = 0;
    char last = 0;
    Q1_CUDA(cudaMemcpyAsync(&total, v + tiles, 8, cudaMemcpyDeviceToHost, st));
    Q1_CUDA(cudaMemcpyAsync(&last, dev_text + bytes - 1, 1, cudaMemcpyDeviceToHost, st));
    Q1_CUDA(cudaStreamSynchronize(st));
    *rows = total + (last != '\n' ? 1u : 0u);
    return Q1_OK;
}

q1_status q1_tbl_parse_device(const char* dev_text, uint64_t bytes, const q1_columns_out* dev_out, uint64_t capacity,
                              uint64_t* rows_out, void* cuda_stream) {
    if (!dev_out || !rows_out || (!dev_text && bytes)) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *rows_out = 0;
    if (!bytes) return Q1_OK;
    if (capacity && (!dev_out->shipdate || !dev_out->quantity || !dev_out->extendedprice || !dev_out->discount ||
                     !dev_out->tax || !dev_out->returnflag || !dev_out->linestatus))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output column");
    auto misaligned = [](const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; };
    if (misaligned(dev_out->shipdate, 4) || misaligned(dev_out->quantity, 8) || misaligned(dev_out->extendedprice, 8) ||
        misaligned(dev_out->discount, 8) || misaligned(dev_out->tax, 8))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "output columns must be aligned to their element size");
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const uint64_t tiles = tbl_tiles(bytes);
    DeviceMem scratch;
    q1_status s = scratch.alloc_async((tiles + 3) * 8, st);
    if (s != Q1_OK) return s;
    auto* v = static_cast<unsigned long long*>(scratch.p);
    unsigned long long* bad = v + tiles + 1;
    Q1_CUDA(cudaMemsetAsync(bad, 0, 8, st));
    Q1_CUDA(cudaMemsetAsync(bad + 1, 0xFF, 8, st));
    Q1_CUDA(launch_tbl_count(dev_text, bytes, v, st));
    Q1_CUDA(launch_tbl_parse(dev_text, bytes, v, dev_out->shipdate, dev_out->quantity, dev_out->extendedprice,
                             dev_out->discount, dev_out->tax, dev_out->returnflag, dev_out->linestatus, capacity, bad,
                             st));
    unsigned long long host[3] = {0, 0, 0};
    char last = 0;
    Q1_CUDA(cudaMemcpyAsync(host, v + tiles, 24, cudaMemcpyDeviceToHost, st));
    Q1_CUDA(cudaMemcpyAsync(&last, dev_text + bytes - 1, 1, cudaMemcpyDeviceToHost, st));
    Q1_CUDA(cudaStreamSynchronize(st));
    const uint64_t rows = host[0] + (last != '\n' ? 1u : 0u);
    *rows_out = rows;
    if (rows > capacity)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "the text holds " + std::to_string(rows) + " rows, the output " +
                                                      std::to_string(capacity));
    if (host[1])
        return set_error(Q1_ERR_INVALID_ARGUMENT, std::to_string(host[1]) + " malformed line(s); the first starts at byte " +
                                                      std::to_string(host[2]));
    return Q1_OK;
}

q1_status q1_tbl_read_file(const char* path, q1_columns_out* out, uint64_t capacity, uint64_t* rows_out) {
    if (!path || !rows_out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    *rows_out = 0;
    uint64_t size = 0;
    q1_status s = file_size(path, &size);
    if (s != Q1_OK) return s;
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(Q1_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path + ": " + strerror(errno));
    // the file in chunks of whole lines: read, copy to the device, parse there, copy the columns back
    // Q1_TBL_CHUNK_BYTES overrides the chunk size (tests use small chunks)
    uint64_t kChunk = 256ull << 20;
    if (const char* env = std::getenv("Q1_TBL_CHUNK_BYTES")) {
        const unsigned long long v = std::strtoull(env, nullptr, 10);
        if (v >= 4096) kChunk = v;
    }
    const uint64_t buf_bytes = std::min<uint64_t>(size, kChunk) + 4096;
    PinnedMem text;
    DeviceMem dtext, dcols;
    cudaStream_t st = nullptr;
    uint64_t total = 0, carry = 0, done = 0;
    // a well-formed row takes more than 16 bytes; a multiple of 64 keeps every column aligned
    const uint64_t max_rows = (buf_bytes / 16 + 64) & ~63ull;
    if ((s = text.alloc(buf_bytes)) != Q1_OK || (s = dtext.alloc(buf_bytes)) != Q1_OK ||
        (s = dcols.alloc(max_rows * 38)) != Q1_OK) {
        fclose(f);
        return s;
    }
    char* h = static_cast<char*>(text.p);
    uint8_t* dc = static_cast<uint8_t*>(dcols.p);
    q1_columns_out dev{reinterpret_cast<int32_t*>(dc), reinterpret_cast<char*>(dc + max_rows * 36),
                       reinterpret_cast<char*>(dc + max_rows * 37), reinterpret_cast<int64_t*>(dc + max_rows * 4),
                       reinterpret_cast<int64_t*>(dc + max_rows * 12), reinterpret_cast<int64_t*>(dc + max_rows * 20),
                       reinterpret_cast<int64_t*>(dc + max_rows * 28)};
    q1_status result = Q1_OK;
    while (done < size || carry) {
        const uint64_t want = std::min<uint64_t>(size - done, buf_bytes - carry - 1);
        const size_t got = want ? fread(h + carry, 1, want, f) : 0;
        if (got != want) {
            result = set_error(Q1_ERR_INVALID_ARGUMENT, std::string("short read from ") + path);
            break;
        }
        done += got;
        uint64_t n = carry + got;
        uint64_t cut = n;
        if (done < size) {   // whole lines only; the rest moves to the next chunk
            while (cut > 0 && h[cut - 1] != '\n') --cut;
            if (cut == 0) {
                result = set_error(Q1_ERR_INVALID_ARGUMENT, "a line is longer than the read buffer");
                break;
            }
        }
        if (cut) {
            const cudaError_t e = cudaMemcpyAsync(dtext.p, h, cut, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) {
                result = cuda_error(e, "copy of the text");
                break;
            }
            uint64_t rows = 0;
            if ((result = q1_tbl_parse_device(static_cast<const char*>(dtext.p), cut, &dev, max_rows, &rows, st)) !=
                Q1_OK) {
                if (rows && result == Q1_ERR_INVALID_ARGUMENT && strstr(q1_last_error(), "malformed"))
                    set_error(Q1_ERR_INVALID_ARGUMENT, std::string(q1_last_error()) + " of the chunk at row " +
                                                           std::to_string(total) + " of " + path);
                break;
            }
            if (out && rows) {
                if (total + rows > capacity) {
                    result = set_error(Q1_ERR_INVALID_ARGUMENT, std::string(path) + " holds more than " +
                                                                    std::to_string(capacity) + " rows");
                    break;
                }
                struct {
                    void* dst;
                    const void* src;
                    size_t elem;
                } cp[7] = {{out->shipdate + total, dev.shipdate, 4},   {out->quantity + total, dev.quantity, 8},
                           {out->extendedprice + total, dev.extendedprice, 8},
                           {out->discount + total, dev.discount, 8},    {out->tax + total, dev.tax, 8},
                           {out->returnflag + total, dev.returnflag, 1}, {out->linestatus + total, dev.linestatus, 1}};
                for (auto& c : cp) {
                    if (!c.dst) continue;
                    const cudaError_t e = cudaMemcpy(c.dst, c.src, rows * c.elem, cudaMemcpyDeviceToHost);
                    if (e != cudaSuccess) {
                        result = cuda_error(e, "copy of the parsed columns");
                        break;
                    }
                }
                if (result != Q1_OK) break;
            }
            total += rows;
        }
        carry = n - cut;
        if (carry) memmove(h, h + cut, carry);
    }
    fclose(f);
    if (result == Q1_OK) *rows_out = total;
    return result;
}

q1_status q1_tbl_load(q1_ctx* ctx, const char* path, q1_layout layout, q1_flag_packing packing,
                      q1_residency residency, uint64_t* rows_out) {
    if (!ctx || !path) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    uint64_t n = 0;
    q1_status s = q1_tbl_read_file(path, nullptr, 0, &n);
    if (s != Q1_OK) return s;
    std::vector<int32_t> ship(n);
    std::vector<char> rf(n), ls(n);
    std::vector<int64_t> disc(n), tax(n), price(n), qty(n);
    q1_columns_out o{ship.data(), rf.data(), ls.data(), disc.data(), tax.data(), price.data(), qty.data()};
    uint64_t got = 0;
    if ((s = q1_tbl_read_file(path, &o, n, &got)) != Q1_OK) return s;
    if (got != n) return set_error(Q1_ERR_INVALID_ARGUMENT, std::string(path) + " changed while it was read");
    q1_columns c{ship.data(), disc.data(), price.data(), tax.data(), qty.data(), rf.data(), ls.data()};
    if ((s = q1_load_columns(ctx, &c, n, layout, packing, residency)) != Q1_OK) return s;
    if (rows_out) *rows_out = n;
    return Q1_OK;
}

q1_status q1_tbl_format(const q1_columns* c, uint64_t first_row, uint64_t rows, char* buf, uint64_t capacity,
                        uint64_t* bytes_out) {
    if (!c || !bytes_out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (rows && (!c->shipdate || !c->quantity || !c->extendedprice || !c->discount || !c->tax || !c->returnflag ||
                 !c->linestatus))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t parts = std::min<uint64_t>(std::max<uint64_t>(1, rows / 65536), hw);
    std::vector<std::string> out(parts);
    std::vector<std::thread> th;
    for (uint64_t p = 0; p < parts; ++p)
        th.emplace_back([&, p]() {
            const uint64_t a = rows * p / parts, b = rows * (p + 1) / parts;
            std::string& s = out[p];
            s.reserve((b - a) * 160);
            for (uint64_t i = a; i < b; ++i) format_row(s, *c, i, first_row + i);
        });
    for (auto& t : th) t.join();
    uint64_t total = 0;
    for (auto& s : out) total += s.size();
    *bytes_out = total;
    if (!buf) return Q1_OK;
    if (total > capacity)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "the text needs " + std::to_string(total) + " bytes, the buffer has " +
                                                      std::to_string(capacity));
    for (auto& s : out) {
        memcpy(buf, s.data(), s.size());
        buf += s.size();
    }
    return Q1_OK;
}

}  // extern "C"
