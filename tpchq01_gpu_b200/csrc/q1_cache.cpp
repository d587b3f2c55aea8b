// Binary column cache in the reference's on-disk format (src/file_access.hpp:19-61, written and
// read by src/main.cu:405-474): one raw native-endian array per lineitem column in a directory,
//   shipdate.bin (int32 day numbers), returnflag.bin, linestatus.bin (char),
//   discount.bin, tax.bin, extendedprice.bin, quantity.bin (int64 hundredths / cents).
// The row count is the size of shipdate.bin / 4; every other file must hold exactly that many
// elements. Unlike the reference, an SF-1-sized cache is not rescaled by the scale factor
// (src/main.cu:412-414, which then fails to read the files).
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "q1.h"
#include "q1_internal.h"

using namespace q1;

namespace {

struct ColumnFile {
    const char* name;
    size_t elem;
};
constexpr ColumnFile kFiles[7] = {{"shipdate.bin", 4},      {"returnflag.bin", 1}, {"linestatus.bin", 1},
                                  {"discount.bin", 8},      {"tax.bin", 8},        {"extendedprice.bin", 8},
                                  {"quantity.bin", 8}};

std::string path_of(const char* dir, const char* name) {
    std::string p(dir);
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name;
}

bool file_size(const std::string& path, uint64_t* size) {
    struct stat sb;
    if (stat(path.c_str(), &sb) != 0) return false;
    *size = (uint64_t)sb.st_size;
    return true;
}

q1_status write_file(const std::string& path, const void* data, size_t elem, uint64_t n) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return set_error(Q1_ERR_INVALID_ARGUMENT, "cannot open " + path + " for writing: " + strerror(errno));
    const size_t written = n ? fwrite(data, elem, n, f) : 0;
    const bool ok = written == n && fclose(f) == 0;
    if (!ok) {
        remove(path.c_str());
        return set_error(Q1_ERR_INVALID_ARGUMENT, "short write to " + path);
    }
    return Q1_OK;
}

q1_status read_file(const std::string& path, void* data, size_t elem, uint64_t n) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return set_error(Q1_ERR_INVALID_ARGUMENT, "cannot open " + path + ": " + strerror(errno));
    const size_t got = n ? fread(data, elem, n, f) : 0;
    fclose(f);
    if (got != n)
        return set_error(Q1_ERR_INVALID_ARGUMENT, "short read from " + path + ": expected " + std::to_string(n) +
                                                      " elements, read " + std::to_string(got));
    return Q1_OK;
}

}  // namespace

extern "C" {

q1_status q1_cache_write(const char* dir, const q1_columns* c, uint64_t rows) {
    if (!dir || !c) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    if (rows && (!c->shipdate || !c->returnflag || !c->linestatus || !c->discount || !c->tax || !c->extendedprice ||
                 !c->quantity))
        return set_error(Q1_ERR_INVALID_ARGUMENT, "missing column");
    mkdir(dir, 0755);   // may exist already
    const void* src[7] = {c->shipdate, c->returnflag, c->linestatus, c->discount, c->tax, c->extendedprice, c->quantity};
    for (int k = 0; k < 7; ++k) {
        q1_status st = write_file(path_of(dir, kFiles[k].name), src[k], kFiles[k].elem, rows);
        if (st != Q1_OK) return st;
    }
    return Q1_OK;
}

q1_status q1_cache_rows(const char* dir, uint64_t* rows) {
    if (!dir || !rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    uint64_t size = 0;
    if (!file_size(path_of(dir, kFiles[0].name), &size))
        return set_error(Q1_ERR_INVALID_ARGUMENT, std::string("no column cache in ") + dir + " (shipdate.bin missing)");
    if (size % kFiles[0].elem) return set_error(Q1_ERR_INVALID_ARGUMENT, "shipdate.bin size is not a multiple of 4");
    const uint64_t n = size / kFiles[0].elem;
    for (int k = 1; k < 7; ++k) {
        uint64_t s = 0;
        const std::string p = path_of(dir, kFiles[k].name);
        if (!file_size(p, &s)) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing " + p);
        if (s != n * kFiles[k].elem)
            return set_error(Q1_ERR_INVALID_ARGUMENT, p + " holds " + std::to_string(s / kFiles[k].elem) +
                                                          " elements, shipdate.bin " + std::to_string(n));
    }
    *rows = n;
    return Q1_OK;
}

q1_status q1_cache_read(const char* dir, uint64_t rows, q1_columns_out* out) {
    if (!dir || !out) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    uint64_t n = 0;
    q1_status st = q1_cache_rows(dir, &n);
    if (st != Q1_OK) return st;
    if (n != rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "row count differs from the cache's");
    void* dst[7] = {out->shipdate, out->returnflag, out->linestatus, out->discount, out->tax, out->extendedprice,
                    out->quantity};
    for (int k = 0; k < 7; ++k) {
        if (!dst[k] && rows) return set_error(Q1_ERR_INVALID_ARGUMENT, "missing output column");
        if ((st = read_file(path_of(dir, kFiles[k].name), dst[k], kFiles[k].elem, rows)) != Q1_OK) return st;
    }
    return Q1_OK;
}

q1_status q1_cache_load(q1_ctx* ctx, const char* dir, q1_layout layout, q1_flag_packing packing,
                        q1_residency residency, uint64_t* rows_out) {
    if (!ctx || !dir) return set_error(Q1_ERR_INVALID_ARGUMENT, "null argument");
    uint64_t n = 0;
    q1_status st = q1_cache_rows(dir, &n);
    if (st != Q1_OK) return st;
    std::vector<int32_t> ship(n);
    std::vector<char> rf(n), ls(n);
    std::vector<int64_t> disc(n), tax(n), price(n), qty(n);
    q1_columns_out o{ship.data(), rf.data(), ls.data(), disc.data(), tax.data(), price.data(), qty.data()};
    if ((st = q1_cache_read(dir, n, &o)) != Q1_OK) return st;
    q1_columns c{ship.data(), disc.data(), price.data(), tax.data(), qty.data(), rf.data(), ls.data()};
    if ((st = q1_load_columns(ctx, &c, n, layout, packing, residency)) != Q1_OK) return st;
    if (rows_out) *rows_out = n;
    return Q1_OK;
}

}  // extern "C"
