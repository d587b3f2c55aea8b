// Boost-free definitions of the three parsing members the reference implements with
// boost::spirit in cpu/tpch_kit.cpp:100-153 (boost is absent in this image). Only Date::Date is
// reached at run time: BaseKernel's cutoff Date("1998-12-01", -1, -90) (cpu/common.cpp:60).
#include <cstdio>
#include <cstring>
#include <cassert>
#include "tpch_kit.hpp"

bool BaseDecimal::parse(const char* first, const char* last, int& intg, int& frac) {
    char buf[64];
    size_t n = (size_t)(last - first);
    if (n >= sizeof(buf)) return false;
    memcpy(buf, first, n);
    buf[n] = 0;
    int consumed = 0;
    if (sscanf(buf, "%d.%d%n", &intg, &frac, &consumed) == 2 && (size_t)consumed == n) return true;
    frac = 0;
    return sscanf(buf, "%d%n", &intg, &consumed) == 1 && (size_t)consumed == n;
}

bool Date::parse(const char* first, const char* last, int& day, int& month, int& year) {
    char buf[64];
    size_t n = (size_t)(last - first);
    if (n >= sizeof(buf)) return false;
    memcpy(buf, first, n);
    buf[n] = 0;
    int consumed = 0;
    return sscanf(buf, "%d-%d-%d%n", &year, &month, &day, &consumed) == 3 && (size_t)consumed == n;
}

Date::Date(const char* v, int64_t len, int plus_days) {
    if (len < 0) len = (int64_t)strlen(v);
    int day = 0, month = 0, year = 0;
    bool ok = parse(v, v + len, day, month, year);
    assert(ok);
    (void)ok;
    dte_val = todate(day, month, year) + plus_days;
}
