// tpch_01 -- drop-in command line of the reference's tpch_01 (src/main.cu:738-916) over the C ABI.
//
// Same flags as the reference's parse_command_line (src/main.cu:255-360), in both the code
// spelling and the README spelling (README.md:47-58): --apply-compression,
// --use-filter-pushdown, --use-coprocessing, --print-results, --device,
// --hash-table-placement=, --scale-factor= | --sf=, --streams=, --threads-per-block=,
// --tuples-per-thread= | --tuples_per_thread=, --tuples-per-kernel-launch= | --tuples-per-kernel=,
// --runs=, --cpu-fraction=.
// Additions: --rows=N (exact row count), --seed=S (generator seed), --cutoff-day=D,
// --data-dir=DIR (the reference's column cache DIR/<scale factor>/*.bin), --cache-dir=DIR (a
// cache directory itself), --write-cache (generate and write the cache when it is missing),
// --resident (keep the table in HBM instead of streaming it from pinned host memory every run,
// which is what the reference does).
// The table comes from the seeded synthetic generator (dbgen's lineitem.tbl is not available);
// rows = scale factor x 6,001,215 (src/constants.hpp:49). Per-run wall times go to results.csv
// (src/main.cu:881-905).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>

#include <fstream>
#include <string>
#include <vector>

#include "q1.h"

static void print_help(const char* argv0) {
    fprintf(stderr, "Unrecognized command line option.\n");
    fprintf(stderr, "Usage: %s [args]\n", argv0);
    fprintf(stderr, "   --apply-compression\n");
    fprintf(stderr, "   --print-results\n");
    fprintf(stderr, "   --use-filter-pushdown\n");
    fprintf(stderr, "   --use-coprocessing\n");
    fprintf(stderr, "   --hash-table-placement=[default:in_registers_per_thread]\n"
                    "     (one of: in_registers, in_registers_per_thread, local_mem, shared_mem_per_thread, global;\n"
                    "      or in-registers, local-mem, per-thread-shared-mem)\n");
    fprintf(stderr, "   --runs=[default:5]\n");
    fprintf(stderr, "   --sf=[default:1.0] | --scale-factor=   --rows=N\n");
    fprintf(stderr, "   --data-dir=DIR | --cache-dir=DIR   --write-cache   --tbl=FILE   --write-tbl\n");
    fprintf(stderr, "   --cpu-fraction=[default:0.5]\n");
    fprintf(stderr, "   --streams=[default:4]\n");
    fprintf(stderr, "   --threads-per-block=[multiple of 32]\n");
    fprintf(stderr, "   --tuples-per-thread=\n");
    fprintf(stderr, "   --tuples-per-kernel-launch=[default:2097152] | --tuples-per-kernel=\n");
    fprintf(stderr, "   --resident   --seed=S   --cutoff-day=D   --device\n");
}

static void print_device() {
    char buf[512];
    if (q1_device_describe(0, buf, sizeof(buf)) != Q1_OK) {
        fprintf(stderr, "%s\n", q1_last_error());
        return;
    }
    printf("%s\n", buf);
}

static void print_dec(const q1_i128& v, int64_t scale, int width) {
    __int128 x = (__int128)(((unsigned __int128)v.hi << 64) | v.lo);
    const bool neg = x < 0;
    if (neg) x = -x;
    const __int128 ip = x / scale, fp = x % scale;
    char buf[64];
    int n = 0;
    __int128 t = ip;
    char digits[48];
    do {
        digits[n++] = (char)('0' + (int)(t % 10));
        t /= 10;
    } while (t);
    int k = 0;
    if (neg) buf[k++] = '-';
    while (n) buf[k++] = digits[--n];
    buf[k] = 0;
    int fd = 0;
    for (int64_t s = scale; s > 1; s /= 10) ++fd;
    printf(" | %*s.%0*lld", width - fd - 1, buf, fd, (long long)fp);
}

static void print_results(const q1_result& r) {
    printf("+---------------------------------------------------- Results ------------------------------------------------------+\n");
    printf("|  LS | RF |  sum_quantity        |  sum_base_price      |  sum_disc_price      |  sum_charge          | count      |\n");
    printf("+-------------------------------------------------------------------------------------------------------------------+\n");
    uint64_t total = 0;
    for (uint32_t g = 0; g < r.num_groups; ++g) {
        const q1_group_result& x = r.groups[g];
        if (!x.count) continue;
        printf("| # %c | %c ", x.returnflag, x.linestatus);
        print_dec(x.sum_qty, 100, 20);
        print_dec(x.sum_base_price, 100, 20);
        print_dec(x.sum_disc_price, 10000, 20);
        print_dec(x.sum_charge, 1000000, 20);
        printf(" | %10llu |", (unsigned long long)x.count);
        printf("  avg_qty %lld.%04lld avg_price %lld.%04lld avg_disc %lld.%04lld\n", (long long)(x.avg_qty_e4 / 10000),
               (long long)llabs(x.avg_qty_e4 % 10000), (long long)(x.avg_price_e4 / 10000),
               (long long)llabs(x.avg_price_e4 % 10000), (long long)(x.avg_disc_e4 / 10000),
               (long long)llabs(x.avg_disc_e4 % 10000));
        total += x.count;
    }
    printf("+-------------------------------------------------------------------------------------------------------------------+\n");
    printf("Total number of elements tuples satisfying the WHERE clause: %llu / %llu = %f\n", (unsigned long long)total,
           (unsigned long long)r.rows_total, r.rows_total ? (double)total / (double)r.rows_total : 0.0);
}

static bool starts(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }

int main(int argc, char** argv) {
    q1_params p;
    q1_params_default(&p);
    double scale_factor = 1.0;
    uint64_t rows = 0;
    uint64_t seed = 20260101;
    bool print = false, resident = false, write_cache = false, write_tbl = false;
    std::string data_dir, cache_dir, tbl_path;
    for (int i = 1; i < argc; ++i) {
        std::string a(argv[i]);
        if (!starts(a, "--")) {
            print_help(argv[0]);
            return EXIT_FAILURE;
        }
        a = a.substr(2);
        const size_t eq = a.find('=');
        std::string name = eq == std::string::npos ? a : a.substr(0, eq);
        const std::string val = eq == std::string::npos ? "" : a.substr(eq + 1);
        for (auto& ch : name)
            if (ch == '_') ch = '-';
        try {
            if (name == "device") {
                print_device();
                return 1;   // the reference exits after printing the device (src/main.cu:266-268)
            } else if (name == "use-coprocessing") p.use_coprocessing = 1;
            else if (name == "apply-compression") p.apply_compression = 1;
            else if (name == "use-filter-pushdown") p.use_filter_pushdown = 1;
            else if (name == "print-results") print = true;
            else if (name == "resident") resident = true;
            else if (name == "data-dir") data_dir = val;
            else if (name == "cache-dir") cache_dir = val;
            else if (name == "write-cache") write_cache = true;
            else if (name == "tbl") tbl_path = val;
            else if (name == "write-tbl") write_tbl = true;
            else if (name == "scale-factor" || name == "sf") {
                scale_factor = std::stod(val);
                if (scale_factor < 0.001) {
                    fprintf(stderr, "Invalid scale factor %f\n", scale_factor);
                    return EXIT_FAILURE;
                }
            } else if (name == "rows") rows = std::stoull(val);
            else if (name == "seed") seed = std::stoull(val);
            else if (name == "cutoff-day") p.cutoff_day = std::stoi(val);
            else if (name == "hash-table-placement") {
                q1_placement pl;
                if (q1_placement_from_name(val.c_str(), &pl) != Q1_OK) {
                    fprintf(stderr, "%s\n", q1_last_error());
                    return EXIT_FAILURE;
                }
                p.placement = pl;
            } else if (name == "streams") p.streams = std::stoi(val);
            else if (name == "tuples-per-thread") p.tuples_per_thread = std::stoi(val);
            else if (name == "threads-per-block") p.threads_per_block = std::stoi(val);
            else if (name == "tuples-per-kernel-launch" || name == "tuples-per-kernel") p.tuples_per_launch = std::stoll(val);
            else if (name == "runs") p.runs = std::stoi(val);
            else if (name == "cpu-fraction") p.cpu_fraction = std::stod(val);
            else {
                print_help(argv[0]);
                return EXIT_FAILURE;
            }
        } catch (const std::exception&) {
            fprintf(stderr, "Cannot parse the value passed after --%s=\n", name.c_str());
            return EXIT_FAILURE;
        }
    }
    if (q1_params_validate(&p) != Q1_OK) {
        fprintf(stderr, "%s\n", q1_last_error());
        return EXIT_FAILURE;
    }
    if (!rows) rows = (uint64_t)(scale_factor * 6001215.0);

    q1_ctx* ctx = nullptr;
    q1_device_opts opts{0, 0};
    if (q1_open(&ctx, &opts) != Q1_OK) {
        fprintf(stderr, "q1_open: %s\n", q1_last_error());
        return EXIT_FAILURE;
    }
    const q1_residency res = resident ? Q1_RESIDENCY_HBM : Q1_RESIDENCY_PINNED_HOST;
    const q1_layout layout = p.apply_compression ? Q1_LAYOUT_COMPRESSED : Q1_LAYOUT_UNCOMPRESSED;
    q1_status st;
    if (!tbl_path.empty()) {
        // a lineitem text file, parsed on the GPU (lineitem::FromFile, cpu/tpch_kit.cpp:155-172)
        printf("Parsing the lineitem table in file %s on the GPU... ", tbl_path.c_str());
        fflush(stdout);
        st = q1_tbl_load(ctx, tbl_path.c_str(), layout, Q1_FLAGS_PAIR_2BIT, res, &rows);
    } else if (!data_dir.empty() || !cache_dir.empty()) {
        // the reference's column cache: <data dir>/<scale factor as std::to_string>/ (src/main.cu:405-409);
        // without one, <dir>/lineitem.tbl is parsed and the cache written (src/main.cu:441-475)
        const std::string dir = !cache_dir.empty() ? cache_dir : data_dir + "/" + std::to_string(scale_factor);
        const std::string tbl = dir + "/lineitem.tbl";
        uint64_t cached = 0;
        if (q1_cache_rows(dir.c_str(), &cached) != Q1_OK) {
            struct stat sb;
            const bool have_tbl = stat(tbl.c_str(), &sb) == 0;
            if (!have_tbl && !write_cache && !write_tbl) {
                fprintf(stderr, "%s and no %s (use --write-cache or --write-tbl to generate one)\n", q1_last_error(),
                        tbl.c_str());
                q1_close(ctx);
                return EXIT_FAILURE;
            }
            if (!data_dir.empty()) mkdir(data_dir.c_str(), 0755);
            mkdir(dir.c_str(), 0755);
            std::vector<int32_t> ship;
            std::vector<int64_t> disc, price, tax, qty;
            std::vector<char> rf, ls;
            auto resize = [&](uint64_t n) {
                ship.resize(n), disc.resize(n), price.resize(n), tax.resize(n), qty.resize(n), rf.resize(n), ls.resize(n);
            };
            q1_status gs = Q1_OK;
            if (have_tbl) {
                printf("Parsing the lineitem table in file %s on the GPU... ", tbl.c_str());
                fflush(stdout);
                uint64_t n = 0;
                gs = q1_tbl_read_file(tbl.c_str(), nullptr, 0, &n);
                if (gs == Q1_OK) {
                    resize(n);
                    q1_columns_out o{ship.data(), rf.data(), ls.data(), disc.data(), tax.data(), price.data(), qty.data()};
                    gs = q1_tbl_read_file(tbl.c_str(), &o, n, &rows);
                }
            } else {
                resize(rows);
                q1_columns c{ship.data(), disc.data(), price.data(), tax.data(), qty.data(), rf.data(), ls.data()};
                gs = q1_generate_host(seed, 0, rows, &c);
                if (gs == Q1_OK && write_tbl) {
                    printf("Writing %llu generated rows to %s... ", (unsigned long long)rows, tbl.c_str());
                    fflush(stdout);
                    uint64_t bytes = 0;
                    gs = q1_tbl_format(&c, 0, rows, nullptr, 0, &bytes);
                    std::vector<char> text(gs == Q1_OK ? bytes : 0);
                    if (gs == Q1_OK) gs = q1_tbl_format(&c, 0, rows, text.data(), bytes, &bytes);
                    FILE* f = gs == Q1_OK ? fopen(tbl.c_str(), "wb") : nullptr;
                    if (gs == Q1_OK && (!f || fwrite(text.data(), 1, bytes, f) != bytes)) {
                        fprintf(stderr, "\ncannot write %s\n", tbl.c_str());
                        if (f) fclose(f);
                        q1_close(ctx);
                        return EXIT_FAILURE;
                    }
                    if (f) fclose(f);
                }
            }
            q1_columns c{ship.data(), disc.data(), price.data(), tax.data(), qty.data(), rf.data(), ls.data()};
            if (gs == Q1_OK && (have_tbl || write_cache)) {
                printf("done (%llu rows).\nWriting the column cache to %s... ", (unsigned long long)rows, dir.c_str());
                fflush(stdout);
                gs = q1_cache_write(dir.c_str(), &c, rows);
            }
            if (gs != Q1_OK) {
                fprintf(stderr, "\n%s\n", q1_last_error());
                q1_close(ctx);
                return EXIT_FAILURE;
            }
            printf("done.\n");
            if (!have_tbl && !write_cache) {
                // --write-tbl alone: load the generated rows directly
                printf("Loading %llu rows... ", (unsigned long long)rows);
                fflush(stdout);
                st = q1_load_columns(ctx, &c, rows, layout, Q1_FLAGS_PAIR_2BIT, res);
                goto loaded;
            }
        }
        printf("Loading the column cache in %s... ", dir.c_str());
        fflush(stdout);
        st = q1_cache_load(ctx, dir.c_str(), layout, Q1_FLAGS_PAIR_2BIT, res, &rows);
    } else {
        printf("Generating %llu lineitem rows (seed %llu, %s, %s)... ", (unsigned long long)rows,
               (unsigned long long)seed, p.apply_compression ? "compressed" : "uncompressed",
               resident ? "HBM-resident" : "pinned host memory, streamed each run");
        fflush(stdout);
        st = q1_generate_table(ctx, seed, 0, rows, layout, Q1_FLAGS_PAIR_2BIT, res);
    }
loaded:
    if (st != Q1_OK) {
        fprintf(stderr, "\nloading the table failed: %s\n", q1_last_error());
        q1_close(ctx);
        return EXIT_FAILURE;
    }
    printf("done (%llu rows).\n", (unsigned long long)rows);
    std::ofstream csv("results.csv", std::ios::out);
    const int runs = p.runs;
    p.runs = 1;
    q1_result r;
    for (int run = 0; run < runs; ++run) {
        printf("Executing TPC-H Query 1, run %d of %d... ", run + 1, runs);
        fflush(stdout);
        st = q1_run(ctx, &p, &r);
        if (st != Q1_OK) {
            fprintf(stderr, "\nq1_run: %s: %s\n", q1_status_string(st), q1_last_error());
            q1_close(ctx);
            return EXIT_FAILURE;
        }
        printf("done.\n");
        csv << r.ms_last_run / 1000.0 << '\n';
        if (print) print_results(r);
    }
    q1_close(ctx);
    return 0;
}
