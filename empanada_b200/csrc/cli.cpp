// cli.cpp -- the `empanada` command (drop-in for the reference's binary).
//
//   empanada input.fastq output.bin [-o N] [-m SIZE] [-r SIZE] [-b SIZE] [-c SIZE]
//
// Argument handling restates config.h:10-140 including its quirks:
//   * positionals first; an option is recognised by its SECOND character
//     only (arg[1] == shortname), so "-o" and "xo" both set -o;
//   * "--long" options print "Not implemented yet. Use short forms instead."
//     (config.h:50-52) and then fall through to "Invalid option";
//   * an unknown option or a missing positional prints the usage and exits
//     with status 0 (config.h:21-35,60-63,66-67);
//   * SIZE is digits with an optional k/K/m/M/g/G binary suffix
//     (hmsize2bytes, config.h:75-100); -o is parsed the same way.
// Differences, on inputs where the reference crashes: an option without a
// value or a SIZE that is not a number prints an error and exits 1.
// Side effects kept: log lines on stdout/stderr, ./timings.csv
// (timer.h:11-62) with this engine's stage times.
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <list>
#include <string>

#include "../../include/empanada.h"

namespace {

struct Option {
    char shortname = 0;
    std::string longname, description, defaultValue, value;
    bool is_required() const { return !shortname; }
};

const char *now_str() {
    static char buf[16];
    std::time_t t = std::time(nullptr);
    std::tm tmv;
    localtime_r(&t, &tmv);
    std::strftime(buf, sizeof buf, "%T", &tmv);
    return buf;
}

#define LOG_INFO(fmt, ...) std::fprintf(stdout, "[%s]\x1B[32mINFO: " fmt "\x1B[0m\n", now_str(), ##__VA_ARGS__)
#define LOG_ERR(fmt, ...) std::fprintf(stderr, "[%s]\x1B[31mERROR: " fmt "\x1B[0m\n", now_str(), ##__VA_ARGS__)

[[noreturn]] void usage_and_exit(const std::list<Option> &options) {
    std::printf("Usage: assembly_v3");
    for (const Option &o : options)
        if (o.is_required()) std::printf(" [%s]", o.description.c_str());
    std::printf(" [options]\n");
    std::printf("Options:\n");
    for (const Option &o : options)
        if (!o.is_required())
            std::printf("  -%c or --%s, %s, default = %s\n", o.shortname, o.longname.c_str(), o.description.c_str(),
                        o.defaultValue.c_str());
    std::exit(0);
}

void parse_args(int argc, char **argv, std::list<Option> &options) {
    auto it = options.begin();
    --argc;
    ++argv;
    while (argc > 0) {
        std::string arg = argv[0];
        if (it != options.end() && it->is_required()) {
            it->value = arg;
            ++it;
            --argc;
            ++argv;
        } else {
            bool found = false;
            for (auto it1 = it; it1 != options.end(); ++it1) {
                const char second = arg.size() > 1 ? arg[1] : '\0';
                if (second == '-') {
                    LOG_ERR("Not implemented yet. Use short forms instead.");
                } else if (second == it1->shortname) {
                    if (argc < 2) {
                        LOG_ERR("Option %s needs a value.", arg.c_str());
                        std::exit(1);
                    }
                    it1->value = argv[1];
                    argc -= 2;
                    argv += 2;
                    found = true;
                }
            }
            if (!found) {
                std::printf("Invalid option %s\n", arg.c_str());
                usage_and_exit(options);
            }
        }
    }
    while (it != options.end()) {
        if (it->is_required()) usage_and_exit(options);
        if (it->value.empty()) it->value = it->defaultValue;
        ++it;
    }
}

uint64_t size_or_die(const std::string &s) {
    uint64_t v = 0;
    emp_status st = emp_parse_size(s.c_str(), &v);
    if (st == EMP_OK) return v;
    if (!s.empty()) {
        const char unit = s.back();
        std::string digits = s.substr(0, s.size() - 1);
        uint64_t dv = 0;
        if (!(unit >= '0' && unit <= '9') && emp_parse_size(digits.c_str(), &dv) == EMP_OK) {
            LOG_ERR("Unknown unit %c.", unit);  // reference keeps the number without the unit
            return dv;
        }
    }
    LOG_ERR("Invalid size %s.", s.c_str());
    std::exit(1);
}

}  // namespace

int main(int argc, char **argv) {
    std::list<Option> options = {
        {0, "", "input fastq", "", ""},
        {0, "", "output gfa", "", ""},
        {'o', "min-overlap", "minimum overlap length", "31", ""},
        {'m', "map-mem", "device memory during the fingerprint generation phase", "1g", ""},
        {'r', "reduce-mem", "device memory during the overlap-detection phase", "1g", ""},
        {'b', "base-blocksz", "block size (count) of transposed bases", "32m", ""},
        {'c', "kv-chunksz", "block size (count) of key-value pairs", "64m", ""},
    };
    parse_args(argc, argv, options);
    auto it = options.begin();
    const std::string input = (it++)->value;
    const std::string output = (it++)->value;
    emp_params p;
    emp_params_default(&p);
    p.min_ovlp = (int32_t)size_or_die((it++)->value);
    p.map_mem = size_or_die((it++)->value);
    p.reduce_mem = size_or_die((it++)->value);
    p.base_blocksz = size_or_die((it++)->value);
    p.kv_chunksz = size_or_die((it++)->value);

    LOG_INFO("Reading file %s", input.c_str());
    static emp_stats st;
    emp_status rc = emp_run_file(input.c_str(), output.c_str(), &p, -1, &st);
    if (rc != EMP_OK) {
        LOG_ERR("%s (%d)", emp_status_string(rc), rc);
        return 1;
    }
    LOG_INFO("Map Phase over..");
    LOG_INFO("%llu duplicates removed.", (unsigned long long)(2 * st.n_reads - st.n_unique));
    for (int r = 0; r < st.n_rounds && r < EMP_MAX_ROUNDS; ++r)
        LOG_INFO("%llu edges created.", (unsigned long long)st.edges[r]);
    std::FILE *t = std::fopen("timings.csv", "w");
    if (t) {
        std::time_t now = std::time(nullptr);
        std::fprintf(t, "## %s", std::asctime(std::localtime(&now)));
        std::fprintf(t, "Phase,Time (us)\n");
        std::fprintf(t, "read_input_h2d,%lld\n", (long long)(st.ms_h2d * 1000.0));
        std::fprintf(t, "map_phase,%lld\n", (long long)(st.ms_map * 1000.0));
        std::fprintf(t, "sort_unique,%lld\n", (long long)(st.ms_dedup * 1000.0));
        std::fprintf(t, "overlap_rounds,%lld\n", (long long)(st.ms_rounds * 1000.0));
        std::fprintf(t, "total_device,%lld\n", (long long)(st.ms_total * 1000.0));
        std::fclose(t);
    }
    return 0;
}
