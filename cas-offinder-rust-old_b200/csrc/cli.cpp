// cli.cpp -- cas-offinder command line on top of libcof.so.
//
//   cof-offinder {input_filename|-} {C|G|A} {output_filename|-}
//
// Input file format and validation follow cas-offinder-cli/src/cli_utils.rs
// (37-148); output (header + 8 tab-separated columns) and the <output>.log
// summary follow cas-offinder-cli/src/main.rs (122-304) and
// cas-offinder-lib/src/log_writer.rs (27-53).  The search always runs on the
// GPU; the device letter only selects the batch size the reference uses for
// that device (C: 64 chunks, search.rs:21; G/A: 16384 chunks, search.rs:22),
// which fixes the reference's batch-boundary rules.
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cof.h"

namespace {

[[noreturn]] void die(const std::string &m) {
    std::cerr << "error: " << m << "\n";
    std::exit(1);
}

bool mixed_str(const std::string &s) {
    static const char *ok = "ACGTRYSWKMBDHVNacgtryswkmbdhvn";
    for (char c : s)
        if (!c || !std::strchr(ok, c)) return false;
    return !s.empty();
}

std::vector<std::string> split_ws(const std::string &l) {
    std::vector<std::string> out;
    std::istringstream is(l);
    std::string w;
    while (is >> w) out.push_back(w);
    return out;
}

bool parse_u32(const std::string &s, uint32_t &v) {
    if (s.empty()) return false;
    unsigned long long x = 0;
    for (char c : s) {
        if (c < '0' || c > '9') return false;
        x = x * 10 + (unsigned)(c - '0');
        if (x > 0xFFFFFFFFull) return false;
    }
    v = (uint32_t)x;
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) die("Too few arguments, expected 3 arguments");
    const auto t0 = std::chrono::steady_clock::now();
    std::string in_path = argv[1], dev = argv[2], out_path = argv[3];
    if (dev.size() != 1 || !std::strchr("CGA", dev[0])) die("2nd argument must be one of {C|G|A}");
    std::ifstream fin;
    std::istream *in = &std::cin;
    if (in_path != "-") {
        fin.open(in_path, std::ios::binary);
        if (!fin) die("cannot open input file " + in_path);
        in = &fin;
    }
    std::string genome, filter, line;
    uint32_t db = 0, rb = 0, mm = 0;
    bool have_mm = false;
    int use_info = -1;
    std::vector<std::string> pats;
    int lineno = 0;
    while (std::getline(*in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        ++lineno;
        if (lineno == 1) { genome = line; continue; }
        auto parts = split_ws(line);
        if (lineno == 2) {
            if (parts.size() == 1) filter = parts[0];
            else if (parts.size() == 3) {
                filter = parts[0];
                if (!parse_u32(parts[1], db)) die("bulge_dna must be a non-negative integer");
                if (!parse_u32(parts[2], rb)) die("bulge_rna must be a non-negative integer");
            } else die("2nd line must be: <search_filter> [<bulge_dna> <bulge_rna>]");
            if (!mixed_str(filter)) die("Pattern in input file needs to be a mixed base string");
            continue;
        }
        if (parts.size() != 2 && parts.size() != 3)
            die("Pattern line must have following elements: <patterns> <mismatches> [<label>]");
        if (!mixed_str(parts[0])) die("Pattern in input file needs to be a mixed base string");
        uint32_t cur;
        if (!parse_u32(parts[1], cur))
            die("2nd element of each pattern in mismatches must be an unsigned integer");
        if (!have_mm) { mm = cur; have_mm = true; }
        if (use_info < 0) use_info = parts.size() == 3;
        if (mm != cur)
            die("In this version of cas-offinder, all mismatches on every line of input file must be the same");
        if (use_info && parts.size() < 3)
            die("Pattern lines in input file must be consistently have either 2 or 3 elements, no mixing and matching allowed");
        if (parts[0].size() != filter.size()) die("All patters in input file must be same length");
        pats.push_back(parts[0]);
    }
    if (lineno < 2) die("Input file must contain at least 3 lines");
    if (!have_mm) die("Input file must contain at least 1 pattern line");

    // COF_CLI_TIMES=1: seconds per stage on stderr (not part of main.rs's output)
    const char *times_env = std::getenv("COF_CLI_TIMES");
    const bool times = times_env && *times_env && std::strcmp(times_env, "0") != 0;
    auto lap = [t = t0]() mutable {
        const auto now = std::chrono::steady_clock::now();
        const double d = std::chrono::duration<double>(now - t).count();
        t = now;
        return d;
    };
    const double t_input = lap();
    // one search per process: timing tile shapes (tens of ms) cannot pay
    // back, so the default shape is used unless COF_AUTOTUNE says otherwise
    ::setenv("COF_AUTOTUNE", "0", 0);
    cof_genome *g = nullptr;
    if (cof_genome_create(0, &g)) die(cof_last_error());
    if (cof_genome_load(g, genome.c_str())) die(cof_last_error());
    const double t_load = lap();
    if (cof_genome_upload(g)) die(cof_last_error());
    const double t_upload = lap();
    std::vector<const char *> pp;
    for (auto &p : pats) pp.push_back(p.c_str());
    cof_request r{};
    r.search_filter = filter.c_str();
    r.pattern_len = filter.size();
    r.patterns = pp.data();
    r.n_patterns = pp.size();
    r.max_mismatches = mm;
    r.max_dna_bulges = db;
    r.max_rna_bulges = rb;
    r.flags = COF_F_ADD_REVCOMP;
    r.chunks_per_search = dev[0] == 'C' ? 64 : 16384;
    cof_result res{};
    if (cof_search(g, &r, &res)) die(cof_last_error());
    const double t_search = lap();
    FILE *out = out_path == "-" ? stdout : std::fopen(out_path.c_str(), "wb");
    if (!out) die("cannot open output file " + out_path);
    std::fputs(COF_HEADER, out);
    std::fwrite(res.text, 1, res.text_len, out);
    if (out != stdout) std::fclose(out);
    const double t_write = lap();
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cerr << "Completed in " << secs << "s\n";
    if (out_path != "-") {
        struct stat st;
        unsigned long long gsize = ::stat(genome.c_str(), &st) ? 0 : (unsigned long long)st.st_size;
        std::ofstream lg(out_path + ".log");
        if (lg) {
            const char *label = dev[0] == 'C' ? "CPU" : dev[0] == 'G' ? "GPU" : "Accelerator";
            lg << "=== Cas-OFFinder Rust ===\n"
               << "Run date (unix timestamp): " << (long long)std::time(nullptr) << "\n\n"
               << "Algorithm: " << ((db || rb) ? "Myers bit-parallel" : "popcount (legacy)") << "\n"
               << "Device: " << label << "\n\n"
               << "Input:\n"
               << "  Genome: " << genome << "\n"
               << "  Genome size: " << gsize << " bytes\n"
               << "  Patterns: " << pats.size() << "\n"
               << "  Search filter: " << filter << "\n"
               << "  Max mismatches: " << mm << "\n"
               << "  Max DNA bulges: " << db << "\n"
               << "  Max RNA bulges: " << rb << "\n\n"
               << "Results:\n"
               << "  Matches found: " << res.n_rows << "\n";
            char buf[64];
            std::snprintf(buf, sizeof buf, "%.3f", secs);
            lg << "  Total elapsed: " << buf << "s\n";
        } else {
            std::cerr << "warning: failed to write log file '" << out_path << ".log'\n";
        }
    }
    cof_result_free(&res);
    cof_genome_free(g);
    if (times)
        std::fprintf(stderr, "stage seconds: input %.4f load %.4f upload %.4f search %.4f "
                             "write %.4f free %.4f\n",
                     t_input, t_load, t_upload, t_search, t_write, lap());
    return 0;
}
