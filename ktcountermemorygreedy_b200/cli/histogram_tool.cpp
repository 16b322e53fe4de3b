// histogram_tool -- drop-in for the reference tool's command line
// (tool/histogram_tool.cpp:176-224, main :905):
//   histogram_tool <precise|approximate> <tmp_dir> <max_threads> <max_memory_gb> <output_file>
//                  [min_freq=1] [max_freq=10000]
// precise merges high.bin and low.bin on the GPU (kc_merge_records) and writes
// the histogram of the exact counts; approximate histograms high.bin only.
// When the records do not fit in max_memory_gb the histogram is summed over
// segments of the k-mers' first bases, each merged on its own (the reference
// falls back to its streaming mode there, tool/histogram_tool.cpp:801-813).
#include <iostream>

#include "cli_common.h"

static int segmented(const std::string &dir, const cli::Layout &L, bool precise, uint32_t lo, uint32_t hi,
                     uint64_t whole, uint64_t budget, const char *out)
{
    std::cout << "estimated_peak_memory_bytes=" << whole << " exceeds max_memory_bytes=" << budget
              << ", falling back to segmented mode" << std::endl;
    std::string err;
    std::vector<uint64_t> ph, pl;
    if (!cli::count_prefixes(dir, L, precise, ph, pl, err)) { std::cerr << err << std::endl; return 255; }
    const cli::SegCost cost = cli::seg_cost(L.k, false, precise, (uint64_t)hi - lo + 1);
    std::vector<cli::Segment> segs;
    uint32_t worst = 0;
    if (!cli::plan_segments(ph, pl, cost, budget, segs, &worst)) {
        std::cerr << cli::no_fit_message(L, ph, pl, cost, worst, budget) << std::endl;
        return 2;
    }
    std::cout << "Segmented mode: " << L.n_high() << " high records in " << segs.size() << " segment(s)" << std::endl;
    std::vector<int64_t> hist((uint64_t)hi - lo + 1, 0), part(hist.size());
    std::vector<uint64_t> hk, lk;
    std::vector<uint32_t> hc;
    for (const cli::Segment &s : segs) {
        if (!cli::load_segment(dir, L, precise, s, hk, hc, lk, err)) { std::cerr << err << std::endl; return 255; }
        uint64_t n = 0;
        int rc = kc_merge_records(hk.data(), hc.data(), hc.size(), precise ? lk.data() : nullptr,
                                  precise ? lk.size() / L.nw : 0, L.k, L.count_max, 1, 0xffffffffu, lo, hi, nullptr,
                                  nullptr, 0, &n, part.data());
        if (rc != KC_OK) { std::cerr << "histogram_tool: " << kc_last_error() << std::endl; return 2; }
        for (size_t i = 0; i < hist.size(); ++i) hist[i] += part[i];
    }
    if (!cli::write_hist(out, hist.data(), lo, hi)) {
        std::cerr << "failed to open output file: " << out << std::endl;
        return 1;
    }
    std::cout << "progress 100%" << std::endl;
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 6 || argc > 8) {
        std::cerr << "Usage: histogram_tool <precise/approximate> <tmp_dir> <max_threads> <max_memory_gb> "
                     "<output_file> [min_freq=1] [max_freq=10000]"
                  << std::endl;
        return 255;
    }
    bool precise;
    if (!std::strcmp(argv[1], "precise")) precise = true;
    else if (!std::strcmp(argv[1], "approximate")) precise = false;
    else {
        std::cerr << "invalid mode: must be 'precise' or 'approximate'" << std::endl;
        return 255;
    }
    uint32_t threads = 0, lo = 1, hi = 10000;
    if (!cli::parse_u32(argv[3], threads)) { std::cerr << "invalid max_threads" << std::endl; return 255; }
    uint64_t budget = 0;
    if (const int e = cli::parse_memory_gib(argv[4], budget)) {
        std::cerr << (e == 1 ? std::string("invalid max_memory_gb: ") + argv[4] : "max_memory_gb is too large")
                  << std::endl;
        return 255;
    }
    if (argc >= 7 && !cli::parse_u32(argv[6], lo)) { std::cerr << "invalid min_freq" << std::endl; return 255; }
    if (argc >= 8 && !cli::parse_u32(argv[7], hi)) { std::cerr << "invalid max_freq" << std::endl; return 255; }
    if (threads == 0) { std::cerr << "invalid max_threads: must be greater than 0" << std::endl; return 255; }
    if (hi < lo) { std::cerr << "invalid max_freq: must be greater than or equal to min_freq" << std::endl; return 255; }
    const std::string dir = cli::with_slash(argv[2]);
    std::string err;
    cli::Layout L;
    if (!cli::read_layout(dir, L, err)) { std::cerr << err << std::endl; return 255; }
    // all records at once: the larger file's bytes, then every decoded record
    const uint64_t kw = 8ull * L.nw;
    const uint64_t whole = std::max(L.high_bytes, L.low_bytes) + (kw + 4) * L.n_high() + kw * L.n_low() +
                           cli::seg_cost(L.k, false, precise, (uint64_t)hi - lo + 1).fixed;
    if (whole > budget) return segmented(dir, L, precise, lo, hi, whole, budget, argv[5]);
    cli::TmpDir t;
    if (!cli::read_tmpdir(dir, t, err)) { std::cerr << err << std::endl; return 255; }
    std::vector<int64_t> hist((uint64_t)hi - lo + 1, 0);
    uint64_t n = 0;
    int rc = kc_merge_records(t.high_keys.data(), t.high_counts.data(), t.n_high(),
                              precise ? t.low_keys.data() : nullptr, precise ? t.n_low() : 0, t.k, t.count_max,
                              1, 0xffffffffu, lo, hi, nullptr, nullptr, 0, &n, hist.data());
    if (rc != KC_OK) { std::cerr << "histogram_tool: " << kc_last_error() << std::endl; return 2; }
    if (!cli::write_hist(argv[5], hist.data(), lo, hi)) {
        std::cerr << "failed to open output file: " << argv[5] << std::endl;
        return 1;
    }
    std::cout << "progress 100%" << std::endl;
    return 0;
}
