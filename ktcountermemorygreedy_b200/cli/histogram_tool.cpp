// histogram_tool -- drop-in for the reference tool's command line
// (tool/histogram_tool.cpp:176-224, main :905):
//   histogram_tool <precise|approximate> <tmp_dir> <max_threads> <max_memory_gb> <output_file>
//                  [min_freq=1] [max_freq=10000]
// precise merges high.bin and low.bin on the GPU (kc_merge_records) and writes
// the histogram of the exact counts; approximate histograms high.bin only.
#include <iostream>

#include "cli_common.h"

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
    double mem = std::atof(argv[4]);
    if (!(mem > 0)) { std::cerr << "invalid max_memory_gb: " << argv[4] << std::endl; return 255; }
    if (argc >= 7 && !cli::parse_u32(argv[6], lo)) { std::cerr << "invalid min_freq" << std::endl; return 255; }
    if (argc >= 8 && !cli::parse_u32(argv[7], hi)) { std::cerr << "invalid max_freq" << std::endl; return 255; }
    if (threads == 0) { std::cerr << "invalid max_threads: must be greater than 0" << std::endl; return 255; }
    if (hi < lo) { std::cerr << "invalid max_freq: must be greater than or equal to min_freq" << std::endl; return 255; }
    cli::TmpDir t;
    std::string err;
    if (!cli::read_tmpdir(cli::with_slash(argv[2]), t, err)) { std::cerr << err << std::endl; return 255; }
    std::vector<int64_t> hist((uint64_t)hi - lo + 1, 0);
    uint64_t n = 0;
    int rc = kc_merge_records(t.high_keys.data(), t.high_counts.data(), t.high_keys.size(),
                              precise ? t.low_keys.data() : nullptr, precise ? t.low_keys.size() : 0, t.k, t.count_max,
                              1, 0xffffffffu, lo, hi, nullptr, nullptr, 0, &n, hist.data());
    if (rc != KC_OK) { std::cerr << "histogram_tool: " << kc_last_error() << std::endl; return 2; }
    if (!cli::write_hist(argv[5], hist.data(), lo, hi)) {
        std::cerr << "failed to open output file: " << argv[5] << std::endl;
        return 1;
    }
    std::cout << "progress 100%" << std::endl;
    return 0;
}
