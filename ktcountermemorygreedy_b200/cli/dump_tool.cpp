// dump_tool -- drop-in for the reference tool's command line
// (tool/dump_tool.cpp:493-537, main :1447):
//   dump_tool <precise|approximate> <tmp_dir> <max_threads> <max_memory_gb> <output_file>
//             [min_freq] [max_freq] [--sort]
// precise writes every k-mer whose exact merged count is in [min_freq,
// max_freq]; approximate writes the high.bin records in range.  Lines are
// always in printed-string order (the --sort order).  For min_freq > 1 the
// reference's precise mode drops k-mers whose high.bin part is below
// min_freq (tool/dump_tool.cpp:717); this tool writes the exact set.
#include <iostream>

#include "cli_common.h"

int main(int argc, char **argv)
{
    if (argc < 6 || argc > 9) {
        std::cerr << "Usage: dump_tool <precise/approximate> <tmp_dir> <max_threads> <max_memory_gb> <output_file> "
                     "[min_freq] [max_freq] [--sort]\n";
        return 255;
    }
    bool precise;
    if (!std::strcmp(argv[1], "precise")) precise = true;
    else if (!std::strcmp(argv[1], "approximate")) precise = false;
    else { std::cerr << "mode must be precise or approximate\n"; return 255; }
    uint32_t threads = 0, lo = 1, hi = 0xffffffffu;
    if (!cli::parse_u32(argv[3], threads) || threads == 0) { std::cerr << "invalid max_threads\n"; return 255; }
    double mem = std::atof(argv[4]);
    if (!(mem > 0)) { std::cerr << "invalid max_memory_gb: " << argv[4] << '\n'; return 255; }
    int next = 6;
    if (argc > next && argv[next][0] != '-') { if (!cli::parse_u32(argv[next++], lo)) { std::cerr << "invalid min_freq\n"; return 255; } }
    if (argc > next && argv[next][0] != '-') { if (!cli::parse_u32(argv[next++], hi)) { std::cerr << "invalid max_freq\n"; return 255; } }
    if (hi < lo) { std::cerr << "max_freq < min_freq\n"; return 255; }
    cli::TmpDir t;
    std::string err;
    if (!cli::read_tmpdir(cli::with_slash(argv[2]), t, err)) { std::cerr << err << '\n'; return 255; }
    const uint64_t cap = t.high_keys.size() + (precise ? t.low_keys.size() : 0);
    std::vector<uint64_t> keys(std::max<uint64_t>(cap, 1));
    std::vector<uint32_t> counts(std::max<uint64_t>(cap, 1));
    uint64_t n = 0;
    int rc = kc_merge_records(t.high_keys.data(), t.high_counts.data(), t.high_keys.size(),
                              precise ? t.low_keys.data() : nullptr, precise ? t.low_keys.size() : 0, t.k, t.count_max,
                              lo, hi, 1, 1, keys.data(), counts.data(), cap, &n, nullptr);
    if (rc != KC_OK) { std::cerr << "dump_tool: " << kc_last_error() << '\n'; return 2; }
    if (!cli::write_dump(argv[5], keys.data(), counts.data(), std::min(n, cap), t.k, err)) {
        std::cerr << "dump_tool: " << err << '\n';
        return 1;
    }
    std::cout << "progress 100%" << std::endl;
    return 0;
}
