// dump_tool -- drop-in for the reference tool's command line
// (tool/dump_tool.cpp:493-537, main :1447):
//   dump_tool <precise|approximate> <tmp_dir> <max_threads> <max_memory_gb> <output_file>
//             [min_freq] [max_freq] [--sort]
// precise writes every k-mer whose exact merged count is in [min_freq,
// max_freq]; approximate writes the high.bin records in range.  Lines are
// always in printed-string order (the --sort order).  For min_freq > 1 the
// reference's precise mode drops k-mers whose high.bin part is below
// min_freq (tool/dump_tool.cpp:717); this tool writes the exact set.  When
// the records do not fit in max_memory_gb they are merged and written in
// segments of the k-mers' first bases, one after the other (the reference
// falls back to its partitioned mode there, tool/dump_tool.cpp:1280-1290).
#include <iostream>

#include "cli_common.h"

static int segmented(const std::string &dir, const cli::Layout &L, bool precise, uint32_t lo, uint32_t hi,
                     uint64_t whole, uint64_t budget, const char *out)
{
    std::cout << "estimated memory " << whole << " exceeds max_memory_bytes=" << budget
              << ", falling back to segmented mode" << std::endl;
    std::string err;
    std::vector<uint64_t> ph, pl;
    if (!cli::count_prefixes(dir, L, precise, ph, pl, err)) { std::cerr << err << '\n'; return 255; }
    const cli::SegCost cost = cli::seg_cost(L.k, true, precise, 0);
    std::vector<cli::Segment> segs;
    uint32_t worst = 0;
    if (!cli::plan_segments(ph, pl, cost, budget, segs, &worst)) {
        std::cerr << cli::no_fit_message(L, ph, pl, cost, worst, budget) << '\n';
        return 2;
    }
    std::cout << "Segmented mode: " << L.n_high() << " high records in " << segs.size() << " segment(s)" << std::endl;
    FILE *f = std::fopen(out, "wb");
    if (!f) { std::cerr << "dump_tool: failed to open " << out << '\n'; return 1; }
    std::vector<uint64_t> hk, lk, keys;
    std::vector<uint32_t> hc, counts;
    for (const cli::Segment &s : segs) {
        if (!cli::load_segment(dir, L, precise, s, hk, hc, lk, err)) {
            std::fclose(f);
            std::cerr << err << '\n';
            return 255;
        }
        const uint64_t cap = hc.size() + lk.size() / L.nw;
        keys.resize(std::max<uint64_t>(cap, 1) * L.nw);
        counts.resize(std::max<uint64_t>(cap, 1));
        uint64_t n = 0;
        int rc = kc_merge_records(hk.data(), hc.data(), hc.size(), precise ? lk.data() : nullptr,
                                  precise ? lk.size() / L.nw : 0, L.k, L.count_max, lo, hi, 1, 1, keys.data(),
                                  counts.data(), cap, &n, nullptr);
        if (rc != KC_OK) {
            std::fclose(f);
            std::cerr << "dump_tool: " << kc_last_error() << '\n';
            return 2;
        }
        if (!cli::append_dump(f, keys.data(), counts.data(), std::min(n, cap), L.k, err)) {
            std::fclose(f);
            std::cerr << "dump_tool: " << err << '\n';
            return 1;
        }
    }
    if (std::fclose(f) != 0) { std::cerr << "dump_tool: failed to write " << out << '\n'; return 1; }
    std::cout << "progress 100%" << std::endl;
    return 0;
}

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
    uint64_t budget = 0;
    if (const int e = cli::parse_memory_gib(argv[4], budget)) {
        std::cerr << (e == 1 ? std::string("invalid max_memory_gb: ") + argv[4] : "max_memory_gb too large") << '\n';
        return 255;
    }
    int next = 6;
    if (argc > next && argv[next][0] != '-') { if (!cli::parse_u32(argv[next++], lo)) { std::cerr << "invalid min_freq\n"; return 255; } }
    if (argc > next && argv[next][0] != '-') { if (!cli::parse_u32(argv[next++], hi)) { std::cerr << "invalid max_freq\n"; return 255; } }
    if (hi < lo) { std::cerr << "max_freq < min_freq\n"; return 255; }
    const std::string dir = cli::with_slash(argv[2]);
    std::string err;
    cli::Layout L;
    if (!cli::read_layout(dir, L, err)) { std::cerr << err << '\n'; return 255; }
    // all records at once: the larger file's bytes, every decoded record, and
    // the merged records with their text
    const uint64_t n_out = L.n_high() + (precise ? L.n_low() : 0);
    const uint64_t kw = 8ull * L.nw;
    const uint64_t whole = std::max(L.high_bytes, L.low_bytes) + (kw + 4) * L.n_high() + kw * L.n_low() +
                           (kw + 16 + (uint64_t)L.k) * n_out + cli::seg_cost(L.k, true, precise, 0).fixed;
    if (whole > budget) return segmented(dir, L, precise, lo, hi, whole, budget, argv[5]);
    cli::TmpDir t;
    if (!cli::read_tmpdir(dir, t, err)) { std::cerr << err << '\n'; return 255; }
    const uint64_t cap = t.n_high() + (precise ? t.n_low() : 0);
    std::vector<uint64_t> keys(std::max<uint64_t>(cap, 1) * t.nw);
    std::vector<uint32_t> counts(std::max<uint64_t>(cap, 1));
    uint64_t n = 0;
    int rc = kc_merge_records(t.high_keys.data(), t.high_counts.data(), t.n_high(),
                              precise ? t.low_keys.data() : nullptr, precise ? t.n_low() : 0, t.k, t.count_max,
                              lo, hi, 1, 1, keys.data(), counts.data(), cap, &n, nullptr);
    if (rc != KC_OK) { std::cerr << "dump_tool: " << kc_last_error() << '\n'; return 2; }
    if (!cli::write_dump(argv[5], keys.data(), counts.data(), std::min(n, cap), t.k, err)) {
        std::cerr << "dump_tool: " << err << '\n';
        return 1;
    }
    std::cout << "progress 100%" << std::endl;
    return 0;
}
