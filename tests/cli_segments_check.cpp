// Test driver for the tools' host-side file and segment logic
// (ktcountermemorygreedy_b200/cli/cli_common.h): no library call, no GPU.
//   cli_segments_check <tmp_dir> <budget_bytes> <dump 0|1> <with_low 0|1> <out_dir>
// writes to out_dir:
//   all_high.bin   key words (N u64), u32 count per record as read_tmpdir decodes high.bin
//   all_low.bin    key words per low.bin k-mer as read_tmpdir decodes it
//   seg_high.bin   key words, u32 count, u32 segment for every record load_segment returns
//   seg_low.bin    key words, u32 segment (with_low)
// (N = 1, 2 or 4 words per key by k)
//   plan.txt       "ok <n> <fixed> <per_high> <per_low>" then "p0 p1 n_high n_low" per segment,
//                  or "nofit <worst>"
#include <cstdio>
#include <string>
#include <vector>

#include "cli_common.h"

int main(int argc, char **argv)
{
    if (argc != 6) return 64;
    const std::string dir = cli::with_slash(argv[1]);
    const uint64_t budget = std::strtoull(argv[2], nullptr, 10);
    const bool dump = argv[3][0] == '1', with_low = argv[4][0] == '1';
    const std::string out = cli::with_slash(argv[5]);
    std::string err;
    cli::TmpDir t;
    if (!cli::read_tmpdir(dir, t, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 2; }
    FILE *f = std::fopen((out + "all_high.bin").c_str(), "wb");
    for (size_t i = 0; i < t.high_counts.size(); ++i) {
        std::fwrite(&t.high_keys[i * t.nw], 8, t.nw, f);
        std::fwrite(&t.high_counts[i], 4, 1, f);
    }
    std::fclose(f);
    f = std::fopen((out + "all_low.bin").c_str(), "wb");
    if (!t.low_keys.empty()) std::fwrite(t.low_keys.data(), 8, t.low_keys.size(), f);
    std::fclose(f);

    cli::Layout L;
    if (!cli::read_layout(dir, L, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 3; }
    std::vector<uint64_t> ph, pl;
    if (!cli::count_prefixes(dir, L, with_low, ph, pl, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 4; }
    const cli::SegCost cost = cli::seg_cost(L.k, dump, with_low, dump ? 0 : 10000);
    std::vector<cli::Segment> segs;
    uint32_t worst = 0;
    FILE *plan = std::fopen((out + "plan.txt").c_str(), "w");
    if (!cli::plan_segments(ph, pl, cost, budget, segs, &worst)) {
        std::fprintf(plan, "nofit %u\n", worst);
        std::fprintf(plan, "%s\n", cli::no_fit_message(L, ph, pl, cost, worst, budget).c_str());
        std::fclose(plan);
        return 0;
    }
    std::fprintf(plan, "ok %zu %llu %llu %llu\n", segs.size(), (unsigned long long)cost.fixed,
                 (unsigned long long)cost.per_high, (unsigned long long)cost.per_low);
    FILE *sh = std::fopen((out + "seg_high.bin").c_str(), "wb");
    FILE *sl = std::fopen((out + "seg_low.bin").c_str(), "wb");
    std::vector<uint64_t> hk, lk;
    std::vector<uint32_t> hc;
    for (uint32_t si = 0; si < segs.size(); ++si) {
        const cli::Segment &s = segs[si];
        std::fprintf(plan, "%u %u %llu %llu\n", s.p0, s.p1, (unsigned long long)s.n_high, (unsigned long long)s.n_low);
        if (!cli::load_segment(dir, L, with_low, s, hk, hc, lk, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 5; }
        for (size_t i = 0; i < hc.size(); ++i) {
            std::fwrite(&hk[i * L.nw], 8, L.nw, sh);
            std::fwrite(&hc[i], 4, 1, sh);
            std::fwrite(&si, 4, 1, sh);
        }
        for (size_t i = 0; i < lk.size() / L.nw; ++i) {
            std::fwrite(&lk[i * L.nw], 8, L.nw, sl);
            std::fwrite(&si, 4, 1, sl);
        }
    }
    std::fclose(sh);
    std::fclose(sl);
    std::fclose(plan);
    return 0;
}
