// fastq_gen -- writes a seeded synthetic FASTQ workload to a file, as a
// program of its own, so that a process timing the reference's CPU programs
// can produce its input without loading any library of this project.
//
//   fastq_gen large <genome_bp> <first_read> <n_reads> <out.fq>
//       the single large job's read stream (seed 2): a genome of <genome_bp>
//       bases, 5% of it from 200 repeat families of 1-5 kbp with 10-500 copies
//       (scaled to the 5% total) at 2% divergence; 150 bp reads at 1%
//       substitutions; reads <first_read> .. <first_read> + <n_reads> - 1 of
//       the stream (the same bytes libkcgen.so writes for those reads).
//
//   fastq_gen outofcore <genome_bp> <first_read> <n_reads> <out.fq>
//       the out-of-core job's read stream (seed 5): 45% of the genome from
//       2000 repeat families of 0.3-6 kbp with 1-10^5 copies (scaled to the
//       45% total), each family at a divergence drawn from U[1%, 15%]; 150 bp
//       reads at 1% substitutions.
//
// Exit status 0 on success, 1 on a usage error, 2 when the file cannot be
// written.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "../csrc/fastq_gen.cpp"

namespace {

int usage()
{
    std::fprintf(stderr, "usage: fastq_gen large|outofcore <genome_bp> <first_read> <n_reads> <out.fq>\n");
    return 1;
}

bool parse_u64(const char *s, uint64_t &v)
{
    char *end = nullptr;
    v = std::strtoull(s, &end, 10);
    return end && *end == '\0' && end != s;
}

}  // namespace

int main(int argc, char **argv)
{
    const std::string mode = argc == 6 ? argv[1] : "";
    if (mode != "large" && mode != "outofcore") return usage();
    const uint64_t seed = mode == "large" ? 2 : 5;
    uint64_t glen = 0, first = 0, n = 0;
    if (!parse_u64(argv[2], glen) || !parse_u64(argv[3], first) || !parse_u64(argv[4], n) || glen < 1000)
        return usage();
    const int threads = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<char> genome(glen);
    if (mode == "large") kcgen_genome(2, glen, 0.05, 200, 1000, 5000, 10, 500, 0.02, genome.data(), threads);
    else kcgen_genome_div(5, glen, 0.45, 2000, 300, 6000, 1, 100000, 0.01, 0.15, genome.data(), threads);
    FILE *f = std::fopen(argv[5], "wb");
    if (!f) {
        std::perror(argv[5]);
        return 2;
    }
    // in pieces of at most 1M reads: the reads are seeded by their index, so
    // the pieces are the bytes of one stream
    const uint64_t piece = 1u << 20;
    std::vector<char> buf;
    for (uint64_t a = 0; a < n; a += piece) {
        const uint64_t m = std::min(piece, n - a);
        const uint64_t size = kcgen_reads_size(seed, first + a, m, 150, 150);
        buf.resize(size);
        if (kcgen_reads(genome.data(), glen, seed, first + a, m, 150, 150, 0.01, 0.0, buf.data(), size, threads) != size ||
            std::fwrite(buf.data(), 1, size, f) != size) {
            std::fclose(f);
            std::fprintf(stderr, "fastq_gen: writing %s failed\n", argv[5]);
            return 2;
        }
    }
    if (std::fclose(f) != 0) return 2;
    return 0;
}
