// fastq_gen.cpp -- seeded synthetic FASTQ for the benchmark and test
// workloads (libkcgen.so).  The reference measures no public dataset; these
// inputs stand in with the shapes of its workloads: uniform-ACGT genomes,
// optional repeat families, reads sampled at uniform positions from either
// strand, uniform substitution errors, optional N bases, Phred+33 qualities
// uniform in [20, 40].
//
// Every read draws from its own generator seeded by (seed, read index), so the
// output is identical for any thread count.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

uint64_t mix_seed(uint64_t a, uint64_t b)
{
    Rng r(a * 0xD1B54A32D192ED03ULL ^ (b + 0x8CB92BA72F3D8DD7ULL));
    r.next();
    return r.next();
}

const char BASES[4] = {'A', 'C', 'G', 'T'};

inline char comp(char c)
{
    switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return 'N';
    }
}

uint32_t digits(uint64_t v)
{
    uint32_t d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
}

template <typename F>
void parallel_for(uint64_t n, int threads, F f)
{
    if (threads <= 1 || n < 1024) { f(0, n); return; }
    std::vector<std::thread> ts;
    uint64_t per = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        uint64_t a = t * per, b = std::min(n, a + per);
        if (a >= b) break;
        ts.emplace_back([=] { f(a, b); });
    }
    for (auto &t : ts) t.join();
}

struct ReadPlan {
    uint64_t n_reads;
    uint32_t len_min, len_max;
    std::vector<uint32_t> lens;
    std::vector<uint64_t> offs;
    uint64_t total = 0;
};

void plan_reads(ReadPlan &p, uint64_t seed, uint64_t first_id)
{
    p.lens.resize(p.n_reads);
    p.offs.resize(p.n_reads + 1);
    uint64_t off = 0;
    for (uint64_t i = 0; i < p.n_reads; ++i) {
        uint32_t L = p.len_min;
        if (p.len_max > p.len_min) {
            Rng r(mix_seed(seed ^ 0x5eedULL, first_id + i));
            L = p.len_min + (uint32_t)r.below(p.len_max - p.len_min + 1);
        }
        p.lens[i] = L;
        p.offs[i] = off;
        off += 2 + digits(first_id + i) + 1 + L + 1 + 2 + L + 1;   // "@r<id>\n<seq>\n+\n<qual>\n"
    }
    p.offs[p.n_reads] = off;
    p.total = off;
}

}  // namespace

extern "C" {

// Genome of `length` bases.  When repeat_frac > 0, n_families family
// sequences of length U[fam_min, fam_max] are drawn, each with a divergence
// U[div_min, div_max] (no draw when they are equal), copy counts
// U[copies_min, copies_max] are scaled so that all copies together cover
// repeat_frac of the genome, and each copy is written at a uniform position
// with its family's per-base substitution rate.  Returns the repeat bases
// placed.
uint64_t kcgen_genome_div(uint64_t seed, uint64_t length, double repeat_frac, uint32_t n_families,
                          uint32_t fam_min, uint32_t fam_max, uint32_t copies_min, uint32_t copies_max,
                          double div_min, double div_max, char *out, int threads)
{
    parallel_for((length + 4095) / 4096, threads, [&](uint64_t a, uint64_t b) {
        for (uint64_t blk = a; blk < b; ++blk) {
            Rng r(mix_seed(seed, blk));
            uint64_t s = blk * 4096, e = std::min(length, s + 4096);
            for (uint64_t i = s; i < e; i += 32) {
                uint64_t v = r.next();
                for (uint64_t j = i; j < std::min(e, i + 32); ++j, v >>= 2) out[j] = BASES[v & 3];
            }
        }
    });
    if (repeat_frac <= 0.0 || n_families == 0) return 0;
    Rng r(mix_seed(seed, 0xfa111e5ULL));
    std::vector<std::string> fams(n_families);
    std::vector<double> copies(n_families), div(n_families, div_min);
    double want = repeat_frac * (double)length, raw = 0.0;
    for (uint32_t f = 0; f < n_families; ++f) {
        uint32_t L = fam_min + (uint32_t)r.below(fam_max - fam_min + 1);
        fams[f].resize(L);
        for (uint32_t i = 0; i < L; ++i) fams[f][i] = BASES[r.next() & 3];
        copies[f] = copies_min + (double)r.below(copies_max - copies_min + 1);
        if (div_max > div_min) div[f] = div_min + (div_max - div_min) * r.uniform();
        raw += copies[f] * L;
    }
    double scale = raw > 0 ? want / raw : 0.0;
    uint64_t placed = 0;
    for (uint32_t f = 0; f < n_families; ++f) {
        uint64_t n = (uint64_t)std::llround(copies[f] * scale);
        const std::string &fam = fams[f];
        if (fam.size() >= length) continue;
        for (uint64_t c = 0; c < n; ++c) {
            uint64_t pos = r.below(length - fam.size());
            for (size_t i = 0; i < fam.size(); ++i) {
                char b = fam[i];
                if (r.uniform() < div[f]) b = BASES[(((b == 'A') ? 0 : (b == 'C') ? 1 : (b == 'G') ? 2 : 3) + 1 + r.below(3)) & 3];
                out[pos + i] = b;
            }
            placed += fam.size();
        }
    }
    return placed;
}

// kcgen_genome_div with one divergence for every family.
uint64_t kcgen_genome(uint64_t seed, uint64_t length, double repeat_frac, uint32_t n_families,
                      uint32_t fam_min, uint32_t fam_max, uint32_t copies_min, uint32_t copies_max,
                      double divergence, char *out, int threads)
{
    return kcgen_genome_div(seed, length, repeat_frac, n_families, fam_min, fam_max, copies_min, copies_max, divergence,
                            divergence, out, threads);
}

// Exact FASTQ size of kcgen_reads with the same arguments.
uint64_t kcgen_reads_size(uint64_t seed, uint64_t first_id, uint64_t n_reads, uint32_t len_min,
                          uint32_t len_max)
{
    ReadPlan p{n_reads, len_min, len_max, {}, {}, 0};
    plan_reads(p, seed, first_id);
    return p.total;
}

// Reads sampled from `genome` as FASTQ records "@r<id>\n<seq>\n+\n<qual>\n".
// Returns the bytes written, or 0 if `cap` is too small.
uint64_t kcgen_reads(const char *genome, uint64_t glen, uint64_t seed, uint64_t first_id,
                     uint64_t n_reads, uint32_t len_min, uint32_t len_max, double sub_rate,
                     double n_rate, char *out, uint64_t cap, int threads)
{
    ReadPlan p{n_reads, len_min, len_max, {}, {}, 0};
    plan_reads(p, seed, first_id);
    if (p.total > cap) return 0;
    parallel_for(n_reads, threads, [&](uint64_t a, uint64_t b) {
        std::vector<char> tmp(std::max(len_max, len_min) + 1);
        for (uint64_t i = a; i < b; ++i) {
            Rng r(mix_seed(seed, first_id + i));
            uint32_t L = p.lens[i];
            char *o = out + p.offs[i];
            *o++ = '@';
            *o++ = 'r';
            uint64_t id = first_id + i;
            uint32_t nd = digits(id);
            for (uint32_t d = 0; d < nd; ++d) { o[nd - 1 - d] = (char)('0' + id % 10); id /= 10; }
            o += nd;
            *o++ = '\n';
            uint64_t pos = glen > L ? r.below(glen - L + 1) : 0;
            bool rev = r.next() & 1;
            for (uint32_t j = 0; j < L; ++j) {
                char c = (pos + j < glen) ? genome[pos + j] : 'A';
                tmp[j] = c;
            }
            if (rev) {
                std::reverse(tmp.begin(), tmp.begin() + L);
                for (uint32_t j = 0; j < L; ++j) tmp[j] = comp(tmp[j]);
            }
            for (uint32_t j = 0; j < L; ++j) {
                char c = tmp[j];
                if (sub_rate > 0 && r.uniform() < sub_rate) {
                    int code = (c == 'A') ? 0 : (c == 'C') ? 1 : (c == 'G') ? 2 : 3;
                    c = BASES[(code + 1 + r.below(3)) & 3];
                }
                if (n_rate > 0 && r.uniform() < n_rate) c = 'N';
                o[j] = c;
            }
            o += L;
            *o++ = '\n';
            *o++ = '+';
            *o++ = '\n';
            for (uint32_t j = 0; j < L; ++j) o[j] = (char)(33 + 20 + r.below(21));
            o += L;
            *o++ = '\n';
        }
    });
    return p.total;
}

}  // extern "C"
