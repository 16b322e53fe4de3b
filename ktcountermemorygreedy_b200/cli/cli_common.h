// cli_common.h -- helpers shared by the reference-compatible command-line
// programs: argument parsing with the reference's messages, file IO in the
// reference's tmp_dir formats, and text output.
#pragma once

#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "kc.h"

namespace cli {

inline bool parse_u32(const char *s, uint32_t &out)
{
    char *end = nullptr;
    errno = 0;
    unsigned long long v = std::strtoull(s, &end, 10);
    if (errno || !end || *end || end == s || v > 0xffffffffULL) return false;
    out = (uint32_t)v;
    return true;
}

inline bool parse_u64(const char *s, uint64_t &out)
{
    char *end = nullptr;
    errno = 0;
    unsigned long long v = std::strtoull(s, &end, 10);
    if (errno || !end || *end || end == s) return false;
    out = v;
    return true;
}

inline std::string with_slash(std::string d)
{
    if (d.empty()) return "./";
    if (d.back() != '/') d += '/';
    return d;
}

inline bool read_file(const std::string &path, std::vector<char> &out)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    size_t got = n > 0 ? std::fread(out.data(), 1, (size_t)n, f) : 0;
    std::fclose(f);
    return got == out.size();
}

// Same input forms as the reference counter (src/main.cpp:498-531): a
// directory (entries not starting with '.', sorted), or a comma list.
inline std::vector<std::string> input_files(const std::string &arg)
{
    std::vector<std::string> names;
    struct stat st;
    if (::stat(arg.c_str(), &st) == 0 && S_ISDIR(st.st_mode)) {
        DIR *d = ::opendir(arg.c_str());
        if (!d) return names;
        while (struct dirent *e = ::readdir(d)) {
            if (e->d_name[0] == '.') continue;
            names.push_back(arg + "/" + e->d_name);
        }
        ::closedir(d);
        std::sort(names.begin(), names.end());
    } else {
        std::string s = arg;
        size_t pos;
        while ((pos = s.find(',')) != std::string::npos) {
            names.push_back(s.substr(0, pos));
            s.erase(0, pos + 1);
        }
        if (!s.empty()) names.push_back(s);
    }
    return names;
}

// 64-bit words of one decoded k-mer: the reference's kmer<N>, N = 1 for
// k <= 32, 2 for k <= 64, 4 for k <= 128 (src/main.cpp:617-633).
inline uint32_t key_words_for(uint32_t k) { return k <= 32 ? 1u : (k <= 64 ? 2u : 4u); }

inline uint32_t count_bytes_for(uint32_t count_max)
{
    return count_max <= 0xFF ? 1 : count_max <= 0xFFFF ? 2 : count_max <= 0xFFFFFF ? 3 : 4;
}

// The records of a tmp_dir; keys are kmer<N> word arrays, nw words each.
struct TmpDir {
    uint32_t k = 0, count_max = 0, count_bytes = 4, nw = 1;
    std::vector<uint64_t> high_keys;
    std::vector<uint32_t> high_counts;
    std::vector<uint64_t> low_keys;
    uint64_t n_high() const { return high_counts.size(); }
    uint64_t n_low() const { return low_keys.size() / nw; }
};

// Record geometry of a tmp_dir, from infos.bin: a k-mer takes kb bytes (full
// words, then the tail bytes of the next word), a high.bin record kb +
// count_bytes (src/main.cpp:590-615, src/FinalDrainWriter.h:71-88); decoded,
// a k-mer is nw words (the reference's kmer<N>, src/main.cpp:617-633).
struct Layout {
    uint32_t k = 0, count_max = 0, count_bytes = 4;
    uint32_t full = 0, tail_bytes = 0, kb = 0, rec = 0, nw = 1;
    uint64_t high_bytes = 0, low_bytes = 0;   // file sizes (read_layout)
    uint64_t n_high() const { return high_bytes / rec; }
    uint64_t n_low() const { return low_bytes / kb; }
};

inline bool read_infos(const std::string &dir, Layout &L, std::string &err)
{
    std::vector<char> b;
    if (!read_file(dir + "infos.bin", b) || b.size() < 8) { err = "failed to read " + dir + "infos.bin"; return false; }
    std::memcpy(&L.k, b.data(), 4);
    std::memcpy(&L.count_max, b.data() + 4, 4);
    L.count_bytes = count_bytes_for(L.count_max);
    if (L.k == 0 || L.k > 128) { err = "invalid k_len from infos.bin: " + std::to_string(L.k); return false; }
    L.tail_bytes = (2 * (L.k % 32) + 7) / 8;
    L.full = L.k / 32;
    L.kb = L.full * 8 + L.tail_bytes;
    L.rec = L.kb + L.count_bytes;
    L.nw = key_words_for(L.k);
    return true;
}

// The kmer<N> words of one packed k-mer (the inverse of the reference's
// packing): the full words, then the tail bytes at the top of the next word.
inline void decode_key(const char *r, const Layout &L, uint64_t *w)
{
    for (uint32_t i = 0; i < L.nw; ++i) w[i] = 0;
    std::memcpy(w, r, L.full * 8);
    if (L.tail_bytes) std::memcpy(reinterpret_cast<char *>(w + L.full) + (8 - L.tail_bytes), r + L.full * 8, L.tail_bytes);
}

// infos.bin, high.bin, low.bin as written by the reference counter
// (src/main.cpp:590-615, src/FinalDrainWriter.h:71-88, src/ExportWriter.h:296-313)
// and read by its tools (tool/histogram_tool.cpp:239-366).
inline bool read_tmpdir(const std::string &dir, TmpDir &t, std::string &err)
{
    Layout L;
    if (!read_infos(dir, L, err)) return false;
    t.k = L.k;
    t.count_max = L.count_max;
    t.count_bytes = L.count_bytes;
    std::vector<char> b;
    if (!read_file(dir + "high.bin", b)) { err = "failed to open " + dir + "high.bin"; return false; }
    if (b.empty()) { err = "empty high.bin file"; return false; }
    if (b.size() % L.rec) { err = "invalid high.bin file size"; return false; }
    size_t n = b.size() / L.rec;
    t.nw = L.nw;
    t.high_keys.resize(n * L.nw);
    t.high_counts.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const char *r = b.data() + i * L.rec;
        uint32_t c = 0;
        std::memcpy(&c, r + L.kb, L.count_bytes);
        decode_key(r, L, t.high_keys.data() + i * L.nw);
        t.high_counts[i] = c;
    }
    if (!read_file(dir + "low.bin", b)) { err = "failed to open " + dir + "low.bin"; return false; }
    if (b.size() % L.kb) { err = "invalid low.bin size"; return false; }
    n = b.size() / L.kb;
    t.low_keys.resize(n * L.nw);
    for (size_t i = 0; i < n; ++i) decode_key(b.data() + i * L.kb, L, t.low_keys.data() + i * L.nw);
    return true;
}

// ---------------------------------------------------------------------------
// Segmented mode: records that do not fit in max_memory_gb
// ---------------------------------------------------------------------------
//
// The reference tools fall back to a streaming histogram over segments of
// high.bin (tool/histogram_tool.cpp:510-600, :801-813) and to a dump over
// hash partitions written to tmp_dir and merged afterwards
// (tool/dump_tool.cpp:938-1110, :1280-1290; tool/Partition.h:472-655) when
// their estimated peak memory exceeds max_memory_gb.  Here a segment is a
// contiguous range of the k-mers' first bases in printed-string order: every
// k-mer's high.bin and low.bin parts fall in the same segment, each segment is
// merged on its own, and the segments' sorted records follow one another in
// the dump's order, so nothing is written to tmp_dir and nothing is merged
// afterwards.  A counting pass over the files plans the segments; each
// segment then reads the files again and keeps its own records.

constexpr uint32_t SEG_LEAD_BASES = 8;                    // first bases that place a k-mer (4^8 ranges)
constexpr uint64_t SEG_BLOCK_BYTES = 1ull << 20;          // file read block
constexpr uint64_t SEG_SLACK_BYTES = 4ull << 20;

inline uint32_t lead_bases(uint32_t k) { return std::min<uint32_t>(k, SEG_LEAD_BASES); }

// Base i of the printed k-mer (kmer_to_buf, tool/dump_tool.cpp:103-124): for
// k <= 32 bit 64 - 2k + 2i of the word; otherwise the first k % 32 bases from
// the top of word k / 32, the others from word k / 32 - 1 downwards, each
// word from its low bits up.
inline uint32_t key_base(const uint64_t *w, uint32_t k, uint32_t i)
{
    if (k <= 32) return (uint32_t)(w[0] >> (64 - 2 * k + 2 * i)) & 3u;
    const uint32_t full = k / 32, tail = k % 32;
    if (i < tail) return (uint32_t)(w[full] >> (64 - 2 * tail + 2 * i)) & 3u;
    const uint32_t off = i - tail;
    return (uint32_t)(w[full - 1 - off / 32] >> (2 * (off % 32))) & 3u;
}

// The first m bases of the printed k-mer as a number, base 0 most significant.
inline uint32_t lead_prefix(const uint64_t *w, uint32_t k, uint32_t m)
{
    uint32_t p = 0;
    for (uint32_t i = 0; i < m; ++i) p = (p << 2) | key_base(w, k, i);
    return p;
}

inline std::string prefix_string(uint32_t p, uint32_t m)
{
    std::string s(m, 'A');
    for (uint32_t i = 0; i < m; ++i) s[m - 1 - i] = "ACGT"[(p >> (2 * i)) & 3];
    return s;
}

// infos.bin plus the sizes of high.bin and low.bin, with read_tmpdir's checks.
inline bool read_layout(const std::string &dir, Layout &L, std::string &err)
{
    if (!read_infos(dir, L, err)) return false;
    struct stat sh, sl;
    if (::stat((dir + "high.bin").c_str(), &sh) != 0 || !S_ISREG(sh.st_mode)) {
        err = "failed to open " + dir + "high.bin";
        return false;
    }
    if (sh.st_size == 0) { err = "empty high.bin file"; return false; }
    if ((uint64_t)sh.st_size % L.rec) { err = "invalid high.bin file size"; return false; }
    if (::stat((dir + "low.bin").c_str(), &sl) != 0 || !S_ISREG(sl.st_mode)) {
        err = "failed to open " + dir + "low.bin";
        return false;
    }
    if ((uint64_t)sl.st_size % L.kb) { err = "invalid low.bin size"; return false; }
    L.high_bytes = (uint64_t)sh.st_size;
    L.low_bytes = (uint64_t)sl.st_size;
    return true;
}

// Calls f(key words, count) for every record of high.bin (low = false) or
// every k-mer of low.bin (low = true, count 0), reading whole records in blocks.
template <class F>
inline bool scan_file(const std::string &dir, const Layout &L, bool low, F &&f, std::string &err)
{
    const std::string path = dir + (low ? "low.bin" : "high.bin");
    const uint64_t rec = low ? L.kb : L.rec;
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) { err = "failed to open " + path; return false; }
    std::vector<char> buf((size_t)(SEG_BLOCK_BYTES / rec * rec));
    const uint64_t total = low ? L.low_bytes : L.high_bytes;
    uint64_t done = 0;
    while (done < total) {
        const size_t want = (size_t)std::min<uint64_t>(buf.size(), total - done);
        if (std::fread(buf.data(), 1, want, fp) != want) {
            std::fclose(fp);
            err = "failed to read " + path;
            return false;
        }
        uint64_t w[4];
        for (size_t o = 0; o < want; o += rec) {
            uint32_t c = 0;
            if (!low) std::memcpy(&c, buf.data() + o + L.kb, L.count_bytes);
            decode_key(buf.data() + o, L, w);
            f(static_cast<const uint64_t *>(w), c);
        }
        done += want;
    }
    std::fclose(fp);
    return true;
}

struct Segment {
    uint32_t p0 = 0, p1 = 0;            // lead prefixes [p0, p1)
    uint64_t n_high = 0, n_low = 0;
};

// Host bytes of one merge: per high.bin record, per low.bin k-mer (0 when
// low.bin is not read), and fixed (read block, prefix counts, histogram, slack).
struct SegCost {
    uint64_t per_high = 0, per_low = 0, fixed = 0;
};

inline SegCost seg_cost(uint32_t k, bool dump, bool with_low, uint64_t hist_bins)
{
    SegCost c;
    // input keys + counts; dump: output keys + counts and the text line (k bases, tab,
    // at most 10 digits, newline)
    const uint64_t kw = 8ull * key_words_for(k);
    const uint64_t out = dump ? kw + 4 + (uint64_t)k + 12 : 0;
    c.per_high = kw + 4 + out;
    c.per_low = with_low ? kw + out : 0;
    const uint64_t prefixes = 1ull << (2 * lead_bases(k));
    c.fixed = SEG_SLACK_BYTES + SEG_BLOCK_BYTES + 2 * prefixes * 8 + hist_bins * 16;
    return c;
}

// Contiguous prefix ranges, each as large as fits in `budget` bytes.  False
// (with the prefix that alone does not fit in *worst) when no plan fits.
inline bool plan_segments(const std::vector<uint64_t> &ph, const std::vector<uint64_t> &pl, const SegCost &c,
                          uint64_t budget, std::vector<Segment> &out, uint32_t *worst)
{
    out.clear();
    if (budget <= c.fixed) {
        if (worst) *worst = ~0u;
        return false;
    }
    const uint64_t room = budget - c.fixed;
    Segment s;
    uint64_t used = 0;
    for (uint32_t p = 0; p < (uint32_t)ph.size(); ++p) {
        const uint64_t b = ph[p] * c.per_high + pl[p] * c.per_low;
        if (b > room) {
            if (worst) *worst = p;
            return false;
        }
        if (used + b > room) {
            s.p1 = p;
            out.push_back(s);
            s = Segment{};
            s.p0 = p;
            used = 0;
        }
        used += b;
        s.n_high += ph[p];
        s.n_low += pl[p];
    }
    s.p1 = (uint32_t)ph.size();
    out.push_back(s);
    return true;
}

// Counting pass: records per lead prefix in high.bin and (with_low) low.bin.
inline bool count_prefixes(const std::string &dir, const Layout &L, bool with_low, std::vector<uint64_t> &ph,
                           std::vector<uint64_t> &pl, std::string &err)
{
    const uint32_t m = lead_bases(L.k);
    ph.assign((size_t)1 << (2 * m), 0);
    pl.assign((size_t)1 << (2 * m), 0);
    if (!scan_file(dir, L, false, [&](const uint64_t *w, uint32_t) { ++ph[lead_prefix(w, L.k, m)]; }, err))
        return false;
    if (with_low && !scan_file(dir, L, true, [&](const uint64_t *w, uint32_t) { ++pl[lead_prefix(w, L.k, m)]; }, err))
        return false;
    return true;
}

// Reads segment s's records: high.bin keys (L.nw words each) and counts,
// low.bin keys (with_low).
inline bool load_segment(const std::string &dir, const Layout &L, bool with_low, const Segment &s,
                         std::vector<uint64_t> &hk, std::vector<uint32_t> &hc, std::vector<uint64_t> &lk,
                         std::string &err)
{
    const uint32_t m = lead_bases(L.k);
    hk.clear();
    hc.clear();
    lk.clear();
    hk.reserve(s.n_high * L.nw);
    hc.reserve(s.n_high);
    if (!scan_file(dir, L, false,
                   [&](const uint64_t *w, uint32_t c) {
                       const uint32_t p = lead_prefix(w, L.k, m);
                       if (p >= s.p0 && p < s.p1) {
                           hk.insert(hk.end(), w, w + L.nw);
                           hc.push_back(c);
                       }
                   },
                   err))
        return false;
    if (with_low) {
        lk.reserve(s.n_low * L.nw);
        if (!scan_file(dir, L, true,
                       [&](const uint64_t *w, uint32_t) {
                           const uint32_t p = lead_prefix(w, L.k, m);
                           if (p >= s.p0 && p < s.p1) lk.insert(lk.end(), w, w + L.nw);
                       },
                       err))
            return false;
    }
    return true;
}

// Why no segment plan fits (return code 2, as the reference's tools give
// when even their largest partition count does not fit).
inline std::string no_fit_message(const Layout &L, const std::vector<uint64_t> &ph, const std::vector<uint64_t> &pl,
                                  const SegCost &c, uint32_t worst, uint64_t budget)
{
    if (worst == ~0u)
        return "insufficient memory: max_memory_bytes=" + std::to_string(budget) + " is below the " +
               std::to_string(c.fixed) + " bytes every segment needs";
    const uint64_t b = c.fixed + ph[worst] * c.per_high + pl[worst] * c.per_low;
    return "insufficient memory: the " + std::to_string(ph[worst] + pl[worst]) + " records whose k-mers start with " +
           prefix_string(worst, lead_bases(L.k)) + " need " + std::to_string(b) + " bytes, more than max_memory_bytes=" +
           std::to_string(budget);
}

// max_memory_gb in bytes: GiB, fractions allowed, the whole argument a
// positive number (tool/histogram_tool.cpp:157-174, tool/dump_tool.cpp:476-491).
// 0 = ok, 1 = not a positive number, 2 = more bytes than 64 bits hold.
inline int parse_memory_gib(const char *s, uint64_t &bytes)
{
    char *end = nullptr;
    errno = 0;
    const long double v = std::strtold(s, &end);
    if (errno || !end || *end || end == s || !(v > 0.0L)) return 1;
    const long double b = v * (long double)(1ull << 30);
    if (b > 18446744073709551615.0L) return 2;
    bytes = (uint64_t)b;
    return 0;
}

// "KMER\tcount\n" lines (tool/dump_tool.cpp:1172-1193), formatted on the
// device (kc_dump_text) into pinned host memory (*buf, kc_host_free it).
inline bool format_dump(const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k, void *&buf,
                        uint64_t &got, std::string &err)
{
    buf = nullptr;
    got = 0;
    uint64_t need = 0;
    if (kc_dump_text(keys, counts, n, k, nullptr, 0, &need) != KC_OK) { err = kc_last_error(); return false; }
    if (need && kc_host_alloc(need, &buf) != KC_OK) {
        buf = nullptr;
        err = kc_last_error();
        return false;
    }
    if (need && kc_dump_text(keys, counts, n, k, static_cast<char *>(buf), need, &got) != KC_OK) {
        err = kc_last_error();
        kc_host_free(buf);
        buf = nullptr;
        return false;
    }
    return true;
}

// The dump lines of one segment, appended to an open file.
inline bool append_dump(FILE *f, const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k,
                        std::string &err)
{
    void *buf = nullptr;
    uint64_t got = 0;
    if (!format_dump(keys, counts, n, k, buf, got, err)) return false;
    const bool ok = !got || std::fwrite(buf, 1, got, f) == got;
    if (buf) kc_host_free(buf);
    if (!ok) err = "failed to write the dump";
    return ok;
}

inline bool write_dump(const std::string &path, const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k,
                       std::string &err)
{
    void *buf = nullptr;
    uint64_t got = 0;
    if (!format_dump(keys, counts, n, k, buf, got, err)) return false;
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "failed to open " + path;
        if (buf) kc_host_free(buf);
        return false;
    }
    bool ok = !got || std::fwrite(buf, 1, got, f) == got;
    ok = (std::fclose(f) == 0) && ok;
    if (buf) kc_host_free(buf);
    if (!ok) err = "failed to write " + path;
    return ok;
}

// "f\tcount\n" for every f in [min, max] (tool/histogram_tool.cpp:462-478).
inline bool write_hist(const std::string &path, const int64_t *hist, uint32_t lo, uint32_t hi)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = true;
    for (uint64_t v = lo; v <= hi; ++v) ok = ok && std::fprintf(f, "%llu\t%lld\n", (unsigned long long)v, (long long)hist[v - lo]) > 0;
    return (std::fclose(f) == 0) && ok;
}

}  // namespace cli
