// cli_common.h -- helpers shared by the reference-compatible command-line
// programs: argument parsing with the reference's messages, file IO in the
// reference's tmp_dir formats, and text output.
#pragma once

#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
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

inline uint32_t count_bytes_for(uint32_t count_max)
{
    return count_max <= 0xFF ? 1 : count_max <= 0xFFFF ? 2 : count_max <= 0xFFFFFF ? 3 : 4;
}

struct TmpDir {
    uint32_t k = 0, count_max = 0, count_bytes = 4;
    std::vector<uint64_t> high_keys;
    std::vector<uint32_t> high_counts;
    std::vector<uint64_t> low_keys;
};

// infos.bin, high.bin, low.bin as written by the reference counter
// (src/main.cpp:590-615, src/FinalDrainWriter.h:71-88, src/ExportWriter.h:296-313)
// and read by its tools (tool/histogram_tool.cpp:239-366).
inline bool read_tmpdir(const std::string &dir, TmpDir &t, std::string &err)
{
    std::vector<char> b;
    if (!read_file(dir + "infos.bin", b) || b.size() < 8) { err = "failed to read " + dir + "infos.bin"; return false; }
    std::memcpy(&t.k, b.data(), 4);
    std::memcpy(&t.count_max, b.data() + 4, 4);
    t.count_bytes = count_bytes_for(t.count_max);
    if (t.k == 0 || t.k > 128) { err = "invalid k_len from infos.bin: " + std::to_string(t.k); return false; }
    if (t.k > 32) { err = "k_len " + std::to_string(t.k) + " is above 32, which this build does not support"; return false; }
    const uint32_t tail_bytes = (2 * (t.k % 32) + 7) / 8, full = t.k / 32;
    const uint32_t kb = full * 8 + tail_bytes, rec = kb + t.count_bytes;
    if (!read_file(dir + "high.bin", b)) { err = "failed to open " + dir + "high.bin"; return false; }
    if (b.empty()) { err = "empty high.bin file"; return false; }
    if (b.size() % rec) { err = "invalid high.bin file size"; return false; }
    size_t n = b.size() / rec;
    t.high_keys.resize(n);
    t.high_counts.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const char *r = b.data() + i * rec;
        uint64_t w = 0;
        if (full) std::memcpy(&w, r, 8);
        else std::memcpy(reinterpret_cast<char *>(&w) + (8 - tail_bytes), r, tail_bytes);
        uint32_t c = 0;
        std::memcpy(&c, r + kb, t.count_bytes);
        t.high_keys[i] = w;
        t.high_counts[i] = c;
    }
    if (!read_file(dir + "low.bin", b)) { err = "failed to open " + dir + "low.bin"; return false; }
    if (b.size() % kb) { err = "invalid low.bin size"; return false; }
    n = b.size() / kb;
    t.low_keys.resize(n);
    for (size_t i = 0; i < n; ++i) {
        uint64_t w = 0;
        if (full) std::memcpy(&w, b.data() + i * kb, 8);
        else std::memcpy(reinterpret_cast<char *>(&w) + (8 - tail_bytes), b.data() + i * kb, tail_bytes);
        t.low_keys[i] = w;
    }
    return true;
}

// "KMER\tcount\n" lines (tool/dump_tool.cpp:1172-1193), formatted on the
// device (kc_dump_text) into pinned host memory, then written out.
inline bool write_dump(const std::string &path, const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k,
                       std::string &err)
{
    uint64_t need = 0;
    if (kc_dump_text(keys, counts, n, k, nullptr, 0, &need) != KC_OK) { err = kc_last_error(); return false; }
    void *buf = nullptr;
    if (need && kc_host_alloc(need, &buf) != KC_OK) { err = kc_last_error(); return false; }
    uint64_t got = 0;
    if (need && kc_dump_text(keys, counts, n, k, static_cast<char *>(buf), need, &got) != KC_OK) {
        err = kc_last_error();
        kc_host_free(buf);
        return false;
    }
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
