// kc_gzip.cpp -- gzip-compressed FASTQ inputs.
//
// The reference reads ".gz" files through zlib's gzread
// (src/FastqReader.h:581-616), which also reads files of several
// concatenated gzip members.  A job's gzip files (recognised by the gzip magic
// bytes 1f 8b) are inflated on the host into pinned blocks before the upload,
// one thread per file; the other files are used as they are.
#include <zlib.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "kc_host.h"

namespace kc {

bool is_gzip(const kc_buffer &b)
{
    const auto *p = reinterpret_cast<const unsigned char *>(b.data);
    return b.data && b.size >= 18 && p[0] == 0x1f && p[1] == 0x8b;
}

uint64_t gzip_size_hint(const kc_buffer &b)
{
    if (!is_gzip(b)) return b.size;
    // ISIZE (the last member's length mod 2^32) and 4x the compressed size
    const auto *p = reinterpret_cast<const unsigned char *>(b.data) + b.size - 4;
    const uint64_t isize = (uint64_t)p[0] | ((uint64_t)p[1] << 8) | ((uint64_t)p[2] << 16) | ((uint64_t)p[3] << 24);
    return std::max<uint64_t>(isize, 4 * b.size);
}

namespace {

// Inflates one gzip file (one or more members) into a pinned block.
void inflate_one(const kc_buffer &in, PinnedBlock &out, uint64_t &size, std::string &err)
{
    size_t cap = (size_t)gzip_size_hint(in) + (1u << 20);
    out.reset(cap);
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, 15 + 32) != Z_OK) {
        err = "zlib inflateInit2 failed";
        return;
    }
    const auto *src = reinterpret_cast<const Bytef *>(in.data);
    uint64_t in_pos = 0, out_pos = 0;
    for (;;) {
        if (zs.avail_in == 0 && in_pos < in.size) {
            const uint64_t n = std::min<uint64_t>(in.size - in_pos, UINT_MAX);
            zs.next_in = const_cast<Bytef *>(src + in_pos);
            zs.avail_in = (uInt)n;
            in_pos += n;
        }
        if (out_pos == out.bytes) {   // the size hint was short: grow
            PinnedBlock bigger;
            bigger.reset(out.bytes * 2);
            std::memcpy(bigger.p, out.p, out_pos);
            std::swap(out, bigger);
        }
        const uint64_t room = std::min<uint64_t>(out.bytes - out_pos, UINT_MAX);
        zs.next_out = static_cast<Bytef *>(out.p) + out_pos;
        zs.avail_out = (uInt)room;
        const int rc = inflate(&zs, Z_NO_FLUSH);
        out_pos += room - zs.avail_out;
        if (rc == Z_STREAM_END) {
            // another member follows when the next bytes are a gzip header;
            // anything else after a member is ignored
            const uint64_t next = in_pos - zs.avail_in;   // first byte after the member
            if (next + 2 <= in.size && src[next] == 0x1f && src[next + 1] == 0x8b) {
                if (inflateReset(&zs) != Z_OK) {
                    err = "zlib inflateReset failed";
                    break;
                }
                continue;
            }
            size = out_pos;
            break;
        }
        if (rc == Z_OK) continue;
        if (rc == Z_BUF_ERROR && (zs.avail_in > 0 || in_pos < in.size || out_pos == out.bytes)) continue;
        err = rc == Z_BUF_ERROR ? "truncated gzip data" : "corrupt gzip data";
        break;
    }
    inflateEnd(&zs);
}

}  // namespace

std::vector<kc_buffer> inflate_inputs(const std::vector<kc_buffer> &files, std::vector<PinnedBlock> &hold)
{
    std::vector<kc_buffer> outv = files;
    std::vector<size_t> gz;
    for (size_t i = 0; i < files.size(); ++i)
        if (is_gzip(files[i])) gz.push_back(i);
    if (gz.empty()) return outv;
    hold.clear();
    hold.resize(gz.size());
    std::vector<uint64_t> sizes(gz.size(), 0);
    std::vector<std::string> errs(gz.size());
    std::vector<std::thread> th;
    const size_t par = std::max<size_t>(1, std::min<size_t>(gz.size(), std::thread::hardware_concurrency()));
    for (size_t w = 0; w < par; ++w)
        th.emplace_back([&, w] {
            for (size_t j = w; j < gz.size(); j += par) {
                try {
                    inflate_one(files[gz[j]], hold[j], sizes[j], errs[j]);
                } catch (const KcError &e) {
                    errs[j] = e.msg;
                }
            }
        });
    for (auto &t : th) t.join();
    for (size_t j = 0; j < gz.size(); ++j) {
        if (!errs[j].empty()) throw KcError{KC_ERR_INVALID, "file " + std::to_string(gz[j]) + ": " + errs[j]};
        outv[gz[j]].data = static_cast<const char *>(hold[j].p);
        outv[gz[j]].size = sizes[j];
    }
    return outv;
}

}  // namespace kc
