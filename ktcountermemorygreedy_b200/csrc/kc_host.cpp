// kc_host.cpp -- shared host helpers and the single-step entry points of
// include/kc.h (kc_extract_kmers, kc_hash_kmers, kc_sort_records,
// kc_bloom_plan).  The single-step calls run synchronously on the current
// device with a private stream.
#include "kc_host.h"
#include "kc_wide.cuh"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include <unistd.h>

#include "kc_plan.h"

namespace kc {

namespace {
thread_local std::string g_err;
}

int set_error(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

namespace {

bool trace_on()
{
    static const bool t = getenv("KC_TRACE") && getenv("KC_TRACE")[0] == '1';
    return t;
}

void *pool_alloc(size_t bytes, cudaStream_t st)
{
    void *p = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (trace_on()) {
        double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > 0.5) fprintf(stderr, "[kc trace] cudaMallocAsync %zu bytes took %.2f ms\n", bytes, ms);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw KcError{KC_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed"};
    }
    return p;
}

}  // namespace

void Workspace::begin_job()
{
    top_ = 0;
    if (max_keep_ && high_ > max_keep_) high_ = max_keep_;
    if (high_ > cap_) {
        // grow once to the high-water mark (plus headroom for jobs that vary)
        CK(cudaStreamSynchronize(st_));
        if (base_) cudaFree(base_);
        base_ = nullptr;
        cap_ = 0;
        // the spilled blocks of earlier jobs are back in the pool: return them
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
            cudaMemPoolTrimTo(pool, 0);
        size_t want = (high_ + high_ / 8 + (64u << 20)) & ~size_t((2u << 20) - 1);
        if (max_keep_ && want > max_keep_) want = max_keep_ & ~size_t((2u << 20) - 1);
        if (cudaMalloc(&base_, want) != cudaSuccess) {
            cudaGetLastError();
            base_ = nullptr;   // keep going from the pool
            return;
        }
        cap_ = want;
        if (trace_on()) fprintf(stderr, "[kc trace] workspace grown to %zu bytes\n", want);
    }
}

void Workspace::reserve(size_t bytes)
{
    high_ = std::max(high_, bytes);
    begin_job();
}

void *Workspace::get(size_t bytes)
{
    if (fail_next_) {
        fail_next_ = false;
        throw KcError{KC_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed (injected)"};
    }
    if (base_ && top_ + bytes <= cap_) {
        void *p = base_ + top_;
        top_ += bytes;
        high_ = std::max(high_, top_);
        return p;
    }
    // the job needs all of the workspace in use plus everything it spilled
    spilled_ += bytes;
    high_ = std::max(high_, top_ + spilled_);
    void *p = pool_alloc(bytes, st_);
    spill_.push_back(p);
    return p;
}

void Workspace::rewind(const Mark &m)
{
    if (m.top <= top_) top_ = m.top;
    while (spill_.size() > m.n_spill) {
        cudaFreeAsync(spill_.back(), st_);
        spill_.pop_back();
    }
}

bool Workspace::release_top(void *p, size_t bytes)
{
    if (base_ && p == base_ + top_ - bytes) {
        top_ -= bytes;
        return true;
    }
    return false;
}

void Workspace::end_job()
{
    fail_next_ = false;
    for (void *p : spill_) cudaFreeAsync(p, st_);
    spill_.clear();
    spilled_ = 0;
    top_ = 0;
}

void Workspace::trim()
{
    end_job();
    cudaStreamSynchronize(st_);
    if (base_) cudaFree(base_);
    base_ = nullptr;
    cap_ = 0;
}

Workspace::~Workspace()
{
    end_job();
    cudaStreamSynchronize(st_);
    if (base_) cudaFree(base_);
}

void *DevScope::get(size_t bytes)
{
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    void *p = ws ? ws->get(bytes) : pool_alloc(bytes, st);
    ptrs.emplace_back(p, bytes);
    return p;
}

void DevScope::release(void *p)
{
    auto it = std::find_if(ptrs.begin(), ptrs.end(), [&](const std::pair<void *, size_t> &x) { return x.first == p; });
    if (it == ptrs.end()) return;
    if (!ws) cudaFreeAsync(p, st);
    else ws->release_top(p, it->second);   // memory further down stays until the job ends
    ptrs.erase(it);
}

void DevScope::rewind(const Mark &m)
{
    if (ws) ws->rewind(m.ws);
    else
        for (size_t i = m.n_ptrs; i < ptrs.size(); ++i) cudaFreeAsync(ptrs[i].first, st);
    if (ptrs.size() > m.n_ptrs) ptrs.resize(m.n_ptrs);
}

DevScope::~DevScope()
{
    if (!ws)
        for (auto &x : ptrs) cudaFreeAsync(x.first, st);
}

uint64_t bit_ceil64(uint64_t x)
{
    if (x <= 1) return 1;
    return 1ULL << (64 - __builtin_clzll(x - 1));
}

struct PinnedPool::Impl {
    std::mutex mu;
    std::multimap<size_t, void *> free_blocks;
    size_t cached = 0;
    struct Arena {
        uint8_t *base;
        size_t size;
        std::map<size_t, size_t> free;   // offset -> length of each free range
    };
    std::vector<Arena> arenas;

    // best-fit range of an arena (caller holds mu); nullptr if none fits
    void *arena_get(size_t bytes)
    {
        Arena *ba = nullptr;
        std::map<size_t, size_t>::iterator bi;
        for (auto &a : arenas)
            for (auto it = a.free.begin(); it != a.free.end(); ++it)
                if (it->second >= bytes && (!ba || it->second < bi->second)) {
                    ba = &a;
                    bi = it;
                }
        if (!ba) return nullptr;
        const size_t off = bi->first, len = bi->second;
        ba->free.erase(bi);
        if (len > bytes) ba->free.emplace(off + bytes, len - bytes);
        return ba->base + off;
    }

    bool arena_put(void *p, size_t bytes)
    {
        uint8_t *q = static_cast<uint8_t *>(p);
        for (auto &a : arenas) {
            if (q < a.base || q >= a.base + a.size) continue;
            size_t off = (size_t)(q - a.base), len = bytes;
            auto next = a.free.lower_bound(off);
            if (next != a.free.end() && off + len == next->first) {   // merge with the range after
                len += next->second;
                next = a.free.erase(next);
            }
            if (next != a.free.begin()) {                              // and with the one before
                auto prev = std::prev(next);
                if (prev->first + prev->second == off) {
                    off = prev->first;
                    len += prev->second;
                    a.free.erase(prev);
                }
            }
            a.free.emplace(off, len);
            return true;
        }
        return false;
    }
};

PinnedPool::PinnedPool() : impl_(new Impl) {}

PinnedPool &PinnedPool::instance()
{
    static PinnedPool pool;
    return pool;
}

void *PinnedPool::get(size_t bytes, size_t &got)
{
    // sizes are rounded up to classes (eight per power of two from 16 MiB,
    // 2 MiB steps below) so that blocks come back for jobs of similar size:
    // pinning new host memory costs far more than the copy it serves
    bytes = std::max<size_t>(bytes, 4096);
    if (bytes >= (16u << 20)) {
        const size_t step = (size_t)bit_ceil64(bytes) / 16;
        bytes = (bytes + step - 1) / step * step;
    } else {
        bytes = (bytes + (2u << 20) - 1) & ~size_t((2u << 20) - 1);
    }
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        if (void *p = impl_->arena_get(bytes)) {
            got = bytes;
            return p;
        }
        auto it = impl_->free_blocks.lower_bound(bytes);
        if (it != impl_->free_blocks.end() && it->first <= bytes + bytes / 4 + (64u << 20)) {
            void *p = it->second;
            got = it->first;
            impl_->cached -= got;
            impl_->free_blocks.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    const size_t want = (bytes + (2u << 20) - 1) & ~size_t((2u << 20) - 1);
    if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        throw KcError{KC_ERR_NOMEM, "pinned host allocation of " + std::to_string(want) + " bytes failed"};
    }
    got = want;
    return p;
}

void PinnedPool::put(void *p, size_t bytes)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        if (impl_->arena_put(p, bytes)) return;
    }
    // keep up to a third of the host's memory pinned for reuse
    static const size_t keep_limit = [] {
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGE_SIZE);
        const size_t phys = (pages > 0 && page > 0) ? (size_t)pages * (size_t)page : (size_t(96) << 30);
        return std::max<size_t>(phys / 3, size_t(8) << 30);
    }();
    {
        std::lock_guard<std::mutex> lk(impl_->mu);
        if (impl_->cached + bytes <= keep_limit) {
            impl_->free_blocks.emplace(bytes, p);
            impl_->cached += bytes;
            return;
        }
    }
    cudaFreeHost(p);
}

void PinnedPool::add_arena(size_t bytes)
{
    bytes = (bytes + (2u << 20) - 1) & ~size_t((2u << 20) - 1);
    if (!bytes) return;
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        throw KcError{KC_ERR_NOMEM, "pinned host arena of " + std::to_string(bytes) + " bytes failed"};
    }
    std::lock_guard<std::mutex> lk(impl_->mu);
    Impl::Arena a{static_cast<uint8_t *>(p), bytes, {}};
    a.free.emplace(0, bytes);
    impl_->arenas.push_back(std::move(a));
}

PinnedPool::~PinnedPool()
{
    // process exit: the driver reclaims pinned memory; freeing here could run
    // after the CUDA runtime has shut down
    delete impl_;
}

void HostRecords::allocate(uint64_t count, uint32_t key_words)
{
    reset();
    n = count;
    words = key_words;
    const size_t need = ((count * 8 * key_words + 255) & ~size_t(255)) + count * 4 + 256;
    block = PinnedPool::instance().get(need, bytes);
}

void HostRecords::reset()
{
    if (block) PinnedPool::instance().put(block, bytes);
    block = nullptr;
    bytes = 0;
    n = 0;
    words = 1;
}

void ChunkedUpload::enqueue(size_t upto)
{
    upto = std::min(upto, ev.size());
    if (queued >= upto) return;
    cudaEvent_t ready;
    CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ready, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ready, 0);
    cudaEventDestroy(ready);   // the wait keeps what it needs
    CK(e);
    for (; queued < upto; ++queued) {
        const uint64_t t0 = queued ? tile_end[queued - 1] : 0, t1 = tile_end[queued];
        const uint64_t b0 = t0 * TILE, b1 = std::min<uint64_t>(len, t1 * TILE);
        if (b1 > b0) CK(cudaMemcpyAsync(dst + b0, src + b0, b1 - b0, cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(ev[queued], cs));
    }
}

ChunkedUpload::~ChunkedUpload()
{
    if (cs) {
        cudaStreamSynchronize(cs);
        cudaStreamDestroy(cs);
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

void build_input(kc_input &in, const kc_buffer *files, uint32_t n_files, cudaStream_t st, DevScope *scope,
                 std::vector<uint32_t> &tile_seg_host, const uint32_t *file_sample, ChunkedUpload *chunked)
{
    if (chunked && n_files != 1) throw KcError{KC_ERR_INVALID, "a chunked upload takes one file"};
    in.segs.clear();
    in.sizes.clear();
    in.total_bytes = 0;
    uint64_t tiles = 0;
    for (uint32_t f = 0; f < n_files; ++f) {
        uint64_t sz = files[f].size;
        in.sizes.push_back(sz);
        in.total_bytes += sz;
        if (sz == 0) continue;
        Seg s{};
        s.first_tile = tiles;
        s.n_tiles = (sz + TILE - 1) / TILE;
        s.len = sz;
        s.sample = file_sample ? file_sample[f] : 0;
        in.segs.push_back(s);
        tiles += s.n_tiles;
    }
    in.n_tiles = tiles;
    const size_t bytes = FRONT_PAD + tiles * (size_t)TILE + 256;
    if (scope) {
        in.base = static_cast<uint8_t *>(scope->get(bytes));
        in.d_tile_seg = scope->n<uint32_t>(std::max<uint64_t>(tiles, 1));
        in.stream_owned = true;
    } else {
        CK(cudaMalloc(&in.base, bytes));
        CK(cudaMalloc(&in.d_tile_seg, std::max<uint64_t>(tiles, 1) * 4));
    }
    in.buf = in.base + FRONT_PAD;
    CK(cudaMemsetAsync(in.base, 0, FRONT_PAD, st));
    CK(cudaMemsetAsync(in.buf + tiles * (size_t)TILE, 0, 256, st));
    tile_seg_host.assign(std::max<uint64_t>(tiles, 1), 0);
    for (uint32_t si = 0; si < in.segs.size(); ++si)
        for (uint64_t t = 0; t < in.segs[si].n_tiles; ++t) tile_seg_host[in.segs[si].first_tile + t] = si;
    // the small table goes before the file bytes: a pageable copy queued behind
    // them would hold the host for the whole upload
    CK(cudaMemcpyAsync(in.d_tile_seg, tile_seg_host.data(), tile_seg_host.size() * 4, cudaMemcpyHostToDevice, st));
    uint32_t si = 0;
    for (uint32_t f = 0; f < n_files; ++f) {
        if (files[f].size == 0) continue;
        const Seg &s = in.segs[si];
        uint8_t *dst = in.buf + s.first_tile * TILE;
        if (chunked) {
            // planned only: the job queues the copies (ChunkedUpload::enqueue)
            CK(cudaStreamCreateWithFlags(&chunked->cs, cudaStreamNonBlocking));
            chunked->st = st;
            chunked->src = reinterpret_cast<const uint8_t *>(files[f].data);
            chunked->dst = dst;
            chunked->len = s.len;
            for (uint64_t t0 = 0; t0 < s.n_tiles; t0 += CHUNKED_UPLOAD_TILES) {
                cudaEvent_t e;
                CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                chunked->ev.push_back(e);
                chunked->tile_end.push_back(s.first_tile + std::min<uint64_t>(s.n_tiles, t0 + CHUNKED_UPLOAD_TILES));
            }
        } else {
            CK(cudaMemcpyAsync(dst, files[f].data, files[f].size, cudaMemcpyHostToDevice, st));
        }
        const uint64_t pad = s.n_tiles * TILE - s.len;
        if (pad) CK(cudaMemsetAsync(dst + s.len, 0, pad, st));
        ++si;
    }
}

namespace {

struct StreamGuard {
    cudaStream_t st = nullptr;
    StreamGuard()
    {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            throw KcError{KC_ERR_NO_DEVICE, "no CUDA device"};
        }
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    }
    ~StreamGuard()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
};

// Newline census + tile line numbers + per-file descriptors for one input.
struct Prepared {
    unsigned long long *tile_prefix = nullptr;
    int32_t *tile_lastnl = nullptr;
    Seg *d_segs = nullptr;
    std::vector<Seg> segs;
};

Prepared prepare(const kc_input &in, uint32_t k, DevScope &ds, cudaStream_t st)
{
    Prepared p;
    const uint64_t T = std::max<uint64_t>(in.n_tiles, 1);
    uint32_t *tile_nl = ds.n<uint32_t>(T);
    p.tile_lastnl = ds.n<int32_t>(T);
    p.tile_prefix = ds.n<unsigned long long>(T);
    unsigned long long *tmp = ds.n<unsigned long long>(scan_tmp_words(T));
    CK(launch_newlines(in.buf, in.n_tiles, tile_nl, p.tile_lastnl, st));
    CK(launch_scan_u32(tile_nl, p.tile_prefix, in.n_tiles, tmp, st));
    p.segs = in.segs;
    for (auto &s : p.segs) s.k = k;
    p.d_segs = ds.n<Seg>(std::max<size_t>(p.segs.size(), 1));
    if (!p.segs.empty())
        CK(cudaMemcpyAsync(p.d_segs, p.segs.data(), p.segs.size() * sizeof(Seg), cudaMemcpyHostToDevice, st));
    return p;
}

}  // namespace

}  // namespace kc

using namespace kc;

extern "C" {

const char *kc_last_error(void) { return kc::g_err.c_str(); }

int kc_extract_kmers(const char *fastq, uint64_t len, uint32_t k, uint64_t *out, uint64_t cap, uint64_t *n_out)
{
    if ((!fastq && len) || (!out && cap) || !n_out) return set_error(KC_ERR_INVALID, "bad argument");
    if (k < 1 || k > 128) return set_error(KC_ERR_INVALID, "k must be in 1..128");
    try {
        const uint32_t nw = key_words(k);
        StreamGuard sg;
        cudaStream_t st = sg.st;
        DevScope ds(st);
        kc_input in;
        std::vector<uint32_t> ts;
        kc_buffer f{fastq, len};
        build_input(in, &f, 1, st, &ds, ts);
        Prepared pr = prepare(in, k, ds, st);
        unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
        CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));
        const uint64_t lcap = std::max<uint64_t>(cap, 1);
        unsigned long long *list = ds.n<unsigned long long>(lcap * nw);
        if (nw == 1) {
            ExtractArgs a{};
            a.buf = in.buf;
            a.n_tiles = in.n_tiles;
            a.tile_prefix = reinterpret_cast<const uint64_t *>(pr.tile_prefix);
            a.tile_seg = in.d_tile_seg;
            a.segs = pr.d_segs;
            a.counters = counters;
            a.list = list;
            a.list_cap = cap;
            CK(launch_extract(MODE_EMIT, a, 0, st));
        } else {
            WideArgs a{};
            a.buf = in.buf;
            a.n_tiles = in.n_tiles;
            a.tile_prefix = reinterpret_cast<const uint64_t *>(pr.tile_prefix);
            a.tile_seg = in.d_tile_seg;
            a.segs = pr.d_segs;
            a.counters = counters;
            a.list = list;
            a.list_cap = cap;
            CK(launch_wide_extract(WMODE_EMIT, k, a, st));
        }
        unsigned long long c[C_COUNT];
        CK(cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c[C_FLAGS] & ERR_WAIT_TIMEOUT) return set_error(KC_ERR_DEVICE, "bounded wait expired");
        *n_out = c[C_EMIT_LEN];
        uint64_t n = std::min<uint64_t>(c[C_EMIT_LEN], cap);
        if (n) CK(cudaMemcpyAsync(out, list, n * nw * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_hash_kmers(const uint64_t *keys, uint64_t n, uint64_t *out)
{
    if ((!keys || !out) && n) return set_error(KC_ERR_INVALID, "bad argument");
    if (!n) return KC_OK;
    try {
        StreamGuard sg;
        DevScope ds(sg.st);
        unsigned long long *dk = ds.n<unsigned long long>(n);
        unsigned long long *dout = ds.n<unsigned long long>(5 * n);
        CK(cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, sg.st));
        CK(launch_hash_batch(dk, n, dout, sg.st));
        CK(cudaMemcpyAsync(out, dout, 5 * n * 8, cudaMemcpyDeviceToHost, sg.st));
        CK(cudaStreamSynchronize(sg.st));
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_sort_records(uint64_t *keys, uint32_t *counts, uint64_t n, uint32_t bits)
{
    if ((!keys || !counts) && n) return set_error(KC_ERR_INVALID, "bad argument");
    if (bits > 64) return set_error(KC_ERR_INVALID, "bits must be <= 64");
    if (n <= 1) return KC_OK;
    try {
        StreamGuard sg;
        DevScope ds(sg.st);
        unsigned long long *dk = ds.n<unsigned long long>(n);
        uint32_t *dv = ds.n<uint32_t>(n);
        void *tmp = ds.get(sort_tmp_bytes(n));
        unsigned long long *dflags = ds.n<unsigned long long>(1);
        CK(cudaMemsetAsync(dflags, 0, 8, sg.st));
        CK(cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, sg.st));
        CK(cudaMemcpyAsync(dv, counts, n * 4, cudaMemcpyHostToDevice, sg.st));
        CK(launch_radix_sort(dk, dv, n, bits, tmp, sg.st, dflags));
        CK(cudaMemcpyAsync(keys, dk, n * 8, cudaMemcpyDeviceToHost, sg.st));
        CK(cudaMemcpyAsync(counts, dv, n * 4, cudaMemcpyDeviceToHost, sg.st));
        unsigned long long flags = 0;
        CK(cudaMemcpyAsync(&flags, dflags, 8, cudaMemcpyDeviceToHost, sg.st));
        CK(cudaStreamSynchronize(sg.st));
        if (flags) return set_error(KC_ERR_DEVICE, "record sort reported error flags");
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_sort_distinct_records(uint64_t *keys, uint32_t *counts, uint64_t n, uint32_t bits)
{
    if ((!keys || !counts) && n) return set_error(KC_ERR_INVALID, "bad argument");
    if (bits > 64) return set_error(KC_ERR_INVALID, "bits must be <= 64");
    if (n <= 1) return KC_OK;
    try {
        StreamGuard sg;
        DevScope ds(sg.st);
        unsigned long long *dk = ds.n<unsigned long long>(n);
        uint32_t *dv = ds.n<uint32_t>(n);
        const bool msd = msd_sort_applies(n, bits);
        void *tmp = ds.get(msd ? msd_sort_tmp_bytes(n, bits) : sort_tmp_bytes(n));
        unsigned long long *dflags = ds.n<unsigned long long>(1);
        CK(cudaMemsetAsync(dflags, 0, 8, sg.st));
        CK(cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, sg.st));
        CK(cudaMemcpyAsync(dv, counts, n * 4, cudaMemcpyHostToDevice, sg.st));
        if (msd) CK(launch_msd_sort(dk, dv, n, bits, tmp, sg.st, dflags, false));
        else CK(launch_radix_sort(dk, dv, n, bits, tmp, sg.st, dflags));
        CK(cudaMemcpyAsync(keys, dk, n * 8, cudaMemcpyDeviceToHost, sg.st));
        CK(cudaMemcpyAsync(counts, dv, n * 4, cudaMemcpyDeviceToHost, sg.st));
        unsigned long long flags = 0;
        CK(cudaMemcpyAsync(&flags, dflags, 8, cudaMemcpyDeviceToHost, sg.st));
        CK(cudaStreamSynchronize(sg.st));
        if (flags) return set_error(KC_ERR_DEVICE, "record sort reported error flags");
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_dump_text(const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k, char *out, uint64_t cap,
                 uint64_t *n_bytes)
{
    if (!n_bytes || (n && (!keys || !counts))) return set_error(KC_ERR_INVALID, "bad argument");
    if (k < 1 || k > 128) return set_error(KC_ERR_INVALID, "k must be in 1..128");
    const uint32_t nw = key_words(k);
    if (!out) {
        // size query: k bases, a tab, the decimal count and a newline per record
        uint64_t need = 0;
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t c = counts[i], d = 1;
            while (c >= 10) { c /= 10; ++d; }
            need += k + 2 + d;
        }
        *n_bytes = need;
        return KC_OK;
    }
    *n_bytes = 0;
    if (!n) return KC_OK;
    try {
        StreamGuard sg;
        // records in chunks, so that device memory stays bounded
        const uint64_t chunk = std::min<uint64_t>(n, 1ull << 25);
        DevScope ds(sg.st);
        unsigned long long *dk = ds.n<unsigned long long>(chunk * nw);
        uint32_t *dc = ds.n<uint32_t>(chunk);
        uint32_t *len = ds.n<uint32_t>(chunk);
        unsigned long long *off = ds.n<unsigned long long>(chunk);
        unsigned long long *tmp = ds.n<unsigned long long>(scan_tmp_words(chunk));
        char *dtxt = static_cast<char *>(ds.get(chunk * (size_t)(k + 12)));
        uint64_t pos = 0;
        for (uint64_t c0 = 0; c0 < n; c0 += chunk) {
            const uint64_t m = std::min(chunk, n - c0);
            CK(cudaMemcpyAsync(dk, keys + c0 * nw, m * nw * 8, cudaMemcpyHostToDevice, sg.st));
            CK(cudaMemcpyAsync(dc, counts + c0, m * 4, cudaMemcpyHostToDevice, sg.st));
            CK(launch_dump_text(dk, dc, m, k, len, off, tmp, dtxt, sg.st));
            unsigned long long last_off = 0;
            uint32_t last_len = 0;
            CK(cudaMemcpyAsync(&last_off, off + m - 1, 8, cudaMemcpyDeviceToHost, sg.st));
            CK(cudaMemcpyAsync(&last_len, len + m - 1, 4, cudaMemcpyDeviceToHost, sg.st));
            CK(cudaStreamSynchronize(sg.st));
            const uint64_t bytes = last_off + last_len;
            if (pos + bytes > cap) {
                *n_bytes = pos;
                return set_error(KC_ERR_INVALID, "output buffer too small for the dump text");
            }
            CK(cudaMemcpyAsync(out + pos, dtxt, bytes, cudaMemcpyDeviceToHost, sg.st));
            CK(cudaStreamSynchronize(sg.st));
            pos += bytes;
        }
        *n_bytes = pos;
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_atomic_peak(uint64_t buffer_bytes, uint32_t repeats, double *atomics_per_s, double *ms_per_launch)
{
    if (!atomics_per_s || !ms_per_launch || !repeats) return set_error(KC_ERR_INVALID, "bad argument");
    if (buffer_bytes < 4096 || (buffer_bytes & (buffer_bytes - 1)))
        return set_error(KC_ERR_INVALID, "buffer_bytes must be a power of two >= 4096");
    try {
        StreamGuard sg;
        DevScope ds(sg.st);
        const uint64_t words = buffer_bytes / 4;
        uint32_t *buf = ds.n<uint32_t>(words);
        CK(cudaMemsetAsync(buf, 0, buffer_bytes, sg.st));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        uint64_t ops = 0;
        const uint32_t iters = 512;
        CK(launch_atomic_peak(buf, words, iters, 1, &ops, sg.st));   // warm-up
        CK(cudaEventRecord(e0, sg.st));
        for (uint32_t r = 0; r < repeats; ++r) CK(launch_atomic_peak(buf, words, iters, 2 + r, &ops, sg.st));
        CK(cudaEventRecord(e1, sg.st));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_per_launch = ms / repeats;
        *atomics_per_s = (double)ops * repeats / (ms * 1e-3);
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_atomic_peak_shared(uint32_t table_bytes, uint32_t repeats, double *atomics_per_s, double *ms_per_launch)
{
    if (!atomics_per_s || !ms_per_launch || !repeats) return set_error(KC_ERR_INVALID, "bad argument");
    if (table_bytes < 4096 || table_bytes > (64u << 10) || (table_bytes & (table_bytes - 1)))
        return set_error(KC_ERR_INVALID, "table_bytes must be a power of two in [4096, 65536]");
    try {
        StreamGuard sg;
        DevScope ds(sg.st);
        uint32_t *out = ds.n<uint32_t>(1);
        CK(cudaMemsetAsync(out, 0, 4, sg.st));
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        uint64_t ops = 0;
        const uint32_t iters = 4096, words = table_bytes / 4;
        CK(launch_atomic_peak_shared(out, words, iters, 1, &ops, sg.st));   // warm-up
        CK(cudaEventRecord(e0, sg.st));
        for (uint32_t r = 0; r < repeats; ++r) CK(launch_atomic_peak_shared(out, words, iters, 2 + r, &ops, sg.st));
        CK(cudaEventRecord(e1, sg.st));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_per_launch = ms / repeats;
        *atomics_per_s = (double)ops * repeats / (ms * 1e-3);
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

int kc_plan_bloom(const uint32_t *raw_prefix_counts, uint32_t avg_quality, uint64_t est_file_size,
                  uint64_t memory_gb, uint32_t k, uint64_t *capacities, uint64_t *max_capacity)
{
    if (!raw_prefix_counts || !capacities || !max_capacity) return set_error(KC_ERR_INVALID, "bad argument");
    if (avg_quality > 255) return set_error(KC_ERR_INVALID, "avg_quality must fit in 8 bits");
    BloomPlan bp = bloom_plan(raw_prefix_counts, (uint8_t)avg_quality, est_file_size, memory_gb, k);
    std::memcpy(capacities, bp.caps, sizeof(bp.caps));
    *max_capacity = bp.max_cap;
    return KC_OK;
}

int kc_bloom_plan(const kc_buffer *files, uint32_t n_files, uint32_t k, uint64_t memory_gb, uint32_t *prefix_counts,
                  uint32_t *avg_quality, uint64_t *capacities, uint64_t *max_capacity)
{
    if (!files || !n_files || !prefix_counts || !avg_quality || !capacities || !max_capacity)
        return set_error(KC_ERR_INVALID, "bad argument");
    if (k < 1 || k > 32) return set_error(KC_ERR_INVALID, "k must be in 1..32");
    try {
        StreamGuard sg;
        cudaStream_t st = sg.st;
        DevScope ds(st);
        kc_input in;
        std::vector<uint32_t> ts;
        build_input(in, files, n_files, st, &ds, ts);
        Prepared pr = prepare(in, k, ds, st);
        const uint64_t limit = n_files == 1 ? (256ULL << 20) : (128ULL << 20);
        std::vector<uint64_t> chunk0(std::max<size_t>(pr.segs.size(), 1), 0);
        uint64_t n_chunks = 0;
        for (size_t i = 0; i < pr.segs.size(); ++i) {
            pr.segs[i].sample_end = std::min(pr.segs[i].len, limit);
            chunk0[i] = n_chunks;
            n_chunks += (pr.segs[i].len + PREPASS_CHUNK - 1) / PREPASS_CHUNK;
        }
        if (!pr.segs.empty())
            CK(cudaMemcpyAsync(pr.d_segs, pr.segs.data(), pr.segs.size() * sizeof(Seg), cudaMemcpyHostToDevice, st));
        int32_t *chunk_lastnl = ds.n<int32_t>(std::max<uint64_t>(n_chunks, 1));
        uint64_t *d_chunk0 = ds.n<uint64_t>(chunk0.size());
        uint32_t *ph = ds.n<uint32_t>(256);
        unsigned long long *qual = ds.n<unsigned long long>(2);
        unsigned long long *occ = ds.n<unsigned long long>(1);
        uint32_t *hll = ds.n<uint32_t>(HLL_M);
        unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
        CK(cudaMemsetAsync(chunk_lastnl, 0xff, std::max<uint64_t>(n_chunks, 1) * 4, st));
        CK(cudaMemcpyAsync(d_chunk0, chunk0.data(), chunk0.size() * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(ph, 0, 1024, st));
        CK(cudaMemsetAsync(qual, 0, 16, st));
        CK(cudaMemsetAsync(occ, 0, 8, st));
        CK(cudaMemsetAsync(hll, 0, HLL_M * 4, st));
        CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));
        CK(launch_chunk_lastnl(pr.tile_lastnl, in.d_tile_seg, pr.d_segs, d_chunk0, in.n_tiles, chunk_lastnl, st));
        ExtractArgs a{};
        a.buf = in.buf;
        a.n_tiles = in.n_tiles;
        a.tile_prefix = reinterpret_cast<const uint64_t *>(pr.tile_prefix);
        a.tile_seg = in.d_tile_seg;
        a.segs = pr.d_segs;
        a.counters = counters;
        a.occ = occ;
        a.hll = nullptr;   // only the pre-pass sample needs k-mers
        a.prepass = 1;
        a.chunk_lastnl = chunk_lastnl;
        a.seg_chunk0 = d_chunk0;
        a.prefix_hist = ph;
        a.qual = qual;
        CK(launch_extract(MODE_SCAN, a, 0, st));
        unsigned long long q[2];
        CK(cudaMemcpyAsync(prefix_counts, ph, 1024, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(q, qual, 16, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        uint8_t avg = q[1] ? (uint8_t)(q[0] / q[1]) : 0;
        *avg_quality = avg;
        BloomPlan bp = bloom_plan(prefix_counts, avg, in.total_bytes, memory_gb, k);
        std::memcpy(capacities, bp.caps, sizeof(bp.caps));
        *max_capacity = bp.max_cap;
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}

}  // extern "C"
