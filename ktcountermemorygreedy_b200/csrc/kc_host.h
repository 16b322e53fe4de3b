// kc_host.h -- host-side helpers shared by the C ABI translation units:
// error type, CUDA check macro, stream-ordered allocation scope, and the
// tile-aligned device layout of FASTQ inputs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "kc.h"
#include "kc_kernels.cuh"

namespace kc {

struct KcError {
    int code;
    std::string msg;
};

int set_error(int code, const std::string &msg);

#define CK(x)                                                                                            \
    do {                                                                                                 \
        cudaError_t e_ = (x);                                                                            \
        if (e_ != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            throw ::kc::KcError{e_ == cudaErrorMemoryAllocation ? KC_ERR_NOMEM : KC_ERR_CUDA,            \
                                std::string(#x) + ": " + cudaGetErrorString(e_)};                        \
        }                                                                                                \
    } while (0)

// Device memory of one worker stream, reused job after job: one block sized
// to the high-water mark of the jobs seen so far, handed out by a bump
// pointer (the most recent allocation can be given back).  Allocation-heavy
// jobs would otherwise spend tens to hundreds of milliseconds per multi-GB
// stream-ordered allocation.  Requests that do not fit go to the stream's
// memory pool for this job; the next job then gets a block that fits all.
class Workspace {
public:
    explicit Workspace(cudaStream_t st) : st_(st) {}
    Workspace(const Workspace &) = delete;
    Workspace &operator=(const Workspace &) = delete;
    void begin_job();
    void reserve(size_t bytes);   // grow the block to at least `bytes` now
    // everything handed out after a mark can be taken back at once
    struct Mark {
        size_t top, n_spill;
    };
    Mark mark() const { return Mark{top_, spill_.size()}; }
    void rewind(const Mark &m);
    void *get(size_t bytes);
    bool release_top(void *p, size_t bytes);
    void end_job();
    ~Workspace();
    size_t capacity() const { return cap_; }
    // failure injection: the next get() fails as a failed device allocation
    // does (KcError KC_ERR_NOMEM)
    void fail_next_get() { fail_next_ = true; }
    // the block kept between jobs is at most this large (0: no limit); a job
    // that needs more takes the rest from the stream-ordered pool, which the
    // other workers of a handle share
    void set_max_keep(size_t bytes) { max_keep_ = bytes; }
    // gives the kept block back to the device between jobs (the next job
    // grows it again to the high-water mark)
    void trim();

private:
    cudaStream_t st_;
    uint8_t *base_ = nullptr;
    size_t cap_ = 0, top_ = 0, high_ = 0;
    size_t spilled_ = 0;   // bytes of this job's blocks taken from the pool
    bool fail_next_ = false;
    size_t max_keep_ = 0;
    std::vector<void *> spill_;
};

// Device allocations of one job step, from a Workspace or (without one)
// from the stream's memory pool.  Everything is released with the scope.
struct DevScope {
    cudaStream_t st = nullptr;
    Workspace *ws = nullptr;
    std::vector<std::pair<void *, size_t>> ptrs;
    explicit DevScope(cudaStream_t s, Workspace *w = nullptr) : st(s), ws(w) {}
    DevScope(const DevScope &) = delete;
    DevScope &operator=(const DevScope &) = delete;
    void *get(size_t bytes);
    template <class T>
    T *n(size_t count)
    {
        return static_cast<T *>(get(count * sizeof(T)));
    }
    void release(void *p);
    // takes back every allocation of this scope made after the mark
    struct Mark {
        size_t n_ptrs;
        Workspace::Mark ws;
    };
    Mark mark() const { return Mark{ptrs.size(), ws ? ws->mark() : Workspace::Mark{0, 0}}; }
    void rewind(const Mark &m);
    ~DevScope();
};

uint64_t bit_ceil64(uint64_t x);

// Pinned host blocks reused across jobs: result copies from the device run at
// link speed and no block is pinned (or zero-filled) twice.
class PinnedPool {
public:
    static PinnedPool &instance();
    void *get(size_t bytes, size_t &got);   // throws KcError on failure
    void put(void *p, size_t bytes);
    // pins `bytes` of host memory once; later blocks are carved from it
    // first (best fit) and returned to it.  Kept until the process exits.
    void add_arena(size_t bytes);           // throws KcError on failure
    ~PinnedPool();

private:
    struct Impl;
    Impl *impl_ = nullptr;
    PinnedPool();
};

// One pinned block from the pool, given back when it goes out of scope.
struct PinnedBlock {
    void *p = nullptr;
    size_t bytes = 0;
    PinnedBlock() = default;
    PinnedBlock(const PinnedBlock &) = delete;
    PinnedBlock &operator=(const PinnedBlock &) = delete;
    PinnedBlock(PinnedBlock &&o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr, o.bytes = 0; }
    PinnedBlock &operator=(PinnedBlock &&o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    void reset(size_t n)   // throws KcError
    {
        release();
        size_t got = 0;
        p = PinnedPool::instance().get(n, got);
        bytes = got;
    }
    void release()
    {
        if (p) PinnedPool::instance().put(p, bytes);
        p = nullptr;
        bytes = 0;
    }
    ~PinnedBlock() { release(); }
};

// gzip inputs (kc_gzip.cpp): detection, an upper estimate of the inflated
// size, and inflation of a job's gzip files into pinned blocks held by `hold`
// (the returned buffers replace the gzip files, the others are unchanged).
bool is_gzip(const kc_buffer &b);
uint64_t gzip_size_hint(const kc_buffer &b);
std::vector<kc_buffer> inflate_inputs(const std::vector<kc_buffer> &files, std::vector<PinnedBlock> &hold);

// (key, count) records of one job in a pinned block; a key is `words`
// 64-bit words (kmer<N>, N = 1, 2 or 4).
struct HostRecords {
    void *block = nullptr;
    size_t bytes = 0;
    uint64_t n = 0;
    uint32_t words = 1;
    HostRecords() = default;
    HostRecords(const HostRecords &) = delete;
    HostRecords &operator=(const HostRecords &) = delete;
    void allocate(uint64_t count, uint32_t key_words = 1);
    uint64_t *keys() const { return static_cast<uint64_t *>(block); }
    uint32_t *counts() const
    {
        return reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(block) + ((n * 8 * words + 255) & ~uint64_t(255)));
    }
    void reset();
    ~HostRecords() { reset(); }
};

}  // namespace kc

struct kc_input {
    uint8_t *base = nullptr;       // allocation (FRONT_PAD zero bytes, then tiles)
    uint8_t *buf = nullptr;        // first byte of tile 0
    uint64_t n_tiles = 0;
    std::vector<kc::Seg> segs;     // k and sample are filled in per job
    uint32_t *d_tile_seg = nullptr;
    std::vector<uint64_t> sizes;   // per file (including empty files)
    uint64_t total_bytes = 0;
    bool stream_owned = false;     // allocated with cudaMallocAsync on a job stream
};

namespace kc {

// An upload of one file in chunks on its own stream: chunk c holds tiles
// [c ? tile_end[c - 1] : 0, tile_end[c]) and is on the device once ev[c] has
// completed, so the job's stream can wait for each chunk before working on
// it.  build_input only plans the chunks; enqueue(upto) queues the copies of
// the chunks before `upto` behind the work queued on the job's stream so far
// (a small upload queued on the job's stream first is not held up behind the
// file's bytes in the copy engine).  A chunk must be queued before the job's
// stream waits for it.  The destructor drains the stream (the host data and
// the device buffer must outlive it: declare it after both).
struct ChunkedUpload {
    cudaStream_t cs = nullptr, st = nullptr;
    std::vector<cudaEvent_t> ev;
    std::vector<uint64_t> tile_end;
    const uint8_t *src = nullptr;
    uint8_t *dst = nullptr;
    uint64_t len = 0;
    size_t queued = 0;
    ChunkedUpload() = default;
    ChunkedUpload(const ChunkedUpload &) = delete;
    ChunkedUpload &operator=(const ChunkedUpload &) = delete;
    void enqueue(size_t upto);   // throws KcError
    ~ChunkedUpload();
};
constexpr uint64_t CHUNKED_UPLOAD_TILES = 16384;   // 128 MiB per chunk

// Lays the files out tile-aligned in one device buffer.  When `scope` is
// given the allocations belong to it (per-job upload), otherwise they are
// long-lived (kc_input_upload).  `file_sample` (optional) assigns each file
// to a sample.  With `chunked` (one file), the file's bytes are planned as
// chunks for chunked->enqueue instead of one copy on st.
void build_input(kc_input &in, const kc_buffer *files, uint32_t n_files, cudaStream_t st, DevScope *scope,
                 std::vector<uint32_t> &tile_seg_host, const uint32_t *file_sample = nullptr,
                 ChunkedUpload *chunked = nullptr);

}  // namespace kc
