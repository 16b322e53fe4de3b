// kc_api.cpp -- C++ host runtime behind include/kc.h.
//
// A handle owns a pool of worker threads, one CUDA stream each.  Submitted
// jobs wait in a FIFO queue and are admitted, in order, when their device
// memory reservation fits the handle's HBM budget (or when nothing else runs),
// so jobs that arrive while others are on the device start as soon as a
// worker slot and memory free up, and their kernels overlap on the GPU.
//
// One job is the reference's counter run followed by its precise tools:
//   upload (tile-aligned, zero padded)  -> newline census -> tile line numbers
//   -> SCAN pass (occurrences, HyperLogLog; Bloom pre-pass statistics)
//   -> plain:  INSERT pass into a table sized from the HyperLogLog estimate
//      Bloom:  BLOOM pass (reference filter sizing and probes), then insert
//              the non-FIRST occurrences and merge the FIRST ones back
//   -> compaction + histogram -> radix sort in printed-string order
//   -> queries -> host.
// All device memory is stream-ordered (cudaMallocAsync on the worker stream)
// from a pool that keeps freed memory for the next job.
#include "kc.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kc_host.h"
#include "kc_kernels.cuh"
#include "kc_plan.h"
#include "kc_wide.cuh"

using namespace kc;

namespace {

double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

double hll_estimate(const uint32_t *regs, uint32_t m)
{
    double sum = 0.0;
    uint32_t zeros = 0;
    for (uint32_t i = 0; i < m; ++i) {
        sum += std::ldexp(1.0, -(int)regs[i]);
        zeros += regs[i] == 0;
    }
    double alpha = 0.7213 / (1.0 + 1.079 / m);
    double e = alpha * m * (double)m / sum;
    if (e <= 2.5 * m && zeros) e = m * std::log((double)m / zeros);
    return e;
}

// Default settings (kc_tuning).  The per-bucket tables of the partitioned
// path are filled while they sit in L2, so memory is cheap there and a low
// load factor (short probe runs, fewer L2 operations per insert) pays: 3x
// took the insert from 43.5 ms (1.6x) to 30.7 ms on the large job.  One-table
// jobs and batched samples keep their tables in HBM, where memory counts.
kc_tuning default_tuning()
{
    kc_tuning t{};
    t.bucket_table_factor = 3.0;
    t.table_factor = 1.6;
    t.sort_group_records = 4ull << 20;
    t.bloom_smem = 1;
    t.record_sort = 1;
    t.sampled_region_keys = 64ull << 20;
    t.count_shape = 1;
    t.part_shape = 1;
    t.scatter_shape = 1;
    return t;
}

// Host inputs of a Bloom job from one file of at least this size are
// uploaded in chunks that the census, SCAN and partition follow.
constexpr uint64_t STREAMED_UPLOAD_MIN_BYTES = 512ull << 20;

// k-mers per sub-bucket the shared-memory Bloom path starts from.  Its table
// (SUB_TABLE_SLOTS, 4096) holds the distinct non-FIRST k-mers: at 30x
// coverage with 1% errors about 1k of 24k, a quarter of the table; a
// sub-bucket with more is cut in two and counted again.
constexpr uint64_t SUB_KEYS_TARGET = 24 * 1024;

// A plain job whose table would hold more slots than this (64 MiB of slots,
// half of L2) is counted through the root-prefix buckets.
constexpr uint64_t PLAIN_PART_MIN_SLOTS = 1ull << 22;

// Slots for an estimated `est` distinct keys: 1.6x (load factor <= 0.63 for
// a fair estimate), rounded up to 256 slots; tables need not be powers of two.
uint64_t table_capacity_for(double est, double factor = 1.6)
{
    const uint64_t want = (uint64_t)std::ceil(std::max(est, 16.0) * factor);
    return std::max<uint64_t>(1024, (want + 255) & ~uint64_t(255));
}

int fail(int code, const std::string &msg) { return set_error(code, msg); }

// Working memory of the sort of a job's n records (k-mers of k bases): the
// MSD sort for large jobs, the LSD sort otherwise; both keep the alternate
// arrays at the start (sort_tmp_alt).
// Sub-bucket regions of a large pass (kc_tuning.sampled_region_keys) are
// sized from a 1-in-SUB_REGION_SAMPLE sample of its work items.
constexpr uint32_t SUB_REGION_SAMPLE = 8;

size_t record_sort_bytes(uint64_t n, uint32_t k)
{
    return msd_sort_applies(n, 2 * k) ? std::max(msd_sort_tmp_bytes(n, 2 * k), sort_tmp_bytes(n)) : sort_tmp_bytes(n);
}

}  // namespace

// ---------------------------------------------------------------------------
// jobs and the handle
// ---------------------------------------------------------------------------

namespace {

enum class JobState { QUEUED, RUNNING, DONE, FAILED };

struct Job {
    kc_job_id id = 0;
    kc_job p{};
    std::vector<kc_buffer> files;
    const kc_input *input = nullptr;
    uint64_t reserve = 0;
    JobState state = JobState::QUEUED;
    std::atomic<bool> cancel{false};   // kc_cancel: stop at the next stage boundary
    int err = KC_OK;
    std::string err_msg;
    double t_submit = 0, t_start = 0, t_end = 0;
    // results
    HostRecords recs;
    std::vector<int64_t> hist;
    std::vector<uint64_t> top_keys;
    std::vector<uint32_t> top_counts;
    HostRecords le2;   // records with count <= 2 (pinned: often most of the records)
    PinnedBlock packed;        // kc_job.pack_high: high.bin bytes packed on the device
    uint64_t packed_bytes = 0;
    bool has_packed = false;
    uint64_t occurrences = 0, distinct = 0, low_only = 0, table_cap = 0;
    uint64_t low_len = 0, high_len = 0, input_bytes = 0, n_records_total = 0;
    uint32_t passes = 1, smem_passes = 0, smem_fallbacks = 0, region_redos = 0;
    uint32_t batch_part = 0;   // sub-batch of a batched job
    uint32_t key_words = 1;    // 64-bit words per k-mer in the records (kmer<N>)
    double device_ms = 0;
    double phase_ms[KC_STAGES] = {0};
    uint64_t phase_launches[KC_STAGES] = {0};
};

// Device time and kernel launches per pipeline stage, from CUDA events on
// the job's stream.  Launches are counted on the worker thread that issues
// them, so overlapping jobs on other workers do not mix in.
struct PhaseClock {
    cudaStream_t st;
    struct Span {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<Span> spans;
    int cur = -1;
    cudaEvent_t cur_a = nullptr;
    unsigned long long l0 = 0;
    uint64_t launches[KC_STAGES] = {0};
    explicit PhaseClock(cudaStream_t s) : st(s) {}
    void begin(int phase)
    {
        CK(cudaEventCreate(&cur_a));
        CK(cudaEventRecord(cur_a, st));
        cur = phase;
        l0 = thread_kernel_launches();
    }
    void end()
    {
        cudaEvent_t b;
        CK(cudaEventCreate(&b));
        CK(cudaEventRecord(b, st));
        spans.push_back({cur, cur_a, b});
        launches[cur] += thread_kernel_launches() - l0;
        cur_a = nullptr;
    }
    void collect(double *ms, uint64_t *ln, cudaEvent_t origin)
    {
        static const bool trace = getenv("KC_TRACE") && getenv("KC_TRACE")[0] == '1';
        for (auto &s : spans) {
            float t = 0;
            if (cudaEventElapsedTime(&t, s.a, s.b) == cudaSuccess) ms[s.phase] += t;
            if (trace) {
                float t0 = 0;
                cudaEventElapsedTime(&t0, origin, s.a);
                fprintf(stderr, "[kc trace] stage %d: %.3f .. %.3f ms\n", s.phase, t0, t0 + t);
            }
        }
        for (int i = 0; i < KC_STAGES; ++i) ln[i] += launches[i];
    }
    ~PhaseClock()
    {
        for (auto &s : spans) {
            cudaEventDestroy(s.a);
            cudaEventDestroy(s.b);
        }
        if (cur_a) cudaEventDestroy(cur_a);
    }
};

struct Task {
    std::vector<std::shared_ptr<Job>> jobs;   // one job, or a batch
    bool batch = false;
    uint64_t reserve = 0;
    kc_tuning tuning{};   // the handle's settings when a worker took the task
};

}  // namespace

struct kc_handle {
    int device = 0;
    kc_tuning tuning = default_tuning();   // settings for jobs that start from now on (guarded by mu)
    uint64_t budget = 0;
    uint64_t workspace_bytes = 0;   // per worker, allocated when the worker starts
    uint32_t workers_n = 1;
    uint64_t reserved = 0;
    uint32_t running = 0;
    // a job larger than one worker's share of the budget runs alone: it is
    // admitted when nothing else runs, the idle workers give their kept
    // workspaces back first, and nothing else starts until it ends
    bool exclusive = false;
    std::vector<kc::Workspace *> spaces;   // every worker's workspace (guarded by mu)
    bool closing = false;
    kc_job_id next_id = 1;
    std::mutex mu;
    std::condition_variable cv_work;
    std::condition_variable cv_done;
    std::deque<std::shared_ptr<Task>> queue;
    std::map<kc_job_id, std::shared_ptr<Job>> jobs;
    std::vector<std::thread> workers;
};

namespace {

// ---------------------------------------------------------------------------
// the counting pipeline of one job
// ---------------------------------------------------------------------------

struct Plan {
    uint32_t k;
    bool bloom;
};

void check_flags(unsigned long long flags, const char *where)
{
    if (flags & ERR_WAIT_TIMEOUT) throw KcError{KC_ERR_DEVICE, std::string(where) + ": bounded wait expired"};
    if (flags & ERR_LIST_FULL) throw KcError{KC_ERR_DEVICE, std::string(where) + ": occurrence list overflow"};
    if (flags & ERR_RECORDS_FULL) throw KcError{KC_ERR_DEVICE, std::string(where) + ": record buffer overflow"};
    if (flags & ERR_HIST_OVERFLOW_FULL) throw KcError{KC_ERR_DEVICE, std::string(where) + ": histogram overflow list full"};
}

// A running job that was cancelled stops here (between stages, with none of
// its kernels depending on the host); the worker gives back its memory.
void check_cancel(const Job &job, const char *where)
{
    if (job.cancel.load(std::memory_order_relaxed))
        throw KcError{KC_ERR_CANCELLED, std::string("cancelled (") + where + ")"};
}

struct Counters {
    unsigned long long v[C_COUNT];
};

Counters read_counters(const unsigned long long *d, cudaStream_t st)
{
    static const bool trace = getenv("KC_TRACE") && getenv("KC_TRACE")[0] == '1';
    Counters c{};
    double t0 = trace ? now_ms() : 0;
    CK(cudaMemcpyAsync(c.v, d, sizeof(c.v), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (trace) fprintf(stderr, "[kc trace] counter read-back waited %.3f ms (host clock %.3f)\n", now_ms() - t0, now_ms());
    return c;
}

// Pinned host staging for one job's small uploads and read-backs.  Copies
// between the device and pinned memory are asynchronous, so several
// read-backs share one synchronisation and an upload does not stall the
// host; a region is written by the host only before its copy is queued and
// never reused within the job.  The blocks belong to the worker thread and
// are reused job after job (no pinned allocation per job); the stream is
// drained when the job's staging ends, before the next job reuses them.
struct HostStage {
    cudaStream_t st;
    size_t blk = 0, top = 0;
    bool used = false;
    static std::vector<PinnedBlock> &blocks()
    {
        static thread_local std::vector<PinnedBlock> b;
        return b;
    }
    explicit HostStage(cudaStream_t s) : st(s) {}
    HostStage(const HostStage &) = delete;
    HostStage &operator=(const HostStage &) = delete;
    void *get(size_t bytes)
    {
        bytes = (bytes + 255) & ~size_t(255);
        auto &bs = blocks();
        while (blk < bs.size() && top + bytes > bs[blk].bytes) {
            ++blk;
            top = 0;
        }
        if (blk == bs.size()) {
            PinnedBlock b;
            b.reset(std::max<size_t>(bytes, size_t(1) << 21));
            bs.push_back(std::move(b));
            top = 0;
        }
        used = true;
        void *p = static_cast<uint8_t *>(bs[blk].p) + top;
        top += bytes;
        return p;
    }
    template <class T>
    T *n(size_t count)
    {
        return static_cast<T *>(get(count * sizeof(T)));
    }
    // a pinned copy of count objects, for an upload
    template <class T>
    const T *up(const T *src, size_t count)
    {
        T *p = n<T>(count);
        if (count) std::memcpy(p, src, count * sizeof(T));
        return p;
    }
    ~HostStage()
    {
        if (used) cudaStreamSynchronize(st);
    }
};

// A root-prefix bucket outgrew the region estimated from the sampled census.
struct CensusOverflow {};

// Device memory one counting pass may use: 70% of the free device memory, the
// part of this worker's workspace the job has not used yet, and what the
// stream-ordered pool holds unused.
uint64_t default_pass_budget(Workspace &ws)
{
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const size_t ws_free = ws.capacity() > ws.mark().top ? ws.capacity() - ws.mark().top : 0;
    uint64_t pool_slack = 0;
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t reserved = 0, used = 0;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
            pool_slack = reserved - used;
    }
    cudaGetLastError();
    return (uint64_t)(0.7 * (double)(free_b + ws_free + pool_slack));
}

// kc_job.pack_high: the high.bin bytes of the job's sorted records (k-mer
// words, printed-string order) packed on the device and copied to pinned host
// memory, for kc_write_tmpdir (stage [11]).
void pack_high_on_device(Job &job, DevScope &ds, const unsigned long long *keys, const uint32_t *counts, uint64_t n,
                         cudaStream_t st, PhaseClock &clk)
{
    const kc_job &P = job.p;
    const uint32_t cb = P.count_max <= 0xFF ? 1 : P.count_max <= 0xFFFF ? 2 : P.count_max <= 0xFFFFFF ? 3 : 4;
    const uint64_t rec = packed_record_bytes(P.k, cb);
    const uint64_t m = std::max<uint64_t>(n, 1);
    clk.begin(11);
    uint32_t *flags = ds.n<uint32_t>(m);
    unsigned long long *pos = ds.n<unsigned long long>(m);
    unsigned long long *tmp = ds.n<unsigned long long>(scan_tmp_words(m));
    uint8_t *out = ds.n<uint8_t>(m * rec);
    unsigned long long *nb = ds.n<unsigned long long>(1);
    CK(launch_pack_high(P.k, keys, counts, n, cb, P.filter_min, P.filter_max, flags, pos, tmp, out, nb, st));
    clk.end();
    unsigned long long hb = 0;
    CK(cudaMemcpyAsync(&hb, nb, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    job.packed.reset(std::max<uint64_t>(hb, 1));
    job.packed_bytes = hb;
    if (hb) CK(cudaMemcpyAsync(job.packed.p, out, hb, cudaMemcpyDeviceToHost, st));
    job.has_packed = true;
}

void run_job_once(Job &job, cudaStream_t st, Workspace &ws, bool exact_census, const kc_tuning &tn)
{
    const kc_job &P = job.p;
    const uint32_t k = P.k;
    if (P.fault_inject & KC_INJECT_NOMEM) ws.fail_next_get();
    DevScope ds(st, &ws);
    std::vector<uint32_t> tile_seg_host;

    // ---- input -----------------------------------------------------------
    kc_input local;
    const kc_input *in = job.input;
    static const bool trace_host = getenv("KC_TRACE") && getenv("KC_TRACE")[0] == '1';
    const double th_start = now_ms();
    std::vector<PinnedBlock> inflated;   // gzip files inflated on the host (kept until the job ends)
    // a Bloom job's one large host file goes up in chunks while the census,
    // SCAN and partition work on the chunks that have arrived (declared after
    // the host and device buffers: it drains its copies before they go)
    ChunkedUpload cu;
    bool streamed = false;
    if (!in) {
        const std::vector<kc_buffer> files = inflate_inputs(job.files, inflated);
        streamed = P.bloom && !exact_census && files.size() == 1 && files[0].size >= STREAMED_UPLOAD_MIN_BYTES;
        build_input(local, files.data(), (uint32_t)files.size(), st, &ds, tile_seg_host, nullptr,
                    streamed ? &cu : nullptr);
        in = &local;
        if (trace_host)
            fprintf(stderr, "[kc trace] job upload of %zu files enqueued after %.3f ms\n", job.files.size(),
                    now_ms() - th_start);
    }
    // small uploads and read-backs through pinned staging: a pageable copy
    // would hold the host (and, behind a streamed upload, wait for it)
    HostStage hs(st);
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evg{ev0, ev1};
    CK(cudaEventRecord(ev0, st));
    PhaseClock clk(st);

    const uint64_t T = in->n_tiles;
    const uint32_t n_seg = (uint32_t)in->segs.size();
    std::vector<Seg> segs = in->segs;
    // the pre-pass samples the first 256 MiB of a single file, 128 MiB of each
    // of several files (src/FastqPreReader.h:98-102)
    const uint64_t sample_limit = (in->sizes.size() == 1) ? (256ULL << 20) : (128ULL << 20);
    std::vector<uint64_t> seg_chunk0(std::max<uint32_t>(n_seg, 1), 0);
    uint64_t n_chunks = 0;
    for (uint32_t i = 0; i < n_seg; ++i) {
        segs[i].k = k;
        segs[i].sample = 0;
        segs[i].sample_end = std::min(segs[i].len, sample_limit);
        seg_chunk0[i] = n_chunks;
        n_chunks += (segs[i].len + PREPASS_CHUNK - 1) / PREPASS_CHUNK;
    }
    Seg *d_segs = ds.n<Seg>(std::max<uint32_t>(n_seg, 1));
    if (n_seg) CK(cudaMemcpyAsync(d_segs, hs.up(segs.data(), n_seg), n_seg * sizeof(Seg), cudaMemcpyHostToDevice, st));

    unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
    CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));

    // ---- line numbers of tile starts --------------------------------------
    uint32_t *tile_nl = ds.n<uint32_t>(std::max<uint64_t>(T, 1));
    int32_t *tile_lastnl = ds.n<int32_t>(std::max<uint64_t>(T, 1));
    unsigned long long *tile_prefix = ds.n<unsigned long long>(std::max<uint64_t>(T, 1));
    unsigned long long *scan_tmp = ds.n<unsigned long long>(scan_tmp_words(std::max<uint64_t>(T, 1)));
    // a streamed upload is censused chunk by chunk: the newline counts of the
    // chunks that have arrived, then the line numbers of every tile so far
    size_t chunks_done = 0;
    uint64_t tiles_ready = streamed ? 0 : T;
    auto census_chunks = [&](size_t upto) {
        cu.enqueue(upto);   // (nothing when already queued)
        for (; chunks_done < upto; ++chunks_done) {
            const uint64_t t0 = chunks_done ? cu.tile_end[chunks_done - 1] : 0, t1 = cu.tile_end[chunks_done];
            CK(cudaStreamWaitEvent(st, cu.ev[chunks_done], 0));
            CK(launch_newlines(in->buf + t0 * TILE, t1 - t0, tile_nl + t0, tile_lastnl + t0, st));
        }
        tiles_ready = chunks_done ? cu.tile_end[chunks_done - 1] : 0;
        CK(launch_scan_u32(tile_nl, tile_prefix, tiles_ready, scan_tmp, st));
    };
    clk.begin(0);
    if (streamed) {
        // first the chunks holding the pre-pass sample (with the 2 MiB chunks
        // it ends in) and at least a quarter of the file: the bucket census
        // and the Bloom sizing come from them
        const uint64_t need = std::max<uint64_t>(
            (segs[0].sample_end + PREPASS_CHUNK - 1) / PREPASS_CHUNK * PREPASS_CHUNK, in->total_bytes / 4);
        size_t first = cu.ev.size();
        for (size_t c = 0; c < cu.ev.size(); ++c)
            if (cu.tile_end[c] * TILE >= need) {
                first = c + 1;
                break;
            }
        census_chunks(first);
    } else {
        CK(launch_newlines(in->buf, T, tile_nl, tile_lastnl, st));
        CK(launch_scan_u32(tile_nl, tile_prefix, T, scan_tmp, st));
    }
    clk.end();
    if (P.fault_inject & KC_INJECT_WAIT_TIMEOUT) {
        // a bounded device wait on a word nothing sets (the counter block's
        // last word, zeroed above and never written): it gives up after 1024
        // polls and the flag check after the SCAN ends the job
        CK(launch_wait_flag(reinterpret_cast<const unsigned int *>(counters + C_COUNT - 1), 1024, counters + C_FLAGS,
                            st));
    }

    // ---- SCAN pass ---------------------------------------------------------
    unsigned long long *occ = ds.n<unsigned long long>(1);
    uint32_t *hll = ds.n<uint32_t>(HLL_M);
    CK(cudaMemsetAsync(occ, 0, 8, st));
    CK(cudaMemsetAsync(hll, 0, HLL_M * 4, st));
    ExtractArgs a{};
    a.buf = in->buf;
    a.n_tiles = T;
    a.tile_prefix = reinterpret_cast<const uint64_t *>(tile_prefix);
    a.tile_seg = in->d_tile_seg;
    a.segs = d_segs;
    a.counters = counters;
    a.occ = occ;
    a.hll = hll;
    a.hll_local = 1;
    uint32_t *prefix_hist = nullptr;
    unsigned long long *qual = nullptr;
    unsigned long long *bucket_hist = nullptr;
    clk.begin(1);
    if (P.bloom) {
        a.hll = nullptr;   // the tables are sized from the non-FIRST occurrences instead
        bucket_hist = ds.n<unsigned long long>(N_BUCKETS);
        CK(cudaMemsetAsync(bucket_hist, 0, N_BUCKETS * 8, st));
        a.bucket_hist = bucket_hist;
        // the bucket census reads every 8th tile of large inputs; buckets get
        // regions with headroom and an outgrown region triggers an exact redo
        a.bucket_sample_mask = (exact_census || T < 512) ? 0 : 7;
        if (a.bucket_sample_mask) {
            // only the census tiles and the pre-pass sample of each file are
            // read; the exact occurrence count comes from the partition pass
            std::vector<uint32_t> visit;
            visit.reserve(T / (a.bucket_sample_mask + 1) + 1);
            for (uint32_t i = 0; i < n_seg; ++i) {
                const uint64_t pre = (segs[i].sample_end + TILE - 1) / TILE;
                for (uint64_t t = segs[i].first_tile; t < segs[i].first_tile + segs[i].n_tiles && t < tiles_ready; ++t)
                    if ((t & a.bucket_sample_mask) == 0 || t - segs[i].first_tile < pre) visit.push_back((uint32_t)t);
            }
            uint32_t *d_visit = ds.n<uint32_t>(std::max<size_t>(visit.size(), 1));
            if (!visit.empty())
                CK(cudaMemcpyAsync(d_visit, hs.up(visit.data(), visit.size()), visit.size() * 4,
                                   cudaMemcpyHostToDevice, st));
            a.visit = d_visit;
            a.n_visit = visit.size();
        }
        int32_t *chunk_lastnl = ds.n<int32_t>(std::max<uint64_t>(n_chunks, 1));
        uint64_t *d_chunk0 = ds.n<uint64_t>(seg_chunk0.size());
        prefix_hist = ds.n<uint32_t>(256);
        qual = ds.n<unsigned long long>(2);
        CK(cudaMemsetAsync(chunk_lastnl, 0xff, std::max<uint64_t>(n_chunks, 1) * 4, st));
        CK(cudaMemcpyAsync(d_chunk0, hs.up(seg_chunk0.data(), seg_chunk0.size()), seg_chunk0.size() * 8,
                           cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(prefix_hist, 0, 256 * 4, st));
        CK(cudaMemsetAsync(qual, 0, 16, st));
        CK(launch_chunk_lastnl(tile_lastnl, in->d_tile_seg, d_segs, d_chunk0, tiles_ready, chunk_lastnl, st));
        a.prepass = 1;
        a.chunk_lastnl = chunk_lastnl;
        a.seg_chunk0 = d_chunk0;
        a.prefix_hist = prefix_hist;
        a.qual = qual;
    } else {
        // plain jobs: an exact root-prefix census beside the distinct
        // estimate, for the partitioned path of large tables
        bucket_hist = ds.n<unsigned long long>(N_BUCKETS);
        CK(cudaMemsetAsync(bucket_hist, 0, N_BUCKETS * 8, st));
        a.bucket_hist = bucket_hist;
        a.bucket_sample_mask = 0;
    }
    CK(launch_extract(MODE_SCAN, a, 0, st));
    clk.end();
    // the SCAN's results (and the bucket census) come back under one sync
    unsigned long long *p_occ = hs.n<unsigned long long>(1);
    uint32_t *p_hll = hs.n<uint32_t>(HLL_M);
    uint32_t *p_ph = hs.n<uint32_t>(256);
    unsigned long long *p_qh = hs.n<unsigned long long>(2);
    unsigned long long *p_bh = hs.n<unsigned long long>(N_BUCKETS);
    unsigned long long *p_c0 = hs.n<unsigned long long>(C_COUNT);
    CK(cudaMemcpyAsync(p_occ, occ, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p_hll, hll, HLL_M * 4, cudaMemcpyDeviceToHost, st));
    if (P.bloom) {
        CK(cudaMemcpyAsync(p_ph, prefix_hist, 256 * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(p_qh, qual, 16, cudaMemcpyDeviceToHost, st));
    }
    if (bucket_hist) CK(cudaMemcpyAsync(p_bh, bucket_hist, N_BUCKETS * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p_c0, counters, C_COUNT * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<uint32_t> hll_h(p_hll, p_hll + HLL_M);
    unsigned long long O = *p_occ;
    std::vector<uint32_t> ph(256, 0);
    unsigned long long qh[2] = {0, 0};
    if (P.bloom) {
        ph.assign(p_ph, p_ph + 256);
        qh[0] = p_qh[0];
        qh[1] = p_qh[1];
    }
    Counters c0{};
    std::memcpy(c0.v, p_c0, sizeof(c0.v));
    check_flags(c0.v[C_FLAGS], "scan");
    check_cancel(job, "after the census");
    job.occurrences = O;

    // ---- counting ---------------------------------------------------------
    const uint32_t count_max = P.count_max ? P.count_max : 255u;
    const uint32_t max_probe_cap = 1u << 16;
    const double est = hll_estimate(hll_h.data(), HLL_M);
    unsigned long long *hist = ds.n<unsigned long long>(HIST_BINS);
    // counts of HIST_BINS or more go to a list: a k-mer that often needs
    // HIST_BINS occurrences, so O / HIST_BINS bounds the list (heavily
    // repeated genomes reach millions of such k-mers)
    const uint64_t ovf_cap = std::max<uint64_t>(1ull << 20, O / HIST_BINS + 1);
    uint32_t *ovf = ds.n<uint32_t>(ovf_cap);
    unsigned long long *n_keys = ds.n<unsigned long long>(1);
    CK(cudaMemsetAsync(hist, 0, HIST_BINS * 8, st));
    unsigned long long low_len = 0, high_len = 0;
    uint64_t table_cap = 0;
    job.distinct = job.low_only = 0;
    job.smem_passes = job.smem_fallbacks = job.region_redos = 0;

    // Records of one counted table: the FIRST occurrences are merged in (Bloom
    // mode), every occupied slot is compacted into new record arrays, and the
    // histogram (shared by all tables of the job) is added to.
    unsigned long long *rec_keys = nullptr;
    uint32_t *rec_counts = nullptr;
    uint64_t n_rec = 0;
    // Slot-order records of a bucket arena are grouped by bucket, and the
    // bucket (root prefix) is the lowest 8 bits of the printed-order sort key:
    // the sort then skips that pass.
    // into_sort_tmp: the records are written into the sort's alternate
    // buffers, from which an odd number of passes ends in rec_keys/rec_counts.
    bool rec_by_bucket = true, rec_in_sort_tmp = false;
    // the records per value of their keys' top 16 bits, when the count made
    // it as it wrote them (a one-pass Bloom job): the sort's bucket histogram
    uint32_t *rec_hist16 = nullptr;
    void *sort_tmp = nullptr;
    auto compact_table = [&](const TableRef &t, uint64_t cap, uint64_t n_low, const unsigned long long *lst,
                             const BucketRanges *low_rg, uint32_t n_low_items, unsigned int *merge_next,
                             const BucketCfg *d_cfg, bool bucket_arena, bool into_sort_tmp) {
        CK(cudaMemsetAsync(counters + C_REC_LEN, 0, 3 * 8, st));   // C_REC_LEN, C_LOW_ONLY, C_DISTINCT
        const bool want1 = P.min_count <= 1 && 1 <= P.max_count;
        bool ordered = true;
        if (n_low && want1) {
            // the FIRST-only k-mers are records too (count 1): the merge
            // appends them as it finds them, then the table's records follow
            ordered = false;
            rec_by_bucket = false;
            CK(cudaMemsetAsync(n_keys, 0, 8, st));
            clk.begin(5);
            CK(launch_count_keys(t.slots, cap, n_keys, st));
            clk.end();
            unsigned long long in_table = 0;
            CK(cudaMemcpyAsync(&in_table, n_keys, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const uint64_t rec_cap = std::max<uint64_t>(in_table + n_low, 1);
            rec_keys = ds.n<unsigned long long>(rec_cap);
            rec_counts = ds.n<uint32_t>(rec_cap);
            clk.begin(4);
            CK(launch_merge_buckets(lst, low_rg, n_low_items, merge_next, d_cfg, t.slots, max_probe_cap,
                                    P.min_count, P.max_count, rec_keys, rec_counts, rec_cap, counters, st));
            clk.end();
            clk.begin(5);
            CK(launch_compact(t, cap, count_max, P.min_count, P.max_count, rec_keys, rec_counts, rec_cap, hist, ovf,
                              ovf_cap, counters, st));
            clk.end();
        } else {
            // merge (no records), count the records of every chunk of slots,
            // place the chunks by a scan, then write the records in slot order
            if (n_low) {
                clk.begin(4);
                CK(launch_merge_buckets(lst, low_rg, n_low_items, merge_next, d_cfg, t.slots, max_probe_cap,
                                        P.min_count, P.max_count, nullptr, nullptr, 0, counters, st));
                clk.end();
            }
            if (!bucket_arena) rec_by_bucket = false;
            const uint64_t n_chunks = std::max<uint64_t>(compact_ordered_chunks(cap), 1);
            uint32_t *chunk_keep = ds.n<uint32_t>(n_chunks);
            unsigned long long *chunk_pos = ds.n<unsigned long long>(n_chunks);
            unsigned long long *scan_tmp = ds.n<unsigned long long>(scan_tmp_words(n_chunks));
            CK(cudaMemsetAsync(chunk_keep, 0, n_chunks * 4, st));
            clk.begin(5);
            CK(launch_compact_ordered(t.slots, cap, count_max, P.min_count, P.max_count, chunk_keep, nullptr, nullptr,
                                      nullptr, 0, hist, ovf, ovf_cap, counters, 1, st));
            CK(launch_scan_u32(chunk_keep, chunk_pos, n_chunks, scan_tmp, st));
            clk.end();
            unsigned long long last_pos = 0;
            uint32_t last_keep = 0;
            CK(cudaMemcpyAsync(&last_pos, chunk_pos + n_chunks - 1, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&last_keep, chunk_keep + n_chunks - 1, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            n_rec = last_pos + last_keep;
            rec_keys = ds.n<unsigned long long>(std::max<uint64_t>(n_rec, 1));
            rec_counts = ds.n<uint32_t>(std::max<uint64_t>(n_rec, 1));
            unsigned long long *wk = rec_keys;
            uint32_t *wc = rec_counts;
            if (into_sort_tmp && n_rec > 1) {
                sort_tmp = ds.get(record_sort_bytes(n_rec, k));
                sort_tmp_alt(sort_tmp, n_rec, &wk, &wc);
                rec_in_sort_tmp = true;
            }
            clk.begin(5);
            CK(launch_compact_ordered(t.slots, cap, count_max, P.min_count, P.max_count, chunk_keep, chunk_pos, wk,
                                      wc, n_rec, hist, ovf, ovf_cap, counters, 0, st));
            clk.end();
        }
        Counters c2 = read_counters(counters, st);
        check_flags(c2.v[C_FLAGS], "compact");
        if (c2.v[C_FLAGS] & ERR_TABLE_FULL) throw KcError{KC_ERR_DEVICE, "counting table lookup overflow"};
        if (!ordered) n_rec = c2.v[C_REC_LEN];
        job.distinct += c2.v[C_DISTINCT] + c2.v[C_LOW_ONLY];
        job.low_only += c2.v[C_LOW_ONLY];
    };

    // a plain job whose table would not fit in L2 takes the partitioned path
    // too (without the Bloom split): scattered by root prefix, every bucket's
    // sub-table is filled while it sits in L2
    const bool plain_part = !P.bloom && table_capacity_for(est, tn.table_factor) > PLAIN_PART_MIN_SLOTS;
    if (!P.bloom && !plain_part) {
        TableRef tr{};
        TableRef *d_tr = ds.n<TableRef>(1);
        uint64_t cap = table_capacity_for(est, tn.table_factor);
        for (int attempt = 0;; ++attempt) {
            if (tr.slots) ds.release(tr.slots);
            tr.slots = static_cast<Slot *>(ds.get(cap * sizeof(Slot)));
            tr.mask = cap - 1;
            CK(launch_init_slots(tr.slots, cap, st));
            CK(cudaMemcpyAsync(d_tr, &tr, sizeof(tr), cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(counters, 0, 8, st));
            a.tables = d_tr;
            a.max_probe = (uint32_t)std::min<uint64_t>(cap, max_probe_cap);
            clk.begin(2);
            CK(launch_extract(MODE_INSERT, a, 0, st));
            clk.end();
            if ((P.fault_inject & KC_INJECT_TABLE_FULL) || (attempt == 0 && (P.fault_inject & KC_INJECT_TABLE_FULL_ONCE)))
                CK(launch_or_flags(counters + C_FLAGS, ERR_TABLE_FULL, st));
            Counters c = read_counters(counters, st);
            check_flags(c.v[C_FLAGS], "insert");
            if (!(c.v[C_FLAGS] & ERR_TABLE_FULL)) break;
            if (attempt >= 3) throw KcError{KC_ERR_DEVICE, "counting table overflow"};
            check_cancel(job, "table regrowth");
            cap *= 2;
        }
        table_cap = cap;
        compact_table(tr, cap, 0, nullptr, nullptr, 0, nullptr, nullptr, false, false);
    } else {
        // ---- root-prefix buckets (the reference's 256 root prefixes,
        // src/NewKmerTree.h:1488-1495): sizes from the SCAN census, one
        // scatter pass, then every bucket's Bloom filter and table slice is
        // processed while it sits in L2
        if (!bucket_hist) throw KcError{KC_ERR_DEVICE, "partitioned job without a bucket census"};
        const std::vector<unsigned long long> bh(p_bh, p_bh + N_BUCKETS);
        std::vector<unsigned long long> region(N_BUCKETS);
        unsigned long long sampled = 0;
        for (uint32_t b = 0; b < N_BUCKETS; ++b) sampled += bh[b];
        const bool exact = a.bucket_sample_mask == 0;
        // SCAN counted the occurrences of the census tiles (all tiles when exact)
        if (sampled != O) throw KcError{KC_ERR_DEVICE, "bucket census does not add up to the occurrences"};
        if (!exact && sampled < 65536) throw CensusOverflow{};   // too thin a sample
        // census tiles: t with (t & mask) == 0 among the tiles censused so far
        const double scale =
            exact ? 1.0
                  : (double)T / (double)((tiles_ready + a.bucket_sample_mask) / (a.bucket_sample_mask + 1));
        for (uint32_t b = 0; b < N_BUCKETS; ++b)
            region[b] = exact ? bh[b] : (unsigned long long)std::ceil((double)bh[b] * scale * 1.15) + 8192;
        std::vector<uint64_t> fcap(N_BUCKETS, 0);
        if (P.bloom) {
            // reference sizing (src/main.cpp:41-153) from the pre-pass statistics
            uint8_t avg_q = qh[1] ? (uint8_t)(qh[0] / qh[1]) : 0;
            BloomPlan bp = bloom_plan(ph.data(), avg_q, in->total_bytes, P.memory_gb, k);
            for (uint32_t b = 0; b < N_BUCKETS; ++b) fcap[b] = bp.caps[b];
        }
        // passes over ranges of buckets, each within the device-memory budget
        // of a pass (k-mer arrays, filters, tables, records of its buckets)
        const uint64_t budget = P.pass_bytes ? P.pass_bytes : default_pass_budget(ws);
        const uint64_t per_occ = P.bloom ? 42 : 48;
        std::vector<std::pair<uint32_t, uint32_t>> ranges;
        {
            uint32_t lo = 0;
            uint64_t need = 0;
            for (uint32_t b = 0; b < N_BUCKETS; ++b) {
                const uint64_t nb = region[b] * per_occ + fcap[b] * 16;
                if (b > lo && need + nb > budget) {
                    ranges.push_back({lo, b});
                    lo = b;
                    need = 0;
                }
                need += nb;
            }
            ranges.push_back({lo, N_BUCKETS});
        }
        const bool multi = ranges.size() > 1;
        if (streamed && multi) census_chunks(cu.ev.size());   // every pass reads every tile
        std::vector<std::unique_ptr<HostRecords>> spilled;
        uint64_t spilled_total = 0, filled_total = 0;
        for (const auto &rg : ranges) {
            const uint32_t lo = rg.first, hi = rg.second;
            const DevScope::Mark mk = ds.mark();
            std::vector<BucketCfg> cfg(N_BUCKETS);
            unsigned long long off = 0, words = 0;
            for (uint32_t b = lo; b < hi; ++b) {
                cfg[b].key_base = off;
                off += region[b];
                cfg[b].bloom_off = words;
                cfg[b].bloom_cap = fcap[b];
                words += 2 * fcap[b];
            }
            const unsigned long long ocap = std::max<unsigned long long>(off, 1);
            // allocation order lets the scattered k-mers and then the filter be
            // given back before the tables are laid out (Bloom mode); without
            // the Bloom split the scattered k-mers are the insert's input
            unsigned long long *list = nullptr, *bits = nullptr, *keys = nullptr;
            unsigned long long list_cap = ocap;
            if (P.bloom) {
                // room for the sub-buckets' estimated regions (their sizes plus
                // about 15% on a large pass)
                list_cap = ocap + ocap / 4 + 65536;
                list = ds.n<unsigned long long>(list_cap);
                bits = ds.n<unsigned long long>(std::max<unsigned long long>(words, 1));
                keys = ds.n<unsigned long long>(ocap);
            } else {
                keys = ds.n<unsigned long long>(ocap);
                list = keys;
            }
            BucketCfg *d_cfg_b = ds.n<BucketCfg>(N_BUCKETS);
            unsigned long long *cursor = ds.n<unsigned long long>(N_BUCKETS);
            unsigned long long *bbase = ds.n<unsigned long long>(2 * N_BUCKETS);
            unsigned long long *lh_cnt = ds.n<unsigned long long>(2 * N_BUCKETS);
            uint32_t *hll_high = ds.n<uint32_t>((size_t)N_BUCKETS * BUCKET_HLL_M);
            unsigned int *next_item = ds.n<unsigned int>(1);
            std::vector<unsigned long long> bb(2 * N_BUCKETS, 0);
            for (uint32_t b = lo; b < hi; ++b) {
                bb[b] = cfg[b].key_base;
                bb[N_BUCKETS + b] = cfg[b].key_base + region[b];
            }
            CK(cudaMemsetAsync(cursor, 0, N_BUCKETS * 8, st));
            CK(cudaMemcpyAsync(bbase, hs.up(bb.data(), bb.size()), 2 * N_BUCKETS * 8, cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(lh_cnt, 0, 2 * N_BUCKETS * 8, st));
            CK(cudaMemsetAsync(hll_high, 0, (size_t)N_BUCKETS * BUCKET_HLL_M * 4, st));
            a.hll = nullptr;
            a.prepass = 0;
            a.bucket_hist = nullptr;
            a.list = keys;
            a.list_cap = ocap;
            a.bucket_cursor = cursor;
            a.bucket_base = bbase;
            a.bucket_end = bbase + N_BUCKETS;
            a.bucket_lo = lo;
            a.bucket_hi = hi;
            clk.begin(2);
            if (streamed && chunks_done < cu.ev.size()) {
                // the rest of the file goes up behind this pass's small uploads;
                // the tiles whose chunks have arrived are partitioned, then each
                // later chunk once it has landed and has its line numbers
                cu.enqueue(cu.ev.size());
                a.tile0 = 0;
                a.n_tiles = tiles_ready;
                CK(launch_extract(MODE_PART, a, 0, st, (uint32_t)tn.part_shape));
                while (chunks_done < cu.ev.size()) {
                    const uint64_t t0 = tiles_ready;
                    census_chunks(chunks_done + 1);
                    a.tile0 = t0;
                    a.n_tiles = tiles_ready - t0;
                    CK(launch_extract(MODE_PART, a, 0, st, (uint32_t)tn.part_shape));
                }
                a.tile0 = 0;
                a.n_tiles = T;
            } else {
                CK(launch_extract(MODE_PART, a, 0, st, (uint32_t)tn.part_shape));
            }
            clk.end();
            unsigned long long *p_fill = hs.n<unsigned long long>(N_BUCKETS);
            CK(cudaMemcpyAsync(p_fill, cursor, N_BUCKETS * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const std::vector<unsigned long long> fill(p_fill, p_fill + N_BUCKETS);
            check_cancel(job, "after the partition");
            for (uint32_t b = lo; b < hi; ++b) {
                if (fill[b] > region[b]) throw CensusOverflow{};
                cfg[b].key_len = fill[b];
                filled_total += fill[b];
            }
            CK(cudaMemcpyAsync(d_cfg_b, hs.up(cfg.data(), N_BUCKETS), N_BUCKETS * sizeof(BucketCfg),
                               cudaMemcpyHostToDevice, st));
            // each bucket-major launch gets its 256 ranges, not a list of items
            auto upload_ranges = [&](BucketRanges &r, uint32_t &n_items) {
                n_items = fill_item_starts(r);
                BucketRanges *d = ds.n<BucketRanges>(1);
                CK(cudaMemcpyAsync(d, hs.up(&r, 1), sizeof(BucketRanges), cudaMemcpyHostToDevice, st));
                return d;
            };
            // Bloom jobs whose records need count >= 2: the Bloom split, the
            // counting and the compaction run per sub-bucket (a slice of its
            // bucket's filter) in shared memory.  A bucket starts with about
            // SUB_KEYS_TARGET k-mers per sub-bucket (and slices of at most
            // SUB_SLICE_BLOCKS blocks); a bucket whose table overflowed is
            // counted again with twice the sub-buckets, and a bucket that
            // cannot be cut further sends the pass to the global-memory path.
            bool sub_done = false;
            if (P.bloom && P.min_count >= 2 && tn.bloom_smem == 1) {
                // the count kernel's block shape: its slice and table sizes
                // set the sub-buckets (a table of 2048 slots takes half the k-mers)
                const uint32_t shape = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(tn.count_shape, 4));
                const uint64_t keys_target = SUB_KEYS_TARGET * sub_table_slots(shape) / SUB_TABLE_SLOTS;
                std::vector<uint32_t> nsub(N_BUCKETS, 0);
                bool eligible = true;
                for (uint32_t b = lo; b < hi; ++b) {
                    const uint64_t f = fcap[b];
                    if (!f || (f & (f - 1))) {
                        eligible = false;
                        break;
                    }
                    uint64_t want = std::max<uint64_t>(f / sub_slice_blocks(shape), (cfg[b].key_len + keys_target - 1) / keys_target);
                    want = std::max<uint64_t>(bit_ceil64(want), 1);
                    if (want > std::min<uint64_t>(f, SUB_MAX_PER_BUCKET)) {
                        eligible = false;
                        break;
                    }
                    nsub[b] = (uint32_t)want;
                }
                // the overflow list's length before the attempts, restored after
                // a failed one (on the device: no round trip)
                unsigned long long *ovf_len_saved = ds.n<unsigned long long>(1);
                CK(cudaMemcpyAsync(ovf_len_saved, counters + C_OVF_LEN, 8, cudaMemcpyDeviceToDevice, st));
                // a large pass sizes the sub-buckets' regions from a sample of
                // its keys instead of counting them all; a sub-bucket that
                // outgrows its region sends the pass back to exact counts
                bool exact_regions = false;
                for (int attempt = 0; eligible && !sub_done; ++attempt) {
                    const DevScope::Mark m0 = ds.mark();
                    std::vector<SubCfg> sc(N_BUCKETS);
                    std::vector<uint8_t> sb;
                    uint32_t n_sub = 0;
                    uint64_t pass_keys = 0;
                    for (uint32_t b = lo; b < hi; ++b) {
                        sc[b].fcap = fcap[b];
                        sc[b].sub_base = n_sub;
                        sc[b].n_sub = nsub[b];
                        sc[b].slice_shift = (uint32_t)__builtin_ctzll(fcap[b] / nsub[b]);
                        n_sub += nsub[b];
                        sb.insert(sb.end(), nsub[b], (uint8_t)b);
                        pass_keys += cfg[b].key_len;
                    }
                    SubCfg *d_sc = ds.n<SubCfg>(N_BUCKETS);
                    uint8_t *d_sb = ds.n<uint8_t>(std::max<uint32_t>(n_sub, 1));
                    uint32_t *sub_count = ds.n<uint32_t>(std::max<uint32_t>(n_sub, 1));
                    unsigned long long *sub_off = ds.n<unsigned long long>(std::max<uint32_t>(n_sub, 1));
                    unsigned long long *sub_cur = ds.n<unsigned long long>(std::max<uint32_t>(n_sub, 1));
                    unsigned long long *sub_tmp =
                        ds.n<unsigned long long>(scan_tmp_words(std::max<uint32_t>(n_sub, 1)));
                    unsigned int *sub_next = ds.n<unsigned int>(1);
                    uint32_t *bucket_ovf = ds.n<uint32_t>(N_BUCKETS);
                    unsigned long long *hist_sub = ds.n<unsigned long long>(HIST_BINS);
                    // a record has count >= 2: at most half the occurrences, and at
                    // most one table of slots per sub-bucket
                    const uint64_t rcap = std::max<uint64_t>(
                        std::min<uint64_t>((uint64_t)n_sub * sub_table_slots(shape), pass_keys / 2 + 1), 1);
                    unsigned long long *rk = ds.n<unsigned long long>(rcap);
                    uint32_t *rc = ds.n<uint32_t>(rcap);
                    BucketRanges br{};
                    for (uint32_t b = lo; b < hi; ++b) {
                        br.begin[b] = cfg[b].key_base;
                        br.len[b] = cfg[b].key_len;
                    }
                    uint32_t n_items = 0;
                    BucketRanges *d_br = upload_ranges(br, n_items);
                    CK(cudaMemcpyAsync(d_sc, hs.up(sc.data(), N_BUCKETS), N_BUCKETS * sizeof(SubCfg),
                                       cudaMemcpyHostToDevice, st));
                    if (n_sub) CK(cudaMemcpyAsync(d_sb, hs.up(sb.data(), n_sub), n_sub, cudaMemcpyHostToDevice, st));
                    CK(cudaMemsetAsync(sub_count, 0, std::max<uint32_t>(n_sub, 1) * 4, st));
                    CK(cudaMemsetAsync(bucket_ovf, 0, N_BUCKETS * 4, st));
                    CK(cudaMemsetAsync(hist_sub, 0, HIST_BINS * 8, st));
                    CK(cudaMemsetAsync(counters + C_LOW_LEN, 0, 2 * 8, st));   // C_LOW_LEN, C_HIGH_LEN
                    CK(cudaMemsetAsync(counters + C_REC_LEN, 0, 3 * 8, st));   // C_REC_LEN, C_LOW_ONLY, C_DISTINCT
                    CK(cudaMemsetAsync(counters + C_SUB_OVF, 0, 2 * 8, st));   // C_SUB_OVF, C_REGION_OVF
                    const bool sampled = !exact_regions && pass_keys >= tn.sampled_region_keys;
                    unsigned long long *sub_end = nullptr;
                    clk.begin(9);
                    if (sampled) {
                        uint32_t *region = ds.n<uint32_t>(std::max<uint32_t>(n_sub, 1));
                        sub_end = ds.n<unsigned long long>(std::max<uint32_t>(n_sub, 1));
                        CK(launch_subpart_count(keys, d_br, n_items, d_sc, sub_count, st, SUB_REGION_SAMPLE));
                        CK(launch_subpart_regions(sub_count, n_sub, SUB_REGION_SAMPLE, region, sub_off, sub_end, sub_cur,
                                                  sub_tmp, st));
                    } else {
                        CK(launch_subpart_count(keys, d_br, n_items, d_sc, sub_count, st));
                        CK(launch_scan_u32(sub_count, sub_off, n_sub, sub_tmp, st));
                        if (n_sub)
                            CK(cudaMemcpyAsync(sub_cur, sub_off, (size_t)n_sub * 8, cudaMemcpyDeviceToDevice, st));
                    }
                    const uint32_t max_sub = *std::max_element(nsub.begin(), nsub.end());
                    BucketRanges bs = br;
                    const uint32_t n_sp_items = fill_item_starts_n(bs, SUB_SCATTER_ITEM_KEYS);
                    BucketRanges *d_bs = ds.n<BucketRanges>(1);
                    CK(cudaMemcpyAsync(d_bs, hs.up(&bs, 1), sizeof(BucketRanges), cudaMemcpyHostToDevice, st));
                    CK(launch_subpart_scatter(keys, d_bs, n_sp_items, sub_next, d_sc, sub_cur, list, list_cap, max_sub,
                                              st, sub_end, (uint32_t)tn.scatter_shape));
                    if (sampled)
                        CK(launch_subpart_sizes(sub_off, sub_cur, sub_end, n_sub, list_cap, sub_count,
                                                counters + C_REGION_OVF, st));
                    clk.end();
                    clk.begin(10);
                    uint32_t *hb16 = nullptr;
                    if (!multi && 2 * k >= 24) {
                        hb16 = ds.n<uint32_t>(1u << 16);
                        CK(cudaMemsetAsync(hb16, 0, (1u << 16) * 4, st));
                    }
                    CK(launch_count_subs(list, sub_off, sub_count, d_sb, n_sub, d_sc, sub_next, count_max,
                                         P.min_count, P.max_count, rk, rc, rcap, hist_sub, ovf, ovf_cap, counters,
                                         bucket_ovf, st, hb16, 2 * k - 16, shape));
                    clk.end();
                    if (attempt == 0 && (P.fault_inject & KC_INJECT_TABLE_FULL_ONCE)) {
                        // as if the first bucket's sub-bucket tables had overflowed
                        CK(cudaMemsetAsync(bucket_ovf + lo, 0x01, 1, st));
                        CK(launch_or_flags(counters + C_SUB_OVF, 1ull, st));
                    }
                    const Counters cs = read_counters(counters, st);
                    check_flags(cs.v[C_FLAGS], "sub-bucket count");
                    if (cs.v[C_REGION_OVF]) {
                        // a sub-bucket outgrew its estimated region: count again
                        // with exact regions (same sub-buckets)
                        CK(cudaMemcpyAsync(counters + C_OVF_LEN, ovf_len_saved, 8, cudaMemcpyDeviceToDevice, st));
                        CK(cudaStreamSynchronize(st));
                        ds.rewind(m0);
                        exact_regions = true;
                        ++job.region_redos;
                        continue;
                    }
                    if (cs.v[C_SUB_OVF] == 0) {
                        CK(launch_add_u64(hist, hist_sub, HIST_BINS, st));
                        rec_keys = rk;
                        rec_counts = rc;
                        n_rec = cs.v[C_REC_LEN];
                        rec_by_bucket = false;
                        rec_hist16 = hb16;
                        job.distinct += cs.v[C_DISTINCT] + cs.v[C_LOW_ONLY];
                        job.low_only += cs.v[C_LOW_ONLY];
                        low_len += cs.v[C_LOW_LEN];
                        high_len += cs.v[C_HIGH_LEN];
                        table_cap = std::max<uint64_t>(table_cap, (uint64_t)n_sub * sub_table_slots(shape));
                        ++job.smem_passes;
                        sub_done = true;
                        break;
                    }
                    // buckets that held more distinct repeated k-mers than their
                    // sub-buckets' tables: twice the sub-buckets next time
                    std::vector<uint32_t> bo(N_BUCKETS);
                    CK(cudaMemcpyAsync(bo.data(), bucket_ovf, N_BUCKETS * 4, cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(counters + C_OVF_LEN, ovf_len_saved, 8, cudaMemcpyDeviceToDevice, st));
                    CK(cudaStreamSynchronize(st));
                    ds.rewind(m0);
                    bool any = false;
                    for (uint32_t b = lo; b < hi; ++b) {
                        if (!bo[b]) continue;
                        any = true;
                        if ((uint64_t)nsub[b] * 2 > std::min<uint64_t>(fcap[b], SUB_MAX_PER_BUCKET)) eligible = false;
                        else nsub[b] *= 2;
                    }
                    if (!any) eligible = false;
                    if (!eligible) ++job.smem_fallbacks;
                }
            }
            if (!sub_done) {
                std::vector<unsigned long long> lh(2 * N_BUCKETS, 0);
                std::vector<uint32_t> hh;
                if (P.bloom) {
                    CK(cudaMemsetAsync(bits, 0, words * 8, st));
                    clk.begin(8);
                    BucketRanges br{};
                    for (uint32_t b = lo; b < hi; ++b) {
                        br.begin[b] = cfg[b].key_base;
                        br.len[b] = cfg[b].key_len;
                    }
                    uint32_t n_items = 0;
                    BucketRanges *d_br = upload_ranges(br, n_items);
                    CK(launch_bloom_buckets(keys, d_br, n_items, next_item, d_cfg_b, bits, list, lh_cnt, lh_cnt + N_BUCKETS,
                                            hll_high, st));
                    clk.end();
                    hh.resize((size_t)N_BUCKETS * BUCKET_HLL_M);
                    CK(cudaMemcpyAsync(lh.data(), lh_cnt, 2 * N_BUCKETS * 8, cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(hh.data(), hll_high, hh.size() * 4, cudaMemcpyDeviceToHost, st));
                    ds.release(d_br);
                } else {
                    // every occurrence goes to the table: the whole bucket is "high"
                    for (uint32_t b = lo; b < hi; ++b) lh[N_BUCKETS + b] = cfg[b].key_len;
                }
                Counters c = read_counters(counters, st);
                check_flags(c.v[C_FLAGS], "partition");
                ds.release(next_item);
                ds.release(hll_high);
                ds.release(lh_cnt);
                ds.release(bbase);
                ds.release(cursor);
                ds.release(d_cfg_b);
                if (P.bloom) {
                    ds.release(keys);
                    ds.release(bits);
                }
                uint64_t pass_low = 0;
                std::vector<uint64_t> bcaps(N_BUCKETS, 0);
                for (uint32_t b = lo; b < hi; ++b) {
                    const unsigned long long hb = lh[N_BUCKETS + b];
                    pass_low += lh[b];
                    high_len += hb;
                    double e;
                    if (P.bloom) {
                        // the registers hold a hash sample of the non-FIRST k-mers
                        e = hb ? (double)(1u << BUCKET_HLL_SAMPLE_BITS) *
                                     hll_estimate(&hh[(size_t)b * BUCKET_HLL_M], BUCKET_HLL_M)
                               : 0.0;
                    } else {
                        // the job's distinct estimate, shared out by occurrences
                        e = O ? est * (double)hb / (double)O : 0.0;
                        e = std::min(e, (double)hb);
                    }
                    e = std::max(e, (double)std::min<unsigned long long>(hb, 4096));
                    bcaps[b] = table_capacity_for(e, tn.bucket_table_factor);
                }
                low_len += pass_low;
                // per-bucket sub-tables in one arena; a bucket whose table
                // overflows gets twice the slots and the insert is repeated
                BucketCfg *d_cfg = ds.n<BucketCfg>(N_BUCKETS);
                unsigned long long *bucket_ovf = ds.n<unsigned long long>(N_BUCKETS);
                next_item = ds.n<unsigned int>(1);
                unsigned int *merge_next = ds.n<unsigned int>(1);
                BucketRanges hr{}, lr{};
                for (uint32_t b = lo; b < hi; ++b) {
                    hr.begin[b] = cfg[b].key_base + cfg[b].key_len - lh[N_BUCKETS + b];
                    hr.len[b] = lh[N_BUCKETS + b];
                    lr.begin[b] = cfg[b].key_base;
                    lr.len[b] = lh[b];
                }
                uint32_t n_high_items = 0, n_low_items = 0;
                BucketRanges *d_hr = upload_ranges(hr, n_high_items);
                BucketRanges *d_lr = upload_ranges(lr, n_low_items);
                TableRef tr{};
                uint64_t cap = 0;
                for (int attempt = 0;; ++attempt) {
                    // sub-tables in the order of the sort key's lowest byte: bucket
                    // b (the internal word's top byte, four bases) is that byte with
                    // its 2-bit groups reversed, so the slot-order records come out
                    // in order of the first sort digit
                    cap = 0;
                    for (uint32_t r = 0; r < N_BUCKETS; ++r) {
                        const uint32_t b = ((r & 3u) << 6) | (((r >> 2) & 3u) << 4) | (((r >> 4) & 3u) << 2) | (r >> 6);
                        cfg[b].slot_base = cap;
                        cfg[b].slot_cap = bcaps[b];
                        cap += bcaps[b];
                    }
                    if (tr.slots) ds.release(tr.slots);
                    tr.slots = static_cast<Slot *>(ds.get(std::max<uint64_t>(cap, 1) * sizeof(Slot)));
                    tr.mask = 0;   // the arena is addressed per bucket
                    CK(launch_init_slots(tr.slots, cap, st));
                    CK(cudaMemcpyAsync(d_cfg, cfg.data(), N_BUCKETS * sizeof(BucketCfg), cudaMemcpyHostToDevice, st));
                    CK(cudaMemsetAsync(bucket_ovf, 0, N_BUCKETS * 8, st));
                    clk.begin(3);
                    CK(launch_insert_buckets(list, d_hr, n_high_items, next_item, d_cfg, tr.slots, max_probe_cap, bucket_ovf,
                                             st));
                    clk.end();
                    std::vector<unsigned long long> ov(N_BUCKETS);
                    CK(cudaMemcpyAsync(ov.data(), bucket_ovf, N_BUCKETS * 8, cudaMemcpyDeviceToHost, st));
                    Counters cc = read_counters(counters, st);
                    check_flags(cc.v[C_FLAGS], "insert");
                    bool any = false;
                    for (uint32_t b = 0; b < N_BUCKETS; ++b)
                        if (ov[b]) {
                            bcaps[b] *= 2;
                            any = true;
                        }
                    if (!any) break;
                    if (attempt >= 3) throw KcError{KC_ERR_DEVICE, "counting table overflow"};
                }
                table_cap = std::max(table_cap, cap);
                // a single pass's records can go straight into the sort's buffers
                // when the sort (first digit skipped) runs an odd number of passes
                compact_table(tr, cap, pass_low, list, d_lr, n_low_items, merge_next, d_cfg, true,
                              !multi && sort_passes_run(2 * k, 8) % 2 == 1);
            }
            if (multi) {
                // this pass's records wait in pinned host memory; its device
                // memory goes to the next pass
                auto hr = std::make_unique<HostRecords>();
                hr->allocate(n_rec);
                if (n_rec) {
                    CK(cudaMemcpyAsync(hr->keys(), rec_keys, n_rec * 8, cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(hr->counts(), rec_counts, n_rec * 4, cudaMemcpyDeviceToHost, st));
                }
                CK(cudaStreamSynchronize(st));
                spilled_total += n_rec;
                spilled.push_back(std::move(hr));
                ds.rewind(mk);
            }
        }
        if (exact && filled_total != O)
            throw KcError{KC_ERR_DEVICE, "partition does not add up to the occurrences"};
        O = filled_total;
        job.occurrences = O;
        job.passes = (uint32_t)ranges.size();
        if (multi) {
            n_rec = spilled_total;
            rec_keys = ds.n<unsigned long long>(std::max<uint64_t>(n_rec, 1));
            rec_counts = ds.n<uint32_t>(std::max<uint64_t>(n_rec, 1));
            uint64_t at = 0;
            for (auto &hr : spilled) {
                if (hr->n) {
                    CK(cudaMemcpyAsync(rec_keys + at, hr->keys(), hr->n * 8, cudaMemcpyHostToDevice, st));
                    CK(cudaMemcpyAsync(rec_counts + at, hr->counts(), hr->n * 4, cudaMemcpyHostToDevice, st));
                }
                at += hr->n;
            }
            CK(cudaStreamSynchronize(st));
        }
    }
    job.table_cap = table_cap;
    check_cancel(job, "before the sort");

    // ---- sort in printed-string order ---------------------------------------
    clk.begin(6);
    bool reversed = false;   // keys back in the k-mer word layout
    if (n_rec > 1) {
        const uint32_t skip = rec_by_bucket && job.passes <= 1 ? 8u : 0u;
        void *stmp = rec_in_sort_tmp ? sort_tmp : ds.get(record_sort_bytes(n_rec, k));
        if (msd_sort_applies(n_rec, 2 * k) && tn.record_sort != 2) {
            // the sort writes the k-mer words back (pair_reverse) as it stores
            CK(launch_msd_sort(rec_keys, rec_counts, n_rec, 2 * k, stmp, st, counters + C_FLAGS, rec_in_sort_tmp,
                               true, rec_hist16));
            reversed = true;
        } else {
            CK(launch_radix_sort(rec_keys, rec_counts, n_rec, 2 * k, stmp, st, counters + C_FLAGS, skip,
                                 rec_in_sort_tmp));
        }
        if (!rec_in_sort_tmp) ds.release(stmp);
    }
    if (!reversed) CK(launch_pair_reverse(rec_keys, n_rec, st));
    clk.end();

    // ---- histogram (with the counters, under one sync) ----------------------
    unsigned long long *p_c2 = hs.n<unsigned long long>(C_COUNT);
    unsigned long long *p_hd = hs.n<unsigned long long>(HIST_BINS);
    CK(cudaMemcpyAsync(p_c2, counters, C_COUNT * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p_hd, hist, HIST_BINS * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    Counters c2{};
    std::memcpy(c2.v, p_c2, sizeof(c2.v));
    check_flags(c2.v[C_FLAGS], "sort");
    std::vector<unsigned long long> hd(p_hd, p_hd + HIST_BINS);
    const uint64_t n_ovf = std::min<uint64_t>(c2.v[C_OVF_LEN], ovf_cap);
    std::vector<uint32_t> ovf_h(n_ovf);
    if (n_ovf) {
        CK(cudaMemcpyAsync(ovf_h.data(), ovf, n_ovf * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    hd[1] += job.low_only;   // FIRST-only k-mers have count 1 (count_max >= 1)
    {
        uint32_t lo = P.hist_min, hi = P.hist_max;
        if (hi < lo) hi = lo;
        uint64_t len = (uint64_t)hi - lo + 1;
        job.hist.assign(len, 0);
        for (uint64_t c = std::max<uint64_t>(lo, 1); c < HIST_BINS && c <= hi; ++c) job.hist[c - lo] = (int64_t)hd[c];
        for (uint32_t c : ovf_h)
            if (c >= lo && c <= hi) job.hist[c - lo]++;
    }

    // ---- queries --------------------------------------------------------------
    if (P.top_n || P.want_le2) {
        clk.begin(7);
        uint32_t *flags = ds.n<uint32_t>(std::max<uint64_t>(n_rec, 1));
        unsigned long long *pos = ds.n<unsigned long long>(std::max<uint64_t>(n_rec, 1));
        unsigned long long *qtmp = ds.n<unsigned long long>(scan_tmp_words(std::max<uint64_t>(n_rec, 1)));
        if (P.top_n && n_rec) {
            // threshold from the histogram restricted to the record range
            auto count_at = [&](uint64_t c) -> uint64_t { return c < HIST_BINS ? hd[c] : 0; };
            std::vector<uint32_t> big;
            for (uint32_t c : ovf_h)
                if (c >= P.min_count && c <= P.max_count) big.push_back(c);
            std::sort(big.begin(), big.end(), std::greater<uint32_t>());
            uint64_t above = 0;
            uint32_t thr = std::max<uint32_t>(P.min_count, 1);
            bool found = false;
            for (size_t i = 0; i < big.size(); ++i) {
                if (above + 1 >= P.top_n) { thr = big[i]; found = true; break; }
                ++above;
            }
            if (!found) {
                uint64_t hi = std::min<uint64_t>((uint64_t)P.max_count, HIST_BINS - 1);
                for (uint64_t c = hi; c >= std::max<uint32_t>(P.min_count, 1); --c) {
                    uint64_t h = count_at(c);
                    if (above + h >= P.top_n) { thr = (uint32_t)c; found = true; break; }
                    above += h;
                    if (c == 0) break;
                }
            }
            // strictly above the threshold
            unsigned long long *ak = ds.n<unsigned long long>(P.top_n);
            uint32_t *ac = ds.n<uint32_t>(P.top_n);
            unsigned long long *bk = ds.n<unsigned long long>(P.top_n);
            uint32_t *bc = ds.n<uint32_t>(P.top_n);
            uint64_t n_above = 0, n_at = 0;
            if (thr < 0xffffffffu) {
                CK(launch_select_range(rec_keys, rec_counts, n_rec, thr + 1, 0xffffffffu, P.top_n, ak, ac, flags, pos,
                                       qtmp, counters, C_SEL_A, st));
            } else {
                CK(cudaMemsetAsync(&counters[C_SEL_A], 0, 8, st));
            }
            Counters ca = read_counters(counters, st);
            n_above = std::min<uint64_t>(ca.v[C_SEL_A], P.top_n);
            uint64_t need = P.top_n - n_above;
            if (need) {
                CK(launch_select_range(rec_keys, rec_counts, n_rec, thr, thr, need, bk, bc, flags, pos, qtmp, counters,
                                       C_SEL_B, st));
                Counters cb = read_counters(counters, st);
                n_at = std::min<uint64_t>(cb.v[C_SEL_B], need);
            }
            std::vector<uint64_t> tk(n_above), tk2(n_at);
            std::vector<uint32_t> tc(n_above), tc2(n_at);
            if (n_above) {
                CK(cudaMemcpyAsync(tk.data(), ak, n_above * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(tc.data(), ac, n_above * 4, cudaMemcpyDeviceToHost, st));
            }
            if (n_at) {
                CK(cudaMemcpyAsync(tk2.data(), bk, n_at * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(tc2.data(), bc, n_at * 4, cudaMemcpyDeviceToHost, st));
            }
            CK(cudaStreamSynchronize(st));
            // records above the threshold: count desc, then printed string asc
            // (they arrive in printed-string order; a stable sort keeps it)
            std::vector<size_t> idx(n_above);
            for (size_t i = 0; i < n_above; ++i) idx[i] = i;
            std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return tc[x] > tc[y]; });
            for (size_t i : idx) { job.top_keys.push_back(tk[i]); job.top_counts.push_back(tc[i]); }
            for (size_t i = 0; i < n_at; ++i) { job.top_keys.push_back(tk2[i]); job.top_counts.push_back(tc2[i]); }
        }
        if (P.want_le2 && n_rec) {
            unsigned long long *lk = ds.n<unsigned long long>(n_rec);
            uint32_t *lc = ds.n<uint32_t>(n_rec);
            CK(launch_select_range(rec_keys, rec_counts, n_rec, 0, 2, n_rec, lk, lc, flags, pos, qtmp, counters, C_SEL_A,
                                   st));
            Counters cl = read_counters(counters, st);
            uint64_t nl = std::min<uint64_t>(cl.v[C_SEL_A], n_rec);
            job.le2.allocate(nl);
            if (nl) {
                CK(cudaMemcpyAsync(job.le2.keys(), lk, nl * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(job.le2.counts(), lc, nl * 4, cudaMemcpyDeviceToHost, st));
            }
        }
        clk.end();
    }
    if (P.pack_high) pack_high_on_device(job, ds, rec_keys, rec_counts, n_rec, st, clk);
    CK(cudaEventRecord(ev1, st));

    // ---- records to host ------------------------------------------------------
    if (trace_host) fprintf(stderr, "[kc trace] records to host from %.3f ms (host clock)\n", now_ms() - th_start);
    if (P.keep_records) {
        job.recs.allocate(n_rec);
        if (n_rec) {
            CK(cudaMemcpyAsync(job.recs.keys(), rec_keys, n_rec * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(job.recs.counts(), rec_counts, n_rec * 4, cudaMemcpyDeviceToHost, st));
        }
    }
    CK(cudaStreamSynchronize(st));
    if (trace_host) fprintf(stderr, "[kc trace] job done at %.3f ms (host clock)\n", now_ms() - th_start);
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    job.device_ms = ms;
    clk.collect(job.phase_ms, job.phase_launches, ev0);
    job.low_len = low_len;
    job.high_len = high_len;
    job.input_bytes = in->total_bytes;
    job.n_records_total = n_rec;
}

// ---------------------------------------------------------------------------
// k-mers of 33..128 bases (the reference's process_main<2> / <4>,
// src/main.cpp:617-633)
// ---------------------------------------------------------------------------
//
// One job: upload -> newline census -> SCAN (occurrences, HyperLogLog,
// occurrences per root prefix) -> per pass over a range of root prefixes:
// INSERT into an N-word table sized from the estimate (regrown when full) ->
// compaction (count, then records + histogram) -> sort of all records in
// printed-string order -> queries -> host.  Jobs whose tables do not fit in
// one pass's memory run in passes, each pass's records held in pinned host
// memory until the final sort.  The Bloom split (kc_job.bloom) only chooses
// which occurrences the reference keeps in memory; the counts are exact
// either way, so these jobs count every occurrence in the table.
void run_wide_job(Job &job, cudaStream_t st, Workspace &ws, const kc_tuning &tn)
{
    const kc_job &P = job.p;
    const uint32_t k = P.k, nw = key_words(k);
    if (P.fault_inject & KC_INJECT_NOMEM) ws.fail_next_get();
    DevScope ds(st, &ws);
    std::vector<uint32_t> tile_seg_host;
    kc_input local;
    const kc_input *in = job.input;
    std::vector<PinnedBlock> inflated;
    if (!in) {
        const std::vector<kc_buffer> files = inflate_inputs(job.files, inflated);
        build_input(local, files.data(), (uint32_t)files.size(), st, &ds, tile_seg_host);
        in = &local;
    }
    HostStage hs(st);
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evg{ev0, ev1};
    CK(cudaEventRecord(ev0, st));
    PhaseClock clk(st);

    const uint64_t T = in->n_tiles;
    const uint32_t n_seg = (uint32_t)in->segs.size();
    std::vector<Seg> segs = in->segs;
    for (auto &sg : segs) {
        sg.k = k;
        sg.sample = 0;
        sg.sample_end = 0;
    }
    Seg *d_segs = ds.n<Seg>(std::max<uint32_t>(n_seg, 1));
    if (n_seg) CK(cudaMemcpyAsync(d_segs, hs.up(segs.data(), n_seg), n_seg * sizeof(Seg), cudaMemcpyHostToDevice, st));
    unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
    CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));

    // ---- line numbers of tile starts ---------------------------------------
    uint32_t *tile_nl = ds.n<uint32_t>(std::max<uint64_t>(T, 1));
    int32_t *tile_lastnl = ds.n<int32_t>(std::max<uint64_t>(T, 1));
    unsigned long long *tile_prefix = ds.n<unsigned long long>(std::max<uint64_t>(T, 1));
    unsigned long long *scan_tmp = ds.n<unsigned long long>(scan_tmp_words(std::max<uint64_t>(T, 1)));
    clk.begin(0);
    CK(launch_newlines(in->buf, T, tile_nl, tile_lastnl, st));
    CK(launch_scan_u32(tile_nl, tile_prefix, T, scan_tmp, st));
    clk.end();
    if (P.fault_inject & KC_INJECT_WAIT_TIMEOUT)
        CK(launch_wait_flag(reinterpret_cast<const unsigned int *>(counters + C_COUNT - 1), 1024, counters + C_FLAGS,
                            st));

    // ---- SCAN: occurrences, distinct estimate, root-prefix histogram ---------
    unsigned long long *scan_out = ds.n<unsigned long long>(1 + N_BUCKETS);   // occurrences, 256 bucket counts
    uint32_t *hll = ds.n<uint32_t>(HLL_M);
    CK(cudaMemsetAsync(scan_out, 0, (1 + N_BUCKETS) * 8, st));
    CK(cudaMemsetAsync(hll, 0, HLL_M * 4, st));
    WideArgs a{};
    a.buf = in->buf;
    a.n_tiles = T;
    a.tile_prefix = reinterpret_cast<const uint64_t *>(tile_prefix);
    a.tile_seg = in->d_tile_seg;
    a.segs = d_segs;
    a.counters = counters;
    a.occ = scan_out;
    a.bucket_hist = scan_out + 1;
    a.hll = hll;
    clk.begin(1);
    CK(launch_wide_extract(WMODE_SCAN, k, a, st));
    clk.end();
    unsigned long long *h_scan = hs.n<unsigned long long>(1 + N_BUCKETS);
    uint32_t *h_hll = hs.n<uint32_t>(HLL_M);
    CK(cudaMemcpyAsync(h_scan, scan_out, (1 + N_BUCKETS) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_hll, hll, HLL_M * 4, cudaMemcpyDeviceToHost, st));
    Counters c0 = read_counters(counters, st);
    check_flags(c0.v[C_FLAGS], "scan");
    const uint64_t O = h_scan[0];
    std::vector<uint64_t> bh(h_scan + 1, h_scan + 1 + N_BUCKETS);
    const double est = hll_estimate(h_hll, HLL_M);
    job.occurrences = O;
    check_cancel(job, "after the scan");

    // ---- passes over ranges of root prefixes ------------------------------------
    // a pass holds its table (slots per estimated distinct k-mer at the
    // handle's table factor) and its records (count pass, then the written
    // records); the final sort holds every record twice plus its temporaries
    const uint64_t slot_bytes = 8ull * nw + 8, rec_bytes = 8ull * nw + 4;
    const double factor = std::max(tn.table_factor, 1.25);
    const uint64_t budget = P.pass_bytes ? P.pass_bytes : default_pass_budget(ws);
    std::vector<std::pair<uint32_t, uint32_t>> ranges;
    {
        uint32_t lo = 0;
        uint64_t need = 0;
        for (uint32_t b = 0; b < N_BUCKETS; ++b) {
            const double share = O ? (double)bh[b] / (double)O : 0.0;
            const uint64_t nb = (uint64_t)(share * est * (factor * slot_bytes + rec_bytes)) + 4096;
            if (b > lo && need + nb > budget) {
                ranges.push_back({lo, b});
                lo = b;
                need = 0;
            }
            need += nb;
        }
        ranges.push_back({lo, N_BUCKETS});
    }
    const bool multi = ranges.size() > 1;
    unsigned long long *hist = ds.n<unsigned long long>(HIST_BINS);
    CK(cudaMemsetAsync(hist, 0, HIST_BINS * 8, st));
    const uint64_t ovf_cap = std::max<uint64_t>(1ull << 20, (uint64_t)(est / HIST_BINS) + 1);
    uint32_t *ovf = ds.n<uint32_t>(ovf_cap);
    std::vector<std::unique_ptr<HostRecords>> spilled;
    uint64_t n_rec = 0, inserted_total = 0, table_cap = 0;
    unsigned long long *rec_keys = nullptr;
    uint32_t *rec_counts = nullptr;
    bool injected_full = false;
    for (const auto &rg : ranges) {
        const DevScope::Mark mk = ds.mark();
        uint64_t occ_r = 0;
        for (uint32_t b = rg.first; b < rg.second; ++b) occ_r += bh[b];
        const double est_r = O ? est * (double)occ_r / (double)O : 0.0;
        uint64_t cap = table_capacity_for(est_r * 1.1, factor);
        WideTable tab{};
        for (int attempt = 0;; ++attempt) {
            check_cancel(job, "before a counting pass");
            tab.cap = cap;
            tab.keys = ds.n<unsigned long long>(cap * nw);
            tab.meta = ds.n<uint32_t>(cap * 2 + 2);
            CK(launch_wide_init(k, tab, st));
            CK(cudaMemsetAsync(counters + C_FLAGS, 0, 8, st));
            CK(cudaMemsetAsync(counters + C_HIGH_LEN, 0, 8, st));
            a.table = tab;
            a.max_probe = (uint32_t)std::min<uint64_t>(cap, 1u << 16);
            a.bucket_lo = rg.first;
            a.bucket_hi = rg.second == N_BUCKETS ? 0 : rg.second;
            clk.begin(2);
            CK(launch_wide_extract(WMODE_INSERT, k, a, st));
            clk.end();
            Counters ci = read_counters(counters, st);
            bool full = (ci.v[C_FLAGS] & ERR_TABLE_FULL) != 0;
            if ((P.fault_inject & KC_INJECT_TABLE_FULL) || ((P.fault_inject & KC_INJECT_TABLE_FULL_ONCE) && !injected_full)) {
                injected_full = true;
                full = true;
            }
            check_flags(ci.v[C_FLAGS] & ~ERR_TABLE_FULL, "insert");
            if (!full) {
                inserted_total += ci.v[C_HIGH_LEN];
                break;
            }
            if (attempt >= 3) throw KcError{KC_ERR_DEVICE, "counting table overflow"};
            ds.release(tab.meta);
            ds.release(tab.keys);
            cap *= 2;
        }
        table_cap = std::max(table_cap, cap);
        // compaction: the records kept, then the records and the histogram
        clk.begin(5);
        CK(cudaMemsetAsync(counters + C_KEPT, 0, 8, st));
        CK(launch_wide_compact(k, tab, P.count_max, P.min_count, P.max_count, nullptr, nullptr, 0, nullptr, nullptr, 0,
                               counters, 1, st));
        Counters ck = read_counters(counters, st);
        const uint64_t kept = ck.v[C_KEPT];
        const uint64_t rec0 = ck.v[C_REC_LEN];
        unsigned long long *rk = ds.n<unsigned long long>(std::max<uint64_t>(kept, 1) * nw);
        uint32_t *rc = ds.n<uint32_t>(std::max<uint64_t>(kept, 1));
        CK(cudaMemsetAsync(counters + C_REC_LEN, 0, 8, st));
        CK(launch_wide_compact(k, tab, P.count_max, P.min_count, P.max_count, rk, rc, kept, hist, ovf, ovf_cap, counters,
                               0, st));
        clk.end();
        (void)rec0;
        if (multi) {
            auto hr = std::make_unique<HostRecords>();
            hr->allocate(kept, nw);
            if (kept) {
                CK(cudaMemcpyAsync(hr->keys(), rk, kept * nw * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(hr->counts(), rc, kept * 4, cudaMemcpyDeviceToHost, st));
            }
            Counters cw = read_counters(counters, st);
            check_flags(cw.v[C_FLAGS], "compaction");
            n_rec += kept;
            spilled.push_back(std::move(hr));
            ds.rewind(mk);
        } else {
            n_rec = kept;
            rec_keys = rk;
            rec_counts = rc;
        }
    }
    if (inserted_total != O) throw KcError{KC_ERR_DEVICE, "counting passes do not add up to the occurrences"};
    job.passes = (uint32_t)ranges.size();
    job.table_cap = table_cap;
    job.high_len = inserted_total;
    if (multi) {
        rec_keys = ds.n<unsigned long long>(std::max<uint64_t>(n_rec, 1) * nw);
        rec_counts = ds.n<uint32_t>(std::max<uint64_t>(n_rec, 1));
        uint64_t at = 0;
        for (auto &hr : spilled) {
            if (hr->n) {
                CK(cudaMemcpyAsync(rec_keys + at * nw, hr->keys(), hr->n * nw * 8, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(rec_counts + at, hr->counts(), hr->n * 4, cudaMemcpyHostToDevice, st));
            }
            at += hr->n;
        }
        CK(cudaStreamSynchronize(st));
        spilled.clear();
    }
    check_cancel(job, "before the sort");

    // ---- sort in printed-string order -----------------------------------------
    clk.begin(6);
    unsigned long long *sk = ds.n<unsigned long long>(std::max<uint64_t>(n_rec, 1) * nw);
    uint32_t *sc = ds.n<uint32_t>(std::max<uint64_t>(n_rec, 1));
    {
        void *stmp = ds.get(wide_sort_tmp_bytes(n_rec));
        CK(launch_wide_sort(k, rec_keys, rec_counts, n_rec, sk, sc, stmp, counters + C_FLAGS, st));
        ds.release(stmp);
    }
    clk.end();

    // ---- histogram and counters ---------------------------------------------------
    unsigned long long *p_c2 = hs.n<unsigned long long>(C_COUNT);
    unsigned long long *p_hd = hs.n<unsigned long long>(HIST_BINS);
    CK(cudaMemcpyAsync(p_c2, counters, C_COUNT * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p_hd, hist, HIST_BINS * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    Counters c2{};
    std::memcpy(c2.v, p_c2, sizeof(c2.v));
    check_flags(c2.v[C_FLAGS], "sort");
    job.distinct = c2.v[C_DISTINCT];
    std::vector<unsigned long long> hd(p_hd, p_hd + HIST_BINS);
    const uint64_t n_ovf = std::min<uint64_t>(c2.v[C_OVF_LEN], ovf_cap);
    std::vector<uint32_t> ovf_h(n_ovf);
    if (n_ovf) {
        CK(cudaMemcpyAsync(ovf_h.data(), ovf, n_ovf * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    {
        uint32_t lo = P.hist_min, hi = P.hist_max;
        if (hi < lo) hi = lo;
        job.hist.assign((uint64_t)hi - lo + 1, 0);
        for (uint64_t c = std::max<uint64_t>(lo, 1); c < HIST_BINS && c <= hi; ++c) job.hist[c - lo] = (int64_t)hd[c];
        for (uint32_t c : ovf_h)
            if (c >= lo && c <= hi) job.hist[c - lo]++;
    }

    // ---- queries: record positions selected by count, their keys gathered --------
    if ((P.top_n || P.want_le2) && n_rec) {
        clk.begin(7);
        unsigned long long *idx = ds.n<unsigned long long>(n_rec);
        CK(launch_iota_u64(idx, n_rec, st));
        uint32_t *flags = ds.n<uint32_t>(n_rec);
        unsigned long long *pos = ds.n<unsigned long long>(n_rec);
        unsigned long long *qtmp = ds.n<unsigned long long>(scan_tmp_words(n_rec));
        auto select = [&](uint32_t lo, uint32_t hi, uint64_t limit, int ctr, std::vector<uint64_t> &keys_out,
                          std::vector<uint32_t> &counts_out) {
            unsigned long long *si = ds.n<unsigned long long>(std::max<uint64_t>(limit, 1));
            uint32_t *scn = ds.n<uint32_t>(std::max<uint64_t>(limit, 1));
            CK(cudaMemsetAsync(&counters[ctr], 0, 8, st));
            CK(launch_select_range(idx, sc, n_rec, lo, hi, limit, si, scn, flags, pos, qtmp, counters, ctr, st));
            Counters cs = read_counters(counters, st);
            const uint64_t m = std::min<uint64_t>(cs.v[ctr], limit);
            unsigned long long *rows = ds.n<unsigned long long>(std::max<uint64_t>(m, 1) * nw);
            CK(launch_wide_gather_rows(k, sk, si, m, rows, st));
            keys_out.resize(m * nw);
            counts_out.resize(m);
            if (m) {
                CK(cudaMemcpyAsync(keys_out.data(), rows, m * nw * 8, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(counts_out.data(), scn, m * 4, cudaMemcpyDeviceToHost, st));
            }
            CK(cudaStreamSynchronize(st));
        };
        if (P.top_n) {
            // the count threshold from the histogram: records above it, then
            // the first ones at it in printed-string order
            std::vector<uint32_t> big;
            for (uint32_t c : ovf_h)
                if (c >= P.min_count && c <= P.max_count) big.push_back(c);
            std::sort(big.begin(), big.end(), std::greater<uint32_t>());
            uint64_t above = 0;
            uint32_t thr = std::max<uint32_t>(P.min_count, 1);
            bool found = false;
            for (size_t i = 0; i < big.size(); ++i) {
                if (above + 1 >= P.top_n) { thr = big[i]; found = true; break; }
                ++above;
            }
            if (!found) {
                const uint64_t hi = std::min<uint64_t>((uint64_t)P.max_count, HIST_BINS - 1);
                for (uint64_t c = hi; c >= std::max<uint32_t>(P.min_count, 1); --c) {
                    const uint64_t h = hd[c];
                    if (above + h >= P.top_n) { thr = (uint32_t)c; break; }
                    above += h;
                    if (c == 0) break;
                }
            }
            std::vector<uint64_t> ka, kb;
            std::vector<uint32_t> ca, cb;
            if (thr < 0xffffffffu) select(thr + 1, 0xffffffffu, P.top_n, C_SEL_A, ka, ca);
            const uint64_t need = P.top_n - std::min<uint64_t>(ca.size(), P.top_n);
            if (need) select(thr, thr, need, C_SEL_B, kb, cb);
            // count desc, then printed string asc (a stable sort of records
            // already in printed-string order)
            std::vector<size_t> order(ca.size());
            for (size_t i = 0; i < order.size(); ++i) order[i] = i;
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return ca[x] > ca[y]; });
            for (size_t i : order) {
                job.top_keys.insert(job.top_keys.end(), ka.begin() + i * nw, ka.begin() + (i + 1) * nw);
                job.top_counts.push_back(ca[i]);
            }
            job.top_keys.insert(job.top_keys.end(), kb.begin(), kb.end());
            job.top_counts.insert(job.top_counts.end(), cb.begin(), cb.end());
        }
        if (P.want_le2) {
            std::vector<uint64_t> kl;
            std::vector<uint32_t> cl;
            select(0, 2, n_rec, C_SEL_A, kl, cl);
            job.le2.allocate(cl.size(), nw);
            if (!cl.empty()) {
                std::memcpy(job.le2.keys(), kl.data(), kl.size() * 8);
                std::memcpy(job.le2.counts(), cl.data(), cl.size() * 4);
            }
        }
        clk.end();
    }
    if (P.pack_high) pack_high_on_device(job, ds, sk, sc, n_rec, st, clk);
    CK(cudaEventRecord(ev1, st));

    // ---- records to host ----------------------------------------------------------
    if (P.keep_records) {
        job.recs.allocate(n_rec, nw);
        if (n_rec) {
            CK(cudaMemcpyAsync(job.recs.keys(), sk, n_rec * nw * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(job.recs.counts(), sc, n_rec * 4, cudaMemcpyDeviceToHost, st));
        }
    }
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    job.device_ms = ms;
    clk.collect(job.phase_ms, job.phase_launches, ev0);
    job.input_bytes = in->total_bytes;
    job.n_records_total = n_rec;
    job.key_words = nw;
}

void validate_job(const kc_job &p)
{
    if (p.k < 1 || p.k > 128) throw KcError{KC_ERR_INVALID, "k must be in 1..128"};
    if (!p.input && p.n_files && !p.files) throw KcError{KC_ERR_INVALID, "files is NULL"};
    if (p.count_max == 0) throw KcError{KC_ERR_INVALID, "count_max must be >= 1"};
    if (p.filter_max < p.filter_min) throw KcError{KC_ERR_INVALID, "filter_max < filter_min"};
    if (p.max_count < p.min_count) throw KcError{KC_ERR_INVALID, "max_count < min_count"};
    if (p.hist_max < p.hist_min) throw KcError{KC_ERR_INVALID, "hist_max < hist_min"};
    if ((uint64_t)p.hist_max - p.hist_min + 1 > (1ULL << 28)) throw KcError{KC_ERR_INVALID, "histogram range too large"};
    if (p.bloom && p.memory_gb == 0) throw KcError{KC_ERR_INVALID, "Bloom mode needs memory_gb >= 1"};
}

uint64_t input_bytes(const kc_job &p)
{
    if (p.input) return 0;
    uint64_t s = 0;
    for (uint32_t i = 0; i < p.n_files; ++i) s += gzip_size_hint(p.files[i]);
    return s;
}

uint64_t reserve_for(const kc_job &p, uint64_t resident_bytes)
{
    uint64_t s = p.input ? resident_bytes : input_bytes(p);
    // input + per-tile tables + table/records/sort sized for distinct <= s/2
    // (k-mers of more than 32 bases take 2 or 4 words)
    return (p.input ? 0 : s) + s / 256 + 24 * (uint64_t)key_words(p.k) * s + (64ULL << 20);
}

void run_job(Job &job, cudaStream_t st, Workspace &ws, const kc_tuning &tn)
{
    if (job.p.k > 32) {
        run_wide_job(job, st, ws, tn);
        return;
    }
    try {
        run_job_once(job, st, ws, false, tn);
    } catch (const CensusOverflow &) {
        // the sampled census missed a skewed bucket: count every tile instead
        CK(cudaStreamSynchronize(st));
        ws.end_job();
        ws.begin_job();
        run_job_once(job, st, ws, true, tn);
    }
}

// Batched jobs: every sample's files in one device buffer, one SCAN and one
// INSERT launch over all tiles (each tile counts into its sample's table in a
// shared slot arena), one batched compaction, one segmented radix sort.
void run_batch(std::vector<std::shared_ptr<Job>> &jobs, cudaStream_t st, Workspace &ws, const kc_tuning &tn)
{
    const uint32_t n = (uint32_t)jobs.size();
    if (n > MAX_BATCH) throw KcError{KC_ERR_INVALID, "more than 4096 jobs in one batch"};
    DevScope ds(st, &ws);
    std::vector<kc_buffer> files;
    std::vector<uint32_t> fsample;
    for (uint32_t i = 0; i < n; ++i)
        for (const auto &f : jobs[i]->files) {
            files.push_back(f);
            fsample.push_back(i);
        }
    kc_input in;
    std::vector<uint32_t> tile_seg_host;
    static const bool trace = getenv("KC_TRACE") && getenv("KC_TRACE")[0] == '1';
    const double th0 = now_ms();
    std::vector<PinnedBlock> inflated;   // gzip files inflated on the host (kept until the batch ends)
    files = inflate_inputs(files, inflated);
    build_input(in, files.data(), (uint32_t)files.size(), st, &ds, tile_seg_host, fsample.data());
    if (trace) fprintf(stderr, "[kc trace] batch upload of %u files enqueued in %.3f ms\n", (uint32_t)files.size(),
                       now_ms() - th0);
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evg{ev0, ev1};
    CK(cudaEventRecord(ev0, st));
    PhaseClock clk(st);

    const uint64_t T = in.n_tiles;
    std::vector<Seg> segs = in.segs;
    uint32_t max_k = 1;
    for (auto &sg : segs) {
        sg.k = jobs[sg.sample]->p.k;
        max_k = std::max(max_k, sg.k);
    }
    Seg *d_segs = ds.n<Seg>(std::max<size_t>(segs.size(), 1));
    if (!segs.empty()) CK(cudaMemcpyAsync(d_segs, segs.data(), segs.size() * sizeof(Seg), cudaMemcpyHostToDevice, st));
    unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
    CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));
    uint32_t *tile_nl = ds.n<uint32_t>(std::max<uint64_t>(T, 1));
    int32_t *tile_lastnl = ds.n<int32_t>(std::max<uint64_t>(T, 1));
    unsigned long long *tile_prefix = ds.n<unsigned long long>(std::max<uint64_t>(T, 1));
    unsigned long long *scan_tmp = ds.n<unsigned long long>(scan_tmp_words(std::max<uint64_t>(T, 1)));
    clk.begin(0);
    CK(launch_newlines(in.buf, T, tile_nl, tile_lastnl, st));
    CK(launch_scan_u32(tile_nl, tile_prefix, T, scan_tmp, st));
    clk.end();

    unsigned long long *occ = ds.n<unsigned long long>(n);
    uint32_t *hll = ds.n<uint32_t>((size_t)n * HLL_M);
    CK(cudaMemsetAsync(occ, 0, (size_t)n * 8, st));
    CK(cudaMemsetAsync(hll, 0, (size_t)n * HLL_M * 4, st));
    ExtractArgs a{};
    a.buf = in.buf;
    a.n_tiles = T;
    a.tile_prefix = reinterpret_cast<const uint64_t *>(tile_prefix);
    a.tile_seg = in.d_tile_seg;
    a.segs = d_segs;
    a.counters = counters;
    a.occ = occ;
    a.hll = hll;
    a.hll_local = n == 1;
    clk.begin(1);
    CK(launch_extract(MODE_SCAN, a, 0, st));
    clk.end();
    std::vector<unsigned long long> occ_h(n);
    std::vector<uint32_t> hll_h((size_t)n * HLL_M);
    CK(cudaMemcpyAsync(occ_h.data(), occ, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hll_h.data(), hll, (size_t)n * HLL_M * 4, cudaMemcpyDeviceToHost, st));
    Counters c0 = read_counters(counters, st);
    check_flags(c0.v[C_FLAGS], "scan");

    std::vector<uint64_t> caps(n);
    for (uint32_t i = 0; i < n; ++i) {
        // one sample: exact registers; several: a 1-in-64 hash sample
        double e = hll_estimate(&hll_h[(size_t)i * HLL_M], HLL_M);
        if (n > 1)
            e = std::max((double)(1u << BATCH_HLL_SAMPLE_BITS) * e, (double)std::min<unsigned long long>(occ_h[i], 4096));
        e = std::min(e, (double)occ_h[i]);
        caps[i] = table_capacity_for(e, tn.table_factor);
    }
    std::vector<SampleCfg> cfg(n);
    Slot *arena = nullptr;
    uint64_t total_slots = 0;
    SampleCfg *d_cfg = ds.n<SampleCfg>(n);
    TableRef *d_tables = ds.n<TableRef>(n);
    for (int attempt = 0;; ++attempt) {
        total_slots = 0;
        for (uint32_t i = 0; i < n; ++i) {
            cfg[i] = SampleCfg{};
            cfg[i].slot_base = total_slots;
            cfg[i].slot_cap = caps[i];
            cfg[i].count_max = jobs[i]->p.count_max;
            cfg[i].min_count = jobs[i]->p.min_count;
            cfg[i].max_count = jobs[i]->p.max_count;
            cfg[i].k = jobs[i]->p.k;
            total_slots += caps[i];
        }
        if (arena) ds.release(arena);
        arena = static_cast<Slot *>(ds.get(total_slots * sizeof(Slot)));
        CK(launch_init_slots(arena, total_slots, st));
        std::vector<TableRef> trs(n);
        for (uint32_t i = 0; i < n; ++i) trs[i] = TableRef{arena + cfg[i].slot_base, caps[i] - 1};
        CK(cudaMemcpyAsync(d_tables, trs.data(), n * sizeof(TableRef), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(counters, 0, 8, st));
        a.tables = d_tables;
        a.max_probe = 1u << 16;
        clk.begin(2);
        CK(launch_extract(MODE_INSERT, a, 0, st));
        clk.end();
        Counters c = read_counters(counters, st);
        check_flags(c.v[C_FLAGS], "insert");
        if (!(c.v[C_FLAGS] & ERR_TABLE_FULL)) break;
        if (attempt >= 3) throw KcError{KC_ERR_DEVICE, "counting table overflow"};
        for (auto &cp : caps) cp *= 2;
    }
    CK(cudaMemcpyAsync(d_cfg, cfg.data(), n * sizeof(SampleCfg), cudaMemcpyHostToDevice, st));
    // compaction in chunks of slots of one sample: count the records of every
    // chunk, scan the counts (the samples' records end up packed in sample
    // order), then write each chunk's records at its offset
    std::vector<uint32_t> chunk0(n + 1, 0);
    uint64_t n_chunks = 0;
    for (uint32_t i = 0; i < n; ++i) {
        chunk0[i] = (uint32_t)n_chunks;
        n_chunks += compact_chunks_of(cfg[i].slot_cap);
    }
    chunk0[n] = (uint32_t)n_chunks;
    uint32_t *d_chunk0 = ds.n<uint32_t>(n + 1);
    uint32_t *chunk_keep = ds.n<uint32_t>(std::max<uint64_t>(n_chunks, 1));
    unsigned long long *chunk_pos = ds.n<unsigned long long>(std::max<uint64_t>(n_chunks, 1));
    unsigned long long *ctmp = ds.n<unsigned long long>(scan_tmp_words(std::max<uint64_t>(n_chunks, 1)));
    unsigned long long *distinct = ds.n<unsigned long long>(n);
    CK(cudaMemcpyAsync(d_chunk0, chunk0.data(), (n + 1) * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(distinct, 0, (size_t)n * 8, st));
    clk.begin(5);
    CK(launch_compact_chunks(arena, d_cfg, d_chunk0, n, n_chunks, chunk_keep, nullptr, nullptr, nullptr, nullptr,
                             nullptr, 0, distinct, counters, 1, st));
    CK(launch_scan_u32(chunk_keep, chunk_pos, n_chunks, ctmp, st));
    clk.end();
    std::vector<unsigned long long> dist_h(n), pos_h(n_chunks);
    uint32_t last_keep = 0;
    CK(cudaMemcpyAsync(dist_h.data(), distinct, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    if (n_chunks) {
        CK(cudaMemcpyAsync(pos_h.data(), chunk_pos, n_chunks * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&last_keep, chunk_keep + n_chunks - 1, 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    const uint64_t total_rec = n_chunks ? pos_h[n_chunks - 1] + last_keep : 0;
    std::vector<unsigned long long> len_h(n);
    for (uint32_t i = 0; i < n; ++i) {
        cfg[i].rec_base = chunk0[i] < n_chunks ? pos_h[chunk0[i]] : total_rec;
        const uint64_t next = chunk0[i + 1] < n_chunks ? pos_h[chunk0[i + 1]] : total_rec;
        len_h[i] = next - cfg[i].rec_base;
        cfg[i].rec_cap = len_h[i];
    }
    unsigned long long *rec_keys = ds.n<unsigned long long>(std::max<uint64_t>(total_rec, 1));
    uint32_t *rec_counts = ds.n<uint32_t>(std::max<uint64_t>(total_rec, 1));
    unsigned long long *hist = ds.n<unsigned long long>((size_t)n * HIST_BINS_BATCH);
    uint64_t occ_total = 0;
    for (uint32_t i = 0; i < n; ++i) occ_total += occ_h[i];
    // counts of HIST_BINS_BATCH or more go to a list, bounded by the
    // occurrences over HIST_BINS_BATCH
    const uint64_t ovf_cap = std::max<uint64_t>(1ull << 20, occ_total / HIST_BINS_BATCH + 1);
    unsigned long long *ovf = ds.n<unsigned long long>(ovf_cap);
    CK(cudaMemsetAsync(hist, 0, (size_t)n * HIST_BINS_BATCH * 8, st));
    clk.begin(5);
    CK(launch_compact_chunks(arena, d_cfg, d_chunk0, n, n_chunks, chunk_keep, chunk_pos, rec_keys, rec_counts, hist,
                             ovf, ovf_cap, nullptr, counters, 0, st));
    clk.end();
    Counters c2 = read_counters(counters, st);
    check_flags(c2.v[C_FLAGS], "compact");

    std::vector<uint64_t> seg_start(n), seg_len(n);
    for (uint32_t i = 0; i < n; ++i) {
        seg_start[i] = cfg[i].rec_base;
        seg_len[i] = len_h[i];
    }
    clk.begin(6);
    if (total_rec > 1) {
        void *stmp = ds.get(sort_tmp_bytes_segmented(total_rec, seg_len.data(), n));
        std::vector<uint32_t> seg_bits(n);
        for (uint32_t i = 0; i < n; ++i) seg_bits[i] = 2 * cfg[i].k;
        CK(launch_radix_sort_segmented(rec_keys, rec_counts, total_rec, seg_start.data(), seg_len.data(), n, 2 * max_k,
                                       stmp, st, counters + C_FLAGS, seg_bits.data(), tn.sort_group_records));
        ds.release(stmp);
    }
    CK(launch_pair_reverse(rec_keys, total_rec, st));
    clk.end();
    CK(cudaEventRecord(ev1, st));
    check_flags(read_counters(counters, st).v[C_FLAGS], "sort");

    std::vector<unsigned long long> hist_h((size_t)n * HIST_BINS_BATCH);
    CK(cudaMemcpyAsync(hist_h.data(), hist, hist_h.size() * 8, cudaMemcpyDeviceToHost, st));
    const uint64_t n_ovf = std::min<uint64_t>(c2.v[C_OVF_LEN], ovf_cap);
    std::vector<unsigned long long> ovf_h(n_ovf);
    if (n_ovf) CK(cudaMemcpyAsync(ovf_h.data(), ovf, n_ovf * 8, cudaMemcpyDeviceToHost, st));
    for (uint32_t i = 0; i < n; ++i) {
        Job &j = *jobs[i];
        j.n_records_total = len_h[i];
        j.input_bytes = 0;
        for (size_t f = 0; f < files.size(); ++f)   // sizes after gzip inflation
            if (fsample[f] == i) j.input_bytes += files[f].size;
        if (!j.p.keep_records) continue;
        j.recs.allocate(len_h[i]);
        if (len_h[i]) {
            CK(cudaMemcpyAsync(j.recs.keys(), rec_keys + cfg[i].rec_base, len_h[i] * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(j.recs.counts(), rec_counts + cfg[i].rec_base, len_h[i] * 4, cudaMemcpyDeviceToHost,
                               st));
        }
    }
    const double th1 = now_ms();
    CK(cudaStreamSynchronize(st));
    if (trace) fprintf(stderr, "[kc trace] batch results to host: %.3f ms after the last enqueue\n", now_ms() - th1);
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    double phase_ms[KC_STAGES] = {0};
    uint64_t phase_launches[KC_STAGES] = {0};
    clk.collect(phase_ms, phase_launches, ev0);
    for (uint32_t i = 0; i < n; ++i) {
        Job &j = *jobs[i];
        j.device_ms = ms;
        for (int q = 0; q < KC_STAGES; ++q) {
            j.phase_ms[q] = phase_ms[q];
            j.phase_launches[q] = phase_launches[q];
        }
        j.occurrences = occ_h[i];
        j.distinct = dist_h[i];
        j.table_cap = caps[i];
        uint32_t lo = j.p.hist_min, hi = std::max(j.p.hist_max, j.p.hist_min);
        j.hist.assign((uint64_t)hi - lo + 1, 0);
        for (uint64_t c = std::max<uint64_t>(lo, 1); c < HIST_BINS_BATCH && c <= hi; ++c)
            j.hist[c - lo] = (int64_t)hist_h[(size_t)i * HIST_BINS_BATCH + c];
    }
    for (unsigned long long e : ovf_h) {
        uint32_t smp = (uint32_t)(e >> 32), c = (uint32_t)e;
        Job &j = *jobs[smp];
        if (c >= j.p.hist_min && c <= j.p.hist_max) j.hist[c - j.p.hist_min]++;
    }
}

void worker_main(kc_handle *h)
{
    cudaSetDevice(h->device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    auto ws = std::make_unique<Workspace>(st);
    // several workers: each keeps at most its share of the budget between
    // jobs, so that one large job does not leave its memory idle in one
    // worker while the others need it
    if (h->workers_n > 1 && !h->workspace_bytes) ws->set_max_keep(h->budget / h->workers_n);
    if (h->workspace_bytes) ws->reserve(h->workspace_bytes);
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->spaces.push_back(ws.get());
    }
    const uint64_t share = h->workers_n > 1 ? h->budget / h->workers_n : UINT64_MAX;
    for (;;) {
        std::shared_ptr<Task> task;
        bool alone = false;
        {
            std::unique_lock<std::mutex> lk(h->mu);
            h->cv_work.wait(lk, [&] {
                if (h->closing) return true;
                if (h->queue.empty() || h->exclusive) return false;
                const auto &f = h->queue.front();
                if (f->reserve > share) return h->running == 0;
                return h->running == 0 || h->reserved + f->reserve <= h->budget;
            });
            if (h->closing) break;
            task = h->queue.front();
            h->queue.pop_front();
            alone = task->reserve > share;
            if (alone) {
                // the other workers are idle (nothing runs): their kept
                // blocks go back to the device for this job's passes
                h->exclusive = true;
                for (Workspace *o : h->spaces)
                    if (o != ws.get()) o->trim();
            }
            h->reserved += task->reserve;
            h->running++;
            task->tuning = h->tuning;
            for (auto &j : task->jobs) {
                j->state = JobState::RUNNING;
                j->t_start = now_ms();
            }
        }
        int code = KC_OK;
        std::string msg;
        try {
            ws->begin_job();
            if (task->batch) run_batch(task->jobs, st, *ws, task->tuning);
            else run_job(*task->jobs[0], st, *ws, task->tuning);
        } catch (const KcError &e) {
            code = e.code;
            msg = e.msg;
        } catch (const std::exception &e) {
            code = KC_ERR_FAILED;
            msg = e.what();
        }
        if (code != KC_OK) cudaStreamSynchronize(st);
        ws->end_job();
        {
            std::lock_guard<std::mutex> lk(h->mu);
            for (auto &j : task->jobs) {
                j->t_end = now_ms();
                int c = code;
                std::string m = msg;
                if (c == KC_OK && j->cancel.load(std::memory_order_relaxed)) {
                    c = KC_ERR_CANCELLED;   // a cancelled sample of a batch that ran on for the others
                    m = "cancelled";
                }
                j->state = c == KC_OK ? JobState::DONE : JobState::FAILED;
                j->err = c;
                j->err_msg = m;
            }
            h->reserved -= task->reserve;
            h->running--;
            if (alone) h->exclusive = false;
        }
        h->cv_work.notify_all();
        h->cv_done.notify_all();
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->spaces.erase(std::find(h->spaces.begin(), h->spaces.end(), ws.get()));
    }
    ws.reset();
    cudaStreamDestroy(st);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

uint64_t kc_kernel_launches(void) { return kernel_launches(); }

uint32_t kc_key_words(uint32_t k) { return (k >= 1 && k <= 128) ? key_words(k) : 0u; }

void kc_job_defaults(kc_job *job)
{
    if (!job) return;
    std::memset(job, 0, sizeof(*job));
    job->k = 31;
    job->count_max = 255;
    job->memory_gb = 4;
    job->filter_min = 2;
    job->filter_max = 0xffffffffu;
    job->min_count = 1;
    job->max_count = 0xffffffffu;
    job->hist_min = 1;
    job->hist_max = 10000;
    job->keep_records = 1;
}

int kc_open(const kc_config *cfg, kc_handle **out)
{
    if (!out) return fail(KC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(KC_ERR_NO_DEVICE, "no CUDA device");
    }
    int dev = cfg ? cfg->device : 0;
    if (dev < 0 || dev >= ndev) return fail(KC_ERR_INVALID, "device ordinal out of range");
    if (cudaSetDevice(dev) != cudaSuccess) return fail(KC_ERR_CUDA, "cudaSetDevice failed");
    // keep freed stream-ordered memory in the pool for the next job
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    auto *h = new kc_handle();
    h->device = dev;
    h->budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (uint64_t)(free_b * 0.9);
    h->workspace_bytes = cfg ? cfg->workspace_bytes : 0;
    if (cfg && cfg->pinned_bytes) {
        try {
            PinnedPool::instance().add_arena(cfg->pinned_bytes);
        } catch (const KcError &e) {
            delete h;
            return fail(e.code, e.msg);
        }
    }
    uint32_t nw = (cfg && cfg->max_inflight_jobs) ? cfg->max_inflight_jobs : 4;
    h->workers_n = nw;
    for (uint32_t i = 0; i < nw; ++i) h->workers.emplace_back(worker_main, h);
    *out = h;
    return KC_OK;
}

void kc_close(kc_handle *h)
{
    if (!h) return;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->closing = true;
        for (auto &t : h->queue)
            for (auto &j : t->jobs) {
                j->state = JobState::FAILED;
                j->err = KC_ERR_FAILED;
                j->err_msg = "handle closed before the job started";
            }
        h->queue.clear();
    }
    h->cv_work.notify_all();
    h->cv_done.notify_all();
    for (auto &w : h->workers) w.join();
    delete h;
}

int kc_input_upload(kc_handle *h, const kc_buffer *files, uint32_t n_files, kc_input **out)
{
    if (!h || !out || (n_files && !files)) return fail(KC_ERR_INVALID, "bad argument");
    try {
        cudaSetDevice(h->device);
        auto *in = new kc_input();
        std::vector<uint32_t> ts;
        cudaStream_t st;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        try {
            std::vector<PinnedBlock> inflated;
            const std::vector<kc_buffer> fv = inflate_inputs(std::vector<kc_buffer>(files, files + n_files), inflated);
            build_input(*in, fv.data(), (uint32_t)fv.size(), st, nullptr, ts);
            CK(cudaStreamSynchronize(st));
        } catch (...) {
            cudaStreamDestroy(st);
            if (in->base) cudaFree(in->base);
            if (in->d_tile_seg) cudaFree(in->d_tile_seg);
            delete in;
            throw;
        }
        cudaStreamDestroy(st);
        *out = in;
        return KC_OK;
    } catch (const KcError &e) {
        return fail(e.code, e.msg);
    }
}

void kc_input_free(kc_handle *h, kc_input *in)
{
    if (!in) return;
    if (h) cudaSetDevice(h->device);
    if (!in->stream_owned) {
        cudaFree(in->base);
        cudaFree(in->d_tile_seg);
    }
    delete in;
}

static int submit_task(kc_handle *h, const kc_job *jobs, uint32_t n, kc_job_id *ids, bool batch)
{
    if (!h || !jobs || !ids || n == 0) return fail(KC_ERR_INVALID, "bad argument");
    // a batch larger than a worker's share of the device-memory budget runs
    // as consecutive sub-batches (each one set of device passes), so that its
    // samples stream through the device while earlier ones are counted
    std::vector<std::shared_ptr<Task>> tasks(1, std::make_shared<Task>());
    tasks[0]->batch = batch;
    const uint64_t group_budget =
        batch ? std::max<uint64_t>(h->budget / std::max<size_t>(h->workers.size(), 1), 1) : UINT64_MAX;
    try {
        for (uint32_t i = 0; i < n; ++i) {
            validate_job(jobs[i]);
            if (batch && jobs[i].bloom) throw KcError{KC_ERR_INVALID, "Bloom mode is not available for batched jobs"};
            if (batch && jobs[i].k > 32)
                throw KcError{KC_ERR_INVALID, "k-mers of more than 32 bases are not available for batched jobs"};
            if (batch && (jobs[i].top_n || jobs[i].want_le2))
                throw KcError{KC_ERR_INVALID, "count queries are not available for batched jobs"};
            if (batch && jobs[i].input) throw KcError{KC_ERR_INVALID, "batched jobs take host files"};
            auto j = std::make_shared<Job>();
            j->p = jobs[i];
            if (!jobs[i].input) j->files.assign(jobs[i].files, jobs[i].files + jobs[i].n_files);
            j->p.files = nullptr;
            j->input = jobs[i].input;
            j->reserve = reserve_for(jobs[i], jobs[i].input ? jobs[i].input->total_bytes : 0);
            if (!tasks.back()->jobs.empty() && tasks.back()->reserve + j->reserve > group_budget) {
                tasks.push_back(std::make_shared<Task>());
                tasks.back()->batch = batch;
            }
            j->batch_part = (uint32_t)(tasks.size() - 1);
            tasks.back()->reserve += j->reserve;
            tasks.back()->jobs.push_back(j);
        }
    } catch (const KcError &e) {
        return fail(e.code, e.msg);
    }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        if (h->closing) return fail(KC_ERR_INVALID, "handle is closing");
        double t = now_ms();
        uint32_t i = 0;
        for (auto &task : tasks) {
            for (auto &j : task->jobs) {
                j->id = h->next_id++;
                j->t_submit = t;
                h->jobs[j->id] = j;
                ids[i++] = j->id;
            }
            h->queue.push_back(task);
        }
    }
    h->cv_work.notify_all();
    return KC_OK;
}

int kc_submit(kc_handle *h, const kc_job *job, kc_job_id *id) { return submit_task(h, job, 1, id, false); }

int kc_get_tuning(kc_handle *h, kc_tuning *out)
{
    if (!h || !out) return fail(KC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(h->mu);
    *out = h->tuning;
    return KC_OK;
}

int kc_set_tuning(kc_handle *h, const kc_tuning *t)
{
    if (!h || !t) return fail(KC_ERR_INVALID, "bad argument");
    if (t->bucket_table_factor > 0 && t->bucket_table_factor < 1.05)
        return fail(KC_ERR_INVALID, "bucket_table_factor must be at least 1.05");
    if (t->table_factor > 0 && t->table_factor < 1.05) return fail(KC_ERR_INVALID, "table_factor must be at least 1.05");
    if (t->bloom_smem > 2) return fail(KC_ERR_INVALID, "bloom_smem must be 1 or 2");
    if (t->record_sort > 2) return fail(KC_ERR_INVALID, "record_sort must be 1 or 2");
    if (t->count_shape > 4) return fail(KC_ERR_INVALID, "count_shape must be 1..4");
    if (t->part_shape > 2) return fail(KC_ERR_INVALID, "part_shape must be 1 or 2");
    if (t->scatter_shape > 2) return fail(KC_ERR_INVALID, "scatter_shape must be 1 or 2");
    std::lock_guard<std::mutex> lk(h->mu);
    if (t->bucket_table_factor > 0) h->tuning.bucket_table_factor = t->bucket_table_factor;
    if (t->table_factor > 0) h->tuning.table_factor = t->table_factor;
    if (t->sort_group_records > 0) h->tuning.sort_group_records = t->sort_group_records;
    if (t->bloom_smem > 0) h->tuning.bloom_smem = t->bloom_smem;
    if (t->record_sort > 0) h->tuning.record_sort = t->record_sort;
    if (t->sampled_region_keys > 0) h->tuning.sampled_region_keys = t->sampled_region_keys;
    if (t->count_shape > 0) h->tuning.count_shape = t->count_shape;
    if (t->part_shape > 0) h->tuning.part_shape = t->part_shape;
    if (t->scatter_shape > 0) h->tuning.scatter_shape = t->scatter_shape;
    return KC_OK;
}

int kc_autotune(kc_handle *h, const kc_job *jobs, uint32_t n_jobs, uint32_t batch, kc_tuning *best)
{
    if (!h || !jobs || !n_jobs) return fail(KC_ERR_INVALID, "bad argument");
    // device time of one run of the jobs with settings t (a batch reports
    // the same device time for all of its samples)
    auto run = [&](const kc_tuning &t, double &ms) -> int {
        {
            std::lock_guard<std::mutex> lk(h->mu);
            h->tuning = t;
        }
        std::vector<kc_job_id> ids(n_jobs);
        int rc = batch ? kc_submit_batch(h, jobs, n_jobs, ids.data()) : KC_OK;
        if (!batch)
            for (uint32_t i = 0; i < n_jobs && rc == KC_OK; ++i) rc = kc_submit(h, &jobs[i], &ids[i]);
        ms = 0;
        int64_t last_part = -1;   // a batch's sub-batches each report their device time once
        for (uint32_t i = 0; i < n_jobs; ++i) {
            if (!ids[i]) continue;
            const int w = kc_wait(h, ids[i], -1);
            if (w == KC_OK) {
                kc_result_t r;
                if (kc_result(h, ids[i], &r) == KC_OK && (!batch || (int64_t)r.batch_part != last_part)) {
                    ms += r.device_ms;
                    last_part = r.batch_part;
                }
            } else if (rc == KC_OK) {
                rc = w;
            }
            kc_release(h, ids[i]);
        }
        return rc;
    };
    kc_tuning cur;
    kc_get_tuning(h, &cur);
    double cur_ms = 0, ms = 0;
    int rc = run(cur, cur_ms);   // warm-up: workspaces and pinned blocks reach this shape
    if (rc == KC_OK) rc = run(cur, cur_ms);
    const double bucket_c[] = {2.0, 3.0, 4.0, 3.0}, table_c[] = {1.3, 1.6, 2.2, 1.6};
    const uint64_t group_c[] = {2ull << 20, 4ull << 20, 8ull << 20, 4ull << 20}, smem_c[] = {1, 2, 1, 1},
                   sort_c[] = {1, 2, 1, 1}, shape_c[] = {1, 2, 3, 4}, part_c[] = {1, 2, 1, 1},
                   scatter_c[] = {1, 2, 1, 1};
    for (int param = 0; param < 8 && rc == KC_OK; ++param)
        for (int c = 0; c < 4 && rc == KC_OK; ++c) {
            kc_tuning t = cur;
            if (param == 0) t.bucket_table_factor = bucket_c[c];
            if (param == 1) t.table_factor = table_c[c];
            if (param == 2) t.sort_group_records = group_c[c];
            if (param == 3) t.bloom_smem = smem_c[c];
            if (param == 4) t.record_sort = sort_c[c];
            if (param == 5) t.count_shape = shape_c[c];
            if (param == 6) t.part_shape = part_c[c];
            if (param == 7) t.scatter_shape = scatter_c[c];
            if (std::memcmp(&t, &cur, sizeof(t)) == 0) continue;
            rc = run(t, ms);
            if (rc == KC_OK && ms < 0.98 * cur_ms) {   // a clear gain only
                cur = t;
                cur_ms = ms;
            }
        }
    {
        std::lock_guard<std::mutex> lk(h->mu);
        h->tuning = cur;
    }
    if (best) *best = cur;
    return rc;
}

int kc_submit_batch(kc_handle *h, const kc_job *jobs, uint32_t n_jobs, kc_job_id *ids)
{
    return submit_task(h, jobs, n_jobs, ids, true);
}

int kc_wait(kc_handle *h, kc_job_id id, int32_t timeout_ms)
{
    if (!h) return fail(KC_ERR_INVALID, "handle is NULL");
    std::unique_lock<std::mutex> lk(h->mu);
    auto it = h->jobs.find(id);
    if (it == h->jobs.end()) return fail(KC_ERR_NOT_FOUND, "unknown job id");
    auto j = it->second;
    auto done = [&] { return j->state == JobState::DONE || j->state == JobState::FAILED; };
    if (timeout_ms < 0) h->cv_done.wait(lk, done);
    else if (!h->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return fail(KC_ERR_TIMEOUT, "job still running");
    if (j->state == JobState::FAILED) return fail(j->err ? j->err : KC_ERR_FAILED, j->err_msg);
    return KC_OK;
}

int kc_result(kc_handle *h, kc_job_id id, kc_result_t *out)
{
    if (!h || !out) return fail(KC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(h->mu);
    auto it = h->jobs.find(id);
    if (it == h->jobs.end()) return fail(KC_ERR_NOT_FOUND, "unknown job id");
    Job &j = *it->second;
    if (j.state != JobState::DONE) return fail(j.state == JobState::FAILED ? j.err : KC_ERR_INVALID, "job not finished");
    std::memset(out, 0, sizeof(*out));
    out->n_records = j.recs.n;
    out->keys = j.recs.n ? j.recs.keys() : nullptr;
    out->counts = j.recs.n ? j.recs.counts() : nullptr;
    out->hist_len = j.hist.size();
    out->hist = j.hist.data();
    out->n_top = j.top_counts.size();   // top_keys holds key_words words per record
    out->top_keys = j.top_keys.data();
    out->top_counts = j.top_counts.data();
    out->n_le2 = j.le2.n;
    out->le2_keys = j.le2.n ? j.le2.keys() : nullptr;
    out->le2_counts = j.le2.n ? j.le2.counts() : nullptr;
    out->occurrences = j.occurrences;
    out->distinct = j.distinct;
    out->low_only = j.low_only;
    out->table_capacity = j.table_cap;
    out->device_ms = j.device_ms;
    out->queue_ms = j.t_start - j.t_submit;
    out->run_ms = j.t_end - j.t_start;
    for (int i = 0; i < KC_STAGES; ++i) {
        out->phase_ms[i] = j.phase_ms[i];
        out->phase_launches[i] = j.phase_launches[i];
    }
    out->low_len = j.low_len;
    out->high_len = j.high_len;
    out->input_bytes = j.input_bytes;
    out->n_records_total = j.n_records_total;
    out->passes = j.passes;
    out->smem_passes = (uint16_t)std::min<uint32_t>(j.smem_passes, 0xFFFF);
    out->smem_fallbacks = (uint16_t)std::min<uint32_t>(j.smem_fallbacks, 0xFFFF);
    out->region_redos = j.region_redos;
    out->batch_part = j.batch_part;
    out->key_words = j.key_words;
    return KC_OK;
}

int kc_cancel(kc_handle *h, kc_job_id id)
{
    if (!h) return fail(KC_ERR_INVALID, "handle is NULL");
    {
        std::lock_guard<std::mutex> lk(h->mu);
        auto it = h->jobs.find(id);
        if (it == h->jobs.end()) return fail(KC_ERR_NOT_FOUND, "unknown job id");
        Job &j = *it->second;
        if (j.state == JobState::DONE || j.state == JobState::FAILED)
            return fail(KC_ERR_INVALID, "job already finished");
        j.cancel.store(true, std::memory_order_relaxed);
        if (j.state == JobState::QUEUED) {
            // a queued task leaves the queue once every job in it is cancelled
            for (auto q = h->queue.begin(); q != h->queue.end(); ++q) {
                auto &jobs = (*q)->jobs;
                if (std::find_if(jobs.begin(), jobs.end(), [&](const std::shared_ptr<Job> &x) { return x->id == id; }) ==
                    jobs.end())
                    continue;
                const bool all = std::all_of(jobs.begin(), jobs.end(), [](const std::shared_ptr<Job> &x) {
                    return x->cancel.load(std::memory_order_relaxed);
                });
                if (all) {
                    const double t = now_ms();
                    for (auto &x : jobs) {
                        x->state = JobState::FAILED;
                        x->err = KC_ERR_CANCELLED;
                        x->err_msg = "cancelled before it started";
                        x->t_start = x->t_end = t;
                    }
                    h->queue.erase(q);
                }
                break;
            }
        }
    }
    h->cv_work.notify_all();
    h->cv_done.notify_all();
    return KC_OK;
}

int kc_release(kc_handle *h, kc_job_id id)
{
    if (!h) return fail(KC_ERR_INVALID, "handle is NULL");
    std::lock_guard<std::mutex> lk(h->mu);
    auto it = h->jobs.find(id);
    if (it == h->jobs.end()) return fail(KC_ERR_NOT_FOUND, "unknown job id");
    if (it->second->state == JobState::QUEUED || it->second->state == JobState::RUNNING)
        return fail(KC_ERR_INVALID, "job still running");
    h->jobs.erase(it);
    return KC_OK;
}

int kc_host_alloc(uint64_t bytes, void **p)
{
    if (!p) return fail(KC_ERR_INVALID, "p is NULL");
    cudaError_t e = cudaHostAlloc(p, bytes ? bytes : 1, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(KC_ERR_NOMEM, cudaGetErrorString(e));
    }
    return KC_OK;
}

int kc_host_free(void *p)
{
    if (p) cudaFreeHost(p);
    return KC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// reference tmp_dir files
// ---------------------------------------------------------------------------

namespace {

bool write_all(FILE *f, const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }

}  // namespace

extern "C" int kc_write_tmpdir(kc_handle *h, kc_job_id id, const char *dir)
{
    if (!h || !dir) return fail(KC_ERR_INVALID, "bad argument");
    std::shared_ptr<Job> jp;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        auto it = h->jobs.find(id);
        if (it == h->jobs.end()) return fail(KC_ERR_NOT_FOUND, "unknown job id");
        jp = it->second;
        if (jp->state != JobState::DONE) return fail(KC_ERR_INVALID, "job not finished");
    }
    const Job &j = *jp;
    if (!j.p.keep_records && !j.has_packed)
        return fail(KC_ERR_INVALID, "job was run without keep_records or pack_high");
    std::string d(dir);
    if (!d.empty() && d.back() != '/') d += '/';
    // infos.bin: u32 k, u32 count_max (src/main.cpp:590-597)
    FILE *f = fopen((d + "infos.bin").c_str(), "wb");
    if (!f) return fail(KC_ERR_IO, "cannot open " + d + "infos.bin");
    uint32_t info[2] = {j.p.k, j.p.count_max};
    bool ok = write_all(f, info, sizeof(info));
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(KC_ERR_IO, "write failed: infos.bin");
    // high.bin: exact counts, record = the full words (k / 32 of them), the
    // tail bytes of the masked next word, the count bytes
    // (src/FinalDrainWriter.h:71-88); the counter-side filter
    // (src/FinalDrainWriter.h:101) is applied to the exact count
    const uint32_t k = j.p.k, nw = j.recs.words;
    const uint32_t tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8, full = k / 32;
    const uint64_t tmask = tail_bits ? (~0ULL << (64 - tail_bits)) : 0;
    const uint32_t cb = j.p.count_max <= 0xFF ? 1 : j.p.count_max <= 0xFFFF ? 2 : j.p.count_max <= 0xFFFFFF ? 3 : 4;
    const uint32_t rec = full * 8 + tail_bytes + cb;
    f = fopen((d + "high.bin").c_str(), "wb");
    if (!f) return fail(KC_ERR_IO, "cannot open " + d + "high.bin");
    if (j.has_packed) {
        // packed on the device (kc_job.pack_high)
        ok = write_all(f, j.packed.p, j.packed_bytes);
        ok = (fclose(f) == 0) && ok;
        if (!ok) return fail(KC_ERR_IO, "write failed: high.bin");
        f = fopen((d + "low.bin").c_str(), "wb");
        if (!f) return fail(KC_ERR_IO, "cannot open " + d + "low.bin");
        if (fclose(f) != 0) return fail(KC_ERR_IO, "write failed: low.bin");
        return KC_OK;
    }
    std::vector<uint8_t> buf;
    buf.reserve(std::min<size_t>(j.recs.n, 1 << 20) * rec);
    for (size_t i = 0; i < j.recs.n; ++i) {
        uint32_t c = j.recs.counts()[i];
        if ((uint64_t)c + 1 < j.p.filter_min || c > j.p.filter_max) continue;
        uint8_t r[48];
        const uint64_t *w = j.recs.keys() + i * nw;
        std::memcpy(r, w, full * 8);
        if (tail_bytes) {
            const uint64_t t = w[full] & tmask;
            std::memcpy(r + full * 8, reinterpret_cast<const uint8_t *>(&t) + (8 - tail_bytes), tail_bytes);
        }
        std::memcpy(r + full * 8 + tail_bytes, &c, cb);
        buf.insert(buf.end(), r, r + rec);
        if (buf.size() >= (64u << 20)) {
            if (!write_all(f, buf.data(), buf.size())) { fclose(f); return fail(KC_ERR_IO, "write failed: high.bin"); }
            buf.clear();
        }
    }
    ok = write_all(f, buf.data(), buf.size());
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(KC_ERR_IO, "write failed: high.bin");
    // low.bin: every k-mer's occurrences are already merged into high.bin
    f = fopen((d + "low.bin").c_str(), "wb");
    if (!f) return fail(KC_ERR_IO, "cannot open " + d + "low.bin");
    if (fclose(f) != 0) return fail(KC_ERR_IO, "write failed: low.bin");
    return KC_OK;
}

