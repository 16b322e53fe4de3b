/*
 * kc.h -- C ABI of the B200 k-mer counter (libkc.so).
 *
 * The reference (ScorchShana/KTCounterMemoryGreedy) has no library API: its
 * boundary is three programs and the files they exchange.  These entry points
 * are what a binding to its counting path needs, one per step of that path:
 *
 *   kc_open / kc_close     replace process start-up and the global state of
 *                          src/main.cpp:481-633 (argv parsing, thread split,
 *                          memory pool of memory_limit GB)
 *   kc_submit / kc_wait    replace process_main<N> (src/main.cpp:246-478):
 *                          FASTQ in -> exact canonical counts
 *   kc_result              the precise outputs of tool/histogram_tool.cpp
 *                          (run_precise_histogram_tool_impl :735) and
 *                          tool/dump_tool.cpp (run_precise_impl :1202,
 *                          --sort), as memory instead of text files
 *   kc_write_tmpdir        the tmp_dir files infos.bin / high.bin / low.bin
 *                          (src/main.cpp:590-597, src/FinalDrainWriter.h:71-146,
 *                          src/ExportWriter.h:296-313) that the unmodified
 *                          reference tools read
 *
 * Conventions: every call returns a status code (KC_OK = 0) and never exits
 * the process; kc_last_error() describes the last failure of the calling
 * thread.  Inputs are caller-owned and only read.  Result memory is owned by
 * the job and stays valid until kc_release() or kc_close().  A handle may be
 * used from several host threads; jobs submitted to one handle run
 * concurrently on the device (one CUDA stream each), admitted in submission
 * order as device memory frees up.
 *
 * k-mer words: a k-mer is the reference's kmer<N> word array (src/kmer.h:15),
 * N = kc_key_words(k): 1 for k <= 32, 2 for k <= 64, 4 for k <= 128 (the
 * dispatch of src/main.cpp:617-633).  For k <= 32, base i of the printed
 * canonical string sits at bit 64 - 2k + 2i of the one word, padding bits
 * are zero.  For k > 32 the newest base sits at data[0]'s top bits and older
 * bases follow towards data[last] (last = (k - 1) / 32), whose low
 * 64 - 2 * (k % 32) bits are zero; words above data[last] are zero.  Key
 * arrays hold N consecutive words per k-mer, data[0] first.  Record arrays
 * are sorted in printed-string order (the order of dump_tool --sort).
 */
#ifndef KC_H
#define KC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KC_OK 0
#define KC_ERR_INVALID 1     /* bad argument */
#define KC_ERR_CUDA 2        /* CUDA runtime failure */
#define KC_ERR_NOMEM 3       /* device or pinned host allocation failed */
#define KC_ERR_TIMEOUT 4     /* kc_wait ran out of time; the job keeps running */
#define KC_ERR_NOT_FOUND 5   /* unknown job id */
#define KC_ERR_DEVICE 6      /* a kernel reported an error flag */
#define KC_ERR_IO 7          /* file write failed */
#define KC_ERR_NO_DEVICE 8   /* no usable CUDA device */
#define KC_ERR_FAILED 9      /* the job failed; kc_last_error after kc_wait says why */
#define KC_ERR_CANCELLED 10  /* the job was cancelled (kc_cancel) before it finished */

/* kc_job.fault_inject: failures a test can force on a job (no counterpart in
 * the reference, whose failures end the process, e.g. src/FastqReader.h:195;
 * its one give-up path is the bounded wait of
 * src/NewKmerTree.h:1225-1254).  Each one goes through the path a real
 * failure of that kind takes. */
#define KC_INJECT_WAIT_TIMEOUT 1u    /* a device wait on a flag nothing sets gives up after a short poll
                                        limit and sets the wait-timeout flag: the job ends KC_ERR_DEVICE */
#define KC_INJECT_TABLE_FULL_ONCE 2u /* the first counting attempt reports its table full (plain jobs) or a
                                        sub-bucket table overflowed (Bloom jobs, shared-memory path): the
                                        job regrows / splits and counts again, with exact results */
#define KC_INJECT_TABLE_FULL 4u      /* every counting attempt reports its table full: KC_ERR_DEVICE after
                                        the retries (plain jobs of one table) */
#define KC_INJECT_NOMEM 8u           /* the job's first device allocation fails as a failed cudaMalloc
                                        does: the job ends KC_ERR_NOMEM, the handle stays usable */

#define KC_STAGES 12         /* entries of kc_result_t.phase_ms */

typedef struct kc_handle kc_handle;
typedef struct kc_input kc_input;
typedef uint64_t kc_job_id;

typedef struct {
    int32_t device;               /* CUDA device ordinal */
    uint32_t max_inflight_jobs;   /* jobs on the device at once (streams); 0 -> 4 */
    uint64_t hbm_budget_bytes;    /* device memory jobs may reserve; 0 -> 90% of free memory */
    uint64_t workspace_bytes;     /* device workspace each worker allocates at kc_open (a server sized
                                     for its largest job never allocates, or synchronizes the device
                                     to grow, while jobs run); 0 -> grown to the largest job seen */
    uint64_t pinned_bytes;        /* pinned host memory kc_open sets aside for job results (records,
                                     count <= 2 sets), shared by all handles of the process and kept
                                     until it exits; results that do not fit use pinned blocks
                                     allocated on demand; 0 -> none */
    uint64_t reserved[4];
} kc_config;

typedef struct {
    const char *data;             /* one FASTQ file, uncompressed, in host memory */
    uint64_t size;
} kc_buffer;

typedef struct {
    /* input: either host files or a device-resident input from kc_input_upload */
    const kc_buffer *files;
    uint32_t n_files;
    uint32_t k;                   /* 1..128 (reference: <k_len>); batched jobs 1..32 */
    const kc_input *input;        /* non-NULL: use this resident input, ignore files */
    uint32_t count_max;           /* saturation of counts (reference [count_max], default 255) */
    uint32_t bloom;               /* 1: reference Bloom singleton split (src/BloomFilter.h) */
    uint64_t memory_gb;           /* reference <memory_limit_gb>, sizes the Bloom filters */
    uint32_t filter_min;          /* reference [filter_min]/[filter_max], applied by */
    uint32_t filter_max;          /*   kc_write_tmpdir to the high.bin records */
    uint32_t min_count;           /* records kept: min_count <= count <= max_count */
    uint32_t max_count;
    uint32_t hist_min;            /* histogram bins hist_min..hist_max */
    uint32_t hist_max;
    uint32_t top_n;               /* 0: no top-N query */
    uint32_t want_le2;            /* 1: the records with count <= 2 */
    uint32_t keep_records;        /* 1: copy the sorted records to host memory */
    uint32_t fault_inject;        /* testing aid: KC_INJECT_* bits, 0 in normal use */
    uint64_t pass_bytes;          /* device memory one counting pass may use; a job that needs more
                                     runs in passes over ranges of root prefixes, each pass's records
                                     held in pinned host memory until the final sort; 0 -> 70% of the
                                     device memory free for the job when its counting starts */
    uint32_t pack_high;           /* 1: the job packs the high.bin records (src/FinalDrainWriter.h:71-101,
                                     filter_min/filter_max applied) on the device, and kc_write_tmpdir
                                     writes those bytes (keep_records may then be 0); single jobs */
    uint32_t reserved_u32;
    uint64_t reserved[4];
} kc_job;

typedef struct {
    uint64_t n_records;           /* sorted records (if keep_records) */
    const uint64_t *keys;
    const uint32_t *counts;
    uint64_t hist_len;            /* hist[i] = k-mers with count hist_min + i */
    const int64_t *hist;
    uint64_t n_top;               /* top_n by count desc, then printed string asc */
    const uint64_t *top_keys;
    const uint32_t *top_counts;
    uint64_t n_le2;               /* records with count <= 2, printed-string order */
    const uint64_t *le2_keys;
    const uint32_t *le2_counts;
    uint64_t occurrences;         /* k-mer occurrences counted */
    uint64_t distinct;            /* distinct canonical k-mers */
    uint64_t low_only;            /* Bloom mode: k-mers seen once and only as FIRST */
    uint64_t table_capacity;      /* slots of the counting table */
    double device_ms;             /* device time of the counting pipeline */
    double queue_ms;              /* submission -> start */
    double run_ms;                /* start -> end (host clock) */
    /* device time per stage (CUDA events on the job's stream):
     * [0] newline census + tile line numbers, [1] SCAN pass, [2] INSERT pass
     * (plain) or scatter into the root-prefix buckets (Bloom), [3] insert of
     * the non-FIRST k-mers, [4] merge of the FIRST k-mers, [5] compaction +
     * histogram, [6] radix sort, [7] queries, [8] Bloom classification,
     * [9] scatter of the buckets into filter sub-buckets and [10] their
     * shared-memory Bloom split + count + compaction (Bloom mode, min count
     * >= 2), [11] packing of the high.bin records (kc_job.pack_high) */
    double phase_ms[KC_STAGES];
    uint64_t phase_launches[KC_STAGES];   /* kernel launches per stage */
    uint64_t low_len;             /* Bloom mode: FIRST occurrences (merged after the inserts) */
    uint64_t high_len;            /* occurrences inserted into root-prefix bucket tables (Bloom mode:
                                     the non-FIRST ones; large plain jobs: all); 0 for one table */
    uint64_t input_bytes;         /* FASTQ bytes of the job */
    uint64_t n_records_total;     /* records on the device (also when keep_records = 0) */
    uint32_t passes;              /* counting passes over ranges of root prefixes (1: the whole job at once) */
    uint16_t smem_passes;         /* passes counted on the shared-memory sub-bucket path (Bloom mode) */
    uint16_t smem_fallbacks;      /* passes that left it after a sub-bucket table overflowed */
    uint32_t region_redos;        /* shared-memory passes counted again because a sub-bucket outgrew the
                                     region estimated from a sample of the pass's keys */
    uint32_t batch_part;          /* batched jobs: the sub-batch (0, 1, ...) the sample was counted in; a
                                     batch larger than a worker's share of the device-memory budget runs
                                     as consecutive sub-batches, and device_ms is that sub-batch's time */
    uint32_t key_words;           /* 64-bit words per k-mer in keys, top_keys and le2_keys (kc_key_words) */
    uint32_t reserved_u32;
} kc_result_t;

/* Settings of a handle that trade memory for speed, chosen by kc_autotune or
 * set by the caller; a job uses the settings in force when it starts. */
typedef struct {
    double bucket_table_factor;   /* table slots per estimated key, per-bucket tables of the partitioned
                                     path (filled while in L2); default 3.0 */
    double table_factor;          /* table slots per estimated key, one-table jobs and batched samples;
                                     default 1.6 */
    uint64_t sort_group_records;  /* records sorted together (kept in L2) by a batch's segmented sort;
                                     default 4M */
    uint64_t bloom_smem;          /* Bloom jobs with min_count >= 2: 1 counts each filter sub-bucket (a slice
                                     of at most 2048 blocks, 32 KiB) in shared memory, 2 uses global-memory
                                     filters and tables; default 1 */
    uint64_t record_sort;         /* records of jobs with at least 1M of them: 1 sorts most significant bits
                                     first (bucket scatter + shared-memory sort per bucket), 2 with the
                                     8-bit LSD radix sort; default 1 */
    uint64_t sampled_region_keys; /* Bloom passes (shared-memory path) with at least this many k-mers size
                                     their sub-buckets from a 1-in-8 sample of the k-mers instead of
                                     counting them all (a sub-bucket that outgrows its estimate sends the
                                     pass back to exact counts); default 64M */
    uint64_t count_shape;         /* block shape of the shared-memory count: 1 = 512-thread blocks, two per
                                     SM, filter slices of up to 2048 blocks, 4096-slot tables; 2 = 256-thread
                                     blocks, four per SM, slices of up to 1024 blocks, 2048-slot tables
                                     (sub-buckets of half the k-mers); 3, 4 = 1, 2 with table slots from one
                                     multiply instead of a 64-bit mix; default 1 */
    uint64_t part_shape;          /* the partition's rounds: 1 = 4096 k-mers staged per round (three blocks
                                     per SM), 2 = 2048 (four blocks per SM); default 1 */
    uint64_t scatter_shape;       /* the sub-bucket scatter: 1 = two blocks per SM, 2 = a variant with fewer
                                     registers, three per SM (passes whose buckets have at most 1024
                                     sub-buckets); default 1 */
    uint64_t reserved[3];
} kc_tuning;

/* 64-bit words of one k-mer: 1 for k <= 32, 2 for k <= 64, 4 for k <= 128,
 * 0 otherwise (the reference's kmer<N>, src/main.cpp:617-633). */
uint32_t kc_key_words(uint32_t k);

/* Kernel launches issued by this process so far (all handles). */
uint64_t kc_kernel_launches(void);

/* ---- handle ------------------------------------------------------------ */
int kc_open(const kc_config *cfg, kc_handle **out);
void kc_close(kc_handle *h);
const char *kc_last_error(void);
void kc_job_defaults(kc_job *job);   /* reference defaults: count_max 255, filter 2..u32max, ... */

int kc_get_tuning(kc_handle *h, kc_tuning *out);
int kc_set_tuning(kc_handle *h, const kc_tuning *t);   /* values <= 0 keep the current one */
/* Autotuner (no counterpart in the reference, whose map capacity is a fixed
 * command-line value, src/main.cpp:539-542): runs the given jobs (as one
 * batch when `batch` is 1) once per candidate setting, one setting at a time
 * with the others fixed, and keeps the setting with the least device time.
 * The handle then uses the best settings, which are also returned. */
int kc_autotune(kc_handle *h, const kc_job *jobs, uint32_t n_jobs, uint32_t batch, kc_tuning *best);

/* ---- device-resident input --------------------------------------------- */
int kc_input_upload(kc_handle *h, const kc_buffer *files, uint32_t n_files, kc_input **out);
void kc_input_free(kc_handle *h, kc_input *in);

/* ---- jobs ---------------------------------------------------------------- */
int kc_submit(kc_handle *h, const kc_job *job, kc_job_id *id);
int kc_wait(kc_handle *h, kc_job_id id, int32_t timeout_ms);   /* <0: no limit */
int kc_result(kc_handle *h, kc_job_id id, kc_result_t *out);
int kc_write_tmpdir(kc_handle *h, kc_job_id id, const char *dir);
int kc_release(kc_handle *h, kc_job_id id);
/* Cancels a job (no counterpart in the reference, which runs one job per
 * process).  A queued job is taken off the queue; a running job stops at its
 * next stage boundary and gives back its device memory.  Either way kc_wait
 * then returns KC_ERR_CANCELLED.  Returns KC_ERR_INVALID when the job had
 * already finished (its results stand). */
int kc_cancel(kc_handle *h, kc_job_id id);

/* Batched jobs: every job of the array is counted in one set of device passes
 * (one persistent extraction kernel over all samples' tiles, per-sample
 * tables in one arena); a batch larger than a worker's share of the
 * device-memory budget is cut into consecutive sub-batches of whole samples.
 * Bloom mode is not available here.  ids[i] is the id of jobs[i]; results
 * are read per id as for kc_submit. */
int kc_submit_batch(kc_handle *h, const kc_job *jobs, uint32_t n_jobs, kc_job_id *ids);

/* ---- pinned host memory (for zero-copy-speed uploads) -------------------- */
int kc_host_alloc(uint64_t bytes, void **p);
int kc_host_free(void *p);

/* ---- single steps of the path, for tests and tools ----------------------- */

/* Canonical k-mer occurrences of one FASTQ file (src/FastqReader.h:559-698
 * record splitting + src/GetKmer.h:58-130 extraction), in no particular
 * order, kc_key_words(k) words each (k 1..128; out holds cap occurrences).
 * *n_out receives the number of occurrences even if it exceeds cap. */
int kc_extract_kmers(const char *fastq, uint64_t len, uint32_t k, uint64_t *out, uint64_t cap,
                     uint64_t *n_out);

/* out[5i..5i+4] = XXH3_128bits.low64, .high64, XXH3_64bits, rapidhash,
 * komihash(seed 0) of the 8-byte word keys[i] (include/xxhash.h 0.8.3,
 * include/rapidhash.h V3, include/komihash.h 5.29 as called at
 * src/BloomFilter.h:217, tool/FlatConcurrentHashMap.h:95,
 * src/ConcurrentMap.h:143-144). */
int kc_hash_kmers(const uint64_t *keys, uint64_t n, uint64_t *out);

/* Stable LSD radix sort of (key, count) pairs on the low `bits` bits of the
 * keys (sort/ExportRecordRadixSort.h:225-269, tool/dump_tool.cpp:373-454). */
int kc_sort_records(uint64_t *keys, uint32_t *counts, uint64_t n, uint32_t bits);

/* Sort of (key, count) records whose keys are all distinct, such as a job's
 * records or the tools' merged records (tool/dump_tool.cpp:373-454 sorts
 * those with an 11-bit LSD radix sort), on the low `bits` bits of the keys.
 * From 1M records and 24 bits on it sorts most significant bits first (a
 * bucket histogram, two scatter passes, one shared-memory sort per bucket),
 * below that with the LSD sort of kc_sort_records.  Equal keys are not
 * allowed (their order is unspecified). */
int kc_sort_distinct_records(uint64_t *keys, uint32_t *counts, uint64_t n, uint32_t bits);

/* kc_sort_records for callers that cannot allocate device memory.  No
 * counterpart in the reference.  Some callers may not call cudaMalloc where
 * they need sorted records (a fixed, pre-accounted device-memory budget owned
 * by another allocator, or a latency-critical path where an allocation can
 * stall or synchronize the device).  This call sorts the caller's DEVICE
 * arrays d_keys/d_counts (n records, low `bits` bits of the keys, stable) in
 * place on `stream` (a cudaStream_t, NULL for the default stream) and returns
 * when the sort is done.  It allocates nothing: its working memory is a fixed
 * 13 MiB device array inside libkc.so that every GPU loading the library holds
 * until the process exits, so n is limited to KC_SORT_NOALLOC_MAX records
 * (larger n is rejected with KC_ERR_INVALID).  The first call on a device
 * does a one-time set-up with the device current: it looks up that array's
 * device address (cudaGetSymbolAddress) and loads the array and the sort
 * kernels onto the device (with CUDA's default lazy module loading they would
 * otherwise be loaded, taking device memory, at first use); a call with n = 0
 * does only this set-up.  Every call waits for its sort to finish on
 * `stream` before returning, so it cannot be part of a CUDA graph: on a
 * stream that is being captured it returns KC_ERR_INVALID and enqueues
 * nothing (make the first, set-up call before any capture).  All
 * calls share the one array: calls that overlap on the GPU (another host
 * thread, another stream) race and must be serialized by the caller. */
#define KC_SORT_NOALLOC_MAX (1u << 20)
int kc_sort_records_noalloc(uint64_t *d_keys, uint32_t *d_counts, uint64_t n, uint32_t bits, void *stream);

/* The sorted dump of the reference's dump_tool (tool/dump_tool.cpp:1172-1193,
 * kmer_to_buf :103-124): one "KMER\tcount\n" line per record, the k-mer's
 * printed string from its kmer<N> words (kc_key_words(k) per record, k
 * 1..128), formatted on the device.  With out ==
 * NULL only *n_bytes (the text's length) is computed; otherwise the text goes
 * to out (cap bytes) and *n_bytes receives its length. */
int kc_dump_text(const uint64_t *keys, const uint32_t *counts, uint64_t n, uint32_t k, char *out, uint64_t cap,
                 uint64_t *n_bytes);

/* Measurement aid, no counterpart in the reference: throughput of random
 * 32-bit atomicAdd (no return value) over a device buffer of buffer_bytes (a
 * power of two), averaged over `repeats` launches.  A buffer far larger than
 * L2 gives the DRAM atomic peak the table insert is compared with; a buffer
 * that fits in L2 gives the L2 atomic peak (the per-bucket tables are sized
 * to stay L2-resident). */
int kc_atomic_peak(uint64_t buffer_bytes, uint32_t repeats, double *atomics_per_s, double *ms_per_launch);

/* Measurement aid, no counterpart in the reference: the same random atomicAdd
 * on a table of table_bytes (a power of two, 4 KiB..64 KiB) in shared memory,
 * one table per block of the shared-memory count's shape.  The peak that
 * count's table inserts are compared with. */
int kc_atomic_peak_shared(uint32_t table_bytes, uint32_t repeats, double *atomics_per_s, double *ms_per_launch);

/* Pre-pass statistics and Bloom sizing of a job (src/main.cpp:262-335 with
 * get_MAX_BLOOM_FILTER_CAPACITY :41 and calculate_bloom_filter_capacity :111):
 * raw root-prefix counts over the sample, average quality, capacities. */
int kc_bloom_plan(const kc_buffer *files, uint32_t n_files, uint32_t k, uint64_t memory_gb,
                  uint32_t *prefix_counts /*256*/, uint32_t *avg_quality,
                  uint64_t *capacities /*256*/, uint64_t *max_capacity);

/* The reference's Bloom filter sizing alone (host arithmetic, no device):
 * src/main.cpp:41-57 and :111-153 applied to raw pre-pass root-prefix counts
 * (counts below 1000 are raised to 1000 as src/main.cpp:306-315 does). */
int kc_plan_bloom(const uint32_t *raw_prefix_counts /*256*/, uint32_t avg_quality, uint64_t est_file_size,
                  uint64_t memory_gb, uint32_t k, uint64_t *capacities /*256*/, uint64_t *max_capacity);

/* The precise merge of the reference tools (tool/histogram_tool.cpp:735-791
 * with tool/LowFrequencyQueryThreadPool.h:186-240; tool/dump_tool.cpp:1202-1272)
 * on the device: high.bin records (keys, counts) and low.bin k-mers become
 * exact counts -- min(high + 1, count_max) for a k-mer in both files, the
 * high count for one only in high.bin, 1 for one only in low.bin.  Records
 * with min_count <= count <= max_count are written sorted in printed-string
 * order (*n_out receives their number even if it exceeds out_cap); hist
 * (hist_max - hist_min + 1 entries, may be NULL) receives the histogram of
 * all merged counts.  k is 1..128; every key array holds kc_key_words(k)
 * words per k-mer. */
int kc_merge_records(const uint64_t *high_keys, const uint32_t *high_counts, uint64_t n_high,
                     const uint64_t *low_keys, uint64_t n_low, uint32_t k, uint32_t count_max,
                     uint32_t min_count, uint32_t max_count, uint32_t hist_min, uint32_t hist_max,
                     uint64_t *out_keys, uint32_t *out_counts, uint64_t out_cap, uint64_t *n_out,
                     int64_t *hist);

#ifdef __cplusplus
}
#endif

#endif
