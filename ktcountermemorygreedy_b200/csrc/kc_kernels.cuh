// kc_kernels.cuh -- host-visible declarations of the device pipeline stages.
// All launches are stream-ordered; none allocates memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kc {

constexpr uint32_t TILE = 8192;         // FASTQ bytes per extraction tile
constexpr uint32_t HALO = 32;           // bytes before a tile read with it (k <= 32)
constexpr uint32_t FRONT_PAD = 256;     // zero bytes before tile 0 in the device buffer
constexpr uint32_t EXT_THREADS = 256;   // one 32-byte segment per thread
constexpr uint32_t STAGE_CAP = 4096;    // staged k-mers per extraction round
constexpr uint32_t HLL_BITS = 12;       // HyperLogLog registers per sample = 2^12
constexpr uint32_t HLL_M = 1u << HLL_BITS;
constexpr uint32_t BATCH_HLL_SAMPLE_BITS = 6;  // batched samples' registers see a 1-in-64 hash sample
constexpr uint32_t HIST_BINS = 1u << 16;  // dense count histogram; larger counts go to a list
constexpr uint32_t HIST_BINS_BATCH = 4096;  // per-sample dense histogram of batched jobs
constexpr uint32_t MAX_BATCH = 4096;        // samples in one batched job
constexpr uint64_t PREPASS_CHUNK = 2ULL * 1024 * 1024;  // reference reader chunk

// error flags (bit mask in counters[C_FLAGS])
constexpr unsigned long long ERR_TABLE_FULL = 1ull << 0;
constexpr unsigned long long ERR_LIST_FULL = 1ull << 1;
constexpr unsigned long long ERR_WAIT_TIMEOUT = 1ull << 2;
constexpr unsigned long long ERR_RECORDS_FULL = 1ull << 3;
constexpr unsigned long long ERR_HIST_OVERFLOW_FULL = 1ull << 4;

// indexes into the per-job device counter block (unsigned long long each)
enum Counter : int {
    C_FLAGS = 0,
    C_LOW_LEN = 1,       // Bloom FIRST occurrences (low list, front of the list buffer)
    C_HIGH_LEN = 2,      // other occurrences (back of the list buffer)
    C_EMIT_LEN = 3,      // plain occurrence list (testing entry point)
    C_REC_LEN = 4,       // output records
    C_LOW_ONLY = 5,      // low k-mers absent from the table (final count 1)
    C_DISTINCT = 6,      // distinct k-mers seen by compaction
    C_OVF_LEN = 7,       // histogram counts >= HIST_BINS
    C_SEL_A = 8,         // query selections
    C_SEL_B = 9,
    C_SUB_OVF = 10,      // sub-buckets whose shared-memory table overflowed
    C_REGION_OVF = 11,   // nonzero: a sub-bucket outgrew its estimated region
    C_KEPT = 12,         // records a counting compaction pass would keep
    C_COUNT = 16
};

// One FASTQ file inside a job's device buffer.  Files start on tile
// boundaries; bytes between a file's end and the next tile boundary are zero.
struct Seg {
    uint64_t first_tile;
    uint64_t n_tiles;
    uint64_t len;          // file bytes
    uint64_t sample_end;   // the pre-pass reads bytes [0, sample_end)
    uint32_t k;
    uint32_t sample;       // owning sample (batched jobs); 0 for a single job
};

struct Slot {              // open-addressing table slot (16 bytes)
    unsigned long long key;
    unsigned int count;
    unsigned int pad;
};

struct TableRef {
    Slot *slots;
    unsigned long long mask;   // capacity - 1 (capacity is a power of two)
};

struct SampleCfg {          // one sample of a batched job
    unsigned long long slot_base, slot_cap;   // its table inside the slot arena
    unsigned long long rec_base, rec_cap;     // its record region
    uint32_t count_max, min_count, max_count, k;
};

struct SortTile {           // one radix-sort tile of a (possibly segmented) sort
    uint64_t begin, end;    // record range
    uint64_t cbase;         // digit-count index of digit 0; digit d at cbase + d * stride
    uint64_t stride;
    uint64_t adjust;        // segment start minus records of earlier segments
};

struct ExtractArgs {
    const uint8_t *buf;             // first byte of tile 0 (FRONT_PAD zero bytes before it)
    uint64_t n_tiles;
    const uint64_t *tile_prefix;    // exclusive newline count before each tile
    const uint32_t *tile_seg;       // file of each tile
    const Seg *segs;
    unsigned long long *counters;   // C_COUNT words
    // scan mode
    unsigned long long *occ;        // occurrences per sample
    uint32_t *hll;                  // HLL_M registers per sample; NULL: no distinct estimate
    int hll_local;                  // single sample: registers kept in shared memory per block
    int prepass;                    // also accumulate the pre-pass statistics
    const int32_t *chunk_lastnl;    // per 2 MiB chunk (global chunk index), last '\n' offset in chunk
    const uint64_t *seg_chunk0;     // first global chunk index of each file
    uint32_t *prefix_hist;          // 256 per sample
    unsigned long long *qual;       // 2 per sample: byte sum, byte count
    // insert mode
    const TableRef *tables;         // per sample
    uint32_t max_probe;
    // bloom mode (single sample)
    const unsigned long long *bloom_off;   // 256 word offsets
    const unsigned long long *bloom_cap;   // 256 capacities (blocks of two words)
    unsigned long long *bloom_bits;
    uint32_t *hll_high;             // HLL registers of the non-FIRST occurrences
    // emit / bloom / part output list
    unsigned long long *list;
    unsigned long long list_cap;
    // root-prefix buckets (single sample): SCAN counts, PART scatters
    unsigned long long *bucket_hist;          // 256 counts (SCAN)
    uint64_t bucket_sample_mask;              // SCAN counts tiles t with (t & mask) == 0
    // SCAN over a subset of the tiles: visit[0..n_visit) ascending tile
    // indexes (NULL: every tile); occurrences are then counted on the census
    // tiles only
    const uint32_t *visit;
    uint64_t n_visit;
    uint32_t bucket_lo, bucket_hi;            // PART keeps buckets lo <= b < hi (hi 0: all)
    uint64_t tile0;                           // without visit: tiles tile0 .. tile0 + n_tiles - 1
    unsigned long long *bucket_cursor;        // 256 fill levels (PART)
    const unsigned long long *bucket_base;    // 256 start offsets in `list` (PART)
    const unsigned long long *bucket_end;     // 256 end offsets in `list` (PART)
};

enum ExtractMode : int { MODE_SCAN = 0, MODE_INSERT = 1, MODE_BLOOM = 2, MODE_EMIT = 3, MODE_PART = 4 };

constexpr uint32_t WORK_ITEM_KEYS = 2048;   // k-mers per work item (8 per thread)
constexpr uint32_t BUCKET_HLL_BITS = 10;    // HyperLogLog registers per bucket = 2^10
constexpr uint32_t BUCKET_HLL_M = 1u << BUCKET_HLL_BITS;
constexpr uint32_t BUCKET_HLL_SAMPLE_BITS = 6;  // the bucket registers see a 1-in-64 hash sample
constexpr uint32_t N_BUCKETS = 256;         // root prefix = top 8 bits of the k-mer word

// A run of k-mers of one root-prefix bucket processed by one block of the
// bucket-major kernels (work items are issued in bucket order, so the blocks
// in flight touch one or two buckets' filters and tables, which stay in L2).
struct WorkItem {
    unsigned long long begin, end;   // range in the key array
    uint32_t bucket;
    uint32_t pad;
};

// The work of one bucket-major launch, 256 ranges instead of a list of work
// items: bucket b's keys [begin[b], begin[b] + len[b]) in runs of
// WORK_ITEM_KEYS, whose first run is item item0[b] (item0[N_BUCKETS] = all).
// A block turns its item number into a bucket and range by itself.
struct BucketRanges {
    unsigned long long begin[N_BUCKETS], len[N_BUCKETS];
    uint32_t item0[N_BUCKETS + 1];
};
uint32_t fill_item_starts(BucketRanges &r);   // sets item0 from len, returns the number of items
uint32_t fill_item_starts_n(BucketRanges &r, uint64_t item_keys);   // items of item_keys keys
constexpr uint32_t SUB_SCATTER_ITEM_KEYS = 4096;   // keys per work item of the sub-bucket scatter

// Shared-memory sub-bucket path of the Bloom split: every bucket is cut
// into n_sub sub-buckets of 2^slice_shift consecutive blocks of its filter (a
// k-mer's sub-bucket follows from its filter block), so one thread block
// holds a sub-bucket's filter slice and counting table in shared memory.
constexpr uint32_t SUB_SLICE_BLOCKS = 2048;     // largest slice (2 words a block): 32 KiB of filter
constexpr uint32_t SUB_TABLE_BITS = 12;
constexpr uint32_t SUB_TABLE_SLOTS = 1u << SUB_TABLE_BITS;   // counting-table slots of a sub-bucket
constexpr uint32_t SUB_MAX_PER_BUCKET = 4096;   // sub-buckets of one bucket
struct SubCfg {
    unsigned long long fcap;    // the bucket's filter blocks (a power of two)
    uint32_t sub_base, n_sub;   // its sub-buckets [sub_base, sub_base + n_sub), n_sub = fcap >> slice_shift
    uint32_t slice_shift;       // log2 of the blocks of one slice, <= log2(SUB_SLICE_BLOCKS)
    uint32_t pad;
};

// Per-bucket state of the partitioned pipeline.
struct BucketCfg {
    unsigned long long key_base, key_len;    // bucket's range in the partitioned key array
    unsigned long long bloom_off, bloom_cap; // its Bloom filter (words offset, blocks)
    unsigned long long slot_base, slot_cap;  // its sub-table in the slot arena
};

size_t extract_smem_bytes();
unsigned long long kernel_launches();          // launches issued by this process
unsigned long long thread_kernel_launches();   // launches issued by the calling thread
cudaError_t launch_newlines(const uint8_t *buf, uint64_t n_tiles, uint32_t *tile_nl, int32_t *tile_lastnl,
                            cudaStream_t st);
cudaError_t launch_chunk_lastnl(const int32_t *tile_lastnl, const uint32_t *tile_seg, const Seg *segs,
                                const uint64_t *seg_chunk0, uint64_t n_tiles, int32_t *chunk_lastnl,
                                cudaStream_t st);
// part_shape (MODE_PART, kc_tuning.part_shape): 1 stages 4096 k-mers a round
// (three blocks per SM), 2 stages 2048 (four blocks per SM).
cudaError_t launch_extract(int mode, const ExtractArgs &a, int grid, cudaStream_t st, uint32_t part_shape = 1);

// Exclusive prefix sum of n 32-bit values into 64-bit outputs.  tmp must
// hold scan_tmp_words(n) 64-bit words.
size_t scan_tmp_words(uint64_t n);
cudaError_t launch_scan_u32(const uint32_t *in, unsigned long long *out, uint64_t n, unsigned long long *tmp,
                            cudaStream_t st);

cudaError_t launch_init_slots(Slot *slots, uint64_t n, cudaStream_t st);
cudaError_t launch_count_keys(const Slot *slots, uint64_t n, unsigned long long *out, cudaStream_t st);
cudaError_t launch_fill_u64(unsigned long long *p, uint64_t n, unsigned long long v, cudaStream_t st);
cudaError_t launch_add_u64(unsigned long long *dst, const unsigned long long *src, uint64_t n, cudaStream_t st);
cudaError_t launch_insert_list(const unsigned long long *keys, uint64_t n, TableRef t, uint32_t max_probe,
                               unsigned long long *counters, cudaStream_t st);
cudaError_t launch_insert_pairs(const unsigned long long *keys, const uint32_t *counts, uint64_t n, TableRef t,
                                uint32_t max_probe, unsigned long long *counters, cudaStream_t st);
cudaError_t launch_merge_low(const unsigned long long *keys, uint64_t n, TableRef t, uint32_t max_probe,
                             uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                             uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *counters,
                             cudaStream_t st);
cudaError_t launch_compact(TableRef t, uint64_t cap, uint32_t count_max, uint32_t min_count, uint32_t max_count,
                           unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                           unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap,
                           unsigned long long *counters, cudaStream_t st);

// Slot-order compaction of one table or bucket arena (records in slot order,
// so a bucket arena gives records grouped by bucket).  Run once with
// count_only = 1 (chunk_keep[c] = records kept by chunk c, C_DISTINCT +=
// occupied slots), scan chunk_keep into chunk_pos, then with count_only = 0
// (records written from chunk_pos[c] on, histogram added to).
uint64_t compact_ordered_chunks(uint64_t cap);
cudaError_t launch_compact_ordered(const Slot *slots, uint64_t cap, uint32_t count_max, uint32_t min_count,
                                   uint32_t max_count, uint32_t *chunk_keep, const unsigned long long *chunk_pos,
                                   unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                                   unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap,
                                   unsigned long long *counters, int count_only, cudaStream_t st);

// LSD radix sort of (key, value) pairs on the low `bits` bits of the keys,
// 8 bits per pass.  Result ends in keys/vals.
size_t sort_tmp_bytes(uint64_t n);
size_t sort_tmp_bytes_segmented(uint64_t n_total, const uint64_t *seg_len, uint32_t n_segs);
cudaError_t launch_radix_sort_segmented(unsigned long long *keys, uint32_t *vals, uint64_t n_total,
                                        const uint64_t *seg_start, const uint64_t *seg_len, uint32_t n_segs,
                                        uint32_t bits, void *tmp, cudaStream_t st, unsigned long long *flags = nullptr,
                                        const uint32_t *seg_bits = nullptr,    // per segment, <= bits
                                        uint64_t group_records = 4ull << 20);  // records per L2-sized group
// One segment, one kernel per 8-bit pass; a look-back wait that gave up sets
// ERR_WAIT_TIMEOUT in *flags (NULL: a word inside tmp).  Keys already in
// order of their low skip_bits bits (a multiple of 8) skip those passes.
// input_in_tmp: the records are in the alternate buffers inside tmp
// (sort_tmp_alt) instead of keys/vals; the result still ends in keys/vals,
// without a final copy when sort_passes_run() is odd.
cudaError_t launch_radix_sort(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits, void *tmp,
                              cudaStream_t st, unsigned long long *flags = nullptr, uint32_t skip_bits = 0,
                              bool input_in_tmp = false);
void sort_tmp_alt(void *tmp, uint64_t n, unsigned long long **k2, uint32_t **v2);
uint32_t sort_passes_run(uint32_t bits, uint32_t skip_bits);

// Compaction of a batched job's slot arena in chunks of slots that each
// belong to one sample: count_only fills chunk_keep (records per chunk) and
// distinct (per sample); the write pass puts chunk c's records at
// chunk_pos[c] (the exclusive scan of chunk_keep) and fills the per-sample
// histograms.  chunk0 has n_samples + 1 entries: first chunk of each sample.
uint64_t compact_chunks_of(uint64_t slot_cap);
cudaError_t launch_compact_chunks(const Slot *slots, const SampleCfg *cfg, const uint32_t *chunk0, uint32_t n_samples,
                                  uint64_t n_chunks, uint32_t *chunk_keep, const unsigned long long *chunk_pos,
                                  unsigned long long *rec_keys, uint32_t *rec_counts, unsigned long long *hist,
                                  unsigned long long *ovf, uint64_t ovf_cap, unsigned long long *distinct,
                                  unsigned long long *counters, int count_only, cudaStream_t st);
// A sort of one segment with every buffer, tile descriptors included, taken
// from tmp (sort_tmp_bytes_in_scratch(n) bytes) and nothing copied from the
// host (digit counts, a scan and a scatter per pass).
size_t sort_tmp_bytes_in_scratch(uint64_t n);
// Loads the kernels launch_radix_sort_in_scratch uses (lazy module loading
// would otherwise load them, and take device memory, at their first launch).
cudaError_t preload_sort_in_scratch();
cudaError_t launch_radix_sort_in_scratch(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits,
                                         void *tmp, cudaStream_t st);

// Sort of distinct keys (a job's records) on their low `bits` bits, most
// significant bits first: a bucket histogram of the top 8..16 bits, a scatter
// pass by the top 8 bits and one by the next bits inside those ranges, then
// every bucket sorted in shared memory (kc_msd_sort.cu).  Synchronizes the
// stream once (the bucket sizes come to the host).  Result in keys/vals; with
// input_in_tmp the records start in the alternate arrays (sort_tmp_alt);
// with reverse_out the sorted keys are written with their 2-bit groups
// reversed (pair_reverse).  For n >= MSD_SORT_MIN_RECORDS and
// 24 <= bits <= 64 (msd_sort_applies).
constexpr uint64_t MSD_SORT_MIN_RECORDS = 1ull << 20;
bool msd_sort_applies(uint64_t n, uint32_t bits);
size_t msd_sort_tmp_bytes(uint64_t n, uint32_t bits);
cudaError_t launch_msd_sort(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits, void *tmp,
                            cudaStream_t st, unsigned long long *flags, bool input_in_tmp, bool reverse_out = false,
                            const uint32_t *hist16 = nullptr);
// hist16: when not NULL, the records per value of the keys' top 16 bits
// (key >> (bits - 16), 65536 counts) made while the records were written;
// the sort then reads no key for its bucket histogram.
// Counts one kernel launch of this library (kernels launched outside kc_kernels.cu).
void note_kernel_launch();

cudaError_t launch_pair_reverse(unsigned long long *keys, uint64_t n, cudaStream_t st);

// Stable selection of records whose count satisfies lo <= c <= hi: writes the
// selected keys/counts in input order.  Uses the scan temp space.
cudaError_t launch_select_range(const unsigned long long *keys, const uint32_t *counts, uint64_t n, uint32_t lo,
                                uint32_t hi, uint64_t limit, unsigned long long *out_keys, uint32_t *out_counts,
                                uint32_t *flags, unsigned long long *pos, unsigned long long *tmp,
                                unsigned long long *counters, int counter_idx, cudaStream_t st);

// Bucket-major kernels of the partitioned pipeline; each resets *next_item.
// Sub-bucket path.  count: sub_count[sub_base + s] += the keys of bucket b
// in sub-bucket s.  scatter: every key to out[sub_cursor[its sub-bucket]++]
// (sub_cursor starts at the exclusive scan of sub_count); its ranges rg are
// cut into items of SUB_SCATTER_ITEM_KEYS keys (fill_item_starts_n).  count_subs: one
// block per sub-bucket at a time runs the Bloom split with the filter slice in
// shared memory, counts the non-FIRST occurrences in a shared-memory table,
// merges the FIRST ones (written back over the front of the sub-bucket's
// keys) and appends (and, with hb16, counts every record's printed-order key
// >> hb16_shift, the record sort's buckets, into hb16[65536]) the table's records (counts saturated at count_max, kept
// when min_count <= count <= max_count) at rec_keys[C_REC_LEN...]; every
// table count goes to hist/ovf, the totals to counters (C_REC_LEN,
// C_LOW_LEN, C_HIGH_LEN, C_LOW_ONLY, C_DISTINCT) and the sub-buckets whose
// table overflowed to C_SUB_OVF and bucket_ovf[their bucket] (the results
// are then incomplete).
// stride > 1: only every stride-th run of 4 keys is counted (a sample).
cudaError_t launch_subpart_count(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 const SubCfg *sc, uint32_t *sub_count, cudaStream_t st, uint32_t stride = 1);
// sub_end non-NULL: the sub-buckets' regions are estimates and a key is
// written only inside its sub-bucket's region [.., sub_end[s]).
cudaError_t launch_subpart_scatter(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                   unsigned int *next_item, const SubCfg *sc, unsigned long long *sub_cursor,
                                   unsigned long long *out, uint64_t out_cap, uint32_t max_sub, cudaStream_t st,
                                   const unsigned long long *sub_end = nullptr, uint32_t scatter_shape = 1);
// scatter_shape 2 (kc_tuning.scatter_shape): launches whose buckets have at
// most 1024 sub-buckets run a variant with fewer registers, three blocks per SM.
// Estimated regions from a 1-in-stride sampled count: region (u32 per
// sub-bucket, scratch), sub_off (their exclusive scan), sub_end = sub_off +
// region, sub_cursor = sub_off.  scan_tmp holds scan_tmp_words(n_sub) words.
cudaError_t launch_subpart_regions(const uint32_t *sampled, uint32_t n_sub, uint32_t stride, uint32_t *region,
                                   unsigned long long *sub_off, unsigned long long *sub_end,
                                   unsigned long long *sub_cursor, unsigned long long *scan_tmp, cudaStream_t st);
// Keys per sub-bucket after a scatter into estimated regions; a sub-bucket
// that outgrew its region sets *overflow (its count is cut to its region).
cudaError_t launch_subpart_sizes(const unsigned long long *sub_off, const unsigned long long *sub_cursor,
                                 const unsigned long long *sub_end, uint32_t n_sub, uint64_t out_cap, uint32_t *count,
                                 unsigned long long *overflow, cudaStream_t st);
cudaError_t launch_count_subs(unsigned long long *keys, const unsigned long long *sub_off, const uint32_t *sub_count,
                              const uint8_t *sub_bucket, uint32_t n_sub, const SubCfg *sc, unsigned int *next_sub,
                              uint32_t count_max, uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                              uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist, uint32_t *ovf,
                              uint64_t ovf_cap, unsigned long long *counters, uint32_t *bucket_ovf, cudaStream_t st,
                              uint32_t *hb16 = nullptr, uint32_t hb16_shift = 0, uint32_t shape = 1);
// Block shapes of the shared-memory count (kc_tuning.count_shape): 1 and 3
// run 512-thread blocks, two per SM, filter slices of up to 2048 blocks and
// 4096-slot tables; 2 and 4 run 256-thread blocks, four per SM, slices of up
// to 1024 blocks and 2048-slot tables (sub-buckets of half the k-mers).  3
// and 4 place keys in the table by one multiply instead of the 64-bit mix.
inline uint32_t sub_slice_blocks(uint32_t shape) { return (shape == 2 || shape == 4) ? 1024u : 2048u; }
inline uint32_t sub_table_slots(uint32_t shape) { return (shape == 2 || shape == 4) ? 2048u : 4096u; }
cudaError_t launch_bloom_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 unsigned int *next_item, const BucketCfg *cfg, unsigned long long *bits,
                                 unsigned long long *out, unsigned long long *low_cnt, unsigned long long *high_cnt,
                                 uint32_t *hll_high, cudaStream_t st);
cudaError_t launch_insert_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                  unsigned int *next_item, const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                  unsigned long long *bucket_ovf, cudaStream_t st);
cudaError_t launch_merge_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 unsigned int *next_item, const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                 uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                                 uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *counters, cudaStream_t st);

// A bounded wait on the device word *flag (nonzero ends it): at most
// poll_limit polls about a microsecond apart, then ERR_WAIT_TIMEOUT is set in
// *flags and the kernel returns.
cudaError_t launch_wait_flag(const unsigned int *flag, uint32_t poll_limit, unsigned long long *flags, cudaStream_t st);
// *word |= bits on the device, in stream order.
cudaError_t launch_or_flags(unsigned long long *word, unsigned long long bits, cudaStream_t st);

// Batch of hash evaluations for the parity tests: out[5*i..5*i+4] =
// xxh3_128.lo, xxh3_128.hi, xxh3_64, rapidhash, komihash (all of keys[i]).
cudaError_t launch_hash_batch(const unsigned long long *keys, uint64_t n, unsigned long long *out,
                              cudaStream_t st);

// "KMER\tcount\n" lines of n records (kmer<N> keys of N words, k <= 128) into out,
// packed; len (n), off (n) and scan_tmp (scan_tmp_words(n)) are scratch, and
// off[n-1] + len[n-1] is the text's length.
cudaError_t launch_dump_text(const unsigned long long *keys, const uint32_t *counts, uint64_t n, uint32_t k,
                             uint32_t *len, unsigned long long *off, unsigned long long *scan_tmp, char *out,
                             cudaStream_t st);

// Random 32-bit atomicAdd microbenchmark over `words` (a power of two) words;
// *ops receives the number of adds the launch performs.
cudaError_t launch_atomic_peak(uint32_t *buf, uint64_t words, uint32_t iters, uint64_t seed, uint64_t *ops,
                               cudaStream_t st);
cudaError_t launch_atomic_peak_shared(uint32_t *out, uint32_t words, uint32_t iters, uint64_t seed, uint64_t *ops,
                                      cudaStream_t st);

}  // namespace kc
