// kc_wide.cuh -- k-mers of 33..128 bases: the reference's kmer<2> (k <= 64)
// and kmer<4> (k <= 128) paths (src/main.cpp:617-633).
//
// A k-mer is its kmer<N> word array (src/kmer.h:15, data[0] first): the
// newest base of the window at data[0]'s top bits, older bases towards
// data[last] (last = (k - 1) / 32), whose low 64 - 2 * (k % 32) bits are
// zero; words above data[last] are zero.  Records are N words + a u32 count,
// the words of record i at keys[i * N .. i * N + N).
#pragma once

#include "kc_kernels.cuh"

namespace kc {

constexpr uint32_t WIDE_HALO = 128;   // bytes before a tile read with it: k - 1 <= 127

inline uint32_t key_words(uint32_t k) { return k <= 32 ? 1u : (k <= 64 ? 2u : 4u); }

// Open-addressing table of N-word keys.
//
// N = 2: a slot is its key, one 16-byte word, all ones when empty (never a
// canonical key: k < 64 leaves low bits of data[1] zero, and at k = 64 the
// all-T key's reverse complement, all A, is smaller).  A probe reads the slot
// with one 128-bit load; an empty slot is claimed by one 128-bit CAS that
// writes the whole key, so no reader can see half a key and nothing waits.
// meta[i] is slot i's count; meta[cap] / meta[cap + 1] hold the count / the
// presence of the all-ones key itself, which only a merge of foreign records
// can bring.
//
// N = 4: a slot is claimed by one CAS of its state (0 -> 1), its key written
// and then published (state 2, release); every other thread compares keys
// only in published slots.  A thread that meets a claimed, unpublished slot
// waits for it (bounded, ERR_WAIT_TIMEOUT).  meta[2i], meta[2i + 1] = state,
// count of slot i.
//
// keys holds cap * N words (slot i at keys[i * N]), meta 2 * cap + 2 words.
struct WideTable {
    unsigned long long *keys;
    uint32_t *meta;
    unsigned long long cap;
};

enum WideMode : int { WMODE_SCAN = 0, WMODE_INSERT = 1, WMODE_EMIT = 2 };

struct WideArgs {
    const uint8_t *buf;               // first byte of tile 0 (FRONT_PAD >= WIDE_HALO zero bytes before it)
    uint64_t n_tiles;
    const uint64_t *tile_prefix;      // exclusive newline count before each tile
    const uint32_t *tile_seg;
    const Seg *segs;
    unsigned long long *counters;     // C_COUNT words
    // SCAN: occurrences, HyperLogLog registers (HLL_M), root-prefix histogram
    unsigned long long *occ;
    uint32_t *hll;
    unsigned long long *bucket_hist;  // 256: occurrences per top byte of data[0]
    // INSERT: the table; a pass keeps root prefixes lo <= b < hi (hi 0: all)
    WideTable table;
    uint32_t max_probe;
    uint32_t bucket_lo, bucket_hi;
    // EMIT: occurrences appended at list[C_EMIT_LEN * N], list_cap k-mers
    unsigned long long *list;
    unsigned long long list_cap;
};

cudaError_t launch_wide_extract(int mode, uint32_t k, const WideArgs &a, cudaStream_t st);
cudaError_t launch_wide_init(uint32_t k, WideTable t, cudaStream_t st);
// (key, count) records into the table (the tools' merge: high.bin records
// with their counts, low.bin k-mers with count 1).
cudaError_t launch_wide_insert_pairs(uint32_t k, const unsigned long long *keys, const uint32_t *counts,
                                     uint32_t count_if_null, uint64_t n, WideTable t, uint32_t max_probe,
                                     unsigned long long *counters, cudaStream_t st);
// Published slots: *kept = slots whose saturated count is in [min, max],
// counters[C_DISTINCT] += published slots.  count_only = 1 writes nothing
// else; 0 appends the kept records at rec_keys / rec_counts (C_REC_LEN, at
// most rec_cap) and adds every slot's count to hist / ovf.
cudaError_t launch_wide_compact(uint32_t k, WideTable t, uint32_t count_max, uint32_t min_count, uint32_t max_count,
                                unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                                unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap,
                                unsigned long long *counters, int count_only, cudaStream_t st);
// Sort of n records in printed-string order: LSD by words (data[0] first,
// each a stable radix sort of its pair-reversed word, data[last] on its
// 2 * (k % 32) bits), then the records permuted into out_keys / out_counts.
// tmp holds wide_sort_tmp_bytes(n) bytes.
size_t wide_sort_tmp_bytes(uint64_t n);
cudaError_t launch_wide_sort(uint32_t k, const unsigned long long *keys, const uint32_t *counts, uint64_t n,
                             unsigned long long *out_keys, uint32_t *out_counts, void *tmp,
                             unsigned long long *flags, cudaStream_t st);
// out rows i = keys rows idx[i] (idx: record positions as 64-bit words).
cudaError_t launch_wide_gather_rows(uint32_t k, const unsigned long long *keys, const unsigned long long *idx,
                                    uint64_t n, unsigned long long *out, cudaStream_t st);
// 0, 1, 2, ... n - 1
cudaError_t launch_iota_u64(unsigned long long *p, uint64_t n, cudaStream_t st);

// high.bin bytes of sorted records (src/FinalDrainWriter.h:71-88): for each
// record whose count c has c + 1 >= filter_min and c <= filter_max
// (src/FinalDrainWriter.h:101), the k / 32 full words (little-endian), the
// top (2 * (k % 32) + 7) / 8 bytes of the next word, the count's low
// count_bytes bytes, written in record order.  keys hold key_words(k)
// words per record.  flags (n) and pos (n) and scan_tmp
// (scan_tmp_words(n)) are scratch; *n_bytes (device) receives the length.
// out holds n * packed_record_bytes(k, count_bytes) bytes.
uint32_t packed_record_bytes(uint32_t k, uint32_t count_bytes);
cudaError_t launch_pack_high(uint32_t k, const unsigned long long *keys, const uint32_t *counts, uint64_t n,
                             uint32_t count_bytes, uint32_t filter_min, uint32_t filter_max, uint32_t *flags,
                             unsigned long long *pos, unsigned long long *scan_tmp, uint8_t *out,
                             unsigned long long *n_bytes, cudaStream_t st);

}  // namespace kc
