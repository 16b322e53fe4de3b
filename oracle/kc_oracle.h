/*
 * kc_oracle.h -- CPU restatement of the reference k-mer counting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against.  Only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py may load it; the product (libkc.so, the CLIs) never links it.
 *
 * Every function cites the reference file:line whose behaviour it restates.
 * Parity of this restatement is pinned by tests/golden/ (vectors produced by
 * the reference's own sources compiled under oracle/_ref/, see oracle/Makefile).
 *
 * k-mers use the reference's internal kmer<1> word (src/kmer.h:15): for the
 * printed canonical string C of length k <= 32, base C[i] sits at bit
 * 64 - 2k + 2i (newest base at the MSB side), padding bits are zero.
 * Multi-word keys (k > 32) are only used by the file-format and tool-merge
 * helpers, laid out exactly like kmer<N>::data.
 */
#ifndef KC_ORACLE_H
#define KC_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- extraction ---------------------------------------------------------- */

/* One FASTQ file held in memory -> canonical k-mer occurrences in input order.
 * Returns the number of occurrences; writes at most `cap` of them. k in 1..32. */
uint64_t kco_extract(const uint8_t *data, uint64_t len, uint32_t k,
                     uint64_t *out, uint64_t cap);

/* k-mers of 33..128 bases: kmer<N> word arrays (N = kco_key_words(k): 1 for
 * k <= 32, 2 for k <= 64, 4 for k <= 128), N words per occurrence in `out`
 * (cap occurrences).  Words above the k-mer's last word are zero (GetKmer<4>
 * leaves stale bases in data[3] at k = 96; see kc_oracle.c). */
uint32_t kco_key_words(uint32_t k);
uint64_t kco_extract_wide(const uint8_t *data, uint64_t len, uint32_t k, uint64_t *out, uint64_t cap);
/* Hash-sampled extraction of N-word k-mers (kco_extract_sampled's rule with
 * the sample hash folded over the words). */
uint64_t kco_sample_hash_wide(const uint64_t *words, uint32_t n_words);
uint64_t kco_extract_wide_sampled(const uint8_t *data, uint64_t len, uint32_t k, uint32_t sample_bits,
                                  uint64_t *out, uint64_t cap);
/* Printed-string order key of one k-mer: N words, most significant first. */
void kco_string_key_wide(const uint64_t *words, uint32_t k, uint64_t *out);

/* Spot-check sample: kco_extract keeping only k-mers w with
 * (kco_sample_hash(w) & (2^sample_bits - 1)) == 0 -- every occurrence of a
 * kept k-mer, so their counts are exact.  The input must start at a record
 * start (a file, or a split point between two records). */
uint64_t kco_sample_hash(uint64_t w);
uint64_t kco_extract_sampled(const uint8_t *data, uint64_t len, uint32_t k, uint32_t sample_bits,
                             uint64_t *out, uint64_t cap);

/* Pre-pass statistics over the first `sample_limit` bytes of one file:
 * root-prefix histogram (top 8 bits of each canonical k-mer) and the sum and
 * count of quality bytes of complete quality lines. */
void kco_prepass(const uint8_t *data, uint64_t len, uint32_t k,
                 uint64_t sample_limit, uint32_t *prefix_counts /*256*/,
                 uint64_t *qual_sum, uint64_t *qual_count);

/* ---- counting ------------------------------------------------------------ */

/* Sorts keys in place (internal u64 order) and run-length encodes them.
 * Returns the number of distinct keys written to ukeys/counts. */
uint64_t kco_count_sorted(uint64_t *keys, uint64_t n, uint64_t *ukeys,
                          uint32_t *counts);

/* Sorts (key, count) records by printed-string order (dump_tool --sort). */
void kco_sort_records_string_order(uint64_t *keys, uint32_t *counts, uint64_t n,
                                   uint32_t k);

/* Printed-string order key: standard 2-bit packing, first base most
 * significant (dump_tool.cpp:346-354 make_sort_key for N == 1). */
uint64_t kco_string_key(uint64_t key, uint32_t k);

/* Text of a k-mer (dump_tool.cpp:103-124 kmer_to_buf), N words generic. */
void kco_kmer_to_string(const uint64_t *words, uint32_t k, char *out);

/* Histogram of counts over [lo, hi]: hist[c - lo] += 1. */
void kco_histogram(const uint32_t *counts, uint64_t n, uint32_t lo, uint32_t hi,
                   int64_t *hist);

/* ---- hashes (8-byte kmer<1> input) --------------------------------------- */

void kco_xxh3_128_8(uint64_t w, uint64_t *lo, uint64_t *hi);
uint64_t kco_xxh3_64_8(uint64_t w);
uint64_t kco_rapidhash_8(uint64_t w);
uint64_t kco_komihash_8(uint64_t w);
uint64_t kco_mix_hash(uint64_t h1, uint64_t h2);
uint64_t kco_concurrent_map_hash(uint64_t w);

/* ---- Bloom singleton filter ---------------------------------------------- */

void kco_bloom_probe(uint64_t w, uint64_t capacity, uint64_t *block,
                     uint64_t *mask);

/* Sequential classification of an occurrence stream against per-root-prefix
 * filters: out[i] = 0 FIRST, 1 SECOND, 2 THIRD_PLUS. */
void kco_bloom_classify(const uint64_t *keys, uint64_t n,
                        const uint64_t *caps /*256*/, uint8_t *out);

/* Reference sizing of the per-prefix filters.  prefix_counts are the raw
 * pre-pass counts (the <1000 clamp is applied here). */
void kco_bloom_capacities(const uint32_t *prefix_counts, uint8_t avg_quality,
                          uint64_t est_file_size, uint64_t memory_gb, uint32_t k,
                          uint64_t *caps_out /*256*/, uint64_t *max_cap_out);

/* ---- reference file formats (generic N words) ---------------------------- */

uint32_t kco_packed_kmer_bytes(uint32_t k);
uint32_t kco_count_bytes(uint32_t count_max);
void kco_pack_kmer(const uint64_t *words, uint32_t k, uint8_t *out);
void kco_unpack_kmer(const uint8_t *in, uint32_t k, uint32_t n_words,
                     uint64_t *words);

/* ---- tool-side precise merge (generic N words) --------------------------- */

/* histogram_tool precise: high records (key words, counts) + low keys ->
 * hist[max - min + 1].  Returns 0, or -1 when high is empty (the tool exits). */
int kco_tool_precise_histogram(const uint64_t *high_words, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_words,
                               uint64_t n_low, uint32_t n_words, uint32_t count_max,
                               uint32_t min_freq, uint32_t max_freq, int64_t *hist);

/* Only the low-frequency query phase (LowFrequencyQueryThreadPool): the deltas
 * applied to hist for each low key against a sealed map of high records. */
void kco_tool_low_query_deltas(const uint64_t *high_words, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_words,
                               uint64_t n_low, uint32_t n_words, uint32_t count_max,
                               uint32_t min_freq, uint32_t max_freq, int64_t *hist);

/* dump_tool precise --sort merge for N == 1, including the reference's
 * min_freq handling.  Writes merged records sorted by string order; returns
 * their number (out arrays sized n_high + n_low). */
uint64_t kco_tool_precise_dump(const uint64_t *high_keys, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_keys,
                               uint64_t n_low, uint32_t k, uint32_t count_max,
                               uint32_t min_freq, uint32_t max_freq,
                               uint64_t *out_keys, uint32_t *out_counts);

#ifdef __cplusplus
}
#endif

#endif
