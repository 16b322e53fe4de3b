/*
 * kc_oracle.c -- CPU restatement of the reference k-mer counting path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py; never by the
 * product.  Plain C, single threaded, written for clarity over speed.
 *
 * Reference citations are file:line within ScorchShana/KTCounterMemoryGreedy.
 * Third-party hashes (xxHash 0.8.3, rapidhash V3, komihash 5.29, all vendored
 * in the reference under include/) are restated from their published
 * algorithms for the 8-byte input that kmer<1> produces.
 */
#include "kc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* small helpers                                                            */
/* ------------------------------------------------------------------------ */

typedef unsigned __int128 u128;

static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

static inline void mul128(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi)
{
    u128 r = (u128)a * (u128)b;
    *lo = (uint64_t)r;
    *hi = (uint64_t)(r >> 64);
}

static inline uint64_t bit_ceil64(uint64_t x)
{
    if (x <= 1) return 1;
    return 1ULL << (64 - __builtin_clzll(x - 1));
}

/* GetKmer.h:22-37: A/a->0, C/c->1, G/g->2, T/t/U/u->3, everything else invalid. */
static inline int base_code(uint8_t c)
{
    switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': case 'U': case 'u': return 3;
    default: return -1;
    }
}

/* Rolling state of GetKmer<1> (GetKmer.h:58-84, batch form :86-130). */
typedef struct {
    uint32_t k;
    uint64_t back_mask;   /* top 2k bits (GetKmer.h:41-44) */
    uint32_t rev_shift;   /* 2*(32 - k%32) (GetKmer.h:43) */
    uint64_t seq, rev, have;
} roll_t;

static void roll_init(roll_t *r, uint32_t k)
{
    r->k = k;
    if (k % 32 != 0) {
        uint32_t rem = k % 32;
        r->back_mask = ((1ULL << (2 * rem)) - 1ULL) << (64 - 2 * rem);
        r->rev_shift = 2 * (32 - rem);
    } else {
        r->back_mask = ~0ULL;
        r->rev_shift = 0;
    }
    r->seq = r->rev = r->have = 0;
}

static inline void roll_clear(roll_t *r) { r->seq = r->rev = r->have = 0; }

/* One byte through GetKmer::get_next_one.  Returns 1 and sets *canon when a
 * full k-mer ends at this byte. */
static inline int roll_push(roll_t *r, uint8_t c, uint64_t *canon)
{
    int code = base_code(c);
    r->have++;
    if (code < 0) { roll_clear(r); return 0; }
    r->seq = ((r->seq >> 2) | ((uint64_t)code << 62)) & r->back_mask;
    r->rev = (r->rev << 2) | ((uint64_t)(code ^ 3) << r->rev_shift);
    if (r->have >= r->k) {
        /* canonicalize: the smaller word (GetKmer.h:181-206) */
        *canon = r->seq < r->rev ? r->seq : r->rev;
        return 1;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* extraction                                                               */
/* ------------------------------------------------------------------------ */

/*
 * FASTQ record splitting follows ReaderThreadPool::reader_worker
 * (FastqReader.h:559-698): a pure 4-line state machine over '\n'
 * (advance_state :478-487).  Only lines 1, 5, 9, ... (the sequence lines) are
 * parsed; each is parsed from a cleared state because the reader appends '\n'
 * after it (:690-693) and '\n' is an invalid base.  Block splitting with the
 * k-1 overlap (:542-557) makes every window of k consecutive valid bases of a
 * sequence line appear exactly once, which is what this loop emits.
 */
uint64_t kco_extract(const uint8_t *data, uint64_t len, uint32_t k,
                     uint64_t *out, uint64_t cap)
{
    roll_t r;
    roll_init(&r, k);
    uint64_t line = 0, n = 0;
    for (uint64_t i = 0; i < len; ++i) {
        uint8_t c = data[i];
        if (c == '\n') { line++; roll_clear(&r); continue; }
        if ((line & 3) != 1) continue;
        uint64_t canon;
        if (roll_push(&r, c, &canon)) {
            if (n < cap) out[n] = canon;
            n++;
        }
    }
    return n;
}

/*
 * k-mers of 33..128 bases (kmer<2> for k <= 64, kmer<4> for k <= 128).  The
 * rolling state restates GetKmer<N> (GetKmer.h:58-84, batch form :86-130) on
 * N words: seq shifts right by one base across the words (kmer.h:102-118,
 * data[i] takes data[i-1]'s low bits) and takes the new base at data[0]'s top,
 * then data[last] is masked to its top 2*(k%32) bits (all of it when k%32 ==
 * 0); rev shifts left across the words (kmer.h:59-75) and takes the
 * complement at data[last] bit 2*(32 - k%32) (0 when k%32 == 0).  The
 * canonical k-mer is the lexicographically smaller word array
 * (GetKmer.h:181-206, kmer.h:21 defaulted <=>).
 *
 * One deviation, on purpose: words above data[last] (data[3] when k <= 96 in
 * kmer<4>) are zero here.  In GetKmer<4> at k = 96 (last = 2, k%32 = 0, so
 * data[2] is not masked) the seq shift carries bases that left the window into
 * data[3], which nothing clears, so the same 96-mer gets different keys in
 * different reads and its count is split.  Exact counts are what the path
 * defines, so the words outside the k-mer stay zero.
 */
static inline uint32_t wide_words(uint32_t k) { return k <= 32 ? 1u : (k <= 64 ? 2u : 4u); }

uint32_t kco_key_words(uint32_t k) { return wide_words(k); }

typedef struct {
    uint32_t k, nw, last;
    uint64_t back_mask;
    uint32_t rev_shift;
    uint64_t seq[4], rev[4], have;
} wroll_t;

static void wroll_clear(wroll_t *r)
{
    memset(r->seq, 0, sizeof(r->seq));
    memset(r->rev, 0, sizeof(r->rev));
    r->have = 0;
}

static void wroll_init(wroll_t *r, uint32_t k)
{
    r->k = k;
    r->nw = wide_words(k);
    r->last = (k - 1) / 32;
    const uint32_t rem = k % 32;
    r->back_mask = rem ? ((1ULL << (2 * rem)) - 1ULL) << (64 - 2 * rem) : ~0ULL;
    r->rev_shift = rem ? 2 * (32 - rem) : 0;
    wroll_clear(r);
}

static inline int wroll_push(wroll_t *r, uint8_t c, uint64_t *canon)
{
    const int code = base_code(c);
    r->have++;
    if (code < 0) { wroll_clear(r); return 0; }
    for (int i = (int)r->nw - 1; i > 0; --i) r->seq[i] = (r->seq[i] >> 2) | (r->seq[i - 1] << 62);
    r->seq[0] = (r->seq[0] >> 2) | ((uint64_t)code << 62);
    r->seq[r->last] &= r->back_mask;
    for (uint32_t i = r->last + 1; i < r->nw; ++i) r->seq[i] = 0;   /* the deviation above */
    for (uint32_t i = 0; i + 1 < r->nw; ++i) r->rev[i] = (r->rev[i] << 2) | (r->rev[i + 1] >> 62);
    r->rev[r->nw - 1] <<= 2;
    r->rev[r->last] |= (uint64_t)(code ^ 3) << r->rev_shift;
    if (r->have < r->k) return 0;
    int less = 0;
    for (uint32_t i = 0; i < r->nw; ++i)
        if (r->seq[i] != r->rev[i]) { less = r->seq[i] < r->rev[i]; break; }
    memcpy(canon, less ? r->seq : r->rev, r->nw * 8);
    return 1;
}

uint64_t kco_extract_wide(const uint8_t *data, uint64_t len, uint32_t k, uint64_t *out, uint64_t cap)
{
    wroll_t r;
    wroll_init(&r, k);
    const uint32_t nw = r.nw;
    uint64_t line = 0, n = 0, canon[4];
    for (uint64_t i = 0; i < len; ++i) {
        const uint8_t c = data[i];
        if (c == '\n') { line++; wroll_clear(&r); continue; }
        if ((line & 3) != 1) continue;
        if (wroll_push(&r, c, canon)) {
            if (n < cap) memcpy(out + n * nw, canon, nw * 8);
            n++;
        }
    }
    return n;
}

/* Spot-check sample of N-word k-mers: the sample hash folded over the
 * words (data[0] first); every occurrence of a kept k-mer is kept. */
uint64_t kco_sample_hash_wide(const uint64_t *words, uint32_t n_words)
{
    uint64_t h = kco_sample_hash(words[0]);
    for (uint32_t i = 1; i < n_words; ++i) h = kco_sample_hash(h ^ words[i]);
    return h;
}

uint64_t kco_extract_wide_sampled(const uint8_t *data, uint64_t len, uint32_t k, uint32_t sample_bits,
                                  uint64_t *out, uint64_t cap)
{
    const uint64_t smask = sample_bits >= 64 ? ~0ULL : ((1ULL << sample_bits) - 1ULL);
    wroll_t r;
    wroll_init(&r, k);
    const uint32_t nw = r.nw;
    uint64_t line = 0, n = 0, canon[4];
    for (uint64_t i = 0; i < len; ++i) {
        const uint8_t c = data[i];
        if (c == '\n') { line++; wroll_clear(&r); continue; }
        if ((line & 3) != 1) continue;
        if (wroll_push(&r, c, canon) && (kco_sample_hash_wide(canon, nw) & smask) == 0) {
            if (n < cap) memcpy(out + n * nw, canon, nw * 8);
            n++;
        }
    }
    return n;
}

/* Printed-string order key of an N-word k-mer: the 2-bit groups of the whole
 * word array reversed (the first base most significant), as N words, most
 * significant first.  Base i of the printed string is extracted as
 * kmer_to_buf does (dump_tool.cpp:103-124). */
void kco_string_key_wide(const uint64_t *words, uint32_t k, uint64_t *out)
{
    const uint32_t nw = wide_words(k), full = k / 32, tail = k % 32;
    memset(out, 0, nw * 8);
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t w, sh;
        if (tail > 0 && i < tail) { w = full; sh = 64 - 2 * tail + 2 * i; }
        else {
            const uint32_t off = i - (tail > 0 ? tail : 0);
            w = full - 1 - off / 32;
            sh = 2 * (off % 32);
        }
        const uint64_t b = (words[w] >> sh) & 3ULL;
        const uint32_t pos = k - 1 - i;   /* 2-bit group from the least significant end */
        out[nw - 1 - pos / 32] |= b << (2 * (pos % 32));
    }
}

/*
 * Spot-check sample of the occurrences of one file: the same record splitting
 * and extraction as kco_extract, keeping only the canonical k-mers whose
 * sample hash has its low `sample_bits` bits zero.  The sample hash is the
 * splitmix64 finaliser, unrelated to every hash on the counting path (Bloom
 * block, table slots, buckets), so the kept k-mers fall in every bucket and
 * filter slice, and every occurrence of a kept k-mer is kept: their exact
 * counts are the full job's counts of those k-mers.
 */
uint64_t kco_sample_hash(uint64_t w)
{
    w ^= w >> 30;
    w *= 0xbf58476d1ce4e5b9ULL;
    w ^= w >> 27;
    w *= 0x94d049bb133111ebULL;
    return w ^ (w >> 31);
}

uint64_t kco_extract_sampled(const uint8_t *data, uint64_t len, uint32_t k, uint32_t sample_bits,
                             uint64_t *out, uint64_t cap)
{
    const uint64_t smask = sample_bits >= 64 ? ~0ULL : ((1ULL << sample_bits) - 1ULL);
    roll_t r;
    roll_init(&r, k);
    uint64_t line = 0, n = 0;
    for (uint64_t i = 0; i < len; ++i) {
        uint8_t c = data[i];
        if (c == '\n') { line++; roll_clear(&r); continue; }
        if ((line & 3) != 1) continue;
        uint64_t canon;
        if (roll_push(&r, c, &canon) && (kco_sample_hash(canon) & smask) == 0) {
            if (n < cap) out[n] = canon;
            n++;
        }
    }
    return n;
}

/*
 * Pre-pass (FastqPreReader::pre_read :98-136, parse_loop :218-288,
 * FastqPrefixCounter::process_block :124-132).  The reader pulls 2 MiB chunks
 * until the limit is reached.  A quality line is summed only from the start of
 * the chunk holding its '\n' (memchr per chunk, :247-256); sequence bytes are
 * parsed across chunks, including a final line cut by the sample limit.
 */
void kco_prepass(const uint8_t *data, uint64_t len, uint32_t k,
                 uint64_t sample_limit, uint32_t *prefix_counts,
                 uint64_t *qual_sum, uint64_t *qual_count)
{
    const uint64_t chunk = 2ULL * 1024 * 1024;   /* FASTQ_FILE_CHUNK_SIZE */
    uint64_t end = len < sample_limit ? len : sample_limit;
    roll_t r;
    roll_init(&r, k);
    uint64_t line = 0, line_start = 0;
    for (uint64_t i = 0; i < end; ++i) {
        uint8_t c = data[i];
        if (c == '\n') {
            if ((line & 3) == 3) {
                uint64_t from = (i / chunk) * chunk;
                if (from < line_start) from = line_start;
                for (uint64_t j = from; j < i; ++j)
                    *qual_sum += (uint64_t)(int64_t)(signed char)data[j];
                *qual_count += i - from;
            }
            line++;
            line_start = i + 1;
            roll_clear(&r);
            continue;
        }
        if ((line & 3) != 1) continue;
        uint64_t canon;
        if (roll_push(&r, c, &canon)) prefix_counts[canon >> 56]++;
    }
}

/* ------------------------------------------------------------------------ */
/* sorting / counting                                                       */
/* ------------------------------------------------------------------------ */

/* LSD radix sort of u64 keys with a u32 payload (11-bit digits). */
static void radix_sort_kv(uint64_t *keys, uint32_t *vals, uint64_t n, uint32_t bits)
{
    if (n <= 1) return;
    uint64_t *tk = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint32_t *tv = vals ? (uint32_t *)malloc(n * sizeof(uint32_t)) : NULL;
    uint64_t *sk = keys, *dk = tk;
    uint32_t *sv = vals, *dv = tv;
    for (uint32_t shift = 0; shift < bits; shift += 11) {
        uint64_t cnt[2048] = {0};
        for (uint64_t i = 0; i < n; ++i) cnt[(sk[i] >> shift) & 2047]++;
        uint64_t sum = 0;
        for (int b = 0; b < 2048; ++b) { uint64_t c = cnt[b]; cnt[b] = sum; sum += c; }
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t p = cnt[(sk[i] >> shift) & 2047]++;
            dk[p] = sk[i];
            if (vals) dv[p] = sv[i];
        }
        uint64_t *t = sk; sk = dk; dk = t;
        uint32_t *u = sv; sv = dv; dv = u;
    }
    if (sk != keys) {
        memcpy(keys, sk, n * sizeof(uint64_t));
        if (vals) memcpy(vals, sv, n * sizeof(uint32_t));
    }
    free(tk);
    free(tv);
}

uint64_t kco_count_sorted(uint64_t *keys, uint64_t n, uint64_t *ukeys, uint32_t *counts)
{
    radix_sort_kv(keys, NULL, n, 64);
    uint64_t u = 0;
    for (uint64_t i = 0; i < n;) {
        uint64_t j = i;
        while (j < n && keys[j] == keys[i]) j++;
        ukeys[u] = keys[i];
        counts[u] = (uint32_t)(j - i);
        u++;
        i = j;
    }
    return u;
}

/*
 * make_sort_key (dump_tool.cpp:346-354) for N == 1: base i of the printed
 * string is read from bit 64 - 2k + 2i (extract_base_at :327-343) and packed
 * first-base-most-significant.  That is a reversal of the 2-bit groups.
 */
uint64_t kco_string_key(uint64_t key, uint32_t k)
{
    uint64_t s = 0;
    for (uint32_t i = 0; i < k; ++i)
        s = (s << 2) | ((key >> (64 - 2 * k + 2 * i)) & 3ULL);
    return s;
}

void kco_sort_records_string_order(uint64_t *keys, uint32_t *counts, uint64_t n, uint32_t k)
{
    uint64_t *sk = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    uint32_t *idx = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; ++i) { sk[i] = kco_string_key(keys[i], k); idx[i] = (uint32_t)i; }
    radix_sort_kv(sk, idx, n, 2 * k);
    uint64_t *ok = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    uint32_t *oc = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; ++i) { ok[i] = keys[idx[i]]; oc[i] = counts[idx[i]]; }
    memcpy(keys, ok, n * sizeof(uint64_t));
    memcpy(counts, oc, n * sizeof(uint32_t));
    free(sk); free(idx); free(ok); free(oc);
}

/* kmer_to_buf (dump_tool.cpp:103-124), N words generic. */
void kco_kmer_to_string(const uint64_t *words, uint32_t k, char *out)
{
    static const char B[4] = {'A', 'C', 'G', 'T'};
    const uint32_t full_words = k / 32, tail = k % 32;
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t w, sh;
        if (tail > 0 && i < tail) { w = full_words; sh = 64 - 2 * tail + 2 * i; }
        else {
            uint32_t off = i - (tail > 0 ? tail : 0);
            w = full_words - 1 - off / 32;
            sh = 2 * (off % 32);
        }
        out[i] = B[(words[w] >> sh) & 3];
    }
    out[k] = 0;
}

void kco_histogram(const uint32_t *counts, uint64_t n, uint32_t lo, uint32_t hi, int64_t *hist)
{
    for (uint64_t i = 0; i < n; ++i)
        if (counts[i] >= lo && counts[i] <= hi) hist[counts[i] - lo]++;
}

/* ------------------------------------------------------------------------ */
/* hashes                                                                   */
/* ------------------------------------------------------------------------ */

/* xxHash 0.8.3 constants (XXH_PRIME64_1, PRIME_MX1/2) and the default-secret
 * words at byte offsets 8, 16 and 24 that the 4..8-byte paths read. */
#define XXP1 0x9E3779B185EBCA87ULL
#define XXMX1 0x165667919E3779F9ULL
#define XXMX2 0x9FB21C651E98DF25ULL
#define XXS8 0x1cad21f72c81017cULL
#define XXS16 0xdb979083e96dd4deULL
#define XXS24 0x1f67b3b7a4a44072ULL

static inline uint64_t xx_avalanche(uint64_t h)
{
    h ^= h >> 37;
    h *= XXMX1;
    h ^= h >> 32;
    return h;
}

/* XXH3_128bits on 8 bytes (XXH3_len_4to8_128b), as called by
 * ConcurrentBloomFilter::prepare_insert (BloomFilter.h:215-222). */
void kco_xxh3_128_8(uint64_t w, uint64_t *lo, uint64_t *hi)
{
    uint64_t keyed = w ^ (XXS16 ^ XXS24);
    uint64_t l, h;
    mul128(keyed, XXP1 + (8ULL << 2), &l, &h);
    h += l << 1;
    l ^= h >> 3;
    l ^= l >> 35;
    l *= XXMX2;
    l ^= l >> 28;
    *lo = l;
    *hi = xx_avalanche(h);
}

/* XXH3_64bits on 8 bytes (XXH3_len_4to8_64b), as called by
 * FlatConcurrentHashMap (tool/FlatConcurrentHashMap.h:95,150). */
uint64_t kco_xxh3_64_8(uint64_t w)
{
    uint64_t in64 = (w >> 32) + ((w & 0xffffffffULL) << 32);
    uint64_t h = in64 ^ (XXS8 ^ XXS16);
    h ^= rotl64(h, 49) ^ rotl64(h, 24);
    h *= XXMX2;
    h ^= (h >> 35) + 8;
    h *= XXMX2;
    return h ^ (h >> 28);
}

/* rapidhash V3 (default secret, seed 0) on 8 bytes; ConcurrentMap.h:144. */
static const uint64_t RAPID_SECRET[8] = {
    0x2d358dccaa6c78a5ULL, 0x8bb84b93962eacc9ULL, 0x4b33a62ed433d4a3ULL, 0x4d5a2da51de1aa47ULL,
    0xa0761d6478bd642fULL, 0xe7037ed1a0b428dbULL, 0x90ed1765281c388cULL, 0xaaaaaaaaaaaaaaaaULL};

static inline uint64_t rapid_mix(uint64_t a, uint64_t b)
{
    uint64_t l, h;
    mul128(a, b, &l, &h);
    return l ^ h;
}

uint64_t kco_rapidhash_8(uint64_t w)
{
    uint64_t seed = rapid_mix(RAPID_SECRET[2], RAPID_SECRET[1]);
    seed ^= 8;
    uint64_t a = w ^ RAPID_SECRET[1], b = w ^ seed;
    uint64_t l, h;
    mul128(a, b, &l, &h);
    return rapid_mix(l ^ RAPID_SECRET[7], h ^ RAPID_SECRET[1] ^ 8);
}

/* komihash 5.29 (seed 0) on 8 bytes; ConcurrentMap.h:143.  Its 128-bit
 * multiply step writes the low half and ADDS the high half into the second
 * operand's state word. */
static inline void komi_m128(uint64_t u, uint64_t v, uint64_t *rl, uint64_t *rha)
{
    uint64_t l, h;
    mul128(u, v, &l, &h);
    *rl = l;
    *rha += h;
}

uint64_t kco_komihash_8(uint64_t w)
{
    uint64_t s1 = 0x243F6A8885A308D3ULL, s5 = 0x452821E638D01377ULL;
    komi_m128(s1, s5, &s1, &s5);   /* hashing round without input */
    s1 ^= s5;
    uint64_t r1h = s1 ^ w;         /* 8 <= len < 12 branch */
    uint64_t r2h = s5 ^ 1ULL;
    komi_m128(r1h, r2h, &s1, &s5); /* finalisation */
    s1 ^= s5;
    komi_m128(s1, s5, &s1, &s5);
    s1 ^= s5;
    return s1;
}

/* mix_hash (HashFunction.h:28-37). */
uint64_t kco_mix_hash(uint64_t h1, uint64_t h2)
{
    const uint64_t K = 0x9ddfea08eb382d69ULL;
    uint64_t a = (h1 ^ h2) * K;
    a ^= a >> 47;
    uint64_t b = (h2 ^ a) * K;
    b ^= b >> 47;
    b *= K;
    return b;
}

/* ConcurrentMap::hash_func (ConcurrentMap.h:141-148). */
uint64_t kco_concurrent_map_hash(uint64_t w)
{
    return kco_mix_hash(kco_komihash_8(w), kco_rapidhash_8(w));
}

/* ------------------------------------------------------------------------ */
/* Bloom filter                                                             */
/* ------------------------------------------------------------------------ */

/* prepare_insert + calculate_insert_num (BloomFilter.h:215-222, :287-296). */
void kco_bloom_probe(uint64_t w, uint64_t capacity, uint64_t *block, uint64_t *mask)
{
    uint64_t lo, hi;
    kco_xxh3_128_8(w, &lo, &hi);
    uint64_t h2 = hi | 1ULL, m = 0;
    for (uint64_t i = 0; i < 3; ++i) m |= 1ULL << ((lo + i * h2) & 63);
    *block = lo & (capacity - 1);
    *mask = m;
}

/* insert_prepared (BloomFilter.h:233-273) run sequentially. */
void kco_bloom_classify(const uint64_t *keys, uint64_t n, const uint64_t *caps, uint8_t *out)
{
    uint64_t *bins[256];
    for (int p = 0; p < 256; ++p) bins[p] = (uint64_t *)calloc(2 * caps[p], sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t w = keys[i], b, m;
        int p = (int)(w >> 56);
        kco_bloom_probe(w, caps[p], &b, &m);
        uint64_t *cell = bins[p] + 2 * b;
        if ((cell[0] & m) == m) { out[i] = 2; continue; }
        if ((cell[1] & m) == m) { cell[0] |= m; out[i] = 1; continue; }
        cell[1] |= m;
        out[i] = 0;
    }
    for (int p = 0; p < 256; ++p) free(bins[p]);
}

/*
 * Filter sizing: get_MAX_BLOOM_FILTER_CAPACITY (main.cpp:41-52),
 * get_estimated_total_kmer (:54-57), calculate_bloom_filter_capacity
 * (:111-153), with the pre-pass clamp of small prefix counts to 1000
 * (main.cpp:306-315).  Same double expressions in the same order.
 */
void kco_bloom_capacities(const uint32_t *prefix_counts, uint8_t avg_quality,
                          uint64_t est_file_size, uint64_t memory_gb, uint32_t k,
                          uint64_t *caps_out, uint64_t *max_cap_out)
{
    const uint64_t MIN_CAP = 1ULL << 12;
    const double error_rate = pow(10.0, -((int)avg_quality - 33) * 0.1);
    const uint64_t quarter = memory_gb * 1024ULL * 1024ULL * 1024ULL / 4 / sizeof(uint64_t) / 256;
    const double singleton = 1.0 - pow(1.0 - error_rate, (double)k);
    const double error_factor = 0.5 + singleton;
    uint64_t corrected = bit_ceil64((uint64_t)((double)quarter * error_factor));
    uint64_t max_cap = corrected > MIN_CAP ? corrected : MIN_CAP;

    const double cap_factor = (0.5 + singleton) < 1.0 ? (0.5 + singleton) : 1.0;
    const uint64_t est_total = est_file_size * 30 / 3 / (k > 31 ? k : 31);
    uint64_t clamped[256], total = 0;
    for (int i = 0; i < 256; ++i) {
        clamped[i] = prefix_counts[i] < 1000 ? 1000 : prefix_counts[i];
        total += clamped[i];
    }
    for (int i = 0; i < 256; ++i) {
        double ratio = (double)clamped[i] / (double)total;
        uint64_t est = (uint64_t)((double)est_total * ratio * 4.81 * cap_factor / 64);
        uint64_t c = bit_ceil64(est);
        if (c < MIN_CAP) c = MIN_CAP;
        if (c > max_cap) c = max_cap;
        caps_out[i] = c;
    }
    *max_cap_out = max_cap;
}

/* ------------------------------------------------------------------------ */
/* file formats                                                             */
/* ------------------------------------------------------------------------ */

/* Record layout of FinalDrainWriter (:43-50, :71-88) / ExportWriter (:296-313). */
uint32_t kco_packed_kmer_bytes(uint32_t k)
{
    return (k / 32) * 8 + (2 * (k % 32) + 7) / 8;
}

/* main.cpp:599-615 */
uint32_t kco_count_bytes(uint32_t count_max)
{
    if (count_max <= 0xFF) return 1;
    if (count_max <= 0xFFFF) return 2;
    if (count_max <= 0xFFFFFF) return 3;
    return 4;
}

void kco_pack_kmer(const uint64_t *words, uint32_t k, uint8_t *out)
{
    const uint32_t full = k / 32, tail_bits = 2 * (k % 32), tail_bytes = (tail_bits + 7) / 8;
    memcpy(out, words, full * 8);
    if (tail_bytes > 0) {
        uint64_t mask = (~0ULL) << (64 - tail_bits);
        uint64_t t = words[full] & mask;
        memcpy(out + full * 8, (const uint8_t *)&t + (8 - tail_bytes), tail_bytes);
    }
}

/* ExportReader / FinalDrainReader unpack (dump_tool.cpp:868-882). */
void kco_unpack_kmer(const uint8_t *in, uint32_t k, uint32_t n_words, uint64_t *words)
{
    const uint32_t full = k / 32, tail_bytes = (2 * (k % 32) + 7) / 8;
    memset(words, 0, n_words * 8);
    memcpy(words, in, full * 8);
    if (tail_bytes > 0) {
        uint64_t t = 0;
        memcpy((uint8_t *)&t + (8 - tail_bytes), in + full * 8, tail_bytes);
        words[full] = t;
    }
}

/* ------------------------------------------------------------------------ */
/* tool-side merge                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    const uint64_t *words;
    uint32_t n;
} keyview_t;

static uint32_t g_cmp_words;

static int cmp_words(const void *a, const void *b)
{
    const uint64_t *x = *(const uint64_t *const *)a, *y = *(const uint64_t *const *)b;
    for (uint32_t i = 0; i < g_cmp_words; ++i) {
        if (x[i] < y[i]) return -1;
        if (x[i] > y[i]) return 1;
    }
    return 0;
}

typedef struct {
    const uint64_t **keys;   /* sorted pointers into the caller's arrays */
    uint32_t *counts;        /* mutable copy, indexed like keys */
    uint64_t n;
    uint32_t nw;
} smap_t;

static void smap_build(smap_t *m, const uint64_t *words, const uint32_t *counts, uint64_t n,
                       uint32_t nw, const uint8_t *keep)
{
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < n; ++i) if (!keep || keep[i]) cnt++;
    const uint64_t **ptrs = (const uint64_t **)malloc((cnt ? cnt : 1) * sizeof(uint64_t *));
    uint64_t j = 0;
    for (uint64_t i = 0; i < n; ++i) if (!keep || keep[i]) ptrs[j++] = words + i * nw;
    g_cmp_words = nw;
    qsort(ptrs, cnt, sizeof(uint64_t *), cmp_words);
    m->keys = ptrs;
    m->n = cnt;
    m->nw = nw;
    m->counts = (uint32_t *)malloc((cnt ? cnt : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < cnt; ++i) m->counts[i] = counts[(ptrs[i] - words) / nw];
}

static int64_t smap_find(const smap_t *m, const uint64_t *key)
{
    uint64_t lo = 0, hi = m->n;
    g_cmp_words = m->nw;
    while (lo < hi) {
        uint64_t mid = (lo + hi) / 2;
        const uint64_t *kp = key;
        int c = cmp_words(&m->keys[mid], &kp);
        if (c == 0) return (int64_t)mid;
        if (c < 0) lo = mid + 1; else hi = mid;
    }
    return -1;
}

static void smap_free(smap_t *m) { free(m->keys); free(m->counts); }

static inline int in_range(uint64_t v, uint32_t lo, uint32_t hi) { return v >= lo && v <= hi; }

/* LowFrequencyQueryThreadPool::process_block (:186-240). */
static void low_phase(const smap_t *m, const uint64_t *low_words, uint64_t n_low, uint32_t nw,
                      uint32_t count_max, uint32_t min_freq, uint32_t max_freq, int64_t *hist)
{
    for (uint64_t i = 0; i < n_low; ++i) {
        int64_t s = smap_find(m, low_words + i * nw);
        if (s >= 0) {
            uint32_t c = m->counts[s];
            if (in_range(c, min_freq, max_freq)) hist[c - min_freq] -= 1;
            uint64_t merged = (uint64_t)c + 1;
            if (merged > count_max) merged = count_max;
            if (in_range(merged, min_freq, max_freq)) hist[merged - min_freq] += 1;
        } else if (in_range(1, min_freq, max_freq)) {
            hist[1 - min_freq] += 1;
        }
    }
}

void kco_tool_low_query_deltas(const uint64_t *high_words, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_words, uint64_t n_low,
                               uint32_t n_words, uint32_t count_max, uint32_t min_freq,
                               uint32_t max_freq, int64_t *hist)
{
    smap_t m;
    smap_build(&m, high_words, high_counts, n_high, n_words, NULL);
    low_phase(&m, low_words, n_low, n_words, count_max, min_freq, max_freq, hist);
    smap_free(&m);
}

/* run_precise_histogram_tool_impl (histogram_tool.cpp:735-791) with
 * HighFrequencyInsertThreadPool::process_block (:150-177). */
int kco_tool_precise_histogram(const uint64_t *high_words, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_words, uint64_t n_low,
                               uint32_t n_words, uint32_t count_max, uint32_t min_freq,
                               uint32_t max_freq, int64_t *hist)
{
    if (n_high == 0) return -1; /* "empty high.bin file" (:296-300) */
    uint8_t *keep = (uint8_t *)calloc(n_high, 1);
    for (uint64_t i = 0; i < n_high; ++i) {
        uint32_t c = high_counts[i];
        if ((uint64_t)c + 1 < min_freq) continue;
        if (in_range(c, min_freq, max_freq)) hist[c - min_freq] += 1;
        keep[i] = 1;
    }
    smap_t m;
    smap_build(&m, high_words, high_counts, n_high, n_words, keep);
    low_phase(&m, low_words, n_low, n_words, count_max, min_freq, max_freq, hist);
    smap_free(&m);
    free(keep);
    return 0;
}

/* run_precise_impl --sort (dump_tool.cpp:1202-1272): build_hash_map (:682-733,
 * keeps only count in [min,max]), process_low_freq_collect (:824-926),
 * collect_remaining_into_vector (:928-936), sort_and_write (:1138-1198). */
uint64_t kco_tool_precise_dump(const uint64_t *high_keys, const uint32_t *high_counts,
                               uint64_t n_high, const uint64_t *low_keys, uint64_t n_low,
                               uint32_t k, uint32_t count_max, uint32_t min_freq,
                               uint32_t max_freq, uint64_t *out_keys, uint32_t *out_counts)
{
    uint8_t *keep = (uint8_t *)calloc(n_high ? n_high : 1, 1);
    for (uint64_t i = 0; i < n_high; ++i) keep[i] = in_range(high_counts[i], min_freq, max_freq);
    smap_t m;
    smap_build(&m, high_keys, high_counts, n_high, 1, keep);
    uint64_t n = 0;
    for (uint64_t i = 0; i < n_low; ++i) {
        int64_t s = smap_find(&m, &low_keys[i]);
        if (s >= 0) {
            uint64_t merged = (uint64_t)m.counts[s] + 1;
            if (merged > count_max) merged = count_max;
            if (in_range(merged, min_freq, max_freq)) { out_keys[n] = low_keys[i]; out_counts[n] = (uint32_t)merged; n++; }
            m.counts[s] = 0;
        } else if (in_range(1, min_freq, max_freq)) {
            out_keys[n] = low_keys[i]; out_counts[n] = 1; n++;
        }
    }
    for (uint64_t i = 0; i < m.n; ++i) {
        if (m.counts[i] > 0 && in_range(m.counts[i], min_freq, max_freq)) {
            out_keys[n] = m.keys[i][0]; out_counts[n] = m.counts[i]; n++;
        }
    }
    smap_free(&m);
    free(keep);
    kco_sort_records_string_order(out_keys, out_counts, n, k);
    return n;
}
