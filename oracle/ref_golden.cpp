// ref_golden.cpp -- golden-vector generator built from the reference's own
// sources.  TEST INFRASTRUCTURE ONLY: oracle/Makefile compiles it against the
// reference tree (REF=...) into oracle/_ref/ref_golden, and
// tests/golden/make_golden.py runs it to produce the committed fixtures.  No
// reference code is copied: the reference's main.cpp is compiled in place with
// its entry point renamed, and this driver calls the reference's own classes
// and functions.
//
//   ref_golden hashes <n> <seed>          per key: w xxh128.lo xxh128.hi xxh64
//                                         rapidhash komihash mix_hash
//                                         bloom_block(cap 2^20) bloom_mask
//   ref_golden getkmer <k> <bases>        canonical k-mer (all words of kmer<N>)
//                                         after each base that completes one
//                                         (GetKmer<N>::get_next_one, N by k)
//   ref_golden prepass <k> <mem_gb> <f>.. root-prefix counts, avgQuality,
//                                         estimated size, Bloom capacities
#define main kc_reference_counter_main
#include "src/main.cpp"
#undef main

#include <cinttypes>
#include <cstdio>

static uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static int run_hashes(uint64_t n, uint64_t seed)
{
    BloomFilter<1> bf(1ULL << 20);
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t w = splitmix(s);
        // every third key is a realistic k=31 word (low two bits clear)
        if (i % 3 == 1) w &= ~3ULL;
        if (i == 0) w = 0;
        if (i == 1) w = ~0ULL;
        kmer<1> km;
        km.data[0] = w;
        XXH128_hash_t h128 = XXH3_128bits(&km, sizeof(km));
        uint64_t h64 = XXH3_64bits(&km, sizeof(km));
        uint64_t r = rapidhash(&km, sizeof(km));
        uint64_t ko = komihash(&km, sizeof(km), 0);
        uint64_t mh = mix_hash(ko, r);
        auto probe = bf.prepare_insert(km);
        std::printf("%016" PRIx64 " %016" PRIx64 " %016" PRIx64 " %016" PRIx64 " %016" PRIx64
                    " %016" PRIx64 " %016" PRIx64 " %" PRIu64 " %016" PRIx64 "\n",
                    w, (uint64_t)h128.low64, (uint64_t)h128.high64, h64, r, ko, mh,
                    probe.block_idx, probe.insert_num);
    }
    return 0;
}

// GetKmer<N> for the reference's dispatch (main.cpp:617-633): N = 1 for
// k <= 32, 2 for k <= 64, 4 for k <= 128.  Prints every word of the canonical
// kmer<N> after each base that completes one.
template <uint32_t N>
static int run_getkmer_n(uint32_t k, const char *bases)
{
    GetKmer<N> g(k);
    for (const char *p = bases; *p; ++p) {
        if (g.get_next_one(static_cast<unsigned char>(*p))) {
            std::printf("%zu", static_cast<size_t>(p - bases));
            for (uint32_t w = 0; w < N; ++w) std::printf(" %016" PRIx64, g.canonical_kmer.data[w]);
            std::printf("\n");
        }
    }
    return 0;
}

static int run_getkmer(uint32_t k, const char *bases)
{
    if (k <= 32) return run_getkmer_n<1>(k, bases);
    if (k <= 64) return run_getkmer_n<2>(k, bases);
    return run_getkmer_n<4>(k, bases);
}

// Mirrors the pre-pass section of process_main<1> (main.cpp:262-335) by
// calling the same reference classes, then the reference's sizing functions.
static int run_prepass(int argc, char **argv)
{
    k_len = static_cast<uint32_t>(std::stoul(argv[2]));
    memory_limit = std::stoull(argv[3]);
    n_thread = 8;
    for (int i = 4; i < argc; ++i) filenames.push_back(argv[i]);

    auto reader_parser_ring_pool = std::make_shared<RingMemoryPool<READER_PARSER_RING_MEMORY_POOL_CAPACITY>>(READER_PARSER_RING_MEMORY_POOL_BLOCK_SIZE, 1);
    auto parser_classifier_ring_pool = std::make_shared<RingMemoryPool<PARSER_CLASSIFIER_RING_MEMORY_POOL_CAPACITY>>(PARSER_CLASSIFIER_RING_MEMORY_POOL_BLOCK_SIZE, 1);
    FastqPreReader<1> pre_reader(filenames, k_len, FASTQ_FILE_CHUNK_SIZE, reader_parser_ring_pool.get());
    estimated_file_size = pre_reader.get_estimated_raw_fastq_file_size();
    auto pre_parser_thread = std::thread([&] {
        FastqPreParser<1> parser(k_len, reader_parser_ring_pool.get(), parser_classifier_ring_pool.get());
        parser.parse_and_push();
        parser_classifier_ring_pool->producer_set_finished();
    });
    std::vector<std::atomic<uint32_t>> prefix_counts(256);
    for (auto &v : prefix_counts) v.store(0);
    std::vector<std::thread> counters;
    for (int t = 0; t < 4; ++t) {
        counters.emplace_back([&] {
            FastqPrefixCounter<1> pc(k_len, parser_classifier_ring_pool.get());
            pc.count_prefixes();
            for (size_t j = 0; j < prefix_counts.size(); ++j)
                prefix_counts[j].fetch_add(pc.prefix_counts[j], std::memory_order_relaxed);
        });
    }
    pre_reader.pre_read();
    pre_parser_thread.join();
    for (auto &t : counters) t.join();

    std::printf("raw_prefix_counts");
    for (auto &v : prefix_counts) std::printf(" %u", v.load());
    std::printf("\n");
    for (auto &v : prefix_counts)
        if (v.load() < 1000) v.store(1000);
    get_MAX_BLOOM_FILTER_CAPACITY();
    calculate_bloom_filter_capacity(prefix_counts, estimated_file_size);
    std::printf("avg_quality %u\n", static_cast<unsigned>(avgQuality));
    std::printf("estimated_file_size %" PRIu64 "\n", estimated_file_size);
    std::printf("max_bloom_capacity %" PRIu64 "\n", MAX_BLOOM_FILTER_CAPACITY);
    std::printf("bloom_capacities");
    for (auto c : bloom_filter_capacity) std::printf(" %" PRIu64, c);
    std::printf("\n");
    return 0;
}

int main(int argc, char **argv)
{
    if (argc >= 4 && std::string(argv[1]) == "hashes")
        return run_hashes(std::stoull(argv[2]), std::stoull(argv[3]));
    if (argc >= 4 && std::string(argv[1]) == "getkmer")
        return run_getkmer(static_cast<uint32_t>(std::stoul(argv[2])), argv[3]);
    if (argc >= 5 && std::string(argv[1]) == "prepass")
        return run_prepass(argc, argv);
    std::fprintf(stderr, "usage: ref_golden hashes <n> <seed> | getkmer <k> <bases> | prepass <k> <mem_gb> <files...>\n");
    return 2;
}
