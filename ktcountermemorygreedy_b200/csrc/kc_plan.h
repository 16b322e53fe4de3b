// kc_plan.h -- the reference's Bloom filter sizing, evaluated on the host.
//
// get_MAX_BLOOM_FILTER_CAPACITY (src/main.cpp:41-52), get_estimated_total_kmer
// (:54-57) and calculate_bloom_filter_capacity (:111-153), applied to the
// pre-pass root-prefix counts after the reference's clamp of counts below 1000
// (:306-315).  The double expressions keep the reference's operand order so
// that every capacity (a power of two) comes out identical, which is what
// makes each Bloom probe pick the same block.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace kc {

struct BloomPlan {
    uint64_t caps[256];
    uint64_t max_cap;
};

inline uint64_t plan_bit_ceil(uint64_t x)
{
    if (x <= 1) return 1;
    return 1ULL << (64 - __builtin_clzll(x - 1));
}

inline BloomPlan bloom_plan(const uint32_t *raw_prefix_counts, uint8_t avg_quality, uint64_t est_file_size,
                            uint64_t memory_gb, uint32_t k)
{
    BloomPlan p{};
    const uint64_t MIN_CAP = 1ULL << 12;
    const double error_rate = std::pow(10.0, -((int)avg_quality - 33) * 0.1);
    const uint64_t quarter = memory_gb * 1024ULL * 1024ULL * 1024ULL / 4 / sizeof(uint64_t) / 256;
    const double singleton = 1.0 - std::pow(1.0 - error_rate, (double)k);
    const double error_factor = 0.5 + singleton;
    const uint64_t corrected = plan_bit_ceil((uint64_t)((double)quarter * error_factor));
    p.max_cap = std::max<uint64_t>(MIN_CAP, corrected);

    const double cap_factor = std::min(0.5 + singleton, 1.0);
    const uint64_t est_total = est_file_size * 30 / 3 / std::max<uint32_t>(k, 31u);
    uint64_t clamped[256], total = 0;
    for (int i = 0; i < 256; ++i) {
        clamped[i] = raw_prefix_counts[i] < 1000 ? 1000 : raw_prefix_counts[i];
        total += clamped[i];
    }
    for (int i = 0; i < 256; ++i) {
        const double ratio = (double)clamped[i] / (double)total;
        const uint64_t est = (uint64_t)((double)est_total * ratio * 4.81 * cap_factor / 64);
        uint64_t c = std::max(plan_bit_ceil(est), MIN_CAP);
        p.caps[i] = std::min(c, p.max_cap);
    }
    return p;
}

}  // namespace kc
