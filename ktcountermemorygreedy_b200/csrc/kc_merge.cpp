// kc_merge.cpp -- the precise merge of the reference tools on the device
// (kc_merge_records in include/kc.h): high.bin records and low.bin k-mers
// become exact counts, then records in printed-string order and a histogram.
#include <algorithm>
#include <cmath>
#include <vector>

#include "kc_host.h"
#include "kc_wide.cuh"

using namespace kc;

namespace {

// k-mers of 33..128 bases: every high.bin record with its count and every
// low.bin k-mer with count 1 into one N-word table (a low k-mer that is also
// in high.bin adds one to its count, as the reference's low-frequency query
// moves it one bin up, tool/histogram_tool.cpp LowFrequencyQueryThreadPool;
// one that is not is a k-mer seen once), then the same compaction, sort and
// histogram as a counting job.
int merge_wide(const uint64_t *high_keys, const uint32_t *high_counts, uint64_t n_high, const uint64_t *low_keys,
               uint64_t n_low, uint32_t k, uint32_t count_max, uint32_t min_count, uint32_t max_count,
               uint32_t hist_min, uint32_t hist_max, uint64_t *out_keys, uint32_t *out_counts, uint64_t out_cap,
               uint64_t *n_out, int64_t *hist, DevScope &ds, unsigned long long *counters, cudaStream_t st)
{
    const uint32_t nw = key_words(k);
    const uint64_t total = n_high + n_low;
    WideTable t{};
    t.cap = std::max<uint64_t>(1024, (uint64_t)std::ceil((double)std::max<uint64_t>(total, 16) * 1.6));
    t.keys = ds.n<unsigned long long>(t.cap * nw);
    t.meta = ds.n<uint32_t>(t.cap * 2 + 2);
    CK(launch_wide_init(k, t, st));
    const uint32_t mp = (uint32_t)std::min<uint64_t>(t.cap, 1u << 16);
    if (n_high) {
        unsigned long long *hk = ds.n<unsigned long long>(n_high * nw);
        uint32_t *hc = ds.n<uint32_t>(n_high);
        CK(cudaMemcpyAsync(hk, high_keys, n_high * nw * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(hc, high_counts, n_high * 4, cudaMemcpyHostToDevice, st));
        CK(launch_wide_insert_pairs(k, hk, hc, 0, n_high, t, mp, counters, st));
    }
    if (n_low) {
        unsigned long long *lk = ds.n<unsigned long long>(n_low * nw);
        CK(cudaMemcpyAsync(lk, low_keys, n_low * nw * 8, cudaMemcpyHostToDevice, st));
        CK(launch_wide_insert_pairs(k, lk, nullptr, 1, n_low, t, mp, counters, st));
    }
    unsigned long long *dh = ds.n<unsigned long long>(HIST_BINS);
    const uint64_t ovf_cap = 1 << 20;
    uint32_t *ovf = ds.n<uint32_t>(ovf_cap);
    CK(cudaMemsetAsync(dh, 0, HIST_BINS * 8, st));
    CK(launch_wide_compact(k, t, count_max, min_count, max_count, nullptr, nullptr, 0, nullptr, nullptr, 0, counters, 1,
                           st));
    unsigned long long c[C_COUNT];
    CK(cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (c[C_FLAGS]) return set_error(KC_ERR_DEVICE, "merge kernel reported error flags");
    const uint64_t kept = c[C_KEPT];
    unsigned long long *rk = ds.n<unsigned long long>(std::max<uint64_t>(kept, 1) * nw);
    uint32_t *rc = ds.n<uint32_t>(std::max<uint64_t>(kept, 1));
    CK(launch_wide_compact(k, t, count_max, min_count, max_count, rk, rc, kept, dh, ovf, ovf_cap, counters, 0, st));
    unsigned long long *sk = ds.n<unsigned long long>(std::max<uint64_t>(kept, 1) * nw);
    uint32_t *sc = ds.n<uint32_t>(std::max<uint64_t>(kept, 1));
    void *tmp = ds.get(wide_sort_tmp_bytes(kept));
    CK(launch_wide_sort(k, rk, rc, kept, sk, sc, tmp, counters + C_FLAGS, st));
    std::vector<unsigned long long> hh(HIST_BINS);
    CK(cudaMemcpyAsync(hh.data(), dh, HIST_BINS * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (c[C_FLAGS]) return set_error(KC_ERR_DEVICE, "merge or sort kernel reported error flags");
    const uint64_t n_ovf = std::min<uint64_t>(c[C_OVF_LEN], ovf_cap);
    std::vector<uint32_t> oh(n_ovf);
    if (n_ovf) CK(cudaMemcpyAsync(oh.data(), ovf, n_ovf * 4, cudaMemcpyDeviceToHost, st));
    const uint64_t n_copy = std::min(kept, out_cap);
    if (n_copy) {
        CK(cudaMemcpyAsync(out_keys, sk, n_copy * nw * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(out_counts, sc, n_copy * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    *n_out = kept;
    if (hist) {
        for (uint64_t v = hist_min; v <= hist_max; ++v) hist[v - hist_min] = (v >= 1 && v < HIST_BINS) ? (int64_t)hh[v] : 0;
        for (uint32_t v : oh)
            if (v >= hist_min && v <= hist_max) hist[v - hist_min]++;
    }
    return KC_OK;
}

}  // namespace

extern "C" int kc_merge_records(const uint64_t *high_keys, const uint32_t *high_counts, uint64_t n_high,
                                const uint64_t *low_keys, uint64_t n_low, uint32_t k, uint32_t count_max,
                                uint32_t min_count, uint32_t max_count, uint32_t hist_min, uint32_t hist_max,
                                uint64_t *out_keys, uint32_t *out_counts, uint64_t out_cap, uint64_t *n_out,
                                int64_t *hist)
{
    if ((n_high && (!high_keys || !high_counts)) || (n_low && !low_keys) || !n_out || (out_cap && (!out_keys || !out_counts)))
        return set_error(KC_ERR_INVALID, "bad argument");
    if (k < 1 || k > 128 || count_max == 0 || max_count < min_count || hist_max < hist_min)
        return set_error(KC_ERR_INVALID, "bad parameter");
    if ((uint64_t)hist_max - hist_min + 1 > (1ULL << 28)) return set_error(KC_ERR_INVALID, "histogram range too large");
    try {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            return set_error(KC_ERR_NO_DEVICE, "no CUDA device");
        }
        cudaStream_t st;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct SG {
            cudaStream_t s;
            ~SG() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        } sg{st};
        DevScope ds(st);
        unsigned long long *counters = ds.n<unsigned long long>(C_COUNT);
        CK(cudaMemsetAsync(counters, 0, C_COUNT * 8, st));
        if (k > 32)
            return merge_wide(high_keys, high_counts, n_high, low_keys, n_low, k, count_max, min_count, max_count,
                              hist_min, hist_max, out_keys, out_counts, out_cap, n_out, hist, ds, counters, st);
        const uint64_t cap = std::max<uint64_t>(1024, bit_ceil64((uint64_t)std::ceil(std::max<double>(n_high, 16) * 1.8)));
        TableRef tr{static_cast<Slot *>(ds.get(cap * sizeof(Slot))), cap - 1};
        CK(launch_init_slots(tr.slots, cap, st));
        const uint32_t mp = (uint32_t)std::min<uint64_t>(cap, 1u << 16);
        unsigned long long *hk = ds.n<unsigned long long>(std::max<uint64_t>(n_high, 1));
        uint32_t *hc = ds.n<uint32_t>(std::max<uint64_t>(n_high, 1));
        if (n_high) {
            CK(cudaMemcpyAsync(hk, high_keys, n_high * 8, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(hc, high_counts, n_high * 4, cudaMemcpyHostToDevice, st));
            CK(launch_insert_pairs(hk, hc, n_high, tr, mp, counters, st));
        }
        const uint64_t rec_cap = std::max<uint64_t>(n_high + n_low, 1);
        unsigned long long *rk = ds.n<unsigned long long>(rec_cap);
        uint32_t *rc = ds.n<uint32_t>(rec_cap);
        unsigned long long *dh = ds.n<unsigned long long>(HIST_BINS);
        const uint64_t ovf_cap = 1 << 20;
        uint32_t *ovf = ds.n<uint32_t>(ovf_cap);
        CK(cudaMemsetAsync(dh, 0, HIST_BINS * 8, st));
        if (n_low) {
            unsigned long long *lk = ds.n<unsigned long long>(n_low);
            CK(cudaMemcpyAsync(lk, low_keys, n_low * 8, cudaMemcpyHostToDevice, st));
            CK(launch_merge_low(lk, n_low, tr, mp, min_count, max_count, rk, rc, rec_cap, counters, st));
        }
        CK(launch_compact(tr, cap, count_max, min_count, max_count, rk, rc, rec_cap, dh, ovf, ovf_cap, counters, st));
        unsigned long long c[C_COUNT];
        CK(cudaMemcpyAsync(c, counters, sizeof(c), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c[C_FLAGS]) return set_error(KC_ERR_DEVICE, "merge kernel reported error flags");
        const uint64_t n_rec = c[C_REC_LEN];
        if (n_rec > 1) {
            void *tmp = ds.get(sort_tmp_bytes(n_rec));
            CK(launch_radix_sort(rk, rc, n_rec, 2 * k, tmp, st, counters + C_FLAGS));
        }
        CK(launch_pair_reverse(rk, n_rec, st));
        std::vector<unsigned long long> hh(HIST_BINS);
        CK(cudaMemcpyAsync(hh.data(), dh, HIST_BINS * 8, cudaMemcpyDeviceToHost, st));
        const uint64_t n_ovf = std::min<uint64_t>(c[C_OVF_LEN], ovf_cap);
        std::vector<uint32_t> oh(n_ovf);
        if (n_ovf) CK(cudaMemcpyAsync(oh.data(), ovf, n_ovf * 4, cudaMemcpyDeviceToHost, st));
        const uint64_t n_copy = std::min(n_rec, out_cap);
        if (n_copy) {
            CK(cudaMemcpyAsync(out_keys, rk, n_copy * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out_counts, rc, n_copy * 4, cudaMemcpyDeviceToHost, st));
        }
        unsigned long long sort_flags = 0;
        CK(cudaMemcpyAsync(&sort_flags, counters + C_FLAGS, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (sort_flags) return set_error(KC_ERR_DEVICE, "record sort reported error flags");
        hh[1] += c[C_LOW_ONLY];
        *n_out = n_rec;
        if (hist) {
            for (uint64_t v = hist_min; v <= hist_max; ++v) hist[v - hist_min] = (v >= 1 && v < HIST_BINS) ? (int64_t)hh[v] : 0;
            for (uint32_t v : oh)
                if (v >= hist_min && v <= hist_max) hist[v - hist_min]++;
        }
        return KC_OK;
    } catch (const KcError &e) {
        return set_error(e.code, e.msg);
    }
}
