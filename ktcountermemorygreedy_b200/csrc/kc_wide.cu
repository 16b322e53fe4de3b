// kc_wide.cu -- device side of k-mers of 33..128 bases (the reference's
// kmer<2> and kmer<4>, src/main.cpp:617-633): extraction from the FASTQ
// tiles, the N-word counting table, compaction and the printed-order sort.
//
// Extraction uses the tile scheme of the kmer<1> path: a bulk copy brings
// 8 KiB of FASTQ and the 128 bytes before it into shared memory; every
// 32-byte segment is classified into 2-bit codes, a valid-base mask and a
// sequence-line mask; the ends of windows of k valid bases come from the run
// of valid bases before each segment; and each window's forward and
// reverse-complement word arrays are read straight out of the packed codes.
// Forward word w holds the 32 codes ending 32w bases before the window's
// end, newest at the top (GetKmer<N>'s seq after its right shifts,
// src/GetKmer.h:70-72, src/kmer.h:102-118); reverse-complement word w holds
// the complemented codes starting 32w bases after the window's start, first
// at the top (its rev after the left shifts, src/GetKmer.h:74-76,
// src/kmer.h:59-75); data[last] of both is masked to its top 2 * (k % 32)
// bits, and the canonical k-mer is the lexicographically smaller array
// (src/GetKmer.h:181-206).  Words above data[last] are zero (GetKmer<4> at
// k = 96 leaves stale bases in data[3]; the counts here are exact instead).
#include <algorithm>

#include "kc_device.cuh"
#include "kc_wide.cuh"

namespace kc {

namespace {

constexpr uint32_t FULLW = 0xffffffffu;
constexpr uint32_t WX_THREADS = 256;          // one 32-byte segment of the tile per thread
constexpr uint32_t WBUF = TILE + WIDE_HALO;   // 8320 bytes, a multiple of 16
constexpr uint32_t WSEGS = WBUF / 32;         // 260 segments, the 4 halo segments first
constexpr uint32_t WH = WIDE_HALO / 32;
constexpr uint32_t WSTRIDE = WSEGS + 4;       // per-segment shared arrays (entry WSEGS stays zero)

int wide_sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

unsigned wide_grid(uint64_t n, uint32_t threads, uint32_t per_sm = 8)
{
    uint64_t g = (n + threads - 1) / threads;
    const uint64_t cap = (uint64_t)wide_sm_count() * per_sm;
    return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
}

__device__ __forceinline__ uint32_t lanes_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over the 256-thread block.
__device__ __forceinline__ uint32_t scan256(uint32_t v, uint32_t *s_warp, uint32_t &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULLW, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < 8 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULLW, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t base = warp ? s_warp[warp - 1] : 0;
    total = s_warp[7];
    __syncthreads();
    return base + x - v;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One 16-byte slot read as a single access (relaxed, device scope).
__device__ __forceinline__ ulonglong2 ld_slot128(const ulonglong2 *p)
{
    ulonglong2 v;
    asm volatile("{\n\t.reg .b128 d;\n\t"
                 "ld.relaxed.gpu.global.b128 d, [%2];\n\t"
                 "mov.b128 {%0, %1}, d;\n\t}"
                 : "=l"(v.x), "=l"(v.y)
                 : "l"(p)
                 : "memory");
    return v;
}

// 16-byte compare-and-swap: writes val where *p == cmp; returns the old slot.
__device__ __forceinline__ ulonglong2 cas_slot128(ulonglong2 *p, ulonglong2 cmp, ulonglong2 val)
{
    ulonglong2 old;
    asm volatile("{\n\t.reg .b128 d, c, v;\n\t"
                 "mov.b128 c, {%3, %4};\n\t"
                 "mov.b128 v, {%5, %6};\n\t"
                 "atom.relaxed.gpu.global.cas.b128 d, [%2], c, v;\n\t"
                 "mov.b128 {%0, %1}, d;\n\t}"
                 : "=l"(old.x), "=l"(old.y)
                 : "l"(p), "l"(cmp.x), "l"(cmp.y), "l"(val.x), "l"(val.y)
                 : "memory");
    return old;
}

constexpr unsigned long long WIDE_EMPTY = ~0ull;   // both words of an empty 16-byte slot

// Placement hash of an N-word key (table slots, HyperLogLog); never affects a count.
template <uint32_t N>
__device__ __forceinline__ uint64_t wide_hash(const uint64_t (&key)[N])
{
    uint64_t h = key[0];
#pragma unroll
    for (uint32_t w = 1; w < N; ++w) h = slot_hash(h) ^ key[w];
    return slot_hash(h);
}

__device__ __forceinline__ void hll_add_s(uint32_t *regs, uint64_t h)
{
    h = slot_hash(h ^ 0x5bd1e9955bd1e995ULL);
    const uint32_t r = (uint32_t)(h >> (64 - HLL_BITS));
    const uint32_t rank = __clzll((h << HLL_BITS) | (1ULL << (HLL_BITS - 1))) + 1;
    if (rank > regs[r]) atomicMax(&regs[r], rank);
}

// Adds c to the count of key, probing at most max_probe slots.  False: no
// slot left on the probe path (the table is too full).
template <uint32_t N>
__device__ bool wide_add(const WideTable &t, const uint64_t (&key)[N], uint32_t c, uint32_t max_probe,
                         unsigned long long *flags)
{
    unsigned long long i = __umul64hi(wide_hash<N>(key), t.cap);
    if constexpr (N == 2) {
        if (key[0] == WIDE_EMPTY && key[1] == WIDE_EMPTY) {
            atomicAdd(&t.meta[t.cap], c);
            atomicOr(&t.meta[t.cap + 1], 1u);
            return true;
        }
        const ulonglong2 want = make_ulonglong2(key[0], key[1]);
        const ulonglong2 empty = make_ulonglong2(WIDE_EMPTY, WIDE_EMPTY);
        ulonglong2 *slots = reinterpret_cast<ulonglong2 *>(t.keys);
        for (uint32_t n = 0; n < max_probe; ++n) {
            // a slot goes from empty to one key once and never changes again
            ulonglong2 v = ld_slot128(slots + i);
            bool vacant = v.x == WIDE_EMPTY && v.y == WIDE_EMPTY;
            if (vacant) {
                v = cas_slot128(slots + i, empty, want);
                vacant = v.x == WIDE_EMPTY && v.y == WIDE_EMPTY;   // claimed by this thread
            }
            if (vacant || (v.x == want.x && v.y == want.y)) {
                atomicAdd(&t.meta[i], c);
                return true;
            }
            i = (i + 1 == t.cap) ? 0 : i + 1;
        }
        return false;
    } else {
        for (uint32_t n = 0; n < max_probe; ++n) {
            uint32_t *st = t.meta + 2 * i;
            uint32_t s = ld_acquire(st);
            if (s == 0) {
                s = atomicCAS(st, 0u, 1u);
                if (s == 0) {
#pragma unroll
                    for (uint32_t w = 0; w < N; ++w) t.keys[i * N + w] = key[w];
                    st_release(st, 2u);   // the key words are visible before the state says so
                    atomicAdd(st + 1, c);
                    return true;
                }
            }
            if (s == 1) {
                // another thread is writing this slot's key: a few stores away
                uint32_t it = 0;
                do {
                    __nanosleep(32);
                    s = ld_acquire(st);
                } while (s == 1 && ++it < SPIN_LIMIT);
                if (s == 1) {
                    atomicOr(flags, ERR_WAIT_TIMEOUT);
                    return true;
                }
            }
            bool eq = true;
#pragma unroll
            for (uint32_t w = 0; w < N; ++w) eq = eq && (__ldcg(&t.keys[i * N + w]) == key[w]);
            if (eq) {
                atomicAdd(st + 1, c);
                return true;
            }
            i = (i + 1 == t.cap) ? 0 : i + 1;
        }
        return false;
    }
}

// The 32 codes of positions e-31..e (e >= 31), position e at bits 62..63.
__device__ __forceinline__ uint64_t fwd_word(const uint64_t *codes, uint32_t e)
{
    const uint32_t s = e >> 5, o = e & 31;
    if (o == 31) return codes[s];
    const uint32_t sh = 2 * (o + 1);
    return (codes[s - 1] >> sh) | (codes[s] << (64 - sh));
}

// The complemented codes of positions a..a+31, position a at bits 62..63
// (rcodes = pair_reverse(~codes): position q of a segment at bits 62-2q).
__device__ __forceinline__ uint64_t rc_word(const uint64_t *rcodes, uint32_t a)
{
    const uint32_t s = a >> 5, o = a & 31;
    if (o == 0) return rcodes[s];
    return (rcodes[s] << (2 * o)) | (rcodes[s + 1] >> (64 - 2 * o));
}

// Canonical kmer<N> of the window of k bases ending at code-stream position P.
template <uint32_t N>
__device__ __forceinline__ void window_key(const uint64_t *codes, const uint64_t *rcodes, uint32_t P, uint32_t k,
                                           uint32_t last, uint64_t back_mask, uint64_t (&key)[N])
{
    uint64_t f[N], r[N];
    const uint32_t S = P - k + 1;
#pragma unroll
    for (uint32_t w = 0; w < N; ++w) {
        f[w] = 0;
        r[w] = 0;
        if (w <= last) {
            f[w] = fwd_word(codes, P - 32 * w);
            r[w] = rc_word(rcodes, S + 32 * w);
            if (w == last) {
                f[w] &= back_mask;
                r[w] &= back_mask;
            }
        }
    }
    int less = -1;
#pragma unroll
    for (uint32_t w = 0; w < N; ++w)
        if (less < 0 && f[w] != r[w]) less = f[w] < r[w] ? 1 : 0;
#pragma unroll
    for (uint32_t w = 0; w < N; ++w) key[w] = less == 1 ? f[w] : r[w];
}

template <uint32_t N, int MODE>
__global__ void __launch_bounds__(WX_THREADS) k_wide_extract(WideArgs a, uint32_t k)
{
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t *sbuf[2] = {smem, smem + WBUF};
    uint64_t *s_codes = reinterpret_cast<uint64_t *>(smem + 2 * WBUF);
    uint64_t *s_rcodes = s_codes + WSTRIDE;
    uint32_t *s_good = reinterpret_cast<uint32_t *>(s_rcodes + WSTRIDE);
    uint32_t *s_chunk = s_good + WSTRIDE;              // <= 4 * WX_THREADS entries
    uint32_t *s_hll = s_chunk + 4 * WX_THREADS;        // SCAN: HLL_M registers
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_bh[MODE == WMODE_SCAN ? 256 : 1];
    __shared__ unsigned long long s_base;

    const int tid = threadIdx.x, lane = tid & 31;
    uint64_t u = blockIdx.x;
    if (u >= a.n_tiles) return;
    const uint32_t last = (k - 1) / 32, rem = k % 32;
    const uint64_t back_mask = rem ? (((1ULL << (2 * rem)) - 1ULL) << (64 - 2 * rem)) : ~0ULL;
    const uint32_t blo = a.bucket_lo, bhi = a.bucket_hi ? a.bucket_hi : 256u;

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
        s_codes[WSEGS] = 0;
        s_rcodes[WSEGS] = 0;
    }
    if (MODE == WMODE_SCAN) {
        s_bh[tid] = 0;
        for (uint32_t i = tid; i < HLL_M; i += WX_THREADS) s_hll[i] = 0;
    }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(&mbar[0], WBUF);
        bulk_load(sbuf[0], a.buf + u * TILE - WIDE_HALO, WBUF, &mbar[0]);
    }
    unsigned long long *flags = &a.counters[C_FLAGS];
    unsigned long long n_occ = 0, n_ins = 0;
    uint32_t iter = 0;
    for (; u < a.n_tiles; u += gridDim.x, ++iter) {
        const int s = iter & 1;
        const uint64_t un = u + gridDim.x;
        const bool pending_next = un < a.n_tiles;
        if (tid == 0 && pending_next) {
            fence_proxy_async_smem();
            mbar_expect_tx(&mbar[s ^ 1], WBUF);
            bulk_load(sbuf[s ^ 1], a.buf + un * TILE - WIDE_HALO, WBUF, &mbar[s ^ 1]);
        }
        const bool ok = mbar_wait(&mbar[s], (iter >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(flags, ERR_WAIT_TIMEOUT);
            if (pending_next) mbar_wait(&mbar[s ^ 1], ((iter + 1) >> 1) & 1);
            return;
        }
        const uint8_t *tb = sbuf[s];
        const uint32_t seg_id = a.tile_seg[u];
        const Seg sg = a.segs[seg_id];
        const bool first = (u == sg.first_tile);
        const uint64_t line0 = a.tile_prefix[u] - a.tile_prefix[sg.first_tile];

        uint64_t codes;
        uint32_t valid, nl;
        classify32(tb + WIDE_HALO + 32 * tid, codes, valid, nl);
        uint32_t tot_nl;
        const uint32_t excl_nl = scan256((uint32_t)__popc(nl), s_warp, tot_nl);
        s_codes[WH + tid] = codes;
        s_rcodes[WH + tid] = pair_reverse(~codes);
        s_good[WH + tid] = valid & line_mask(line0 + excl_nl, nl, 1);
        if (tid < 32) {
            // the halo: the 128 bytes before the tile, the end of the file's
            // previous tile (nothing for a file's first tile); line numbers
            // counted back from the tile's first line
            uint64_t hc = 0;
            uint32_t hv = 0, hn = 0;
            if (lane < (int)WH && !first) classify32(tb + 32 * lane, hc, hv, hn);
            uint32_t x = lane < (int)WH ? (uint32_t)__popc(hn) : 0u;
            x += __shfl_down_sync(FULLW, x, 1);
            x += __shfl_down_sync(FULLW, x, 2);   // lane j: newlines of halo segments j..3
            if (lane < (int)WH) {
                s_codes[lane] = hc;
                s_rcodes[lane] = pair_reverse(~hc);
                s_good[lane] = first ? 0u : (hv & line_mask(line0 - x, hn, 1));
            }
        }
        __syncthreads();

        // windows of k valid bases ending in this thread's segment: the run
        // of valid bases before it comes from the four segments before
        const uint32_t g = s_good[WH + tid];
        uint32_t ends = 0;
        if (g) {
            uint32_t run = 0;
            for (int j = (int)(WH + tid) - 1; j >= tid; --j) {
                const uint32_t gj = s_good[j];
                if (gj == FULLW) {
                    run += 32;
                    continue;
                }
                run += (uint32_t)__clz(~gj);
                break;
            }
#pragma unroll
            for (uint32_t q = 0; q < 32; ++q) {
                run = ((g >> q) & 1u) ? run + 1 : 0u;
                if (run >= k) ends |= 1u << q;
            }
        }
        n_occ += (unsigned long long)__popc(ends);

        // chunks of 8 positions holding window ends, listed so that the
        // threads share the windows of the tile's sequence segments
        uint32_t nq = 0;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) nq += ((ends >> (8 * q)) & 0xFFu) ? 1u : 0u;
        uint32_t packed_tot;
        const uint32_t packed = scan256((uint32_t)__popc(ends) | (nq << 16), s_warp, packed_tot);
        const uint32_t n_windows = packed_tot & 0xFFFFu, n_chunks = packed_tot >> 16;
        {
            // chunk = first window index << 18 | segment << 10 | quarter << 8 | its 8 end bits
            uint32_t idx = packed & 0xFFFFu, c = packed >> 16;
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                const uint32_t e8 = (ends >> (8 * q)) & 0xFFu;
                if (e8) s_chunk[c++] = (idx << 18) | ((uint32_t)tid << 10) | (q << 8) | e8;
                idx += (uint32_t)__popc(e8);
            }
        }
        if (MODE == WMODE_EMIT && tid == 0)
            s_base = n_windows ? atomicAdd(&a.counters[C_EMIT_LEN], (unsigned long long)n_windows) : 0ull;
        __syncthreads();
        for (uint32_t ci = tid; ci < n_chunks; ci += WX_THREADS) {
            const uint32_t ch = s_chunk[ci], e8 = ch & 0xFFu;
            const uint32_t sgm = (ch >> 10) & 0xFFu, q0 = ((ch >> 8) & 3u) * 8;
            uint32_t idx = ch >> 18;
            const uint32_t pos0 = 32 * (WH + sgm) + q0;
#pragma unroll 1
            for (uint32_t p = 0; p < 8; ++p) {
                if (!((e8 >> p) & 1u)) continue;
                uint64_t key[N];
                window_key<N>(s_codes, s_rcodes, pos0 + p, k, last, back_mask, key);
                if (MODE == WMODE_SCAN) {
                    hll_add_s(s_hll, wide_hash<N>(key));
                    atomicAdd(&s_bh[(uint32_t)(key[0] >> 56)], 1u);
                } else if (MODE == WMODE_INSERT) {
                    const uint32_t b = (uint32_t)(key[0] >> 56);
                    if (b >= blo && b < bhi) {
                        ++n_ins;
                        if (!wide_add<N>(a.table, key, 1u, a.max_probe, flags)) atomicOr(flags, ERR_TABLE_FULL);
                    }
                } else {
                    const unsigned long long o = s_base + idx;
                    if (o < a.list_cap) {
#pragma unroll
                        for (uint32_t w = 0; w < N; ++w) a.list[o * N + w] = key[w];
                    } else {
                        atomicOr(flags, ERR_LIST_FULL);
                    }
                    ++idx;
                }
            }
        }
        __syncthreads();
    }

    for (int o = 16; o > 0; o >>= 1) {
        n_occ += __shfl_down_sync(FULLW, n_occ, o);
        n_ins += __shfl_down_sync(FULLW, n_ins, o);
    }
    if (MODE == WMODE_SCAN) {
        if (lane == 0 && n_occ && a.occ) atomicAdd(a.occ, n_occ);
        __syncthreads();
        if (a.bucket_hist && s_bh[tid]) atomicAdd(&a.bucket_hist[tid], (unsigned long long)s_bh[tid]);
        if (a.hll)
            for (uint32_t i = tid; i < HLL_M; i += WX_THREADS) {
                const uint32_t v = s_hll[i];
                if (v > *(volatile uint32_t *)&a.hll[i]) atomicMax(&a.hll[i], v);
            }
    } else if (MODE == WMODE_INSERT) {
        if (lane == 0 && n_ins) atomicAdd(&a.counters[C_HIGH_LEN], n_ins);
    }
}

template <uint32_t N, int MODE>
cudaError_t launch_wide_extract_t(uint32_t k, const WideArgs &a, cudaStream_t st)
{
    const size_t smem = 2 * WBUF + 2 * WSTRIDE * 8 + WSTRIDE * 4 + 4 * WX_THREADS * 4 +
                        (MODE == WMODE_SCAN ? HLL_M * 4 : 0);
    cudaError_t e = cudaFuncSetAttribute(k_wide_extract<N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wide_extract<N, MODE>, WX_THREADS, smem);
    if (e != cudaSuccess) return e;
    const uint64_t grid = std::min<uint64_t>(a.n_tiles, (uint64_t)wide_sm_count() * std::max(per_sm, 1));
    note_kernel_launch();
    k_wide_extract<N, MODE><<<(unsigned)grid, WX_THREADS, smem, st>>>(a, k);
    return cudaGetLastError();
}

// N = 2: every key slot all ones, every count 0; N = 4: every state and count 0.
template <uint32_t N>
__global__ void __launch_bounds__(256) k_wide_init(WideTable t)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= t.cap; i += (uint64_t)gridDim.x * blockDim.x) {
        reinterpret_cast<uint2 *>(t.meta)[i] = make_uint2(0u, 0u);
        if (N == 2 && i < t.cap)
            reinterpret_cast<ulonglong2 *>(t.keys)[i] = make_ulonglong2(WIDE_EMPTY, WIDE_EMPTY);
    }
}

template <uint32_t N>
__global__ void __launch_bounds__(256) k_wide_insert_pairs(const unsigned long long *keys, const uint32_t *counts,
                                                           uint32_t cnull, uint64_t n, WideTable t, uint32_t max_probe,
                                                           unsigned long long *counters)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key[N];
#pragma unroll
        for (uint32_t w = 0; w < N; ++w) key[w] = keys[i * N + w];
        if (!wide_add<N>(t, key, counts ? counts[i] : cnull, max_probe, &counters[C_FLAGS]))
            atomicOr(&counters[C_FLAGS], ERR_TABLE_FULL);
    }
}

template <uint32_t N>
__global__ void __launch_bounds__(256) k_wide_compact(WideTable t, uint32_t count_max, uint32_t min_count,
                                                      uint32_t max_count, unsigned long long *rec_keys,
                                                      uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist,
                                                      uint32_t *ovf, uint64_t ovf_cap, unsigned long long *counters,
                                                      int count_only)
{
    __shared__ uint32_t s_hist[2048];
    if (!count_only)
        for (int i = threadIdx.x; i < 2048; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // N = 2 also visits index cap: the all-ones key's own count
    const uint64_t n_slots = t.cap + (N == 2 ? 1 : 0);
    const uint64_t rounds = (n_slots + stride - 1) / stride;
    uint32_t distinct = 0, kept = 0;
    for (uint64_t r = 0; r < rounds; ++r) {
        const uint64_t i = r * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        bool keep = false;
        uint32_t c = 0;
        if (i < n_slots) {
            bool used;
            uint32_t cnt;
            if (N == 2) {
                if (i < t.cap) {
                    const ulonglong2 kw = reinterpret_cast<const ulonglong2 *>(t.keys)[i];
                    used = !(kw.x == WIDE_EMPTY && kw.y == WIDE_EMPTY);
                    cnt = used ? t.meta[i] : 0u;
                } else {
                    used = t.meta[t.cap + 1] != 0u;
                    cnt = t.meta[t.cap];
                }
            } else {
                const uint2 m = reinterpret_cast<const uint2 *>(t.meta)[i];
                used = m.x == 2u;
                cnt = m.y;
            }
            if (used) {
                ++distinct;
                c = cnt < count_max ? cnt : count_max;
                keep = c >= min_count && c <= max_count;
                if (!count_only) {
                    if (c < 2048) atomicAdd(&s_hist[c], 1u);
                    else if (c < HIST_BINS) atomicAdd(&hist[c], 1ull);
                    else {
                        const unsigned long long p = atomicAdd(&counters[C_OVF_LEN], 1ull);
                        if (p < ovf_cap) ovf[p] = c;
                        else atomicOr(&counters[C_FLAGS], ERR_HIST_OVERFLOW_FULL);
                    }
                }
            }
        }
        kept += keep ? 1u : 0u;
        if (!count_only) {
            const uint32_t b = __ballot_sync(FULLW, keep);
            if (b) {
                const int leader = __ffs(b) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&counters[C_REC_LEN], (unsigned long long)__popc(b));
                base = __shfl_sync(FULLW, base, leader);
                if (keep) {
                    const unsigned long long pos = base + (unsigned)__popc(b & lanes_lt());
                    if (pos < rec_cap) {
#pragma unroll
                        for (uint32_t w = 0; w < N; ++w) rec_keys[pos * N + w] = i < t.cap ? t.keys[i * N + w] : WIDE_EMPTY;
                        rec_counts[pos] = c;
                    } else {
                        atomicOr(&counters[C_FLAGS], ERR_RECORDS_FULL);
                    }
                }
            }
        }
    }
    const unsigned d = __reduce_add_sync(FULLW, distinct), kk = __reduce_add_sync(FULLW, kept);
    if (lane == 0) {
        if (count_only && kk) atomicAdd(&counters[C_KEPT], (unsigned long long)kk);
        if (!count_only && d) atomicAdd(&counters[C_DISTINCT], (unsigned long long)d);
    }
    if (!count_only) {
        __syncthreads();
        for (int i = threadIdx.x; i < 2048; i += blockDim.x)
            if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
    }
}

__global__ void k_iota_u32(uint32_t *p, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

__global__ void k_iota_u64(unsigned long long *p, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = i;
}

// skey[i] = word w of record perm[i], its 2-bit groups reversed (printed order)
template <uint32_t N>
__global__ void k_wide_sort_word(const unsigned long long *keys, const uint32_t *perm, uint64_t n, uint32_t w,
                                 unsigned long long *skey)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        skey[i] = pair_reverse(keys[(uint64_t)perm[i] * N + w]);
}

template <uint32_t N>
__global__ void k_wide_permute(const unsigned long long *keys, const uint32_t *counts, const uint32_t *perm,
                               uint64_t n, unsigned long long *out_keys, uint32_t *out_counts)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = perm[i];
#pragma unroll
        for (uint32_t w = 0; w < N; ++w) out_keys[i * N + w] = keys[j * N + w];
        out_counts[i] = counts[j];
    }
}

template <uint32_t N>
__global__ void k_wide_gather_rows(const unsigned long long *keys, const unsigned long long *idx, uint64_t n,
                                   unsigned long long *out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = idx[i];
#pragma unroll
        for (uint32_t w = 0; w < N; ++w) out[i * N + w] = keys[j * N + w];
    }
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

__global__ void k_pack_flags(const uint32_t *counts, uint64_t n, uint32_t filter_min, uint32_t filter_max,
                             uint32_t *flags)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = counts[i];
        flags[i] = (c + 1 >= filter_min && c <= filter_max) ? 1u : 0u;
    }
}

// One record per thread; consecutive threads write consecutive records, so a
// warp's byte stores cover one contiguous run.
template <uint32_t N>
__global__ void k_pack_write(const unsigned long long *keys, const uint32_t *counts, const uint32_t *flags,
                             const unsigned long long *pos, uint64_t n, uint32_t full, uint32_t tail_bytes,
                             uint32_t count_bytes, uint8_t *out, unsigned long long *n_bytes)
{
    const uint32_t rec = full * 8 + tail_bytes + count_bytes;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (i == n - 1) *n_bytes = (pos[i] + flags[i]) * rec;
        if (!flags[i]) continue;
        uint8_t *o = out + pos[i] * rec;
        uint32_t b = 0;
        for (uint32_t w = 0; w < full; ++w) {
            const uint64_t x = keys[i * N + w];
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) o[b++] = (uint8_t)(x >> (8 * j));
        }
        if (tail_bytes) {
            const uint64_t x = keys[i * N + full];   // its low bits below the k-mer are zero
            for (uint32_t j = 8 - tail_bytes; j < 8; ++j) o[b++] = (uint8_t)(x >> (8 * j));
        }
        const uint32_t c = counts[i];
        for (uint32_t j = 0; j < count_bytes; ++j) o[b++] = (uint8_t)(c >> (8 * j));
    }
}

}  // namespace

cudaError_t launch_wide_extract(int mode, uint32_t k, const WideArgs &a, cudaStream_t st)
{
    if (!a.n_tiles) return cudaSuccess;
    if (k <= 32 || k > 128) return cudaErrorInvalidValue;
    const uint32_t nw = key_words(k);
    if (nw == 2) {
        if (mode == WMODE_SCAN) return launch_wide_extract_t<2, WMODE_SCAN>(k, a, st);
        if (mode == WMODE_INSERT) return launch_wide_extract_t<2, WMODE_INSERT>(k, a, st);
        return launch_wide_extract_t<2, WMODE_EMIT>(k, a, st);
    }
    if (mode == WMODE_SCAN) return launch_wide_extract_t<4, WMODE_SCAN>(k, a, st);
    if (mode == WMODE_INSERT) return launch_wide_extract_t<4, WMODE_INSERT>(k, a, st);
    return launch_wide_extract_t<4, WMODE_EMIT>(k, a, st);
}

cudaError_t launch_wide_init(uint32_t k, WideTable t, cudaStream_t st)
{
    if (!t.cap) return cudaSuccess;
    note_kernel_launch();
    if (key_words(k) == 2)
        k_wide_init<2><<<wide_grid(t.cap + 1, 256), 256, 0, st>>>(t);
    else
        k_wide_init<4><<<wide_grid(t.cap + 1, 256), 256, 0, st>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_wide_insert_pairs(uint32_t k, const unsigned long long *keys, const uint32_t *counts,
                                     uint32_t count_if_null, uint64_t n, WideTable t, uint32_t max_probe,
                                     unsigned long long *counters, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_kernel_launch();
    if (key_words(k) == 2)
        k_wide_insert_pairs<2><<<wide_grid(n, 256), 256, 0, st>>>(keys, counts, count_if_null, n, t, max_probe, counters);
    else
        k_wide_insert_pairs<4><<<wide_grid(n, 256), 256, 0, st>>>(keys, counts, count_if_null, n, t, max_probe, counters);
    return cudaGetLastError();
}

cudaError_t launch_wide_compact(uint32_t k, WideTable t, uint32_t count_max, uint32_t min_count, uint32_t max_count,
                                unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                                unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap,
                                unsigned long long *counters, int count_only, cudaStream_t st)
{
    if (!t.cap) return cudaSuccess;
    note_kernel_launch();
    const unsigned g = wide_grid(t.cap, 256);
    if (key_words(k) == 2)
        k_wide_compact<2><<<g, 256, 0, st>>>(t, count_max, min_count, max_count, rec_keys, rec_counts, rec_cap, hist,
                                             ovf, ovf_cap, counters, count_only);
    else
        k_wide_compact<4><<<g, 256, 0, st>>>(t, count_max, min_count, max_count, rec_keys, rec_counts, rec_cap, hist,
                                             ovf, ovf_cap, counters, count_only);
    return cudaGetLastError();
}

size_t wide_sort_tmp_bytes(uint64_t n)
{
    n = std::max<uint64_t>(n, 1);
    return align256(n * 4) + align256(n * 8) + sort_tmp_bytes(n);
}

cudaError_t launch_wide_sort(uint32_t k, const unsigned long long *keys, const uint32_t *counts, uint64_t n,
                             unsigned long long *out_keys, uint32_t *out_counts, void *tmp,
                             unsigned long long *flags, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    const uint32_t nw = key_words(k), last = (k - 1) / 32, rem = k % 32;
    uint8_t *p = static_cast<uint8_t *>(tmp);
    uint32_t *perm = reinterpret_cast<uint32_t *>(p);
    unsigned long long *skey = reinterpret_cast<unsigned long long *>(p + align256(n * 4));
    void *rtmp = p + align256(n * 4) + align256(n * 8);
    const unsigned g = wide_grid(n, 256);
    note_kernel_launch();
    k_iota_u32<<<g, 256, 0, st>>>(perm, n);
    cudaError_t e = cudaGetLastError();
    // least significant word first: data[0] holds the last 32 bases of the
    // printed string, data[last] the first k - 32 * last
    for (uint32_t w = 0; w <= last && e == cudaSuccess; ++w) {
        note_kernel_launch();
        if (nw == 2) k_wide_sort_word<2><<<g, 256, 0, st>>>(keys, perm, n, w, skey);
        else k_wide_sort_word<4><<<g, 256, 0, st>>>(keys, perm, n, w, skey);
        e = cudaGetLastError();
        if (e == cudaSuccess && n > 1)
            e = launch_radix_sort(skey, perm, n, (w == last && rem) ? 2 * rem : 64u, rtmp, st, flags);
    }
    if (e != cudaSuccess) return e;
    note_kernel_launch();
    if (nw == 2) k_wide_permute<2><<<g, 256, 0, st>>>(keys, counts, perm, n, out_keys, out_counts);
    else k_wide_permute<4><<<g, 256, 0, st>>>(keys, counts, perm, n, out_keys, out_counts);
    return cudaGetLastError();
}

cudaError_t launch_wide_gather_rows(uint32_t k, const unsigned long long *keys, const unsigned long long *idx,
                                    uint64_t n, unsigned long long *out, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_kernel_launch();
    if (key_words(k) == 2) k_wide_gather_rows<2><<<wide_grid(n, 256), 256, 0, st>>>(keys, idx, n, out);
    else k_wide_gather_rows<4><<<wide_grid(n, 256), 256, 0, st>>>(keys, idx, n, out);
    return cudaGetLastError();
}

uint32_t packed_record_bytes(uint32_t k, uint32_t count_bytes)
{
    return (k / 32) * 8 + (2 * (k % 32) + 7) / 8 + count_bytes;
}

cudaError_t launch_pack_high(uint32_t k, const unsigned long long *keys, const uint32_t *counts, uint64_t n,
                             uint32_t count_bytes, uint32_t filter_min, uint32_t filter_max, uint32_t *flags,
                             unsigned long long *pos, unsigned long long *scan_tmp, uint8_t *out,
                             unsigned long long *n_bytes, cudaStream_t st)
{
    if (!n) return cudaMemsetAsync(n_bytes, 0, 8, st);
    const unsigned g = wide_grid(n, 256);
    note_kernel_launch();
    k_pack_flags<<<g, 256, 0, st>>>(counts, n, filter_min, filter_max, flags);
    cudaError_t e = launch_scan_u32(flags, pos, n, scan_tmp, st);
    if (e != cudaSuccess) return e;
    const uint32_t full = k / 32, tail = (2 * (k % 32) + 7) / 8;
    note_kernel_launch();
    if (k <= 32) k_pack_write<1><<<g, 256, 0, st>>>(keys, counts, flags, pos, n, full, tail, count_bytes, out, n_bytes);
    else if (k <= 64) k_pack_write<2><<<g, 256, 0, st>>>(keys, counts, flags, pos, n, full, tail, count_bytes, out, n_bytes);
    else k_pack_write<4><<<g, 256, 0, st>>>(keys, counts, flags, pos, n, full, tail, count_bytes, out, n_bytes);
    return cudaGetLastError();
}

cudaError_t launch_iota_u64(unsigned long long *p, uint64_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_kernel_launch();
    k_iota_u64<<<wide_grid(n, 256), 256, 0, st>>>(p, n);
    return cudaGetLastError();
}

}  // namespace kc
