// kc_kernels.cu -- the sm_100a device pipeline of the k-mer counter.
//
// Stages (one job; batched jobs run the same kernels over many files):
//   k_newlines      per-tile '\n' count and last '\n' offset (16-byte loads)
//   scan            exclusive prefix of the tile counts -> line number of
//                   every tile start (FASTQ line state machine without a
//                   sequential pass)
//   k_extract<M>    TMA-bulk-loaded 8 KiB tiles; per 32-byte segment the
//                   2-bit codes, valid-base mask and sequence-line mask; the
//                   ends of all windows of k valid bases found with a
//                   bit-parallel run test; canonical words formed directly
//                   from the packed codes.  The mode decides what happens to
//                   each canonical k-mer: count + HyperLogLog (SCAN), insert
//                   into the open-addressing table (INSERT), classify with the
//                   reference's two-level Bloom filter (BLOOM) or append to a
//                   list (EMIT).
//   k_insert_list   insert a k-mer list (Bloom non-FIRST occurrences)
//   k_merge_low     add the FIRST occurrences back (exact merged counts)
//   k_compact       table -> (string-order key, count) records + histogram
//   radix sort      LSD, 8-bit digits, warp match ranking, stable
//   selection       stable range selection for the count queries
#include <algorithm>
#include <atomic>
#include <utility>
#include <vector>

#include "kc_device.cuh"
#include "kc_kernels.cuh"

namespace kc {

namespace {

constexpr uint32_t FULL = 0xffffffffu;
constexpr uint32_t BUF_BYTES = TILE + HALO;   // 8224, a multiple of 16

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *s_warp, uint32_t &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < 8 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            uint32_t y = __shfl_up_sync(FULL, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t base = warp ? s_warp[warp - 1] : 0;
    total = s_warp[7];
    __syncthreads();
    return base + x - v;
}

// Bit b (b >= 32) of the result is set when bits b-k+1 .. b of g are all set.
__device__ __forceinline__ uint32_t run_ends(uint64_t g, uint32_t k)
{
    uint64_t r1 = g, r2 = r1 & (r1 << 1), r4 = r2 & (r2 << 2), r8 = r4 & (r4 << 4), r16 = r8 & (r8 << 8);
    uint64_t acc = ~0ULL;
    uint32_t sh = 0;
    if (k & 32) { acc &= r16 & (r16 << 16); sh = 32; }
    if (k & 16) { acc &= r16 << sh; sh += 16; }
    if (k & 8) { acc &= r8 << sh; sh += 8; }
    if (k & 4) { acc &= r4 << sh; sh += 4; }
    if (k & 2) { acc &= r2 << sh; sh += 2; }
    if (k & 1) { acc &= r1 << sh; sh += 1; }
    return (uint32_t)(acc >> 32);
}

struct KParams {
    uint32_t k;
    uint64_t kmask;     // low 2k bits
    uint64_t topmask;   // high 2k bits
    uint32_t fwd_shift; // 64 - 2k
};

__device__ __forceinline__ KParams kparams(uint32_t k)
{
    KParams p;
    p.k = k;
    p.kmask = k >= 32 ? ~0ULL : ((1ULL << (2 * k)) - 1ULL);
    p.fwd_shift = 64 - 2 * k;
    p.topmask = k >= 32 ? ~0ULL : (~0ULL << p.fwd_shift);
    return p;
}

// Forward and reverse-complement words of the window ending just before
// position q0 (0..31) of the current segment (for q0 = 0, the window ending at
// the previous segment's last position), the start of a roll along the
// segment: for each next base c, fwd = fwd >> 2 | c << 62 and
// rc = rc << 2 | (3 - c) << (64 - 2k), and the window's canonical word is
// min(fwd & topmask, rc) (the smaller word, as GetKmer::canonicalize).  fwd
// has stale bits below bit 64 - 2k (dropped by the mask); rc is exact.
// prev/cur hold the 2-bit codes of the previous and current segments (base q
// at bits 2q); the forward word puts base i of the window at bit 64-2k+2i (the
// reference's kmer<1> layout), so the 128-bit value (cur:prev) shifted right
// by 2q0 gives it.  rprev/rcur = pair_reverse(~codes) of the two segments: in
// the 128-bit value (rprev:rcur) span position q sits at 2-bit group 63 - q,
// so the reverse-complement word (complemented codes in reverse order) of the
// window is that value shifted right by 2k - 2q0 (left when negative).
__device__ __forceinline__ void window_words(uint64_t prev, uint64_t cur, uint64_t rprev, uint64_t rcur, uint32_t q0,
                                             const KParams &kp, uint64_t &fwd, uint64_t &rc)
{
    fwd = q0 ? (prev >> (2 * q0)) | (cur << (64 - 2 * q0)) : prev;
    const int t = 2 * (int)kp.k - 2 * (int)q0;
    uint64_t r;
    if (t == 0) r = rcur;
    else if (t > 0 && t < 64) r = (rcur >> t) | (rprev << (64 - t));
    else if (t >= 64) r = rprev;   // k = 32, q0 = 0
    else r = rcur << (-t);
    rc = r & kp.topmask;
}

__device__ __forceinline__ void hll_add(uint32_t *regs, unsigned long long key)
{
    uint64_t h = slot_hash(key ^ 0x5bd1e9955bd1e995ULL);
    uint32_t r = (uint32_t)(h >> (64 - HLL_BITS));
    uint32_t rank = __clzll((h << HLL_BITS) | (1ULL << (HLL_BITS - 1))) + 1;
    if (rank > *(volatile uint32_t *)&regs[r]) atomicMax(&regs[r], rank);
}

// Batched jobs keep one register set per sample in global memory, shared by
// all blocks: only a 1-in-64 hash sample of the k-mers updates them (the host
// scales the estimate by 64), and an update is skipped when the register
// already holds the rank.
__device__ __forceinline__ void hll_add_sampled(uint32_t *regs, unsigned long long key)
{
    uint64_t h = slot_hash(key ^ 0x5bd1e9955bd1e995ULL);
    if (h & ((1u << BATCH_HLL_SAMPLE_BITS) - 1)) return;
    uint32_t r = (uint32_t)(h >> (64 - HLL_BITS));
    uint32_t rank = __clzll((h << HLL_BITS) | (1ULL << (HLL_BITS + BATCH_HLL_SAMPLE_BITS - 1))) + 1;
    if (rank > *(volatile uint32_t *)&regs[r]) atomicMax(&regs[r], rank);
}

__device__ __forceinline__ void hll_add_shared(uint32_t *regs, unsigned long long key)
{
    uint64_t h = slot_hash(key ^ 0x5bd1e9955bd1e995ULL);
    uint32_t r = (uint32_t)(h >> (64 - HLL_BITS));
    uint32_t rank = __clzll((h << HLL_BITS) | (1ULL << (HLL_BITS - 1))) + 1;
    if (rank > regs[r]) atomicMax(&regs[r], rank);
}

// Tables have any capacity (mask = capacity - 1): a key's home slot is the
// high half of hash * capacity, probing is linear and wraps at the end.
__device__ __forceinline__ unsigned long long home_slot(unsigned long long key, unsigned long long mask)
{
    return __umul64hi(slot_hash(key), mask + 1);
}

__device__ __forceinline__ unsigned long long next_slot(unsigned long long i, unsigned long long mask)
{
    return i == mask ? 0 : i + 1;
}

// Adds c to key's count, probing at most max_probe slots from slot i.
__device__ __forceinline__ bool table_add_at(Slot *slots, unsigned long long mask, unsigned long long key,
                                             unsigned int c, uint32_t max_probe, unsigned long long i)
{
    for (uint32_t n = 0; n < max_probe; ++n) {
        unsigned long long cur = __ldcg(&slots[i].key);
        if (cur == key) {
            atomicAdd(&slots[i].count, c);
            return true;
        }
        if (cur == EMPTY_KEY) {
            unsigned long long prev = atomicCAS(&slots[i].key, EMPTY_KEY, key);
            if (prev == EMPTY_KEY || prev == key) {
                atomicAdd(&slots[i].count, c);
                return true;
            }
        }
        i = next_slot(i, mask);
    }
    return false;
}

__device__ __forceinline__ bool table_add(Slot *slots, unsigned long long mask, unsigned long long key,
                                          unsigned int c, uint32_t max_probe)
{
    return table_add_at(slots, mask, key, c, max_probe, home_slot(key, mask));
}

__device__ __forceinline__ Slot *table_find_at(Slot *slots, unsigned long long mask, unsigned long long key,
                                               uint32_t max_probe, bool &overflow, unsigned long long i)
{
    for (uint32_t n = 0; n < max_probe; ++n) {
        unsigned long long cur = __ldcg(&slots[i].key);
        if (cur == key) return &slots[i];
        if (cur == EMPTY_KEY) return nullptr;
        i = next_slot(i, mask);
    }
    overflow = true;
    return nullptr;
}

__device__ __forceinline__ Slot *table_find(Slot *slots, unsigned long long mask, unsigned long long key,
                                            uint32_t max_probe, bool &overflow)
{
    return table_find_at(slots, mask, key, max_probe, overflow, home_slot(key, mask));
}

// Grouped probes: the home slots of a thread's G keys are read with their
// loads in flight together, then each key is resolved in turn.  A slot only
// ever changes from empty to a key, so an early read is never wrong: a key
// found there is final, an empty slot is claimed by CAS (which reports a key
// that arrived meanwhile), and another key sends the probe on to the next slot.
template <uint32_t G>
__device__ __forceinline__ bool table_add_group(Slot *slots, unsigned long long mask, const unsigned long long *key,
                                                uint32_t act, uint32_t max_probe)
{
    unsigned long long i[G], cur[G];
#pragma unroll
    for (uint32_t u = 0; u < G; ++u) {
        i[u] = home_slot(key[u], mask);
        cur[u] = ((act >> u) & 1u) ? __ldcg(&slots[i[u]].key) : EMPTY_KEY;
    }
    bool ok = true;
#pragma unroll
    for (uint32_t u = 0; u < G; ++u) {
        if (!((act >> u) & 1u)) continue;
        if (cur[u] == key[u]) {
            atomicAdd(&slots[i[u]].count, 1u);
            continue;
        }
        if (cur[u] == EMPTY_KEY) {
            const unsigned long long prev = atomicCAS(&slots[i[u]].key, EMPTY_KEY, key[u]);
            if (prev == EMPTY_KEY || prev == key[u]) {
                atomicAdd(&slots[i[u]].count, 1u);
                continue;
            }
        }
        if (max_probe < 2 || !table_add_at(slots, mask, key[u], 1u, max_probe - 1, next_slot(i[u], mask))) ok = false;
    }
    return ok;
}

// Warp-aggregated insert: lanes holding the same k-mer elect one leader that
// adds the group's size.
__device__ __forceinline__ void warp_insert(bool act, unsigned long long key, const TableRef &tr,
                                            uint32_t max_probe, unsigned long long *flags)
{
    unsigned long long k = act ? key : EMPTY_KEY;
    uint32_t peers = __match_any_sync(FULL, k);
    if (act && (int)(threadIdx.x & 31) == __ffs(peers) - 1) {
        if (!table_add(tr.slots, tr.mask, k, __popc(peers), max_probe)) atomicOr(flags, ERR_TABLE_FULL);
    }
}

// ---------------------------------------------------------------------------
// newline census
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_newlines(const uint8_t *buf, uint64_t n_tiles, uint32_t *tile_nl,
                                                  int32_t *tile_lastnl)
{
    __shared__ uint32_t s_cnt[8];
    __shared__ int32_t s_last[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const uint4 *p = reinterpret_cast<const uint4 *>(buf + t * TILE + 32 * tid);
        uint4 a = __ldcs(p), b = __ldcs(p + 1);
        const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        uint32_t cnt = 0;
        int32_t last = -1;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint32_t eq = __vcmpeq4(w[i], 0x0a0a0a0au);
            cnt += __popc(eq) >> 3;
            if (eq) last = 32 * tid + 4 * i + (31 - __clz(eq)) / 8;
        }
        cnt = __reduce_add_sync(FULL, cnt);
        last = __reduce_max_sync(FULL, last);
        if (lane == 0) { s_cnt[warp] = cnt; s_last[warp] = last; }
        __syncthreads();
        if (tid == 0) {
            uint32_t c = 0;
            int32_t l = -1;
            for (int i = 0; i < 8; ++i) { c += s_cnt[i]; l = max(l, s_last[i]); }
            tile_nl[t] = c;
            tile_lastnl[t] = l;
        }
        __syncthreads();
    }
}

__global__ void k_chunk_lastnl(const int32_t *tile_lastnl, const uint32_t *tile_seg, const Seg *segs,
                               const uint64_t *seg_chunk0, uint64_t n_tiles, int32_t *chunk_lastnl)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n_tiles; t += (uint64_t)gridDim.x * blockDim.x) {
        int32_t l = tile_lastnl[t];
        if (l < 0) continue;
        uint32_t s = tile_seg[t];
        uint64_t fo = (t - segs[s].first_tile) * TILE;
        uint64_t c = seg_chunk0[s] + fo / PREPASS_CHUNK;
        atomicMax(&chunk_lastnl[c], (int32_t)(fo % PREPASS_CHUNK) + l);
    }
}

// ---------------------------------------------------------------------------
// extraction
// ---------------------------------------------------------------------------

// SCAP: the most k-mers staged per round (the PART reorder holds SCAP /
// EXT_THREADS of them per thread in registers); a PART launch with
// SCAP = 2048 fits four blocks per SM instead of three.
template <int MODE, uint32_t SCAP = STAGE_CAP>
__global__ void __launch_bounds__(EXT_THREADS, MODE == MODE_SCAN ? 5 : (SCAP <= 2048 ? 4 : 3))
    k_extract(ExtractArgs a, uint32_t stage_cap)
{
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t *sbuf[2] = {smem, smem + BUF_BYTES};
    uint64_t *s_codes = reinterpret_cast<uint64_t *>(smem + 2 * BUF_BYTES);   // 257 used
    uint64_t *s_rcodes = s_codes + 264;                                       // 257 used
    uint32_t *s_good = reinterpret_cast<uint32_t *>(s_rcodes + 264);          // 257 used
    unsigned long long *s_stage = reinterpret_cast<unsigned long long *>(s_good + 264);
    uint32_t *s_hll = reinterpret_cast<uint32_t *>(s_good + 264);   // SCAN mode: registers of sample 0
    const bool hll_local = MODE == MODE_SCAN && a.hll && a.hll_local;

    // staged modes: (segment, position) of each window, then (PART mode) the
    // rank of each staged k-mer inside its bucket's share of the tile
    uint16_t *s_rank = reinterpret_cast<uint16_t *>(s_stage + stage_cap);

    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_hist[256];
    __shared__ uint32_t s_bhist[MODE == MODE_SCAN || MODE == MODE_PART ? 256 : 1];
    __shared__ unsigned long long s_bpos[MODE == MODE_PART ? 256 : 1];
    __shared__ unsigned long long s_bcast[2];
    __shared__ unsigned long long s_boff[MODE == MODE_BLOOM ? 256 : 1];
    __shared__ unsigned long long s_bcap[MODE == MODE_BLOOM ? 256 : 1];

    const int tid = threadIdx.x, lane = tid & 31;
    // u walks the visited tiles (all tiles, or the SCAN subset a.visit)
    const uint64_t n_iter = (MODE == MODE_SCAN && a.visit) ? a.n_visit : a.n_tiles;
    uint64_t u = blockIdx.x;
    if (u >= n_iter) return;
    uint64_t t = (MODE == MODE_SCAN && a.visit) ? (uint64_t)a.visit[u] : a.tile0 + u;

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    if (MODE == MODE_SCAN) {
        s_hist[tid] = 0;
        s_bhist[tid] = 0;
    }
    if (hll_local)
        for (uint32_t i = tid; i < HLL_M; i += EXT_THREADS) s_hll[i] = 0;
    if (MODE == MODE_BLOOM) {
        s_boff[tid] = a.bloom_off[tid];
        s_bcap[tid] = a.bloom_cap[tid];
    }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(&mbar[0], BUF_BYTES);
        bulk_load(sbuf[0], a.buf + t * TILE - HALO, BUF_BYTES, &mbar[0]);
    }

    unsigned long long *flags = &a.counters[C_FLAGS];
    uint32_t iter = 0;
    bool pending_next = false;
    for (; u < n_iter; u += gridDim.x, ++iter) {
        t = (MODE == MODE_SCAN && a.visit) ? (uint64_t)a.visit[u] : a.tile0 + u;
        const int s = iter & 1;
        const uint64_t un = u + gridDim.x;
        pending_next = un < n_iter;
        if (tid == 0 && pending_next) {
            const uint64_t tn = (MODE == MODE_SCAN && a.visit) ? (uint64_t)a.visit[un] : a.tile0 + un;
            fence_proxy_async_smem();
            mbar_expect_tx(&mbar[s ^ 1], BUF_BYTES);
            bulk_load(sbuf[s ^ 1], a.buf + tn * TILE - HALO, BUF_BYTES, &mbar[s ^ 1]);
        }
        bool ok = mbar_wait(&mbar[s], (iter >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(flags, ERR_WAIT_TIMEOUT);
            if (pending_next) mbar_wait(&mbar[s ^ 1], ((iter + 1) >> 1) & 1);
            return;
        }
        const uint8_t *tb = sbuf[s];

        const uint32_t seg_id = a.tile_seg[t];
        const Seg sg = a.segs[seg_id];
        const bool first = (t == sg.first_tile);
        const uint64_t line0 = a.tile_prefix[t] - a.tile_prefix[sg.first_tile];
        const uint64_t fo = (t - sg.first_tile) * TILE;
        const KParams kp = kparams(sg.k);

        // per-segment classification
        uint64_t codes;
        uint32_t valid, nl;
        classify32(tb + HALO + 32 * tid, codes, valid, nl);
        uint32_t tot_nl;
        const uint32_t excl_nl = block_excl_scan(__popc(nl), s_warp, tot_nl);
        const uint64_t lstart = line0 + excl_nl;
        s_codes[tid + 1] = codes;
        s_rcodes[tid + 1] = pair_reverse(~codes);
        s_good[tid + 1] = valid & line_mask(lstart, nl, 1);
        if (tid == 0) {
            if (first) {
                s_codes[0] = 0;
                s_rcodes[0] = ~0ULL;
                s_good[0] = 0;
            } else {
                uint64_t c0;
                uint32_t v0, n0;
                classify32(tb, c0, v0, n0);
                s_codes[0] = c0;
                s_rcodes[0] = pair_reverse(~c0);
                s_good[0] = v0 & line_mask(line0 - __popc(n0), n0, 1);
            }
        }
        const uint64_t seg_pos = fo + 32 * (uint64_t)tid;   // file offset of this thread's segment
        if (MODE == MODE_SCAN && a.prepass) {
            // quality bytes of complete quality lines, counted from the start
            // of the 2 MiB chunk holding the line's '\n' (the reference's
            // reader sums per chunk)
            uint32_t qm = 0;
            if (seg_pos < sg.sample_end) {
                qm = line_mask(lstart, nl, 3) & ~nl;
                uint64_t lim = sg.sample_end - seg_pos;
                if (lim < 32) qm &= (1u << lim) - 1u;
                int32_t cl = a.chunk_lastnl[a.seg_chunk0[seg_id] + seg_pos / PREPASS_CHUNK];
                int64_t room = (int64_t)cl - (int64_t)(seg_pos % PREPASS_CHUNK);
                if (room <= 0) qm = 0;
                else if (room < 32) qm &= (1u << room) - 1u;
            }
            long long qs = 0;
            const uint8_t *pb = tb + HALO + 32 * tid;
            for (uint32_t m = qm; m; m &= m - 1) qs += (long long)(signed char)pb[__ffs(m) - 1];
            unsigned qn = __reduce_add_sync(FULL, (unsigned)__popc(qm));
            for (int o = 16; o > 0; o >>= 1) qs += __shfl_down_sync(FULL, qs, o);
            if (lane == 0 && qn) {
                atomicAdd(&a.qual[2 * sg.sample], (unsigned long long)qs);
                atomicAdd(&a.qual[2 * sg.sample + 1], (unsigned long long)qn);
            }
        }
        __syncthreads();

        // windows of k valid bases ending in this thread's segment
        const uint64_t g = (uint64_t)s_good[tid] | ((uint64_t)s_good[tid + 1] << 32);
        uint32_t ends = run_ends(g, kp.k);

        if (MODE == MODE_SCAN) {
            uint32_t sample_ok = 0;
            if (a.prepass && seg_pos < sg.sample_end) {
                uint64_t lim = sg.sample_end - seg_pos;
                sample_ok = lim >= 32 ? FULL : ((1u << lim) - 1u);
            }
            // keys are needed for the HyperLogLog, the bucket census (every
            // tile, or a 1-in-2^n sample of the tiles) and the pre-pass
            // sample; otherwise only the windows are counted
            const bool census = a.bucket_hist && (t & a.bucket_sample_mask) == 0;
            const uint32_t e = (a.hll || census) ? ends : (ends & sample_ok);
            // the k-mers are formed per chunk of 8 positions holding such
            // windows, rolled along the chunk, as in the staged modes (the
            // chunk list goes to the tile buffer, free once classified)
            uint32_t nq = 0;
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) nq += ((e >> (8 * q)) & 0xFFu) ? 1u : 0u;
            uint32_t n_chunks;
            const uint32_t coff = block_excl_scan(nq, s_warp, n_chunks);
            uint32_t *s_chunk = reinterpret_cast<uint32_t *>(sbuf[s]);   // <= 4 * EXT_THREADS entries
            {
                uint32_t c = coff;
#pragma unroll
                for (uint32_t q = 0; q < 4; ++q) {
                    const uint32_t e8 = (e >> (8 * q)) & 0xFFu;
                    if (e8) s_chunk[c++] = ((uint32_t)tid << 10) | (q << 8) | e8;
                }
            }
            __syncthreads();
            const uint32_t hll_base = sg.sample * HLL_M;
            for (uint32_t ci = tid; ci < n_chunks; ci += EXT_THREADS) {
                const uint32_t ch = s_chunk[ci], e8 = ch & 0xFFu;
                const uint32_t sgm = (ch >> 10) & 0xFFu, q0 = ((ch >> 8) & 3u) * 8;
                uint32_t sok = 0;   // the chunk segment's pre-pass sample positions
                if (a.prepass) {
                    const uint64_t sp = fo + 32 * (uint64_t)sgm;
                    if (sp < sg.sample_end) {
                        const uint64_t lim = sg.sample_end - sp;
                        sok = lim >= 32 ? FULL : ((1u << lim) - 1u);
                    }
                }
                const uint64_t cseg = s_codes[sgm + 1];
                uint64_t fwd, rc;
                window_words(s_codes[sgm], cseg, s_rcodes[sgm], s_rcodes[sgm + 1], q0, kp, fwd, rc);
                const uint32_t cw = (uint32_t)(cseg >> (2 * q0));
#pragma unroll
                for (uint32_t p = 0; p < 8; ++p) {
                    const uint32_t cb = (cw >> (2 * p)) & 3u;
                    fwd = (fwd >> 2) | ((uint64_t)cb << 62);
                    rc = (rc << 2) | ((uint64_t)(cb ^ 3u) << kp.fwd_shift);
                    if ((e8 >> p) & 1u) {
                        const uint64_t f = fwd & kp.topmask;
                        const unsigned long long key = f < rc ? f : rc;
                        if (hll_local) hll_add_shared(s_hll, key);
                        else if (a.hll) hll_add_sampled(a.hll + hll_base, key);
                        if (census) atomicAdd(&s_bhist[key >> 56], 1u);
                        if ((sok >> (q0 + p)) & 1u) atomicAdd(&s_hist[key >> 56], 1u);
                    }
                }
            }
            if (!a.visit || census) {
                unsigned n = __reduce_add_sync(FULL, (unsigned)__popc(ends));
                if (lane == 0 && n) atomicAdd(&a.occ[sg.sample], (unsigned long long)n);
            }
            // the chunk list went into the tile buffer through the generic
            // proxy; the next bulk copy into that buffer is an async-proxy write
            fence_proxy_async_smem();
        } else {
            // the windows are emitted per chunk of 8 positions (a quarter of a
            // segment) holding at least one window end: the chunks of all
            // segments are listed (in the tile buffer, which is free once
            // classified), then each thread rolls the forward and reverse-
            // complement words along its chunks.  Segments of header and
            // quality lines have no chunks, so working per owning segment
            // would leave most lanes idle.  One scan gives each segment its
            // first window index (low half) and first chunk (high half).
            uint32_t nq = 0;
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) nq += ((ends >> (8 * q)) & 0xFFu) ? 1u : 0u;
            uint32_t packed_tot;
            const uint32_t packed = block_excl_scan((uint32_t)__popc(ends) | (nq << 16), s_warp, packed_tot);
            const uint32_t tot = packed_tot & 0xFFFFu, n_chunks = packed_tot >> 16;
            uint32_t *s_chunk = reinterpret_cast<uint32_t *>(sbuf[s]);   // <= 4 * EXT_THREADS entries
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
            if (MODE == MODE_PART) s_bhist[tid] = 0;
            __syncthreads();
            const uint32_t blo = a.bucket_lo, bhi = a.bucket_hi ? a.bucket_hi : N_BUCKETS;
            for (uint32_t base = 0; base < tot; base += stage_cap) {
                const uint32_t nr = min(stage_cap, tot - base);
                for (uint32_t ci = tid; ci < n_chunks; ci += EXT_THREADS) {
                    const uint32_t ch = s_chunk[ci], e8 = ch & 0xFFu;
                    uint32_t idx = ch >> 18;
                    if (idx >= base + nr || idx + (uint32_t)__popc(e8) <= base) continue;   // not in this round
                    const uint32_t sgm = (ch >> 10) & 0xFFu, q0 = ((ch >> 8) & 3u) * 8;
                    const uint64_t cur = s_codes[sgm + 1];
                    uint64_t fwd, rc;
                    window_words(s_codes[sgm], cur, s_rcodes[sgm], s_rcodes[sgm + 1], q0, kp, fwd, rc);
                    const uint32_t cw = (uint32_t)(cur >> (2 * q0));
#pragma unroll
                    for (uint32_t p = 0; p < 8; ++p) {
                        const uint32_t c = (cw >> (2 * p)) & 3u;
                        fwd = (fwd >> 2) | ((uint64_t)c << 62);
                        rc = (rc << 2) | ((uint64_t)(c ^ 3u) << kp.fwd_shift);
                        if ((e8 >> p) & 1u) {
                            if (idx >= base && idx < base + nr) {
                                const uint64_t f = fwd & kp.topmask;
                                const unsigned long long key = f < rc ? f : rc;
                                s_stage[idx - base] = key;
                                if (MODE == MODE_PART) {
                                    // rank inside the tile's share of its bucket (a
                                    // pass of a multi-pass job keeps only its range)
                                    const uint32_t bk = (uint32_t)(key >> 56);
                                    s_rank[idx - base] =
                                        (bk >= blo && bk < bhi) ? (uint16_t)atomicAdd(&s_bhist[bk], 1u) : (uint16_t)0xFFFFu;
                                }
                            }
                            ++idx;
                        }
                    }
                }
                __syncthreads();
                if (MODE == MODE_INSERT) {
                    const TableRef tr = a.tables[sg.sample];
                    for (uint32_t r0 = 0; r0 < nr; r0 += EXT_THREADS) {
                        uint32_t i = r0 + tid;
                        bool act = i < nr;
                        warp_insert(act, act ? s_stage[i] : EMPTY_KEY, tr, a.max_probe, flags);
                    }
                } else if (MODE == MODE_PART) {
                    // scatter into the root-prefix buckets (ranks were taken
                    // as the k-mers were formed), one cursor update per bucket;
                    // the round's k-mers are reordered by bucket in shared
                    // memory, so that consecutive threads store consecutive
                    // addresses of one bucket's region (a warp's store then
                    // touches a few sectors instead of one per k-mer)
                    uint32_t tot_b;
                    const uint32_t c = s_bhist[tid];
                    s_bhist[tid] = 0;   // the next round's ranks (emission is done)
                    const uint32_t bstart = block_excl_scan(c, s_warp, tot_b);
                    s_hist[tid] = bstart;
                    // this tile's range of bucket tid: the cursor update is in
                    // flight during the reorder and consumed only after it
                    const unsigned long long cur = c ? atomicAdd(&a.bucket_cursor[tid], (unsigned long long)c) : 0ull;
                    __syncthreads();
                    unsigned long long kr[SCAP / EXT_THREADS];
#pragma unroll
                    for (uint32_t r = 0; r < SCAP / EXT_THREADS; ++r) {
                        const uint32_t i = tid + r * EXT_THREADS;
                        if (i < nr && s_rank[i] != 0xFFFFu) {
                            kr[r] = s_stage[i];
                            s_rank[i] = (uint16_t)(s_hist[(uint32_t)(kr[r] >> 56)] + s_rank[i]);
                        }
                    }
                    __syncthreads();
#pragma unroll
                    for (uint32_t r = 0; r < SCAP / EXT_THREADS; ++r) {
                        const uint32_t i = tid + r * EXT_THREADS;
                        if (i < nr && s_rank[i] != 0xFFFFu) s_stage[s_rank[i]] = kr[r];
                    }
                    // destination of sorted index i of bucket b: s_bpos[b] + i,
                    // written while i < s_hist[b] (inside the bucket's region
                    // and the list: a bucket that outgrows its estimated
                    // region is reported by its cursor and redone)
                    {
                        const unsigned long long bp = c ? a.bucket_base[tid] + cur - bstart : 0ull;
                        s_bpos[tid] = bp;
                        const unsigned long long lim = a.bucket_end[tid] < a.list_cap ? a.bucket_end[tid] : a.list_cap;
                        s_hist[tid] = lim > bp ? (uint32_t)(lim - bp < 0xFFFFFFFFull ? lim - bp : 0xFFFFFFFFull) : 0u;
                    }
                    __syncthreads();
                    for (uint32_t i = tid; i < tot_b; i += EXT_THREADS) {
                        const unsigned long long key = s_stage[i];
                        const uint32_t b = (uint32_t)(key >> 56);
                        if (i < s_hist[b]) a.list[s_bpos[b] + i] = key;
                    }
                } else if (MODE == MODE_EMIT) {
                    if (tid == 0) s_bcast[0] = atomicAdd(&a.counters[C_EMIT_LEN], (unsigned long long)nr);
                    __syncthreads();
                    const unsigned long long b0 = s_bcast[0];
                    for (uint32_t i = tid; i < nr; i += EXT_THREADS) {
                        if (b0 + i < a.list_cap) a.list[b0 + i] = s_stage[i];
                        else atomicOr(flags, ERR_LIST_FULL);
                    }
                } else if (MODE == MODE_BLOOM) {
                    uint32_t firsts = 0, highs = 0;
                    for (uint32_t r = 0, i = tid; i < nr; ++r, i += EXT_THREADS) {
                        unsigned long long key = s_stage[i];
                        uint32_t p = (uint32_t)(key >> 56);
                        uint64_t block, m;
                        bloom_probe(key, s_bcap[p], block, m);
                        unsigned long long *cell = a.bloom_bits + s_boff[p] + 2 * block;
                        // ConcurrentBloomFilter::insert_prepared (src/BloomFilter.h:233-273)
                        bool first_occ = false;
                        unsigned long long bf1 = __ldcg(&cell[0]);
                        if ((bf1 & m) != m) {
                            unsigned long long bf2 = __ldcg(&cell[1]);
                            if ((bf2 & m) == m) {
                                atomicOr(&cell[0], (unsigned long long)m);
                            } else {
                                unsigned long long old2 = atomicOr(&cell[1], (unsigned long long)m);
                                if ((old2 & m) == m) atomicOr(&cell[0], (unsigned long long)m);
                                else first_occ = true;
                            }
                        }
                        if (first_occ) firsts |= 1u << r;
                        else {
                            highs |= 1u << r;
                            hll_add(a.hll_high, key);
                        }
                    }
                    uint32_t tf, th;
                    const uint32_t of = block_excl_scan(__popc(firsts), s_warp, tf);
                    const uint32_t oh = block_excl_scan(__popc(highs), s_warp, th);
                    if (tid == 0) {
                        s_bcast[0] = atomicAdd(&a.counters[C_LOW_LEN], (unsigned long long)tf);
                        s_bcast[1] = atomicAdd(&a.counters[C_HIGH_LEN], (unsigned long long)th);
                    }
                    __syncthreads();
                    const unsigned long long lb = s_bcast[0] + of, hb = s_bcast[1] + oh;
                    uint32_t nf = 0, nh = 0;
                    for (uint32_t r = 0, i = tid; i < nr; ++r, i += EXT_THREADS) {
                        unsigned long long key = s_stage[i];
                        if ((firsts >> r) & 1u) {
                            unsigned long long pos = lb + nf++;
                            if (pos < a.list_cap) a.list[pos] = key;
                            else atomicOr(flags, ERR_LIST_FULL);
                        } else {
                            unsigned long long pos = hb + nh++;
                            if (pos < a.list_cap) a.list[a.list_cap - 1 - pos] = key;
                            else atomicOr(flags, ERR_LIST_FULL);
                        }
                    }
                }
                __syncthreads();
            }
            // the chunk list went into the tile buffer through the generic
            // proxy; the next bulk copy into that buffer is an async-proxy write
            fence_proxy_async_smem();
        }
        __syncthreads();
    }

    if (MODE == MODE_SCAN && a.prepass) {
        // one file-sample per job in Bloom mode; the histogram belongs to sample 0
        uint32_t v = s_hist[tid];
        if (v) atomicAdd(&a.prefix_hist[tid], v);
    }
    if (MODE == MODE_SCAN && a.bucket_hist) {
        uint32_t v = s_bhist[tid];
        if (v) atomicAdd(&a.bucket_hist[tid], (unsigned long long)v);
    }
    if (hll_local) {
        for (uint32_t i = tid; i < HLL_M; i += EXT_THREADS) {
            uint32_t v = s_hll[i];
            if (v > *(volatile uint32_t *)&a.hll[i]) atomicMax(&a.hll[i], v);
        }
    }
}

// ---------------------------------------------------------------------------
// table phases
// ---------------------------------------------------------------------------

__global__ void k_init_slots(Slot *slots, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        slots[i].key = EMPTY_KEY;
        slots[i].count = 0;
        slots[i].pad = 0;
    }
}

__global__ void k_count_keys(const Slot *slots, uint64_t n, unsigned long long *out)
{
    unsigned c = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += slots[i].key != EMPTY_KEY;
    c = __reduce_add_sync(FULL, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

__global__ void k_fill_u64(unsigned long long *p, uint64_t n, unsigned long long v)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void __launch_bounds__(256) k_insert_list(const unsigned long long *keys, uint64_t n, TableRef t,
                                                     uint32_t max_probe, unsigned long long *counters)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // whole warps iterate together so __match_any_sync sees all lanes
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        uint64_t i = base + (threadIdx.x & 31);
        bool act = i < n;
        warp_insert(act, act ? keys[i] : EMPTY_KEY, t, max_probe, &counters[C_FLAGS]);
    }
}

__global__ void k_insert_pairs(const unsigned long long *keys, const uint32_t *counts, uint64_t n, TableRef t,
                               uint32_t max_probe, unsigned long long *counters)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (!table_add(t.slots, t.mask, keys[i], counts[i], max_probe)) atomicOr(&counters[C_FLAGS], ERR_TABLE_FULL);
}

// Block-aggregated append of (string key, count) records.
__device__ __forceinline__ void append_records(bool keep, unsigned long long skey, uint32_t c,
                                               unsigned long long *rec_keys, uint32_t *rec_counts,
                                               uint64_t rec_cap, unsigned long long *counters,
                                               uint32_t *s_warp, unsigned long long *s_base)
{
    uint32_t tot;
    uint32_t off = block_excl_scan(keep ? 1u : 0u, s_warp, tot);
    if (threadIdx.x == 0) *s_base = tot ? atomicAdd(&counters[C_REC_LEN], (unsigned long long)tot) : 0ull;
    __syncthreads();
    unsigned long long pos = *s_base + off;
    if (keep) {
        if (pos < rec_cap) {
            rec_keys[pos] = skey;
            rec_counts[pos] = c;
        } else {
            atomicOr(&counters[C_FLAGS], ERR_RECORDS_FULL);
        }
    }
    __syncthreads();
}

// FIRST occurrences: a hit adds the low-list occurrence to the table count
// (the tools' merge, LowFrequencyQueryThreadPool::process_block); a miss is a
// k-mer whose only occurrence is this one.
__global__ void __launch_bounds__(256) k_merge_low(const unsigned long long *keys, uint64_t n, TableRef t,
                                                   uint32_t max_probe, uint32_t min_count, uint32_t max_count,
                                                   unsigned long long *rec_keys, uint32_t *rec_counts,
                                                   uint64_t rec_cap, unsigned long long *counters)
{
    __shared__ uint32_t s_warp[8];
    __shared__ unsigned long long s_base;
    const bool want1 = (min_count <= 1 && 1 <= max_count);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t rounds = (n + stride - 1) / stride;
    for (uint64_t r = 0; r < rounds; ++r) {
        uint64_t i = r * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        bool miss = false;
        unsigned long long key = 0;
        if (i < n) {
            key = keys[i];
            bool ovf = false;
            Slot *sl = table_find(t.slots, t.mask, key, max_probe, ovf);
            if (ovf) atomicOr(&counters[C_FLAGS], ERR_TABLE_FULL);
            if (sl) atomicAdd(&sl->count, 1u);
            else miss = true;
        }
        unsigned m = __reduce_add_sync(FULL, miss ? 1u : 0u);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(&counters[C_LOW_ONLY], (unsigned long long)m);
        append_records(miss && want1, pair_reverse(key), 1u, rec_keys, rec_counts, rec_cap, counters, s_warp, &s_base);
    }
}

__global__ void __launch_bounds__(256) k_compact(TableRef t, uint64_t cap, uint32_t count_max, uint32_t min_count,
                                                 uint32_t max_count, unsigned long long *rec_keys,
                                                 uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist,
                                                 uint32_t *ovf, uint64_t ovf_cap, unsigned long long *counters)
{
    __shared__ uint32_t s_warp[8];
    __shared__ unsigned long long s_base;
    __shared__ uint32_t s_hist[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t rounds = (cap + stride - 1) / stride;
    uint32_t distinct = 0;
    for (uint64_t r = 0; r < rounds; ++r) {
        uint64_t i = r * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        bool keep = false;
        unsigned long long skey = 0;
        uint32_t c = 0;
        if (i < cap) {
            Slot sl = t.slots[i];
            if (sl.key != EMPTY_KEY) {
                ++distinct;
                c = sl.count < count_max ? sl.count : count_max;
                if (c < 2048) atomicAdd(&s_hist[c], 1u);
                else if (c < HIST_BINS) atomicAdd(&hist[c], 1ull);
                else {
                    unsigned long long p = atomicAdd(&counters[C_OVF_LEN], 1ull);
                    if (p < ovf_cap) ovf[p] = c;
                    else atomicOr(&counters[C_FLAGS], ERR_HIST_OVERFLOW_FULL);
                }
                keep = (c >= min_count && c <= max_count);
                skey = pair_reverse(sl.key);
            }
        }
        append_records(keep, skey, c, rec_keys, rec_counts, rec_cap, counters, s_warp, &s_base);
    }
    unsigned d = __reduce_add_sync(FULL, distinct);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(&counters[C_DISTINCT], (unsigned long long)d);
    __syncthreads();
    for (int i = threadIdx.x; i < 2048; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
}

// Compaction of one table (or one bucket arena) in slot order, without a
// global atomic per record or per chunk.  The slots are cut into chunks of
// ORDERED_CHUNK, one per block at a time; warp w owns 256 consecutive slots
// of a chunk, 8 per lane.  count_only: chunk_keep[c] = records chunk c keeps
// and C_DISTINCT += the occupied slots.  Otherwise chunk c writes its records
// from chunk_pos[c] (the exclusive scan of chunk_keep) on, in slot order, so
// a bucket arena's records come out grouped by bucket, and adds every count
// to the histogram.
constexpr uint32_t ORDERED_CHUNK = 2048;
constexpr uint32_t ORDERED_PER_LANE = ORDERED_CHUNK / 256;

__global__ void __launch_bounds__(256) k_compact_ordered(const Slot *slots, uint64_t cap, uint32_t count_max,
                                                         uint32_t min_count, uint32_t max_count,
                                                         uint32_t *chunk_keep, const unsigned long long *chunk_pos,
                                                         unsigned long long *rec_keys, uint32_t *rec_counts,
                                                         uint64_t rec_cap, unsigned long long *hist, uint32_t *ovf,
                                                         uint64_t ovf_cap, unsigned long long *counters, int count_only)
{
    __shared__ uint32_t s_hist[2048];
    __shared__ uint32_t s_wk[2][8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (!count_only)
        for (int i = tid; i < 2048; i += 256) s_hist[i] = 0;
    __syncthreads();
    const uint64_t n_chunks = (cap + ORDERED_CHUNK - 1) / ORDERED_CHUNK;
    const uint32_t lt = lanemask_lt();
    uint32_t present = 0, par = 0;
    bool full = false;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x, par ^= 1u) {
        const uint64_t w0 = c * ORDERED_CHUNK + (uint64_t)warp * (32 * ORDERED_PER_LANE);
        unsigned long long key[ORDERED_PER_LANE];
        uint32_t cnt[ORDERED_PER_LANE];
#pragma unroll
        for (uint32_t r = 0; r < ORDERED_PER_LANE; ++r) {
            const uint64_t i = w0 + r * 32 + lane;
            key[r] = EMPTY_KEY;
            cnt[r] = 0;
            if (i < cap) {
                const Slot sl = slots[i];
                key[r] = sl.key;
                cnt[r] = sl.count < count_max ? sl.count : count_max;
            }
        }
        uint32_t keep = 0, wtot = 0;
#pragma unroll
        for (uint32_t r = 0; r < ORDERED_PER_LANE; ++r) {
            const bool occ = key[r] != EMPTY_KEY;
            present += occ ? 1u : 0u;
            const bool k = occ && cnt[r] >= min_count && cnt[r] <= max_count;
            keep |= (k ? 1u : 0u) << r;
            wtot += (uint32_t)__popc(__ballot_sync(FULL, k));
        }
        if (lane == 0) s_wk[par][warp] = wtot;
        __syncthreads();
        uint32_t before = 0, ctot = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint32_t v = s_wk[par][w];
            before += w < warp ? v : 0u;
            ctot += v;
        }
        if (count_only) {
            if (tid == 0) chunk_keep[c] = ctot;
            continue;
        }
        unsigned long long pos = chunk_pos[c] + before;
#pragma unroll
        for (uint32_t r = 0; r < ORDERED_PER_LANE; ++r) {
            const bool k = (keep >> r) & 1u;
            const uint32_t b = __ballot_sync(FULL, k);
            if (k) {
                const unsigned long long q = pos + (uint32_t)__popc(b & lt);
                if (q < rec_cap) {
                    rec_keys[q] = pair_reverse(key[r]);
                    rec_counts[q] = cnt[r];
                } else {
                    full = true;
                }
            }
            pos += (uint32_t)__popc(b);
            if (key[r] != EMPTY_KEY) {
                const uint32_t cc = cnt[r];
                if (cc < 2048) atomicAdd(&s_hist[cc], 1u);
                else if (cc < HIST_BINS) atomicAdd(&hist[cc], 1ull);
                else {
                    const unsigned long long p = atomicAdd(&counters[C_OVF_LEN], 1ull);
                    if (p < ovf_cap) ovf[p] = cc;
                    else atomicOr(&counters[C_FLAGS], ERR_HIST_OVERFLOW_FULL);
                }
            }
        }
    }
    if (full) atomicOr(&counters[C_FLAGS], ERR_RECORDS_FULL);
    if (count_only) {
        const unsigned d = __reduce_add_sync(FULL, present);
        if (lane == 0 && d) atomicAdd(&counters[C_DISTINCT], (unsigned long long)d);
        return;
    }
    __syncthreads();
    for (int i = tid; i < 2048; i += 256)
        if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
}

// Batched jobs keep all samples' tables in one slot arena.  Sample s owns
// slots [slot_base, slot_base + slot_cap), cut into chunks of COMPACT_CHUNK
// slots; chunk0[s] is the index of its first chunk (chunk0[n] = all chunks),
// so every chunk belongs to one sample.
constexpr uint32_t COMPACT_CHUNK = 4096;

__device__ __forceinline__ uint32_t sample_of_chunk(const uint32_t *s_chunk0, uint32_t n, uint64_t c)
{
    uint32_t lo = 0, hi = n;   // last sample whose first chunk is <= c
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_chunk0[mid] <= c) lo = mid; else hi = mid;
    }
    return lo;
}

// count_only: chunk_keep[c] = records chunk c keeps, distinct[s] += its
// occupied slots.  Otherwise chunk c writes its records from
// rec_keys[chunk_pos[c]] on (chunk_pos = exclusive scan of chunk_keep, so the
// samples' records are packed one after the other in sample order) and adds
// its counts to the sample's histogram through a shared-memory histogram.
__global__ void __launch_bounds__(256) k_compact_chunks(const Slot *slots, const SampleCfg *cfg,
                                                        const uint32_t *chunk0, uint32_t n_samples,
                                                        uint64_t n_chunks, uint32_t *chunk_keep,
                                                        const unsigned long long *chunk_pos,
                                                        unsigned long long *rec_keys, uint32_t *rec_counts,
                                                        unsigned long long *hist, unsigned long long *ovf,
                                                        uint64_t ovf_cap, unsigned long long *distinct,
                                                        unsigned long long *counters, int count_only)
{
    extern __shared__ uint32_t s_chunk0[];   // n_samples + 1
    __shared__ uint32_t s_hist[2048];
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_red[2][8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i <= n_samples; i += 256) s_chunk0[i] = chunk0[i];
    for (uint32_t i = tid; i < 2048; i += 256) s_hist[i] = 0;
    __syncthreads();
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const uint32_t smp = sample_of_chunk(s_chunk0, n_samples, c);
        const SampleCfg sc = cfg[smp];
        const uint64_t lo = sc.slot_base + (c - s_chunk0[smp]) * COMPACT_CHUNK;
        const uint64_t end = sc.slot_base + sc.slot_cap;
        const uint64_t hi = lo + COMPACT_CHUNK < end ? lo + COMPACT_CHUNK : end;
        if (count_only) {
            uint32_t present = 0, keep = 0;
            for (uint64_t i = lo + tid; i < hi; i += 256) {
                const Slot sl = slots[i];
                if (sl.key == EMPTY_KEY) continue;
                ++present;
                const uint32_t cnt = sl.count < sc.count_max ? sl.count : sc.count_max;
                keep += (cnt >= sc.min_count && cnt <= sc.max_count);
            }
            present = __reduce_add_sync(FULL, present);
            keep = __reduce_add_sync(FULL, keep);
            if (lane == 0) { s_red[0][warp] = present; s_red[1][warp] = keep; }
            __syncthreads();
            if (tid == 0) {
                uint32_t p = 0, k = 0;
                for (int w = 0; w < 8; ++w) { p += s_red[0][w]; k += s_red[1][w]; }
                chunk_keep[c] = k;
                if (p) atomicAdd(&distinct[smp], (unsigned long long)p);
            }
            __syncthreads();
            continue;
        }
        unsigned long long run = chunk_pos[c];
        for (uint64_t base = lo; base < hi; base += 256) {
            const uint64_t i = base + tid;
            bool keep = false;
            uint32_t cnt = 0;
            unsigned long long key = EMPTY_KEY;
            if (i < hi) {
                const Slot sl = slots[i];
                key = sl.key;
                if (key != EMPTY_KEY) {
                    cnt = sl.count < sc.count_max ? sl.count : sc.count_max;
                    if (cnt < 2048) atomicAdd(&s_hist[cnt], 1u);
                    else if (cnt < HIST_BINS_BATCH) atomicAdd(&hist[(uint64_t)smp * HIST_BINS_BATCH + cnt], 1ull);
                    else {
                        const unsigned long long p = atomicAdd(&counters[C_OVF_LEN], 1ull);
                        if (p < ovf_cap) ovf[p] = ((unsigned long long)smp << 32) | cnt;
                        else atomicOr(&counters[C_FLAGS], ERR_HIST_OVERFLOW_FULL);
                    }
                    keep = cnt >= sc.min_count && cnt <= sc.max_count;
                }
            }
            uint32_t tot;
            const uint32_t off = block_excl_scan(keep ? 1u : 0u, s_warp, tot);
            if (keep) {
                rec_keys[run + off] = pair_reverse(key);
                rec_counts[run + off] = cnt;
            }
            run += tot;
        }
        __syncthreads();
        for (uint32_t b = tid; b < 2048; b += 256) {
            const uint32_t v = s_hist[b];
            if (v) {
                atomicAdd(&hist[(uint64_t)smp * HIST_BINS_BATCH + b], (unsigned long long)v);
                s_hist[b] = 0;
            }
        }
        __syncthreads();
    }
}

__global__ void k_pair_reverse(unsigned long long *keys, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = pair_reverse(keys[i]);
}

// ---------------------------------------------------------------------------
// scan
// ---------------------------------------------------------------------------

constexpr uint32_t SCAN_ITEMS = 8;
constexpr uint32_t SCAN_BLOCK = 256 * SCAN_ITEMS;

__global__ void __launch_bounds__(256) k_scan_reduce(const uint32_t *in, uint64_t n, unsigned long long *sums)
{
    __shared__ unsigned long long s[8];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_BLOCK;
    unsigned long long acc = 0;
    for (uint32_t j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + j * 256 + threadIdx.x;
        if (i < n) acc += in[i];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < 8; ++i) t += s[i];
        sums[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_scan_top(unsigned long long *sums, uint64_t nb)
{
    __shared__ unsigned long long s[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t b0 = 0; b0 < nb; b0 += 1024) {
        uint64_t i = b0 + threadIdx.x;
        unsigned long long v = i < nb ? sums[i] : 0, x = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = s[lane];
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(FULL, w, o);
                if (lane >= o) w += y;
            }
            s[lane] = w;
        }
        __syncthreads();
        unsigned long long excl = carry + (warp ? s[warp - 1] : 0) + x - v;
        if (i < nb) sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += s[31];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_scan_down(const uint32_t *in, uint64_t n, const unsigned long long *sums,
                                                   unsigned long long *out)
{
    __shared__ unsigned long long s[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_BLOCK;
    // each thread owns SCAN_ITEMS consecutive items
    uint32_t v[SCAN_ITEMS];
    unsigned long long local = 0;
    for (uint32_t j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + threadIdx.x * SCAN_ITEMS + j;
        v[j] = i < n ? in[i] : 0;
        local += v[j];
    }
    unsigned long long x = local;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long c = 0;
        for (int i = 0; i < 8; ++i) { unsigned long long t = s[i]; s[i] = c; c += t; }
    }
    __syncthreads();
    unsigned long long run = sums[blockIdx.x] + s[warp] + x - local;
    for (uint32_t j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + threadIdx.x * SCAN_ITEMS + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
}

// ---------------------------------------------------------------------------
// radix sort (LSD, 8-bit digits)
// ---------------------------------------------------------------------------

constexpr uint32_t RS_THREADS = 256;
constexpr uint32_t RS_ITEMS = 16;
constexpr uint32_t RS_TILE = RS_THREADS * RS_ITEMS;   // 4096
constexpr uint32_t RS_WARP_ITEMS = 32 * RS_ITEMS;     // 512 contiguous items per warp

__global__ void __launch_bounds__(RS_THREADS) k_radix_count(const unsigned long long *keys, const SortTile *tiles,
                                                            uint32_t shift, uint32_t *counts)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const SortTile tl = tiles[blockIdx.x];
    for (uint32_t j = 0; j < RS_ITEMS; ++j) {
        uint64_t i = tl.begin + j * RS_THREADS + threadIdx.x;
        if (i < tl.end) atomicAdd(&h[(keys[i] >> shift) & 255], 1u);
    }
    __syncthreads();
    counts[tl.cbase + (uint64_t)threadIdx.x * tl.stride] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const unsigned long long *kin, const uint32_t *vin,
                                                              unsigned long long *kout, uint32_t *vout,
                                                              const SortTile *tiles, uint32_t shift,
                                                              const unsigned long long *offsets)
{
    extern __shared__ __align__(16) uint8_t rs_smem[];
    unsigned long long *s_keys = reinterpret_cast<unsigned long long *>(rs_smem);       // RS_TILE
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + RS_TILE);                   // RS_TILE
    uint32_t *s_wcnt = s_vals + RS_TILE;                                                 // 8 x 256
    uint32_t *s_start = s_wcnt + 8 * 256;                                                // 256
    __shared__ uint32_t s_warp[8];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 8 * 256; i += RS_THREADS) s_wcnt[i] = 0;
    __syncthreads();

    const SortTile tl = tiles[blockIdx.x];
    const uint64_t tile_base = tl.begin;
    const uint64_t tile_n = tl.end - tl.begin;
    unsigned long long k[RS_ITEMS];
    uint32_t v[RS_ITEMS];
    uint16_t rank[RS_ITEMS];
    uint16_t dig[RS_ITEMS];
    uint32_t *wc = s_wcnt + warp * 256;
#pragma unroll
    for (uint32_t r = 0; r < RS_ITEMS; ++r) {
        uint64_t li = warp * RS_WARP_ITEMS + r * 32 + lane;
        bool act = li < tile_n;
        k[r] = act ? kin[tile_base + li] : 0;
        v[r] = act ? vin[tile_base + li] : 0;
        uint32_t d = act ? (uint32_t)((k[r] >> shift) & 255) : 256u;
        uint32_t peers = __match_any_sync(FULL, d);
        uint32_t before = __popc(peers & lanemask_lt());
        uint32_t cnt = act ? wc[d] : 0;
        __syncwarp();
        if (act && before == 0) wc[d] = cnt + __popc(peers);
        __syncwarp();
        rank[r] = (uint16_t)(cnt + before);
        dig[r] = (uint16_t)d;
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, total for the tile
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        uint32_t c = s_wcnt[w * 256 + tid];
        s_wcnt[w * 256 + tid] = run;
        run += c;
    }
    uint32_t tot;
    uint32_t start = block_excl_scan(run, s_warp, tot);
    s_start[tid] = start;
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < RS_ITEMS; ++r) {
        if (dig[r] < 256) {
            uint32_t pos = s_start[dig[r]] + s_wcnt[warp * 256 + dig[r]] + rank[r];
            s_keys[pos] = k[r];
            s_vals[pos] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
        unsigned long long key = s_keys[i];
        uint32_t d = (uint32_t)((key >> shift) & 255);
        unsigned long long dst = offsets[tl.cbase + (uint64_t)d * tl.stride] + tl.adjust + (i - s_start[d]);
        kout[dst] = key;
        vout[dst] = s_vals[i];
    }
}

// ---------------------------------------------------------------------------
// radix sort of one segment, one kernel per pass (single-pass prefix with
// decoupled look-back: every tile publishes its per-digit counts, then adds up
// its predecessors' counts until it meets a published inclusive prefix)
// ---------------------------------------------------------------------------

constexpr uint32_t OS_MAX_PASSES = 8;
constexpr int LB_VALUE_BITS = 40;                                // count field of a look-back word
constexpr unsigned long long LB_VALUE_MASK = (1ull << LB_VALUE_BITS) - 1;

// With segment tiles (segmented sort), each tile belongs to one segment: the
// look-back stops at the segment's first tile, and the digit offsets come from
// that segment's histograms and start.
struct OsTile {
    uint64_t begin, end;    // key range of the tile
    uint64_t seg_start;     // first key of the tile's segment
    uint32_t first_tile;    // index of the segment's first tile
    uint32_t seg;           // segment index (its histograms)
    uint32_t passes;        // 8-bit passes the segment needs (it sits out later ones)
    uint32_t pad;
};

// Digit histograms of every pass in one read of the keys.
__global__ void __launch_bounds__(256) k_radix_hist_all(const unsigned long long *keys, uint64_t n, uint32_t passes,
                                                        unsigned long long *hist)
{
    __shared__ uint32_t h[OS_MAX_PASSES * 256];
    for (uint32_t i = threadIdx.x; i < OS_MAX_PASSES * 256; i += 256) h[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (uint64_t)gridDim.x * 256) {
        const unsigned long long k = __ldcs(&keys[i]);
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&h[p * 256 + (uint32_t)((k >> (8 * p)) & 255)], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * 256; i += 256)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

// Digit histograms of every pass per segment: each block takes a run of
// consecutive tiles and adds its counts to the segment's histograms when the
// segment changes and at the end.
__global__ void __launch_bounds__(256) k_radix_hist_seg(const unsigned long long *keys, const OsTile *tiles,
                                                        uint64_t n_tiles, uint64_t tiles_per_block, uint32_t passes,
                                                        unsigned long long *hist)
{
    __shared__ uint32_t h[OS_MAX_PASSES * 256];
    const uint64_t t0 = blockIdx.x * tiles_per_block;
    const uint64_t t1 = t0 + tiles_per_block < n_tiles ? t0 + tiles_per_block : n_tiles;
    if (t0 >= t1) return;
    for (uint32_t i = threadIdx.x; i < OS_MAX_PASSES * 256; i += 256) h[i] = 0;
    uint32_t seg = tiles[t0].seg;
    __syncthreads();
    for (uint64_t t = t0; t < t1; ++t) {
        const OsTile tl = tiles[t];
        if (tl.seg != seg) {
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < passes * 256; i += 256) {
                if (h[i]) atomicAdd(&hist[(uint64_t)seg * OS_MAX_PASSES * 256 + i], (unsigned long long)h[i]);
                h[i] = 0;
            }
            seg = tl.seg;
            __syncthreads();
        }
        // lanes with the same digit add once (the high digits of short keys
        // are all zero, and 32 lanes adding to one bin would serialize)
        const uint32_t np = tl.passes < passes ? tl.passes : passes;
        for (uint64_t b = tl.begin; b < tl.end; b += 256) {
            const uint64_t i = b + threadIdx.x;
            const bool act = i < tl.end;
            const unsigned long long k = act ? __ldcs(&keys[i]) : 0;
            for (uint32_t p = 0; p < np; ++p) {
                const uint32_t d = act ? (uint32_t)((k >> (8 * p)) & 255) : 256u;
                const uint32_t peers = __match_any_sync(FULL, d);
                if (act && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[p * 256 + d], __popc(peers));
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < passes * 256; i += 256)
        if (h[i]) atomicAdd(&hist[(uint64_t)seg * OS_MAX_PASSES * 256 + i], (unsigned long long)h[i]);
}

// Exclusive prefix sum over the block's 256 threads of 64-bit values.
__device__ __forceinline__ unsigned long long block_excl_scan64(unsigned long long v, unsigned long long *s_w)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    unsigned long long base = 0;
    for (int w = 0; w < warp; ++w) base += s_w[w];
    __syncthreads();
    return base + x - v;
}

// One LSD pass over 8 bits at `shift`.  Tiles are taken in launch order from
// tile_ctr, so every tile a block waits on belongs to a block that is already
// running and publishes its counts before it waits itself.  Look-back words:
// bits 40.. hold the tag (2*pass+1: tile count, 2*pass+2: inclusive prefix),
// bits 0..39 the value; the array starts zeroed, and older passes' tags are
// smaller, so it is reused across passes.  A wait that exceeds the spin limit
// sets ERR_WAIT_TIMEOUT in *flags and carries on.
__global__ void __launch_bounds__(RS_THREADS, 3) k_radix_onesweep(const unsigned long long *kin, const uint32_t *vin,
                                                                  unsigned long long *kout, uint32_t *vout,
                                                                  uint64_t n, uint32_t pass,
                                                                  const unsigned long long *hist,
                                                                  unsigned long long *look, unsigned int *tile_ctr,
                                                                  unsigned long long *flags, const OsTile *tiles)
{
    extern __shared__ __align__(16) uint8_t rs_smem[];
    unsigned long long *s_keys = reinterpret_cast<unsigned long long *>(rs_smem);       // RS_TILE
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + RS_TILE);                   // RS_TILE
    uint32_t *s_wcnt = s_vals + RS_TILE;                                                 // 8 x 256
    __shared__ uint32_t s_start[256], s_warp[8], s_tile;
    __shared__ unsigned long long s_dst[256], s_w64[8];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t shift = 8 * pass;
    if (tid == 0) s_tile = atomicAdd(&tile_ctr[pass], 1u);
    for (int i = tid; i < 8 * 256; i += RS_THREADS) s_wcnt[i] = 0;
    __syncthreads();
    const uint64_t j = s_tile;
    uint64_t base, first = 0, seg_start = 0;
    uint32_t tile_n;
    const unsigned long long *hp = hist;
    if (tiles) {
        const OsTile tl = tiles[j];
        base = tl.begin;
        tile_n = (uint32_t)(tl.end - tl.begin);
        first = tl.first_tile;
        seg_start = tl.seg_start;
        hp = hist + (uint64_t)tl.seg * OS_MAX_PASSES * 256;
        if (pass >= tl.passes) return;   // the segment is sorted already (no tile of it waits or is waited on)
    } else {
        base = j * RS_TILE;
        tile_n = (uint32_t)(n - base < RS_TILE ? n - base : RS_TILE);
    }

    // stable rank of every key among the tile's keys with the same digit
    unsigned long long k[RS_ITEMS];
    uint32_t v[RS_ITEMS];
    uint32_t rd[RS_ITEMS];   // rank << 16 | digit (digit 256: no key)
    uint32_t *wc = s_wcnt + warp * 256;
#pragma unroll
    for (uint32_t r = 0; r < RS_ITEMS; ++r) {
        const uint32_t li = warp * RS_WARP_ITEMS + r * 32 + lane;
        const bool act = li < tile_n;
        k[r] = act ? __ldcs(&kin[base + li]) : 0;
        v[r] = act ? __ldcs(&vin[base + li]) : 0u;
        const uint32_t d = act ? (uint32_t)((k[r] >> shift) & 255) : 256u;
        const uint32_t peers = __match_any_sync(FULL, d);
        const uint32_t before = __popc(peers & lanemask_lt());
        const uint32_t cnt = act ? wc[d] : 0;
        __syncwarp();
        if (act && before == 0) wc[d] = cnt + __popc(peers);
        __syncwarp();
        rd[r] = ((cnt + before) << 16) | d;
    }
    __syncthreads();
    uint32_t own = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const uint32_t c = s_wcnt[w * 256 + tid];
        s_wcnt[w * 256 + tid] = own;
        own += c;
    }
    // publish this tile's count of digit tid, then find the keys of digit tid
    // in the tiles before it
    const unsigned long long tag_a = 2ull * pass + 1, tag_i = 2ull * pass + 2;
    volatile unsigned long long *mine = look + j * 256 + tid;
    *mine = ((j == first ? tag_i : tag_a) << LB_VALUE_BITS) | own;
    uint32_t tot;
    const uint32_t start = block_excl_scan(own, s_warp, tot);
    s_start[tid] = start;
    unsigned long long excl = 0;
    if (j > first) {
        bool gave_up = false;
        for (int64_t p = (int64_t)j - 1; p >= (int64_t)first; --p) {
            const volatile unsigned long long *w = look + (uint64_t)p * 256 + tid;
            unsigned long long v = *w;
            uint32_t spins = 0;
            while ((v >> LB_VALUE_BITS) < tag_a) {
                if (++spins > SPIN_LIMIT) { gave_up = true; break; }
                __nanosleep(32);
                v = *w;
            }
            if (gave_up) break;
            excl += v & LB_VALUE_MASK;
            if ((v >> LB_VALUE_BITS) >= tag_i) break;
        }
        if (gave_up) atomicOr(flags, ERR_WAIT_TIMEOUT);
        *mine = (tag_i << LB_VALUE_BITS) | (excl + own);
    }
    const unsigned long long gofs = seg_start + block_excl_scan64(hp[pass * 256 + tid], s_w64);
    s_dst[tid] = gofs + excl - start;
    __syncthreads();
    // reorder the tile by digit in shared memory, then write runs of equal
    // digits to consecutive addresses
#pragma unroll
    for (uint32_t r = 0; r < RS_ITEMS; ++r) {
        const uint32_t d = rd[r] & 0xFFFFu;
        if (d < 256) {
            const uint32_t pos = s_start[d] + s_wcnt[warp * 256 + d] + (rd[r] >> 16);
            s_keys[pos] = k[r];
            s_vals[pos] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < tile_n; i += RS_THREADS) {
        const unsigned long long key = s_keys[i];
        const unsigned long long dst = s_dst[(uint32_t)((key >> shift) & 255)] + i;
        if (dst < n) {   // only a look-back that gave up can point elsewhere
            kout[dst] = key;
            vout[dst] = s_vals[i];
        }
    }
}

// ---------------------------------------------------------------------------
// selection
// ---------------------------------------------------------------------------

__global__ void k_range_flags(const uint32_t *counts, uint64_t n, uint32_t lo, uint32_t hi, uint32_t *flags)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flags[i] = (counts[i] >= lo && counts[i] <= hi) ? 1u : 0u;
}

__global__ void k_scatter_selected(const unsigned long long *keys, const uint32_t *counts, const uint32_t *flags,
                                   const unsigned long long *pos, uint64_t n, uint64_t limit,
                                   unsigned long long *out_keys, uint32_t *out_counts, unsigned long long *counters,
                                   int counter_idx)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (flags[i] && pos[i] < limit) {
            out_keys[pos[i]] = keys[i];
            out_counts[pos[i]] = counts[i];
        }
        if (i == n - 1) counters[counter_idx] = pos[i] + flags[i];
    }
}

// ---------------------------------------------------------------------------
// bucket-major kernels of the partitioned pipeline
// ---------------------------------------------------------------------------

constexpr uint32_t ITEM_PER_THREAD = WORK_ITEM_KEYS / 256;
// keys per thread whose first table probes are in flight together
constexpr uint32_t INSERT_GROUP = 2;

// Claims the next work item for the whole block; false when none is left.
// Work item `it` of a launch: its bucket is the last one whose first item is
// at or before it (empty buckets share their first item with the next one).
__device__ __forceinline__ WorkItem work_item_n(const BucketRanges *rg, const uint32_t *s_item0, uint32_t it,
                                                uint32_t item_keys)
{
    uint32_t lo = 0, hi = N_BUCKETS;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_item0[mid] <= it) lo = mid; else hi = mid;
    }
    WorkItem w;
    w.bucket = lo;
    const unsigned long long b0 = rg->begin[lo], e0 = b0 + rg->len[lo];
    w.begin = b0 + (unsigned long long)(it - s_item0[lo]) * item_keys;
    w.end = w.begin + item_keys < e0 ? w.begin + item_keys : e0;
    w.pad = 0;
    return w;
}

__device__ __forceinline__ WorkItem work_item(const BucketRanges *rg, const uint32_t *s_item0, uint32_t it)
{
    return work_item_n(rg, s_item0, it, WORK_ITEM_KEYS);
}

__device__ __forceinline__ void load_item_starts(const BucketRanges *rg, uint32_t *s_item0)
{
    for (uint32_t i = threadIdx.x; i <= N_BUCKETS; i += blockDim.x) s_item0[i] = rg->item0[i];
    __syncthreads();
}

__device__ __forceinline__ bool next_work(unsigned int *next_item, uint32_t n_items, uint32_t *s_item, uint32_t &it)
{
    if (threadIdx.x == 0) *s_item = atomicAdd(next_item, 1u);
    __syncthreads();
    it = *s_item;
    __syncthreads();
    return it < n_items;
}

// HyperLogLog of a 1-in-64 hash sample of the non-FIRST k-mers, from the
// high 64 bits h of their XXH3-128 hash (the estimate is scaled by 64 on the
// host).  hll_token packs (register << 8 | rank), 0 for a hash outside the
// sample.  The sample is thin because all blocks working on a bucket update
// the same 1024 registers; an update is skipped when the register already
// holds the rank.
__device__ __forceinline__ uint32_t hll_token(uint64_t h, uint32_t bits)
{
    if (h & ((1u << BUCKET_HLL_SAMPLE_BITS) - 1)) return 0;
    const uint32_t r = (uint32_t)(h >> (64 - bits));
    const uint32_t rank = __clzll((h << bits) | (1ULL << (bits + BUCKET_HLL_SAMPLE_BITS - 1))) + 1;
    return (r << 8) | rank;
}

__device__ __forceinline__ void hll_add_token(uint32_t *regs, uint32_t tok)
{
    if (!tok) return;
    uint32_t *p = &regs[tok >> 8];
    if ((tok & 0xFFu) > *(volatile uint32_t *)p) atomicMax(p, tok & 0xFFu);
}

// The reference's two-level Bloom classification (src/BloomFilter.h:233-273)
// over the partitioned k-mers.  FIRST occurrences go to the front of the
// bucket's range in `out`, the others to its back.  Only FIRST versus not
// FIRST matters downstream, so both filter words are read with one 16-byte
// load and the first word is set without reading its old value.
// k-mers per thread whose filter words are in flight together: two keep the
// kernel at 40 registers (six blocks per SM); four needed 64 (four blocks).
constexpr uint32_t BLOOM_GROUP = 2;

__global__ void __launch_bounds__(256, 6) k_bloom_buckets(const unsigned long long *keys, const BucketRanges *rg,
                                                       uint32_t n_items, unsigned int *next_item,
                                                       const BucketCfg *cfg, unsigned long long *bits,
                                                       unsigned long long *out, unsigned long long *low_cnt,
                                                       unsigned long long *high_cnt, uint32_t *hll_high)
{
    __shared__ uint32_t s_item0[N_BUCKETS + 1];
    load_item_starts(rg, s_item0);
    __shared__ uint32_t s_item, s_warp[8];
    __shared__ unsigned long long s_lb, s_hb;
    // each thread's k-mers wait here (not in registers) while their filter
    // words are read; a thread only reads back what it wrote itself
    __shared__ unsigned long long s_k[WORK_ITEM_KEYS];
    const int tid = threadIdx.x;
    uint32_t it;
    while (next_work(next_item, n_items, &s_item, it)) {
        const WorkItem w = work_item(rg, s_item0, it);
        const BucketCfg bc = cfg[w.bucket];
        const uint64_t n = w.end - w.begin;
        uint32_t firsts = 0, highs = 0;
        // the k-mer stream is read once: keep it from evicting filter lines
#pragma unroll
        for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r) {
            const uint64_t i = (uint64_t)r * 256 + tid;
            s_k[r * 256 + tid] = i < n ? __ldcs(&keys[w.begin + i]) : EMPTY_KEY;
        }
        uint32_t *regs = hll_high + (size_t)w.bucket * BUCKET_HLL_M;
#pragma unroll
        for (uint32_t g = 0; g < ITEM_PER_THREAD; g += BLOOM_GROUP) {
            unsigned long long m[BLOOM_GROUP];
            uint32_t tok[BLOOM_GROUP];
            ulonglong2 *cell[BLOOM_GROUP];
            ulonglong2 v[BLOOM_GROUP];
#pragma unroll
            for (uint32_t u = 0; u < BLOOM_GROUP; ++u) {
                const uint64_t i = (uint64_t)(g + u) * 256 + tid;
                uint64_t block = 0, mask = 0, hi = 0;
                if (i < n) bloom_probe_hi(s_k[(g + u) * 256 + tid], bc.bloom_cap, block, mask, hi);
                m[u] = mask;
                tok[u] = hll_token(hi, BUCKET_HLL_BITS);
                cell[u] = reinterpret_cast<ulonglong2 *>(bits + bc.bloom_off + 2 * block);
            }
#pragma unroll
            for (uint32_t u = 0; u < BLOOM_GROUP; ++u)
                if ((uint64_t)(g + u) * 256 + tid < n) v[u] = __ldcg(cell[u]);
            // occurrences not yet known to be repeats set their bits in the
            // seen-once word; the group's returning atomics are issued back to
            // back and their old values examined afterwards
            unsigned long long old2[BLOOM_GROUP];
            uint32_t pending = 0;
#pragma unroll
            for (uint32_t u = 0; u < BLOOM_GROUP; ++u) {
                if ((uint64_t)(g + u) * 256 + tid >= n) continue;
                unsigned long long *c = reinterpret_cast<unsigned long long *>(cell[u]);
                if ((v[u].x & m[u]) == m[u]) continue;              // seen twice already
                if ((v[u].y & m[u]) == m[u]) atomicOr(&c[0], m[u]);   // seen once: now twice
                else {
                    old2[u] = atomicOr(&c[1], m[u]);
                    pending |= 1u << u;
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < BLOOM_GROUP; ++u) {
                if ((uint64_t)(g + u) * 256 + tid >= n) continue;
                bool first = false;
                if ((pending >> u) & 1u) {
                    unsigned long long *c = reinterpret_cast<unsigned long long *>(cell[u]);
                    if ((old2[u] & m[u]) == m[u]) atomicOr(&c[0], m[u]);
                    else first = true;
                }
                if (first) firsts |= 1u << (g + u);
                else {
                    highs |= 1u << (g + u);
                    hll_add_token(regs, tok[u]);
                }
            }
        }
        uint32_t tf, th;
        const uint32_t of = block_excl_scan(__popc(firsts), s_warp, tf);
        const uint32_t oh = block_excl_scan(__popc(highs), s_warp, th);
        if (tid == 0) {
            s_lb = atomicAdd(&low_cnt[w.bucket], (unsigned long long)tf);
            s_hb = atomicAdd(&high_cnt[w.bucket], (unsigned long long)th);
        }
        __syncthreads();
        unsigned long long lp = bc.key_base + s_lb + of;
        unsigned long long hp = bc.key_base + bc.key_len - 1 - (s_hb + oh);
#pragma unroll
        for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r) {
            if ((firsts >> r) & 1u) __stcs(&out[lp++], s_k[r * 256 + tid]);
            else if ((highs >> r) & 1u) __stcs(&out[hp--], s_k[r * 256 + tid]);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_insert_buckets(const unsigned long long *keys, const BucketRanges *rg,
                                                        uint32_t n_items, unsigned int *next_item,
                                                        const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                                        unsigned long long *bucket_ovf)
{
    __shared__ uint32_t s_item0[N_BUCKETS + 1];
    load_item_starts(rg, s_item0);
    __shared__ uint32_t s_item;
    const int tid = threadIdx.x;
    uint32_t it;
    while (next_work(next_item, n_items, &s_item, it)) {
        const WorkItem w = work_item(rg, s_item0, it);
        const BucketCfg bc = cfg[w.bucket];
        const TableRef tr{arena + bc.slot_base, bc.slot_cap - 1};
        const uint64_t n = w.end - w.begin;
        unsigned long long k[ITEM_PER_THREAD];
#pragma unroll
        for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r) {
            const uint64_t i = (uint64_t)r * 256 + tid;
            k[r] = i < n ? __ldcs(&keys[w.begin + i]) : EMPTY_KEY;
        }
        // a bucket list is in extraction order, so a warp almost never holds
        // two copies of one k-mer: every thread inserts its own k-mers (no
        // warp aggregation), INSERT_GROUP at a time
        bool ok = true;
#pragma unroll
        for (uint32_t g = 0; g < ITEM_PER_THREAD; g += INSERT_GROUP) {
            uint32_t act = 0;
#pragma unroll
            for (uint32_t u = 0; u < INSERT_GROUP; ++u)
                if ((uint64_t)(g + u) * 256 + tid < n) act |= 1u << u;
            if (act && !table_add_group<INSERT_GROUP>(tr.slots, tr.mask, k + g, act, max_probe)) ok = false;
        }
        if (!ok) atomicOr(&bucket_ovf[w.bucket], ERR_TABLE_FULL);
    }
}

__global__ void __launch_bounds__(256) k_merge_buckets(const unsigned long long *keys, const BucketRanges *rg,
                                                       uint32_t n_items, unsigned int *next_item,
                                                       const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                                       uint32_t min_count, uint32_t max_count,
                                                       unsigned long long *rec_keys, uint32_t *rec_counts,
                                                       uint64_t rec_cap, unsigned long long *counters)
{
    __shared__ uint32_t s_item0[N_BUCKETS + 1];
    load_item_starts(rg, s_item0);
    __shared__ uint32_t s_item, s_warp[8];
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x;
    const bool want1 = (min_count <= 1 && 1 <= max_count);
    uint32_t it;
    while (next_work(next_item, n_items, &s_item, it)) {
        const WorkItem w = work_item(rg, s_item0, it);
        const BucketCfg bc = cfg[w.bucket];
        const TableRef tr{arena + bc.slot_base, bc.slot_cap - 1};
        const uint64_t n = w.end - w.begin;
        unsigned long long k[ITEM_PER_THREAD];
#pragma unroll
        for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r) {
            const uint64_t i = (uint64_t)r * 256 + tid;
            k[r] = i < n ? __ldcs(&keys[w.begin + i]) : EMPTY_KEY;
        }
        uint32_t misses = 0;
#pragma unroll
        for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r) {
            if ((uint64_t)r * 256 + tid >= n) continue;
            bool ovf = false;
            Slot *sl = table_find(tr.slots, tr.mask, k[r], max_probe, ovf);
            if (ovf) atomicOr(&counters[C_FLAGS], ERR_TABLE_FULL);
            if (sl) atomicAdd(&sl->count, 1u);
            else misses |= 1u << r;
        }
        unsigned nm = __reduce_add_sync(FULL, (unsigned)__popc(misses));
        if ((tid & 31) == 0 && nm) atomicAdd(&counters[C_LOW_ONLY], (unsigned long long)nm);
        if (want1) {
#pragma unroll
            for (uint32_t r = 0; r < ITEM_PER_THREAD; ++r)
                append_records((misses >> r) & 1u, pair_reverse(k[r]), 1u, rec_keys, rec_counts, rec_cap, counters,
                               s_warp, &s_base);
        }
    }
}

// ---------------------------------------------------------------------------
// shared-memory sub-bucket path of the Bloom split
// ---------------------------------------------------------------------------

// Sub-bucket of a k-mer inside its bucket: its filter block (the reference's
// block = XXH3-128.low64 & (cap - 1), src/BloomFilter.h:215-222) divided by
// the slice size.
__device__ __forceinline__ uint32_t sub_of(unsigned long long key, const SubCfg &c)
{
    uint64_t lo, hi;
    xxh3_128_8(key, lo, hi);
    return (uint32_t)((lo & (c.fcap - 1)) >> c.slice_shift);
}

// Each block counts a contiguous run of work items (bucket-major, so a block
// meets one or two buckets) in a shared histogram, flushed per bucket.
constexpr uint32_t SPC_PER_THREAD = WORK_ITEM_KEYS / 256;
__global__ void __launch_bounds__(256) k_subpart_count(const unsigned long long *keys, const BucketRanges *rg,
                                                       uint32_t n_items, const SubCfg *sc, uint32_t *sub_count,
                                                       uint32_t stride)
{
    __shared__ uint32_t s_item0[N_BUCKETS + 1];
    __shared__ uint32_t s_h[SUB_MAX_PER_BUCKET];
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < SUB_MAX_PER_BUCKET; i += 256) s_h[i] = 0;
    load_item_starts(rg, s_item0);
    const uint32_t per = (n_items + gridDim.x - 1) / gridDim.x;
    const uint32_t it0 = blockIdx.x * per, it1 = min(n_items, it0 + per);
    uint32_t cur = N_BUCKETS;
    SubCfg c{};
    for (uint32_t it = it0; it < it1; ++it) {
        const WorkItem w = work_item(rg, s_item0, it);
        if (w.bucket != cur) {
            if (cur != N_BUCKETS) {
                __syncthreads();
                for (uint32_t i = tid; i < c.n_sub; i += 256)
                    if (s_h[i]) {
                        atomicAdd(&sub_count[c.sub_base + i], s_h[i]);
                        s_h[i] = 0;
                    }
                __syncthreads();
            }
            cur = w.bucket;
            c = sc[cur];
        }
        if (stride > 1) {
            // a sample: every stride-th run of 4 keys (one 32-byte sector).
            // Sampling single sectors rather than whole work items keeps the
            // sampled count of a sub-bucket close to binomial: a work item
            // holds several keys of each sub-bucket, and sampling items would
            // multiply the count's variance by about that number.
            for (unsigned long long j = tid;; j += 256) {
                const unsigned long long i = w.begin + 4ull * stride * (j >> 2) + (j & 3);
                if (i >= w.end) break;
                atomicAdd(&s_h[sub_of(__ldcs(&keys[i]), c)], 1u);
            }
            continue;
        }
        // a work item is 8 keys per thread: their loads are issued together
        for (unsigned long long i0 = w.begin + tid; i0 < w.end; i0 += 256 * SPC_PER_THREAD) {
            unsigned long long kk[SPC_PER_THREAD];
#pragma unroll
            for (uint32_t r = 0; r < SPC_PER_THREAD; ++r) {
                const unsigned long long i = i0 + r * 256;
                kk[r] = i < w.end ? __ldcs(&keys[i]) : 0ull;
            }
#pragma unroll
            for (uint32_t r = 0; r < SPC_PER_THREAD; ++r)
                if (i0 + r * 256 < w.end) atomicAdd(&s_h[sub_of(kk[r], c)], 1u);
        }
    }
    __syncthreads();
    if (cur != N_BUCKETS)
        for (uint32_t i = tid; i < c.n_sub; i += 256)
            if (s_h[i]) atomicAdd(&sub_count[c.sub_base + i], s_h[i]);
}

// Regions of the sub-buckets estimated from a 1-in-stride sample of the
// keys (sectors of 4 keys): n = stride * sampled count, region = n +
// 20 sqrt(n) + 64; the estimate's standard deviation is about
// sqrt(stride * n), under 2.9 sqrt(n) for stride 8, so the margin is about
// 7 of them.
__global__ void k_subpart_regions(const uint32_t *sampled, uint32_t n_sub, uint32_t stride, uint32_t *region)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sub; s += gridDim.x * blockDim.x) {
        const double n = (double)sampled[s] * stride;
        const double r = n + 20.0 * sqrt(n) + 64.0;
        region[s] = r < 2.0e9 ? (uint32_t)r : 2000000000u;
    }
}

// After the scatter into estimated regions: the cursors start at sub_off and
// end past each sub-bucket's keys.  count[s] = keys of sub-bucket s; a
// sub-bucket that outgrew its region (or a region past the key array's end)
// sets *overflow, and its count is cut to what was written.
__global__ void k_subpart_sizes(const unsigned long long *sub_off, const unsigned long long *sub_cursor,
                                const unsigned long long *sub_end, uint32_t n_sub, uint64_t out_cap, uint32_t *count,
                                unsigned long long *overflow)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sub; s += gridDim.x * blockDim.x) {
        const unsigned long long a = sub_off[s], e = sub_end[s] < out_cap ? sub_end[s] : out_cap;
        unsigned long long b = sub_cursor[s];
        if (b > e) {
            atomicOr(overflow, 1ull);
            b = e;
        }
        count[s] = (uint32_t)(b > a ? b - a : 0);
    }
}

// sub_end[s] = sub_off[s] + region[s]; the cursors start at sub_off.
__global__ void k_subpart_ends(const unsigned long long *sub_off, const uint32_t *region, uint32_t n_sub,
                               unsigned long long *sub_end, unsigned long long *sub_cursor)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sub; s += gridDim.x * blockDim.x) {
        sub_end[s] = sub_off[s] + region[s];
        sub_cursor[s] = sub_off[s];
    }
}

// Exclusive scan of one value per thread over a block of up to 1024 threads
// (a multiple of 32).
__device__ __forceinline__ uint32_t block_excl_scan_1024(uint32_t v, uint32_t *s_warp, uint32_t &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < nw ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        s_warp[lane] = s;   // inclusive
    }
    __syncthreads();
    total = s_warp[nw - 1];
    const uint32_t base = warp ? s_warp[warp - 1] : 0u;
    __syncthreads();
    return base + x - v;
}

// One work item (SUB_SCATTER_ITEM_KEYS keys of one bucket) per round: the
// keys are ranked by sub-bucket in shared memory, every sub-bucket of the
// item takes its range with one cursor update, and the item's keys are
// written reordered by sub-bucket (consecutive threads store consecutive
// addresses).  Items are larger than the other bucket kernels' so that a
// sub-bucket's run in an item spans several sectors.
constexpr uint32_t SP_THREADS = 512;
constexpr uint32_t SP_PER_THREAD = SUB_SCATTER_ITEM_KEYS / SP_THREADS;
constexpr uint32_t SP_MAX_BINS = (SUB_MAX_PER_BUCKET + SP_THREADS - 1) / SP_THREADS;   // sub-buckets per thread
static_assert(SUB_SCATTER_ITEM_KEYS % SP_THREADS == 0 && SUB_SCATTER_ITEM_KEYS <= 65536, "item layout");

// MAXB: sub-buckets per thread in the rank scan (the cursor updates held in
// registers until after the reorder); launches whose buckets have at most
// 2 * SP_THREADS sub-buckets use MAXB = 2 and fit three blocks per SM.
template <uint32_t MAXB, uint32_t BPSM>
__global__ void __launch_bounds__(SP_THREADS, BPSM) k_subpart_scatter(const unsigned long long *keys,
                                                                      const BucketRanges *rg, uint32_t n_items,
                                                                      unsigned int *next_item, const SubCfg *sc,
                                                                      unsigned long long *sub_cursor,
                                                                      const unsigned long long *sub_end,
                                                                      unsigned long long *out, uint64_t out_cap,
                                                                      uint32_t max_sub)
{
    // shared arrays per sub-bucket hold max_sub entries (the most of any
    // bucket of the launch)
    extern __shared__ __align__(16) uint8_t sp_smem[];
    unsigned long long *s_sorted = reinterpret_cast<unsigned long long *>(sp_smem);          // SUB_SCATTER_ITEM_KEYS
    unsigned long long *s_dst = s_sorted + SUB_SCATTER_ITEM_KEYS;                             // max_sub
    uint32_t *s_cnt = reinterpret_cast<uint32_t *>(s_dst + max_sub);                          // max_sub
    uint32_t *s_start = s_cnt + max_sub;                                                      // max_sub
    uint16_t *s_sub = reinterpret_cast<uint16_t *>(s_start + max_sub);                        // SUB_SCATTER_ITEM_KEYS
    __shared__ uint32_t s_item0[N_BUCKETS + 1];
    __shared__ uint32_t s_item, s_warp[32];
    const int tid = threadIdx.x;
    for (uint32_t i = tid; i < max_sub; i += SP_THREADS) s_cnt[i] = 0;
    load_item_starts(rg, s_item0);
    uint32_t it;
    while (next_work(next_item, n_items, &s_item, it)) {
        const WorkItem w = work_item_n(rg, s_item0, it, SUB_SCATTER_ITEM_KEYS);
        const SubCfg c = sc[w.bucket];
        const uint32_t n = (uint32_t)(w.end - w.begin);
        unsigned long long k[SP_PER_THREAD];
        uint32_t sr[SP_PER_THREAD];   // rank << 16 | sub (sub 0xFFFF: no key)
#pragma unroll
        for (uint32_t r = 0; r < SP_PER_THREAD; ++r) {
            const uint32_t i = r * SP_THREADS + tid;
            if (i < n) k[r] = __ldcs(&keys[w.begin + i]);
        }
#pragma unroll
        for (uint32_t r = 0; r < SP_PER_THREAD; ++r) {
            const uint32_t i = r * SP_THREADS + tid;
            sr[r] = 0xFFFFu;
            if (i < n) {
                const uint32_t sub = sub_of(k[r], c);
                sr[r] = (atomicAdd(&s_cnt[sub], 1u) << 16) | sub;
            }
        }
        __syncthreads();
        // exclusive scan of the n_sub counts, a few per thread
        const uint32_t per = (c.n_sub + SP_THREADS - 1) / SP_THREADS, b0 = tid * per;
        uint32_t local = 0;
        for (uint32_t j = 0; j < per; ++j)
            if (b0 + j < c.n_sub) local += s_cnt[b0 + j];
        uint32_t tot;
        uint32_t run = block_excl_scan_1024(local, s_warp, tot);
        // the sub-buckets' cursor updates are in flight during the reorder
        // and consumed only after it
        unsigned long long cur[MAXB];
        uint32_t first[MAXB];
#pragma unroll
        for (uint32_t j = 0; j < MAXB; ++j) {
            const uint32_t s = b0 + j;
            cur[j] = 0ull;
            first[j] = run;
            if (j < per && s < c.n_sub) {
                const uint32_t cnt = s_cnt[s];
                s_start[s] = run;
                if (cnt) cur[j] = atomicAdd(&sub_cursor[c.sub_base + s], (unsigned long long)cnt);
                run += cnt;
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t r = 0; r < SP_PER_THREAD; ++r) {
            const uint32_t sub = sr[r] & 0xFFFFu;
            if (sub != 0xFFFFu) {
                const uint32_t p = s_start[sub] + (sr[r] >> 16);
                s_sorted[p] = k[r];
                s_sub[p] = (uint16_t)sub;
            }
        }
        // destination of sorted index i of sub-bucket s: s_dst[s] + i
#pragma unroll
        for (uint32_t j = 0; j < MAXB; ++j)
            if (j < per && b0 + j < c.n_sub) s_dst[b0 + j] = cur[j] - first[j];
        __syncthreads();
        for (uint32_t i = tid; i < n; i += SP_THREADS) {
            const uint32_t sb = s_sub[i];
            const unsigned long long d = s_dst[sb] + i;
            // estimated regions: a sub-bucket that outgrew its region is
            // reported by its cursor (k_subpart_sizes) and counted exactly
            if (d < out_cap && (!sub_end || d < sub_end[c.sub_base + sb])) out[d] = s_sorted[i];
        }
        for (uint32_t i = tid; i < c.n_sub; i += SP_THREADS) s_cnt[i] = 0;
        __syncthreads();
    }
}

// Shared-memory counting table of one sub-bucket (2^TBITS slots): linear
// probing from the key's hash, claims by CAS; a slot only changes from empty
// to a key.  The home slot is the top TBITS bits of the 64-bit mix
// (slot_hash), or with FIB of the key times 2^64 / golden ratio (one
// multiply: placement only, it never affects a count).
constexpr uint32_t SUB_MAX_PROBE = 512;

template <uint32_t TBITS, bool FIB>
__device__ __forceinline__ uint32_t sub_table_slot(unsigned long long key)
{
    return FIB ? (uint32_t)((key * 0x9E3779B97F4A7C15ULL) >> (64 - TBITS))
               : (uint32_t)(slot_hash(key) >> (64 - TBITS));
}

template <uint32_t TBITS, bool FIB>
__device__ __forceinline__ bool sub_table_add(unsigned long long *tk, uint32_t *tc, unsigned long long key)
{
    uint32_t i = sub_table_slot<TBITS, FIB>(key);
    for (uint32_t n = 0; n < SUB_MAX_PROBE; ++n) {
        const unsigned long long cur = *(volatile unsigned long long *)&tk[i];
        if (cur == key) {
            atomicAdd(&tc[i], 1u);
            return true;
        }
        if (cur == EMPTY_KEY) {
            const unsigned long long prev = atomicCAS(&tk[i], EMPTY_KEY, key);
            if (prev == EMPTY_KEY || prev == key) {
                atomicAdd(&tc[i], 1u);
                return true;
            }
        }
        i = (i + 1) & ((1u << TBITS) - 1);
    }
    return false;
}

template <uint32_t TBITS, bool FIB>
__device__ __forceinline__ int sub_table_find(const unsigned long long *tk, unsigned long long key)
{
    uint32_t i = sub_table_slot<TBITS, FIB>(key);
    for (uint32_t n = 0; n < SUB_MAX_PROBE; ++n) {
        const unsigned long long cur = tk[i];
        if (cur == key) return (int)i;
        if (cur == EMPTY_KEY) return -1;
        i = (i + 1) & ((1u << TBITS) - 1);
    }
    return -1;
}

constexpr uint32_t SUB_PER_THREAD = 4;

// THREADS per block, BPSM blocks per SM, filter slices of at most SLICE
// blocks, tables of 2^TBITS slots, counts below HBINS histogrammed in shared
// memory (the two shapes are SubShape 1 and 2 in kc_kernels.cuh).
template <uint32_t THREADS, uint32_t BPSM, uint32_t SLICE, uint32_t TBITS, uint32_t HBINS, bool FIB>
__global__ void __launch_bounds__(THREADS, BPSM) k_count_subs(
    unsigned long long *keys, const unsigned long long *sub_off, const uint32_t *sub_count, const uint8_t *sub_bucket,
    uint32_t n_sub, const SubCfg *sc, unsigned int *next_sub, uint32_t count_max, uint32_t min_count,
    uint32_t max_count, unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist,
    uint32_t *ovf, uint64_t ovf_cap, unsigned long long *counters, uint32_t *bucket_ovf, uint32_t *hb16,
    uint32_t hb16_shift)
{
    extern __shared__ __align__(16) uint8_t cs_smem[];
    unsigned long long *s_filter = reinterpret_cast<unsigned long long *>(cs_smem);   // 2 * SLICE
    unsigned long long *s_tk = s_filter + 2 * SLICE;                       // (1u << TBITS)
    uint32_t *s_tc = reinterpret_cast<uint32_t *>(s_tk + (1u << TBITS));            // (1u << TBITS)
    uint32_t *s_hist = s_tc + (1u << TBITS);                                        // HBINS
    unsigned long long *s_queue = reinterpret_cast<unsigned long long *>(s_hist + HBINS);   // (THREADS * SUB_PER_THREAD)
    __shared__ uint32_t s_warp[32], s_sub, s_lo;   // s_lo: FIRST keys written back
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    for (uint32_t i = tid; i < HBINS; i += THREADS) s_hist[i] = 0;
    unsigned long long n_high = 0, n_low = 0, n_low_only = 0, n_distinct = 0;
    uint32_t n_ovf_subs = 0;
    bool rec_full = false;
    for (;;) {
        if (tid == 0) s_sub = atomicAdd(next_sub, 1u);
        __syncthreads();
        const uint32_t sub = s_sub;
        __syncthreads();
        if (sub >= n_sub) break;
        const uint32_t n = sub_count[sub];
        if (n == 0) continue;
        const unsigned long long base = sub_off[sub];
        const uint32_t bucket = sub_bucket[sub];
        const unsigned long long fcap = sc[bucket].fcap;
        const uint32_t slice = 1u << sc[bucket].slice_shift;
        if (tid == 0) s_lo = 0;
        for (uint32_t i = tid; i < 2 * slice; i += THREADS) s_filter[i] = 0;
        for (uint32_t i = tid; i < (1u << TBITS); i += THREADS) {
            s_tk[i] = EMPTY_KEY;
            s_tc[i] = 0;
        }
        __syncthreads();
        // 1. the reference's two-level Bloom classification (src/BloomFilter.h:233-273)
        // on the slice; non-FIRST occurrences counted in the table, FIRST ones
        // written back over the front of the sub-bucket's keys
        bool full = false;
        // the next tile's k-mers are loaded while this one is classified (a
        // tile's FIRST write-back only reaches positions already loaded)
        unsigned long long kn[SUB_PER_THREAD];
#pragma unroll
        for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
            const uint32_t i = r * THREADS + tid;
            kn[r] = i < n ? __ldcs(&keys[base + i]) : EMPTY_KEY;
        }
        __syncthreads();   // the first tile is loaded by every warp before any write-back
        for (uint32_t t0 = 0; t0 < n; t0 += (THREADS * SUB_PER_THREAD)) {
            unsigned long long k[SUB_PER_THREAD];
            uint32_t firsts = 0, highs = 0;
#pragma unroll
            for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                k[r] = kn[r];
                const uint32_t i = t0 + (THREADS * SUB_PER_THREAD) + r * THREADS + tid;
                kn[r] = i < n ? __ldcs(&keys[base + i]) : EMPTY_KEY;
            }
#pragma unroll
            for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                if (t0 + r * THREADS + tid >= n) continue;
                uint64_t block, m, hi;
                bloom_probe_hi(k[r], fcap, block, m, hi);
                unsigned long long *cell = s_filter + 2 * (block & (slice - 1));
                // a k-mer seen twice already (most of them) needs no update;
                // otherwise it is FIRST exactly when the seen-once word lacked
                // its bits (the seen-twice bits are always a subset of the
                // seen-once bits, so this is the reference's three-way test,
                // and setting bits already set changes nothing)
                bool first = false;
                if ((*(volatile unsigned long long *)&cell[0] & m) != m) {
                    const unsigned long long old2 = atomicOr(&cell[1], (unsigned long long)m);
                    first = (old2 & m) != m;
                    if (!first) atomicOr(&cell[0], (unsigned long long)m);
                }
                if (first) firsts |= 1u << r;
                else highs |= 1u << r;
            }
            n_high += (uint64_t)__popc(highs);
            // the warp's non-FIRST k-mers are queued so that every lane inserts
            {
                unsigned long long *q = s_queue + warp * (32 * SUB_PER_THREAD);
                uint32_t qn = 0;
#pragma unroll
                for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                    const bool h = (highs >> r) & 1u;
                    const uint32_t b = __ballot_sync(FULL, h);
                    if (h) q[qn + (uint32_t)__popc(b & lt)] = k[r];
                    qn += (uint32_t)__popc(b);
                }
                __syncwarp();
                for (uint32_t j = lane; j < qn; j += 32)
                    if (!sub_table_add<TBITS, FIB>(s_tk, s_tc, q[j])) full = true;
                __syncwarp();
            }
            // FIRST write-back: each warp takes its positions with one
            // shared-memory atomic.  They lie below the keys classified so
            // far, i.e. in this tile or earlier ones, whose keys every warp
            // holds in registers (the barrier at the end of the previous tile
            // came after every warp's loads of this one)
            {
                uint32_t wb[SUB_PER_THREAD], wtot = 0;
#pragma unroll
                for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                    wb[r] = __ballot_sync(FULL, (firsts >> r) & 1u);
                    wtot += (uint32_t)__popc(wb[r]);
                }
                uint32_t wbase = 0;
                if (lane == 0 && wtot) wbase = atomicAdd(&s_lo, wtot);
                wbase = __shfl_sync(FULL, wbase, 0);
                uint32_t before = 0;
#pragma unroll
                for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                    if ((firsts >> r) & 1u) keys[base + wbase + before + (uint32_t)__popc(wb[r] & lt)] = k[r];
                    before += (uint32_t)__popc(wb[r]);
                }
            }
            n_low += (uint64_t)__popc(firsts);
            __syncthreads();
        }
        if (__syncthreads_or(full)) {
            if (tid == 0) {
                ++n_ovf_subs;
                atomicOr(&bucket_ovf[bucket], 1u);
            }
            continue;   // incomplete: the host counts the pass again with more sub-buckets
        }
        // 2. FIRST occurrences: a hit adds one to the table count, a miss is a
        // k-mer seen once (counted, not a record: min_count >= 2)
        const uint32_t lo_cnt = s_lo;
        for (uint32_t i0 = tid; i0 < lo_cnt; i0 += THREADS * SUB_PER_THREAD) {
            unsigned long long kk[SUB_PER_THREAD];
#pragma unroll
            for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                const uint32_t i = i0 + r * THREADS;
                kk[r] = i < lo_cnt ? __ldcg(&keys[base + i]) : EMPTY_KEY;
            }
#pragma unroll
            for (uint32_t r = 0; r < SUB_PER_THREAD; ++r) {
                if (i0 + r * THREADS >= lo_cnt) continue;
                const int sl = sub_table_find<TBITS, FIB>(s_tk, kk[r]);
                if (sl >= 0) atomicAdd(&s_tc[sl], 1u);
                else ++n_low_only;
            }
        }
        __syncthreads();
        // 3. the table's records and histogram
        uint32_t keep = 0;
        for (uint32_t i = tid; i < (1u << TBITS); i += THREADS) {
            if (s_tk[i] == EMPTY_KEY) continue;
            ++n_distinct;
            const uint32_t c = s_tc[i] < count_max ? s_tc[i] : count_max;
            if (c < HBINS) atomicAdd(&s_hist[c], 1u);
            else if (c < HIST_BINS) atomicAdd(&hist[c], 1ull);
            else {
                const unsigned long long q = atomicAdd(&counters[C_OVF_LEN], 1ull);
                if (q < ovf_cap) ovf[q] = c;
                else atomicOr(&counters[C_FLAGS], ERR_HIST_OVERFLOW_FULL);
            }
            keep += (c >= min_count && c <= max_count) ? 1u : 0u;
        }
        uint32_t tk;
        const uint32_t ok = block_excl_scan_1024(keep, s_warp, tk);
        if (tid == 0) s_base = tk ? atomicAdd(&counters[C_REC_LEN], (unsigned long long)tk) : 0ull;
        __syncthreads();
        unsigned long long q = s_base + ok;
        for (uint32_t i = tid; i < (1u << TBITS); i += THREADS) {
            if (s_tk[i] == EMPTY_KEY) continue;
            const uint32_t c = s_tc[i] < count_max ? s_tc[i] : count_max;
            if (c < min_count || c > max_count) continue;
            if (q < rec_cap) {
                const unsigned long long sk = pair_reverse(s_tk[i]);
                rec_keys[q] = sk;
                rec_counts[q] = c;
                if (hb16) atomicAdd(&hb16[(uint32_t)(sk >> hb16_shift) & 0xFFFFu], 1u);   // the record sort's buckets
            } else {
                rec_full = true;
            }
            ++q;
        }
        __syncthreads();
    }
    __syncthreads();
    for (uint32_t i = tid; i < HBINS; i += THREADS)
        if (s_hist[i]) atomicAdd(&hist[i], (unsigned long long)s_hist[i]);
    if (rec_full) atomicOr(&counters[C_FLAGS], ERR_RECORDS_FULL);
    const unsigned long long v[4] = {n_high, n_low, n_low_only, n_distinct};
    const int idx[4] = {C_HIGH_LEN, C_LOW_LEN, C_LOW_ONLY, C_DISTINCT};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        unsigned long long x = v[j];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
        if ((tid & 31) == 0 && x) atomicAdd(&counters[idx[j]], x);
    }
    if (tid == 0 && n_ovf_subs) atomicAdd(&counters[C_SUB_OVF], (unsigned long long)n_ovf_subs);
}

__global__ void k_hash_batch(const unsigned long long *keys, uint64_t n, unsigned long long *out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t w = keys[i], lo, hi;
        xxh3_128_8(w, lo, hi);
        out[5 * i + 0] = lo;
        out[5 * i + 1] = hi;
        out[5 * i + 2] = xxh3_64_8(w);
        out[5 * i + 3] = rapidhash_8(w);
        out[5 * i + 4] = komihash_8(w);
    }
}

// Failure detection: a wait on a device word, polled at most poll_limit
// times (about a microsecond apart), the same way every wait of the pipeline
// is bounded.  A wait that runs out sets ERR_WAIT_TIMEOUT in *flags and
// returns, so the host reads a status and the context stays usable.
__global__ void k_wait_flag(const unsigned int *flag, uint32_t poll_limit, unsigned long long *flags)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const volatile unsigned int *f = flag;
    for (uint32_t i = 0; i < poll_limit; ++i) {
        if (*f != 0u) return;
        __nanosleep(1000);
    }
    atomicOr(flags, ERR_WAIT_TIMEOUT);
}

__global__ void k_or_flags(unsigned long long *word, unsigned long long bits)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(word, bits);
}

std::atomic<unsigned long long> g_launches{0};
thread_local unsigned long long t_launches = 0;

inline void note_launch()
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    ++t_launches;
}

int sm_count()
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

int grid_for(uint64_t n, int threads, int per_sm = 8)
{
    uint64_t g = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)sm_count() * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

unsigned long long kernel_launches() { return g_launches.load(std::memory_order_relaxed); }
unsigned long long thread_kernel_launches() { return t_launches; }

void note_kernel_launch() { note_launch(); }

size_t extract_smem_bytes_for(int mode, uint32_t stage_cap)
{
    size_t b = 2 * BUF_BYTES + 264 * 8 * 2 + 264 * 4;
    if (mode != MODE_SCAN) b += (size_t)stage_cap * 8;
    else b += HLL_M * 4;
    if (mode != MODE_SCAN) b += (size_t)stage_cap * 2;
    return b;
}

size_t extract_smem_bytes() { return extract_smem_bytes_for(MODE_INSERT, STAGE_CAP); }

cudaError_t launch_newlines(const uint8_t *buf, uint64_t n_tiles, uint32_t *tile_nl, int32_t *tile_lastnl,
                            cudaStream_t st)
{
    if (!n_tiles) return cudaSuccess;
    note_launch();
    k_newlines<<<grid_for(n_tiles, 1, 16), 256, 0, st>>>(buf, n_tiles, tile_nl, tile_lastnl);
    return cudaGetLastError();
}

cudaError_t launch_chunk_lastnl(const int32_t *tile_lastnl, const uint32_t *tile_seg, const Seg *segs,
                                const uint64_t *seg_chunk0, uint64_t n_tiles, int32_t *chunk_lastnl, cudaStream_t st)
{
    if (!n_tiles) return cudaSuccess;
    note_launch();
    k_chunk_lastnl<<<grid_for(n_tiles, 256), 256, 0, st>>>(tile_lastnl, tile_seg, segs, seg_chunk0, n_tiles,
                                                           chunk_lastnl);
    return cudaGetLastError();
}

template <int M, uint32_t SCAP = STAGE_CAP>
static cudaError_t launch_extract_t(const ExtractArgs &a, int grid, uint32_t stage_cap, cudaStream_t st)
{
    size_t smem = extract_smem_bytes_for(M, stage_cap);
    auto kern = k_extract<M, SCAP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (grid <= 0) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, EXT_THREADS, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        grid = sm_count() * per_sm;
    }
    const uint64_t n_iter = (M == MODE_SCAN && a.visit) ? a.n_visit : a.n_tiles;
    if (!n_iter) return cudaSuccess;
    if ((uint64_t)grid > n_iter) grid = (int)n_iter;
    note_launch();
    kern<<<grid, EXT_THREADS, smem, st>>>(a, stage_cap);
    return cudaGetLastError();
}

cudaError_t launch_extract(int mode, const ExtractArgs &a, int grid, cudaStream_t st, uint32_t part_shape)
{
    if (!a.n_tiles) return cudaSuccess;
    switch (mode) {
    case MODE_SCAN: return launch_extract_t<MODE_SCAN>(a, grid, STAGE_CAP, st);
    case MODE_INSERT: return launch_extract_t<MODE_INSERT>(a, grid, STAGE_CAP, st);
    case MODE_BLOOM: return launch_extract_t<MODE_BLOOM>(a, grid, STAGE_CAP, st);
    case MODE_EMIT: return launch_extract_t<MODE_EMIT>(a, grid, STAGE_CAP, st);
    case MODE_PART:
        return part_shape == 2 ? launch_extract_t<MODE_PART, 2048>(a, grid, 2048, st)
                               : launch_extract_t<MODE_PART>(a, grid, STAGE_CAP, st);
    default: return cudaErrorInvalidValue;
    }
}

size_t scan_tmp_words(uint64_t n) { return (n + SCAN_BLOCK - 1) / SCAN_BLOCK + 1; }

cudaError_t launch_scan_u32(const uint32_t *in, unsigned long long *out, uint64_t n, unsigned long long *tmp,
                            cudaStream_t st)
{
    if (!n) return cudaSuccess;
    uint64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    note_launch();
    k_scan_reduce<<<(unsigned)nb, 256, 0, st>>>(in, n, tmp);
    note_launch();
    k_scan_top<<<1, 1024, 0, st>>>(tmp, nb);
    note_launch();
    k_scan_down<<<(unsigned)nb, 256, 0, st>>>(in, n, tmp, out);
    return cudaGetLastError();
}

__global__ void k_add_u64(unsigned long long *dst, const unsigned long long *src, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (src[i]) dst[i] += src[i];
}

cudaError_t launch_add_u64(unsigned long long *dst, const unsigned long long *src, uint64_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_add_u64<<<grid_for(n, 256), 256, 0, st>>>(dst, src, n);
    return cudaGetLastError();
}

cudaError_t launch_fill_u64(unsigned long long *p, uint64_t n, unsigned long long v, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_fill_u64<<<grid_for(n, 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_init_slots(Slot *slots, uint64_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_init_slots<<<grid_for(n, 256), 256, 0, st>>>(slots, n);
    return cudaGetLastError();
}

cudaError_t launch_count_keys(const Slot *slots, uint64_t n, unsigned long long *out, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_count_keys<<<grid_for(n, 256), 256, 0, st>>>(slots, n, out);
    return cudaGetLastError();
}

cudaError_t launch_insert_list(const unsigned long long *keys, uint64_t n, TableRef t, uint32_t max_probe,
                               unsigned long long *counters, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_insert_list<<<grid_for(n, 256), 256, 0, st>>>(keys, n, t, max_probe, counters);
    return cudaGetLastError();
}

cudaError_t launch_insert_pairs(const unsigned long long *keys, const uint32_t *counts, uint64_t n, TableRef t,
                                uint32_t max_probe, unsigned long long *counters, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_insert_pairs<<<grid_for(n, 256), 256, 0, st>>>(keys, counts, n, t, max_probe, counters);
    return cudaGetLastError();
}

cudaError_t launch_merge_low(const unsigned long long *keys, uint64_t n, TableRef t, uint32_t max_probe,
                             uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys, uint32_t *rec_counts,
                             uint64_t rec_cap, unsigned long long *counters, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_merge_low<<<grid_for(n, 256), 256, 0, st>>>(keys, n, t, max_probe, min_count, max_count, rec_keys, rec_counts,
                                                  rec_cap, counters);
    return cudaGetLastError();
}

cudaError_t launch_compact(TableRef t, uint64_t cap, uint32_t count_max, uint32_t min_count, uint32_t max_count,
                           unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                           unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap, unsigned long long *counters,
                           cudaStream_t st)
{
    if (!cap) return cudaSuccess;
    note_launch();
    k_compact<<<grid_for(cap, 256, 4), 256, 0, st>>>(t, cap, count_max, min_count, max_count, rec_keys, rec_counts,
                                                     rec_cap, hist, ovf, ovf_cap, counters);
    return cudaGetLastError();
}

uint64_t compact_ordered_chunks(uint64_t cap) { return (cap + ORDERED_CHUNK - 1) / ORDERED_CHUNK; }

cudaError_t launch_compact_ordered(const Slot *slots, uint64_t cap, uint32_t count_max, uint32_t min_count,
                                   uint32_t max_count, uint32_t *chunk_keep, const unsigned long long *chunk_pos,
                                   unsigned long long *rec_keys, uint32_t *rec_counts, uint64_t rec_cap,
                                   unsigned long long *hist, uint32_t *ovf, uint64_t ovf_cap,
                                   unsigned long long *counters, int count_only, cudaStream_t st)
{
    if (!cap) return cudaSuccess;
    const uint64_t n_chunks = compact_ordered_chunks(cap);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_compact_ordered, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint64_t grid = std::min<uint64_t>(n_chunks, (uint64_t)sm_count() * per_sm);
    note_launch();
    k_compact_ordered<<<(unsigned)grid, 256, 0, st>>>(slots, cap, count_max, min_count, max_count, chunk_keep,
                                                      chunk_pos, rec_keys, rec_counts, rec_cap, hist, ovf, ovf_cap,
                                                      counters, count_only);
    return cudaGetLastError();
}

static uint64_t sort_tiles_for(const uint64_t *seg_len, uint32_t n_segs)
{
    uint64_t t = 0;
    for (uint32_t i = 0; i < n_segs; ++i) t += (seg_len[i] + RS_TILE - 1) / RS_TILE;
    return t;
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// working memory of the digit-count/scan/scatter sort kept for
// launch_radix_sort_in_scratch: second key/value arrays, per-tile digit counts
// and offsets, the scan's temporary words and the tile descriptors
static size_t scratch_sort_bytes(uint64_t n)
{
    const uint64_t n_tiles = (n + RS_TILE - 1) / RS_TILE;
    const uint64_t nc = 256 * std::max<uint64_t>(n_tiles, 1);
    return align256(n * 8) + align256(n * 4) + align256(nc * 4) + align256(nc * 8) + align256(scan_tmp_words(nc) * 8) +
           align256(std::max<uint64_t>(n_tiles, 1) * sizeof(SortTile));
}

// working memory of launch_radix_sort_segmented: second key/value arrays,
// per-segment digit histograms of all passes, the look-back words, the pass
// tile counters and an error word, and the tile descriptors
size_t sort_tmp_bytes_segmented(uint64_t n_total, const uint64_t *seg_len, uint32_t n_segs)
{
    const uint64_t n_tiles = std::max<uint64_t>(sort_tiles_for(seg_len, n_segs), 1);
    return align256(n_total * 8) + align256(n_total * 4) +
           align256((uint64_t)std::max<uint32_t>(n_segs, 1) * OS_MAX_PASSES * 256 * 8) + align256(n_tiles * 256 * 8) +
           align256(OS_MAX_PASSES * 4 + 8) + align256(n_tiles * sizeof(OsTile));
}

// working memory of launch_radix_sort: second key/value arrays, the digit
// histograms of all passes, one look-back word per (tile, digit), the tile
// counters of the passes and an error word
static size_t onesweep_tmp_bytes(uint64_t n)
{
    const uint64_t n_tiles = std::max<uint64_t>((n + RS_TILE - 1) / RS_TILE, 1);
    return align256(n * 8) + align256(n * 4) + align256(OS_MAX_PASSES * 256 * 8) + align256(n_tiles * 256 * 8) +
           align256(OS_MAX_PASSES * 4 + 8);
}

size_t sort_tmp_bytes(uint64_t n) { return onesweep_tmp_bytes(n); }

void sort_tmp_alt(void *tmp, uint64_t n, unsigned long long **k2, uint32_t **v2)
{
    uint8_t *p = static_cast<uint8_t *>(tmp);
    *k2 = reinterpret_cast<unsigned long long *>(p);
    *v2 = reinterpret_cast<uint32_t *>(p + align256(n * 8));
}

uint32_t sort_passes_run(uint32_t bits, uint32_t skip_bits)
{
    const uint32_t passes = (bits + 7) / 8, skipped = skip_bits / 8;
    return skipped < passes ? passes - skipped : 0;
}

size_t sort_tmp_bytes_in_scratch(uint64_t n) { return scratch_sort_bytes(n); }

// Segments [seg_start[i], seg_start[i] + seg_len[i]) of the arrays are sorted
// independently; they must be disjoint and in increasing address order.
// Consecutive segments are sorted in groups of about group_records records
// (4M: 48 MiB of keys + values), every pass of a group before the next group,
// so that a group's keys and values stay in L2 across its passes.

cudaError_t launch_radix_sort_segmented(unsigned long long *keys, uint32_t *vals, uint64_t n_total,
                                        const uint64_t *seg_start, const uint64_t *seg_len, uint32_t n_segs,
                                        uint32_t bits, void *tmp, cudaStream_t st, unsigned long long *flags,
                                        const uint32_t *seg_bits, uint64_t group_records_max)
{
    const uint64_t n_tiles = sort_tiles_for(seg_len, n_segs);
    if (n_tiles == 0 || bits == 0) return cudaSuccess;
    if (bits > 64) return cudaErrorInvalidValue;
    // groups of whole segments; a tile's first_tile is relative to its group
    struct Group {
        uint64_t t0, t1;
        uint32_t passes;
    };
    std::vector<Group> groups;
    std::vector<OsTile> tiles;
    tiles.reserve(n_tiles);
    uint64_t group_records = 0;
    for (uint32_t sgi = 0; sgi < n_segs; ++sgi) {
        const uint64_t nt = (seg_len[sgi] + RS_TILE - 1) / RS_TILE;
        if (!nt) continue;
        const uint32_t b = seg_bits ? std::min(seg_bits[sgi], bits) : bits;
        const uint32_t sp = (b + 7) / 8;
        if (groups.empty() || group_records + seg_len[sgi] > group_records_max) {
            groups.push_back(Group{tiles.size(), tiles.size(), 0});
            group_records = 0;
        }
        Group &g = groups.back();
        const uint32_t first = (uint32_t)(tiles.size() - g.t0);
        for (uint64_t j = 0; j < nt; ++j) {
            OsTile t;
            t.begin = seg_start[sgi] + j * RS_TILE;
            t.end = std::min(seg_start[sgi] + seg_len[sgi], t.begin + RS_TILE);
            t.seg_start = seg_start[sgi];
            t.first_tile = first;
            t.seg = sgi;
            t.passes = sp;
            t.pad = 0;
            tiles.push_back(t);
        }
        g.t1 = tiles.size();
        g.passes = std::max(g.passes, sp);
        group_records += seg_len[sgi];
    }
    uint8_t *p = static_cast<uint8_t *>(tmp);
    unsigned long long *k2 = reinterpret_cast<unsigned long long *>(p);
    p += align256(n_total * 8);
    uint32_t *v2 = reinterpret_cast<uint32_t *>(p);
    p += align256(n_total * 4);
    unsigned long long *hist = reinterpret_cast<unsigned long long *>(p);
    const size_t hist_bytes = (size_t)std::max<uint32_t>(n_segs, 1) * OS_MAX_PASSES * 256 * 8;
    p += align256(hist_bytes);
    unsigned long long *look = reinterpret_cast<unsigned long long *>(p);
    p += align256(n_tiles * 256 * 8);
    unsigned int *tile_ctr = reinterpret_cast<unsigned int *>(p);
    unsigned long long *own_flags = reinterpret_cast<unsigned long long *>(p + OS_MAX_PASSES * 4);
    p += align256(OS_MAX_PASSES * 4 + 8);
    OsTile *d_tiles = reinterpret_cast<OsTile *>(p);
    if (!flags) flags = own_flags;
    cudaError_t e = cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(OsTile), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, hist_bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(look, 0, n_tiles * 256 * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(own_flags, 0, 8, st);
    if (e != cudaSuccess) return e;
    const size_t smem = RS_TILE * 8 + RS_TILE * 4 + 8 * 256 * 4;
    e = cudaFuncSetAttribute(k_radix_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    for (const Group &g : groups) {
        const uint64_t gt = g.t1 - g.t0;
        e = cudaMemsetAsync(tile_ctr, 0, OS_MAX_PASSES * 4, st);
        if (e != cudaSuccess) return e;
        const uint64_t hblocks = std::min<uint64_t>(gt, (uint64_t)sm_count() * 8);
        const uint64_t per_block = (gt + hblocks - 1) / hblocks;
        note_launch();
        k_radix_hist_seg<<<(unsigned)((gt + per_block - 1) / per_block), 256, 0, st>>>(keys, d_tiles + g.t0, gt,
                                                                                         per_block, g.passes, hist);
        unsigned long long *ks = keys, *kd = k2;
        uint32_t *vs = vals, *vd = v2;
        for (uint32_t pass = 0; pass < g.passes; ++pass) {
            note_launch();
            k_radix_onesweep<<<(unsigned)gt, RS_THREADS, smem, st>>>(ks, vs, kd, vd, n_total, pass, hist,
                                                                     look + g.t0 * 256, tile_ctr, flags,
                                                                     d_tiles + g.t0);
            std::swap(ks, kd);
            std::swap(vs, vd);
        }
    }
    // a segment that took an odd number of passes ends in the second arrays
    for (uint32_t sgi = 0; sgi < n_segs; ++sgi) {
        const uint32_t b = seg_bits ? std::min(seg_bits[sgi], bits) : bits;
        if (!seg_len[sgi] || ((b + 7) / 8) % 2 == 0) continue;
        e = cudaMemcpyAsync(keys + seg_start[sgi], k2 + seg_start[sgi], seg_len[sgi] * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(vals + seg_start[sgi], v2 + seg_start[sgi], seg_len[sgi] * 4, cudaMemcpyDeviceToDevice,
                                st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

// Tile descriptors of a one-segment sort, written by the device.
__global__ void k_single_segment_tiles(SortTile *tiles, uint64_t n, uint64_t n_tiles)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n_tiles; t += (uint64_t)gridDim.x * blockDim.x) {
        SortTile d;
        d.begin = t * RS_TILE;
        d.end = n < d.begin + RS_TILE ? n : d.begin + RS_TILE;
        d.cbase = t;
        d.stride = n_tiles;
        d.adjust = 0;
        tiles[t] = d;
    }
}

// Under lazy module loading a kernel's code is loaded (device memory taken)
// at its first launch; querying each kernel's attributes loads them now.
cudaError_t preload_sort_in_scratch()
{
    cudaFuncAttributes fa;
    const void *fns[] = {reinterpret_cast<const void *>(k_single_segment_tiles),
                         reinterpret_cast<const void *>(k_radix_count), reinterpret_cast<const void *>(k_radix_scatter),
                         reinterpret_cast<const void *>(k_scan_reduce), reinterpret_cast<const void *>(k_scan_top),
                         reinterpret_cast<const void *>(k_scan_down)};
    for (const void *f : fns) {
        const cudaError_t e = cudaFuncGetAttributes(&fa, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_radix_sort_in_scratch(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits,
                                         void *tmp, cudaStream_t st)
{
    if (n <= 1 || bits == 0) return cudaSuccess;
    const uint64_t n_tiles = (n + RS_TILE - 1) / RS_TILE;
    const uint64_t nc = 256 * n_tiles;
    uint8_t *p = static_cast<uint8_t *>(tmp);
    unsigned long long *k2 = reinterpret_cast<unsigned long long *>(p);
    p += align256(n * 8);
    uint32_t *v2 = reinterpret_cast<uint32_t *>(p);
    p += align256(n * 4);
    uint32_t *counts = reinterpret_cast<uint32_t *>(p);
    p += align256(nc * 4);
    unsigned long long *offs = reinterpret_cast<unsigned long long *>(p);
    p += align256(nc * 8);
    unsigned long long *stmp = reinterpret_cast<unsigned long long *>(p);
    p += align256(scan_tmp_words(nc) * 8);
    SortTile *d_tiles = reinterpret_cast<SortTile *>(p);
    note_launch();
    k_single_segment_tiles<<<grid_for(n_tiles, 256), 256, 0, st>>>(d_tiles, n, n_tiles);
    const size_t smem = RS_TILE * 8 + RS_TILE * 4 + 8 * 256 * 4 + 256 * 4;
    cudaError_t e = cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    unsigned long long *ks = keys, *kd = k2;
    uint32_t *vs = vals, *vd = v2;
    const uint32_t passes = (bits + 7) / 8;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t shift = pass * 8;
        note_launch();
        k_radix_count<<<(unsigned)n_tiles, RS_THREADS, 0, st>>>(ks, d_tiles, shift, counts);
        e = launch_scan_u32(counts, offs, nc, stmp, st);
        if (e != cudaSuccess) return e;
        note_launch();
        k_radix_scatter<<<(unsigned)n_tiles, RS_THREADS, smem, st>>>(ks, vs, kd, vd, d_tiles, shift, offs);
        std::swap(ks, kd);
        std::swap(vs, vd);
    }
    if (ks != keys) {
        e = cudaMemcpyAsync(keys, ks, n * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vals, vs, n * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_radix_sort(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits, void *tmp,
                              cudaStream_t st, unsigned long long *flags, uint32_t skip_bits, bool input_in_tmp)
{
    if (bits > 64 || skip_bits % 8) return cudaErrorInvalidValue;
    const uint32_t passes = (bits + 7) / 8;
    const uint64_t n_tiles = (n + RS_TILE - 1) / RS_TILE;
    uint8_t *p = static_cast<uint8_t *>(tmp);
    unsigned long long *k2 = reinterpret_cast<unsigned long long *>(p);
    p += align256(n * 8);
    uint32_t *v2 = reinterpret_cast<uint32_t *>(p);
    p += align256(n * 4);
    unsigned long long *hist = reinterpret_cast<unsigned long long *>(p);
    p += align256(OS_MAX_PASSES * 256 * 8);
    unsigned long long *look = reinterpret_cast<unsigned long long *>(p);
    p += align256(n_tiles * 256 * 8);
    unsigned int *tile_ctr = reinterpret_cast<unsigned int *>(p);
    unsigned long long *own_flags = reinterpret_cast<unsigned long long *>(p + OS_MAX_PASSES * 4);
    if (!flags) flags = own_flags;
    // records placed in the alternate buffers (input_in_tmp) end in keys/vals
    // after an odd number of passes without the final copy
    unsigned long long *ks = keys, *kd = k2;
    uint32_t *vs = vals, *vd = v2;
    if (input_in_tmp) {
        std::swap(ks, kd);
        std::swap(vs, vd);
    }
    cudaError_t e = cudaSuccess;
    if (n > 1 && bits && skip_bits / 8 < passes) {
        e = cudaMemsetAsync(hist, 0, OS_MAX_PASSES * 256 * 8, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(look, 0, n_tiles * 256 * 8, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(tile_ctr, 0, OS_MAX_PASSES * 4 + 8, st);
        if (e != cudaSuccess) return e;
        note_launch();
        k_radix_hist_all<<<grid_for(n, 256, 4), 256, 0, st>>>(ks, n, passes, hist);
    }
    const size_t smem = RS_TILE * 8 + RS_TILE * 4 + 8 * 256 * 4;
    e = cudaFuncSetAttribute(k_radix_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    for (uint32_t pass = skip_bits / 8; n > 1 && pass < passes; ++pass) {
        note_launch();
        k_radix_onesweep<<<(unsigned)n_tiles, RS_THREADS, smem, st>>>(ks, vs, kd, vd, n, pass, hist, look, tile_ctr,
                                                                      flags, nullptr);
        std::swap(ks, kd);
        std::swap(vs, vd);
    }
    if (ks != keys && n) {
        e = cudaMemcpyAsync(keys, ks, n * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vals, vs, n * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

uint64_t compact_chunks_of(uint64_t slot_cap) { return (slot_cap + COMPACT_CHUNK - 1) / COMPACT_CHUNK; }

cudaError_t launch_compact_chunks(const Slot *slots, const SampleCfg *cfg, const uint32_t *chunk0, uint32_t n_samples,
                                  uint64_t n_chunks, uint32_t *chunk_keep, const unsigned long long *chunk_pos,
                                  unsigned long long *rec_keys, uint32_t *rec_counts, unsigned long long *hist,
                                  unsigned long long *ovf, uint64_t ovf_cap, unsigned long long *distinct,
                                  unsigned long long *counters, int count_only, cudaStream_t st)
{
    if (!n_chunks || !n_samples) return cudaSuccess;
    const size_t smem = ((size_t)n_samples + 1) * 4;
    cudaError_t e = cudaFuncSetAttribute(k_compact_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint64_t grid = std::min<uint64_t>(n_chunks, (uint64_t)sm_count() * 8);
    note_launch();
    k_compact_chunks<<<(unsigned)grid, 256, smem, st>>>(slots, cfg, chunk0, n_samples, n_chunks, chunk_keep, chunk_pos,
                                                         rec_keys, rec_counts, hist, ovf, ovf_cap, distinct, counters,
                                                         count_only);
    return cudaGetLastError();
}

cudaError_t launch_pair_reverse(unsigned long long *keys, uint64_t n, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_pair_reverse<<<grid_for(n, 256), 256, 0, st>>>(keys, n);
    return cudaGetLastError();
}

cudaError_t launch_select_range(const unsigned long long *keys, const uint32_t *counts, uint64_t n, uint32_t lo,
                                uint32_t hi, uint64_t limit, unsigned long long *out_keys, uint32_t *out_counts,
                                uint32_t *flags, unsigned long long *pos, unsigned long long *tmp,
                                unsigned long long *counters, int counter_idx, cudaStream_t st)
{
    if (!n) return cudaMemsetAsync(&counters[counter_idx], 0, 8, st);
    note_launch();
    k_range_flags<<<grid_for(n, 256), 256, 0, st>>>(counts, n, lo, hi, flags);
    cudaError_t e = launch_scan_u32(flags, pos, n, tmp, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_scatter_selected<<<grid_for(n, 256), 256, 0, st>>>(keys, counts, flags, pos, n, limit, out_keys, out_counts,
                                                         counters, counter_idx);
    return cudaGetLastError();
}

template <typename K>
static int persistent_grid(K kernel)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return sm_count() * per_sm;
}

uint32_t fill_item_starts_n(BucketRanges &r, uint64_t item_keys)
{
    uint32_t n = 0;
    for (uint32_t b = 0; b < N_BUCKETS; ++b) {
        r.item0[b] = n;
        n += (uint32_t)((r.len[b] + item_keys - 1) / item_keys);
    }
    r.item0[N_BUCKETS] = n;
    return n;
}

uint32_t fill_item_starts(BucketRanges &r) { return fill_item_starts_n(r, WORK_ITEM_KEYS); }

cudaError_t launch_bloom_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 unsigned int *next_item, const BucketCfg *cfg, unsigned long long *bits,
                                 unsigned long long *out, unsigned long long *low_cnt, unsigned long long *high_cnt,
                                 uint32_t *hll_high, cudaStream_t st)
{
    if (!n_items) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next_item, 0, 4, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_bloom_buckets<<<std::min<int>(persistent_grid(k_bloom_buckets), n_items), 256, 0, st>>>(
        keys, rg, n_items, next_item, cfg, bits, out, low_cnt, high_cnt, hll_high);
    return cudaGetLastError();
}

cudaError_t launch_insert_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                  unsigned int *next_item, const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                  unsigned long long *bucket_ovf, cudaStream_t st)
{
    if (!n_items) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next_item, 0, 4, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_insert_buckets<<<std::min<int>(persistent_grid(k_insert_buckets), n_items), 256, 0, st>>>(
        keys, rg, n_items, next_item, cfg, arena, max_probe, bucket_ovf);
    return cudaGetLastError();
}

cudaError_t launch_merge_buckets(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 unsigned int *next_item, const BucketCfg *cfg, Slot *arena, uint32_t max_probe,
                                 uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                                 uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *counters, cudaStream_t st)
{
    if (!n_items) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(next_item, 0, 4, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_merge_buckets<<<std::min<int>(persistent_grid(k_merge_buckets), n_items), 256, 0, st>>>(
        keys, rg, n_items, next_item, cfg, arena, max_probe, min_count, max_count, rec_keys, rec_counts, rec_cap,
        counters);
    return cudaGetLastError();
}

cudaError_t launch_subpart_count(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                 const SubCfg *sc, uint32_t *sub_count, cudaStream_t st, uint32_t stride)
{
    if (!n_items) return cudaSuccess;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subpart_count, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint32_t grid = std::min<uint32_t>(n_items, (uint32_t)(sm_count() * per_sm));
    note_launch();
    k_subpart_count<<<grid, 256, 0, st>>>(keys, rg, n_items, sc, sub_count, stride < 1 ? 1u : stride);
    return cudaGetLastError();
}

cudaError_t launch_subpart_regions(const uint32_t *sampled, uint32_t n_sub, uint32_t stride, uint32_t *region,
                                   unsigned long long *sub_off, unsigned long long *sub_end,
                                   unsigned long long *sub_cursor, unsigned long long *scan_tmp, cudaStream_t st)
{
    if (!n_sub) return cudaSuccess;
    note_launch();
    k_subpart_regions<<<grid_for(n_sub, 256), 256, 0, st>>>(sampled, n_sub, stride, region);
    cudaError_t e = launch_scan_u32(region, sub_off, n_sub, scan_tmp, st);
    if (e != cudaSuccess) return e;
    note_launch();
    k_subpart_ends<<<grid_for(n_sub, 256), 256, 0, st>>>(sub_off, region, n_sub, sub_end, sub_cursor);
    return cudaGetLastError();
}

cudaError_t launch_subpart_sizes(const unsigned long long *sub_off, const unsigned long long *sub_cursor,
                                 const unsigned long long *sub_end, uint32_t n_sub, uint64_t out_cap, uint32_t *count,
                                 unsigned long long *overflow, cudaStream_t st)
{
    if (!n_sub) return cudaSuccess;
    note_launch();
    k_subpart_sizes<<<grid_for(n_sub, 256), 256, 0, st>>>(sub_off, sub_cursor, sub_end, n_sub, out_cap, count, overflow);
    return cudaGetLastError();
}

static size_t subpart_scatter_smem(uint32_t max_sub)
{
    return (size_t)SUB_SCATTER_ITEM_KEYS * (8 + 2) + (size_t)max_sub * (8 + 4 + 4);
}

cudaError_t launch_subpart_scatter(const unsigned long long *keys, const BucketRanges *rg, uint32_t n_items,
                                   unsigned int *next_item, const SubCfg *sc, unsigned long long *sub_cursor,
                                   unsigned long long *out, uint64_t out_cap, uint32_t max_sub, cudaStream_t st,
                                   const unsigned long long *sub_end, uint32_t scatter_shape)
{
    if (!n_items) return cudaSuccess;
    if (!max_sub || max_sub > SUB_MAX_PER_BUCKET) return cudaErrorInvalidValue;
    max_sub = (max_sub + 1) & ~1u;   // keeps the 2-byte array after the 4-byte ones aligned
    cudaError_t e = cudaMemsetAsync(next_item, 0, 4, st);
    if (e != cudaSuccess) return e;
    const size_t smem = subpart_scatter_smem(max_sub);
    auto kern = (scatter_shape == 2 && max_sub <= 2 * SP_THREADS) ? k_subpart_scatter<2, 3>
                                                                  : k_subpart_scatter<SP_MAX_BINS, 2>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SP_THREADS, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint32_t grid = std::min<uint32_t>(n_items, (uint32_t)(sm_count() * per_sm));
    note_launch();
    kern<<<grid, SP_THREADS, smem, st>>>(keys, rg, n_items, next_item, sc, sub_cursor, sub_end, out, out_cap, max_sub);
    return cudaGetLastError();
}

template <uint32_t THREADS, uint32_t BPSM, uint32_t SLICE, uint32_t TBITS, uint32_t HBINS, bool FIB>
static cudaError_t launch_count_subs_t(unsigned long long *keys, const unsigned long long *sub_off,
                                       const uint32_t *sub_count, const uint8_t *sub_bucket, uint32_t n_sub,
                                       const SubCfg *sc, unsigned int *next_sub, uint32_t count_max,
                                       uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                                       uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist, uint32_t *ovf,
                                       uint64_t ovf_cap, unsigned long long *counters, uint32_t *bucket_ovf,
                                       cudaStream_t st, uint32_t *hb16, uint32_t hb16_shift)
{
    const size_t smem = (size_t)2 * SLICE * 8 + ((size_t)1 << TBITS) * (8 + 4) + HBINS * 4 +
                        (size_t)THREADS * SUB_PER_THREAD * 8;
    auto kern = k_count_subs<THREADS, BPSM, SLICE, TBITS, HBINS, FIB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t grid = std::min<uint32_t>(n_sub, (uint32_t)sm_count() * BPSM);
    note_launch();
    kern<<<grid, THREADS, smem, st>>>(keys, sub_off, sub_count, sub_bucket, n_sub, sc, next_sub, count_max, min_count,
                                      max_count, rec_keys, rec_counts, rec_cap, hist, ovf, ovf_cap, counters, bucket_ovf,
                                      hb16, hb16_shift);
    return cudaGetLastError();
}

cudaError_t launch_count_subs(unsigned long long *keys, const unsigned long long *sub_off, const uint32_t *sub_count,
                              const uint8_t *sub_bucket, uint32_t n_sub, const SubCfg *sc, unsigned int *next_sub,
                              uint32_t count_max, uint32_t min_count, uint32_t max_count, unsigned long long *rec_keys,
                              uint32_t *rec_counts, uint64_t rec_cap, unsigned long long *hist, uint32_t *ovf,
                              uint64_t ovf_cap, unsigned long long *counters, uint32_t *bucket_ovf, cudaStream_t st,
                              uint32_t *hb16, uint32_t hb16_shift, uint32_t shape)
{
    if (!n_sub) return cudaSuccess;
    if (min_count < 2) return cudaErrorInvalidValue;   // singletons are not records on this path
    cudaError_t e = cudaMemsetAsync(next_sub, 0, 4, st);
    if (e != cudaSuccess) return e;
#define KC_COUNT_SUBS_ARGS                                                                                         \
    keys, sub_off, sub_count, sub_bucket, n_sub, sc, next_sub, count_max, min_count, max_count, rec_keys, rec_counts, \
        rec_cap, hist, ovf, ovf_cap, counters, bucket_ovf, st, hb16, hb16_shift
    switch (shape) {
    case 2: return launch_count_subs_t<256, 4, 1024, 11, 1024, false>(KC_COUNT_SUBS_ARGS);
    case 3: return launch_count_subs_t<512, 2, 2048, 12, 2048, true>(KC_COUNT_SUBS_ARGS);
    case 4: return launch_count_subs_t<256, 4, 1024, 11, 1024, true>(KC_COUNT_SUBS_ARGS);
    default: return launch_count_subs_t<512, 2, 2048, 12, 2048, false>(KC_COUNT_SUBS_ARGS);
    }
#undef KC_COUNT_SUBS_ARGS
}

cudaError_t launch_wait_flag(const unsigned int *flag, uint32_t poll_limit, unsigned long long *flags, cudaStream_t st)
{
    note_launch();
    k_wait_flag<<<1, 32, 0, st>>>(flag, poll_limit, flags);
    return cudaGetLastError();
}

cudaError_t launch_or_flags(unsigned long long *word, unsigned long long bits, cudaStream_t st)
{
    note_launch();
    k_or_flags<<<1, 32, 0, st>>>(word, bits);
    return cudaGetLastError();
}

cudaError_t launch_hash_batch(const unsigned long long *keys, uint64_t n, unsigned long long *out, cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_hash_batch<<<grid_for(n, 256), 256, 0, st>>>(keys, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// text dump (the reference dump_tool's "KMER\tcount\n" lines)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t dec_digits(uint32_t v)
{
    uint32_t d = 1;
    while (v >= 10) {
        v /= 10;
        ++d;
    }
    return d;
}

// Length of record i's line: k bases, a tab, the count in decimal, a newline.
__global__ void k_dump_lengths(const uint32_t *counts, uint64_t n, uint32_t k, uint32_t *len)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        len[i] = k + 2 + dec_digits(counts[i]);
}

// Base i of the printed string of a kmer<N> key (kmer_to_buf,
// tool/dump_tool.cpp:103-124): for N = 1 bit 64-2k+2i of the word; for
// N > 1 the first k % 32 bases from data[k / 32]'s top bits, the rest from
// data[k / 32 - 1] downwards, each word from its low bits up.
template <uint32_t N>
__device__ __forceinline__ uint32_t key_base(const unsigned long long *w, uint32_t k, uint32_t i)
{
    if (N == 1) return (uint32_t)(w[0] >> (64 - 2 * k + 2 * i)) & 3u;
    const uint32_t full = k / 32, tail = k % 32;
    if (i < tail) return (uint32_t)(w[full] >> (64 - 2 * tail + 2 * i)) & 3u;
    const uint32_t off = i - tail;
    return (uint32_t)(w[full - 1 - off / 32] >> (2 * (off % 32))) & 3u;
}

// Each block formats 256 consecutive lines into shared memory and copies them
// out as one run of bytes starting at the first line's offset.
constexpr uint32_t DUMP_MAX_LINE = 128 + 2 + 10;

template <uint32_t N>
__global__ void __launch_bounds__(256) k_dump_write(const unsigned long long *keys, const uint32_t *counts,
                                                    uint64_t n, uint32_t k, const unsigned long long *off,
                                                    char *out)
{
    __shared__ char s_txt[256 * DUMP_MAX_LINE];
    const uint64_t first = blockIdx.x * 256ull;
    if (first >= n) return;
    const uint64_t last = first + 256 < n ? first + 255 : n - 1;
    const unsigned long long base = off[first];
    const uint64_t i = first + threadIdx.x;
    if (i < n) {
        char *p = s_txt + (off[i] - base);
        unsigned long long w[N];
#pragma unroll
        for (uint32_t j = 0; j < N; ++j) w[j] = keys[i * N + j];
        for (uint32_t b = 0; b < k; ++b) p[b] = "ACGT"[key_base<N>(w, k, b)];
        p[k] = '\t';
        uint32_t c = counts[i];
        const uint32_t nd = dec_digits(c);
        for (uint32_t d = nd; d > 0; --d) {
            p[k + d] = (char)('0' + c % 10);
            c /= 10;
        }
        p[k + 1 + nd] = '\n';
    }
    __syncthreads();
    const uint64_t bytes = off[last] + k + 2 + dec_digits(counts[last]) - base;
    for (uint64_t j = threadIdx.x; j < bytes; j += 256) out[base + j] = s_txt[j];
}

cudaError_t launch_dump_text(const unsigned long long *keys, const uint32_t *counts, uint64_t n, uint32_t k,
                             uint32_t *len, unsigned long long *off, unsigned long long *scan_tmp, char *out,
                             cudaStream_t st)
{
    if (!n) return cudaSuccess;
    note_launch();
    k_dump_lengths<<<grid_for(n, 256), 256, 0, st>>>(counts, n, k, len);
    cudaError_t e = launch_scan_u32(len, off, n, scan_tmp, st);
    if (e != cudaSuccess) return e;
    note_launch();
    const unsigned g = (unsigned)((n + 255) / 256);
    if (k <= 32) k_dump_write<1><<<g, 256, 0, st>>>(keys, counts, n, k, off, out);
    else if (k <= 64) k_dump_write<2><<<g, 256, 0, st>>>(keys, counts, n, k, off, out);
    else k_dump_write<4><<<g, 256, 0, st>>>(keys, counts, n, k, off, out);
    return cudaGetLastError();
}

// Random 32-bit atomicAdd throughput: every thread adds 1 at `iters`
// pseudo-random word indexes (xorshift64*, independent per thread) of a buffer
// of mask+1 words.  With a buffer far larger than L2 each add is a DRAM
// read-modify-write of one 32-byte sector; with a buffer that fits in L2 it
// measures the L2 atomic units.  The adds do not use their return value (the
// counting tables' count increments do not either).
__global__ void __launch_bounds__(256) k_atomic_peak(uint32_t *buf, uint64_t mask, uint32_t iters, uint64_t seed)
{
    uint64_t x = seed ^ ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x + 1) * 0x9E3779B97F4A7C15ull);
    x ^= x >> 31;
    if (!x) x = 1;
#pragma unroll 4
    for (uint32_t i = 0; i < iters; ++i) {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        atomicAdd(buf + ((x * 0x2545F4914F6CDD1Dull) >> 20 & mask), 1u);
    }
}

cudaError_t launch_atomic_peak(uint32_t *buf, uint64_t words, uint32_t iters, uint64_t seed, uint64_t *ops,
                               cudaStream_t st)
{
    const unsigned grid = (unsigned)sm_count() * 8;
    *ops = (uint64_t)grid * 256 * iters;
    note_launch();
    k_atomic_peak<<<grid, 256, 0, st>>>(buf, words - 1, iters, seed);
    return cudaGetLastError();
}

// The same random atomicAdd on a table of mask+1 words in shared memory, one
// table per block, with the shared-memory count's block shape (512 threads,
// two blocks per SM).  Each block adds its table into `out` at the end so
// that the adds are not dead code.
__global__ void __launch_bounds__(512, 2) k_atomic_peak_shared(uint32_t *out, uint32_t mask,
                                                                                        uint32_t iters, uint64_t seed)
{
    extern __shared__ uint32_t s_tab[];
    for (uint32_t i = threadIdx.x; i <= mask; i += blockDim.x) s_tab[i] = 0;
    __syncthreads();
    uint64_t x = seed ^ ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x + 1) * 0x9E3779B97F4A7C15ull);
    x ^= x >> 31;
    if (!x) x = 1;
#pragma unroll 4
    for (uint32_t i = 0; i < iters; ++i) {
        x ^= x >> 12;
        x ^= x << 25;
        x ^= x >> 27;
        atomicAdd(&s_tab[(uint32_t)((x * 0x2545F4914F6CDD1Dull) >> 32) & mask], 1u);
    }
    __syncthreads();
    uint32_t sum = 0;
    for (uint32_t i = threadIdx.x; i <= mask; i += blockDim.x) sum += s_tab[i];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(FULL, sum, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, sum);
}

cudaError_t launch_atomic_peak_shared(uint32_t *out, uint32_t words, uint32_t iters, uint64_t seed, uint64_t *ops,
                                      cudaStream_t st)
{
    const unsigned grid = (unsigned)sm_count() * 2 * 4;
    const size_t smem = (size_t)words * 4;
    cudaError_t e = cudaFuncSetAttribute(k_atomic_peak_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    *ops = (uint64_t)grid * 512 * iters;
    note_launch();
    k_atomic_peak_shared<<<grid, 512, smem, st>>>(out, words - 1, iters, seed);
    return cudaGetLastError();
}

}  // namespace kc
