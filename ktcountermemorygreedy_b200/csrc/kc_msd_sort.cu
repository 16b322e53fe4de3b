// kc_msd_sort.cu -- the sort of a job's records in printed-string order,
// most significant bits first (the reference sorts its dump with an 11-bit
// LSD radix sort over the whole key, tool/dump_tool.cpp:357-454).
//
// The records' keys are distinct, so a sort needs no stability across equal
// keys.  Three passes over the records instead of one per 8-bit digit:
//   1. bucket histogram: the top P bits of each key (P = 8 + P2, P2 <= 8,
//      chosen so that a bucket holds about 1.5K records on average);
//   2. scatter by the top 8 bits, then within each of those 256 ranges by the
//      next P2 bits (each a single pass: ranks inside a tile by warp match,
//      across tiles by decoupled look-back, output offsets from the scanned
//      bucket histogram, records reordered in shared memory so that runs of one
//      digit are written to consecutive addresses);
//   3. every bucket sorted in shared memory: placed by the next 8 bits (warp
//      match ranks), then each of the 256 resulting runs of a few records
//      sorted by insertion; written back in place.
// Buckets larger than one block's shared memory (rare: the keys come from
// genome sequence, spread over the prefixes) are sorted afterwards one by one
// by the count/scan/scatter LSD sort on the bits below the prefix.
#include <algorithm>
#include <vector>

#include "kc_device.cuh"
#include "kc_kernels.cuh"

namespace kc {

namespace {

constexpr uint32_t FULLW = 0xffffffffu;
constexpr uint32_t MS_THREADS = 256;
constexpr uint32_t MS_ITEMS = 16;
constexpr uint32_t MS_TILE = MS_THREADS * MS_ITEMS;   // records per scatter tile and per bucket block
constexpr uint32_t MS_WARP_ITEMS = 32 * MS_ITEMS;
constexpr int LB_BITS = 40;                             // value field of a look-back word
constexpr unsigned long long LB_MASK = (1ull << LB_BITS) - 1;
constexpr unsigned long long TAG_AGG = 1, TAG_INC = 2;  // tile aggregate / inclusive prefix

struct MsdTile {
    uint64_t begin, end;   // record range
    uint32_t first_tile;   // first tile of the tile's segment (the look-back stops there)
    uint32_t seg;          // segment (pass 2: the records' top 8 bits)
};

__device__ __forceinline__ uint32_t lanes_below()
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
        uint32_t w = lane < 8 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULLW, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t base = warp ? s_warp[warp - 1] : 0u;
    total = s_warp[7];
    __syncthreads();
    return base + x - v;
}

// Records per bucket: hb[(key >> shift) & bmask] += 1 (the mask keeps bits
// above the sorted ones out of the index).
__global__ void __launch_bounds__(256) k_msd_hist(const unsigned long long *keys, uint64_t n, uint32_t shift,
                                                  uint32_t bmask, uint32_t *hb)
{
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (uint64_t)gridDim.x * 256)
        atomicAdd(&hb[(uint32_t)(__ldcs(&keys[i]) >> shift) & bmask], 1u);
}

// hb[b] = the 2^(16 - P) counts of hist16 under bucket b (the top P of the
// key's top 16 bits).
__global__ void k_msd_hist_fold(const uint32_t *hist16, uint32_t p_bits, uint32_t *hb)
{
    const uint32_t nb = 1u << p_bits, per = 1u << (16 - p_bits);
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (uint32_t j = 0; j < per; ++j) c += hist16[b * per + j];
        hb[b] = c;
    }
}

// Stable ranks of the items of one block among the items with the same digit,
// in item order: items are blocked per warp (warp w holds items
// w * per_warp + r * 32 + lane, r < steps), so per-warp digit counters taken
// in order and then added up over the warps give the ranks.  rd[r] = rank << 16
// | digit (digit 256: no item).  On return s_wcnt[w * 256 + d] holds the
// items of digit d in warps before w, s_start[d] the items of smaller digits.
__device__ __forceinline__ void rank_items(const unsigned long long (&k)[MS_ITEMS], uint32_t (&rd)[MS_ITEMS],
                                           uint32_t base_item, uint32_t n_items, uint32_t shift, uint32_t dmask,
                                           uint32_t steps, uint32_t *s_wcnt, uint32_t *s_start, uint32_t *s_warp,
                                           uint32_t &own_out)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 8 * 256; i += MS_THREADS) s_wcnt[i] = 0;
    __syncthreads();
    uint32_t *wc = s_wcnt + warp * 256;
    const uint32_t lt = lanes_below();
#pragma unroll
    for (uint32_t r = 0; r < MS_ITEMS; ++r) {
        if (r >= steps) break;
        const uint32_t li = base_item + r * 32 + lane;
        const bool act = li < n_items;
        const uint32_t d = act ? (uint32_t)((k[r] >> shift) & dmask) : 256u;
        const uint32_t peers = __match_any_sync(FULLW, d);
        const uint32_t before = __popc(peers & lt);
        const uint32_t cnt = act ? wc[d] : 0u;
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
    uint32_t tot;
    s_start[tid] = scan256(own, s_warp, tot);
    own_out = own;
    __syncthreads();
}

// One scatter pass by the digit (key >> shift) & dmask.  Records of digit d
// in segment s go to ob[(s << seg_sh) | (d << dig_sh)] plus their rank among
// the segment's records of that digit.  Tiles are taken in launch order from
// *tile_ctr, so a tile only waits on tiles of blocks that already run; a wait
// that exceeds SPIN_LIMIT polls sets ERR_WAIT_TIMEOUT in *flags, and the
// writes stay inside [0, n).
__global__ void __launch_bounds__(MS_THREADS, 2) k_msd_scatter(const unsigned long long *kin, const uint32_t *vin,
                                                               unsigned long long *kout, uint32_t *vout, uint64_t n,
                                                               const MsdTile *tiles, uint32_t shift, uint32_t dmask,
                                                               uint32_t seg_sh, uint32_t dig_sh,
                                                               const unsigned long long *ob, unsigned long long *look,
                                                               unsigned int *tile_ctr, unsigned long long *flags)
{
    extern __shared__ __align__(16) uint8_t ms_smem[];
    unsigned long long *s_keys = reinterpret_cast<unsigned long long *>(ms_smem);   // MS_TILE
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + MS_TILE);              // MS_TILE
    uint32_t *s_wcnt = s_vals + MS_TILE;                                            // 8 x 256
    __shared__ uint32_t s_start[256], s_warp[8], s_tile;
    __shared__ unsigned long long s_dst[256];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t j = s_tile;
    const MsdTile tl = tiles[j];
    const uint32_t tile_n = (uint32_t)(tl.end - tl.begin);

    unsigned long long k[MS_ITEMS];
    uint32_t v[MS_ITEMS], rd[MS_ITEMS];
#pragma unroll
    for (uint32_t r = 0; r < MS_ITEMS; ++r) {
        const uint32_t li = warp * MS_WARP_ITEMS + r * 32 + lane;
        const bool act = li < tile_n;
        k[r] = act ? __ldcs(&kin[tl.begin + li]) : 0ull;
        v[r] = act ? __ldcs(&vin[tl.begin + li]) : 0u;
    }
    uint32_t own;
    rank_items(k, rd, warp * MS_WARP_ITEMS, tile_n, shift, dmask, MS_ITEMS, s_wcnt, s_start, s_warp, own);

    // publish this tile's count of digit tid, then add up the tiles before it
    volatile unsigned long long *mine = look + (uint64_t)j * 256 + tid;
    *mine = ((j == tl.first_tile ? TAG_INC : TAG_AGG) << LB_BITS) | own;
    unsigned long long excl = 0;
    if (j > tl.first_tile) {
        bool gave_up = false;
        for (int64_t p = (int64_t)j - 1; p >= (int64_t)tl.first_tile; --p) {
            const volatile unsigned long long *w = look + (uint64_t)p * 256 + tid;
            unsigned long long x = *w;
            uint32_t spins = 0;
            while ((x >> LB_BITS) < TAG_AGG) {
                if (++spins > SPIN_LIMIT) {
                    gave_up = true;
                    break;
                }
                __nanosleep(32);
                x = *w;
            }
            if (gave_up) break;
            excl += x & LB_MASK;
            if ((x >> LB_BITS) >= TAG_INC) break;
        }
        if (gave_up) atomicOr(flags, ERR_WAIT_TIMEOUT);
        *mine = (TAG_INC << LB_BITS) | (excl + own);
    }
    if ((uint32_t)tid <= dmask) s_dst[tid] = ob[((uint64_t)tl.seg << seg_sh) | ((uint64_t)tid << dig_sh)] + excl - s_start[tid];
    // reorder the tile by digit in shared memory
#pragma unroll
    for (uint32_t r = 0; r < MS_ITEMS; ++r) {
        const uint32_t d = rd[r] & 0xFFFFu;
        if (d < 256) {
            const uint32_t pos = s_start[d] + s_wcnt[warp * 256 + d] + (rd[r] >> 16);
            s_keys[pos] = k[r];
            s_vals[pos] = v[r];
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < tile_n; i += MS_THREADS) {
        const unsigned long long key = s_keys[i];
        const unsigned long long dst = s_dst[(uint32_t)((key >> shift) & dmask)] + i;
        if (dst < n) {   // only a look-back that gave up can point elsewhere
            kout[dst] = key;
            vout[dst] = s_vals[i];
        }
    }
}

// A bucket of at most ITEMS * 256 records is sorted in shared memory by one
// block.  Its records are loaded into registers in one batch (one memory
// latency per bucket) and placed by the 8 bits just below the bucket prefix
// (per-warp match ranks in record order: a pass to count, a pass to place),
// which cuts the bucket into 256 runs of a few records each; thread t then
// sorts run t by insertion on the key's low `bits` bits (all records of a run
// share every bit above the 8 placed ones, so this orders the whole bucket).
// Written back in place when kin == kout, with the 2-bit groups reversed when
// reverse_out.  The buckets come in size classes (blist: the buckets of this
// class), each class with as many blocks per SM as its registers and shared
// memory allow; buckets larger than BS_CAP go to the fallback.
constexpr uint32_t BS_CAP = MS_THREADS * 32;   // 8192

template <uint32_t ITEMS>
__global__ void __launch_bounds__(MS_THREADS, ITEMS <= 8 ? 5 : (ITEMS <= 16 ? 3 : 2))
    k_bucket_sort(const unsigned long long *kin, const uint32_t *vin, unsigned long long *kout, uint32_t *vout,
                  const uint32_t *hb, const unsigned long long *ob, const uint32_t *blist, uint32_t n_list,
                  uint32_t low_bits, uint32_t bits, int reverse_out)
{
    constexpr uint32_t BS_ITEMS = ITEMS, CAP = MS_THREADS * ITEMS;
    extern __shared__ __align__(16) uint8_t bs_smem[];
    unsigned long long *s_keys = reinterpret_cast<unsigned long long *>(bs_smem);   // CAP
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + CAP);                  // CAP
    uint32_t *s_wcnt = s_vals + CAP;                                                // 8 x 256
    __shared__ uint32_t s_start[257], s_warp[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t dsh = low_bits > 8 ? low_bits - 8 : 0;
    const uint32_t dmask = low_bits >= 8 ? 255u : ((1u << low_bits) - 1u);
    const unsigned long long kmask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);
    const uint32_t lt = lanes_below();
    uint32_t *wc = s_wcnt + warp * 256;
    for (uint32_t bi = blockIdx.x; bi < n_list; bi += gridDim.x) {
        const uint32_t b = blist[bi];
        const uint32_t m = hb[b];
        const unsigned long long base = ob[b];
        if (m > CAP) continue;   // not in this class (the host lists never do this)
        if (m <= 1 || low_bits == 0) {
            for (uint32_t i = tid; i < m; i += MS_THREADS) {
                kout[base + i] = reverse_out ? pair_reverse(kin[base + i]) : kin[base + i];
                vout[base + i] = vin[base + i];
            }
            continue;
        }
        // records blocked per warp: warp w holds [w * per, (w + 1) * per),
        // loaded into registers together (one memory latency per bucket)
        const uint32_t per = ((m + 8 * 32 - 1) / (8 * 32)) * 32;
        const uint32_t steps = per / 32, first = warp * per;
        unsigned long long k[BS_ITEMS];
        uint32_t v[BS_ITEMS];
#pragma unroll
        for (uint32_t r = 0; r < BS_ITEMS; ++r) {
            const uint32_t li = first + r * 32 + lane;
            const bool act = r < steps && li < m;
            k[r] = act ? kin[base + li] : 0ull;
            v[r] = act ? vin[base + li] : 0u;
        }
        for (int i = tid; i < 8 * 256; i += MS_THREADS) s_wcnt[i] = 0;
        __syncthreads();
        // 1. count the records of every digit, per warp
#pragma unroll
        for (uint32_t r = 0; r < BS_ITEMS; ++r) {
            if (r >= steps) break;
            const bool act = first + r * 32 + lane < m;
            const uint32_t d = act ? (uint32_t)((k[r] >> dsh) & dmask) : 256u;
            const uint32_t peers = __match_any_sync(FULLW, d);
            const uint32_t before = __popc(peers & lt);
            const uint32_t cnt = act ? wc[d] : 0u;
            __syncwarp();
            if (act && before == 0) wc[d] = cnt + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t own = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint32_t c = s_wcnt[w * 256 + tid];
            s_wcnt[w * 256 + tid] = own;
            own += c;
        }
        uint32_t tot;
        s_start[tid] = scan256(own, s_warp, tot);
        if (tid == 0) s_start[256] = m;
        __syncthreads();
        // 2. place every record after the records of smaller digits and of
        // earlier warps, in record order within the warp
#pragma unroll
        for (uint32_t r = 0; r < BS_ITEMS; ++r) {
            if (r >= steps) break;
            const bool act = first + r * 32 + lane < m;
            const uint32_t d = act ? (uint32_t)((k[r] >> dsh) & dmask) : 256u;
            const uint32_t peers = __match_any_sync(FULLW, d);
            const uint32_t before = __popc(peers & lt);
            const uint32_t cnt = act ? wc[d] : 0u;
            __syncwarp();
            if (act && before == 0) wc[d] = cnt + __popc(peers);
            __syncwarp();
            if (act) {
                const uint32_t pos = s_start[d] + cnt + before;
                s_keys[pos] = k[r];
                s_vals[pos] = v[r];
            }
        }
        __syncthreads();
        // 3. run tid sorted by insertion
        {
            const uint32_t lo = s_start[tid], hi = s_start[tid + 1];
            for (uint32_t i = lo + 1; i < hi; ++i) {
                const unsigned long long key = s_keys[i];
                const unsigned long long km = key & kmask;
                const uint32_t val = s_vals[i];
                uint32_t j = i;
                while (j > lo && (s_keys[j - 1] & kmask) > km) {
                    s_keys[j] = s_keys[j - 1];
                    s_vals[j] = s_vals[j - 1];
                    --j;
                }
                s_keys[j] = key;
                s_vals[j] = val;
            }
        }
        __syncthreads();
        for (uint32_t i = tid; i < m; i += MS_THREADS) {
            kout[base + i] = reverse_out ? pair_reverse(s_keys[i]) : s_keys[i];
            vout[base + i] = s_vals[i];
        }
        __syncthreads();
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

int n_sms()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

// Prefix bits of the buckets for n records of `bits` bits: 8 + P2 with the
// average bucket near 1.5K records, at most 16 and leaving bits below.
uint32_t msd_prefix_bits(uint64_t n, uint32_t bits)
{
    uint32_t p = 8;
    while (p < 16 && p + 1 < bits && (n >> p) > 1536) ++p;
    return p;
}

uint64_t msd_max_tiles(uint64_t n) { return (n + MS_TILE - 1) / MS_TILE + 256; }

template <uint32_t ITEMS>
cudaError_t launch_bucket_class(const unsigned long long *kin, const uint32_t *vin, unsigned long long *kout,
                                uint32_t *vout, const uint32_t *hb, const unsigned long long *ob, const uint32_t *blist,
                                uint32_t n_list, uint32_t low_bits, uint32_t bits, bool reverse_out, cudaStream_t st)
{
    const size_t smem = (size_t)MS_THREADS * ITEMS * 12 + 8 * 256 * 4;
    cudaError_t e = cudaFuncSetAttribute(k_bucket_sort<ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bucket_sort<ITEMS>, MS_THREADS, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    note_kernel_launch();
    k_bucket_sort<ITEMS><<<(unsigned)std::min<uint64_t>(n_list, (uint64_t)n_sms() * per_sm), MS_THREADS, smem, st>>>(
        kin, vin, kout, vout, hb, ob, blist, n_list, low_bits, bits, reverse_out ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace

// Up to 2^16 buckets of about 3K records on average (BS_CAP leaves room for
// the skew of canonical k-mers' prefixes, whose first base is A or C more
// often); larger record sets take the LSD sort.
bool msd_sort_applies(uint64_t n, uint32_t bits)
{
    return n >= MSD_SORT_MIN_RECORDS && n <= (3072ull << 16) && bits >= 24 && bits <= 64;
}

// Working memory: the alternate key/value arrays at its start (the layout
// sort_tmp_alt describes), inside a region large enough for the fallback
// sort of any one bucket (sort_tmp_bytes_in_scratch(n)), then the bucket
// histogram and offsets, the scan's words, the look-back words and tile
// descriptors of both scatter passes, the tile counters and an error word.
size_t msd_sort_tmp_bytes(uint64_t n, uint32_t bits)
{
    const uint64_t nb = 1ull << msd_prefix_bits(n, bits);
    const uint64_t nt = msd_max_tiles(n);
    return align256(std::max<size_t>(sort_tmp_bytes_in_scratch(n), align256(n * 8) + align256(n * 4))) +
           align256(nb * 4) + align256(nb * 8) + align256(scan_tmp_words(nb) * 8) + align256(2 * nt * 256 * 8) +
           align256(2 * nt * sizeof(MsdTile)) + align256(16) + align256(nb * 4);
}

cudaError_t launch_msd_sort(unsigned long long *keys, uint32_t *vals, uint64_t n, uint32_t bits, void *tmp,
                            cudaStream_t st, unsigned long long *flags, bool input_in_tmp, bool reverse_out,
                            const uint32_t *hist16)
{
    if (!msd_sort_applies(n, bits)) return cudaErrorInvalidValue;
    const uint32_t P = msd_prefix_bits(n, bits), P2 = P - 8;
    const uint64_t nb = 1ull << P;
    const uint64_t nt_max = msd_max_tiles(n);
    uint8_t *p = static_cast<uint8_t *>(tmp);
    unsigned long long *k2 = reinterpret_cast<unsigned long long *>(p);
    uint32_t *v2 = reinterpret_cast<uint32_t *>(p + align256(n * 8));
    void *fallback_tmp = p;   // free again once the buckets are sorted
    p += align256(std::max<size_t>(sort_tmp_bytes_in_scratch(n), align256(n * 8) + align256(n * 4)));
    uint32_t *hb = reinterpret_cast<uint32_t *>(p);
    p += align256(nb * 4);
    unsigned long long *ob = reinterpret_cast<unsigned long long *>(p);
    p += align256(nb * 8);
    unsigned long long *stmp = reinterpret_cast<unsigned long long *>(p);
    p += align256(scan_tmp_words(nb) * 8);
    unsigned long long *look = reinterpret_cast<unsigned long long *>(p);
    p += align256(2 * nt_max * 256 * 8);
    MsdTile *d_tiles = reinterpret_cast<MsdTile *>(p);
    p += align256(2 * nt_max * sizeof(MsdTile));
    unsigned int *tile_ctr = reinterpret_cast<unsigned int *>(p);
    unsigned long long *own_flags = reinterpret_cast<unsigned long long *>(p + 8);
    uint32_t *d_blist = reinterpret_cast<uint32_t *>(p + align256(16));   // the buckets by size class
    if (!flags) flags = own_flags;

    // the records start in keys/vals (A), or in the alternate arrays (B)
    unsigned long long *ka = keys, *kb = k2;
    uint32_t *va = vals, *vb = v2;
    if (input_in_tmp) {
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    const uint32_t shift2 = bits - P;   // bits below the bucket prefix
    cudaError_t e = cudaMemsetAsync(hb, 0, nb * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(tile_ctr, 0, 16, st);
    if (e != cudaSuccess) return e;
    note_kernel_launch();
    if (hist16 && P <= 16)
        k_msd_hist_fold<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(hist16, P, hb);
    else
        k_msd_hist<<<n_sms() * 8, 256, 0, st>>>(ka, n, shift2, (uint32_t)(nb - 1), hb);
    e = launch_scan_u32(hb, ob, nb, stmp, st);
    if (e != cudaSuccess) return e;
    // the bucket sizes come to the host once: the second pass's tiles follow
    // the top-8-bit ranges, and oversized buckets go to the fallback
    std::vector<uint32_t> h(nb);
    e = cudaMemcpyAsync(h.data(), hb, nb * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    std::vector<MsdTile> tiles;
    tiles.reserve(2 * nt_max);
    const uint64_t nt1 = (n + MS_TILE - 1) / MS_TILE;
    for (uint64_t t = 0; t < nt1; ++t) tiles.push_back(MsdTile{t * MS_TILE, std::min<uint64_t>(n, (t + 1) * MS_TILE), 0, 0});
    std::vector<uint64_t> big_start, big_len;   // buckets of more than BS_CAP records
    std::vector<uint32_t> lists[3];               // buckets of at most 2048, 4096, 8192 records
    uint64_t at = 0;
    for (uint32_t s = 0; s < 256; ++s) {
        uint64_t len = 0;
        for (uint64_t d = 0; d < (1ull << P2); ++d) {
            const uint64_t b = ((uint64_t)s << P2) | d, m = h[b];
            if (m > BS_CAP) {
                big_start.push_back(at + len);
                big_len.push_back(m);
            } else {
                lists[m <= 2048 ? 0 : (m <= 4096 ? 1 : 2)].push_back((uint32_t)b);
            }
            len += m;
        }
        const uint32_t first = (uint32_t)(tiles.size() - nt1);
        for (uint64_t o = 0; o < len; o += MS_TILE)
            tiles.push_back(MsdTile{at + o, at + std::min<uint64_t>(len, o + MS_TILE), first, s});
        at += len;
    }
    if (at != n) return cudaErrorInvalidValue;
    const uint64_t nt2 = tiles.size() - nt1;
    std::vector<uint32_t> blist;
    blist.reserve(nb);
    for (auto &l : lists) blist.insert(blist.end(), l.begin(), l.end());
    if (!blist.empty()) e = cudaMemcpyAsync(d_blist, blist.data(), blist.size() * 4, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(MsdTile), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(look, 0, (nt1 + nt2) * 256 * 8, st);
    if (e != cudaSuccess) return e;
    const size_t smem = MS_TILE * 12 + 8 * 256 * 4;
    e = cudaFuncSetAttribute(k_msd_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // pass 1: top 8 bits, A -> B; pass 2: the next P2 bits inside each top-8 range, B -> A
    note_kernel_launch();
    k_msd_scatter<<<(unsigned)nt1, MS_THREADS, smem, st>>>(ka, va, kb, vb, n, d_tiles, bits - 8, 255u, 0, P2, ob, look,
                                                          tile_ctr, flags);
    if (P2) {
        note_kernel_launch();
        k_msd_scatter<<<(unsigned)nt2, MS_THREADS, smem, st>>>(kb, vb, ka, va, n, d_tiles + nt1, shift2,
                                                              (1u << P2) - 1u, P2, 0, ob, look + nt1 * 256,
                                                              tile_ctr + 1, flags);
    }
    unsigned long long *ks = P2 ? ka : kb;   // where the bucketed records are
    uint32_t *vs = P2 ? va : vb;
    uint32_t off = 0;
    for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
        const uint32_t nl = (uint32_t)lists[c].size();
        if (nl) {
            if (c == 0) e = launch_bucket_class<8>(ks, vs, keys, vals, hb, ob, d_blist + off, nl, shift2, bits, reverse_out, st);
            if (c == 1) e = launch_bucket_class<16>(ks, vs, keys, vals, hb, ob, d_blist + off, nl, shift2, bits, reverse_out, st);
            if (c == 2) e = launch_bucket_class<32>(ks, vs, keys, vals, hb, ob, d_blist + off, nl, shift2, bits, reverse_out, st);
        }
        off += nl;
    }
    // the buckets too large for a block start where the fallback sorts them
    if (ks != keys)
        for (size_t i = 0; i < big_start.size() && e == cudaSuccess; ++i) {
            e = cudaMemcpyAsync(keys + big_start[i], ks + big_start[i], big_len[i] * 8, cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(vals + big_start[i], vs + big_start[i], big_len[i] * 4, cudaMemcpyDeviceToDevice, st);
        }
    if (e != cudaSuccess) return e;
    // buckets too large for one block: each sorted on its own on the bits
    // below the prefix, with the alternate arrays as working memory
    for (size_t i = 0; i < big_start.size() && e == cudaSuccess; ++i) {
        e = launch_radix_sort_in_scratch(keys + big_start[i], vals + big_start[i], big_len[i], shift2, fallback_tmp, st);
        if (e == cudaSuccess && reverse_out) e = launch_pair_reverse(keys + big_start[i], big_len[i], st);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace kc
