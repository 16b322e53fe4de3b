// kc_device.cuh -- device-side building blocks shared by the kernels:
// 2-bit k-mer word helpers, the reference's hash functions reproduced
// bit-for-bit for the 8-byte kmer<1> input, and the bounded-spin helpers.
#pragma once

#include <cstdint>

namespace kc {

constexpr uint64_t EMPTY_KEY = 0xFFFFFFFFFFFFFFFFULL;  // never a canonical k-mer word

// ---------------------------------------------------------------------------
// k-mer words
// ---------------------------------------------------------------------------

// Reverses the order of the 32 two-bit groups of a word.  It maps the
// reference's internal kmer<1> word (base i of the printed string at bit
// 64-2k+2i) to the printed-string order key (base i at bit 2(k-1-i)) and back.
__device__ __forceinline__ uint64_t pair_reverse(uint64_t x)
{
    uint64_t r = ((uint64_t)__brev((uint32_t)x) << 32) | (uint64_t)__brev((uint32_t)(x >> 32));
    return ((r >> 1) & 0x5555555555555555ULL) | ((r & 0x5555555555555555ULL) << 1);
}

// 64-bit mixer for table slots and HyperLogLog registers (the MurmurHash3
// 64-bit finaliser).  Placement only; it never affects a count.
__device__ __forceinline__ uint64_t slot_hash(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// ---------------------------------------------------------------------------
// FASTQ bytes
// ---------------------------------------------------------------------------

// Bit i of the result is bit 0 of byte i of x (x's bytes hold 0 or 1).
__device__ __forceinline__ uint32_t byte_bits4(uint32_t x)
{
    return (x * 0x01020408u) >> 24 & 0xFu;
}

// 2-bit codes (A0 C1 G2 T/U3, case-insensitive, as the reference's
// char_to_2bit table and its AVX2 classifier), valid-base mask and newline
// mask of 32 bytes at p (16-byte aligned shared memory), four bytes per
// 32-bit word at a time.  With u = byte & 0xDF (upper case), the valid
// letters A C G T U are 0x41 0x43 0x47 0x54 0x55: bit 7 clear, bit 6 set,
// bit 3 clear, and either bit 4 clear, bit 0 set and not (bit 2 set with
// bit 1 clear) -- 00001 00011 00111 -- or bit 4 set, bit 2 set, bit 1 clear
// -- 10100 10101.  The code is ((u >> 1) & 3) ^ ((u >> 2) & 1).
__device__ __forceinline__ void classify32(const uint8_t *p, uint64_t &codes, uint32_t &valid, uint32_t &nl)
{
    const uint4 a = *reinterpret_cast<const uint4 *>(p);
    const uint4 b = *reinterpret_cast<const uint4 *>(p + 16);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint64_t c = 0;
    uint32_t v = 0, n = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t x = w[i];
        // newline bytes: zero bytes of x ^ 0x0a0a0a0a (exact, no borrow)
        const uint32_t z = x ^ 0x0a0a0a0au;
        const uint32_t nz = (((z & 0x7f7f7f7fu) + 0x7f7f7f7fu) | z) & 0x80808080u;   // 0x80 where byte != 0
        n |= byte_bits4((~nz & 0x80808080u) >> 7) << (4 * i);
        const uint32_t u = x & 0xdfdfdfdfu;
        const uint32_t x0 = u, x1 = u >> 1, x2 = u >> 2, x3 = u >> 3, x4 = u >> 4, x6 = u >> 6, x7 = u >> 7;
        const uint32_t ok = x6 & ~x7 & ~x3 & ((~x4 & x0 & ~(x2 & ~x1)) | (x4 & x2 & ~x1)) & 0x01010101u;
        v |= byte_bits4(ok) << (4 * i);
        // four 2-bit codes, one per byte, packed into 8 bits
        const uint32_t c4 = ((u >> 1) & 0x03030303u) ^ ((u >> 2) & 0x01010101u);
        const uint32_t c2 = c4 | (c4 >> 6);                       // bytes 0 and 2 hold two codes each
        const uint32_t c8 = (c2 & 0xfu) | ((c2 >> 12) & 0xf0u);
        c |= (uint64_t)c8 << (8 * i);
    }
    codes = c;
    valid = v;
    nl = n;
}

__device__ __forceinline__ uint32_t range_mask(uint32_t a, uint32_t b)
{
    uint32_t hi = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    uint32_t lo = a >= 32 ? 0xffffffffu : ((1u << a) - 1u);
    return hi & ~lo;
}

// Bytes of the 32-byte segment that lie in lines whose number is
// `want` mod 4, given the line number at the segment start.
__device__ __forceinline__ uint32_t line_mask(uint64_t line0, uint32_t nl, uint32_t want)
{
    uint32_t m = 0, pos = 0, bits = nl;
    uint64_t cur = line0;
    while (bits) {
        uint32_t j = __ffs(bits) - 1;
        if ((cur & 3) == want) m |= range_mask(pos, j);
        ++cur;
        pos = j + 1;
        bits &= bits - 1;
    }
    if ((cur & 3) == want) m |= range_mask(pos, 32);
    return m;
}

// ---------------------------------------------------------------------------
// Reference hashes on the 8-byte kmer<1> word (little-endian bytes of w)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

__device__ __forceinline__ void mul128(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi)
{
    lo = a * b;
    hi = __umul64hi(a, b);
}

// xxHash 0.8.3 XXH3_128bits, 4..8-byte path, seed 0.  The two constants are
// XXH_PRIME64_1 and PRIME_MX2/PRIME_MX1 of the published algorithm; the
// secret words are bytes 16..32 of its default secret.
__device__ __forceinline__ void xxh3_128_8(uint64_t w, uint64_t &lo, uint64_t &hi)
{
    const uint64_t P1 = 0x9E3779B185EBCA87ULL, MX1 = 0x165667919E3779F9ULL, MX2 = 0x9FB21C651E98DF25ULL;
    const uint64_t S16 = 0xdb979083e96dd4deULL, S24 = 0x1f67b3b7a4a44072ULL;
    uint64_t keyed = w ^ (S16 ^ S24);
    uint64_t l, h;
    mul128(keyed, P1 + (8ULL << 2), l, h);
    h += l << 1;
    l ^= h >> 3;
    l ^= l >> 35;
    l *= MX2;
    l ^= l >> 28;
    h ^= h >> 37;
    h *= MX1;
    h ^= h >> 32;
    lo = l;
    hi = h;
}

// xxHash 0.8.3 XXH3_64bits, 4..8-byte path, seed 0 (secret bytes 8..24).
__device__ __forceinline__ uint64_t xxh3_64_8(uint64_t w)
{
    const uint64_t MX2 = 0x9FB21C651E98DF25ULL;
    const uint64_t S8 = 0x1cad21f72c81017cULL, S16 = 0xdb979083e96dd4deULL;
    uint64_t in64 = (w >> 32) + ((w & 0xffffffffULL) << 32);
    uint64_t h = in64 ^ (S8 ^ S16);
    h ^= rotl64(h, 49) ^ rotl64(h, 24);
    h *= MX2;
    h ^= (h >> 35) + 8;
    h *= MX2;
    return h ^ (h >> 28);
}

// rapidhash V3, default secret, seed 0, 8-byte input.
__device__ __forceinline__ uint64_t rapidhash_8(uint64_t w)
{
    const uint64_t s1 = 0x8bb84b93962eacc9ULL, s2 = 0x4b33a62ed433d4a3ULL, s7 = 0xaaaaaaaaaaaaaaaaULL;
    uint64_t l, h;
    mul128(s2, s1, l, h);
    uint64_t seed = (l ^ h) ^ 8ULL;
    mul128(w ^ s1, w ^ seed, l, h);
    uint64_t l2, h2;
    mul128(l ^ s7, h ^ s1 ^ 8ULL, l2, h2);
    return l2 ^ h2;
}

// komihash 5.29, seed 0, 8-byte input.  Its multiply step keeps the low half
// and adds the high half into the second state word.
__device__ __forceinline__ uint64_t komihash_8(uint64_t w)
{
    uint64_t s1 = 0x243F6A8885A308D3ULL, s5 = 0x452821E638D01377ULL, l, h;
    mul128(s1, s5, l, h);
    s1 = l;
    s5 += h;
    s1 ^= s5;
    uint64_t r1h = s1 ^ w, r2h = s5 ^ 1ULL;
    mul128(r1h, r2h, l, h);
    s1 = l;
    s5 += h;
    s1 ^= s5;
    mul128(s1, s5, l, h);
    s1 = l;
    s5 += h;
    return s1 ^ s5;
}

// mix_hash of the reference (src/HashFunction.h:28-37).
__device__ __forceinline__ uint64_t mix_hash(uint64_t h1, uint64_t h2)
{
    const uint64_t K = 0x9ddfea08eb382d69ULL;
    uint64_t a = (h1 ^ h2) * K;
    a ^= a >> 47;
    uint64_t b = (h2 ^ a) * K;
    b ^= b >> 47;
    return b * K;
}

// Bloom probe of the reference (src/BloomFilter.h:215-222, :287-296):
// block = xxh3.lo & (cap - 1); three bits (lo + i*(hi|1)) & 63.
__device__ __forceinline__ void bloom_probe(uint64_t w, uint64_t cap, uint64_t &block, uint64_t &mask)
{
    uint64_t lo, hi;
    xxh3_128_8(w, lo, hi);
    uint64_t h2 = hi | 1ULL;
    mask = (1ULL << (lo & 63)) | (1ULL << ((lo + h2) & 63)) | (1ULL << ((lo + 2 * h2) & 63));
    block = lo & (cap - 1);
}

// The same probe, also returning the high 64 bits of the hash (used as the
// hash of the k-mer for sampled distinct counting).
__device__ __forceinline__ void bloom_probe_hi(uint64_t w, uint64_t cap, uint64_t &block, uint64_t &mask,
                                               uint64_t &hi_out)
{
    uint64_t lo, hi;
    xxh3_128_8(w, lo, hi);
    uint64_t h2 = hi | 1ULL;
    mask = (1ULL << (lo & 63)) | (1ULL << ((lo + h2) & 63)) | (1ULL << ((lo + 2 * h2) & 63));
    block = lo & (cap - 1);
    hi_out = hi;
}

// ---------------------------------------------------------------------------
// bounded waits
// ---------------------------------------------------------------------------

constexpr uint32_t SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}

// One-dimensional bulk copy global -> shared completing on an mbarrier.
// Source, destination and size must be 16-byte aligned.
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar)
{
    uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
        "l"(gmem_src), "r"(bytes), "r"(b)
        : "memory");
}

// Waits for the mbarrier phase with the given parity; gives up after
// SPIN_LIMIT polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace kc
