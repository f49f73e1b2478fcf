// gkc_device.cuh -- device helpers shared by the k-mer counter's kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gkc {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr uint64_t EMPTY_KEY = ~0ull;  // never a canonical k-mer: for k=32 the
                                       // canonical form of TT..T is AA..A = 0

// Four ASCII bases in one 32-bit word -> four 2-bit codes, one per byte
// (A/a=0 C/c=1 G/g=2 T/t=3; N, U and every other byte read as 0).  The same
// mapping as the reference's basemap (cpu_funcs.cpp:20-54, gpu_skmgen.cu:25-58)
// for A/C/G/T/N/U; the xor of the bytes shifted by one and two bits gives
// the code of every letter of ACGTN in either case.
__device__ __forceinline__ uint32_t codes4(uint32_t w) {
    uint32_t c = ((w >> 1) ^ (w >> 2)) & 0x03030303u;
    uint32_t l = w | 0x20202020u;  // lower case
    uint32_t ok = __vcmpeq4(l, 0x61616161u) | __vcmpeq4(l, 0x63636363u) |
                  __vcmpeq4(l, 0x67676767u) | __vcmpeq4(l, 0x74747474u);
    return c & ok;
}

__device__ __forceinline__ uint32_t code1(uint8_t b) { return codes4(b) & 3u; }

// Default minimizer filter (minimizer_filter.h:20): invalid when the first
// three bases are AAA/ACA/CAA/CCA or the last three are AAA.
__device__ __forceinline__ bool mm_valid(uint32_t v, int p) {
    return (((v >> ((p - 3) * 2)) & 0x2Bu) != 0) & ((v & 0x3Fu) != 0);
}

// Reverse complement of a p-mer held in the low 2p bits (p <= 16).
__device__ __forceinline__ uint32_t rc32(uint32_t v, int p) {
    uint32_t r = __brev(~v);
    r = ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
    return r >> (32 - 2 * p);
}

// Reverse complement of a k-mer held in the low 2k bits (k <= 32).
__device__ __forceinline__ uint64_t rc64(uint64_t v, int k) {
    uint64_t r = __brevll(~v);
    r = ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);
    return r >> (64 - 2 * k);
}

__device__ __forceinline__ uint64_t kmask(int k) {
    return k >= 32 ? ~0ull : ((1ull << (2 * k)) - 1);
}

// 64-bit finaliser (splitmix64) for hash-table slots.
__device__ __forceinline__ uint64_t hash64(uint64_t z) {
    z ^= z >> 31;
    z *= 0x7FB5D329728EA185ull;
    z ^= z >> 27;
    z *= 0x81DADEF4BC2DD44Dull;
    z ^= z >> 33;
    return z;
}

// Superkmer record written by phase 1 (one per superkmer):
//   pos   global position of the superkmer's first base in the read batch
//   len   number of k-mers (>= 1)
//   key   minimizer key (partition = (~key) % P, gpu_skmgen.cu:276-278)
// pos also carries, in bits 56-57, (first base - read start) % 3, the packing
// phase, and in bits 58-59 the number of read bases after the superkmer's
// last base, capped at 3 (both needed to rebuild the reference's bytes).
struct SkmRecord {
    uint64_t pos;
    uint32_t len;
    uint32_t key;
};
static_assert(sizeof(SkmRecord) == 16, "record layout");
constexpr int REC_POS_BITS = 48;
__device__ __host__ __forceinline__ uint64_t rec_pack_pos(uint64_t pos, uint32_t phase, uint32_t tail) {
    return pos | ((uint64_t)phase << 56) | ((uint64_t)tail << 58);
}
__device__ __host__ __forceinline__ uint64_t rec_base(uint64_t w) { return w & ((1ull << REC_POS_BITS) - 1); }
__device__ __host__ __forceinline__ uint32_t rec_phase(uint64_t w) { return (uint32_t)(w >> 56) & 3u; }
__device__ __host__ __forceinline__ uint32_t rec_tail(uint64_t w) { return (uint32_t)(w >> 58) & 3u; }

// Bytes of a superkmer in the reference's 3-bases-per-byte format
// (cpu_funcs.cpp:216-218): ((beg%3) + L + k - 1 + 3) / 3.
__device__ __host__ __forceinline__ uint32_t skm_nbytes(uint32_t phase, uint32_t len, int k) {
    return (phase + len + (uint32_t)k - 1 + 3) / 3;
}

// Superkmer index entry (phase 2 input): byte offset of the superkmer inside
// its partition (low 40 bits) and its k-mer count (high 24 bits).
constexpr int IDX_OFF_BITS = 40;
constexpr uint32_t IDX_MAX_LEN = (1u << 24) - 1;
__device__ __host__ __forceinline__ uint64_t idx_pack(uint64_t off, uint32_t len) {
    return off | ((uint64_t)len << IDX_OFF_BITS);
}
__device__ __host__ __forceinline__ uint64_t idx_off(uint64_t e) { return e & ((1ull << IDX_OFF_BITS) - 1); }
__device__ __host__ __forceinline__ uint32_t idx_len(uint64_t e) { return (uint32_t)(e >> IDX_OFF_BITS); }

// Error flags raised by kernels (OR-ed into a device word, read by the host).
enum : uint32_t {
    ERR_RECORD_OVERFLOW = 1u << 0,  // phase-1 record region full (host retries larger)
    ERR_SKM_TOO_LONG = 1u << 1,     // superkmer longer than IDX_MAX_LEN k-mers
    ERR_TABLE_FULL = 1u << 2,       // hash table probe limit (host retries larger)
    ERR_OUTPUT_FULL = 1u << 3,      // output capacity exceeded
    ERR_DECODE = 1u << 4,           // malformed superkmer stream
    ERR_CAPACITY = 1u << 5,         // phase-1 store chunk capacity exceeded (host redoes the batch)
};

}  // namespace gkc

namespace gkc {

// Calls f(canonical k-mer) for every k-mer of the superkmer described by
// index entry e, in order (the decode of cpu_funcs.cpp:437-515 and
// gpu_kmercounting.cu:90-165).  `bytes` is the start of its partition.  The
// first byte's header gives the number of valid bases it holds in its low
// bits; the k+L-1 bases follow three per byte; the terminal byte is never
// read past.
template <bool CANONICAL, class F>
__device__ __forceinline__ void for_each_kmer(const uint8_t *bytes, uint64_t e, int k, F &&f) {
    const uint8_t *s = bytes + idx_off(e);
    const uint32_t L = idx_len(e);
    const uint64_t mask = kmask(k);
    const int sh = 2 * k - 2;
    uint32_t cur = s[0];
    uint32_t slot = 3 - (cur >> 6);
    uint32_t bi = 0;
    uint64_t fwd = 0, rc = 0;
    const uint32_t nbases = (uint32_t)k + L - 1;
    for (uint32_t j = 0; j < nbases; j++) {
        uint32_t c = (cur >> (4 - 2 * slot)) & 3u;
        fwd = ((fwd << 2) | c) & mask;
        rc = (rc >> 2) | ((uint64_t)(3u - c) << sh);
        if (j + 1 >= (uint32_t)k) {
            if (CANONICAL) f(fwd < rc ? fwd : rc);
            else f(fwd);
        }
        if (++slot == 3) { slot = 0; cur = s[++bi]; }
    }
}

// k-mers of 33 to 64 bases: the reference's LONGERKMER build keeps them in an
// unsigned __int128 (types.h:34-35); stored as two u64 words, low word first.
using u128 = unsigned __int128;

// for_each_kmer<true> for k <= 64: calls f(canonical u128 k-mer).
template <class F>
__device__ __forceinline__ void for_each_kmer_wide(const uint8_t *bytes, uint64_t e, int k, F &&f) {
    const uint8_t *s = bytes + idx_off(e);
    const uint32_t L = idx_len(e);
    const u128 mask = k >= 64 ? ~(u128)0 : (((u128)1 << (2 * k)) - 1);
    const int sh = 2 * k - 2;
    uint32_t cur = s[0];
    uint32_t slot = 3 - (cur >> 6);
    uint32_t bi = 0;
    u128 fwd = 0, rc = 0;
    const uint32_t nbases = (uint32_t)k + L - 1;
    for (uint32_t j = 0; j < nbases; j++) {
        const uint32_t c = (cur >> (4 - 2 * slot)) & 3u;
        fwd = ((fwd << 2) | c) & mask;
        rc = (rc >> 2) | ((u128)(3u - c) << sh);
        if (j + 1 >= (uint32_t)k) f(fwd < rc ? fwd : rc);
        if (++slot == 3) { slot = 0; cur = s[++bi]; }
    }
}

// Exclusive scan of one value per thread over a block of NT threads.
// Returns the prefix; *total receives the block total.  `ws` holds NT/32
// words of shared memory.  Must be called by every thread of the block.
template <int NT, class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *total, T *ws) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T s = lane < NT / 32 ? ws[lane] : T(0);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T y = __shfl_up_sync(FULL, s, d);
            if (lane >= d) s += y;
        }
        if (lane < NT / 32) ws[lane] = s;  // inclusive warp totals
    }
    __syncthreads();
    T warp_prefix = warp ? ws[warp - 1] : T(0);
    *total = ws[NT / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// ---------------------------------------------------------------------------
// Tie-break of the learned order: a fixed bijection of `bits` bits (odd
// multipliers are bijections modulo 2^bits, and so are xor-shifts).
constexpr uint32_t ORDER_MIX_KEY = 0x5BD1E995u;

__host__ __device__ __forceinline__ uint32_t mix_bits(uint32_t x, int bits, uint32_t key) {
    const uint32_t mask = bits >= 32 ? 0xFFFFFFFFu : (1u << bits) - 1;
    const int h = bits > 1 ? bits / 2 : 1;
    x = (x ^ key) & mask;
    x = (x * 0x9E3779B1u) & mask;
    x ^= x >> h;
    x = (x * 0x85EBCA77u) & mask;
    x ^= x >> h;
    return x;
}

}  // namespace gkc
