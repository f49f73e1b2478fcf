// skm_load.cu -- superkmer stores from the reference's .skm bytes.
//
// A .skm file (skmstore.hpp:129-141, one per partition) is the partition's
// superkmers in skm_3x bytes, concatenated with no index.  A superkmer is a
// first byte (1-3 valid bases in its low slots), full bytes, and a terminal
// byte (0-2 valid bases in its high slots; cpu_funcs.cpp:219-250).  Parsing it
// is a two-state automaton -- state 0: the next byte starts a superkmer;
// state 1: inside one, where a non-full byte ends it -- so the bounds of
// every superkmer follow from composable per-span transforms, as in the
// FASTQ scanner: tiles are scanned in parallel (skm_tile_kernel), composed by
// one CTA (skm_carry_kernel), and rescanned to write each superkmer's start
// (skm_starts_kernel).  skm_index_kernel then gives each superkmer its index
// entry (offset in its partition, k-mer count) and its minimizer key,
// recomputed under the context's order from its first k-mer, and checks that
// the key maps to the partition the bytes came in.
#include "gkc_device.cuh"

namespace gkc {

constexpr int SL_THREADS = 256, SL_PER = 64, SL_TILE = SL_THREADS * SL_PER;
constexpr int SL_CARRY_THREADS = 256;

enum : uint32_t {
    SKM_ERR_TRUNCATED = 1u,   // a partition ends inside a superkmer
    SKM_ERR_SHORT = 2u,       // a superkmer holds fewer than k bases
    SKM_ERR_PARTITION = 4u,   // a superkmer's minimizer maps to another partition
};

struct SlT {            // effect of a span, per state at its start (0 or 1)
    uint8_t next[2];
    uint64_t starts[2];  // superkmers starting in the span
};

__device__ __forceinline__ SlT sl_identity() {
    SlT t;
    t.next[0] = 0;
    t.next[1] = 1;
    t.starts[0] = t.starts[1] = 0;
    return t;
}

__device__ __forceinline__ SlT sl_compose(const SlT &a, const SlT &b) {
    SlT t;
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int m = a.next[s];
        t.next[s] = b.next[m];
        t.starts[s] = a.starts[s] + b.starts[m];
    }
    return t;
}

template <int NT>
__device__ __forceinline__ SlT sl_block_scan(SlT v, SlT *sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int d = 1; d < NT; d <<= 1) {
        SlT o = t >= d ? sh[t - d] : sl_identity();
        __syncthreads();
        if (t >= d) v = sl_compose(o, v);
        sh[t] = v;
        __syncthreads();
    }
    return v;
}

struct SlParams {
    const uint8_t *bytes;
    uint64_t n;
    const unsigned long long *part_off;  // [P+1] partition starts in bytes
    uint32_t P;
    SlT *tiles;
    uint64_t ntiles;
    uint8_t *tile_state;
    uint64_t *tile_starts;
    uint64_t *result;       // [0] superkmers
    uint64_t *starts;       // [superkmers] byte position of each superkmer
    uint32_t *err;
};

// first index j of off[0..P] with off[j] > pos (ge: off[j] >= pos); P + 1 when none
template <bool GE = false>
__device__ __forceinline__ uint32_t sl_next_part(const unsigned long long *off, uint32_t P, uint64_t pos) {
    uint32_t lo = 0, hi = P + 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (GE ? off[mid] >= pos : off[mid] > pos) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// Walks bytes [pos, pos + len) from state s; a partition start resets the
// state to 0 (a truncated superkmer there sets *trunc).  Calls at(i) for the
// position of each superkmer start when `Emit`.
template <bool Emit, class F>
__device__ __forceinline__ int sl_walk(const SlParams &a, uint64_t pos, int len, int s, uint64_t *starts,
                                       bool *trunc, F at) {
    uint32_t np = sl_next_part<true>(a.part_off, a.P, pos);
    uint64_t nb = np <= a.P ? a.part_off[np] : ~0ull;  // next partition start at or after pos
    for (int i = 0; i < len; i++) {
        const uint64_t q = pos + i;
        if (q == nb) {  // (empty partitions repeat a start)
            if (s == 1) *trunc = true;
            s = 0;
            while (np <= a.P && a.part_off[np] <= q) np++;
            nb = np <= a.P ? a.part_off[np] : ~0ull;
        }
        const uint8_t c = a.bytes[q];
        if (s == 0) {
            ++*starts;
            if (Emit) at(q);
            s = 1;
        } else if ((c >> 6) != 3u) {
            s = 0;
        }
    }
    return s;
}

__device__ __forceinline__ SlT sl_thread_transform(const SlParams &a, uint64_t pos, int len) {
    SlT t;
    bool tr = false;
#pragma unroll
    for (int s = 0; s < 2; s++) {
        uint64_t st = 0;
        t.next[s] = (uint8_t)sl_walk<false>(a, pos, len, s, &st, &tr, [](uint64_t) {});
        t.starts[s] = st;
    }
    return t;
}

__global__ void __launch_bounds__(SL_THREADS) skm_tile_kernel(SlParams a) {
    __shared__ SlT sh[SL_THREADS];
    const uint64_t pos = blockIdx.x * (uint64_t)SL_TILE + (uint64_t)threadIdx.x * SL_PER;
    const int len = pos < a.n ? (int)(a.n - pos < (uint64_t)SL_PER ? a.n - pos : SL_PER) : 0;
    const SlT v = sl_block_scan<SL_THREADS>(sl_thread_transform(a, pos, len), sh);
    if (threadIdx.x == SL_THREADS - 1) a.tiles[blockIdx.x] = v;
}

__global__ void __launch_bounds__(SL_CARRY_THREADS) skm_carry_kernel(SlParams a) {
    __shared__ SlT sh[SL_CARRY_THREADS];
    const uint64_t per = (a.ntiles + SL_CARRY_THREADS - 1) / SL_CARRY_THREADS;
    const uint64_t t0 = threadIdx.x * per, t1 = t0 + per < a.ntiles ? t0 + per : a.ntiles;
    SlT v = sl_identity();
    for (uint64_t t = t0; t < t1; t++) v = sl_compose(v, a.tiles[t]);
    const SlT inc = sl_block_scan<SL_CARRY_THREADS>(v, sh);
    const SlT ex = threadIdx.x ? sh[threadIdx.x - 1] : sl_identity();
    int s = ex.next[0];
    uint64_t starts = ex.starts[0];
    for (uint64_t t = t0; t < t1; t++) {
        a.tile_state[t] = (uint8_t)s;
        a.tile_starts[t] = starts;
        starts += a.tiles[t].starts[s];
        s = a.tiles[t].next[s];
    }
    if (threadIdx.x == SL_CARRY_THREADS - 1) {
        a.result[0] = inc.starts[0];
        if (inc.next[0] != 0) atomicOr(a.err, SKM_ERR_TRUNCATED);  // the last superkmer has no end
    }
}

__global__ void __launch_bounds__(SL_THREADS) skm_starts_kernel(SlParams a) {
    __shared__ SlT sh[SL_THREADS];
    const uint64_t pos = blockIdx.x * (uint64_t)SL_TILE + (uint64_t)threadIdx.x * SL_PER;
    const int len = pos < a.n ? (int)(a.n - pos < (uint64_t)SL_PER ? a.n - pos : SL_PER) : 0;
    sl_block_scan<SL_THREADS>(sl_thread_transform(a, pos, len), sh);
    const SlT ex = threadIdx.x ? sh[threadIdx.x - 1] : sl_identity();
    const int ts = a.tile_state[blockIdx.x];
    uint64_t idx = a.tile_starts[blockIdx.x] + ex.starts[ts];
    bool trunc = false;
    uint64_t cnt = 0;
    sl_walk<true>(a, pos, len, ex.next[ts], &cnt, &trunc, [&](uint64_t q) { a.starts[idx++] = q; });
    if (trunc) atomicOr(a.err, SKM_ERR_TRUNCATED);
}

struct SiParams {
    const uint8_t *bytes;
    uint64_t n;
    const unsigned long long *part_off;  // [P+1] starts of partitions part0 .. part0 + P in bytes
    uint32_t P;
    uint32_t part0;             // the store partition of part_off[0]
    uint32_t P_store;           // the store's partitions (the key -> partition map)
    uint64_t pmod;              // fastmod multiplier of P_store
    int k, p;
    const uint32_t *lut;        // canonical order table, or null for the default order
    const uint64_t *starts;
    uint64_t nskm;
    uint64_t *idx;              // out: offset in the partition | k-mers << 40
    uint32_t *keys;             // out: minimizer key
    uint32_t *part_kmers32;     // out: k-mers of each superkmer (for the per-partition sums)
    uint32_t *err;
};

// One thread per superkmer.
template <bool LUT>
__global__ void __launch_bounds__(256) skm_index_kernel(SiParams a) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.nskm;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = a.starts[i];
        const uint32_t part = sl_next_part(a.part_off, a.P, s) - 1;  // off[part] <= s < off[part+1]
        uint64_t e = i + 1 < a.nskm ? a.starts[i + 1] : a.n;
        if (e > a.part_off[part + 1]) e = a.part_off[part + 1];
        const uint64_t nb = e - s;
        uint32_t bases = nb >= 1 ? (a.bytes[s] >> 6) : 0u;
        if (nb >= 2) bases += 3u * (uint32_t)(nb - 2) + (a.bytes[e - 1] >> 6);
        uint32_t kmers = bases >= (uint32_t)a.k ? bases - a.k + 1 : 0u;
        if (!kmers || kmers > IDX_MAX_LEN) {
            atomicOr(a.err, SKM_ERR_SHORT);
            kmers = 0;
        }
        // the first k bases: the first byte's low slots, then 3 per byte
        const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * a.p);
        uint32_t f = 0, best = 0xFFFFFFFFu;
        int have = 0;
        for (uint64_t q = s; q < e && have < a.k; q++) {
            const uint8_t c = a.bytes[q];
            const int h = c >> 6;
            const int t0 = q == s ? 3 - h : 0, t1 = q == s ? 3 : h;
            for (int t = t0; t < t1 && have < a.k; t++) {
                f = ((f << 2) | ((c >> (4 - 2 * t)) & 3u)) & pmask;
                if (++have >= a.p) {
                    uint32_t m;
                    if (LUT) {
                        m = __ldg(a.lut + f);
                    } else {
                        const uint32_t r = rc32(f, a.p);
                        const uint32_t kf = pmer_key(f, a.p, pmask), kr = pmer_key(r, a.p, pmask);
                        m = kf < kr ? kf : kr;
                    }
                    best = m < best ? m : best;
                }
            }
        }
        if (kmers && fastmod(~best, a.pmod, a.P_store) != a.part0 + part) atomicOr(a.err, SKM_ERR_PARTITION);
        a.idx[i] = idx_pack(s - a.part_off[part], kmers);
        a.keys[i] = best;
        a.part_kmers32[i] = kmers;
    }
}

// Per partition: superkmers (first start at or after its first byte) and
// k-mers (a sum over its superkmers).  One CTA per partition.
__global__ void __launch_bounds__(256) skm_part_totals_kernel(const unsigned long long *part_off, uint32_t P,
                                                              const uint64_t *starts, uint64_t nskm,
                                                              const uint32_t *kmers32,
                                                              unsigned long long *skm_off,
                                                              unsigned long long *part_kmers) {
    __shared__ unsigned long long ws[8];
    __shared__ uint64_t range[2];
    const uint32_t p = blockIdx.x;
    if (threadIdx.x < 2) {  // first superkmer starting at or after part_off[p + t]
        const uint64_t x = part_off[p + threadIdx.x];
        uint64_t lo = 0, hi = nskm;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (starts[mid] < x) lo = mid + 1; else hi = mid;
        }
        range[threadIdx.x] = lo;
    }
    __syncthreads();
    unsigned long long sum = 0, tot;
    for (uint64_t i = range[0] + threadIdx.x; i < range[1]; i += 256) sum += kmers32[i];
    block_exclusive_scan<256>(sum, &tot, ws);
    if (threadIdx.x == 0) {
        skm_off[p] = range[0];
        if (p + 1 == P) skm_off[P] = range[1];
        part_kmers[p] = tot;
    }
}

}  // namespace gkc
