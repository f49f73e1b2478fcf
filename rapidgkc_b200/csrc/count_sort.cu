// count_sort.cu -- phase 2, sort counter: superkmers -> sorted (k-mer, count).
//
// Replaces the reference's Extract_Kmers + thrust::transform(canonicalkmer)
// + thrust::sort + sameasprev/sequence/remove_if chain and its host-side
// count differences (gpu_kmercounting.cu:257-523):
//   extract  one lane per superkmer decodes its canonical k-mers into a
//            per-warp shared-memory stage; the warp copies them to its
//            partitions' segments of the key buffer in coalesced runs;
//   sort     a hand-written stable LSD radix sort over only the 2k meaningful
//            bits, all partitions at once as independent segments
//            (count_onesweep.cu; the three-kernel form below, a tile
//            histogram, a device-wide scan of the segment-major
//            [segment][digit][tile] counts and a scatter per digit, is kept
//            for partitions of 2^30 keys or more);
//   rle      heads of equal-key runs -> distinct keys and run lengths
//            (counts saturate at 2^32-1, types.h:101-102) -> threshold
//            [cmin, cmax] (utilities.hpp:190) -> compaction that keeps the
//            ascending order inside every partition.
// Keys are u64 for k <= 32 and u128 for k <= 64 (the reference's LONGERKMER
// build, types.h:34-35): every kernel is a template over the key type.
#include "gkc_device.cuh"

namespace gkc {

// ---------------------------------------------------------------------------
// extract
struct SExtractParams {
    const uint8_t *bytes;                // store chunk bytes
    const uint64_t *idx;                 // store chunk superkmer index
    uint64_t i_begin, n_skm;             // index range [i_begin, n_skm) to extract
    const unsigned long long *part_skm_off;   // [P+1] partition ranges in idx
    const unsigned long long *part_byte_off;  // [P] partition starts in bytes
    uint32_t P;
    int k;
    int canonical;
    void *keys;                          // key buffer (u64, or u128 for k > 32)
    const unsigned long long *seg_off;   // [P] partition segment starts in keys
    unsigned long long *seg_cursor;      // [P] keys written per partition
};

constexpr int SX_THREADS = 256;
constexpr int SX_WARPS = SX_THREADS / 32;
template <class KT> constexpr int sx_stage() { return 4096 / (int)sizeof(KT); }  // 4 KB per warp

// A warp takes 32 superkmers at a time.  Each lane reserves its k-mers'
// range in its partition's segment (one atomic per partition group of the
// warp), decodes them in order into the warp's shared-memory stage, and the
// warp then copies the stage out with consecutive lanes on consecutive keys
// (within a partition group the ranges are contiguous).  A superkmer that
// does not fit the stage's remainder is written straight to global memory.
template <class KT>
__global__ void __launch_bounds__(SX_THREADS)
sort_extract_kernel(SExtractParams a) {
    constexpr int ST = sx_stage<KT>();
    __shared__ KT stage[SX_WARPS][ST];
    KT *keys = static_cast<KT *>(a.keys);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    KT *sw = stage[warp];
    for (uint64_t base = a.i_begin + blockIdx.x * (uint64_t)SX_THREADS + warp * 32; base < a.n_skm;
         base += (uint64_t)gridDim.x * SX_THREADS) {
        const uint64_t i = base + lane;
        const bool has = i < a.n_skm;
        uint32_t part = 0xFFFFFFFFu, L = 0;
        uint64_t e = 0;
        if (has) {
            e = a.idx[i];
            L = idx_len(e);
            uint32_t lo = 0, hi = a.P;  // part_skm_off[lo] <= i < part_skm_off[hi]
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (a.part_skm_off[mid] <= i) lo = mid; else hi = mid;
            }
            part = lo;
        }
        // k-mer prefix over the warp (lanes of one partition are contiguous)
        uint32_t incl = L;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t excl = incl - L;
        const unsigned grp = __match_any_sync(FULL, part);
        const int first = __ffs(grp) - 1, last = 31 - __clz(grp);
        const uint32_t excl_first = __shfl_sync(FULL, excl, first);
        const uint32_t incl_last = __shfl_sync(FULL, incl, last);
        unsigned long long b = 0;
        if (has && lane == first) b = atomicAdd(a.seg_cursor + part, (unsigned long long)(incl_last - excl_first));
        b = __shfl_sync(FULL, b, first);
        // global position of stage element x of this lane's group: x + delta
        const uint64_t delta = has ? a.seg_off[part] + b - excl_first : 0;
        const uint64_t dst = delta + excl;
        const bool staged = has && incl <= (uint32_t)ST;
        if (has) {
            const uint8_t *pb = a.bytes + a.part_byte_off[part];
            if (staged) {
                uint32_t o = excl;
                if constexpr (sizeof(KT) == 16)
                    for_each_kmer_wide(pb, e, a.k, [&](u128 key) { sw[o++] = key; });
                else if (a.canonical)
                    for_each_kmer<true>(pb, e, a.k, [&](uint64_t key) { sw[o++] = key; });
                else
                    for_each_kmer<false>(pb, e, a.k, [&](uint64_t key) { sw[o++] = key; });
            } else {
                uint64_t o = dst;
                if constexpr (sizeof(KT) == 16)
                    for_each_kmer_wide(pb, e, a.k, [&](u128 key) { keys[o++] = key; });
                else if (a.canonical)
                    for_each_kmer<true>(pb, e, a.k, [&](uint64_t key) { keys[o++] = key; });
                else
                    for_each_kmer<false>(pb, e, a.k, [&](uint64_t key) { keys[o++] = key; });
            }
        }
        __syncwarp();
        // the staged prefix of the warp's k-mers, out in order
        const unsigned sb = __ballot_sync(FULL, staged);  // a prefix of the lanes
        const uint32_t n_st = sb ? __shfl_sync(FULL, incl, 31 - __clz(sb)) : 0u;
        const unsigned gb = __ballot_sync(FULL, has && lane == first);  // group leaders
        if (__popc(gb) <= 1) {  // one partition: one contiguous range
            const uint64_t d0 = __shfl_sync(FULL, delta, 0);
            for (uint32_t x = lane; x < n_st; x += 32) keys[d0 + x] = sw[x];
        } else {
            // every lane takes every step (the owner search shuffles), the
            // store is predicated
            for (uint32_t x0 = 0; x0 < n_st; x0 += 32) {
                const uint32_t x = x0 + lane;
                int own = 0;  // the last lane whose range starts at or before x
#pragma unroll
                for (int st = 16; st; st >>= 1) {
                    const int cand = own + st;
                    if (__shfl_sync(FULL, excl, cand) <= x) own = cand;
                }
                const uint64_t dl = __shfl_sync(FULL, delta, own);
                if (x < n_st) keys[dl + x] = sw[x];
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// device-wide exclusive scan, u32 counts -> u64 offsets
constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 16;
constexpr int SC_PER_BLOCK = SC_THREADS * SC_ITEMS;

__global__ void __launch_bounds__(SC_THREADS)
scan_reduce_kernel(const uint32_t *in, uint64_t n, unsigned long long *block_sums) {
    __shared__ unsigned long long ws[SC_THREADS / 32];
    uint64_t b0 = blockIdx.x * (uint64_t)SC_PER_BLOCK;
    unsigned long long s = 0;
#pragma unroll
    for (int t = 0; t < SC_ITEMS; t++) {
        uint64_t i = b0 + (uint64_t)t * SC_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    unsigned long long tot;
    block_exclusive_scan<SC_THREADS>(s, &tot, ws);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of the block sums in place; *total = sum.
__global__ void __launch_bounds__(1024)
scan_blocksums_kernel(unsigned long long *sums, uint64_t nb, unsigned long long *total) {
    __shared__ unsigned long long ws[32];
    unsigned long long carry = 0;
    for (uint64_t b0 = 0; b0 < nb; b0 += 1024) {
        uint64_t i = b0 + threadIdx.x;
        unsigned long long v = i < nb ? sums[i] : 0ull;
        unsigned long long tot;
        unsigned long long pre = block_exclusive_scan<1024>(v, &tot, ws);
        if (i < nb) sums[i] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(SC_THREADS)
scan_down_kernel(const uint32_t *in, uint64_t n, const unsigned long long *block_off, uint64_t *out) {
    __shared__ unsigned long long ws[SC_THREADS / 32];
    uint64_t b0 = blockIdx.x * (uint64_t)SC_PER_BLOCK;
    // thread t owns SC_ITEMS consecutive elements (blocked) for an ordered scan
    uint64_t t0 = b0 + (uint64_t)threadIdx.x * SC_ITEMS;
    uint32_t v[SC_ITEMS];
    unsigned long long s = 0;
#pragma unroll
    for (int t = 0; t < SC_ITEMS; t++) {
        uint64_t i = t0 + t;
        v[t] = i < n ? in[i] : 0u;
        s += v[t];
    }
    unsigned long long tot;
    unsigned long long pre = block_exclusive_scan<SC_THREADS>(s, &tot, ws) + block_off[blockIdx.x];
#pragma unroll
    for (int t = 0; t < SC_ITEMS; t++) {
        uint64_t i = t0 + t;
        if (i < n) out[i] = pre;
        pre += v[t];
    }
}

// ---------------------------------------------------------------------------
// segmented LSD radix sort
struct TileDesc {
    uint64_t start;     // first key of the tile
    uint64_t cnt_base;  // base of the tile's segment in the counts array
    uint32_t n;         // keys in the tile
    uint32_t t;         // tile index inside its segment
    uint32_t nt;        // tiles in the segment
    uint32_t pad;
};
static_assert(sizeof(TileDesc) == 32, "tile layout");

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
// keys per thread: 16 u64, or 8 u128 (the scatter holds them in registers)
template <class KT> constexpr int rs_items() { return sizeof(KT) == 16 ? 8 : 16; }
template <class KT> constexpr int rs_tile() { return RS_THREADS * rs_items<KT>(); }

template <int RB, class KT>
__global__ void __launch_bounds__(RS_THREADS)
radix_hist_kernel(const KT *keys, const TileDesc *tiles, int shift, uint32_t *counts) {
    constexpr int NB = 1 << RB;
    __shared__ uint32_t hist[NB];
    const TileDesc td = tiles[blockIdx.x];
    for (int d = threadIdx.x; d < NB; d += RS_THREADS) hist[d] = 0;
    __syncthreads();
    const uint64_t dmask = NB - 1;
#pragma unroll 4
    for (int i = 0; i < rs_items<KT>(); i++) {
        uint32_t j = (uint32_t)i * RS_THREADS + threadIdx.x;
        if (j < td.n) atomicAdd(&hist[(uint32_t)((keys[td.start + j] >> shift) & dmask)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < NB; d += RS_THREADS)
        counts[td.cnt_base + (uint64_t)d * td.nt + td.t] = hist[d];
}

template <int RB, class KT>
__global__ void __launch_bounds__(RS_THREADS)
radix_scatter_kernel(const KT *in, KT *out, const TileDesc *tiles, int shift, const uint64_t *offsets) {
    constexpr int NB = 1 << RB;
    __shared__ uint32_t wcnt[RS_WARPS][NB];
    const TileDesc td = tiles[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1;
    for (int d = threadIdx.x; d < RS_WARPS * NB; d += RS_THREADS) (&wcnt[0][0])[d] = 0;
    __syncthreads();
    const uint64_t dmask = NB - 1;
    KT key[rs_items<KT>()];
    uint32_t rank[rs_items<KT>()];
    // warp-striped: warp w owns keys [w*32*ITEMS, (w+1)*32*ITEMS) of the tile
#pragma unroll
    for (int i = 0; i < rs_items<KT>(); i++) {
        uint32_t j = (uint32_t)warp * 32 * rs_items<KT>() + (uint32_t)i * 32 + lane;
        bool valid = j < td.n;
        key[i] = valid ? in[td.start + j] : KT(0);
        unsigned act = __ballot_sync(FULL, valid);
        rank[i] = 0;
        if (valid) {
            uint32_t dig = (uint32_t)((key[i] >> shift) & dmask);
            unsigned grp = __match_any_sync(act, dig);
            uint32_t pre = wcnt[warp][dig];
            rank[i] = pre + __popc(grp & lt);
            __syncwarp(act);
            if ((grp & lt) == 0) wcnt[warp][dig] = pre + __popc(grp);
        }
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps for every digit
    for (int d = threadIdx.x; d < NB; d += RS_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) {
            uint32_t t = wcnt[w][d];
            wcnt[w][d] = s;
            s += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < rs_items<KT>(); i++) {
        uint32_t j = (uint32_t)warp * 32 * rs_items<KT>() + (uint32_t)i * 32 + lane;
        if (j < td.n) {
            uint32_t dig = (uint32_t)((key[i] >> shift) & dmask);
            uint64_t pos = offsets[td.cnt_base + (uint64_t)dig * td.nt + td.t] + wcnt[warp][dig] + rank[i];
            out[pos] = key[i];
        }
    }
}

// ---------------------------------------------------------------------------
// run-length encoding + threshold over the sorted buffer.  A CTA takes a tile
// of RL_TILE keys and each warp a contiguous chunk of RL_ITEMS x 32 of them,
// read 32 consecutive keys a step (coalesced); a key is a run head when it
// differs from the key before it (a shuffle, and the previous step's last key
// for lane 0), and a head's rank is the heads of the earlier steps and lanes
// (ballots), so the heads come out in key order.
constexpr int RL_THREADS = 256;
constexpr int RL_ITEMS = 16;
constexpr int RL_WARPS = RL_THREADS / 32;
constexpr int RL_TILE = RL_THREADS * RL_ITEMS;

// Warp shuffles of a key (u64, or u128 as two words).
__device__ __forceinline__ uint64_t key_shfl_up(uint64_t v, int d) { return __shfl_up_sync(FULL, v, d); }
__device__ __forceinline__ uint64_t key_shfl(uint64_t v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ u128 key_shfl_up(u128 v, int d) {
    const uint64_t lo = __shfl_up_sync(FULL, (uint64_t)v, d), hi = __shfl_up_sync(FULL, (uint64_t)(v >> 64), d);
    return ((u128)hi << 64) | lo;
}
__device__ __forceinline__ u128 key_shfl(u128 v, int src) {
    const uint64_t lo = __shfl_sync(FULL, (uint64_t)v, src), hi = __shfl_sync(FULL, (uint64_t)(v >> 64), src);
    return ((u128)hi << 64) | lo;
}

// Heads of the warp's chunk [c0, c0 + 32 * RL_ITEMS), as one ballot mask per
// step; equal keys never straddle two partitions (a canonical k-mer has one
// minimizer, so one partition).
template <class KT>
__device__ __forceinline__ void rl_heads(const KT *keys, uint64_t n, uint64_t c0, unsigned (&hm)[RL_ITEMS], KT (&kv)[RL_ITEMS]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        const uint64_t i = c0 + (uint64_t)t * 32 + lane;
        kv[t] = i < n ? keys[i] : KT(0);
    }
    KT prev = (lane == 0 && c0 > 0 && c0 - 1 < n) ? keys[c0 - 1] : KT(0);
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        const uint64_t i = c0 + (uint64_t)t * 32 + lane;
        KT up = key_shfl_up(kv[t], 1);
        if (lane == 0) up = prev;
        prev = key_shfl(kv[t], 31);
        hm[t] = __ballot_sync(FULL, i < n && (i == 0 || kv[t] != up));
    }
}

template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
rle_count_kernel(const KT *keys, uint64_t n, uint32_t *tile_cnt) {
    __shared__ uint32_t ws[RL_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t c0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)warp * 32 * RL_ITEMS;
    unsigned hm[RL_ITEMS];
    KT kv[RL_ITEMS];
    rl_heads(keys, n, c0, hm, kv);
    uint32_t c = 0;
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) c += __popc(hm[t]);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < RL_WARPS; w++) s += ws[w];
        tile_cnt[blockIdx.x] = s;
    }
}

template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
rle_write_kernel(const KT *keys, uint64_t n, const uint64_t *tile_off, uint64_t *head_pos, KT *head_key) {
    __shared__ uint32_t ws[RL_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1;
    const uint64_t c0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)warp * 32 * RL_ITEMS;
    unsigned hm[RL_ITEMS];
    KT kv[RL_ITEMS];
    rl_heads(keys, n, c0, hm, kv);
    uint32_t c = 0;
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) c += __popc(hm[t]);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    uint64_t o = tile_off[blockIdx.x];
    for (int w = 0; w < warp; w++) o += ws[w];
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        if ((hm[t] >> lane) & 1) {
            const uint64_t q = o + __popc(hm[t] & lt);
            head_pos[q] = c0 + (uint64_t)t * 32 + lane;
            head_key[q] = kv[t];
        }
        o += __popc(hm[t]);
    }
}

// Run j's count: the next head's position (or n) minus its own, saturated
// at 2^32 - 1 (types.h:101-102).  Heads are read 32 a step like the keys.
__device__ __forceinline__ void rl_runs(const uint64_t *head_pos, uint64_t d, uint64_t n, uint64_t c0, uint32_t cmin,
                                        uint32_t cmax, unsigned (&km)[RL_ITEMS], uint32_t (&cnt)[RL_ITEMS]) {
    const int lane = threadIdx.x & 31;
    uint64_t hp[RL_ITEMS];
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        const uint64_t j = c0 + (uint64_t)t * 32 + lane;
        hp[t] = j < d ? head_pos[j] : n;
    }
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        const uint64_t j = c0 + (uint64_t)t * 32 + lane;
        uint64_t nx = __shfl_down_sync(FULL, hp[t], 1);
        if (lane == 31) nx = j + 1 < d ? head_pos[j + 1] : n;
        const uint64_t r = nx - hp[t];
        cnt[t] = r > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)r;
        km[t] = __ballot_sync(FULL, j < d && cnt[t] >= cmin && cnt[t] <= cmax);
    }
}

__global__ void __launch_bounds__(RL_THREADS)
keep_count_kernel(const uint64_t *head_pos, uint64_t d, uint64_t n, uint32_t cmin, uint32_t cmax,
                  uint32_t *tile_cnt) {
    __shared__ uint32_t ws[RL_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t c0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)warp * 32 * RL_ITEMS;
    unsigned km[RL_ITEMS];
    uint32_t cnt[RL_ITEMS];
    rl_runs(head_pos, d, n, c0, cmin, cmax, km, cnt);
    uint32_t c = 0;
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) c += __popc(km[t]);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < RL_WARPS; w++) s += ws[w];
        tile_cnt[blockIdx.x] = s;
    }
}

template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
keep_write_kernel(const uint64_t *head_pos, const KT *head_key, uint64_t d, uint64_t n, uint32_t cmin,
                  uint32_t cmax, const uint64_t *tile_off, KT *out_k, uint32_t *out_c) {
    __shared__ uint32_t ws[RL_WARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1;
    const uint64_t c0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)warp * 32 * RL_ITEMS;
    unsigned km[RL_ITEMS];
    uint32_t cnt[RL_ITEMS];
    rl_runs(head_pos, d, n, c0, cmin, cmax, km, cnt);
    uint32_t c = 0;
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) c += __popc(km[t]);
    if (lane == 0) ws[warp] = c;
    __syncthreads();
    uint64_t o = tile_off[blockIdx.x];
    for (int w = 0; w < warp; w++) o += ws[w];
#pragma unroll
    for (int t = 0; t < RL_ITEMS; t++) {
        if ((km[t] >> lane) & 1) {
            const uint64_t q = o + __popc(km[t] & lt);
            out_k[q] = head_key[c0 + (uint64_t)t * 32 + lane];
            out_c[q] = cnt[t];
        }
        o += __popc(km[t]);
    }
}

}  // namespace gkc
