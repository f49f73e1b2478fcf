// count_sort.cu -- phase 2, sort counter: superkmers -> sorted (k-mer, count).
//
// Replaces the reference's Extract_Kmers + thrust::transform(canonicalkmer)
// + thrust::sort + sameasprev/sequence/remove_if chain and its host-side
// count differences (gpu_kmercounting.cu:257-523):
//   extract  one thread per superkmer writes its canonical k-mers into its
//            partition's segment of the key buffer (warp-aggregated cursor);
//   sort     a hand-written stable LSD radix sort over only the 2k meaningful
//            bits, all partitions at once as independent segments: per pass
//            a tile histogram, one device-wide scan of the segment-major
//            [segment][digit][tile] counts, and a scatter whose in-tile ranks
//            come from __match_any_sync over per-warp digit counters;
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

template <class KT>
__global__ void __launch_bounds__(SX_THREADS)
sort_extract_kernel(SExtractParams a) {
    KT *keys = static_cast<KT *>(a.keys);
    const int lane = threadIdx.x & 31;
    for (uint64_t base = a.i_begin + blockIdx.x * (uint64_t)SX_THREADS; base < a.n_skm;
         base += (uint64_t)gridDim.x * SX_THREADS) {
        uint64_t i = base + threadIdx.x;
        bool has = i < a.n_skm;
        uint32_t part = 0, L = 0;
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
        // warp-aggregated reservation: lanes of one partition are contiguous
        unsigned act = __ballot_sync(FULL, has);
        uint64_t dst = 0;
        if (has) {
            unsigned grp = __match_any_sync(act, part);
            uint32_t incl = L;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                uint32_t y = __shfl_up_sync(act, incl, d);
                if (lane >= d && ((act >> (lane - d)) & 1)) incl += y;
            }
            // all lanes below `lane` are active (has is a prefix of the warp)
            int first = __ffs(grp) - 1;
            uint32_t excl_first = __shfl_sync(grp, incl - L, first);
            int last = 31 - __clz(grp);
            uint32_t incl_last = __shfl_sync(grp, incl, last);
            unsigned long long b = 0;
            if (lane == first) b = atomicAdd(a.seg_cursor + part, (unsigned long long)(incl_last - excl_first));
            b = __shfl_sync(grp, b, first);
            dst = a.seg_off[part] + b + (incl - L - excl_first);
        }
        if (has) {
            const uint8_t *pb = a.bytes + a.part_byte_off[part];
            uint64_t o = dst;
            if constexpr (sizeof(KT) == 16)
                for_each_kmer_wide(pb, e, a.k, [&](u128 key) { keys[o++] = key; });
            else if (a.canonical)
                for_each_kmer<true>(pb, e, a.k, [&](uint64_t key) { keys[o++] = key; });
            else
                for_each_kmer<false>(pb, e, a.k, [&](uint64_t key) { keys[o++] = key; });
        }
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
// run-length encoding + threshold over the sorted buffer
constexpr int RL_THREADS = 256;
constexpr int RL_ITEMS = 16;
constexpr int RL_TILE = RL_THREADS * RL_ITEMS;

// Heads per tile: i == 0 or key[i] != key[i-1].  Equal keys never straddle
// two partitions (a canonical k-mer has one minimizer, so one partition).
template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
rle_count_kernel(const KT *keys, uint64_t n, uint32_t *tile_cnt) {
    __shared__ uint32_t ws[RL_THREADS / 32];
    uint64_t t0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)threadIdx.x * RL_ITEMS;
    uint32_t c = 0;
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t i = t0 + t;
        if (i < n && (i == 0 || keys[i] != keys[i - 1])) c++;
    }
    uint32_t tot;
    block_exclusive_scan<RL_THREADS>(c, &tot, ws);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
rle_write_kernel(const KT *keys, uint64_t n, const uint64_t *tile_off, uint64_t *head_pos, KT *head_key) {
    __shared__ uint32_t ws[RL_THREADS / 32];
    uint64_t t0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)threadIdx.x * RL_ITEMS;
    uint32_t c = 0;
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t i = t0 + t;
        if (i < n && (i == 0 || keys[i] != keys[i - 1])) c++;
    }
    uint32_t tot;
    uint64_t o = tile_off[blockIdx.x] + block_exclusive_scan<RL_THREADS>(c, &tot, ws);
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t i = t0 + t;
        if (i < n && (i == 0 || keys[i] != keys[i - 1])) {
            head_pos[o] = i;
            head_key[o] = keys[i];
            o++;
        }
    }
}

__device__ __forceinline__ uint32_t run_count(const uint64_t *head_pos, uint64_t d, uint64_t j, uint64_t n) {
    uint64_t c = ((j + 1 < d) ? head_pos[j + 1] : n) - head_pos[j];
    return c > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)c;
}

__global__ void __launch_bounds__(RL_THREADS)
keep_count_kernel(const uint64_t *head_pos, uint64_t d, uint64_t n, uint32_t cmin, uint32_t cmax,
                  uint32_t *tile_cnt) {
    __shared__ uint32_t ws[RL_THREADS / 32];
    uint64_t t0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)threadIdx.x * RL_ITEMS;
    uint32_t c = 0;
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t j = t0 + t;
        if (j < d) {
            uint32_t r = run_count(head_pos, d, j, n);
            c += (r >= cmin && r <= cmax);
        }
    }
    uint32_t tot;
    block_exclusive_scan<RL_THREADS>(c, &tot, ws);
    if (threadIdx.x == 0) tile_cnt[blockIdx.x] = tot;
}

template <class KT>
__global__ void __launch_bounds__(RL_THREADS)
keep_write_kernel(const uint64_t *head_pos, const KT *head_key, uint64_t d, uint64_t n, uint32_t cmin,
                  uint32_t cmax, const uint64_t *tile_off, KT *out_k, uint32_t *out_c) {
    __shared__ uint32_t ws[RL_THREADS / 32];
    uint64_t t0 = blockIdx.x * (uint64_t)RL_TILE + (uint64_t)threadIdx.x * RL_ITEMS;
    uint32_t c = 0;
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t j = t0 + t;
        if (j < d) {
            uint32_t r = run_count(head_pos, d, j, n);
            c += (r >= cmin && r <= cmax);
        }
    }
    uint32_t tot;
    uint64_t o = tile_off[blockIdx.x] + block_exclusive_scan<RL_THREADS>(c, &tot, ws);
    for (int t = 0; t < RL_ITEMS; t++) {
        uint64_t j = t0 + t;
        if (j < d) {
            uint32_t r = run_count(head_pos, d, j, n);
            if (r >= cmin && r <= cmax) {
                out_k[o] = head_key[j];
                out_c[o] = r;
                o++;
            }
        }
    }
}

}  // namespace gkc
