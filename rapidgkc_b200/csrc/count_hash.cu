// count_hash.cu -- phase 2, hash counter: superkmers -> (k-mer, count).
//
// The reference's hash counter (gpu_hash_counter.cu:171-493, not in its
// build) locks each bucket entry with a CAS 0->1->2 spin and counts keys seen
// at least twice.  This one is lock-free open addressing with linear probing
// over a table of 64-bit keys (EMPTY = all ones) and 32-bit counts sized to
// stay resident in L2 for one partition at a time:
//   insert  one thread per superkmer decodes its canonical k-mers; equal
//           consecutive k-mers (poly-A and other low-complexity runs) are
//           merged in registers, equal keys across the warp are merged with
//           __match_any_sync / __reduce_add_sync, and the group leader does
//           one CAS (only for a new key) and one atomicAdd;
//   collect one pass over the table writes the entries whose count lies in
//           [cmin, cmax], counts the distinct keys, and clears the slots so the
//           table is ready for the next partition.
#include "gkc_device.cuh"

namespace gkc {

constexpr int H_THREADS = 256;
constexpr uint32_t H_MAX_PROBE = 4096;

__device__ __forceinline__ void table_add(unsigned long long *keys, uint32_t *cnts, uint64_t mask,
                                          uint64_t key, uint32_t c, uint32_t *err) {
    uint64_t h = hash64(key) & mask;
    for (uint32_t pr = 0; pr < H_MAX_PROBE; pr++) {
        unsigned long long cur = __ldcg(keys + h);
        if (cur == key) { atomicAdd(cnts + h, c); return; }
        if (cur == EMPTY_KEY) {
            unsigned long long old = atomicCAS(keys + h, (unsigned long long)EMPTY_KEY, (unsigned long long)key);
            if (old == EMPTY_KEY || old == key) { atomicAdd(cnts + h, c); return; }
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, ERR_TABLE_FULL);
}

// Merges equal keys across the lanes that flush together, then inserts.
__device__ __forceinline__ void flush_key(unsigned long long *keys, uint32_t *cnts, uint64_t mask,
                                          uint64_t key, uint32_t run, uint32_t *err) {
    unsigned act = __activemask();
    unsigned grp = __match_any_sync(act, (unsigned long long)key);
    uint32_t tot = __reduce_add_sync(grp, run);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(grp) - 1)) table_add(keys, cnts, mask, key, tot, err);
}

struct HInsertParams {
    const uint8_t *bytes;   // partition bytes
    const uint64_t *idx;    // partition superkmer index
    uint64_t n_skm;
    int k;
    unsigned long long *keys;
    uint32_t *cnts;
    uint64_t mask;          // table capacity - 1 (power of two)
    uint32_t *err;
};

__global__ void __launch_bounds__(H_THREADS)
hash_insert_kernel(HInsertParams a) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.n_skm;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t e = a.idx[i];
        uint64_t last = EMPTY_KEY;
        uint32_t run = 0;
        for_each_kmer<true>(a.bytes, e, a.k, [&](uint64_t key) {
            if (key == last) {
                run++;
            } else {
                if (run) flush_key(a.keys, a.cnts, a.mask, last, run, a.err);
                last = key;
                run = 1;
            }
        });
        if (run) flush_key(a.keys, a.cnts, a.mask, last, run, a.err);
    }
}

// Raw 64-bit keys (no canonical step): the reference hash counter's own
// known-answer test counts plain integers (gpu_hash_counter.cu:693-708).
__global__ void __launch_bounds__(H_THREADS)
hash_insert_keys_kernel(const uint64_t *in, uint64_t n, unsigned long long *keys, uint32_t *cnts,
                        uint64_t mask, uint32_t *err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = in[i];
        if (key == EMPTY_KEY) { atomicOr(err, ERR_DECODE); continue; }
        flush_key(keys, cnts, mask, key, 1u, err);
    }
}

constexpr int HC_ITEMS = 8;

struct HCollectParams {
    unsigned long long *keys;
    uint32_t *cnts;
    uint64_t cap;
    uint32_t cmin, cmax;
    uint64_t *out_k;
    uint32_t *out_c;
    unsigned long long *out_cursor;  // number of entries written so far
    uint64_t out_cap;
    unsigned long long *distinct;
    uint32_t *err;
    const uint32_t *part_err;        // flags of this partition's insert; a
                                     // failed insert is cleared, not output
};

__global__ void __launch_bounds__(H_THREADS)
hash_collect_kernel(HCollectParams a) {
    __shared__ uint32_t ws[H_THREADS / 32];
    __shared__ unsigned long long base_s;
    const uint64_t per_block = (uint64_t)H_THREADS * HC_ITEMS;
    const bool failed = (*a.part_err & ERR_TABLE_FULL) != 0;
    for (uint64_t b0 = blockIdx.x * per_block; b0 < a.cap; b0 += (uint64_t)gridDim.x * per_block) {
        uint64_t kk[HC_ITEMS];
        uint32_t cc[HC_ITEMS];
        uint32_t keep = 0, occ = 0;
#pragma unroll
        for (int t = 0; t < HC_ITEMS; t++) {
            uint64_t s = b0 + (uint64_t)t * H_THREADS + threadIdx.x;
            kk[t] = EMPTY_KEY;
            cc[t] = 0;
            if (s < a.cap) {
                kk[t] = a.keys[s];
                if (kk[t] != EMPTY_KEY) {
                    cc[t] = a.cnts[s];
                    a.keys[s] = EMPTY_KEY;
                    a.cnts[s] = 0;
                    occ++;
                    if (!failed && cc[t] >= a.cmin && cc[t] <= a.cmax) keep++;
                    else kk[t] = EMPTY_KEY;
                }
            }
        }
        uint32_t tot;
        uint32_t pre = block_exclusive_scan<H_THREADS>(keep, &tot, ws);
        uint32_t occ_tot;
        block_exclusive_scan<H_THREADS>(occ, &occ_tot, ws);
        if (threadIdx.x == 0) {
            base_s = tot ? atomicAdd(a.out_cursor, (unsigned long long)tot) : 0ull;
            if (occ_tot && !failed) atomicAdd(a.distinct, (unsigned long long)occ_tot);
        }
        __syncthreads();
        unsigned long long base = base_s;
        __syncthreads();
        if (keep) {
            uint64_t o = base + pre;
#pragma unroll
            for (int t = 0; t < HC_ITEMS; t++) {
                if (kk[t] != EMPTY_KEY) {
                    if (o < a.out_cap) { a.out_k[o] = kk[t]; a.out_c[o] = cc[t]; }
                    else atomicOr(a.err, ERR_OUTPUT_FULL);
                    o++;
                }
            }
        }
    }
}

}  // namespace gkc
