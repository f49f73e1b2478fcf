// count_hash.cu -- phase 2, hash counter: superkmers -> (k-mer, count).
//
// The reference's hash counter (gpu_hash_counter.cu:171-493, not in its
// build) locks each bucket entry with a CAS 0->1->2 spin and counts keys seen
// at least twice.  This one is lock-free open addressing with linear probing
// over 16-byte slots {64-bit key (EMPTY = all ones), 32-bit count}, so a probe
// and its count update touch one 32-byte sector.  The table is sized to stay
// resident in L2 for one partition at a time:
//   insert  a new key costs one CAS, a present key one atomicAdd; callers
//           merge equal consecutive k-mers first, so a hot key costs one atomic
//           per run (count_bucket.cu decodes superkmers into this table for
//           the sub-buckets that overflow shared memory);
//   collect every thread loads its slots before storing anything, writes the
//           entries whose count lies in [cmin, cmax] (block-aggregated cursor),
//           counts the distinct keys and clears the slots for the next
//           partition.
#include "gkc_device.cuh"

namespace gkc {

constexpr int H_THREADS = 256;
constexpr uint32_t H_MAX_PROBE = 4096;

struct __align__(16) HSlot {
    unsigned long long key;
    uint32_t cnt;
    uint32_t pad;
};
static_assert(sizeof(HSlot) == 16, "slot layout");

// Once any insert of the pass has given up (ERR_TABLE_FULL), the pass is
// redone with a larger table or failed, so the others stop probing too: every
// 64 probes a thread looks at the flag.
__device__ __forceinline__ void table_add(HSlot *tab, uint64_t mask, uint64_t key, uint32_t c, uint32_t *err) {
    uint64_t h = hash64(key) & mask;
    for (uint32_t pr = 0; pr < H_MAX_PROBE; pr++) {
        if ((pr & 63) == 63 && (__ldcg(err) & ERR_TABLE_FULL)) return;
        unsigned long long cur = __ldcg(&tab[h].key);
        if (cur == key) {
            atomicAdd(&tab[h].cnt, c);
            return;
        }
        if (cur == EMPTY_KEY) {
            unsigned long long old = atomicCAS(&tab[h].key, (unsigned long long)EMPTY_KEY, (unsigned long long)key);
            if (old == EMPTY_KEY || old == key) {
                atomicAdd(&tab[h].cnt, c);
                return;
            }
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, ERR_TABLE_FULL);
}

// Raw 64-bit keys (no canonical step): the reference hash counter's own
// known-answer test counts plain integers (gpu_hash_counter.cu:693-708).
__global__ void __launch_bounds__(H_THREADS)
hash_insert_keys_kernel(const uint64_t *in, uint64_t n, HSlot *tab, uint64_t mask, uint32_t *err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = in[i];
        if (key == EMPTY_KEY) {
            atomicOr(err, ERR_DECODE);
            continue;
        }
        table_add(tab, mask, key, 1u, err);
    }
}

__global__ void hash_init_kernel(HSlot *tab, uint64_t cap) {
    const ulonglong2 empty = make_ulonglong2(EMPTY_KEY, 0ull);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x)
        reinterpret_cast<ulonglong2 *>(tab)[i] = empty;
}

constexpr int HC_ITEMS = 4;

struct HCollectParams {
    HSlot *tab;
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
    const ulonglong2 empty = make_ulonglong2(EMPTY_KEY, 0ull);
    for (uint64_t b0 = blockIdx.x * per_block; b0 < a.cap; b0 += (uint64_t)gridDim.x * per_block) {
        ulonglong2 v[HC_ITEMS];
#pragma unroll
        for (int t = 0; t < HC_ITEMS; t++) {
            uint64_t s = b0 + (uint64_t)t * H_THREADS + threadIdx.x;
            v[t] = s < a.cap ? __ldcg(reinterpret_cast<const ulonglong2 *>(a.tab) + s) : empty;
        }
        uint32_t keep = 0, occ = 0;
#pragma unroll
        for (int t = 0; t < HC_ITEMS; t++) {
            if (v[t].x != EMPTY_KEY) {
                uint64_t s = b0 + (uint64_t)t * H_THREADS + threadIdx.x;
                reinterpret_cast<ulonglong2 *>(a.tab)[s] = empty;
                occ++;
                uint32_t c = (uint32_t)v[t].y;
                if (!failed && c >= a.cmin && c <= a.cmax) keep++;
                else v[t].x = EMPTY_KEY;
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
                if (v[t].x != EMPTY_KEY) {
                    if (o < a.out_cap) {
                        a.out_k[o] = v[t].x;
                        a.out_c[o] = (uint32_t)v[t].y;
                    } else {
                        atomicOr(a.err, ERR_OUTPUT_FULL);
                    }
                    o++;
                }
            }
        }
    }
}

}  // namespace gkc
