// count_records.cu -- phase 2, second level of the shared-memory hash counter.
//
// A minimizer sub-bucket holding a heavy minimizer (typically one inside a
// repeat family) can have more distinct k-mers than a CTA's shared-memory
// table.  Such sub-buckets are re-split by a hash of the k-mer itself, which
// spreads distinct k-mers uniformly:
//   split    the sub-bucket's superkmers are decoded, equal consecutive
//            k-mers merged, and each (k-mer, run) record is written to the
//            record sub-bucket hash(k-mer) >> (64 - r_log).  Pass 0 counts
//            records per record sub-bucket; pass 1 counts a CTA's records in
//            shared memory, reserves one block per record sub-bucket and
//            writes them;
//   count    one CTA per record sub-bucket adds its records into a
//            shared-memory table (equal keys of a warp merged with
//            __match_any_sync first) and writes the k-mers within [cmin, cmax].
// A record sub-bucket that still overflows (more distinct k-mers than its
// instance estimate allowed) is listed and counted through the L2 table.
#include "count_bucket.cu"

namespace gkc {

struct KRec {
    unsigned long long key;
    uint32_t cnt;
    uint32_t pad;
};
static_assert(sizeof(KRec) == 16, "record layout");

// One piece of an overflowed sub-bucket: its entries [e0, e1) split into the
// 2^r_log record sub-buckets starting at rb_base.
struct RWork {
    uint64_t e0, e1;
    uint32_t rb_base, r_log;
};
static_assert(sizeof(RWork) == 24, "work layout");

constexpr int RS_MAX_LOG = 11;     // at most 2048 record sub-buckets per sub-bucket
constexpr int RSP_THREADS = 256;
constexpr int RW_ENTRIES = 1024;   // entries per work item

struct RSplitParams {
    const BEntry *entries;
    const RWork *work;
    int k;
    uint32_t *rcount;               // [NR] records per record sub-bucket (pass 0)
    unsigned long long *rcursor;    // [NR] next free record (pass 1)
    KRec *recs;
    int pass;
};

__device__ __forceinline__ uint32_t rec_bucket(uint64_t key, uint32_t r_log) {
    // The table slot of smem_add is the top bits of key * 0x9E37..; the
    // record sub-bucket must not depend on those bits, or the records of one
    // record sub-bucket would share a fraction of the table.  splitmix64's
    // top bits are independent of them.
    return r_log ? (uint32_t)(hash64(key) >> (64 - r_log)) : 0u;
}

// Calls f(key, run) for the run-merged k-mers of entries [e0, e1); warps take
// 32 entries at a time.  Deterministic for a given block size, so both split
// passes see the same records.
template <class F>
__device__ __forceinline__ void for_each_run(const BEntry *ent, uint64_t e0, uint64_t e1, int k, F &&f) {
    const uint64_t mask = kmask(k);
    for (uint64_t bb = e0 + (threadIdx.x & ~31u); bb < e1; bb += blockDim.x) {
        warp_kmers<true>(ent, bb, e1, k, mask, [&](uint64_t key, bool valid) {
            uint32_t run;
            if (warp_run_head(key, valid, &run)) f(key, run);
        });
    }
}

__global__ void __launch_bounds__(RSP_THREADS)
rec_split_kernel(RSplitParams a) {
    __shared__ uint32_t cnt[1 << RS_MAX_LOG];
    __shared__ unsigned long long base[1 << RS_MAX_LOG];
    const RWork w = a.work[blockIdx.x];
    const uint32_t R = 1u << w.r_log;
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS) cnt[t] = 0;
    __syncthreads();
    for_each_run(a.entries, w.e0, w.e1, a.k, [&](uint64_t key, uint32_t) {
        atomicAdd(&cnt[rec_bucket(key, w.r_log)], 1u);
    });
    __syncthreads();
    if (a.pass == 0) {
        for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS)
            if (cnt[t]) atomicAdd(a.rcount + w.rb_base + t, cnt[t]);
        return;
    }
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS) {
        base[t] = cnt[t] ? atomicAdd(a.rcursor + w.rb_base + t, (unsigned long long)cnt[t]) : 0ull;
        cnt[t] = 0;
    }
    __syncthreads();
    for_each_run(a.entries, w.e0, w.e1, a.k, [&](uint64_t key, uint32_t run) {
        uint32_t r = rec_bucket(key, w.r_log);
        KRec rec;
        rec.key = key;
        rec.cnt = run;
        rec.pad = 0;
        a.recs[base[r] + atomicAdd(&cnt[r], 1u)] = rec;
    });
}

struct RCountParams {
    const KRec *recs;
    const uint64_t *roff;        // [NR+1]
    uint32_t cmin, cmax;
    uint64_t *out_k;
    uint32_t *out_c;
    unsigned long long *out_cursor;
    uint64_t out_cap;
    unsigned long long *distinct;
    uint32_t *failed;            // [1 + NR]: count, then the record sub-buckets left over
    uint32_t *err;
};

template <int TS>
__global__ void __launch_bounds__(BC_THREADS)
rec_count_kernel(RCountParams a) {
    extern __shared__ unsigned long long tk[];             // [TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + TS);  // [TS] counts
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    const uint32_t r = blockIdx.x;
    const uint64_t e0 = a.roff[r], e1 = a.roff[r + 1];
    if (e0 == e1) return;
    for (int t = threadIdx.x; t < TS; t += BC_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    // whole warps walk the records so equal keys of a warp can be merged; the
    // overflow check is a warp vote so every lane leaves the loop together
    for (uint64_t i0 = e0 + (threadIdx.x & ~31u); i0 < e1; i0 += BC_THREADS) {
        if (__any_sync(FULL, over != 0)) break;
        const uint64_t i = i0 + (threadIdx.x & 31);
        const bool has = i < e1;
        KRec rec;
        rec.key = EMPTY_KEY;
        rec.cnt = 0;
        if (has) rec = a.recs[i];
        const unsigned act = __ballot_sync(FULL, has);
        if (has) {
            const unsigned grp = __match_any_sync(act, rec.key);
            const uint32_t tot = __reduce_add_sync(grp, rec.cnt);
            if ((threadIdx.x & 31) == (unsigned)(__ffs(grp) - 1)) smem_add<TS>(tk, tc, &over, rec.key, tot);
        }
    }
    __syncthreads();
    if (over) {
        if (threadIdx.x == 0) {
            uint32_t j = atomicAdd(a.failed, 1u);
            a.failed[1 + j] = r;
        }
        return;
    }
    smem_collect<TS, BC_THREADS>(tk, tc, a.cmin, a.cmax, a.out_k, a.out_c, a.out_cursor, a.out_cap, a.distinct,
                                 a.err, ws, &base_s);
}

// L2-table insert of records (record sub-buckets that overflow shared memory).
__global__ void __launch_bounds__(H_THREADS)
hash_insert_records_kernel(const KRec *recs, uint64_t n, HSlot *tab, uint64_t mask, uint32_t *err) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        KRec r = recs[i];
        table_add(tab, mask, r.key, r.cnt, err);
    }
}

}  // namespace gkc
