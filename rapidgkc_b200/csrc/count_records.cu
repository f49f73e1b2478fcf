// count_records.cu -- phase 2, second level of the shared-memory hash counter.
//
// A minimizer sub-bucket holding a heavy minimizer (a low-complexity run, or
// a minimizer common in a repeat family) can have more k-mer instances or more
// distinct k-mers than one CTA should count.  Such sub-buckets are re-split
// by a hash of the k-mer itself, which spreads distinct k-mers uniformly.
// Their superkmers are cut into work items of RW_ENTRIES entries:
//   inst     the k-mer instances of every work item, scanned into the offsets
//            of per-item record segments (a record stands for at least one
//            instance, so a segment never overflows);
//   agg      one CTA per work item decodes its k-mers once and counts them in
//            a shared-memory table (pre-aggregation: a low-complexity run
//            collapses to a few records); a k-mer that finds no free slot is
//            written out as a record at once.  The table is then written to
//            the segment as (k-mer, count, record sub-bucket) records, where
//            the record sub-bucket is hash(k-mer) >> (64 - r_log) of the work
//            item's sub-bucket, and records are counted per record sub-bucket;
//   scatter  one CTA per work item moves its segment into record-sub-bucket
//            order (no decoding: the segment is re-read from L2);
//   count    one CTA per window of about RC_WINDOW records (whole record
//            sub-buckets) adds them into a shared-memory table and writes the
//            k-mers within [cmin, cmax].
// A record sub-bucket that still overflows (more distinct k-mers than its
// instance estimate allowed) is listed and counted through the L2 table.
#include "count_bucket.cu"

namespace gkc {

struct KRec {
    unsigned long long key;
    uint32_t cnt;
    uint32_t rb;     // record sub-bucket (segment records); unused in sorted records
};
static_assert(sizeof(KRec) == 16, "record layout");

// One piece of a listed sub-bucket: its entries [e0, e1) split into the
// 2^r_log record sub-buckets starting at rb_base.
struct RWork {
    uint64_t e0, e1;
    uint32_t rb_base, r_log;
};
static_assert(sizeof(RWork) == 24, "work layout");

constexpr int RS_MAX_LOG = 11;     // at most 2048 record sub-buckets per sub-bucket
constexpr int RSP_THREADS = 256;
constexpr int RW_ENTRIES = 256;    // entries per work item: their k-mers fit u32
constexpr int RS_TS = 4096;        // pre-aggregation table slots
constexpr uint32_t RS_MAX_PROBE = 64;
// dynamic shared memory of rec_agg_kernel: keys, counts, per-record-sub-bucket counts
constexpr size_t RA_SMEM = (size_t)RS_TS * 12 + (size_t)(1 << RS_MAX_LOG) * 4;

__device__ __forceinline__ uint32_t rec_bucket(uint64_t key, uint32_t r_log) {
    // The table slot of smem_add is the top bits of key * 0x9E37..; the
    // record sub-bucket must not depend on those bits, or the records of one
    // record sub-bucket would share a fraction of the table.  splitmix64's
    // top bits are independent of them.
    return r_log ? (uint32_t)(hash64(key) >> (64 - r_log)) : 0u;
}

// k-mer instances of each work item (one warp per item).
__global__ void __launch_bounds__(256)
work_inst_kernel(const BEntry *ent, const RWork *work, uint32_t nwork, uint32_t *winst) {
    const uint32_t w = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (w >= nwork) return;
    const RWork wk = work[w];
    uint32_t s = 0;
    for (uint64_t i = wk.e0 + (threadIdx.x & 31); i < wk.e1; i += 32) s += ent[i].len;
#pragma unroll
    for (int d = 16; d; d >>= 1) s += __shfl_xor_sync(FULL, s, d);
    if ((threadIdx.x & 31) == 0) winst[w] = s;
}

struct RAggParams {
    const BEntry *entries;
    const RWork *work;
    const uint64_t *woff;           // [work items] segment offsets
    int k;
    KRec *stage;                    // segments
    uint32_t *wrec;                 // [work items] records written
    uint32_t *rcount;               // [NR] records per record sub-bucket
};

// Shared-memory insert; false when the probe found no slot within
// RS_MAX_PROBE (the table is nearly full).
__device__ __forceinline__ bool smem_try_add(unsigned long long *tk, uint32_t *tc, uint64_t key, uint32_t c) {
    constexpr int LOG = __builtin_ctz(RS_TS);
    uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> (64 - LOG));
    for (uint32_t pr = 0; pr < RS_MAX_PROBE; pr++) {
        unsigned long long cur = tk[h];
        if (cur == key) {
            atomicAdd(&tc[h], c);
            return true;
        }
        if (cur == EMPTY_KEY) {
            unsigned long long old = atomicCAS(&tk[h], (unsigned long long)EMPTY_KEY, (unsigned long long)key);
            if (old == EMPTY_KEY || old == key) {
                atomicAdd(&tc[h], c);
                return true;
            }
        }
        h = (h + 1) & (RS_TS - 1);
    }
    return false;
}

__global__ void __launch_bounds__(RSP_THREADS)
rec_agg_kernel(RAggParams a) {
    extern __shared__ unsigned long long ra_smem[];
    unsigned long long *tk = ra_smem;                         // [RS_TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + RS_TS);  // [RS_TS] counts
    uint32_t *cnt = tc + RS_TS;                               // [2^RS_MAX_LOG]
    __shared__ uint32_t lcur;
    __shared__ uint32_t ws[RSP_THREADS / 32];
    const RWork w = a.work[blockIdx.x];
    const uint32_t R = 1u << w.r_log;
    KRec *seg = a.stage + a.woff[blockIdx.x];
    for (int t = threadIdx.x; t < RS_TS; t += RSP_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS) cnt[t] = 0;
    if (threadIdx.x == 0) lcur = 0;
    __syncthreads();
    const uint64_t mask = kmask(a.k);
    for (uint64_t bb = w.e0 + (threadIdx.x & ~31u); bb < w.e1; bb += RSP_THREADS) {
        warp_kmer_runs(a.entries, bb, w.e1, a.k, mask, [&](uint64_t key, uint32_t run) {
            if (!smem_try_add(tk, tc, key, run)) {
                const uint32_t r = rec_bucket(key, w.r_log);
                KRec rec;
                rec.key = key;
                rec.cnt = run;
                rec.rb = w.rb_base + r;
                seg[atomicAdd(&lcur, 1u)] = rec;
                atomicAdd(&cnt[r], 1u);
            }
        });
    }
    __syncthreads();
    // the table: thread i owns slots i, i + NT, ...
    constexpr int PER = RS_TS / RSP_THREADS;
    uint32_t n = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) n += tk[t * RSP_THREADS + threadIdx.x] != EMPTY_KEY;
    uint32_t tot;
    uint32_t o = block_exclusive_scan<RSP_THREADS>(n, &tot, ws) + lcur;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        const int sl = t * RSP_THREADS + threadIdx.x;
        const unsigned long long key = tk[sl];
        if (key != EMPTY_KEY) {
            const uint32_t r = rec_bucket(key, w.r_log);
            KRec rec;
            rec.key = key;
            rec.cnt = tc[sl];
            rec.rb = w.rb_base + r;
            seg[o++] = rec;
            atomicAdd(&cnt[r], 1u);
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS)
        if (cnt[t]) atomicAdd(a.rcount + w.rb_base + t, cnt[t]);
    if (threadIdx.x == 0) a.wrec[blockIdx.x] = lcur + tot;
}

struct RScatterParams {
    const RWork *work;
    const uint64_t *woff;
    const uint32_t *wrec;
    const KRec *stage;
    unsigned long long *rcursor;    // [NR] next free record
    KRec *recs;                     // records in record-sub-bucket order
};

__global__ void __launch_bounds__(RSP_THREADS)
rec_scatter_kernel(RScatterParams a) {
    __shared__ uint32_t cnt[1 << RS_MAX_LOG];
    __shared__ unsigned long long base[1 << RS_MAX_LOG];
    const RWork w = a.work[blockIdx.x];
    const uint32_t R = 1u << w.r_log;
    const KRec *seg = a.stage + a.woff[blockIdx.x];
    const uint32_t n = a.wrec[blockIdx.x];
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS) cnt[t] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += RSP_THREADS) atomicAdd(&cnt[seg[i].rb - w.rb_base], 1u);
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < R; t += RSP_THREADS) {
        base[t] = cnt[t] ? atomicAdd(a.rcursor + w.rb_base + t, (unsigned long long)cnt[t]) : 0ull;
        cnt[t] = 0;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += RSP_THREADS) {
        const KRec rec = seg[i];
        const uint32_t r = rec.rb - w.rb_base;
        a.recs[base[r] + atomicAdd(&cnt[r], 1u)] = rec;
    }
}

// rec_count_kernel: CTA c counts the record sub-buckets whose first record
// lies in [c * RC_WINDOW, (c + 1) * RC_WINDOW): whole record sub-buckets (their
// key sets are disjoint, so they share one table), about RC_WINDOW records.
// A record sub-bucket holds at most ~4.3k instances, so a CTA sees at most
// ~7.4k distinct k-mers.
constexpr uint64_t RC_WINDOW = 3072;

struct RCountParams {
    const KRec *recs;
    const uint64_t *roff;        // [NR+1]
    uint64_t nr;                 // record sub-buckets
    uint32_t cmin, cmax;
    uint64_t *out_k;
    uint32_t *out_c;
    unsigned long long *out_cursor;
    uint64_t out_cap;
    unsigned long long *distinct;
    uint32_t *failed;            // [1 + CTAs]: count, then the windows left over
    uint32_t *err;
};

// First index i in [0, n] with off[i] >= v (off ascending).
__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t *off, uint64_t n, uint64_t v) {
    uint64_t lo = 0, hi = n + 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (off[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <int TS>
__global__ void __launch_bounds__(BC_THREADS)
rec_count_kernel(RCountParams a) {
    extern __shared__ unsigned long long tk[];             // [TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + TS);  // [TS] counts
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    const uint32_t r = blockIdx.x;
    const uint64_t lo = lower_bound_u64(a.roff, a.nr, r * RC_WINDOW);
    const uint64_t hi = min(lower_bound_u64(a.roff, a.nr, (r + 1) * RC_WINDOW), a.nr);
    if (lo >= hi || lo >= a.nr) return;
    const uint64_t e0 = a.roff[lo], e1 = a.roff[hi];
    if (e0 == e1) return;
    for (int t = threadIdx.x; t < TS; t += BC_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    // records were aggregated per work item, so equal keys are rare here:
    // one shared-memory insert per record.  The overflow check is a warp vote
    // so every lane of a warp leaves the loop together.
    for (uint64_t i0 = e0 + (threadIdx.x & ~31u); i0 < e1; i0 += BC_THREADS) {
        if (__any_sync(FULL, over != 0)) break;
        const uint64_t i = i0 + (threadIdx.x & 31);
        if (i < e1) {
            const KRec rec = a.recs[i];
            smem_add<TS>(tk, tc, &over, rec.key, rec.cnt);
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
