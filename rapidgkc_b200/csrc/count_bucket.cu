// count_bucket.cu -- phase 2, shared-memory hash counter over sub-buckets.
//
// Every partition of the store is split into S sub-buckets by a hash of the
// superkmers' minimizer keys.  A canonical k-mer has one minimizer, so all its
// occurrences land in one sub-bucket, and a sub-bucket can be counted on its
// own.  Sub-buckets are sized (S chosen from the partition sizes) so that their
// distinct k-mers fit an open-addressing table in one CTA's shared memory:
//   split    over all superkmers of all store chunks: a histogram of
//            superkmers per sub-bucket (shared-memory aggregated), a scan,
//            then a scatter of 16-byte entries {first byte address, k-mer
//            count} into sub-bucket order;
//   count    one CTA per sub-bucket decodes its superkmers warp-synchronously
//            (two streams per lane, equal consecutive k-mers merged) into a
//            shared-memory table with shared-memory atomics, then writes the
//            k-mers whose count lies in [cmin, cmax] with one global atomic
//            per CTA.  A sub-bucket whose distinct k-mers outgrow the table is
//            abandoned and listed; the host counts those through the L2 hash
//            table (count_hash.cu), so the result does not depend on skew.
#include "count_hash.cu"

namespace gkc {

struct BEntry {
    const uint8_t *ptr;  // first byte of the superkmer
    uint32_t len;        // k-mers
    uint32_t pad;
};
static_assert(sizeof(BEntry) == 16, "entry layout");

__device__ __forceinline__ uint32_t bucket_of(uint32_t key, int s_log) {
    return s_log ? (uint32_t)(hash64(key) >> (64 - s_log)) : 0u;
}

constexpr int BS_THREADS = 256;
constexpr int BS_PER_CTA = 2048;   // superkmers per split CTA
constexpr int BS_MAX_PARTS = 4;    // partitions a split CTA aggregates in shared memory
constexpr int BS_MAX_LOG = 9;      // at most 512 sub-buckets per partition

struct BSplitParams {
    const uint64_t *idx;                       // chunk superkmer index (partition-ordered)
    const uint32_t *keys;                      // chunk superkmer minimizer keys
    const uint8_t *bytes;                      // chunk bytes
    uint64_t i_begin, n_skm;                   // superkmer index range [i_begin, n_skm)
    const unsigned long long *part_skm_off;    // [P+1]
    const unsigned long long *part_byte_off;   // [P]
    uint32_t P;
    int s_log;                                 // S = 2^s_log sub-buckets per partition
    uint32_t *bucket_skms;                     // [P*S] superkmers per sub-bucket (pass 0)
    unsigned long long *bucket_kmers;          // [P*S] k-mers per sub-bucket (pass 0)
    unsigned long long *bucket_cursor;         // [P*S] next free entry (pass 1)
    BEntry *entries;                           // [total superkmers] (pass 1)
    int pass;
};

__device__ __forceinline__ uint32_t part_of_index(const unsigned long long *off, uint32_t P, uint64_t i) {
    uint32_t lo = 0, hi = P;  // off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Pass 0 counts superkmers per sub-bucket; pass 1 scatters entries.  A CTA
// covers BS_PER_CTA consecutive superkmers, which span few partitions: the
// sub-buckets of its first BS_MAX_PARTS partitions are aggregated in shared
// memory (one global atomic per sub-bucket per CTA), any further partition
// goes straight to global atomics.
__global__ void __launch_bounds__(BS_THREADS)
bucket_split_kernel(BSplitParams a) {
    constexpr int NB = BS_MAX_PARTS << BS_MAX_LOG;
    __shared__ uint32_t cnt[NB];
    __shared__ unsigned long long base[NB];
    __shared__ uint32_t p_first_s;
    const uint32_t S = 1u << a.s_log;  // s_log <= BS_MAX_LOG
    const uint64_t i0 = a.i_begin + blockIdx.x * (uint64_t)BS_PER_CTA;
    if (i0 >= a.n_skm) return;
    const uint64_t i1 = min(a.n_skm, i0 + BS_PER_CTA);
    if (threadIdx.x == 0) p_first_s = part_of_index(a.part_skm_off, a.P, i0);
    for (int t = threadIdx.x; t < NB; t += BS_THREADS) cnt[t] = 0, base[t] = 0;
    __syncthreads();
    const uint32_t pf = p_first_s;
    auto part = [&](uint64_t i) {
        return (i < a.part_skm_off[pf + 1]) ? pf : part_of_index(a.part_skm_off, a.P, i);
    };
    // count this CTA's superkmers (and, pass 0, k-mers) per shared sub-bucket
    // (global atomics for the rest); pass 0 sums k-mers in `base`
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += BS_THREADS) {
        uint32_t p = part(i);
        uint32_t b = bucket_of(a.keys[i], a.s_log);
        if (p - pf < BS_MAX_PARTS) {
            atomicAdd(&cnt[((p - pf) << BS_MAX_LOG) + b], 1u);
            if (a.pass == 0) atomicAdd(&base[((p - pf) << BS_MAX_LOG) + b], (unsigned long long)idx_len(a.idx[i]));
        } else if (a.pass == 0) {
            atomicAdd(a.bucket_skms + p * S + b, 1u);
            atomicAdd(a.bucket_kmers + p * S + b, (unsigned long long)idx_len(a.idx[i]));
        }
    }
    __syncthreads();
    if (a.pass == 0) {
        for (int t = threadIdx.x; t < NB; t += BS_THREADS)
            if (cnt[t]) {
                atomicAdd(a.bucket_skms + (pf + (t >> BS_MAX_LOG)) * S + (t & ((1 << BS_MAX_LOG) - 1)), cnt[t]);
                atomicAdd(a.bucket_kmers + (pf + (t >> BS_MAX_LOG)) * S + (t & ((1 << BS_MAX_LOG) - 1)), base[t]);
            }
        return;
    }
    // pass 1: reserve each shared sub-bucket's block, then write entries
    for (int t = threadIdx.x; t < NB; t += BS_THREADS) {
        base[t] = cnt[t] ? atomicAdd(a.bucket_cursor + (pf + (t >> BS_MAX_LOG)) * S + (t & ((1 << BS_MAX_LOG) - 1)), (unsigned long long)cnt[t])
                         : 0ull;
        cnt[t] = 0;
    }
    __syncthreads();
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += BS_THREADS) {
        uint32_t p = part(i);
        uint32_t b = bucket_of(a.keys[i], a.s_log);
        uint64_t slot;
        if (p - pf < BS_MAX_PARTS) {
            uint32_t t = ((p - pf) << BS_MAX_LOG) + b;
            slot = base[t] + atomicAdd(&cnt[t], 1u);
        } else {
            slot = atomicAdd(a.bucket_cursor + p * S + b, 1ull);
        }
        uint64_t e = a.idx[i];
        BEntry en;
        en.ptr = a.bytes + a.part_byte_off[p] + idx_off(e);
        en.len = idx_len(e);
        en.pad = 0;
        a.entries[slot] = en;
    }
}

// Decoder state over one entry stream.  The first k-mer needs at most the
// superkmer's first 12 bytes (k <= 32): they are fetched with three aligned
// 8-byte loads issued together (store buffers carry 32 bytes of padding) and
// assembled in registers.
__device__ __forceinline__ void entry_begin(SkmCursor &c, const BEntry &en, int k, uint64_t mask) {
    c.s = en.ptr;
    c.left = en.len - 1;
    const uintptr_t a = reinterpret_cast<uintptr_t>(en.ptr);
    const uint64_t *w = reinterpret_cast<const uint64_t *>(a & ~(uintptr_t)7);
    const uint32_t sh = 8 * (uint32_t)(a & 7);
    const uint64_t w0 = w[0], w1 = w[1], w2 = w[2];
    const uint64_t lo = sh ? (w0 >> sh) | (w1 << (64 - sh)) : w0;  // bytes 0..7
    const uint64_t hi = sh ? (w1 >> sh) | (w2 << (64 - sh)) : w1;  // bytes 8..15
    auto byte = [&](uint32_t i) -> uint32_t { return (uint32_t)((i < 8 ? lo >> (8 * i) : hi >> (8 * (i - 8))) & 0xFF); };
    const uint32_t b0 = (uint32_t)(lo & 0xFF);
    const uint32_t h = b0 >> 6;
    uint64_t f = b0 & ((1u << (2 * h)) - 1);
    const uint32_t need = (uint32_t)k - h;
    const uint32_t full = need / 3, part = need % 3;
    for (uint32_t t = 1; t <= full; t++) f = (f << 6) | (byte(t) & 63u);
    const uint32_t nxt = byte(full + 1);
    if (part) f = (f << (2 * part)) | ((nxt & 63u) >> (6 - 2 * part));
    c.fwd = f & mask;
    c.rc = rc64(c.fwd, k);
    c.bi = full + 1;
    c.slot = part;
    c.cur = nxt;
}

struct EStream {
    SkmCursor c;
    uint64_t next, step;
    uint64_t last;
    uint32_t run;
    __device__ __forceinline__ bool advance(const BEntry *ent, uint64_t end, int k, uint64_t mask, bool &flush,
                                            uint64_t &fk, uint32_t &fc) {
        flush = false;
        bool have = false;
        if (c.left) {
            skm_step(c, k, mask);
            have = true;
        } else if (next < end) {
            entry_begin(c, ent[next], k, mask);
            next += step;
            have = true;
        }
        if (have) {
            uint64_t key = c.fwd < c.rc ? c.fwd : c.rc;
            if (key == last) {
                run++;
            } else {
                flush = run != 0;
                fk = last;
                fc = run;
                last = key;
                run = 1;
            }
        }
        return have;
    }
};

constexpr int BC_THREADS = 512;

struct BCountParams {
    const BEntry *entries;
    const uint64_t *bucket_off;   // [nb+1] entry ranges of the sub-buckets
    uint32_t b0;                  // first sub-bucket of this launch
    int k;
    uint32_t cmin, cmax;
    uint64_t *out_k;
    uint32_t *out_c;
    unsigned long long *out_cursor;
    uint64_t out_cap;
    unsigned long long *distinct;
    uint32_t *failed;             // [1 + nb]: count, then the abandoned sub-buckets
    uint32_t *err;
};

// Shared-memory table insert.  A probe sequence longer than SM_MAX_PROBE
// (the table is nearly full) raises *over instead of inserting; the caller
// then abandons the table.  No shared fill counter: one would serialise
// every new key of the CTA on a single shared-memory word.
constexpr uint32_t SM_MAX_PROBE = 128;

template <int TS>
__device__ __forceinline__ void smem_add(unsigned long long *tk, uint32_t *tc, volatile uint32_t *over,
                                         uint64_t key, uint32_t c) {
    uint32_t h = (uint32_t)hash64(key) & (TS - 1);
    for (uint32_t pr = 0; pr < SM_MAX_PROBE; pr++) {
        unsigned long long cur = tk[h];
        if (cur == key) {
            atomicAdd(&tc[h], c);
            return;
        }
        if (cur == EMPTY_KEY) {
            unsigned long long old = atomicCAS(&tk[h], (unsigned long long)EMPTY_KEY, (unsigned long long)key);
            if (old == EMPTY_KEY || old == key) {
                atomicAdd(&tc[h], c);
                return;
            }
        }
        h = (h + 1) & (TS - 1);
    }
    *over = 1;
}

template <int TS>
__global__ void __launch_bounds__(BC_THREADS)
bucket_count_kernel(BCountParams a) {
    extern __shared__ unsigned long long tk[];  // [TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + TS);  // [TS] counts
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    const uint32_t b = a.b0 + blockIdx.x;
    const uint64_t e0 = a.bucket_off[b], e1 = a.bucket_off[b + 1];
    if (e0 == e1) return;
    for (int t = threadIdx.x; t < TS; t += BC_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t mask = kmask(a.k);
    constexpr int NWARP = BC_THREADS / 32;
    EStream s0, s1;
    s0.c.left = s1.c.left = 0;
    s0.next = e0 + (uint64_t)warp * 64 + lane;
    s1.next = s0.next + 32;
    s0.step = s1.step = (uint64_t)NWARP * 64;
    s0.last = s1.last = EMPTY_KEY;
    s0.run = s1.run = 0;
    for (;;) {
        bool f0, f1;
        uint64_t k0 = 0, k1 = 0;
        uint32_t c0 = 0, c1 = 0;
        bool h0 = s0.advance(a.entries, e1, a.k, mask, f0, k0, c0);
        bool h1 = s1.advance(a.entries, e1, a.k, mask, f1, k1, c1);
        // a warp vote, so every lane of the warp leaves the loop together
        if (!__any_sync(FULL, (h0 || h1) && over == 0)) break;
        if (f0) smem_add<TS>(tk, tc, &over, k0, c0);
        if (f1) smem_add<TS>(tk, tc, &over, k1, c1);
    }
    if (!over) {
        if (s0.run) smem_add<TS>(tk, tc, &over, s0.last, s0.run);
        if (s1.run) smem_add<TS>(tk, tc, &over, s1.last, s1.run);
    }
    __syncthreads();
    if (over) {
        if (threadIdx.x == 0) {
            uint32_t i = atomicAdd(a.failed, 1u);
            a.failed[1 + i] = b;
        }
        return;
    }
    // collect: each thread owns TS/BC_THREADS consecutive slots
    constexpr int PER = TS / BC_THREADS;
    uint32_t keep = 0, occ = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        int s = threadIdx.x * PER + t;
        if (tk[s] != EMPTY_KEY) {
            occ++;
            keep += (tc[s] >= a.cmin && tc[s] <= a.cmax);
        }
    }
    uint32_t tot, occ_tot;
    uint32_t pre = block_exclusive_scan<BC_THREADS>(keep, &tot, ws);
    block_exclusive_scan<BC_THREADS>(occ, &occ_tot, ws);
    if (threadIdx.x == 0) {
        base_s = tot ? atomicAdd(a.out_cursor, (unsigned long long)tot) : 0ull;
        atomicAdd(a.distinct, (unsigned long long)occ_tot);
    }
    __syncthreads();
    uint64_t o = base_s + pre;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        int s = threadIdx.x * PER + t;
        if (tk[s] != EMPTY_KEY && tc[s] >= a.cmin && tc[s] <= a.cmax) {
            if (o < a.out_cap) {
                a.out_k[o] = tk[s];
                a.out_c[o] = tc[s];
            } else {
                atomicOr(a.err, ERR_OUTPUT_FULL);
            }
            o++;
        }
    }
}

// L2-table insert of one sub-bucket's entries (the fallback of abandoned
// sub-buckets).
__global__ void __launch_bounds__(H_THREADS)
hash_insert_entries_kernel(const BEntry *ent, uint64_t n, int k, HSlot *tab, uint64_t tmask, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = (uint64_t)gridDim.x * (H_THREADS / 32);
    const uint64_t gw = blockIdx.x * (uint64_t)(H_THREADS / 32) + (threadIdx.x >> 5);
    const uint64_t mask = kmask(k);
    EStream s0, s1;
    s0.c.left = s1.c.left = 0;
    s0.next = gw * 64 + lane;
    s1.next = s0.next + 32;
    s0.step = s1.step = nw * 64;
    s0.last = s1.last = EMPTY_KEY;
    s0.run = s1.run = 0;
    for (;;) {
        bool f0, f1;
        uint64_t k0 = 0, k1 = 0;
        uint32_t c0 = 0, c1 = 0;
        bool h0 = s0.advance(ent, n, k, mask, f0, k0, c0);
        bool h1 = s1.advance(ent, n, k, mask, f1, k1, c1);
        if (!__any_sync(FULL, h0 || h1)) break;
        const uint64_t p0 = hash64(k0) & tmask, p1 = hash64(k1) & tmask;
        const unsigned long long v0 = f0 ? __ldcg(&tab[p0].key) : 0ull;
        const unsigned long long v1 = f1 ? __ldcg(&tab[p1].key) : 0ull;
        if (f0) table_add_from(tab, tmask, k0, c0, p0, v0, err);
        if (f1) table_add_from(tab, tmask, k1, c1, p1, v1, err);
    }
    if (s0.run) table_add(tab, tmask, s0.last, s0.run, err);
    if (s1.run) table_add(tab, tmask, s1.last, s1.run, err);
}

}  // namespace gkc
