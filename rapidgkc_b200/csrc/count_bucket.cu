// count_bucket.cu -- phase 2, shared-memory hash counter over sub-buckets.
//
// Every partition p of the store is split into 2^s_p sub-buckets by a hash of
// the superkmers' minimizer keys.  A canonical k-mer has one minimizer, so all
// its occurrences land in one sub-bucket, and a sub-bucket can be counted on
// its own.  s_p is chosen from partition p's k-mer count (about 8k instances
// per sub-bucket), so that a sub-bucket's distinct k-mers fit an
// open-addressing table in one CTA's shared memory however skewed the
// partitions are:
//   split    over all superkmers of all store chunks: a histogram of
//            superkmers and k-mers per sub-bucket (shared-memory aggregated),
//            a scan, then a scatter of 16-byte entries {first byte address,
//            k-mer count} into sub-bucket order;
//   count    one CTA per sub-bucket: warps take groups of 32 superkmers from
//            a shared-memory counter (groups differ in k-mers, so a fixed
//            round robin left warps idle at the barrier), decode them 32 quads
//            of up to four consecutive k-mers at a time (warp_kmer_runs
//            below), merge equal neighbouring k-mers into runs, and add the
//            runs to a shared-memory table with
//            shared-memory atomics; then the k-mers whose count lies in
//            [cmin, cmax] are written with one global atomic per CTA.  A
//            sub-bucket whose distinct k-mers outgrow the table is abandoned
//            and listed; the host re-splits those by k-mer hash
//            (count_records.cu), so the result does not depend on skew.  A
//            sub-bucket of more than heavy_kmers instances (one minimizer of
//            a low-complexity run can hold millions) is listed without being
//            counted: one CTA would take as long as the rest of the launch,
//            while the record split spreads it over many CTAs.
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

// ---------------------------------------------------------------------------
// Warp-cooperative superkmer decoding.
//
// Superkmer bytes hold three 2-bit bases in their low six bits, first base
// highest; a superkmer's first byte holds 3 - (its header) bases of padding
// before its first base.  The j-th k-mer of a superkmer therefore starts at
// base slot u = pad + j, i.e. byte u/3, slot u%3.

// Six-bit fields of eight bytes (byte 0 first) packed into 48 bits, byte 0's
// bases highest.
__device__ __forceinline__ uint64_t pack6x8(uint64_t le) {
    uint64_t x = ((uint64_t)__byte_perm((uint32_t)le, 0, 0x0123) << 32) | __byte_perm((uint32_t)(le >> 32), 0, 0x0123);
    x &= 0x3F3F3F3F3F3F3F3Full;
    x = ((x >> 2) & 0x0FC00FC00FC00FC0ull) | (x & 0x003F003F003F003Full);
    x = ((x >> 4) & 0x00FFF00000FFF000ull) | (x & 0x00000FFF00000FFFull);
    x = ((x >> 8) & 0x0000FFFFFF000000ull) | (x & 0x0000000000FFFFFFull);
    return x;
}

constexpr int KQ = 4;  // k-mers per lane per step (a quad)

// Calls f(key, run) for the canonical k-mers of quad qi of a superkmer (first
// byte p, pad bases of padding, len k-mers), equal consecutive k-mers merged
// into runs.  A quad is up to KQ consecutive k-mers.  Its first k-mer is
// decoded from a 48-base window (16 bytes from three aligned 8-byte loads;
// store buffers carry 32 bytes of padding); the others roll in one base each,
// forward and reverse complement.  f must not use warp collectives.
template <class F>
__device__ __forceinline__ void quad_runs(const uint8_t *p, uint32_t pad, uint32_t len, uint32_t qi, int k,
                                          uint64_t mask, F &&f) {
    const uint32_t j0 = KQ * qi;
    const uint32_t nk = len - j0 < (uint32_t)KQ ? len - j0 : (uint32_t)KQ;
    const uint32_t u = pad + j0, bi = u / 3, s = u - 3 * bi;
    const uintptr_t addr = (uintptr_t)p + bi;
    const uint64_t *w = reinterpret_cast<const uint64_t *>(addr & ~(uintptr_t)7);
    const uint32_t sh = 8 * (uint32_t)(addr & 7);
    const uint64_t w0 = w[0], w1 = w[1], w2 = w[2];
    const uint64_t lo = sh ? (w0 >> sh) | (w1 << (64 - sh)) : w0;  // bytes 0..7
    const uint64_t hi = sh ? (w1 >> sh) | (w2 << (64 - sh)) : w1;  // bytes 8..15
    // 48 bases, slot 0 first: A holds slots 0-23 (48 bits), B slots 24-47.
    // The 96-bit value A:B shifted right by d is, in its low 64 bits (all
    // that the masks below keep), (A << (48 - d)) | (B >> d) for d <= 48
    // and A >> (d - 48) beyond: 64-bit shifts, no 128-bit one.
    const uint64_t A = pack6x8(lo), B = pack6x8(hi);
    auto shr96 = [&](uint32_t dd) -> uint64_t { return dd <= 48 ? (A << (48 - dd)) | (B >> dd) : A >> (dd - 48); };
    const uint32_t d = 96 - 2 * (s + (uint32_t)k);  // 30..34 for k = 31
    uint64_t x = shr96(d) & mask;
    // the quad's KQ-1 entering bases (slots s+k .. s+k+KQ-2), the last in bits 1-0
    const uint32_t nxt = (uint32_t)shr96(d - 2 * (KQ - 1));
    uint64_t r = rc64(x, k);
    uint64_t last = x < r ? x : r;
    uint32_t run = 1;
#pragma unroll
    for (uint32_t t = 1; t < (uint32_t)KQ; t++) {
        if (t >= nk) break;
        const uint32_t bt = (nxt >> (2 * (KQ - 1 - t))) & 3u;  // the entering base
        x = ((x << 2) | bt) & mask;
        r = (r >> 2) | ((uint64_t)(3u - bt) << (2 * k - 2));
        const uint64_t key = x < r ? x : r;
        if (key == last) {
            run++;
        } else {
            f(last, run);
            last = key;
            run = 1;
        }
    }
    f(last, run);
}

// Calls f(key, run) for every canonical k-mer of the entries ent[b .. b+32)
// of a warp (entry b + lane exists when b + lane < end), equal consecutive
// k-mers merged into runs (quad_runs).  A warp step gives each lane one quad
// (a shuffle prefix sum and owner search over the 32 entries).  Must be
// called by the whole warp; f is called by single lanes.
template <class F>
__device__ __forceinline__ void warp_kmer_runs(const BEntry *ent, uint64_t b, uint64_t end, int k, uint64_t mask,
                                               F &&f) {
    const int lane = threadIdx.x & 31;
    const bool has = b + lane < end;
    BEntry en;
    en.ptr = nullptr;
    en.len = 0;
    if (has) en = ent[b + lane];
    const uint32_t pad = has ? 3u - (en.ptr[0] >> 6) : 0u;
    const uint32_t nq = (en.len + KQ - 1) / KQ;
    uint32_t incl = nq;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, incl, d);
        if (lane >= d) incl += y;
    }
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    const uint32_t excl = incl - nq;
    const uint64_t pv = reinterpret_cast<uint64_t>(en.ptr);
    for (uint32_t c0 = 0; c0 < total; c0 += 32) {
        const uint32_t g = c0 + lane;
        int own = 0;  // the last lane whose first quad index is <= g
#pragma unroll
        for (int st = 16; st; st >>= 1) {
            const int cand = own + st;
            if (__shfl_sync(FULL, excl, cand) <= g) own = cand;
        }
        const uint32_t qi = g - __shfl_sync(FULL, excl, own);
        const uint64_t po = __shfl_sync(FULL, pv, own);
        const uint32_t opad = __shfl_sync(FULL, pad, own), olen = __shfl_sync(FULL, en.len, own);
        if (g >= total) continue;
        quad_runs(reinterpret_cast<const uint8_t *>(po), opad, olen, qi, k, mask, f);
    }
}

// ---------------------------------------------------------------------------
// split
constexpr int BS_THREADS = 512;
constexpr int BS_PER_CTA = 8192;   // superkmers per split CTA
constexpr int BS_MAX_PARTS = 4;    // partitions a split CTA aggregates in shared memory
constexpr int BS_SLOTS = 4096;     // shared-memory sub-bucket counters per split CTA
constexpr int BS_LOG_LIMIT = 16;   // at most 65536 sub-buckets per partition
constexpr size_t BS_SMEM = (size_t)BS_SLOTS * 12;  // dynamic shared memory

// One store chunk's part of a split launch.
struct BSChunk {
    const uint64_t *idx;                       // chunk superkmer index (partition-ordered)
    const uint32_t *keys;                      // chunk superkmer minimizer keys
    const uint8_t *bytes;                      // chunk bytes
    uint64_t i_begin, n_skm;                   // superkmer index range [i_begin, n_skm)
    const unsigned long long *part_skm_off;    // [P+1]
    const unsigned long long *part_byte_off;   // [P]
    uint32_t cta0;                             // the chunk's first CTA in the launch
};

struct BSplitParams {
    const BSChunk *chunks;                     // ascending cta0; one launch covers them all
    uint32_t nchunks;
    uint32_t P;
    const uint32_t *part_slog;                 // [P] s_p: partition p has 2^s_p sub-buckets
    const uint32_t *part_bbase;                // [P] index of partition p's first sub-bucket
    uint32_t *bucket_skms;                     // [NB] superkmers per sub-bucket (pass 0)
    unsigned long long *bucket_kmers;          // [NB] k-mers per sub-bucket (pass 0)
    unsigned long long *bucket_cursor;         // [NB] next free entry (pass 1)
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

// Pass 0 counts superkmers and k-mers per sub-bucket; pass 1 scatters
// entries.  One launch covers every chunk of a group (chunk of a CTA: the last
// with cta0 <= blockIdx.x).  A CTA covers BS_PER_CTA consecutive superkmers of
// its chunk, which span few
// partitions: its first BS_MAX_PARTS partitions get consecutive ranges of
// BS_SLOTS shared-memory counters, 2^s_p each, while they fit, so their
// sub-buckets cost one global atomic per CTA; any other superkmer goes
// straight to global atomics.
__global__ void __launch_bounds__(BS_THREADS)
bucket_split_kernel(BSplitParams a) {
    extern __shared__ unsigned long long bs_smem[];
    unsigned long long *base = bs_smem;                                // pass 0: k-mers; pass 1: reserved block
    uint32_t *cnt = reinterpret_cast<uint32_t *>(bs_smem + BS_SLOTS);  // superkmers
    __shared__ uint32_t soff[BS_MAX_PARTS + 1];  // shared range of partition pf + q: [soff[q], soff[q + 1])
    __shared__ uint32_t p_first_s, nq_s;
    uint32_t lo = 0, hi = a.nchunks;  // chunks[lo].cta0 <= blockIdx.x < chunks[hi].cta0
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.chunks[mid].cta0 <= blockIdx.x) lo = mid; else hi = mid;
    }
    const BSChunk ch = a.chunks[lo];
    const uint64_t i0 = ch.i_begin + (blockIdx.x - ch.cta0) * (uint64_t)BS_PER_CTA;
    if (i0 >= ch.n_skm) return;
    const uint64_t i1 = min(ch.n_skm, i0 + BS_PER_CTA);
    if (threadIdx.x == 0) {
        const uint32_t pf = part_of_index(ch.part_skm_off, a.P, i0);
        uint32_t q = 0, o = 0;
        soff[0] = 0;
        while (q < BS_MAX_PARTS && pf + q < a.P && o + (1u << a.part_slog[pf + q]) <= BS_SLOTS) {
            o += 1u << a.part_slog[pf + q];
            soff[++q] = o;
        }
        p_first_s = pf;
        nq_s = q;
    }
    for (int t = threadIdx.x; t < BS_SLOTS; t += BS_THREADS) cnt[t] = 0, base[t] = 0;
    __syncthreads();
    const uint32_t pf = p_first_s, nq = nq_s;
    auto part = [&](uint64_t i) {
        return (i < ch.part_skm_off[pf + 1]) ? pf : part_of_index(ch.part_skm_off, a.P, i);
    };
    // global sub-bucket of shared counter t (t < soff[nq])
    auto global_of = [&](uint32_t t) {
        uint32_t q = 0;
        while (t >= soff[q + 1]) q++;
        return a.part_bbase[pf + q] + (t - soff[q]);
    };
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += BS_THREADS) {
        const uint32_t p = part(i);
        const uint32_t b = bucket_of(ch.keys[i], (int)__ldg(a.part_slog + p));
        if (p - pf < nq) {
            const uint32_t t = soff[p - pf] + b;
            atomicAdd(&cnt[t], 1u);
            if (a.pass == 0) atomicAdd(&base[t], (unsigned long long)idx_len(ch.idx[i]));
        } else if (a.pass == 0) {
            const uint32_t g = __ldg(a.part_bbase + p) + b;
            atomicAdd(a.bucket_skms + g, 1u);
            atomicAdd(a.bucket_kmers + g, (unsigned long long)idx_len(ch.idx[i]));
        }
    }
    __syncthreads();
    const uint32_t ns = soff[nq];
    if (a.pass == 0) {
        for (uint32_t t = threadIdx.x; t < ns; t += BS_THREADS)
            if (cnt[t]) {
                const uint32_t g = global_of(t);
                atomicAdd(a.bucket_skms + g, cnt[t]);
                atomicAdd(a.bucket_kmers + g, base[t]);
            }
        return;
    }
    // pass 1: reserve each shared sub-bucket's block, then write entries
    for (uint32_t t = threadIdx.x; t < ns; t += BS_THREADS) {
        if (cnt[t]) base[t] = atomicAdd(a.bucket_cursor + global_of(t), (unsigned long long)cnt[t]);
        cnt[t] = 0;
    }
    __syncthreads();
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += BS_THREADS) {
        const uint32_t p = part(i);
        const uint32_t b = bucket_of(ch.keys[i], (int)__ldg(a.part_slog + p));
        uint64_t slot;
        if (p - pf < nq) {
            const uint32_t t = soff[p - pf] + b;
            slot = base[t] + atomicAdd(&cnt[t], 1u);
        } else {
            slot = atomicAdd(a.bucket_cursor + __ldg(a.part_bbase + p) + b, 1ull);
        }
        const uint64_t e = ch.idx[i];
        BEntry en;
        en.ptr = ch.bytes + ch.part_byte_off[p] + idx_off(e);
        en.len = idx_len(e);
        en.pad = 0;
        a.entries[slot] = en;
    }
}

// ---------------------------------------------------------------------------
// shared-memory counting
constexpr int BC_THREADS = 512;

struct BCountParams {
    const BEntry *entries;
    const uint64_t *bucket_off;   // [nb+1] entry ranges of the sub-buckets
    const unsigned long long *bucket_kmers;  // [nb] k-mer instances per sub-bucket
    uint64_t heavy_kmers;         // larger sub-buckets are listed, not counted
    uint32_t b0;                  // first sub-bucket of this launch
    const uint32_t *ids;          // or, when not null: CTA i counts sub-bucket ids[i]
    int k;
    uint32_t cmin, cmax;
    uint64_t *out_k;
    uint32_t *out_c;
    unsigned long long *out_cursor;
    uint64_t out_cap;
    unsigned long long *distinct;
    uint32_t *failed;             // [1 + nb]: count, then the abandoned sub-buckets
    uint32_t *err;
    // 128-bit counter only: when not null, CTA i counts piece (piece[2i] of
    // piece[2i+1]) of sub-bucket ids[i] (wide_piece) and lists i, not the
    // sub-bucket, when it fails
    const uint32_t *piece = nullptr;
};

// Quads of a sub-bucket spread evenly over a CTA (the 128-bit counter,
// count_wide.cu).  The entries are taken in chunks of QS_CH (one per thread):
// a block scan of their quad counts gives each entry its first quad, and
// warps claim the chunk's 32-quad steps one at a time from a shared counter.
// A lane finds its quad's entry in a window of 32 entries from the owner of
// the step's first quad (two ballots over the chunk; every entry has at least
// one quad, so the window covers the step).  At large k a sub-bucket of about
// 4k instances holds only about 150 superkmers, so groups of 32 entries per
// warp (bucket_count_kernel) left most warps at the barrier: 96.8 -> 40.0 ms
// for the 128-bit counter on 3 Gbp at k = 63.  With the short superkmers of
// k <= 32 the groups balance well enough, and their cheaper steps win
// (29.8 vs 32.7 ms on 3 Gbp at k = 31).
constexpr int QS_CH = BC_THREADS;
constexpr int QS_STRIDE = QS_CH / 32;
static_assert(QS_CH == 32 * QS_STRIDE && QS_STRIDE <= 32, "chunk search in two ballots");
constexpr uint32_t QS_LEN_MASK = 0x3FFFFFFFu;  // ql: k-mers in bits 0-29, padding bases in 30-31

struct QStage {
    uint32_t qx[QS_CH + 32];  // first quad of each entry of the chunk; UINT32_MAX past its end
    const uint8_t *qp[QS_CH];  // first byte of each entry
    uint32_t ql[QS_CH];       // k-mers | padding << 30
    uint32_t next;            // the next step to claim
};

// Calls q(p, pad, len, qi) for every quad qi of every entry of ent[e0, e1)
// (entries of fewer than 2^30 k-mers).  Must be called by the whole CTA of
// NT == QS_CH threads; it starts and ends with a barrier's worth of
// synchronisation (the block scan and a final __syncthreads), so shared state
// written before it is visible to q and everything q wrote is visible after
// it.  A warp stops taking steps once *over is set.
template <int NT, class QF>
__device__ __forceinline__ void cta_quads(const BEntry *ent, uint64_t e0, uint64_t e1, QStage &qs, uint32_t *ws,
                                          volatile uint32_t *over, QF &&q) {
    static_assert(NT == QS_CH, "one entry per thread per chunk");
    constexpr int NW = NT / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint64_t c0 = e0; c0 < e1; c0 += QS_CH) {
        const uint32_t n = (uint32_t)(e1 - c0 < (uint64_t)QS_CH ? e1 - c0 : (uint64_t)QS_CH);
        uint32_t nq = 0;
        if (threadIdx.x < n) {
            const BEntry en = ent[c0 + threadIdx.x];
            const uint32_t pad = 3u - (en.ptr[0] >> 6);
            nq = en.len ? (en.len + KQ - 1) / KQ : 1u;  // an empty entry keeps one (skipped) quad
            qs.qp[threadIdx.x] = en.ptr;
            qs.ql[threadIdx.x] = (en.len & QS_LEN_MASK) | (pad << 30);
        }
        uint32_t nquads;
        const uint32_t ex = block_exclusive_scan<NT>(nq, &nquads, ws);
        qs.qx[threadIdx.x] = threadIdx.x < n ? ex : 0xFFFFFFFFu;
        if (threadIdx.x < 32) qs.qx[QS_CH + threadIdx.x] = 0xFFFFFFFFu;
        if (threadIdx.x == 0) qs.next = NW;
        __syncthreads();
        const uint32_t S = (nquads + 31) / 32;
        // steps are claimed one at a time from a shared counter (warp w starts at step w)
        uint32_t s = warp;
        while (s < S) {
            if (__any_sync(FULL, *over != 0)) break;  // a warp vote: the warp leaves together
            // c: the owner of quad 32 s, the last entry whose first quad is <= 32 s
            // (qx[0] = 0, so both ballots have lane 0 set)
            const uint32_t t0 = 32 * s;
            uint32_t m = __ballot_sync(FULL, qs.qx[lane * QS_STRIDE] <= t0);
            uint32_t c = (31 - __clz(m)) * QS_STRIDE;
            m = __ballot_sync(FULL, lane < QS_STRIDE && qs.qx[c + lane] <= t0);
            c += 31 - __clz(m);
            const uint32_t v = qs.qx[c + lane];  // c < n, so c + lane < QS_CH + 32
            const uint32_t g = t0 + lane;
            int own = 0;  // the last window entry whose first quad is <= g
#pragma unroll
            for (int st = 16; st; st >>= 1) {
                const int cand = own + st;
                if (__shfl_sync(FULL, v, cand) <= g) own = cand;
            }
            const uint32_t first = __shfl_sync(FULL, v, own);
            uint32_t nx = 0;
            if (lane == 0) nx = atomicAdd(&qs.next, 1u);
            if (g < nquads) {
                const uint32_t l = qs.ql[c + own];
                if (l & QS_LEN_MASK) q(qs.qp[c + own], l >> 30, l & QS_LEN_MASK, g - first);
            }
            s = __shfl_sync(FULL, nx, 0);
        }
        __syncthreads();
    }
}

// Shared-memory table insert (multiplicative hash on the top bits).  A probe
// sequence longer than SM_MAX_PROBE (the table is nearly full) raises *over
// instead of inserting; the caller then abandons the table.
constexpr uint32_t SM_MAX_PROBE = 128;

// TS need not be a power of two: the slot is the top 32 bits of the hash
// scaled to [0, TS) (for TS = 2^L, its top L bits), and probes wrap at TS.
template <int TS>
__device__ __forceinline__ void smem_add(unsigned long long *tk, uint32_t *tc, volatile uint32_t *over,
                                         uint64_t key, uint32_t c) {
    uint32_t h = (uint32_t)((((key * 0x9E3779B97F4A7C15ull) >> 32) * (uint64_t)TS) >> 32);
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
        h = h + 1 == (uint32_t)TS ? 0u : h + 1;
    }
    *over = 1;
}

// Writes the table's k-mers with count in [cmin, cmax] (one global atomic per
// CTA), adds its distinct keys to *distinct.  Called by the whole CTA.
template <int TS, int NT>
__device__ __forceinline__ void smem_collect(const unsigned long long *tk, const uint32_t *tc, uint32_t cmin,
                                             uint32_t cmax, uint64_t *out_k, uint32_t *out_c,
                                             unsigned long long *out_cursor, uint64_t out_cap,
                                             unsigned long long *distinct, uint32_t *err, uint32_t *ws,
                                             unsigned long long *base_s) {
    // thread i owns slots i, i + NT, i + 2 NT, ...: conflict-free loads (the
    // output order inside a table does not matter)
    static_assert(TS % NT == 0, "whole slots per thread");
    constexpr int PER = TS / NT;
    uint32_t keep = 0, occ = 0;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        int s = t * NT + threadIdx.x;
        if (tk[s] != EMPTY_KEY) {
            occ++;
            keep += (tc[s] >= cmin && tc[s] <= cmax);
        }
    }
    uint32_t tot, occ_tot;
    uint32_t pre = block_exclusive_scan<NT>(keep, &tot, ws);
    block_exclusive_scan<NT>(occ, &occ_tot, ws);
    if (threadIdx.x == 0) {
        *base_s = tot ? atomicAdd(out_cursor, (unsigned long long)tot) : 0ull;
        if (occ_tot) atomicAdd(distinct, (unsigned long long)occ_tot);
    }
    __syncthreads();
    uint64_t o = *base_s + pre;
#pragma unroll
    for (int t = 0; t < PER; t++) {
        int s = t * NT + threadIdx.x;
        if (tk[s] != EMPTY_KEY && tc[s] >= cmin && tc[s] <= cmax) {
            if (o < out_cap) {
                out_k[o] = tk[s];
                out_c[o] = tc[s];
            } else {
                atomicOr(err, ERR_OUTPUT_FULL);
            }
            o++;
        }
    }
}

// CTAs per SM that a table of TS slots (12 bytes each) allows in 228 KB of
// shared memory, as the launch bound's minimum.
constexpr int bc_min_ctas(int ts) { return ts <= 4096 ? 4 : ts <= 6144 ? 3 : ts <= 8192 ? 2 : 1; }

template <int TS>
__global__ void __launch_bounds__(BC_THREADS, bc_min_ctas(TS))
bucket_count_kernel(BCountParams a) {
    extern __shared__ unsigned long long tk[];             // [TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + TS);  // [TS] counts
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    const uint32_t b = a.ids ? a.ids[blockIdx.x] : a.b0 + blockIdx.x;
    const uint64_t e0 = a.bucket_off[b], e1 = a.bucket_off[b + 1];
    if (e0 == e1) return;
    if (a.bucket_kmers[b] > a.heavy_kmers) {
        if (threadIdx.x == 0) {
            uint32_t i = atomicAdd(a.failed, 1u);
            a.failed[1 + i] = b;
        }
        return;
    }
    for (int t = threadIdx.x; t < TS; t += BC_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    __shared__ uint32_t next_grp;  // the next group of 32 entries to take
    if (threadIdx.x == 0) {
        over = 0;
        next_grp = BC_THREADS / 32;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t mask = kmask(a.k);
    for (uint64_t bb = e0 + (uint64_t)warp * 32; bb < e1;) {
        if (__any_sync(FULL, over != 0)) break;  // a warp vote: the warp leaves together
        warp_kmer_runs(a.entries, bb, e1, a.k, mask,
                       [&](uint64_t key, uint32_t run) { smem_add<TS>(tk, tc, &over, key, run); });
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(&next_grp, 1u);
        bb = e0 + 32ull * __shfl_sync(FULL, g, 0);
    }
    __syncthreads();
    if (over) {
        if (threadIdx.x == 0) {
            uint32_t i = atomicAdd(a.failed, 1u);
            a.failed[1 + i] = b;
        }
        return;
    }
    smem_collect<TS, BC_THREADS>(tk, tc, a.cmin, a.cmax, a.out_k, a.out_c, a.out_cursor, a.out_cap, a.distinct,
                                 a.err, ws, &base_s);
}

// smem_add that also lists each slot it claims in tl (nl counts them), so
// that the table can be collected and cleared by its occupied slots alone.
template <int TS>
__device__ __forceinline__ void smem_add_listed(unsigned long long *tk, uint32_t *tc, uint16_t *tl, uint32_t *nl,
                                                volatile uint32_t *over, uint64_t key, uint32_t c) {
    uint32_t h = (uint32_t)((((key * 0x9E3779B97F4A7C15ull) >> 32) * (uint64_t)TS) >> 32);
    for (uint32_t pr = 0; pr < SM_MAX_PROBE; pr++) {
        unsigned long long cur = tk[h];
        if (cur == key) {
            atomicAdd(&tc[h], c);
            return;
        }
        if (cur == EMPTY_KEY) {
            unsigned long long old = atomicCAS(&tk[h], (unsigned long long)EMPTY_KEY, (unsigned long long)key);
            if (old == EMPTY_KEY) {
                tl[atomicAdd(nl, 1u)] = (uint16_t)h;
                atomicAdd(&tc[h], c);
                return;
            }
            if (old == key) {
                atomicAdd(&tc[h], c);
                return;
            }
        }
        h = h + 1 == (uint32_t)TS ? 0u : h + 1;
    }
    *over = 1;
}

// The first pass of the sub-bucket counter as a persistent kernel: each CTA
// clears its table once, then takes sub-buckets b0 + i (i from the counter
// *next, below nb) one after another.  A sub-bucket is counted as in
// bucket_count_kernel, but every claimed slot is listed, and the table is
// collected and cleared through that list: a sub-bucket of 8k instances holds
// about 1-2k distinct k-mers, so clearing and scanning all 8192 slots for
// each of a million sub-buckets cost more than its decode (11.5 of the
// 50 ms the launch took on 6 Gbp).  TS <= 65536 (u16 slot list).
constexpr int BC_TAIL = 256;  // entries at a sub-bucket's end handed out in groups of 16

template <int TS>
__global__ void __launch_bounds__(BC_THREADS, bc_min_ctas(TS))
bucket_count_persistent_kernel(BCountParams a, uint32_t nb, uint32_t *next) {
    static_assert(TS <= 65536, "u16 slot list");
    extern __shared__ unsigned long long tk[];             // [TS] keys
    uint32_t *tc = reinterpret_cast<uint32_t *>(tk + TS);  // [TS] counts
    uint16_t *tl = reinterpret_cast<uint16_t *>(tc + TS);  // [TS] claimed slots
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    __shared__ uint32_t next_grp, cur_i, nl;
    for (int t = threadIdx.x; t < TS; t += BC_THREADS) {
        tk[t] = EMPTY_KEY;
        tc[t] = 0;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t mask = kmask(a.k);
    for (;;) {
        if (threadIdx.x == 0) {
            cur_i = atomicAdd(next, 1u);
            over = 0;
            nl = 0;
            next_grp = BC_THREADS / 32;
        }
        __syncthreads();  // also orders the previous sub-bucket's clearing before this one's inserts
        const uint32_t i = cur_i;
        if (i >= nb) break;
        const uint32_t b = a.b0 + i;
        const uint64_t e0 = a.bucket_off[b], e1 = a.bucket_off[b + 1];
        if (e0 != e1 && a.bucket_kmers[b] > a.heavy_kmers) {
            if (threadIdx.x == 0) {
                const uint32_t f = atomicAdd(a.failed, 1u);
                a.failed[1 + f] = b;
            }
        } else if (e0 != e1) {
            // group g: 32 entries, except the sub-bucket's last BC_TAIL entries,
            // which go in groups of 16 so that the warps finish close together
            const uint64_t E = e1 - e0, tail = E < (uint64_t)BC_TAIL ? E : (uint64_t)BC_TAIL;
            const uint64_t head = E - tail, nbig = (head + 31) / 32;
            for (uint64_t g = warp;;) {
                const uint64_t g0 = g < nbig ? 32 * g : head + 16 * (g - nbig);
                if (g0 >= E) break;
                const uint64_t g1 = g < nbig ? (32 * g + 32 < head ? 32 * g + 32 : head) : (g0 + 16 < E ? g0 + 16 : E);
                if (__any_sync(FULL, over != 0)) break;  // a warp vote: the warp leaves together
                warp_kmer_runs(a.entries, e0 + g0, e0 + g1, a.k, mask, [&](uint64_t key, uint32_t run) {
                    smem_add_listed<TS>(tk, tc, tl, &nl, &over, key, run);
                });
                uint32_t gn = 0;
                if (lane == 0) gn = atomicAdd(&next_grp, 1u);
                g = __shfl_sync(FULL, gn, 0);
            }
            __syncthreads();
            const uint32_t n = nl;  // <= TS: a slot is claimed once
            if (over) {
                if (threadIdx.x == 0) {
                    const uint32_t f = atomicAdd(a.failed, 1u);
                    a.failed[1 + f] = b;
                }
                for (uint32_t j = threadIdx.x; j < n; j += BC_THREADS) {
                    const uint32_t sl = tl[j];
                    tk[sl] = EMPTY_KEY;
                    tc[sl] = 0;
                }
            } else {
                // collect through the list (thread t takes entries t, t + NT, ...
                // in both loops, so its prefix offsets line up), clearing as it goes
                uint32_t keep = 0;
                for (uint32_t j = threadIdx.x; j < n; j += BC_THREADS) {
                    const uint32_t c = tc[tl[j]];
                    keep += (c >= a.cmin && c <= a.cmax);
                }
                uint32_t tot;
                const uint32_t pre = block_exclusive_scan<BC_THREADS>(keep, &tot, ws);
                if (threadIdx.x == 0) {
                    base_s = tot ? atomicAdd(a.out_cursor, (unsigned long long)tot) : 0ull;
                    if (n) atomicAdd(a.distinct, (unsigned long long)n);
                }
                __syncthreads();
                uint64_t o = base_s + pre;
                for (uint32_t j = threadIdx.x; j < n; j += BC_THREADS) {
                    const uint32_t sl = tl[j];
                    const uint32_t c = tc[sl];
                    if (c >= a.cmin && c <= a.cmax) {
                        if (o < a.out_cap) {
                            a.out_k[o] = tk[sl];
                            a.out_c[o] = c;
                        } else {
                            atomicOr(a.err, ERR_OUTPUT_FULL);
                        }
                        o++;
                    }
                    tk[sl] = EMPTY_KEY;
                    tc[sl] = 0;
                }
            }
        }
        __syncthreads();  // cur_i, nl and the list are rewritten at the top
    }
}

// L2-table insert of one sub-bucket's entries (hash_l2_only mode).
__global__ void __launch_bounds__(H_THREADS)
hash_insert_entries_kernel(const BEntry *ent, uint64_t n, int k, HSlot *tab, uint64_t tmask, uint32_t *err) {
    const uint64_t nw = (uint64_t)gridDim.x * (H_THREADS / 32);
    const uint64_t gw = blockIdx.x * (uint64_t)(H_THREADS / 32) + (threadIdx.x >> 5);
    const uint64_t mask = kmask(k);
    for (uint64_t bb = gw * 32; bb < n; bb += nw * 32) {
        warp_kmer_runs(ent, bb, n, k, mask, [&](uint64_t key, uint32_t run) { table_add(tab, tmask, key, run, err); });
    }
}

}  // namespace gkc
