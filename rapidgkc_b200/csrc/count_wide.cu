// count_wide.cu -- phase 2, the sub-bucket hash counter for k-mers of 33 to
// 64 bases: u128 keys, the values of the reference's LONGERKMER build
// (types.h:34-35, unsigned __int128 T_kmer; first base in the most
// significant position, masked to 2k bits, canonical min(x, revcomp(x)),
// gpu_kmercounting.cu:63-74).  The reference counts these with its sort path
// only; here they take the same sub-bucket scheme as the 64-bit counter
// (count_bucket.cu), with four differences:
//   * a lane's quad of k-mers is decoded from a 72-base window (24 bytes,
//     three 48-bit fields) instead of 48 bases;
//   * the shared-memory table holds 16-byte keys, which no atomic claims in
//     one step: a slot is claimed through a 32-bit state word (empty ->
//     being written -> ready) and its key is compared only once ready;
//     4096 slots in 96 KB (8192 in the second pass), so sub-buckets are
//     sized at about 4k instances;
//   * a sub-bucket's quads are spread over the whole CTA (cta_quads): at
//     large k a sub-bucket holds few, long superkmers;
//   * sub-buckets that overflow, and heavy ones, are not split into records:
//     they are counted in pieces by a hash of the key (wide_piece), each
//     piece one CTA that decodes the whole sub-bucket and inserts its own
//     keys; a piece that overflows splits in two, and pieces past the decode
//     limit have their instances extracted into the key buffer and counted by
//     the 128-bit radix sort (count_onesweep.cu).
// Included by engine.cu after count_bucket.cu.

namespace gkc {

// Reverse complement of a k-mer in the low 2k bits of a u128 (k <= 64).
__device__ __forceinline__ u128 rc128(u128 v, int k) {
    const uint64_t lo = (uint64_t)v, hi = (uint64_t)(v >> 64);
    // the 128 bits reversed: the words swap places and each is reversed;
    // then the two bits of every base swap back
    uint64_t rl = __brevll(~hi), rh = __brevll(~lo);
    rl = ((rl >> 1) & 0x5555555555555555ull) | ((rl & 0x5555555555555555ull) << 1);
    rh = ((rh >> 1) & 0x5555555555555555ull) | ((rh & 0x5555555555555555ull) << 1);
    return (((u128)rh << 64) | rl) >> (128 - 2 * k);
}

__device__ __forceinline__ u128 kmask128(int k) { return k >= 64 ? ~(u128)0 : (((u128)1 << (2 * k)) - 1); }

// quad_runs (count_bucket.cu) for 33 <= k <= 64: calls f(key, run) for the
// canonical k-mers of quad qi of a superkmer (first byte p, pad bases of
// padding, len k-mers), equal consecutive k-mers merged into runs.  The
// quad's first k-mer is taken from a 72-base window: 24 bytes from four
// aligned 8-byte loads (store buffers carry 32 bytes of padding) as three
// 48-bit fields A (slots 0-23), B (24-47) and C (48-71).  f must not use
// warp collectives.
template <class F>
__device__ __forceinline__ void quad_runs_wide(const uint8_t *p, uint32_t pad, uint32_t len, uint32_t qi, int k,
                                               u128 mask, F &&f) {
    const uint32_t j0 = KQ * qi;
    const uint32_t nk = len - j0 < (uint32_t)KQ ? len - j0 : (uint32_t)KQ;
    const uint32_t u = pad + j0, bi = u / 3, s = u - 3 * bi;
    const uintptr_t addr = (uintptr_t)p + bi;
    const uint64_t *w = reinterpret_cast<const uint64_t *>(addr & ~(uintptr_t)7);
    const uint32_t sh = 8 * (uint32_t)(addr & 7);
    const uint64_t w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
    auto fs = [&](uint64_t x, uint64_t y) -> uint64_t { return sh ? (x >> sh) | (y << (64 - sh)) : x; };
    const uint64_t A = pack6x8(fs(w0, w1)), B = pack6x8(fs(w1, w2)), C = pack6x8(fs(w2, w3));
    // the 144-bit A:B:C shifted right by d, low 128 bits (6 <= d <= 78 here)
    auto shr144 = [&](uint32_t d) -> u128 {
        u128 r = (u128)A << (96 - d);
        r |= d <= 48 ? ((u128)B << (48 - d)) : (u128)(B >> (d - 48));
        if (d < 48) r |= (u128)(C >> d);
        return r;
    };
    const uint32_t d = 144 - 2 * (s + (uint32_t)k);
    u128 x = shr144(d) & mask;
    // the quad's KQ-1 entering bases (slots s+k .. s+k+KQ-2), the last in bits 1-0
    const uint32_t nxt = (uint32_t)shr144(d - 2 * (KQ - 1));
    u128 r = rc128(x, k);
    u128 last = x < r ? x : r;
    uint32_t run = 1;
#pragma unroll
    for (uint32_t t = 1; t < (uint32_t)KQ; t++) {
        if (t >= nk) break;
        const uint32_t bt = (nxt >> (2 * (KQ - 1 - t))) & 3u;  // the entering base
        x = ((x << 2) | bt) & mask;
        r = (r >> 2) | ((u128)(3u - bt) << (2 * k - 2));
        const u128 key = x < r ? x : r;
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

// warp_kmer_runs (count_bucket.cu) for 33 <= k <= 64: calls f(key, run) for
// every canonical k-mer of the entries ent[b .. b+32) of a warp, by
// quad_runs_wide.  Must be called by the whole warp; f is called by single
// lanes and must not use warp collectives.
template <class F>
__device__ __forceinline__ void warp_kmer_runs_wide(const BEntry *ent, uint64_t b, uint64_t end, int k, u128 mask,
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
        quad_runs_wide(reinterpret_cast<const uint8_t *>(po), opad, olen, qi, k, mask, f);
    }
}

// ---------------------------------------------------------------------------
// Shared-memory table of 16-byte keys.  Slot state: 0 empty, 1 being
// written, 2 ready.  A thread claims an empty slot by compare-and-swap of its
// state, writes the key and its count, and publishes the slot as ready;
// another thread that meets a slot being written waits for it (a bounded
// wait: past it the table is abandoned like a full one).
struct WideTable {
    unsigned long long *klo, *khi;
    uint32_t *st, *cnt;
};

template <int TS>
__device__ __forceinline__ WideTable wide_table(unsigned long long *smem) {
    WideTable t;
    t.klo = smem;
    t.khi = smem + TS;
    t.st = reinterpret_cast<uint32_t *>(smem + 2 * TS);
    t.cnt = t.st + TS;
    return t;
}

constexpr uint32_t WIDE_MAX_WAIT = 1u << 20;  // polls of a slot being written before giving up

// The piece of n (n >= 1) that a key belongs to when a sub-bucket is counted
// in n pieces by key hash: [0, n), from the top 32 bits of a mix of the key
// that is independent of the table's slot hash.  Piece r of n is exactly
// pieces 2r and 2r + 1 of 2n, so a piece that overflows splits in two.
__device__ __forceinline__ uint32_t wide_piece(u128 key, uint32_t n) {
    uint64_t x = (uint64_t)key ^ ((uint64_t)(key >> 64) * 0xC2B2AE3D27D4EB4Full);
    x ^= x >> 33;
    x *= 0xFF51AFD7ED558CCDull;
    x ^= x >> 29;
    return (uint32_t)(((x >> 32) * (uint64_t)n) >> 32);
}

template <int TS>
__device__ __forceinline__ void wide_add(const WideTable &t, volatile uint32_t *over, u128 key, uint32_t c) {
    constexpr int LOG = __builtin_ctz(TS);
    const uint64_t lo = (uint64_t)key, hi = (uint64_t)(key >> 64);
    uint32_t h = (uint32_t)(((lo ^ (hi * 0x9E3779B97F4A7C15ull)) * 0xD6E8FEB86659FD93ull) >> (64 - LOG));
    volatile uint32_t *vst = t.st;
    volatile unsigned long long *vlo = t.klo, *vhi = t.khi;
    uint32_t waits = 0;
    for (uint32_t pr = 0; pr < SM_MAX_PROBE;) {
        const uint32_t s = vst[h];
        if (s == 2u) {
            if (vlo[h] == lo && vhi[h] == hi) {
                atomicAdd(&t.cnt[h], c);
                return;
            }
            h = (h + 1) & (TS - 1);
            pr++;
        } else if (s == 0u) {
            if (atomicCAS(&t.st[h], 0u, 1u) == 0u) {
                vlo[h] = lo;
                vhi[h] = hi;
                atomicAdd(&t.cnt[h], c);
                __threadfence_block();
                atomicExch(&t.st[h], 2u);
                return;
            }
            // another thread claimed it first: look at the slot again
        } else if (++waits > WIDE_MAX_WAIT) {
            *over = 1;
            return;
        }
    }
    *over = 1;
}

// bucket_count_kernel (count_bucket.cu) with 16-byte keys: one CTA counts a
// sub-bucket (b0 + CTA, or ids[CTA]) in a TS-slot table and writes its k-mers
// with count in [cmin, cmax] as two u64 words each (low word first); a
// sub-bucket whose table overflows, or of more than heavy_kmers instances, is
// listed in failed instead.
template <int TS>
__global__ void __launch_bounds__(BC_THREADS)
bucket_count_wide_kernel(BCountParams a) {
    extern __shared__ unsigned long long wt_smem[];
    const WideTable t = wide_table<TS>(wt_smem);
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t over;
    __shared__ unsigned long long base_s;
    __shared__ QStage qs;
    const uint32_t b = a.ids ? a.ids[blockIdx.x] : a.b0 + blockIdx.x;
    const uint32_t pr = a.piece ? a.piece[2 * blockIdx.x] : 0u, pn = a.piece ? a.piece[2 * blockIdx.x + 1] : 1u;
    const uint32_t fail_id = a.piece ? blockIdx.x : b;
    const uint64_t e0 = a.bucket_off[b], e1 = a.bucket_off[b + 1];
    if (e0 == e1) return;
    if (a.bucket_kmers[b] > a.heavy_kmers) {
        if (threadIdx.x == 0) {
            const uint32_t i = atomicAdd(a.failed, 1u);
            a.failed[1 + i] = fail_id;
        }
        return;
    }
    for (int x = threadIdx.x; x < TS; x += BC_THREADS) {
        t.st[x] = 0;
        t.cnt[x] = 0;
    }
    if (threadIdx.x == 0) over = 0;
    __syncthreads();
    const u128 mask = kmask128(a.k);
    cta_quads<BC_THREADS>(a.entries, e0, e1, qs, ws, &over, [&](const uint8_t *p, uint32_t pad, uint32_t len,
                                                                uint32_t qi) {
        quad_runs_wide(p, pad, len, qi, a.k, mask, [&](u128 key, uint32_t run) {
            if (pn == 1u || wide_piece(key, pn) == pr) wide_add<TS>(t, &over, key, run);
        });
    });
    if (over) {
        if (threadIdx.x == 0) {
            const uint32_t i = atomicAdd(a.failed, 1u);
            a.failed[1 + i] = fail_id;
        }
        return;
    }
    // collect: thread i owns slots i, i + NT, ...
    constexpr int PER = TS / BC_THREADS;
    uint32_t keep = 0, occ = 0;
#pragma unroll
    for (int x = 0; x < PER; x++) {
        const int sl = x * BC_THREADS + threadIdx.x;
        if (t.st[sl] == 2u) {
            occ++;
            keep += (t.cnt[sl] >= a.cmin && t.cnt[sl] <= a.cmax);
        }
    }
    uint32_t tot, occ_tot;
    const uint32_t pre = block_exclusive_scan<BC_THREADS>(keep, &tot, ws);
    block_exclusive_scan<BC_THREADS>(occ, &occ_tot, ws);
    if (threadIdx.x == 0) {
        base_s = tot ? atomicAdd(a.out_cursor, (unsigned long long)tot) : 0ull;
        if (occ_tot) atomicAdd(a.distinct, (unsigned long long)occ_tot);
    }
    __syncthreads();
    uint64_t o = base_s + pre;
#pragma unroll
    for (int x = 0; x < PER; x++) {
        const int sl = x * BC_THREADS + threadIdx.x;
        if (t.st[sl] == 2u && t.cnt[sl] >= a.cmin && t.cnt[sl] <= a.cmax) {
            if (o < a.out_cap) {
                a.out_k[2 * o] = t.klo[sl];
                a.out_k[2 * o + 1] = t.khi[sl];
                a.out_c[o] = t.cnt[sl];
            } else {
                atomicOr(a.err, ERR_OUTPUT_FULL);
            }
            o++;
        }
    }
}

// The k-mer instances of listed pieces of sub-buckets written to keys, one
// key per instance (runs expanded), in any order: the radix sort that counts
// them does not care.  Work item i covers the entries [range[2i],
// range[2i+1]) of one sub-bucket and keeps the keys of piece piece[2i] of
// piece[2i+1] (wide_piece); a large sub-bucket is cut into many items, so
// that one low-complexity run does not hold a single CTA.  Its keys go to
// keys from key_off[i] on; with keys null, the item's instances are only
// counted, into counts[i].
struct BExtractParams {
    const BEntry *entries;
    const unsigned long long *range;
    const uint32_t *piece;
    const unsigned long long *key_off;
    int k;
    u128 *keys;
    unsigned long long *counts;
};

__global__ void __launch_bounds__(BC_THREADS) bucket_extract_wide_kernel(BExtractParams a) {
    __shared__ QStage qs;
    __shared__ uint32_t ws[BC_THREADS / 32];
    __shared__ volatile uint32_t never;  // cta_quads' stop flag: extraction does not stop
    __shared__ unsigned long long cur;
    const uint32_t pr = a.piece[2 * blockIdx.x], pn = a.piece[2 * blockIdx.x + 1];
    const uint64_t e0 = a.range[2 * blockIdx.x], e1 = a.range[2 * blockIdx.x + 1];
    if (threadIdx.x == 0) {
        cur = 0;
        never = 0;
    }
    __syncthreads();
    const bool write = a.keys != nullptr;
    u128 *out = write ? a.keys + a.key_off[blockIdx.x] : nullptr;
    const u128 mask = kmask128(a.k);
    uint32_t mine = 0;  // count mode: this thread's instances
    cta_quads<BC_THREADS>(a.entries, e0, e1, qs, ws, &never, [&](const uint8_t *p, uint32_t pad, uint32_t len,
                                                                  uint32_t qi) {
        quad_runs_wide(p, pad, len, qi, a.k, mask, [&](u128 key, uint32_t run) {
            if (pn != 1u && wide_piece(key, pn) != pr) return;
            if (!write) {
                mine += run;
                return;
            }
            const unsigned long long o = atomicAdd(&cur, (unsigned long long)run);
            for (uint32_t r = 0; r < run; r++) out[o + r] = key;
        });
    });
    if (!write) {
        if (mine) atomicAdd(&cur, (unsigned long long)mine);
        __syncthreads();
        if (threadIdx.x == 0) a.counts[blockIdx.x] = cur;
    }
}

}  // namespace gkc
