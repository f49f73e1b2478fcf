// skmgen.cu -- phase 1: reads -> superkmers in per-partition device buffers.
//
// Replaces the reference's GPU_GenMinimizer / GPU_GenSKMOffs /
// GPU_ReadCompression / GPU_ExtractSKM chain (gpu_skmgen.cu:218-470) and the
// host round trip per 2000-read batch (gpu_skmgen.cu:504-718).
//
// Kernel 0 (tile_reads) finds, for every tile of 4096 bases, the read that
// holds the tile's first staged base (one binary search per tile, all tiles in
// parallel).
//
// Kernel 1 (find_superkmers) walks the concatenated read bases tile by tile.
// A CTA stages its tile's ASCII bytes in shared memory as 2-bit codes (16-byte
// vector loads) and a bitmap of read boundaries, and writes the tile's codes
// back to global memory packed 16 bases per word.  Each warp then walks a
// strip of the tile 32 positions at a time: lane l evaluates the canonical
// p-mer key at position c0+l; the minimum over the window of w = k-p+1 p-mers
// is a sparse-table doubling over a 64-wide register window (this chunk and
// the next) built from shuffles.  A superkmer starts at a valid k-mer that
// begins a read or whose key differs from its predecessor's, and ends at the
// next start or invalid position; both are ballots over the chunk.  The
// lanes where a superkmer ends build its record (begin, k-mer count, key,
// packing phase, trailing bases) in the warp's shared-memory queue; every 32
// queued records the warp's lanes emit one each into a per-CTA region and add
// it to per-partition byte/superkmer/k-mer counts in shared memory, which the
// CTA also writes out (cta_hist).  Emitting 32 at a time keeps every lane busy
// (a chunk ends about 3 superkmers): find took 11% less time than emitting
// each record in the chunk where it ends.
//
// cta_offsets_kernel lays out, from those counts, each CTA's contiguous range
// of every partition's byte and index buffers (CTA order: deterministic).
//
// Kernel 2 (scatter_superkmers) makes one pass over a CTA's records and writes
// every superkmer in the reference's 3-bases-per-byte format
// (cpu_funcs.cpp:200-250): a copy of the packed read whose first byte's
// header says 3-beg%3 valid bases and whose last byte's header says
// (end-1+k)%3, so the bytes are bit-identical to the reference's.
#include "gkc_device.cuh"

namespace gkc {

constexpr int P1_WARPS = 8;
constexpr int P1_THREADS = P1_WARPS * 32;
// chunks of 32 positions per warp strip: a strip pays a warm-up chunk and,
// usually, one chunk past its end for the superkmer still open there, so
// longer strips waste less (32 chunks: phase 1 5% faster than 16)
constexpr int P1_CHUNKS = 32;
constexpr int P1_STRIP = 32 * P1_CHUNKS;              // 1024 positions
constexpr int P1_TILE = P1_WARPS * P1_STRIP;          // 8192 positions per tile
constexpr int P1_TILE_WORDS = P1_TILE / 16;           // packed code words per tile
constexpr int P1_HALO = 512;                          // staged positions past the tile
constexpr int P1_STAGE = P1_TILE + 32 + P1_HALO + 128;  // staged positions (from tile-32)
constexpr int P1_CODE_WORDS = P1_STAGE / 16 + 2;      // 16 bases per word
constexpr int P1_BM_WORDS = P1_STAGE / 32 + 2;        // 32 positions per word

struct P1Params {
    const uint8_t *reads;      // concatenated ASCII bases
    const uint64_t *offs;      // n_reads+1 read offsets
    int64_t n_reads;
    uint64_t total;            // offs[n_reads]
    int k, p;
    uint32_t P;
    uint64_t pmod;             // fastmod multiplier of P
    const uint32_t *lut;       // canonical order table: lut[v] = min(rank(v), rank(rc(v))),
                               // or null for the default order
    int vec_ok;                // reads pointer is 16-byte aligned
    const int64_t *tile_read;  // [ntiles] read holding the tile's first staged base
    uint32_t *codes;           // [ntiles * P1_TILE_WORDS] packed 2-bit codes (out)
    SkmRecord *records;        // gridDim.x regions of `region_cap` records
    uint32_t region_cap;
    uint32_t *region_count;    // [gridDim.x]
    unsigned long long *part_bytes, *part_skms, *part_kmers;  // [P]
    uint32_t *cta_hist;        // [gridDim.x][2P]: this CTA's bytes, then superkmers, per partition
    uint32_t *err;
};

// x % d for 32-bit x from the precomputed m = 2^64 / d + 1 (Lemire, Kaser and
// Kurz, "Faster remainder by direct computation", 2019).
__device__ __host__ __forceinline__ uint64_t fastmod_m(uint32_t d) { return ~0ull / d + 1; }
__device__ __forceinline__ uint32_t fastmod(uint32_t x, uint64_t m, uint32_t d) {
    return (uint32_t)__umul64hi(m * x, d);
}

// Packs four 2-bit codes held one per byte (byte 0 first) into 8 bits with the
// first base in bits 7-6.
__device__ __forceinline__ uint32_t pack4(uint32_t c) {
    uint32_t r = __byte_perm(c, 0, 0x0123);
    return (r | (r >> 6) | (r >> 12) | (r >> 18)) & 0xFFu;
}

// Reverse complement of 16 packed codes (first base in the top bits).
__device__ __forceinline__ uint32_t rc16(uint32_t w) {
    uint32_t r = __brev(~w);
    return ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
}

// Index of the read containing position q (largest r with offs[r] <= q).
__device__ int64_t read_of(const uint64_t *offs, int64_t n_reads, uint64_t q) {
    int64_t lo = 0, hi = n_reads;  // offs[lo] <= q < offs[hi] (virtually)
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (offs[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void tile_reads_kernel(const uint64_t *offs, int64_t n_reads, uint64_t ntiles, int64_t *out) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ntiles;
         t += (uint64_t)gridDim.x * blockDim.x) {
        int64_t q = (int64_t)(t * P1_TILE) - 32;
        out[t] = read_of(offs, n_reads, q < 0 ? 0 : (uint64_t)q);
    }
}

// Default order: the p-mer's value, or the sentinel pmask when the
// "rapidgkc" filter rejects it (minimizer_filter.h:20).
__device__ __forceinline__ uint32_t pmer_key(uint32_t v, int p, uint32_t pmask) {
    return mm_valid(v, p) ? v : pmask;
}

// Minimizer key of k-mer q computed directly from global memory (used only
// for superkmers that run past the staged halo).
template <bool LUT>
__device__ uint32_t kmer_key_global(const P1Params &a, uint64_t q) {
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * a.p);
    uint32_t f = 0, best = 0xFFFFFFFFu;
    for (int j = 0; j < a.k; j++) {
        f = ((f << 2) | code1(a.reads[q + j])) & pmask;
        if (j >= a.p - 1) {
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
    return best;
}

// Read bases after a superkmer's last base x, capped at 3, from the boundary
// bits at x+1..x+3 (the terminal byte can hold three bases past x; the
// reference copies whatever the packed read has there).
__device__ __forceinline__ uint32_t tail_of(uint32_t b3) {
    return (b3 & 1) ? 0u : (b3 & 2) ? 1u : (b3 & 4) ? 2u : 3u;
}

constexpr int P1_RC_BASES = 16 * P1_CODE_WORDS;

struct P1Smem {
    uint32_t codes[P1_CODE_WORDS];   // staged 2-bit codes, position j at word j/16
    uint32_t rcodes[P1_CODE_WORDS + 1];  // complement codes in reverse: position j at
                                         // P1_RC_BASES-1-j (+1 word read past by the funnel)
    uint32_t bm[P1_BM_WORDS];
    uint32_t region_n;
    uint64_t rs0;  // start of the read containing the first staged position
};

__device__ __forceinline__ void emit_record(const P1Params &a, uint32_t *h, uint32_t slot, uint64_t pos,
                                            uint32_t len, uint32_t key, uint32_t phase, uint32_t tail) {
    uint32_t part = fastmod(~key, a.pmod, a.P);
    uint32_t nb = skm_nbytes(phase, len, a.k);
    if (len > IDX_MAX_LEN) atomicOr(a.err, ERR_SKM_TOO_LONG);
    atomicAdd(h + part, nb);
    atomicAdd(h + a.P + part, 1u);
    atomicAdd(h + 2 * a.P + part, len);
    if (slot < a.region_cap) {
        SkmRecord r;
        r.pos = rec_pack_pos(pos, phase, tail);
        r.len = len;
        r.key = key;
        a.records[(uint64_t)blockIdx.x * a.region_cap + slot] = r;
    } else {
        atomicOr(a.err, ERR_RECORD_OVERFLOW);
    }
}

// Adds a record built by a warp's lanes (pos already packed with phase and
// tail) to the CTA's region and partition counts.
__device__ __forceinline__ void emit_packed(const P1Params &a, uint32_t *h, uint32_t slot, const SkmRecord &r) {
    const uint32_t part = fastmod(~r.key, a.pmod, a.P);
    const uint32_t nb = skm_nbytes(rec_phase(r.pos), r.len, a.k);
    if (r.len > IDX_MAX_LEN) atomicOr(a.err, ERR_SKM_TOO_LONG);
    atomicAdd(h + part, nb);
    atomicAdd(h + a.P + part, 1u);
    atomicAdd(h + 2 * a.P + part, r.len);
    if (slot < a.region_cap) a.records[(uint64_t)blockIdx.x * a.region_cap + slot] = r;
    else atomicOr(a.err, ERR_RECORD_OVERFLOW);
}

// LOG = log2 of the largest power of two <= w (the doubling levels); LUT: the
// key of a position is a.lut[p-mer] (an order table, already canonical), else
// the default order over both strands.  KW: k > 32 (the reference's 128-bit
// LONGERKMER build, k <= 64): a k-mer's read-boundary test spans 64 bits, and
// LOG = 5 takes windows of 32 < w <= 62 p-mers over three chunks in
// registers: the 32-wide minimum of this chunk and of the next, combined at
// offset w - 32.
template <int LOG, bool LUT, bool KW>
__global__ void __launch_bounds__(P1_THREADS, 6)  // 6 CTAs (48 warps) per SM
find_superkmers_kernel(P1Params a) {
    extern __shared__ uint32_t hist[];  // [3P]: bytes, superkmers, k-mers per partition
    __shared__ P1Smem sm;
    // per warp: records found but not yet emitted; emitted 32 at a time, one
    // per lane (a chunk ends ~3 superkmers, so emitting them where they end
    // would run the emission with most lanes idle)
    __shared__ SkmRecord pend[P1_WARPS][64];
    static_assert(LOG < 5 || KW, "windows of more than 31 p-mers need k > 32");
    constexpr bool W3 = LOG == 5;  // three-chunk window
    constexpr int L2 = 1 << (W3 ? 4 : LOG);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = a.k, p = a.p, w = k - p + 1;
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * p);
    const unsigned lt_mask = (1u << lane) - 1;

    for (uint32_t i = threadIdx.x; i < 3 * a.P; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) sm.region_n = 0;

    const uint64_t ntiles = (a.total + P1_TILE - 1) / P1_TILE;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        const int64_t t0 = (int64_t)(tile * P1_TILE);
        const int64_t sbeg = t0 - 32;  // first staged position (multiple of 16)
        const int64_t r0 = a.tile_read[tile];
        // ---- stage 2-bit codes, forward and reverse complement ----
        for (int i = threadIdx.x; i < P1_CODE_WORDS; i += blockDim.x) {
            int64_t q = sbeg + 16 * (int64_t)i;
            uint32_t word = 0;
            if (q >= 0 && q + 16 <= (int64_t)a.total && a.vec_ok) {
                uint4 v = __ldg(reinterpret_cast<const uint4 *>(a.reads + q));
                word = (pack4(codes4(v.x)) << 24) | (pack4(codes4(v.y)) << 16) |
                       (pack4(codes4(v.z)) << 8) | pack4(codes4(v.w));
            } else {
                for (int t = 0; t < 16; t++) {
                    int64_t qq = q + t;
                    uint32_t c = (qq >= 0 && qq < (int64_t)a.total) ? code1(a.reads[qq]) : 0u;
                    word |= c << (30 - 2 * t);
                }
            }
            sm.codes[i] = word;
            if (!LUT) sm.rcodes[P1_CODE_WORDS - 1 - i] = rc16(word);
            if (i >= 2 && i < 2 + P1_TILE_WORDS) a.codes[tile * P1_TILE_WORDS + (i - 2)] = word;
        }
        for (int i = threadIdx.x; i < P1_BM_WORDS; i += blockDim.x) sm.bm[i] = 0;
        if (threadIdx.x == 0) sm.rs0 = a.offs[r0];
        __syncthreads();
        // ---- read-boundary bitmap: bit j <=> some offs[r] == sbeg + j ----
        {
            const int64_t send = sbeg + P1_STAGE;
            for (int64_t r = r0 + threadIdx.x; r <= a.n_reads; r += blockDim.x) {
                int64_t o = (int64_t)a.offs[r];
                if (o >= send) break;
                if (o >= sbeg) atomicOr(&sm.bm[(o - sbeg) >> 5], 1u << ((o - sbeg) & 31));
            }
        }
        __syncthreads();
        // ---- each warp walks its strip ----
        const int64_t strip0 = t0 + (int64_t)warp * P1_STRIP;
        if (strip0 >= (int64_t)a.total) continue;
        // staged-relative limits
        const int jstrip0 = (int)(strip0 - sbeg), jstrip1 = jstrip0 + P1_STRIP;
        const int jmin = sbeg < 0 ? (int)(-sbeg) : 0;                     // first position >= 0
        const int64_t jk64 = (int64_t)a.total - k - sbeg;                 // last valid k-mer start
        const int jmaxk = jk64 > (int64_t)P1_STAGE ? P1_STAGE : (int)jk64;
        const int64_t jt64 = (int64_t)a.total - sbeg;
        const int jtotal = jt64 > (int64_t)P1_STAGE ? P1_STAGE : (int)jt64;
        // last chunk start whose next chunk's p-mers and boundary bits are staged
        const int jlimit = P1_STAGE - (128 + k);
        const int shp = 32 - 2 * p;

        auto pk_at = [&](int j) -> uint32_t {  // canonical p-mer key at staged position j
            int i = j >> 4, o = j & 15;
            uint32_t f = __funnelshift_l(sm.codes[i + 1], sm.codes[i], 2 * o) >> shp;
            if (LUT) return __ldg(a.lut + f);  // the table is canonical: one read
            int rj = P1_RC_BASES - j - p;  // reverse-complement p-mer start in rcodes
            int ri = rj >> 4, ro = rj & 15;
            uint32_t r = __funnelshift_l(sm.rcodes[ri + 1], sm.rcodes[ri], 2 * ro) >> shp;
            uint32_t kf = pmer_key(f, p, pmask), kr = pmer_key(r, p, pmask);
            return kf < kr ? kf : kr;
        };
        auto bits_at = [&](int j) -> uint32_t {  // 32 boundary bits from staged position j
            return __funnelshift_r(sm.bm[j >> 5], sm.bm[(j >> 5) + 1], j & 31);
        };
        const uint32_t vmask = (1u << ((k - 1) & 31)) - 1;  // k <= 32
        const uint64_t vmask64 = (1ull << ((k - 1) & 63)) - 1;  // KW: k <= 64
        // minimum over [lane, lane + 32) of the 64 keys of two chunks (W3)
        auto win32 = [&](uint32_t ma, uint32_t mb) -> uint32_t {
#pragma unroll
            for (int x = 1; x < 32; x <<= 1) {
                const uint32_t t = __shfl_sync(FULL, lane >= x ? ma : mb, (lane + x) & 31);
                const uint32_t tb = __shfl_down_sync(FULL, mb, x);
                ma = min(ma, t);
                mb = min(mb, tb);
            }
            return ma;
        };
        // read start of the warm-up chunk's first position: the last boundary
        // bit at or before it, else the start of the read containing sbeg.
        int64_t rs;
        {
            const int j = jstrip0 - 32;  // multiple of 32
            int64_t found = -1;
            for (int base = (j >> 5); found < 0 && base >= 0; base -= 32) {
                int idx = base - lane;
                uint32_t v = idx >= 0 ? sm.bm[idx] : 0u;
                if (idx == (j >> 5)) v &= 1u;  // only position j itself in its own word
                unsigned bal = __ballot_sync(FULL, v != 0);
                if (bal) {
                    int src = __ffs(bal) - 1;  // lowest lane = highest word index
                    uint32_t vv = __shfl_sync(FULL, v, src);
                    found = sbeg + ((int64_t)(base - src) << 5) + (31 - __clz(vv));
                }
            }
            rs = found >= 0 ? found : (int64_t)sm.rs0;
        }

        // pipeline: A = p-mer keys of chunk c, B = of chunk c+1
        int cj = jstrip0 - 32;
        uint32_t A = pk_at(cj + lane), B = pk_at(cj + 32 + lane);
        // W3: C = keys of chunk c+2, F = 32-wide minima of chunk c
        uint32_t C = 0xFFFFFFFFu, F = 0xFFFFFFFFu;
        if (W3) {
            C = pk_at(cj + 64 + lane);
            F = win32(A, B);
        }
        uint32_t carried_key = 0xFFFFFFFFu;
        uint32_t npend = 0;  // records in pend[warp] (warp-uniform)
        SkmRecord *wp = pend[warp];
        // emits pend[warp][0, n), n <= 32, one per lane
        auto flush = [&](uint32_t n) {
            __syncwarp();
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&sm.region_n, n);
            base = __shfl_sync(FULL, base, 0);
            if ((uint32_t)lane < n) emit_packed(a, hist, base + lane, wp[lane]);
            __syncwarp();
        };
        bool open = false;  // a superkmer of this warp whose end is not found yet
        int64_t o_pos = 0;
        uint32_t o_key = 0, o_phase = 0;
        for (;;) {
            const bool warm = cj < jstrip0;
            const bool cont = cj >= jstrip1;
            if (cont && !open) break;
            if (cj > jlimit || cj >= jtotal) break;
            // ---- window minimum over w p-mers for the k-mer at cj+lane ----
            uint32_t key, Fn = 0xFFFFFFFFu;
            if (W3) {
                // [lane, lane + w) = [lane, lane + 32) u [lane + d, lane + d + 32)
                Fn = win32(B, C);
                const int d = w - 32;
                const uint32_t t = __shfl_sync(FULL, lane >= d ? F : Fn, (lane + d) & 31);
                key = min(F, t);
            } else {
                uint32_t ma = A, mb = B;
#pragma unroll
                for (int x = 1; x < L2; x <<= 1) {
                    uint32_t t = __shfl_sync(FULL, lane >= x ? ma : mb, (lane + x) & 31);
                    uint32_t tb = __shfl_down_sync(FULL, mb, x);
                    ma = min(ma, t);
                    mb = min(mb, tb);
                }
                key = ma;
                if (w > L2) {
                    int d = w - L2;
                    uint32_t t = __shfl_sync(FULL, lane >= d ? ma : mb, (lane + d) & 31);
                    key = min(ma, t);
                }
            }
            const int j = cj + lane;
            uint32_t prevkey = __shfl_up_sync(FULL, key, 1);
            if (lane == 0) prevkey = carried_key;
            const uint32_t bits = bits_at(j);
            bool valid;
            if (KW) {  // no read start at j+1 .. j+k-1 (k <= 64)
                const uint64_t b64 = bits | ((uint64_t)bits_at(j + 32) << 32);
                valid = j >= jmin && j <= jmaxk && ((b64 >> 1) & vmask64) == 0;
            } else {
                valid = j >= jmin && j <= jmaxk && ((bits >> 1) & vmask) == 0;
            }
            const bool isrs = j >= jmin && (bits & 1u);
            const bool start = valid && (isrs || key != prevkey);
            const unsigned RSB = __ballot_sync(FULL, isrs);
            const unsigned E = __ballot_sync(FULL, start || !valid);
            const unsigned S = __ballot_sync(FULL, start);

            if (!warm) {
                // a superkmer ends at each E lane whose nearest E bit below is
                // an owned start, or (none below) at the first E lane if one
                // is open from an earlier chunk
                const unsigned below = E & lt_mask;
                const int src = below ? 31 - __clz(below) : 0;
                const uint32_t skey = __shfl_sync(FULL, key, src);
                const bool isE = (E >> lane) & 1u;
                const bool emit = isE && (below ? (((S >> src) & 1u) && !cont) : open);
                const unsigned EM = __ballot_sync(FULL, emit);
                if (EM) {
                    if (emit) {
                        const int64_t e = sbeg + j;  // exclusive end (k-mer index)
                        int64_t b = o_pos;
                        uint32_t phase = o_phase, skey2 = o_key;
                        if (below) {
                            // read start at or before src: last boundary bit in
                            // the chunk up to src, else the carried one
                            const unsigned rsb = RSB & ((2u << src) - 1);
                            const int64_t rss = rsb ? sbeg + cj + 31 - __clz(rsb) : rs;
                            b = sbeg + cj + src;
                            phase = (uint32_t)(b - rss) % 3u;
                            skey2 = skey;
                        }
                        const uint32_t tail = tail_of(bits_at(j + k - 1) & 7u);
                        SkmRecord r;
                        r.pos = rec_pack_pos((uint64_t)b, phase, tail);
                        r.len = (uint32_t)(e - b);
                        r.key = skey2;
                        wp[npend + __popc(EM & lt_mask)] = r;
                    }
                    npend += __popc(EM);
                    if (npend >= 32) {  // emit the first 32, keep the rest
                        flush(32);
                        npend -= 32;
                        if ((uint32_t)lane < npend) wp[lane] = wp[32 + lane];
                        __syncwarp();
                    }
                }
                // the last start with no end in this chunk stays open
                if (E) {
                    const int last = 31 - __clz(E);
                    open = ((S >> last) & 1u) && !cont;
                    if (open) {
                        const unsigned rsb = RSB & ((2u << last) - 1);
                        const int64_t rsl = rsb ? sbeg + cj + 31 - __clz(rsb) : rs;
                        o_pos = sbeg + cj + last;
                        o_key = __shfl_sync(FULL, key, last);
                        o_phase = (uint32_t)(o_pos - rsl) % 3u;
                    }
                }
            }
            carried_key = __shfl_sync(FULL, key, 31);
            if (RSB) rs = sbeg + cj + 31 - __clz(RSB);
            // advance
            cj += 32;
            if (W3) {
                F = Fn;
                B = C;
                C = (cj + 95 < P1_STAGE - 16) ? pk_at(cj + 64 + lane) : 0xFFFFFFFFu;
            } else {
                A = B;
                B = (cj + 63 < P1_STAGE - 16) ? pk_at(cj + 32 + lane) : 0xFFFFFFFFu;
            }
        }
        if (npend) flush(npend);
        // superkmer running past the staged range: finish it from global memory
        if (open) {
            if (lane == 0) {
                const int64_t c0 = sbeg + cj;
                int64_t r = read_of(a.offs, a.n_reads, (uint64_t)o_pos);
                int64_t re = (int64_t)a.offs[r + 1];
                int64_t e = c0 > o_pos + 1 ? c0 : o_pos + 1;
                while (e + k <= re && kmer_key_global<LUT>(a, (uint64_t)e) == o_key) e++;
                int64_t after = re - (e + k - 1);
                uint32_t tail = after >= 3 ? 3 : (uint32_t)after;
                uint32_t slot = atomicAdd(&sm.region_n, 1u);
                emit_record(a, hist, slot, (uint64_t)o_pos, (uint32_t)(e - o_pos), o_key, o_phase, tail);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    uint32_t *ch = a.cta_hist + (uint64_t)blockIdx.x * 2 * a.P;
    for (uint32_t i = threadIdx.x; i < a.P; i += blockDim.x) {
        ch[i] = hist[i];
        ch[a.P + i] = hist[a.P + i];
        if (hist[a.P + i]) {
            atomicAdd(a.part_bytes + i, (unsigned long long)hist[i]);
            atomicAdd(a.part_skms + i, (unsigned long long)hist[a.P + i]);
            atomicAdd(a.part_kmers + i, (unsigned long long)hist[2 * a.P + i]);
        }
    }
    if (threadIdx.x == 0) a.region_count[blockIdx.x] = sm.region_n;
}

// Per-CTA base offsets in every partition: CTA c's range of partition p
// starts after the bytes (superkmers) of CTAs 0..c-1 in p.  One CTA per
// partition: each thread sums a contiguous run of CTAs, a block scan orders
// the runs, and the thread writes its run's bases (CTA order: deterministic).
constexpr int CO_THREADS = 256;
__global__ void __launch_bounds__(CO_THREADS) cta_offsets_kernel(const uint32_t *cta_hist, uint32_t ncta, uint32_t P,
                                                                  const unsigned long long *part_byte_off,
                                                                  const unsigned long long *part_skm_off,
                                                                  unsigned long long *cta_base, const uint32_t *flags) {
    __shared__ unsigned long long ws[CO_THREADS / 32];
    if (*flags & (ERR_RECORD_OVERFLOW | ERR_CAPACITY)) return;  // the batch is redone (uniform over the grid)
    const uint32_t p = blockIdx.x;
    const uint32_t per = (ncta + CO_THREADS - 1) / CO_THREADS;
    const uint32_t c0 = threadIdx.x * per, c1 = c0 + per < ncta ? c0 + per : ncta;
    unsigned long long b = 0, s = 0, tb, ts;
    for (uint32_t c = c0; c < c1; c++) {
        const uint64_t o = (uint64_t)c * 2 * P;
        b += cta_hist[o + p];
        s += cta_hist[o + P + p];
    }
    b = part_byte_off[p] + block_exclusive_scan<CO_THREADS>(b, &tb, ws);
    s = part_skm_off[p] + block_exclusive_scan<CO_THREADS>(s, &ts, ws);
    for (uint32_t c = c0; c < c1; c++) {
        const uint64_t o = (uint64_t)c * 2 * P;
        cta_base[o + p] = b;
        cta_base[o + P + p] = s;
        b += cta_hist[o + p];
        s += cta_hist[o + P + p];
    }
}

// Offsets of a batch's read set relative to its first read (device copy of
// a slice of the caller's offsets).
__global__ void rebase_offsets_kernel(uint64_t *offs, uint64_t n, uint64_t base) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        offs[i] -= base;
}

// Batch cuts of device-resident reads: cut j (0 < j < ncut) is the last read
// boundary at or below j * bb bases, found by binary search over the offsets
// (offs[0] == 0); cut 0 is read 0 and cut ncut is n_reads.  cut_idx[j] = read
// index, cut_off[j] = offs[that read].
__global__ void batch_cuts_kernel(const uint64_t *__restrict__ offs, uint64_t n_reads, uint64_t bb, uint32_t ncut,
                                  uint64_t *cut_idx, uint64_t *cut_off) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > ncut) return;
    uint64_t r;
    if (j == 0) {
        r = 0;
    } else if (j == ncut) {
        r = n_reads;
    } else {
        const uint64_t target = (uint64_t)j * bb;
        uint64_t lo = 0, hi = n_reads;  // offs[lo] <= target holds (offs[0] == 0)
        while (lo < hi) {
            const uint64_t mid = (lo + hi + 1) >> 1;
            if (offs[mid] <= target) lo = mid; else hi = mid - 1;
        }
        r = lo;
    }
    cut_idx[j] = r;
    cut_off[j] = offs[r];
}

// A batch's store chunk layout from its partition totals (hist: bytes,
// superkmers, k-mers per partition): exclusive scans into byte_off / skm_off
// [P+1], k-mers copied out.  Raises ERR_CAPACITY when the chunk's preallocated
// capacity is too small (cta_offsets and scatter then write nothing and the
// host redoes the batch).  One CTA of PO_THREADS.
constexpr int PO_THREADS = 1024;

__global__ void __launch_bounds__(PO_THREADS)
part_offsets_kernel(const unsigned long long *hist, uint32_t P, uint64_t byte_cap, uint64_t skm_cap,
                    unsigned long long *byte_off, unsigned long long *skm_off, unsigned long long *kmers,
                    uint32_t *flags) {
    __shared__ unsigned long long ws[PO_THREADS / 32];
    const uint32_t per = (P + PO_THREADS - 1) / PO_THREADS, p0 = threadIdx.x * per;
    unsigned long long sb = 0, ss = 0;
    for (uint32_t p = p0; p < p0 + per && p < P; p++) {
        sb += hist[p];
        ss += hist[P + p];
        kmers[p] = hist[2 * P + p];
    }
    unsigned long long tb, ts;
    unsigned long long ob = block_exclusive_scan<PO_THREADS>(sb, &tb, ws);
    unsigned long long os = block_exclusive_scan<PO_THREADS>(ss, &ts, ws);
    for (uint32_t p = p0; p < p0 + per && p < P; p++) {
        byte_off[p] = ob;
        skm_off[p] = os;
        ob += hist[p];
        os += hist[P + p];
    }
    if (threadIdx.x == 0) {
        byte_off[P] = tb;
        skm_off[P] = ts;
        if (tb > byte_cap || ts > skm_cap) atomicOr(flags, ERR_CAPACITY);
    }
}

// ---------------------------------------------------------------------------
// Kernel 2: scatter records into per-partition byte and index buffers.
struct P2Params {
    const uint32_t *codes;     // packed 2-bit codes of the batch (16 per word)
    const SkmRecord *records;
    uint32_t region_cap;
    const uint32_t *region_count;
    int k;
    uint32_t P;
    uint64_t pmod;
    const unsigned long long *part_byte_off;  // [P] partition start in `bytes`
    const unsigned long long *cta_base;       // [gridDim.x][2P] this CTA's first byte, superkmer per partition
    const uint32_t *flags;                    // the batch's error flags: nothing is written after an overflow
    uint8_t *bytes;
    uint64_t *idx;
    uint32_t *keys;  // minimizer key of each superkmer, indexed like idx
};

// One thread per record at a time; 1024-thread CTAs timed faster than
// 256 x 6 or 512 x 3 with their register caps.
constexpr int P2_THREADS = 1024;

__global__ void __launch_bounds__(P2_THREADS)
scatter_superkmers_kernel(P2Params a) {
    extern __shared__ unsigned long long sbase[];  // [2P] CTA bases in each partition
    uint32_t *lcnt = reinterpret_cast<uint32_t *>(sbase + 2 * a.P);  // [2P] CTA-local cursors
    if (*a.flags & (ERR_RECORD_OVERFLOW | ERR_CAPACITY)) return;  // the batch is redone
    const uint32_t n = a.region_count[blockIdx.x] < a.region_cap ? a.region_count[blockIdx.x] : a.region_cap;
    const SkmRecord *rec = a.records + (uint64_t)blockIdx.x * a.region_cap;
    // this CTA's ranges, laid out by cta_offsets_kernel from the find kernel's
    // per-CTA counts: one pass over the records
    const unsigned long long *cb = a.cta_base + (uint64_t)blockIdx.x * 2 * a.P;
    for (uint32_t i = threadIdx.x; i < 2 * a.P; i += blockDim.x) {
        sbase[i] = cb[i];
        lcnt[i] = 0;
    }
    __syncthreads();
    // Warps take 32 records at a time.  Each lane sets up its own record
    // (destination, code slot, headers); then the warp writes the records'
    // destination words cooperatively, one aligned 4-byte word per lane per
    // step (no lane waits for a longer superkmer, and consecutive lanes
    // write consecutive words).
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = blockDim.x >> 5;
    for (uint32_t base = (threadIdx.x >> 5) * 32; base < n; base += nwarps * 32) {
        const uint32_t i = base + lane;
        const bool has = i < n;
        uint64_t dst = 0, pos = 0;
        uint32_t nb = 0, rlim = 0, hdr = 0, nw = 0;
        if (has) {
            const SkmRecord r = rec[i];
            const uint32_t part = fastmod(~r.key, a.pmod, a.P);
            const uint32_t phase = rec_phase(r.pos), tail = rec_tail(r.pos);
            nb = skm_nbytes(phase, r.len, a.k);
            const uint32_t ob = atomicAdd(&lcnt[part], nb);
            const uint32_t os = atomicAdd(&lcnt[a.P + part], 1u);
            const uint64_t pbase = sbase[part] - a.part_byte_off[part];  // this CTA's range in the partition
            dst = reinterpret_cast<uint64_t>(a.bytes + sbase[part] + ob);
            pos = rec_base(r.pos) - phase;              // first code slot of the first byte
            rlim = phase + r.len + (uint32_t)a.k - 1 + tail;  // read bases used, from pos
            hdr = (3 - phase) | (((phase + r.len + (uint32_t)a.k - 1) % 3) << 2);  // first, last byte headers
            nw = (uint32_t)((((dst + nb + 3) & ~3ull) - (dst & ~3ull)) >> 2);
            a.idx[sbase[a.P + part] + os] = idx_pack(pbase + ob, r.len);
            a.keys[sbase[a.P + part] + os] = r.key;
        }
        uint32_t incl = nw;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31), excl = incl - nw;
        for (uint32_t c0 = 0; c0 < total; c0 += 32) {
            const uint32_t gi = c0 + lane;
            int own = 0;  // the last lane whose first word index is <= gi
#pragma unroll
            for (int st = 16; st; st >>= 1) {
                const int cand = own + st;
                if (__shfl_sync(FULL, excl, cand) <= gi) own = cand;
            }
            const uint32_t s = gi - __shfl_sync(FULL, excl, own);
            const uint64_t odst = __shfl_sync(FULL, dst, own), opos = __shfl_sync(FULL, pos, own);
            const uint32_t onb = __shfl_sync(FULL, nb, own), olim = __shfl_sync(FULL, rlim, own);
            const uint32_t ohdr = __shfl_sync(FULL, hdr, own);
            if (gi >= total) continue;
            const uint64_t A = (odst & ~3ull) + 4ull * s;    // this lane's destination word
            const int b0 = (int)((int64_t)A - (int64_t)odst);  // superkmer byte at A (may be < 0)
            auto codes_at = [&](uint64_t q) -> uint64_t {   // base q in bits 63-62, >= 17 bases
                const uint64_t wi = q >> 4;
                return (((uint64_t)__ldg(a.codes + wi) << 32) | __ldg(a.codes + wi + 1)) << (2 * (uint32_t)(q & 15));
            };
            if (b0 >= 1 && b0 + 4 < (int)onb) {
                // interior: 12 bases -> 4 bytes of 6 code bits + header 3 (little-endian)
                const uint32_t x = (uint32_t)(codes_at(opos + 3ull * (uint32_t)b0) >> 40);
                *reinterpret_cast<uint32_t *>(A) = (x >> 18) | (((x >> 12) & 63u) << 8) | (((x >> 6) & 63u) << 16) |
                                                   ((x & 63u) << 24) | 0xC0C0C0C0u;
            } else {
                // first or last word: byte by byte, only the superkmer's bytes
                uint32_t word = 0, nvalid = 0;
                for (int j = 0; j < 4; j++) {
                    const int bb = b0 + j;
                    if (bb < 0 || bb >= (int)onb) continue;
                    const uint32_t q = 3u * (uint32_t)bb;  // slot of byte bb, from opos
                    uint32_t v = (uint32_t)(codes_at(opos + q) >> 58), h = 3;
                    if (bb == (int)onb - 1) {
                        const uint32_t keep = olim > q ? (olim - q < 3 ? olim - q : 3u) : 0u;
                        v &= ~((1u << (6 - 2 * keep)) - 1) & 63u;
                        h = ohdr >> 2;
                    } else if (bb == 0) {
                        h = ohdr & 3;
                    }
                    word |= (v | (h << 6)) << (8 * j);
                    nvalid++;
                }
                if (nvalid == 4) {
                    *reinterpret_cast<uint32_t *>(A) = word;
                } else {
                    for (int j = 0; j < 4; j++) {
                        const int bb = b0 + j;
                        if (bb >= 0 && bb < (int)onb) reinterpret_cast<uint8_t *>(A)[j] = (uint8_t)(word >> (8 * j));
                    }
                }
            }
        }
    }
}

}  // namespace gkc
