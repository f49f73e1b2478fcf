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
// vector loads) and a bitmap of read boundaries, writes the tile's codes back
// to global memory packed 16 bases per word, and puts the p-mer key of every
// staged position in shared memory.  Each lane then owns 32 consecutive k-mer
// starts and works through them serially: the minimum over each window of
// w = k-p+1 keys from block suffix and prefix minima (van Herk / Gil-Werman),
// and 32-bit masks of valid k-mers, superkmer starts (a valid k-mer that
// begins a read or whose key differs from its predecessor's) and end events
// (a start or an invalid k-mer).  A superkmer ends at the next end event after
// its start, found in the lane's mask, the later lanes' (a suffix minimum over
// the warp), the later strips' (published per warp) or, past the tile, in the
// staged halo.  Each lane writes the records (begin, k-mer count, key, packing
// phase, trailing bases) of the superkmers that start in it into a per-CTA
// region and adds them to per-partition byte/superkmer/k-mer counts in shared
// memory, which the CTA also writes out (cta_hist).  Against one position per
// lane per step (a shuffle doubling for the window and ballots for the
// boundaries every 32 positions), this cuts the instructions per base about
// tenfold: the window, boundary and record work is done once per position
// instead of once per lane per step.
//
// cta_offsets_kernel lays out, from those counts, each CTA's contiguous range
// of every partition's byte and index buffers (CTA order: deterministic).
//
// Kernel 2 (scatter_superkmers) makes one pass over a CTA's records and writes
// every superkmer in the reference's 3-bases-per-byte format
// (cpu_funcs.cpp:200-250): a copy of the packed read whose first byte's
// header says 3-beg%3 valid bases and whose last byte's header says
// (end-1+k)%3, so the bytes are bit-identical to the reference's.
#include <type_traits>

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
    const uint8_t *reads;      // concatenated ASCII bases, or
    const uint32_t *packed;    // (when not null) the same bases as 2-bit codes, 16 to a word
                               // (first base highest: the words staged below); then they
                               // are also the batch's codes, and `codes` is not written
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

// 2-bit code of base q of the batch, from the ASCII or the packed words.
__device__ __forceinline__ uint32_t base_code(const P1Params &a, uint64_t q) {
    return a.packed ? (__ldg(a.packed + (q >> 4)) >> (30 - 2 * (uint32_t)(q & 15))) & 3u : code1(a.reads[q]);
}

// Minimizer key of k-mer q computed directly from global memory (used only
// for superkmers that run past the staged halo).
template <bool LUT>
__device__ uint32_t kmer_key_global(const P1Params &a, uint64_t q) {
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * a.p);
    uint32_t f = 0, best = 0xFFFFFFFFu;
    for (int j = 0; j < a.k; j++) {
        f = ((f << 2) | base_code(a, q + j)) & pmask;
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

// Skewed shared-memory index of staged position j: lane l of a warp reads
// positions 32 l + t in step t, and the skew puts them in 32 different banks.
__device__ __forceinline__ int p1_sk(int j) { return j + (j >> 5); }
constexpr int P1_NKEYS = P1_STAGE - 16;                 // staged positions with a p-mer key
constexpr int P1_KEY_SLOTS = P1_NKEYS + P1_NKEYS / 32 + 2;
constexpr int P1_INF = 0x7FFFFFFF;

// LUT: the key of a position is a.lut[p-mer] (an order table, already
// canonical), else the default order over both strands.  KW: k > 32 (the
// reference's 128-bit LONGERKMER build, k <= 64): read-boundary windows of up
// to 63 bits and minimizer windows of up to 62 p-mers.
//
// Per tile: (A) every staged position's p-mer key into shared memory; (B)
// lane l of warp w owns the 32 k-mer starts [32 l, 32 l + 32) of strip w and
// computes their window minima serially -- blocks of w keys from the lane's
// first position, suffix minima backwards, prefix minima forwards, window =
// min(suffix at its first key, prefix at its last key) (van Herk / Gil-Werman)
// -- then its superkmer starts and ends as 32-bit masks: valid (no read start
// inside the k-mer), start = valid and (read start or key change), end event =
// start or invalid.  Each start's end is the next end event: in the lane, in
// a later lane (a suffix minimum over lanes), in a later strip (published per
// warp), or past the tile (the owning warp scans the staged halo, then global
// memory).  Each lane then writes its records.
// Four CTAs per SM for k <= 32 (64 registers; a few bytes spill) hide the
// order table's L2 latency better than two (111 registers): 55.4 -> 43.7 ms
// per 6 Gbp; three for k > 32, whose wider windows spill more at 64.
template <bool LUT, bool KW>
__global__ void __launch_bounds__(P1_THREADS, KW ? 3 : 4)
find_superkmers_kernel(P1Params a) {
    extern __shared__ uint32_t hist[];  // [3P]: bytes, superkmers, k-mers per partition
    __shared__ P1Smem sm;
    __shared__ uint32_t skey[P1_KEY_SLOTS];  // keys, then (tile positions) window minima
    __shared__ int fe_warp[P1_WARPS];        // first end event of each strip (staged index)
    using BM = typename std::conditional<KW, u128, uint64_t>::type;
    constexpr int TMAX = KW ? 96 : 64;  // > the last local index the backward pass reads, for any w
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = a.k, p = a.p, w = k - p + 1;
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * p);
    const int shp = 32 - 2 * p;
    // blocks of w keys from the lane's local index 0 (its first k-mer's predecessor)
    BM bend = 0;  // bit t: local index t ends a block
    for (int t = w - 1; t < TMAX; t += w) bend |= (BM)1 << t;
    uint64_t bfirst = 0;  // bit i (1..32): local index i + w - 1 starts a block
    for (int i = 1; i < 33; i += w) bfirst |= 1ull << i;
    const int top = (32 / w + 1) * w - 1;  // end of the block that holds local index 32
    const uint32_t vmask = (1u << ((k - 1) & 31)) - 1;      // k <= 32
    const uint64_t vmask64 = (1ull << ((k - 1) & 63)) - 1;  // KW: k <= 64

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
            if (a.packed) {  // q is a multiple of 16: one word (0 past the batch's end)
                if (q >= 0 && q < (int64_t)a.total) word = __ldg(a.packed + (q >> 4));
            } else if (q >= 0 && q + 16 <= (int64_t)a.total && a.vec_ok) {
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
            if (!a.packed && i >= 2 && i < 2 + P1_TILE_WORDS) a.codes[tile * P1_TILE_WORDS + (i - 2)] = word;
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
        // ---- (A) the p-mer key of every staged position ----
        // (unrolled: the table reads of one thread are in flight together)
        constexpr int NA = (P1_NKEYS + P1_THREADS - 1) / P1_THREADS;
#pragma unroll
        for (int r = 0; r < NA; r++) {
            const int j = threadIdx.x + r * P1_THREADS;
            if (j < P1_NKEYS) skey[p1_sk(j)] = pk_at(j);
        }
        __syncthreads();

        // ---- (B) lane-serial window minima over the lane's 32 k-mer starts ----
        const int jstrip0 = 32 + warp * P1_STRIP;            // staged index of the strip's first k-mer
        const int jb = jstrip0 + 32 * lane;                  // the lane's first k-mer (multiple of 32)
        const int64_t q0 = sbeg + jb;
        const int64_t jk64 = (int64_t)a.total - k - sbeg;    // last valid k-mer start
        const int jmaxk = jk64 > (int64_t)P1_STAGE ? P1_STAGE : (int)jk64;
        uint32_t M[33];  // M[i]: minimum over local keys [i, i + w), the k-mer at jb - 1 + i
        {
            uint32_t suf = 0xFFFFFFFFu;
#pragma unroll
            for (int t = TMAX - 1; t >= 0; t--) {
                if (t <= top) {
                    const uint32_t kk = skey[p1_sk(jb - 1 + t)];
                    suf = ((bend >> t) & 1) ? kk : min(suf, kk);
                    if (t < 33) M[t] = suf;
                }
            }
            uint32_t pre = M[0];  // local keys [0, w) are block 0
#pragma unroll
            for (int i = 1; i < 33; i++) {
                const uint32_t kk = skey[p1_sk(jb + i + w - 2)];
                pre = ((bfirst >> i) & 1) ? kk : min(pre, kk);
                M[i] = min(M[i], pre);
            }
        }
        uint32_t D = 0;  // bit i: the key of k-mer jb + i differs from its predecessor's
#pragma unroll
        for (int i = 0; i < 32; i++) D |= (uint32_t)(M[i + 1] != M[i]) << i;
        // validity: no read start at jb + i + 1 .. jb + i + k - 1, and a k-mer inside the input
        const int wb = jb >> 5;
        const uint32_t RS = sm.bm[wb];  // read starts at jb .. jb + 31
        BM X;
        if (KW) {
            const u128 lo = (u128)sm.bm[wb] | ((u128)sm.bm[wb + 1] << 32) | ((u128)sm.bm[wb + 2] << 64) |
                            ((u128)sm.bm[wb + 3] << 96);
            X = (BM)(lo >> 1);
        } else {
            const uint64_t lo = (uint64_t)sm.bm[wb] | ((uint64_t)sm.bm[wb + 1] << 32);
            X = (BM)((lo >> 1) | ((uint64_t)sm.bm[wb + 2] << 63));
        }
        {  // X bit i = OR of read-start bits i .. i + k - 2 (from jb + 1)
            const int n = k - 1;
            int s = 1;
            while (2 * s <= n) {
                X |= X >> s;
                s *= 2;
            }
            if (n > s) X |= X >> (n - s);
        }
        const int lim = jmaxk - jb;
        uint32_t V = ~(uint32_t)X;
        V &= lim >= 31 ? 0xFFFFFFFFu : lim < 0 ? 0u : ((2u << lim) - 1);
        const uint32_t S = V & (RS | D);
        const uint32_t E = S | ~V;
        // the first end event after this lane: a suffix minimum over lanes
        const int fe = E ? jb + __ffs(E) - 1 : P1_INF;
        int sfx = fe;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_down_sync(FULL, sfx, d);
            if (lane + d < 32) sfx = min(sfx, o);
        }
        int after = __shfl_down_sync(FULL, sfx, 1);
        if (lane == 31) after = P1_INF;
        if (lane == 0) fe_warp[warp] = sfx;
        // last read start before the strip (its base may lie before the staged range)
        int64_t rs_before;
        {
            int64_t found = -1;
            for (int base = (jstrip0 >> 5) - 1; found < 0 && base >= 0; base -= 32) {
                const int idx = base - lane;
                const uint32_t v = idx >= 0 ? sm.bm[idx] : 0u;
                const unsigned bal = __ballot_sync(FULL, v != 0);
                if (bal) {
                    const int src = __ffs(bal) - 1;  // lowest lane = highest word index
                    const uint32_t vv = __shfl_sync(FULL, v, src);
                    found = sbeg + ((int64_t)(base - src) << 5) + (31 - __clz(vv));
                }
            }
            const int64_t rs_strip = found >= 0 ? found : (int64_t)sm.rs0;
            // ... then before each lane: the last read start of the lanes below
            int64_t incl = RS ? q0 + 31 - __clz(RS) : -1;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int64_t o = __shfl_up_sync(FULL, incl, d);
                if (lane >= d) incl = max(incl, o);
            }
            rs_before = __shfl_up_sync(FULL, incl, 1);
            if (lane == 0) rs_before = -1;
            rs_before = max(rs_before, rs_strip);
        }
        __syncthreads();  // keys read by every lane; strip end events published
#pragma unroll
        for (int i = 0; i < 32; i++) skey[p1_sk(jb + i)] = M[i + 1];  // window minimum of k-mer jb + i
        __syncwarp();
        // ---- records: each lane writes those that start in it ----
        const uint32_t cnt = __popc(S);
        uint32_t pre = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(FULL, pre, d);
            if (lane >= d) pre += o;
        }
        const uint32_t wtot = __shfl_sync(FULL, pre, 31);
        uint32_t base = 0;
        if (lane == 0 && wtot) base = atomicAdd(&sm.region_n, wtot);
        uint32_t slot = __shfl_sync(FULL, base, 0) + pre - cnt;
        bool open = false;  // this lane's last superkmer runs past the tile
        int64_t o_pos = 0;
        uint32_t o_key = 0, o_phase = 0, o_slot = 0;
        uint32_t s = S;
        while (s) {
            const int i = __ffs(s) - 1;
            s &= s - 1;
            const int bj = jb + i;
            const uint32_t above = i == 31 ? 0u : (E >> (i + 1));
            int ej;
            if (above) {
                ej = bj + __ffs(above);
            } else if (after != P1_INF) {
                ej = after;
            } else {
                ej = P1_INF;
                for (int w2 = warp + 1; w2 < P1_WARPS; w2++)
                    if (fe_warp[w2] != P1_INF) {
                        ej = fe_warp[w2];
                        break;
                    }
            }
            const uint32_t key = skey[p1_sk(bj)];
            const int64_t b = sbeg + bj;
            const uint32_t rsb = RS & (i == 31 ? 0xFFFFFFFFu : ((2u << i) - 1));
            const int64_t rs = rsb ? q0 + 31 - __clz(rsb) : rs_before;
            const uint32_t phase = (uint32_t)(b - rs) % 3u;
            if (ej == P1_INF) {  // ends past the tile: the warp finds its end below
                open = true;
                o_pos = b;
                o_key = key;
                o_phase = phase;
                o_slot = slot++;
                continue;
            }
            SkmRecord r;
            r.pos = rec_pack_pos((uint64_t)b, phase, tail_of(bits_at(ej + k - 1) & 7u));
            r.len = (uint32_t)(ej - bj);
            r.key = key;
            emit_packed(a, hist, slot++, r);
        }
        // ---- the superkmer that runs past the tile: its end in the staged halo ----
        const unsigned op = __ballot_sync(FULL, open);
        if (op) {
            const int src = __ffs(op) - 1;
            o_pos = __shfl_sync(FULL, o_pos, src);
            o_key = __shfl_sync(FULL, o_key, src);
            o_phase = __shfl_sync(FULL, o_phase, src);
            o_slot = __shfl_sync(FULL, o_slot, src);
            const int jlimit = P1_STAGE - (128 + k);  // last chunk start whose keys and bits are staged
            int cj = 32 + P1_TILE, ej = P1_INF;
            for (; cj <= jlimit; cj += 32) {
                const int j = cj + lane;
                uint32_t m = 0xFFFFFFFFu;
                for (int x = 0; x < w; x++) m = min(m, skey[p1_sk(j + x)]);
                const uint32_t bits = bits_at(j);
                bool valid;
                if (KW) {
                    const uint64_t b64 = bits | ((uint64_t)bits_at(j + 32) << 32);
                    valid = j <= jmaxk && ((b64 >> 1) & vmask64) == 0;
                } else {
                    valid = j <= jmaxk && ((bits >> 1) & vmask) == 0;
                }
                const unsigned eb = __ballot_sync(FULL, !valid || (bits & 1u) || m != o_key);
                if (eb) {
                    ej = cj + __ffs(eb) - 1;
                    break;
                }
            }
            if (lane == src) {
                if (ej != P1_INF) {
                    SkmRecord r;
                    r.pos = rec_pack_pos((uint64_t)o_pos, o_phase, tail_of(bits_at(ej + k - 1) & 7u));
                    r.len = (uint32_t)(sbeg + ej - o_pos);
                    r.key = o_key;
                    emit_packed(a, hist, o_slot, r);
                } else {  // past the staged range too: from global memory
                    const int64_t c0 = sbeg + cj;
                    const int64_t rr = read_of(a.offs, a.n_reads, (uint64_t)o_pos);
                    const int64_t re = (int64_t)a.offs[rr + 1];
                    int64_t e = c0 > o_pos + 1 ? c0 : o_pos + 1;
                    while (e + k <= re && kmer_key_global<LUT>(a, (uint64_t)e) == o_key) e++;
                    const int64_t rest = re - (e + k - 1);
                    emit_record(a, hist, o_slot, (uint64_t)o_pos, (uint32_t)(e - o_pos), o_key, o_phase,
                                rest >= 3 ? 3u : (uint32_t)rest);
                }
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

// 1024-thread CTAs.  A CTA's records are taken in chunks of P2_CHUNK, each
// put in partition order first (a counting sort in shared memory), so that a
// warp's 32 records fall into a few runs of one partition each: a run
// reserves its bytes and index slots with one atomic, and its superkmers
// leave as contiguous, mostly whole sectors.  In record order every record of
// a warp went to another partition's write front (296-592 CTAs x P fronts),
// and partial sectors were completed by read-modify-write in DRAM.
constexpr int P2_THREADS = 1024;
constexpr int P2_CHUNK = 8192;  // records per chunk (8 per thread)

// Dynamic shared memory of the scatter: CTA bases (2P u64), cursors (2P),
// chunk counts and starts (P each), the chunk order (u16 per record).
__host__ __device__ inline size_t p2_smem(uint32_t P) {
    return 2ull * P * 8 + 2ull * P * 4 + 2ull * P * 4 + (size_t)P2_CHUNK * 2;
}

__global__ void __launch_bounds__(P2_THREADS, 2)
scatter_superkmers_kernel(P2Params a) {
    extern __shared__ unsigned long long sbase[];                    // [2P] CTA bases in each partition
    uint32_t *lcnt = reinterpret_cast<uint32_t *>(sbase + 2 * a.P);  // [2P] CTA-local cursors (bytes, superkmers)
    uint32_t *ccnt = lcnt + 2 * a.P;                                 // [P] records of the chunk per partition
    uint32_t *cstart = ccnt + a.P;                                   // [P] their first place in chunk order
    uint16_t *order = reinterpret_cast<uint16_t *>(cstart + a.P);    // [P2_CHUNK] chunk records by partition
    __shared__ uint32_t ws[P2_THREADS / 32];
    if (*a.flags & (ERR_RECORD_OVERFLOW | ERR_CAPACITY)) return;  // the batch is redone
    const uint32_t n = a.region_count[blockIdx.x] < a.region_cap ? a.region_count[blockIdx.x] : a.region_cap;
    const SkmRecord *rec = a.records + (uint64_t)blockIdx.x * a.region_cap;
    // this CTA's ranges, laid out by cta_offsets_kernel from the find kernel's
    // per-CTA counts
    const unsigned long long *cb = a.cta_base + (uint64_t)blockIdx.x * 2 * a.P;
    for (uint32_t i = threadIdx.x; i < 2 * a.P; i += blockDim.x) {
        sbase[i] = cb[i];
        lcnt[i] = 0;
    }
    const int lane = threadIdx.x & 31;
    const unsigned lanes_le = 0xFFFFFFFFu >> (31 - lane);
    constexpr int PER = P2_CHUNK / P2_THREADS;
    for (uint32_t c0 = 0; c0 < n; c0 += P2_CHUNK) {
        const uint32_t m = n - c0 < (uint32_t)P2_CHUNK ? n - c0 : (uint32_t)P2_CHUNK;
        for (uint32_t i = threadIdx.x; i < a.P; i += blockDim.x) ccnt[i] = 0;
        __syncthreads();
        // ---- the chunk's records counted per partition (rank within it) ----
        uint32_t pr[PER];  // partition << 16 | rank (ranks < P2_CHUNK)
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const uint32_t j = threadIdx.x + t * P2_THREADS;
            pr[t] = 0;
            if (j < m) {
                const uint32_t part = fastmod(~rec[c0 + j].key, a.pmod, a.P);
                pr[t] = (part << 16) | atomicAdd(&ccnt[part], 1u);
            }
        }
        __syncthreads();
        // ---- each partition's first place in chunk order ----
        {
            const uint32_t per = (a.P + P2_THREADS - 1) / P2_THREADS, p0 = threadIdx.x * per;
            uint32_t sum = 0, tot;
            for (uint32_t p = p0; p < p0 + per && p < a.P; p++) sum += ccnt[p];
            uint32_t pre = block_exclusive_scan<P2_THREADS>(sum, &tot, ws);
            for (uint32_t p = p0; p < p0 + per && p < a.P; p++) {
                cstart[p] = pre;
                pre += ccnt[p];
            }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < PER; t++) {
            const uint32_t j = threadIdx.x + t * P2_THREADS;
            if (j < m) order[cstart[pr[t] >> 16] + (pr[t] & 0xFFFFu)] = (uint16_t)j;
        }
        __syncthreads();
        // ---- warps take 32 records in partition order at a time.  Each lane
        //      sets up its own record (destination, code slot, headers); the
        //      lanes of one partition form a run that reserves its bytes and
        //      index slots with one atomic.  Then the warp writes the records'
        //      destination words cooperatively, one aligned 4-byte word per
        //      lane per step (no lane waits for a longer superkmer, and
        //      consecutive lanes write consecutive words). ----
        const uint32_t nwarps = blockDim.x >> 5;
        for (uint32_t base = (threadIdx.x >> 5) * 32; base < m; base += nwarps * 32) {
            const uint32_t i = base + lane;
            const bool has = i < m;
            SkmRecord r;
            r.pos = 0;
            r.len = 0;
            r.key = 0;
            uint32_t part = 0xFFFFFFFFu, nb = 0;
            if (has) {
                r = rec[c0 + order[i]];
                part = fastmod(~r.key, a.pmod, a.P);
                nb = skm_nbytes(rec_phase(r.pos), r.len, a.k);
            }
            // runs of one partition: heads, inclusive byte prefix, run bounds
            const uint32_t prev = __shfl_up_sync(FULL, part, 1);
            const unsigned heads = __ballot_sync(FULL, lane == 0 || prev != part);
            uint32_t incl = nb;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, incl, d);
                if (lane >= d) incl += y;
            }
            const int hs = 31 - __clz(heads & lanes_le);                   // this run's first lane
            const unsigned later = heads & ~lanes_le;                      // heads after this lane
            const int he = later ? __ffs(later) - 2 : 31;                  // this run's last lane
            const uint32_t excl_s = __shfl_sync(FULL, incl - nb, hs);      // bytes before the run
            const uint32_t run_bytes = __shfl_sync(FULL, incl, he) - excl_s;
            uint32_t rb = 0, rs = 0;
            if (has && lane == hs) {
                rb = atomicAdd(&lcnt[part], run_bytes);
                rs = atomicAdd(&lcnt[a.P + part], (uint32_t)(he - hs + 1));
            }
            rb = __shfl_sync(FULL, rb, hs);
            rs = __shfl_sync(FULL, rs, hs);
            uint64_t dst = 0, pos = 0;
            uint32_t rlim = 0, hdr = 0, nw = 0;
            if (has) {
                const uint32_t phase = rec_phase(r.pos), tail = rec_tail(r.pos);
                const uint32_t ob = rb + (incl - nb - excl_s);
                const uint32_t os = rs + (uint32_t)(lane - hs);
                const uint64_t pbase = sbase[part] - a.part_byte_off[part];  // this CTA's range in the partition
                dst = reinterpret_cast<uint64_t>(a.bytes + sbase[part] + ob);
                pos = rec_base(r.pos) - phase;              // first code slot of the first byte
                rlim = phase + r.len + (uint32_t)a.k - 1 + tail;  // read bases used, from pos
                hdr = (3 - phase) | (((phase + r.len + (uint32_t)a.k - 1) % 3) << 2);  // first, last byte headers
                nw = (uint32_t)((((dst + nb + 3) & ~3ull) - (dst & ~3ull)) >> 2);
                a.idx[sbase[a.P + part] + os] = idx_pack(pbase + ob, r.len);
                a.keys[sbase[a.P + part] + os] = r.key;
            }
            uint32_t wincl = nw;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, wincl, d);
                if (lane >= d) wincl += y;
            }
            const uint32_t total = __shfl_sync(FULL, wincl, 31), excl = wincl - nw;
            for (uint32_t w0 = 0; w0 < total; w0 += 32) {
                const uint32_t gi = w0 + lane;
                int own = 0;  // the last lane whose first word index is <= gi
#pragma unroll
                for (int st = 16; st; st >>= 1) {
                    const int cand = own + st;
                    if (__shfl_sync(FULL, excl, cand) <= gi) own = cand;
                }
                const uint32_t sw = gi - __shfl_sync(FULL, excl, own);
                const uint64_t odst = __shfl_sync(FULL, dst, own), opos = __shfl_sync(FULL, pos, own);
                const uint32_t onb = __shfl_sync(FULL, nb, own), olim = __shfl_sync(FULL, rlim, own);
                const uint32_t ohdr = __shfl_sync(FULL, hdr, own);
                if (gi >= total) continue;
                const uint64_t A = (odst & ~3ull) + 4ull * sw;   // this lane's destination word
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
        __syncthreads();  // ccnt, cstart and order are reused by the next chunk
    }
}

}  // namespace gkc
