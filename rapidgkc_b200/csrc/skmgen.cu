// skmgen.cu -- phase 1: reads -> superkmers in per-partition device buffers.
//
// Replaces the reference's GPU_GenMinimizer / GPU_GenSKMOffs /
// GPU_ReadCompression / GPU_ExtractSKM chain (gpu_skmgen.cu:218-470) and the
// host round trip per 2048-read batch (gpu_skmgen.cu:504-718).
//
// Kernel 1 (find_superkmers) walks the concatenated read bases in tiles.  A
// CTA stages its tile's ASCII bytes in shared memory as 2-bit codes (16-byte
// vector loads) together with a bitmap of read boundaries.  Each warp then
// walks a strip of the tile 32 positions at a time: lane l evaluates the
// canonical p-mer key at position c0+l; the minimum over the window of
// w = k-p+1 p-mers is a sparse-table doubling over a 64-wide register window
// (this chunk and the next) built from shuffles; superkmer starts and ends
// are ballots over the chunk.  Closed superkmers are written as compact
// records into a per-CTA region, and per-partition byte/superkmer/k-mer
// counts accumulate in shared memory.
//
// Kernel 2 (scatter_superkmers) reserves, per CTA and per partition, a
// contiguous range of each partition's byte and index buffers, then writes
// every superkmer in the reference's 3-bases-per-byte format
// (cpu_funcs.cpp:200-250): a copy of the packed read whose first byte's
// header says 3-beg%3 valid bases and whose last byte's header says
// (end-1+k)%3, so the bytes are bit-identical to the reference's.
#include "gkc_device.cuh"

namespace gkc {

constexpr int P1_WARPS = 8;
constexpr int P1_THREADS = P1_WARPS * 32;
constexpr int P1_CHUNKS = 8;                          // chunks of 32 positions per warp strip
constexpr int P1_STRIP = 32 * P1_CHUNKS;              // 256 positions
constexpr int P1_TILE = P1_WARPS * P1_STRIP;          // 2048 positions per tile
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
    const uint32_t *lut;       // 4^p ranks, or null for the default order
    int vec_ok;                // reads pointer is 16-byte aligned
    SkmRecord *records;        // gridDim.x regions of `region_cap` records
    uint32_t region_cap;
    uint32_t *region_count;    // [gridDim.x]
    unsigned long long *part_bytes, *part_skms, *part_kmers;  // [P]
    int smem_hist;             // per-CTA histograms in shared memory (P <= 4096)
    uint32_t *err;
};

// Packs four 2-bit codes held one per byte (byte 0 first) into 8 bits with the
// first base in bits 7-6.
__device__ __forceinline__ uint32_t pack4(uint32_t c) {
    uint32_t r = __byte_perm(c, 0, 0x0123);
    return (r | (r >> 6) | (r >> 12) | (r >> 18)) & 0xFFu;
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

__device__ __forceinline__ uint32_t pmer_key(uint32_t v, int p, uint32_t pmask, const uint32_t *lut) {
    if (lut) return __ldg(lut + v);
    return mm_valid(v, p) ? v : pmask;
}

// Minimizer key of k-mer q computed directly from global memory (used only
// for superkmers that run past the staged halo).
__device__ uint32_t kmer_key_global(const P1Params &a, uint64_t q) {
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * a.p);
    uint32_t f = 0, best = 0xFFFFFFFFu;
    for (int j = 0; j < a.k; j++) {
        f = ((f << 2) | code1(a.reads[q + j])) & pmask;
        if (j >= a.p - 1) {
            uint32_t r = rc32(f, a.p);
            uint32_t kf = pmer_key(f, a.p, pmask, a.lut), kr = pmer_key(r, a.p, pmask, a.lut);
            uint32_t m = kf < kr ? kf : kr;
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

struct P1Smem {
    uint32_t codes[P1_CODE_WORDS];
    uint32_t bm[P1_BM_WORDS];
    uint32_t region_n;
    uint64_t rs0;  // start of the read containing the first staged position
};

__device__ __forceinline__ void emit_record(const P1Params &a, P1Smem &sm, uint32_t *h_bytes,
                                            uint32_t *h_skms, uint32_t *h_kmers, uint32_t slot,
                                            uint64_t pos, uint32_t len, uint32_t key,
                                            uint32_t phase, uint32_t tail) {
    uint32_t part = (~key) % a.P;
    uint32_t nb = skm_nbytes(phase, len, a.k);
    if (len > IDX_MAX_LEN) atomicOr(a.err, ERR_SKM_TOO_LONG);
    if (a.smem_hist) {
        atomicAdd(h_bytes + part, nb);
        atomicAdd(h_skms + part, 1u);
        atomicAdd(h_kmers + part, len);
    } else {
        atomicAdd(a.part_bytes + part, (unsigned long long)nb);
        atomicAdd(a.part_skms + part, 1ull);
        atomicAdd(a.part_kmers + part, (unsigned long long)len);
    }
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

__global__ void __launch_bounds__(P1_THREADS)
find_superkmers_kernel(P1Params a) {
    extern __shared__ uint32_t dyn[];
    __shared__ P1Smem sm;
    uint32_t *h_bytes = dyn, *h_skms = dyn + a.P, *h_kmers = dyn + 2 * a.P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = a.k, p = a.p, w = k - p + 1;
    const uint32_t pmask = 0xFFFFFFFFu >> (32 - 2 * p);
    int L2 = 1;
    while (L2 * 2 <= w) L2 *= 2;  // largest power of two <= w
    const unsigned lt_mask = (1u << lane) - 1, le_mask = lt_mask | (1u << lane);

    if (a.smem_hist)
        for (uint32_t i = threadIdx.x; i < 3 * a.P; i += blockDim.x) dyn[i] = 0;
    if (threadIdx.x == 0) sm.region_n = 0;

    const uint64_t ntiles = (a.total + P1_TILE - 1) / P1_TILE;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        const int64_t t0 = (int64_t)(tile * P1_TILE);
        const int64_t sbeg = t0 - 32;  // first staged position (multiple of 16)
        // ---- stage 2-bit codes ----
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
        }
        for (int i = threadIdx.x; i < P1_BM_WORDS; i += blockDim.x) sm.bm[i] = 0;
        __syncthreads();
        // ---- read-boundary bitmap: bit j <=> some offs[r] == sbeg + j ----
        {
            __shared__ int64_t r0s;
            if (threadIdx.x == 0) {
                uint64_t q0 = sbeg < 0 ? 0 : (uint64_t)sbeg;
                int64_t r0 = read_of(a.offs, a.n_reads, q0);
                r0s = r0;
                sm.rs0 = a.offs[r0];
            }
            __syncthreads();
            const int64_t send = sbeg + P1_STAGE;
            for (int64_t r = r0s + threadIdx.x; r <= a.n_reads; r += blockDim.x) {
                int64_t o = (int64_t)a.offs[r];
                if (o >= send) break;
                if (o >= sbeg) atomicOr(&sm.bm[(o - sbeg) >> 5], 1u << ((o - sbeg) & 31));
            }
            __syncthreads();
        }
        // ---- each warp walks its strip ----
        const int64_t strip0 = t0 + (int64_t)warp * P1_STRIP;
        if (strip0 >= (int64_t)a.total) continue;
        const int64_t strip1 = strip0 + P1_STRIP;

        auto pk_at = [&](int64_t q) -> uint32_t {  // canonical p-mer key at staged position q
            int64_t j = q - sbeg;
            int i = (int)(j >> 4), o = (int)(j & 15);
            uint64_t v = ((uint64_t)sm.codes[i] << 32) | sm.codes[i + 1];
            uint32_t f = (uint32_t)(v >> (64 - 2 * (o + p))) & pmask;
            uint32_t r = rc32(f, p);
            uint32_t kf = pmer_key(f, p, pmask, a.lut), kr = pmer_key(r, p, pmask, a.lut);
            return kf < kr ? kf : kr;
        };
        auto bits_at = [&](int64_t q, int n) -> uint32_t {  // n (<=31) boundary bits from q
            int64_t j = q - sbeg;
            int i = (int)(j >> 5), o = (int)(j & 31);
            uint64_t v = (uint64_t)sm.bm[i] | ((uint64_t)sm.bm[i + 1] << 32);
            return (uint32_t)(v >> o) & ((n >= 32) ? 0xFFFFFFFFu : ((1u << n) - 1));
        };
        // read start of the warm-up chunk's first position: the last boundary
        // bit at or before it, else the start of the read containing sbeg.
        int64_t rs;
        {
            int64_t q0 = strip0 - 32;
            int64_t j = q0 - sbeg;  // >= 0
            int wi = (int)(j >> 5);
            uint32_t own = sm.bm[wi] & (((j & 31) == 31) ? 0xFFFFFFFFu : ((2u << (j & 31)) - 1));
            int64_t found = -1;
            if (own) found = sbeg + ((int64_t)wi << 5) + (31 - __clz(own));
            for (int base = wi - 1; found < 0 && base >= 0; base -= 32) {
                int idx = base - lane;
                uint32_t v = idx >= 0 ? sm.bm[idx] : 0u;
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
        int64_t c0 = strip0 - 32;
        uint32_t A = pk_at(c0 + lane), B = pk_at(c0 + 32 + lane);
        uint32_t carried_key = 0xFFFFFFFFu;
        bool open = false;         // a superkmer of this warp whose end is not found yet
        int64_t o_pos = 0;
        uint32_t o_key = 0, o_phase = 0;
        // last chunk start whose next chunk's p-mers and boundary bits are staged
        const int64_t stage_limit = sbeg + P1_STAGE - (128 + k);
        for (;;) {
            const bool warm = c0 < strip0;
            const bool cont = c0 >= strip1;
            if (cont && !open) break;
            if (c0 > stage_limit || c0 >= (int64_t)a.total) break;
            // ---- window minimum over w p-mers for the k-mer at c0+lane ----
            uint32_t ma = A, mb = B;
            for (int x = 1; x < L2; x <<= 1) {
                uint32_t t = __shfl_sync(FULL, lane >= x ? ma : mb, (lane + x) & 31);
                uint32_t tb = __shfl_down_sync(FULL, mb, x);
                ma = min(ma, t);
                mb = min(mb, tb);
            }
            uint32_t key = ma;
            if (w > L2) {
                int d = w - L2;
                uint32_t t = __shfl_sync(FULL, lane >= d ? ma : mb, (lane + d) & 31);
                key = min(ma, t);
            }
            const int64_t q = c0 + lane;
            uint32_t prevkey = __shfl_up_sync(FULL, key, 1);
            if (lane == 0) prevkey = carried_key;
            const bool valid = q >= 0 && (uint64_t)(q + k) <= a.total && bits_at(q + 1, k - 1) == 0;
            const bool isrs = q >= 0 && bits_at(q, 1) != 0;
            const bool start = valid && (isrs || key != prevkey);
            const unsigned RSB = __ballot_sync(FULL, isrs);
            const unsigned E = __ballot_sync(FULL, start || !valid);
            const unsigned S = __ballot_sync(FULL, start);
            // read start of this lane's position
            const unsigned rsle = RSB & le_mask;
            const int64_t my_rs = rsle ? (c0 + 31 - __clz(rsle)) : rs;

            if (!warm) {
                // close the carried superkmer at the first end/start of this chunk
                uint32_t emit_carried = 0;
                int64_t c_end = 0;
                if (open && E) { emit_carried = 1; c_end = c0 + __ffs(E) - 1; }
                // superkmers starting in this chunk (owned strip only)
                bool my_start = start && !cont;
                unsigned above = E & ~le_mask;
                bool my_close = my_start && above != 0;
                unsigned CL = __ballot_sync(FULL, my_close);
                uint32_t n = __popc(CL) + emit_carried;
                uint32_t base = 0;
                if (n) {
                    if (lane == 0) base = atomicAdd(&sm.region_n, n);
                    base = __shfl_sync(FULL, base, 0);
                }
                if (emit_carried && lane == 0) {
                    int64_t x = c_end + k - 2;  // last base
                    uint32_t tail = tail_of(bits_at(x + 1, 3));
                    emit_record(a, sm, h_bytes, h_skms, h_kmers, base, (uint64_t)o_pos,
                                (uint32_t)(c_end - o_pos), o_key, o_phase, tail);
                }
                if (my_close) {
                    int64_t e = c0 + __ffs(above) - 1;
                    int64_t x = e + k - 2;
                    uint32_t tail = tail_of(bits_at(x + 1, 3));
                    uint32_t phase = (uint32_t)((q - my_rs) % 3);
                    emit_record(a, sm, h_bytes, h_skms, h_kmers,
                                base + emit_carried + __popc(CL & lt_mask), (uint64_t)q,
                                (uint32_t)(e - q), key, phase, tail);
                }
                if (emit_carried) open = false;
                // a start with no end in this chunk becomes the open superkmer
                unsigned OPEN = __ballot_sync(FULL, my_start && above == 0);
                if (OPEN) {
                    int src = 31 - __clz(OPEN);
                    open = true;
                    o_pos = c0 + src;
                    o_key = __shfl_sync(FULL, key, src);
                    uint32_t ph = (uint32_t)((q - my_rs) % 3);
                    o_phase = __shfl_sync(FULL, ph, src);
                }
                (void)S;
            }
            carried_key = __shfl_sync(FULL, key, 31);
            if (RSB) rs = c0 + 31 - __clz(RSB);
            // advance
            c0 += 32;
            A = B;
            B = (c0 + 32 + 31 - sbeg < (int64_t)P1_STAGE - 16) ? pk_at(c0 + 32 + lane) : 0xFFFFFFFFu;
        }
        // superkmer running past the staged range: finish it from global memory
        if (open) {
            uint32_t slot = 0;
            if (lane == 0) {
                int64_t r = read_of(a.offs, a.n_reads, (uint64_t)o_pos);
                int64_t re = (int64_t)a.offs[r + 1];
                int64_t e = c0 > o_pos + 1 ? c0 : o_pos + 1;
                while (e + k <= re && kmer_key_global(a, (uint64_t)e) == o_key) e++;
                int64_t after = re - (e + k - 1);
                uint32_t tail = after >= 3 ? 3 : (uint32_t)after;
                slot = atomicAdd(&sm.region_n, 1u);
                emit_record(a, sm, h_bytes, h_skms, h_kmers, slot, (uint64_t)o_pos,
                            (uint32_t)(e - o_pos), o_key, o_phase, tail);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (a.smem_hist) {
        for (uint32_t i = threadIdx.x; i < a.P; i += blockDim.x) {
            if (h_skms[i]) {
                atomicAdd(a.part_bytes + i, (unsigned long long)h_bytes[i]);
                atomicAdd(a.part_skms + i, (unsigned long long)h_skms[i]);
                atomicAdd(a.part_kmers + i, (unsigned long long)h_kmers[i]);
            }
        }
    }
    if (threadIdx.x == 0) a.region_count[blockIdx.x] = sm.region_n;
}

// ---------------------------------------------------------------------------
// Kernel 2: scatter records into per-partition byte and index buffers.
struct P2Params {
    const uint8_t *reads;
    const SkmRecord *records;
    uint32_t region_cap;
    const uint32_t *region_count;
    int k;
    uint32_t P;
    const unsigned long long *part_byte_off;  // [P] partition start in `bytes`
    const unsigned long long *part_skm_off;   // [P] partition start in `idx`
    unsigned long long *cur_bytes, *cur_skms;  // [P] zeroed cursors
    uint8_t *bytes;
    uint64_t *idx;
};

constexpr int P2_THREADS = 512;

__device__ __forceinline__ uint8_t skm_byte(const uint8_t *reads, uint64_t s, uint64_t limit, uint32_t b,
                                            uint32_t nb, uint32_t first_h, uint32_t last_h) {
    uint64_t q = s + 3ull * b;
    uint32_t v = 0;
#pragma unroll
    for (int t = 0; t < 3; t++) {
        uint32_t c = (q + t < limit) ? code1(reads[q + t]) : 0u;
        v |= c << (4 - 2 * t);
    }
    uint32_t h = (b == nb - 1) ? last_h : (b == 0 ? first_h : 3u);
    return (uint8_t)(v | (h << 6));
}

__global__ void __launch_bounds__(P2_THREADS)
scatter_superkmers_kernel(P2Params a) {
    extern __shared__ unsigned long long cur[];  // [2P]: byte and superkmer cursors
    const uint32_t n = a.region_count[blockIdx.x] < a.region_cap ? a.region_count[blockIdx.x] : a.region_cap;
    const SkmRecord *rec = a.records + (uint64_t)blockIdx.x * a.region_cap;
    for (uint32_t i = threadIdx.x; i < 2 * a.P; i += blockDim.x) cur[i] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        SkmRecord r = rec[i];
        uint32_t part = (~r.key) % a.P;
        atomicAdd(&cur[part], (unsigned long long)skm_nbytes(rec_phase(r.pos), r.len, a.k));
        atomicAdd(&cur[a.P + part], 1ull);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < a.P; i += blockDim.x) {
        unsigned long long nbp = cur[i], nsp = cur[a.P + i];
        cur[i] = nbp ? atomicAdd(a.cur_bytes + i, nbp) : 0ull;
        cur[a.P + i] = nsp ? atomicAdd(a.cur_skms + i, nsp) : 0ull;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        SkmRecord r = rec[i];
        uint32_t part = (~r.key) % a.P;
        uint32_t phase = rec_phase(r.pos), tail = rec_tail(r.pos);
        uint64_t g = rec_base(r.pos);
        uint32_t nb = skm_nbytes(phase, r.len, a.k);
        unsigned long long ob = atomicAdd(&cur[part], (unsigned long long)nb);
        unsigned long long os = atomicAdd(&cur[a.P + part], 1ull);
        uint8_t *dst = a.bytes + a.part_byte_off[part] + ob;
        uint64_t s = g - phase;                                 // first slot of the first byte
        uint64_t limit = g + r.len + (uint64_t)a.k - 1 + tail;  // end of read bases used
        uint32_t first_h = 3 - phase, last_h = (phase + r.len + (uint32_t)a.k - 1) % 3;
        for (uint32_t b = 0; b < nb; b++) dst[b] = skm_byte(a.reads, s, limit, b, nb, first_h, last_h);
        a.idx[a.part_skm_off[part] + os] = idx_pack(ob, r.len);
    }
}

}  // namespace gkc
