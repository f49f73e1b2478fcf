// fastx.cu -- FASTQ / FASTA record scanning on the device: text in, a CSR of
// reads (sequence bytes + u64 offsets) out, ready for phase 1.
//
// The reference's loader (fileloader.hpp:201-232, 269-330) finds newlines on
// the host and takes every 4th line of FASTQ (line 4i+1) as a read, carrying
// the line phase across buffers.  Here the same line phase is computed for all
// bytes at once.  A span of text (a thread's 64 bytes, a CTA's 16 KiB tile,
// a run of tiles) is summarised as a transform over the state at its start:
//   FASTQ  state = line phase 0..3 (0 header, 1 sequence, 2 '+', 3 quality);
//          a byte is kept when its phase is 1; a read starts after each
//          newline that ends a phase-0 line;
//   FASTA  state = type of the current line (0 sequence, 1 header '>'); a
//          line's type is set by its first byte, so the state only matters up
//          to the span's first line start; a read starts at each header line;
//          the sequence lines of a record are concatenated.
// '\n' and '\r' are never kept.  Transforms compose associatively, so tiles
// are scanned in parallel (fastx_tile_kernel), the tile transforms are scanned
// by one CTA (fastx_carry_kernel), and each tile is rescanned to write its
// bytes and read offsets (fastx_write_kernel).
#pragma once

#include "gkc_device.cuh"

constexpr int FX_THREADS = 256, FX_PER = 64, FX_TILE = FX_THREADS * FX_PER;  // 16 KiB tiles
constexpr int FX_CARRY_THREADS = 256;

struct FxT {               // the effect of a span, per state at its start
    uint8_t next[4];       // state after the span
    uint64_t kept[4];      // bytes kept
    uint64_t reads[4];     // reads started
};

__device__ __forceinline__ FxT fx_identity() {
    FxT t;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        t.next[s] = (uint8_t)s;
        t.kept[s] = 0;
        t.reads[s] = 0;
    }
    return t;
}

// a then b
__device__ __forceinline__ FxT fx_compose(const FxT &a, const FxT &b) {
    FxT t;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int m = a.next[s];
        t.next[s] = b.next[m];
        t.kept[s] = a.kept[s] + b.kept[m];
        t.reads[s] = a.reads[s] + b.reads[m];
    }
    return t;
}

// Counts over a span from which its transform follows for every start
// state: FASTQ keeps counts indexed by the newlines seen so far (mod 4),
// FASTA splits the keepable bytes at the span's first line start.
struct FxSpan {
    uint32_t cnt[4];   // FASTQ: keepable bytes by newlines-before mod 4
    uint32_t nlc[4];   // FASTQ: newlines by newlines-before mod 4
    uint32_t nl;       // FASTQ: newlines
    uint32_t pre;      // FASTA: keepable bytes before the first line start
    uint32_t rest;     // FASTA: keepable bytes in lines starting in the span
    uint32_t heads;    // FASTA: header line starts
    int last_type;     // FASTA: type of the last line start (-1: none)
};

__device__ __forceinline__ bool fx_keepable(uint8_t c) { return c != '\n' && c != '\r'; }

// the counts of bytes b[0, len); prev: the byte before b ('\n' at the text's start)
template <bool FASTA>
__device__ __forceinline__ FxSpan fx_count(const uint8_t *b, int len, uint8_t prev) {
    FxSpan r;
#pragma unroll
    for (int i = 0; i < 4; i++) r.cnt[i] = r.nlc[i] = 0;
    r.nl = r.pre = r.rest = r.heads = 0;
    r.last_type = -1;
    int type = -1;  // FASTA: type of the current line if it started in the span
    for (int i = 0; i < len; i++) {
        const uint8_t c = b[i];
        if (FASTA) {
            if (prev == '\n') {
                type = c == '>';
                r.last_type = type;
                r.heads += (uint32_t)type;
            }
            if (fx_keepable(c)) {
                if (type < 0) r.pre++;
                else if (type == 0) r.rest++;
            }
        } else {
            if (c == '\n') {
                r.nlc[r.nl & 3]++;
                r.nl++;
            } else if (c != '\r') {
                r.cnt[r.nl & 3]++;
            }
        }
        prev = c;
    }
    return r;
}

template <bool FASTA>
__device__ __forceinline__ FxT fx_transform(const FxSpan &r) {
    FxT t;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        if (FASTA) {
            t.next[s] = (uint8_t)(r.last_type >= 0 ? r.last_type : s);
            t.kept[s] = r.rest + (s == 0 ? r.pre : 0);
            t.reads[s] = r.heads;
        } else {
            t.next[s] = (uint8_t)((s + r.nl) & 3);
            t.kept[s] = r.cnt[(1 - s) & 3];
            t.reads[s] = r.nlc[(4 - s) & 3];
        }
    }
    return t;
}

// inclusive block scan of transforms (Hillis-Steele, one shared buffer)
template <int NT>
__device__ __forceinline__ FxT fx_block_scan(FxT v, FxT *sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int d = 1; d < NT; d <<= 1) {
        FxT o = t >= d ? sh[t - d] : fx_identity();
        __syncthreads();
        if (t >= d) v = fx_compose(o, v);
        sh[t] = v;
        __syncthreads();
    }
    return v;
}

struct FxParams {
    const uint8_t *text;
    uint64_t n;
    FxT *tiles;            // [ntiles] tile transforms
    uint64_t ntiles;
    // carry results per tile
    uint8_t *tile_state;   // state at the tile's start
    uint64_t *tile_kept;   // bytes kept before the tile
    uint64_t *tile_reads;  // reads started before the tile
    uint64_t *result;      // [0] bytes kept, [1] reads, [2] state at the end
    int state_in;          // state at the text's start
    uint8_t *out;          // kept bytes
    uint64_t *offs;        // read offsets (offs[reads] = bytes kept)
};

template <bool FASTA>
__device__ __forceinline__ FxSpan fx_thread_span(const FxParams &a, uint64_t tile, int *len_out) {
    const uint64_t pos = tile * FX_TILE + (uint64_t)threadIdx.x * FX_PER;
    const int len = pos < a.n ? (int)(a.n - pos < (uint64_t)FX_PER ? a.n - pos : FX_PER) : 0;
    *len_out = len;
    const uint8_t prev = pos == 0 ? (uint8_t)'\n' : (pos <= a.n ? a.text[pos - 1] : (uint8_t)0);
    uint8_t buf[FX_PER];
    if (len == FX_PER && (reinterpret_cast<uintptr_t>(a.text + pos) & 15) == 0) {
        const uint4 *p = reinterpret_cast<const uint4 *>(a.text + pos);
#pragma unroll
        for (int i = 0; i < FX_PER / 16; i++) reinterpret_cast<uint4 *>(buf)[i] = p[i];
    } else {
        for (int i = 0; i < len; i++) buf[i] = a.text[pos + i];
    }
    return fx_count<FASTA>(buf, len, prev);
}

template <bool FASTA>
__global__ void __launch_bounds__(FX_THREADS) fastx_tile_kernel(FxParams a) {
    __shared__ FxT sh[FX_THREADS];
    int len;
    const FxSpan r = fx_thread_span<FASTA>(a, blockIdx.x, &len);
    const FxT v = fx_block_scan<FX_THREADS>(fx_transform<FASTA>(r), sh);
    if (threadIdx.x == FX_THREADS - 1) a.tiles[blockIdx.x] = v;
}

// One CTA: each thread composes a contiguous run of tiles, the runs are
// scanned, and each thread walks its run from the text's start state.
__global__ void __launch_bounds__(FX_CARRY_THREADS) fastx_carry_kernel(FxParams a, int virtual_read) {
    __shared__ FxT sh[FX_CARRY_THREADS];
    const uint64_t per = (a.ntiles + FX_CARRY_THREADS - 1) / FX_CARRY_THREADS;
    const uint64_t t0 = threadIdx.x * per, t1 = t0 + per < a.ntiles ? t0 + per : a.ntiles;
    FxT v = fx_identity();
    for (uint64_t t = t0; t < t1; t++) v = fx_compose(v, a.tiles[t]);
    const FxT inc = fx_block_scan<FX_CARRY_THREADS>(v, sh);
    // exclusive prefix: the inclusive value of the thread before
    const FxT ex = threadIdx.x ? sh[threadIdx.x - 1] : fx_identity();
    const int s0 = a.state_in;
    int s = ex.next[s0];
    uint64_t kept = ex.kept[s0], reads = ex.reads[s0] + (uint64_t)virtual_read;
    for (uint64_t t = t0; t < t1; t++) {
        a.tile_state[t] = (uint8_t)s;
        a.tile_kept[t] = kept;
        a.tile_reads[t] = reads;
        const FxT &x = a.tiles[t];
        kept += x.kept[s];
        reads += x.reads[s];
        s = x.next[s];
    }
    if (threadIdx.x == FX_CARRY_THREADS - 1) {
        a.result[0] = inc.kept[s0];
        a.result[1] = inc.reads[s0] + (uint64_t)virtual_read;
        a.result[2] = inc.next[s0];
    }
}

// Rescans a tile from its start state: kept bytes are compacted in shared
// memory and written out coalesced; each read start writes its offset.
template <bool FASTA>
__global__ void __launch_bounds__(FX_THREADS) fastx_write_kernel(FxParams a) {
    __shared__ FxT sh[FX_THREADS];
    __shared__ uint8_t stage[FX_TILE];
    const uint64_t tile = blockIdx.x;
    int len;
    const FxSpan r = fx_thread_span<FASTA>(a, tile, &len);
    const FxT mine = fx_transform<FASTA>(r);
    fx_block_scan<FX_THREADS>(mine, sh);
    const FxT ex = threadIdx.x ? sh[threadIdx.x - 1] : fx_identity();
    const int ts = a.tile_state[tile];
    int s = ex.next[ts];
    const uint64_t kept_tile = a.tile_kept[tile];
    uint32_t k = (uint32_t)ex.kept[ts];               // position in the tile's kept bytes
    uint64_t rd = a.tile_reads[tile] + ex.reads[ts];  // next read index
    const uint64_t pos = tile * FX_TILE + (uint64_t)threadIdx.x * FX_PER;
    uint8_t prev = pos == 0 ? (uint8_t)'\n' : (pos <= a.n ? a.text[pos - 1] : (uint8_t)0);
    for (int i = 0; i < len; i++) {
        const uint8_t c = a.text[pos + i];
        if (FASTA) {
            if (prev == '\n') {
                s = c == '>';
                if (s == 1) a.offs[rd++] = kept_tile + k;  // the record's bytes start here
            }
            if (s == 0 && fx_keepable(c)) stage[k++] = c;
        } else {
            if (c == '\n') {
                if (s == 0) a.offs[rd++] = kept_tile + k;  // the next line is a read
                s = (s + 1) & 3;
            } else if (s == 1 && c != '\r') {
                stage[k++] = c;
            }
        }
        prev = c;
    }
    __syncthreads();
    const FxT &tot = sh[FX_THREADS - 1];
    const uint32_t nk = (uint32_t)tot.kept[ts];
    for (uint32_t i = threadIdx.x; i < nk; i += FX_THREADS) a.out[kept_tile + i] = stage[i];
}
