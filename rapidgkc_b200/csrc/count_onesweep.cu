// count_onesweep.cu -- the sort counter's LSD radix sort, one pass over the
// keys per digit.
//
// The reference sorts each partition's k-mers with thrust::sort
// (gpu_kmercounting.cu:428).  Here every partition of a group is a segment of
// one key buffer and all segments are sorted at once, least significant digit
// first, over only the 2k meaningful bits:
//
//   os_hist_kernel   reads the keys once and counts, per segment, the keys of
//                    every digit value of every pass (one histogram per pass);
//   os_scan_kernel   turns those counts into each digit's first position in
//                    its segment, for every pass;
//   os_pass_kernel   one launch per digit: a CTA takes the next tile of keys
//                    (tile ids from an atomic counter, so every tile before
//                    it is already running), ranks them by digit in shared
//                    memory (per-warp digit counters and __match_any_sync,
//                    stable; a chain of one ballot per digit bit measured
//                    slower), publishes its per-digit counts, and reads the
//                    earlier tiles' counts of its segment back to its own
//                    offsets (decoupled look-back: each tile publishes its
//                    count first and its inclusive prefix once known, and a
//                    reader stops at the first inclusive prefix).  It then
//                    writes its keys in digit order from shared memory, so
//                    the keys of one digit leave as a contiguous run.
//
// Per pass the keys are read once and written once; the look-back statuses
// add NB x 4 bytes per tile.  Digits are up to 11 bits (6 passes over the 62
// bits of a 31-mer); 8 bits is the default (8 passes): with 8-bit digits a
// tile's runs average 16 keys (128 bytes, whole sectors), where 11-bit digits
// leave 2-key runs and partial sectors.  A thread owns one digit (8 bits) in
// the look-back and reads four earlier tiles' statuses per step; the pass is
// latency-bound unless three CTAs share an SM, so the look-back keeps its
// loads few (one base address, constant row offsets) and the register count
// under the three-CTA bound.  A status word holds a 2-bit flag and a 30-bit count,
// so segments are limited to 2^30 - 1 keys (larger ones use the
// three-kernel sort of count_sort.cu).  The flags cycle through three
// (aggregate, inclusive) pairs, so statuses left by the previous pass never
// read as the current pass's and the array is cleared once per sort.
#include "gkc_device.cuh"

namespace gkc {

constexpr int OS_THREADS = 256;
constexpr int OS_WARPS = OS_THREADS / 32;
constexpr int OS_MAX_PASSES = 32;
constexpr uint32_t OS_SEG_MAX = (1u << 30) - 1;
constexpr uint64_t OS_WAIT_NS = 100000000ull;  // a look-back gives up after 0.1 s of waiting
constexpr uint32_t ERR_LOOKBACK = 1u << 10;   // a look-back wait ran out

// keys per thread: 16 u64 or 8 u128, so a tile's keys take 32 KB either way
template <class KT> constexpr int os_items() { return sizeof(KT) == 16 ? 8 : 16; }
template <class KT> constexpr int os_tile() { return OS_THREADS * os_items<KT>(); }

// The segments of one sort: segment s holds keys [key0[s], key0[s+1]) of the
// key buffer, pass tiles [tile0[s], tile0[s+1]) and histogram chunks
// [chunk0[s], chunk0[s+1]).  Kernels find a tile's or chunk's segment by a
// binary search, so no per-tile descriptor is built on the host.
struct OsSegs {
    const unsigned long long *key0;  // [nseg + 1]
    const uint32_t *tile0;           // [nseg + 1]
    const uint32_t *chunk0;          // [nseg + 1]
    uint32_t nseg;
};

// The segment holding item x: the largest s with first[s] <= x (first[0] = 0,
// first[nseg] > x; empty segments repeat a value and are skipped).
__device__ __forceinline__ uint32_t os_seg_of(const uint32_t *first, uint32_t nseg, uint32_t x) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(first + mid) <= x) lo = mid; else hi = mid;
    }
    return lo;
}

struct OsTile {
    uint64_t start;      // first key of the tile
    uint64_t seg_start;  // first key of its segment
    uint32_t n;          // keys in the tile
    uint32_t t;          // tile index in its segment
    uint32_t seg;        // segment index
    uint32_t seg_n;      // keys in the segment
};

// The descriptor of every pass tile (T keys), written once per sort: a pass
// CTA then reads its next tile's descriptor with one load, issued while it
// works on the current tile.
template <int T>
__global__ void os_tiles_kernel(OsSegs sg, uint32_t ntiles, OsTile *tiles) {
    const uint32_t tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const uint32_t s = os_seg_of(sg.tile0, sg.nseg, tile);
    const uint64_t s0 = sg.key0[s], sn = sg.key0[s + 1] - s0;
    OsTile td;
    td.t = tile - sg.tile0[s];
    td.seg = s;
    td.seg_start = s0;
    td.seg_n = (uint32_t)sn;
    td.start = s0 + (uint64_t)td.t * T;
    td.n = (uint32_t)(sn - (uint64_t)td.t * T < (uint64_t)T ? sn - (uint64_t)td.t * T : (uint64_t)T);
    tiles[tile] = td;
}

struct OsPasses {
    int n;                        // passes
    int shift[OS_MAX_PASSES];     // lowest bit of each pass's digit
    int width[OS_MAX_PASSES];     // bits of each pass's digit (<= RB)
};

template <class KT>
__device__ __forceinline__ uint32_t os_digit(const KT &key, int shift, uint32_t mask) {
    return (uint32_t)(key >> shift) & mask;
}

// ---------------------------------------------------------------------------
// Per-segment histograms of every pass.  A CTA counts one chunk (OS_HCHUNK
// keys of one segment) in shared memory and adds the nonzero counts to
// ghist[seg][pass][digit].
constexpr uint32_t OS_HCHUNK = 1u << 16;

template <int RB, class KT>
__global__ void __launch_bounds__(OS_THREADS)
os_hist_kernel(const KT *__restrict__ keys, OsSegs sg, OsPasses ps, uint32_t *ghist) {
    constexpr int NB = 1 << RB;
    extern __shared__ uint32_t h[];  // [ps.n][NB]
    const uint32_t seg = os_seg_of(sg.chunk0, sg.nseg, blockIdx.x);
    const uint64_t s0 = sg.key0[seg], s1 = sg.key0[seg + 1];
    const uint64_t c0 = s0 + (uint64_t)(blockIdx.x - sg.chunk0[seg]) * OS_HCHUNK;
    const uint32_t n = (uint32_t)(s1 - c0 < OS_HCHUNK ? s1 - c0 : OS_HCHUNK);
    for (int i = threadIdx.x; i < ps.n * NB; i += OS_THREADS) h[i] = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < n; j += OS_THREADS) {
        const KT key = keys[c0 + j];
        for (int p = 0; p < ps.n; p++)
            atomicAdd(&h[p * NB + os_digit(key, ps.shift[p], (1u << ps.width[p]) - 1)], 1u);
    }
    __syncthreads();
    uint32_t *g = ghist + (uint64_t)seg * ps.n * NB;
    for (int i = threadIdx.x; i < ps.n * NB; i += OS_THREADS)
        if (h[i]) atomicAdd(g + i, h[i]);
}

// Exclusive scan of one (segment, pass) histogram over its digits, in place:
// the digit's first position in the segment's output.
template <int RB>
__global__ void __launch_bounds__(1024) os_scan_kernel(uint32_t *ghist) {
    constexpr int NB = 1 << RB;
    constexpr int PER = NB > 1024 ? NB / 1024 : 1;
    __shared__ uint32_t ws[32];
    uint32_t *g = ghist + (uint64_t)blockIdx.x * NB;
    uint32_t v[PER], s = 0;
    const int b0 = threadIdx.x * PER;
#pragma unroll
    for (int i = 0; i < PER; i++) {
        v[i] = b0 + i < NB ? g[b0 + i] : 0u;
        s += v[i];
    }
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<1024>(s, &tot, ws);
#pragma unroll
    for (int i = 0; i < PER; i++) {
        if (b0 + i < NB) g[b0 + i] = pre;
        pre += v[i];
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t os_now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t os_load_status(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void os_store_status(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct OsPassParams {
    const void *in;
    void *out;
    const OsTile *tiles;
    uint32_t ntiles;
    uint32_t *status;         // [ntiles][NB]
    const uint32_t *gbase;    // [nseg][npass][NB] digit starts in the segment
    int npass, pass, shift, width;
    uint32_t agg, inc;        // this pass's flags (2 bits, shifted to 31..30)
    uint32_t *tile_ctr;       // next tile of this pass
    uint32_t *err;
};

// CTAs per SM the register budget must allow: three with 16 u64 keys a thread
// (80 registers, no spills; four would spill), four with 8 u128 keys
template <class KT> constexpr int os_min_ctas() { return sizeof(KT) == 16 ? 4 : 3; }

// Shared memory of a pass CTA besides the dynamic key / counter area.
struct OsShared {
    uint32_t ws[32];
    OsTile td;
    __align__(16) OsTile td_next;  // the next tile's descriptor, fetched by cp.async
    uint32_t tile;
    uint32_t lb_fail;  // a look-back of this tile gave up: its keys are not written
};

// Thread 0 fetches a tile descriptor (32 bytes) into shared memory without
// waiting for it; os_desc_wait makes the copy complete.
__device__ __forceinline__ void os_desc_fetch(OsTile *dst, const OsTile *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d + 16), "l"(reinterpret_cast<const char *>(src) + 16)
                 : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void os_desc_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One tile of a pass.  (A bounds-check-free body for full tiles measured no
// faster: with its loads unconditional the compiler holds all of them at
// once and spills under the three-CTA register budget.)
template <int RB, class KT>
__device__ __forceinline__ void os_pass_tile(const OsPassParams &a, OsShared &sh, uint32_t next) {
    constexpr int NB = 1 << RB;
    constexpr int ITEMS = os_items<KT>();
    constexpr int T = os_tile<KT>();
    extern __shared__ __align__(16) unsigned char os_smem[];
    // the key staging area doubles as the per-warp digit counters (u16)
    KT *skeys = reinterpret_cast<KT *>(os_smem);
    uint16_t *wcnt = reinterpret_cast<uint16_t *>(os_smem);           // [OS_WARPS][NB]
    uint32_t *bstart = reinterpret_cast<uint32_t *>(os_smem + T * sizeof(KT));  // [NB] tile-local run starts
    int32_t *bdelta = reinterpret_cast<int32_t *>(bstart + NB);       // [NB] segment position - local index
    uint16_t *tcount = reinterpret_cast<uint16_t *>(bdelta + NB);     // [NB] tile counts
    const KT *in = static_cast<const KT *>(a.in);
    KT *out = static_cast<KT *>(a.out);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1;
    const uint32_t dmask = (1u << a.width) - 1;
    const uint32_t tile = sh.tile;
    const OsTile td = sh.td;
    constexpr int BPT = NB >= OS_THREADS ? NB / OS_THREADS : 1;  // digits per thread in the look-back
    // earlier tiles read at once per digit: the frontier advances at most
    // this many tiles per L2 round trip; tiles start in order, so the tile
    // before is usually already inclusive or nearly so
    constexpr int LB_ROWS = BPT >= 4 ? 1 : 4 / BPT;
    auto has = [&](uint32_t j) { return j < td.n; };

    // ---- load (all loads in flight first), then rank; warp w owns keys
    //      [w * 32 * ITEMS, (w + 1) * 32 * ITEMS) ----
    KT key[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const uint32_t j = (uint32_t)warp * 32 * ITEMS + (uint32_t)i * 32 + lane;
        key[i] = has(j) ? in[td.start + j] : KT(0);
    }
    uint32_t rank[(ITEMS + 1) / 2];  // 16-bit ranks, two to a register
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const uint32_t j = (uint32_t)warp * 32 * ITEMS + (uint32_t)i * 32 + lane;
        const bool valid = has(j);
        const uint32_t dig = valid ? os_digit(key[i], a.shift, dmask) : (uint32_t)NB;
        const unsigned grp = __match_any_sync(FULL, dig);
        uint32_t pre = 0;
        if (valid) pre = wcnt[warp * NB + dig];
        const uint32_t rk = pre + __popc(grp & lt);
        if (i & 1) rank[i >> 1] |= rk << 16; else rank[i >> 1] = rk;
        __syncwarp();
        if (valid && (grp & lt) == 0) wcnt[warp * NB + dig] = (uint16_t)(pre + __popc(grp));
        __syncwarp();
    }
    // thread 0: the next tile's descriptor, needed only at the next tile's
    // start (its id came back from the atomic long ago)
    if (threadIdx.x == 0 && next < a.ntiles) os_desc_fetch(&sh.td_next, a.tiles + next);
    __syncthreads();
    // ---- per digit: exclusive prefix over warps, tile count, published at once ----
    uint32_t *st = a.status + (uint64_t)tile * NB;
    for (int b = threadIdx.x; b < NB; b += OS_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < OS_WARPS; w++) {
            const uint32_t c = wcnt[w * NB + b];
            wcnt[w * NB + b] = (uint16_t)s;
            s += c;
        }
        tcount[b] = (uint16_t)s;
        os_store_status(st + b, (td.t == 0 ? a.inc : a.agg) | s);
    }
    __syncthreads();
    // ---- tile-local run starts: exclusive scan of the counts over digits ----
    {
        constexpr int PER = NB / OS_THREADS > 0 ? NB / OS_THREADS : 1;
        const int b0 = threadIdx.x * PER;
        uint32_t s = 0;
#pragma unroll
        for (int i = 0; i < PER; i++) s += b0 + i < NB ? tcount[b0 + i] : 0u;
        uint32_t tot;
        uint32_t pre = block_exclusive_scan<OS_THREADS>(s, &tot, sh.ws);
#pragma unroll
        for (int i = 0; i < PER; i++)
            if (b0 + i < NB) {
                bstart[b0 + i] = pre;
                pre += tcount[b0 + i];
            }
    }
    __syncthreads();
    // ---- stage the keys in digit order (the counters' area takes the keys) ----
    {
        // each key's place in the tile, written over its rank (16 bits each)
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t j = (uint32_t)warp * 32 * ITEMS + (uint32_t)i * 32 + lane;
            uint32_t lp = 0;
            if (has(j)) {
                const uint32_t dig = os_digit(key[i], a.shift, dmask);
                lp = bstart[dig] + wcnt[warp * NB + dig] + ((rank[i >> 1] >> (16 * (i & 1))) & 0xFFFFu);
            }
            rank[i >> 1] = (i & 1) ? (rank[i >> 1] & 0xFFFFu) | (lp << 16) : (rank[i >> 1] & 0xFFFF0000u) | lp;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t j = (uint32_t)warp * 32 * ITEMS + (uint32_t)i * 32 + lane;
            if (has(j)) skeys[(rank[i >> 1] >> (16 * (i & 1))) & 0xFFFFu] = key[i];
        }
    }
    // ---- look back: each thread's digits together, LB_ROWS earlier tiles a step ----
    {
        const uint32_t *gb = a.gbase + ((uint64_t)td.seg * a.npass + a.pass) * NB;
        uint32_t excl[BPT], jn[BPT], left[BPT];
        uint32_t pending = 0;  // digits still looking back
#pragma unroll
        for (int x = 0; x < BPT; x++) {
            excl[x] = 0;
            jn[x] = tile - 1;
            left[x] = td.t;  // earlier tiles of the segment
            if (td.t != 0 && x * OS_THREADS + (int)threadIdx.x < NB) pending |= 1u << x;
        }
        uint64_t t_wait = 0;  // when this thread first waited
        bool failed = false;
        while (pending) {
            uint32_t v[BPT][LB_ROWS];
#pragma unroll
            for (int x = 0; x < BPT; x++) {
                // row jn - r of digit slot x: one base, constant offsets
                const uint32_t *row = a.status + (uint64_t)jn[x] * NB + x * OS_THREADS + threadIdx.x;
#pragma unroll
                for (int r = 0; r < LB_ROWS; r++)
                    v[x][r] = ((pending >> x) & 1) && (uint32_t)r < left[x] ? os_load_status(row - r * NB) : 0u;
            }
            bool waited = false;
#pragma unroll
            for (int x = 0; x < BPT; x++) {
                if (!((pending >> x) & 1)) continue;
                const uint32_t nr = left[x] < (uint32_t)LB_ROWS ? left[x] : (uint32_t)LB_ROWS;
                uint32_t r = 0;  // rows consumed
#pragma unroll
                for (int rr = 0; rr < LB_ROWS; rr++) {
                    if ((uint32_t)rr >= nr) break;
                    const uint32_t f = v[x][rr] & 0xC0000000u;
                    if (f == a.inc) {
                        excl[x] += v[x][rr] & 0x3FFFFFFFu;
                        pending &= ~(1u << x);
                        break;
                    }
                    if (f != a.agg) {  // not published yet: this row is read again next step
                        waited = true;
                        break;
                    }
                    excl[x] += v[x][rr] & 0x3FFFFFFFu;
                    r++;
                }
                if ((pending >> x) & 1) {
                    jn[x] -= r;
                    left[x] -= r;
                    // the segment's first tile publishes its inclusive prefix at once,
                    // so the walk cannot run past it
                    if (left[x] == 0) {
                        atomicOr(a.err, ERR_LOOKBACK);
                        failed = true;
                        pending &= ~(1u << x);
                    }
                }
            }
            if (waited) {
                // never expected: an earlier tile that does not publish.  Give
                // up after OS_WAIT_NS, or at once when another tile gave up,
                // record it and go on (the host then fails the call)
                const uint64_t now = os_now_ns();
                if (!t_wait) t_wait = now;
                if (now - t_wait > OS_WAIT_NS || (os_load_status(a.err) & ERR_LOOKBACK)) {
                    if (!(atomicOr(a.err, ERR_LOOKBACK) & ERR_LOOKBACK)) {  // the first to give up
                        a.err[1] = tile;
                        a.err[2] = (uint32_t)__ffs(pending) - 1 + 0;  // the digit slot still waiting
                        a.err[3] = td.t;
                    }
                    failed = true;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (failed) sh.lb_fail = 1;
#pragma unroll
        for (int x = 0; x < BPT; x++) {
            const int b = x * OS_THREADS + threadIdx.x;
            if (b < NB) {
                if (td.t != 0) os_store_status(st + b, a.inc | ((excl[x] + tcount[b]) & 0x3FFFFFFFu));
                bdelta[b] = (int32_t)(gb[b] + excl[x]) - (int32_t)bstart[b];
            }
        }
    }
    __syncthreads();
    // ---- write: consecutive threads, consecutive keys of one digit run.
    //      Every position is inside the segment by construction (the
    //      segment's histogram counts exactly its keys); a tile whose
    //      look-back gave up writes nothing (the host fails the call). ----
    if (!sh.lb_fail) {
        KT *o = out + td.seg_start;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t idx = (uint32_t)i * OS_THREADS + threadIdx.x;
            if (has(idx)) {
                const KT k = skeys[idx];
                o[(int64_t)bdelta[os_digit(k, a.shift, dmask)] + idx] = k;
            }
        }
    }
}

template <int RB, class KT>
__global__ void __launch_bounds__(OS_THREADS, os_min_ctas<KT>())
os_pass_kernel(OsPassParams a) {
    constexpr int NB = 1 << RB;
    constexpr int T = os_tile<KT>();
    static_assert(OS_WARPS * NB * 2 <= T * (int)sizeof(KT), "warp counters fit the key staging area");
    extern __shared__ __align__(16) unsigned char os_smem[];
    uint16_t *wcnt = reinterpret_cast<uint16_t *>(os_smem);
    __shared__ OsShared sh;
    // The next tile's id is taken while the current tile runs, and its
    // descriptor read once the id is back, so neither round trip is on the
    // critical path.  A CTA's next tile is always later
    // than its current one, so the earliest unfinished tile is always running
    // and every look-back ends.
    uint32_t next = 0;  // thread 0: the next tile
    if (threadIdx.x == 0) {
        next = atomicAdd(a.tile_ctr, 1u);
        if (next < a.ntiles) os_desc_fetch(&sh.td_next, a.tiles + next);
    }
    for (;;) {
        if (threadIdx.x == 0) {
            os_desc_wait();
            sh.tile = next;
            sh.td = sh.td_next;
            sh.lb_fail = 0;
            if (next < a.ntiles) next = atomicAdd(a.tile_ctr, 1u);
        }
        for (int i = threadIdx.x; i < OS_WARPS * NB / 2; i += OS_THREADS) reinterpret_cast<uint32_t *>(wcnt)[i] = 0;
        __syncthreads();
        if (sh.tile >= a.ntiles) break;
        os_pass_tile<RB, KT>(a, sh, next);
        __syncthreads();  // the staging area is cleared for the next tile
    }
}

template <int RB, class KT>
constexpr size_t os_pass_smem() {
    return (size_t)os_tile<KT>() * sizeof(KT) + (size_t)(1 << RB) * (4 + 4 + 2);
}

}  // namespace gkc
