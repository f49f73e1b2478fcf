// engine.cu -- host orchestration and the C ABI of the B200 k-mer counter.
//
// One translation unit: the kernels of skmgen.cu, count_hash.cu and
// count_sort.cu are compiled here together with the host code that drives
// them.  The data path is
//   host/device CSR reads --(H2D, overlapped, batches)--> phase 1 kernels
//   --> partition store (one chunk per batch: partition-ordered superkmer
//   bytes + index, on the device or spilled to pinned host memory)
//   --> phase 2 (hash: groups of partitions split into sub-buckets counted
//   in shared memory; sort: groups of partitions through the segmented
//   radix sort)
//   --> thresholded (k-mer, count) arrays on the device.
#include "../../include/gkc_capi.h"

#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "count_records.cu"
#include "count_sort.cu"
#include "count_onesweep.cu"
#include "count_wide.cu"
#include "order_mlp.cu"
#include "skmgen.cu"
#include "store_pack.cu"
#include "fastx.cu"
#include "skm_load.cu"
#include "hpc.cu"

using namespace gkc;

namespace gkc_host {
// pack_host.cpp: n ASCII bases -> nwords 2-bit words on the host's threads
void pack_bases(const uint8_t *src, uint64_t n, uint32_t *words, uint64_t nwords);
}  // namespace gkc_host

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        // 1/8 headroom: sizes that vary a little between calls (the overflow
        // set of the shared-memory counter) do not reallocate every call
        size_t want = std::max<size_t>(bytes + bytes / 8, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want; else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct PinBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 8, 256);
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want; else p = nullptr;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// /proc/meminfo fields in bytes (0 when unreadable)
static uint64_t meminfo(const char *key) {
    FILE *f = fopen("/proc/meminfo", "r");
    if (!f) return 0;
    char line[256];
    uint64_t v = 0;
    const size_t kl = strlen(key);
    while (fgets(line, sizeof line, f))
        if (!strncmp(line, key, kl) && line[kl] == ':') {
            v = strtoull(line + kl + 1, nullptr, 10) * 1024;
            break;
        }
    fclose(f);
    return v;
}
static uint64_t mem_available() { return meminfo("MemAvailable"); }
static uint64_t mem_total() { return meminfo("MemTotal"); }

// Pinned host memory for spilled chunks.  Pinning is slower than the
// device-to-host copy, so it is done once: regions are handed out first-fit
// from slabs of at least 4 GiB, rewound when the store is cleared, and
// gkc_reserve_host can pin slabs ahead of time (also from another thread
// while batches run).  Only the slab list is shared with that thread.
struct HostArena {
    struct Slab {
        uint8_t *p;
        size_t cap, used;
    };
    static constexpr size_t SLAB_MIN = 4ull << 30;
    std::mutex mu;
    std::vector<Slab> slabs;
    size_t cur = 0;  // first slab that may have room

    // A slab is anonymous memory backed by transparent huge pages, faulted in
    // by several threads and then registered with the driver: about ten
    // times faster than cudaHostAlloc, which zeroes and pins 4 KB pages one
    // by one while holding the driver's lock.
    cudaError_t add_slab(size_t bytes) {  // called without the lock held
        const size_t cap = (std::max(bytes, SLAB_MIN) + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
        // never pin the host into swapping or the out-of-memory killer: keep
        // an eighth of physical memory (at least 8 GiB) available
        const uint64_t avail = mem_available(), total = mem_total();
        if (avail && cap + std::max<uint64_t>(total / 8, 8ull << 30) > avail) return cudaErrorMemoryAllocation;
        void *p = mmap(nullptr, cap, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) return cudaErrorMemoryAllocation;
        madvise(p, cap, MADV_HUGEPAGE);  // advisory: 4 KB pages still work
        const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        const size_t per = (cap / nt + 4095) & ~(size_t)4095;
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; t++)
            th.emplace_back([p, per, cap, t]() {
                volatile uint8_t *b = (uint8_t *)p;
                for (size_t o = t * per; o < std::min(cap, (t + 1) * per); o += 4096) b[o] = 0;
            });
        for (auto &x : th) x.join();
        cudaError_t e = cudaHostRegister(p, cap, cudaHostRegisterDefault);
        if (e != cudaSuccess) {
            munmap(p, cap);
            return e;
        }
        std::lock_guard<std::mutex> g(mu);
        slabs.push_back({(uint8_t *)p, cap, 0});
        return cudaSuccess;
    }
    size_t pinned() {
        std::lock_guard<std::mutex> g(mu);
        size_t f = 0;
        for (auto &s : slabs) f += s.cap;
        return f;
    }
    // Pins slabs until the arena holds `bytes` in all, used or free (batches
    // may be taking slabs meanwhile).  One SLAB_MIN slab at a time: the
    // registration holds the driver's lock (about 0.1 s per slab), so
    // batches running on another thread wait at most that long.
    cudaError_t reserve(size_t bytes) {
        while (pinned() < bytes) {
            cudaError_t e = add_slab(SLAB_MIN);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // `bytes` of pinned memory, 256-byte aligned; valid until rewind().
    // First fit over the slabs; `cur` skips slabs with no useful room left.
    cudaError_t take(size_t bytes, uint8_t **out) {
        bytes = (bytes + 255) & ~(size_t)255;
        for (;;) {
            {
                std::lock_guard<std::mutex> g(mu);
                while (cur < slabs.size() && slabs[cur].cap - slabs[cur].used < (1u << 20)) cur++;
                for (size_t i = cur; i < slabs.size(); i++) {
                    Slab &s = slabs[i];
                    if (s.cap - s.used >= bytes) {
                        *out = s.p + s.used;
                        s.used += bytes;
                        return cudaSuccess;
                    }
                }
            }
            cudaError_t e = add_slab(bytes);
            if (e != cudaSuccess) return e;
        }
    }
    void rewind() {
        std::lock_guard<std::mutex> g(mu);
        for (auto &s : slabs) s.used = 0;
        cur = 0;
    }
    void release() {
        std::lock_guard<std::mutex> g(mu);
        for (auto &s : slabs) {
            cudaHostUnregister(s.p);
            munmap(s.p, s.cap);
        }
        slabs.clear();
        cur = 0;
    }
};

// One phase-1 batch worth of superkmers, partition-ordered.
// Chunks are pooled: a cleared store keeps its buffers for the next batch,
// so steady-state batches allocate nothing.
struct StoreChunk {
    bool on_host = false;
    uint8_t *bytes = nullptr;  // in dbytes, or in the context's host arena
    uint64_t *idx = nullptr;   // in didx, or in the host arena
    uint32_t *keys = nullptr;  // in dkeys, or in the host arena: minimizer key of each superkmer
    uint64_t nbytes = 0, nskm = 0;
    std::vector<uint64_t> byte_off, skm_off;  // [P+1]
    std::vector<uint64_t> kmers;              // [P]
    DevBuf dbytes, didx, dkeys;               // device storage
    DevBuf d_byte_off, d_skm_off;             // device copies of the offsets
    // laid out on the device (phase1_async): k-mers per partition, error
    // flags, and their pinned host mirror read back after the batch
    DevBuf d_kmers, d_flags;
    PinBuf h_meta;                            // byte_off [P+1], skm_off [P+1], kmers [P], flags
    bool pending = false;
    uint64_t batch = 0;                       // the batch of this chunk in the last gkc_add_reads
    uint64_t bases = 0;                       // read bases of the batch
    int64_t pend_find = -1, pend_scatter = -1;  // profiled launches whose bytes wait for the layout
    void release() {
        d_kmers.release();
        d_flags.release();
        h_meta.release();
        dbytes.release();
        didx.release();
        dkeys.release();
        d_byte_off.release();
        d_skm_off.release();
    }
};

uint64_t next_pow2(uint64_t v) {
    uint64_t r = 1;
    while (r < v) r <<= 1;
    return r;
}

}  // namespace

struct gkc_ctx {
    int device = 0;
    gkc_options opt{};
    int sms = 148;
    cudaStream_t s = nullptr, cs = nullptr, own_s = nullptr;
    // spilled chunks: two device staging slots, copied to the host arena on
    // their own stream so the next batch's phase 1 overlaps the copy
    cudaStream_t ss = nullptr;
    // a spilled store's staged ranges get their index entries rebuilt here,
    // beside the copy stream's next copies
    cudaStream_t rs = nullptr;
    cudaEvent_t spill_ready = nullptr, spill_done[2] = {nullptr, nullptr};
    int spill_slot = 0;

    // per-kernel-class profiling (events resolved after each public call)
    struct Pending {
        int cls;
        cudaEvent_t a, b;
        double bytes;
    };
    bool prof = false;
    std::vector<Pending> pend;
    std::vector<cudaEvent_t> evpool;
    double kms[GKC_K_CLASSES] = {}, kbytes[GKC_K_CLASSES] = {};
    uint64_t klaunch[GKC_K_CLASSES] = {};
    cudaEvent_t take_event() {
        if (!evpool.empty()) {
            cudaEvent_t e = evpool.back();
            evpool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void prof_flush() {
        for (auto &q : pend) {
            float ms = 0;
            if (cudaEventSynchronize(q.b) == cudaSuccess && cudaEventElapsedTime(&ms, q.a, q.b) == cudaSuccess) {
                kms[q.cls] += ms;
                klaunch[q.cls]++;
                kbytes[q.cls] += q.bytes;
            }
            evpool.push_back(q.a);
            evpool.push_back(q.b);
        }
        pend.clear();
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
    std::string err;
    uint64_t launches = 0;
    double times[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // see gkc_last_timings

    // phase 1 buffers
    // host batches: NSLOT device slots, so a batch's copy does not wait for the
    // phase 1 of the batch before it in the same slot
    static constexpr int NSLOT = 3;
    DevBuf reads[NSLOT], offs[NSLOT];
    PinBuf offs_pin[2];
    PinBuf pk_host[2];                   // host batches packed to 2-bit words (pinned), one per slot
    uint64_t h2d_bytes = 0;              // bytes the last gkc_add_reads copied host to device
    const uint32_t *p1_packed = nullptr;  // the batch in phase 1 as packed words (device), or null: ASCII
    cudaEvent_t buf_free[NSLOT] = {}, buf_ready[NSLOT] = {};
    cudaEvent_t pk_copied[2] = {nullptr, nullptr};  // the last copy from pk_host[i] is done
    DevBuf cta_hist, cta_base;  // phase 1: per-CTA partition counts and base offsets
    DevBuf records, region_count, hist, flags, cursors, part_off, tile_read, codes;
    PinBuf h_hist, h_flags;
    DevBuf lut;             // canonical order table: min(rank(v), rank(rc(v)))
    bool has_lut = false;
    // learned order: network training and scoring
    DevBuf ord_loads, ord_stage, ord_list, mlp_p, mlp_m, mlp_v, mlp_g, mlp_t, mlp_w, mlp_s, mlp_scalar;
    // FASTQ / FASTA scanning: staged text, tile transforms and carries, the CSR
    DevBuf fx_text, fx_tiles, fx_state, fx_kept, fx_reads, fx_res, fx_out, fx_offs;
    // .skm loading: tile transforms and carries, superkmer starts, k-mer counts
    DevBuf sk_tiles, sk_state, sk_tstarts, sk_res, sk_starts, sk_k32, sk_po;
    DevBuf hpc_tiles, hpc_tbase, hpc_reads, hpc_offs;  // homopolymer-compressed batch
    std::vector<StoreChunk *> store;

    // phase 2 buffers
    DevBuf table;  // HSlot[tcap]
    uint64_t tcap = 0;
    DevBuf out_k, out_c;
    uint64_t out_cap = 0, n_out = 0, n_distinct = 0;
    int res_kw = 1;  // u64 words per k-mer of the result: 2 for k > 32 (u128, low word first)
    // host arrays that the hash counter fills group by group while it counts
    // (gkc_count_reads with host output); `streamed` entries are there
    uint64_t *stream_k = nullptr;
    uint32_t *stream_c = nullptr;
    uint64_t stream_cap = 0, streamed = 0;
    bool has_result = false;
    std::vector<char> counted;  // partitions already counted by gkc_count_partitions
    std::vector<cudaEvent_t> batch_ev;  // start / end of each batch of the last gkc_add_reads
    std::vector<double> batch_ms;       // latency of each batch: its copy start to its phase-1 end
    DevBuf keysA, keysB, tiles, counts, offsets, blocksums, heads_pos, heads_key, tilecnt, tileoff;
    DevBuf os_status, os_hist, os_segs, os_ctr;  // one-pass-per-digit radix sort
    PinBuf h_segs;                               // its segment tables, staged for the copy
    DevBuf segoff, segcur, part_err, scal;
    DevBuf stage_bytes, stage_idx, stage_keys;
    DevBuf spill_bytes[2], spill_idx[2], spill_keys[2];  // device staging of chunks being spilled
    // shared-memory bucket counter
    DevBuf bk_skms, bk_kmers, bk_off, bk_cur, bk_entries, bk_failed, bk_arena, bk_part, bk_desc;
    DevBuf bk_arena2;  // second staging arena: a spilled store's next group is staged beside the current one
    DevBuf bk_ids2, bk_failed2;  // the second counting pass: its sub-buckets and those that failed again
    DevBuf bk_piece;             // 128-bit counter: (piece, pieces) of each second-pass CTA
    DevBuf bk_next;              // the persistent first pass's sub-bucket counter
    PinBuf h_ids2;
    DevBuf r_work, r_count, r_off, r_cur, r_recs, r_failed;  // record sub-buckets
    DevBuf r_stage, r_winst, r_woff, r_wrec;                  // per-work-item record segments
    uint64_t fallback_buckets = 0;  // sub-buckets counted through the L2 table
    PinBuf h_scal;
    PinBuf h_off, h_km, h_ids, h_work;  // pinned staging of the record path's host round trips
    PinBuf h_desc;                      // split descriptors of a group
    PinBuf h_cur;                       // output cursor, distinct count and error flags of a group
    uint64_t free_hint = 0;             // free device memory at the start of the count

    std::vector<StoreChunk *> pool;  // cleared chunks kept for reuse
    HostArena arena;                 // pinned host memory of spilled chunks

    StoreChunk *take_chunk() {
        if (pool.empty()) return new StoreChunk();
        StoreChunk *c = pool.back();
        pool.pop_back();
        return c;
    }
    void clear_store() {
        for (auto *c : store) pool.push_back(c);
        store.clear();
        arena.rewind();
    }

    ~gkc_ctx() {
        if (ss) cudaStreamSynchronize(ss);  // spill copies into the arena
        for (auto *c : store) delete_chunk(c);
        for (auto *c : pool) delete_chunk(c);
        store.clear();
        pool.clear();
        DevBuf *ds[] = {&reads[0], &reads[1], &reads[2], &offs[0], &offs[1], &offs[2], &records, &region_count, &cta_hist, &cta_base,
                        &hist, &flags,
                        &cursors, &part_off, &tile_read, &codes, &lut, &table, &out_k, &out_c, &keysA, &keysB, &tiles,
                        &counts, &offsets, &blocksums, &heads_pos, &heads_key, &tilecnt, &tileoff, &segoff,
                        &segcur, &part_err, &scal, &stage_bytes, &stage_idx, &spill_bytes[0], &spill_idx[0], &spill_keys[0],
                        &spill_bytes[1], &spill_idx[1], &spill_keys[1],
                        &bk_skms, &bk_kmers, &bk_off, &bk_cur, &bk_entries, &bk_failed, &bk_arena, &bk_part, &bk_desc,
                        &bk_arena2,
                        &r_work, &r_count, &r_off, &r_cur, &r_recs, &r_failed, &r_stage, &r_winst,
                        &r_woff, &r_wrec, &ord_loads, &ord_stage, &ord_list, &mlp_p, &mlp_m, &mlp_v, &mlp_g, &mlp_t,
                        &mlp_w, &mlp_s, &mlp_scalar, &fx_text, &fx_tiles, &fx_state, &fx_kept,
                        &fx_reads, &fx_res, &fx_out, &fx_offs, &sk_tiles, &sk_state, &sk_tstarts, &sk_res,
                        &sk_starts, &sk_k32, &hpc_tiles, &hpc_tbase, &hpc_reads, &hpc_offs, &os_status, &os_hist,
                        &os_segs, &os_ctr, &bk_ids2, &bk_failed2, &bk_piece, &bk_next};
        for (auto *d : ds) d->release();
        PinBuf *ps[] = {&offs_pin[0], &offs_pin[1], &pk_host[0], &pk_host[1], &h_hist, &h_flags, &h_scal, &h_off, &h_km, &h_ids, &h_work,
                        &h_desc, &h_cur, &h_segs, &h_ids2};
        for (auto *p : ps) p->release();
        arena.release();
        cudaEvent_t evs[] = {e0, e1, e2, e3, buf_free[0], buf_free[1], buf_free[2], buf_ready[0], buf_ready[1], buf_ready[2], spill_ready,
                             spill_done[0], spill_done[1], pk_copied[0], pk_copied[1]};
        for (auto e : evs) if (e) cudaEventDestroy(e);
        for (auto e : batch_ev) cudaEventDestroy(e);
        prof_flush();
        for (auto e : evpool) cudaEventDestroy(e);
        if (own_s) cudaStreamDestroy(own_s);
        if (cs) cudaStreamDestroy(cs);
        if (ss) cudaStreamDestroy(ss);
        if (rs) cudaStreamDestroy(rs);
    }
    static void delete_chunk(StoreChunk *c) {
        c->release();
        delete c;
    }
    int fail(int code, const char *fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
};

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess)                                                            \
            return ctx->fail(_e == cudaErrorMemoryAllocation ? GKC_ENOMEM : GKC_ECUDA,    \
                             "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

#define LAUNCHED()                          \
    do {                                    \
        ctx->launches++;                    \
        CK(cudaPeekAtLastError());          \
    } while (0)

#define RET(call)                \
    do {                         \
        int _r = (call);         \
        if (_r != GKC_OK) return _r; \
    } while (0)

namespace {

// Brackets one kernel launch with events when profiling is on.
struct KScope {
    gkc_ctx *c;
    int cls;
    double bytes;
    cudaEvent_t a = nullptr;
    KScope(gkc_ctx *ctx, int k, double b) : c(ctx), cls(k), bytes(b) {
        if (c->prof) {
            a = c->take_event();
            cudaEventRecord(a, c->s);
        }
    }
    ~KScope() {
        if (c->prof && a) {
            cudaEvent_t b = c->take_event();
            cudaEventRecord(b, c->s);
            c->pend.push_back({cls, a, b, bytes});
        }
    }
};

}  // namespace

namespace {

// device-wide exclusive scan u32 -> u64; total (optional) on the device
int scan_u32(gkc_ctx *ctx, const uint32_t *in, uint64_t n, uint64_t *out, unsigned long long *total) {
    uint64_t nb = (n + SC_PER_BLOCK - 1) / SC_PER_BLOCK;
    if (nb == 0) {
        if (total) CK(cudaMemsetAsync(total, 0, sizeof(unsigned long long), ctx->s));
        return GKC_OK;
    }
    CK(ctx->blocksums.ensure(nb * sizeof(unsigned long long)));
    auto *bs = ctx->blocksums.as<unsigned long long>();
    {
        KScope ks(ctx, GKC_K_SCAN, 4.0 * n + 8.0 * nb);
        scan_reduce_kernel<<<(unsigned)nb, SC_THREADS, 0, ctx->s>>>(in, n, bs);
        LAUNCHED();
    }
    {
        KScope ks(ctx, GKC_K_SCAN, 16.0 * nb);
        scan_blocksums_kernel<<<1, 1024, 0, ctx->s>>>(bs, nb, total);
        LAUNCHED();
    }
    {
        KScope ks(ctx, GKC_K_SCAN, 12.0 * n + 8.0 * nb);
        scan_down_kernel<<<(unsigned)nb, SC_THREADS, 0, ctx->s>>>(in, n, bs, out);
        LAUNCHED();
    }
    return GKC_OK;
}

// Hash table of at least C slots, every slot empty (the collect kernel leaves
// the slots it reads empty, so only a new allocation is initialised).
int ensure_table(gkc_ctx *ctx, uint64_t C) {
    if (C <= ctx->tcap && ctx->table.p) return GKC_OK;
    CK(cudaStreamSynchronize(ctx->s));
    ctx->table.release();
    CK(ctx->table.ensure(C * sizeof(HSlot)));
    uint32_t g = (uint32_t)std::min<uint64_t>((C + 255) / 256, (uint64_t)ctx->sms * 16);
    hash_init_kernel<<<g, 256, 0, ctx->s>>>(ctx->table.as<HSlot>(), C);
    LAUNCHED();
    ctx->tcap = C;
    return GKC_OK;
}

// Releases the pooled scratch that no counting group holds between groups:
// phase-1 batch buffers, spill staging, the record path's slices, the L2
// table, and (hash counter) the sort buffers.  Called when an allocation of
// the output fails; the buffers are allocated again when next needed.
void trim_scratch(gkc_ctx *ctx) {
    cudaStreamSynchronize(ctx->s);
    DevBuf *ds[] = {&ctx->reads[0], &ctx->reads[1], &ctx->reads[2], &ctx->offs[0], &ctx->offs[1], &ctx->offs[2],
                    &ctx->records, &ctx->codes,
                    &ctx->tile_read, &ctx->cta_hist, &ctx->cta_base, &ctx->spill_bytes[0], &ctx->spill_bytes[1],
                    &ctx->spill_idx[0], &ctx->spill_idx[1], &ctx->spill_keys[0], &ctx->spill_keys[1],
                    &ctx->stage_bytes, &ctx->stage_idx, &ctx->stage_keys, &ctx->r_work, &ctx->r_count, &ctx->r_off,
                    &ctx->r_cur, &ctx->r_recs, &ctx->r_failed, &ctx->r_stage, &ctx->r_winst, &ctx->r_woff,
                    &ctx->r_wrec, &ctx->fx_text, &ctx->fx_reads, &ctx->fx_out, &ctx->hpc_reads};
    for (auto *d : ds) d->release();
    ctx->table.release();
    ctx->tcap = 0;
    if (ctx->opt.counter == GKC_COUNTER_HASH && ctx->opt.k <= 32) {
        DevBuf *sb[] = {&ctx->keysA, &ctx->keysB, &ctx->heads_pos, &ctx->heads_key, &ctx->os_status};
        for (auto *d : sb) d->release();
    }
}

// Output capacity of at least `need` entries; a new buffer keeps the first
// `keep` entries of the old one.  If the device is short of memory, the
// pooled scratch is released (trim_scratch) and the allocation tried again.
int ensure_out(gkc_ctx *ctx, uint64_t need, uint64_t keep) {
    if (need <= ctx->out_cap && ctx->out_k.p) return GKC_OK;
    const uint64_t kb = ctx->opt.k > 32 ? 16 : 8;  // key bytes per entry
    uint64_t cap = std::max<uint64_t>(need, 1024);
    DevBuf nk, nc;
    if (nk.ensure(cap * kb) != cudaSuccess || nc.ensure(cap * 4) != cudaSuccess) {
        cudaGetLastError();  // the failed allocation's error, not sticky
        nk.release();
        nc.release();
        trim_scratch(ctx);
        CK(nk.ensure(cap * kb));
        CK(nc.ensure(cap * 4));
    }
    keep = std::min<uint64_t>(keep, ctx->out_cap);
    if (keep && ctx->out_k.p) {
        CK(cudaMemcpyAsync(nk.p, ctx->out_k.p, keep * kb, cudaMemcpyDeviceToDevice, ctx->s));
        CK(cudaMemcpyAsync(nc.p, ctx->out_c.p, keep * 4, cudaMemcpyDeviceToDevice, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
    }
    ctx->out_k.release();
    ctx->out_c.release();
    ctx->out_k = nk;
    ctx->out_c = nc;
    nk.p = nullptr;
    nc.p = nullptr;
    ctx->out_cap = cap;
    return GKC_OK;
}

// ---------------------------------------------------------------------------
// phase 1 on a device-resident batch (offs[0] == 0)
// Launch shape of phase 1 for a batch of `total` bases.
struct P1Plan {
    uint64_t ntiles = 0, tiles_per_cta = 0, cap = 0, cap_max = 0;
    uint32_t grid = 0;
    size_t dyn = 0;
    void (*kfind)(P1Params) = nullptr;
};

int p1_plan(gkc_ctx *ctx, uint64_t total, P1Plan *pl) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    pl->ntiles = (total + P1_TILE - 1) / P1_TILE;
    if (ctx->opt.k > 32)
        pl->kfind = ctx->has_lut ? find_superkmers_kernel<true, true> : find_superkmers_kernel<false, true>;
    else
        pl->kfind = ctx->has_lut ? find_superkmers_kernel<true, false> : find_superkmers_kernel<false, false>;
    pl->dyn = 3ull * P * sizeof(uint32_t);
    CK(cudaFuncSetAttribute(pl->kfind, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl->dyn));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->kfind, P1_THREADS, pl->dyn));
    pl->grid = (uint32_t)std::min<uint64_t>(pl->ntiles, (uint64_t)ctx->sms * std::max(per_sm, 1));
    pl->tiles_per_cta = (pl->ntiles + pl->grid - 1) / pl->grid;
    pl->cap = std::min<uint64_t>(pl->tiles_per_cta * P1_TILE / 4 + 4096, UINT32_MAX);  // records per CTA
    pl->cap_max = pl->tiles_per_cta * P1_TILE + 64;
    const size_t dyn2 = p2_smem(P);
    CK(cudaFuncSetAttribute(scatter_superkmers_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn2));
    // per-context buffers every batch of this size needs
    CK(ctx->region_count.ensure(pl->grid * sizeof(uint32_t)));
    CK(ctx->cta_hist.ensure(2ull * P * pl->grid * sizeof(uint32_t)));
    CK(ctx->cta_base.ensure(2ull * P * pl->grid * sizeof(unsigned long long)));
    CK(ctx->hist.ensure(3ull * P * sizeof(unsigned long long)));
    CK(ctx->tile_read.ensure(pl->ntiles * sizeof(int64_t)));
    CK(ctx->codes.ensure((pl->ntiles * P1_TILE_WORDS + 4) * sizeof(uint32_t)));
    CK(ctx->records.ensure(pl->cap * pl->grid * sizeof(SkmRecord)));
    return GKC_OK;
}

// tile_reads + find_superkmers of a batch (stream work only).
int launch_find(gkc_ctx *ctx, const P1Plan &pl, const uint8_t *d_reads, const uint64_t *d_offs, uint64_t n_reads,
                uint64_t total, uint64_t cap, uint32_t *flags) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    auto *hist = ctx->hist.as<unsigned long long>();
    if (!ctx->p1_packed) CK(cudaMemsetAsync(ctx->codes.as<uint32_t>() + pl.ntiles * P1_TILE_WORDS, 0, 16, ctx->s));
    {
        uint32_t g = (uint32_t)std::min<uint64_t>((pl.ntiles + 255) / 256, (uint64_t)ctx->sms * 8);
        tile_reads_kernel<<<g, 256, 0, ctx->s>>>(d_offs, (int64_t)n_reads, pl.ntiles, ctx->tile_read.as<int64_t>());
        LAUNCHED();
    }
    CK(cudaMemsetAsync(hist, 0, 3ull * P * sizeof(unsigned long long), ctx->s));
    CK(cudaMemsetAsync(flags, 0, 4, ctx->s));
    P1Params a;
    a.reads = d_reads;
    a.packed = ctx->p1_packed;
    a.offs = d_offs;
    a.n_reads = (int64_t)n_reads;
    a.total = total;
    a.k = ctx->opt.k;
    a.p = ctx->opt.p;
    a.P = P;
    a.pmod = fastmod_m(P);
    a.lut = ctx->has_lut ? ctx->lut.as<uint32_t>() : nullptr;
    a.vec_ok = ((uintptr_t)d_reads & 15) == 0;
    a.tile_read = ctx->tile_read.as<int64_t>();
    a.codes = ctx->codes.as<uint32_t>();
    a.records = ctx->records.as<SkmRecord>();
    a.region_cap = (uint32_t)cap;
    a.region_count = ctx->region_count.as<uint32_t>();
    a.part_bytes = hist;
    a.part_skms = hist + P;
    a.part_kmers = hist + 2 * P;
    a.cta_hist = ctx->cta_hist.as<uint32_t>();
    a.err = flags;
    // reads (ASCII in, 2-bit codes out; or packed words in) + offsets (records
    // are added by the caller)
    KScope ks(ctx, GKC_K_FIND_SUPERKMERS, (ctx->p1_packed ? 0.25 : 1.25) * (double)total + 8.0 * (n_reads + 1));
    pl.kfind<<<pl.grid, P1_THREADS, pl.dyn, ctx->s>>>(a);
    LAUNCHED();
    return GKC_OK;
}

// cta_offsets + scatter of a batch into chunk c's device buffers (stream work only).
int launch_scatter(gkc_ctx *ctx, const P1Plan &pl, StoreChunk *c, uint64_t total, uint64_t cap,
                   const uint32_t *flags, double nskm_hint, double nbytes_hint) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    {
        KScope ks(ctx, GKC_K_SCAN, 24.0 * P * pl.grid);
        cta_offsets_kernel<<<P, CO_THREADS, 0, ctx->s>>>(
            ctx->cta_hist.as<uint32_t>(), pl.grid, P, c->d_byte_off.as<unsigned long long>(),
            c->d_skm_off.as<unsigned long long>(), ctx->cta_base.as<unsigned long long>(), flags);
        LAUNCHED();
    }
    P2Params b;
    b.codes = ctx->p1_packed ? ctx->p1_packed : ctx->codes.as<uint32_t>();
    b.records = ctx->records.as<SkmRecord>();
    b.region_cap = (uint32_t)cap;
    b.region_count = ctx->region_count.as<uint32_t>();
    b.k = ctx->opt.k;
    b.P = P;
    b.pmod = fastmod_m(P);
    b.part_byte_off = c->d_byte_off.as<unsigned long long>();
    b.cta_base = ctx->cta_base.as<unsigned long long>();
    b.flags = flags;
    b.bytes = c->bytes;
    b.idx = c->idx;
    b.keys = c->keys;
    const size_t dyn2 = p2_smem(P);
    // records (16 B) and codes in; superkmer bytes, index (8 B) and keys (4 B) out
    KScope ks(ctx, GKC_K_SCATTER, 28.0 * nskm_hint + 0.25 * (double)total + nbytes_hint);
    scatter_superkmers_kernel<<<pl.grid, P2_THREADS, dyn2, ctx->s>>>(b);
    LAUNCHED();
    return GKC_OK;
}

// Waits for every spill copy in flight: called before spilled chunks are
// read, staged back, or their arena memory is rewound or freed.
int spill_sync(gkc_ctx *ctx) {
    if (ctx->ss) CK(cudaStreamSynchronize(ctx->ss));
    return GKC_OK;
}

// Device staging slot for the next spilled chunk: waits until the copy that
// last read the slot is done, then sizes it.
int spill_slot(gkc_ctx *ctx, uint64_t nbytes, uint64_t nskm, DevBuf **db, DevBuf **di, DevBuf **dk) {
    const int j = ctx->spill_slot;
    CK(cudaEventSynchronize(ctx->spill_done[j]));
    CK(ctx->spill_bytes[j].ensure(nbytes + 32));
    CK(ctx->spill_idx[j].ensure(std::max<uint64_t>(nskm, 1) * 8));
    CK(ctx->spill_keys[j].ensure(std::max<uint64_t>(nskm, 1) * 4));
    *db = &ctx->spill_bytes[j];
    *di = &ctx->spill_idx[j];
    *dk = &ctx->spill_keys[j];
    return GKC_OK;
}

// Copies a chunk from the current device staging slot (c->bytes, idx, keys,
// written on ctx->s) to pinned host memory of the context's arena, on the
// spill stream; the slot is released by spill_done when the copy ends.
// Only the superkmer bytes are kept: a spilled chunk's index entries and
// minimizer keys follow from its bytes and partition offsets, and are rebuilt
// on the device when a range of it is staged back (stage_spilled).  That
// halves the pinned memory and the PCIe traffic of a spilled store.
int spill_chunk(gkc_ctx *ctx, StoreChunk *c) {
    uint8_t *hb = nullptr;
    cudaError_t ea = ctx->arena.take(c->nbytes + 16, &hb);
    if (ea != cudaSuccess) return ctx->fail(GKC_ENOMEM, "pinned spill allocation: %s", cudaGetErrorString(ea));
    // the copy waits for the chunk's kernels, not the other way round:
    // readers of spilled chunks call spill_sync first
    CK(cudaEventRecord(ctx->spill_ready, ctx->s));
    CK(cudaStreamWaitEvent(ctx->ss, ctx->spill_ready, 0));
    CK(cudaMemcpyAsync(hb, c->bytes, c->nbytes, cudaMemcpyDeviceToHost, ctx->ss));
    CK(cudaEventRecord(ctx->spill_done[ctx->spill_slot], ctx->ss));
    ctx->spill_slot ^= 1;
    c->bytes = hb;
    c->idx = nullptr;
    c->keys = nullptr;
    c->on_host = true;
    return GKC_OK;
}

// Stages partitions [p0, p1) of spilled chunk c on stream st: its bytes to pb
// (then 32 zero bytes of padding), and its index entries and minimizer keys,
// rebuilt from the bytes by the .skm parse (skm_load.cu) under the context's
// order, to pi / pk (one per superkmer of the range, in byte order; the
// order of a partition's entries does not matter to any reader).
// Scratch of the index rebuild for a staged range of n bytes, nskm
// superkmers and np partitions.  A staging loop sizes it for its largest
// range first, so that no buffer grows (cudaFree waits for the device) while
// the staging overlaps the counting.
int stage_scratch(gkc_ctx *ctx, uint64_t n, uint64_t nskm, uint32_t np) {
    const uint64_t ntiles = (n + gkc::SL_TILE - 1) / gkc::SL_TILE;
    CK(ctx->sk_po.ensure((np + 1) * 8ull));
    CK(ctx->sk_tiles.ensure(std::max<uint64_t>(ntiles, 1) * sizeof(gkc::SlT)));
    CK(ctx->sk_state.ensure(std::max<uint64_t>(ntiles, 1)));
    CK(ctx->sk_tstarts.ensure(std::max<uint64_t>(ntiles, 1) * 8));
    CK(ctx->sk_res.ensure(64));
    CK(ctx->sk_starts.ensure(std::max<uint64_t>(nskm, 1) * 8));
    CK(ctx->sk_k32.ensure(std::max<uint64_t>(nskm, 1) * 4));
    return GKC_OK;
}

// Stages partitions [p0, p1) of spilled chunk c back to the device: the
// superkmer bytes to pb (copy, on stream st), then their index entries to pi
// and minimizer keys to pk (rebuild).  STAGE_BOTH does both on st; a staging
// loop may issue every copy first and the rebuilds on another stream.
enum { STAGE_COPY = 1, STAGE_REBUILD = 2, STAGE_BOTH = 3 };

int stage_spilled(gkc_ctx *ctx, StoreChunk *c, uint32_t p0, uint32_t p1, uint8_t *pb, uint64_t *pi, uint32_t *pk,
                  cudaStream_t st, int what = STAGE_BOTH) {
    const uint64_t b0 = c->byte_off[p0], b1 = c->byte_off[p1], s0 = c->skm_off[p0], s1 = c->skm_off[p1];
    const uint64_t n = b1 - b0, nskm = s1 - s0;
    if (what & STAGE_COPY) {
        CK(cudaMemcpyAsync(pb, c->bytes + b0, n, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(pb + n, 0, 32, st));
    }
    if (!(what & STAGE_REBUILD) || !nskm) return GKC_OK;
    const uint32_t np = p1 - p0;
    const uint64_t ntiles = (n + gkc::SL_TILE - 1) / gkc::SL_TILE;
    RET(stage_scratch(ctx, n, nskm, np));
    // the partition offsets, rebased to the staged range, from the chunk's
    // device copy (no host copy: a pageable one may wait for the stream)
    CK(cudaMemcpyAsync(ctx->sk_po.p, c->d_byte_off.as<unsigned long long>() + p0, (np + 1) * 8ull,
                       cudaMemcpyDeviceToDevice, st));
    gkc::rebase_offsets_kernel<<<1, 256, 0, st>>>(ctx->sk_po.as<uint64_t>(), np + 1, b0);
    LAUNCHED();
    CK(cudaMemsetAsync(ctx->sk_res.p, 0, 64, st));
    gkc::SlParams a;
    a.bytes = pb;
    a.n = n;
    a.part_off = ctx->sk_po.as<unsigned long long>();
    a.P = np;
    a.tiles = ctx->sk_tiles.as<gkc::SlT>();
    a.ntiles = ntiles;
    a.tile_state = ctx->sk_state.as<uint8_t>();
    a.tile_starts = ctx->sk_tstarts.as<uint64_t>();
    a.result = ctx->sk_res.as<uint64_t>();
    a.err = reinterpret_cast<uint32_t *>(ctx->sk_res.as<uint64_t>() + 1);
    a.starts = ctx->sk_starts.as<uint64_t>();
    gkc::skm_tile_kernel<<<(uint32_t)ntiles, gkc::SL_THREADS, 0, st>>>(a);
    LAUNCHED();
    gkc::skm_carry_kernel<<<1, gkc::SL_CARRY_THREADS, 0, st>>>(a);
    LAUNCHED();
    gkc::skm_starts_kernel<<<(uint32_t)ntiles, gkc::SL_THREADS, 0, st>>>(a);
    LAUNCHED();
    gkc::SiParams x;
    x.bytes = pb;
    x.n = n;
    x.part_off = a.part_off;
    x.P = np;
    x.part0 = p0;
    x.P_store = (uint32_t)ctx->opt.partitions;
    x.pmod = gkc::fastmod_m(x.P_store);
    x.k = ctx->opt.k;
    x.p = ctx->opt.p;
    x.lut = ctx->has_lut ? ctx->lut.as<uint32_t>() : nullptr;
    x.starts = a.starts;
    x.nskm = nskm;
    x.idx = pi;
    x.keys = pk;
    x.part_kmers32 = ctx->sk_k32.as<uint32_t>();
    x.err = a.err;
    const uint32_t g = (uint32_t)std::min<uint64_t>((nskm + 255) / 256, (uint64_t)ctx->sms * 8);
    if (x.lut) gkc::skm_index_kernel<true><<<g, 256, 0, st>>>(x);
    else gkc::skm_index_kernel<false><<<g, 256, 0, st>>>(x);
    LAUNCHED();
    return GKC_OK;
}

// ---------------------------------------------------------------------------
// Phase 1 of one device-resident batch (offs[0] == 0), synchronously: the
// partition totals are read back after find_superkmers and the chunk is
// allocated to the exact size.  Used for spilled stores (the chunk is then
// copied to pinned host memory) and to redo a batch that overflowed
// phase1_async's capacities.
int phase1_exact(gkc_ctx *ctx, const uint8_t *d_reads, const uint64_t *d_offs, uint64_t n_reads,
                 uint64_t total) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    if (total == 0 || n_reads == 0) return GKC_OK;
    P1Plan pl;
    RET(p1_plan(ctx, total, &pl));
    CK(ctx->flags.ensure(64));
    CK(ctx->h_hist.ensure(3ull * P * sizeof(unsigned long long)));
    CK(ctx->h_flags.ensure(64));
    auto *hh = ctx->h_hist.as<unsigned long long>();
    uint64_t cap = pl.cap;
    for (int attempt = 0;; attempt++) {
        CK(ctx->records.ensure(cap * pl.grid * sizeof(SkmRecord)));
        CK(cudaEventRecord(ctx->e0, ctx->s));
        RET(launch_find(ctx, pl, d_reads, d_offs, n_reads, total, cap, ctx->flags.as<uint32_t>()));
        CK(cudaEventRecord(ctx->e1, ctx->s));
        CK(cudaMemcpyAsync(hh, ctx->hist.p, 3ull * P * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaMemcpyAsync(ctx->h_flags.p, ctx->flags.p, 4, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->e0, ctx->e1));
        ctx->times[1] += ms;
        uint32_t f = *ctx->h_flags.as<uint32_t>();
        if (f & ERR_SKM_TOO_LONG) return ctx->fail(GKC_EINVAL, "a superkmer exceeds %u k-mers", IDX_MAX_LEN);
        if (f & ERR_RECORD_OVERFLOW) {
            if (cap >= pl.cap_max || attempt >= 3)
                return ctx->fail(GKC_EINTERNAL, "superkmer record region overflow at capacity %llu",
                                 (unsigned long long)cap);
            cap = std::min<uint64_t>(std::min<uint64_t>(cap * 4, pl.cap_max), UINT32_MAX);
            continue;
        }
        break;
    }
    // ---- partition offsets, store chunk ----
    StoreChunk *c = ctx->take_chunk();
    c->byte_off.assign(P + 1, 0);
    c->skm_off.assign(P + 1, 0);
    c->kmers.assign(P, 0);
    for (uint32_t i = 0; i < P; i++) {
        c->byte_off[i + 1] = c->byte_off[i] + hh[i];
        c->skm_off[i + 1] = c->skm_off[i] + hh[P + i];
        c->kmers[i] = hh[2 * P + i];
    }
    c->nbytes = c->byte_off[P];
    c->nskm = c->skm_off[P];
    c->on_host = false;
    c->pending = false;
    if (ctx->prof && !ctx->pend.empty()) ctx->pend.back().bytes += 16.0 * c->nskm;  // records written
    // a spilled chunk is scattered into shared device staging, then copied out
    DevBuf *db = &c->dbytes, *di = &c->didx, *dk = &c->dkeys;
    if (ctx->opt.spill_host) {
        const int rc = spill_slot(ctx, c->nbytes, c->nskm, &db, &di, &dk);
        if (rc != GKC_OK) {
            ctx->pool.push_back(c);
            return rc;
        }
    }
    cudaError_t e1 = db->ensure(c->nbytes + 32);
    cudaError_t e2 = e1 == cudaSuccess ? di->ensure(std::max<uint64_t>(c->nskm, 1) * 8) : e1;
    cudaError_t e2k = e2 == cudaSuccess ? dk->ensure(std::max<uint64_t>(c->nskm, 1) * 4) : e2;
    cudaError_t e3 = e2k == cudaSuccess ? c->d_byte_off.ensure((P + 1) * 8) : e2k;
    cudaError_t e4 = e3 == cudaSuccess ? c->d_skm_off.ensure((P + 1) * 8) : e3;
    if (e4 != cudaSuccess) {
        ctx->pool.push_back(c);
        return ctx->fail(GKC_ENOMEM, "store chunk allocation (%llu bytes): %s",
                         (unsigned long long)c->nbytes, cudaGetErrorString(e4));
    }
    c->bytes = db->as<uint8_t>();
    c->idx = di->as<uint64_t>();
    c->keys = dk->as<uint32_t>();
    CK(cudaMemcpyAsync(c->d_byte_off.p, c->byte_off.data(), (P + 1) * 8, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemcpyAsync(c->d_skm_off.p, c->skm_off.data(), (P + 1) * 8, cudaMemcpyHostToDevice, ctx->s));
    RET(launch_scatter(ctx, pl, c, total, cap, ctx->flags.as<uint32_t>(), (double)c->nskm, (double)c->nbytes));
    if (ctx->opt.spill_host) {
        const int rc = spill_chunk(ctx, c);
        if (rc != GKC_OK) {
            ctx->pool.push_back(c);
            return rc;
        }
    }
    ctx->store.push_back(c);
    return GKC_OK;
}

// Phase 1 of one device-resident batch without waiting for the device: the
// chunk gets capacity for 2 bytes and 0.25 superkmers per base (typical data
// needs about 1.2 and 0.09), the layout is computed on the device
// (part_offsets_kernel), and the batch's launches are captured into one CUDA
// graph and launched.  `rebase` != 0 first subtracts it from the batch's
// offsets (a slice of the caller's offsets).  The chunk's layout is copied back
// to pinned memory; phase1_finish reads it after the stream is synchronised.
int phase1_async(gkc_ctx *ctx, const uint8_t *d_reads, uint64_t *d_offs, uint64_t n_reads, uint64_t total,
                 uint64_t rebase, uint64_t batch) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    if (total == 0 || n_reads == 0) return GKC_OK;
    P1Plan pl;
    RET(p1_plan(ctx, total, &pl));
    const uint64_t byte_cap = 2 * total + 65536, skm_cap = total / 4 + 4096;
    StoreChunk *c = ctx->take_chunk();
    cudaError_t e = c->dbytes.ensure(byte_cap + 32);
    if (e == cudaSuccess) e = c->didx.ensure(skm_cap * 8);
    if (e == cudaSuccess) e = c->dkeys.ensure(skm_cap * 4);
    if (e == cudaSuccess) e = c->d_byte_off.ensure((P + 1) * 8);
    if (e == cudaSuccess) e = c->d_skm_off.ensure((P + 1) * 8);
    if (e == cudaSuccess) e = c->d_kmers.ensure(P * 8ull);
    if (e == cudaSuccess) e = c->d_flags.ensure(64);
    if (e == cudaSuccess) e = c->h_meta.ensure((3ull * P + 3) * 8);
    if (e != cudaSuccess) {
        ctx->pool.push_back(c);
        return ctx->fail(GKC_ENOMEM, "store chunk allocation: %s", cudaGetErrorString(e));
    }
    c->bytes = c->dbytes.as<uint8_t>();
    c->idx = c->didx.as<uint64_t>();
    c->keys = c->dkeys.as<uint32_t>();
    c->on_host = false;
    c->batch = batch;
    uint32_t *flags = c->d_flags.as<uint32_t>();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    c->bases = total;
    c->pend_find = c->pend_scatter = -1;
    auto work = [&]() -> int {
        if (rebase) {
            const uint32_t g = (uint32_t)std::min<uint64_t>((n_reads + 256) / 256, (uint64_t)ctx->sms * 8);
            rebase_offsets_kernel<<<g, 256, 0, ctx->s>>>(d_offs, n_reads + 1, rebase);
            LAUNCHED();
        }
        RET(launch_find(ctx, pl, d_reads, d_offs, n_reads, total, pl.cap, flags));
        if (ctx->prof) c->pend_find = (int64_t)ctx->pend.size() - 1;
        part_offsets_kernel<<<1, PO_THREADS, 0, ctx->s>>>(
            ctx->hist.as<unsigned long long>(), P, byte_cap, skm_cap, c->d_byte_off.as<unsigned long long>(),
            c->d_skm_off.as<unsigned long long>(), c->d_kmers.as<unsigned long long>(), flags);
        LAUNCHED();
        RET(launch_scatter(ctx, pl, c, total, pl.cap, flags, 0.09 * (double)total, 1.2 * (double)total));
        if (ctx->prof) c->pend_scatter = (int64_t)ctx->pend.size() - 1;
        return GKC_OK;
    };
    if (ctx->prof) {
        // profiling brackets each launch with timing events, which do not time
        // inside a graph: the same launches go straight to the stream
        const int rc = work();
        if (rc != GKC_OK) {
            ctx->pool.push_back(c);
            return rc;
        }
    } else {
        CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
        const int rc = work();
        const cudaError_t ec = cudaStreamEndCapture(ctx->s, &graph);  // also ends a capture that failed
        if (rc != GKC_OK || ec != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            ctx->pool.push_back(c);
            return rc != GKC_OK ? rc : ctx->fail(GKC_ECUDA, "phase-1 graph capture: %s", cudaGetErrorString(ec));
        }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec, ctx->s);
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ctx->pool.push_back(c);
            return ctx->fail(GKC_ECUDA, "phase-1 graph launch: %s", cudaGetErrorString(e));
        }
    }
    auto *hm = c->h_meta.as<unsigned long long>();
    CK(cudaMemcpyAsync(hm, c->d_byte_off.p, (P + 1) * 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(hm + P + 1, c->d_skm_off.p, (P + 1) * 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(hm + 2 * P + 2, c->d_kmers.p, P * 8ull, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(hm + 3 * P + 2, c->d_flags.p, 4, cudaMemcpyDeviceToHost, ctx->s));
    c->pending = true;
    ctx->store.push_back(c);
    return GKC_OK;
}

// After the stream is synchronised: fills the host view of every chunk
// phase1_async wrote.  Chunks that overflowed are taken out of the store;
// their batches are listed in `redo` (the caller runs them with phase1_exact).
int phase1_finish(gkc_ctx *ctx, std::vector<uint64_t> *redo) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    std::vector<StoreChunk *> keep;
    int rc = GKC_OK;
    for (StoreChunk *c : ctx->store) {
        if (!c->pending) {
            keep.push_back(c);
            continue;
        }
        c->pending = false;
        const auto *hm = c->h_meta.as<unsigned long long>();
        const uint32_t f = (uint32_t)hm[3 * P + 2];
        if (f & ERR_SKM_TOO_LONG) rc = ctx->fail(GKC_EINVAL, "a superkmer exceeds %u k-mers", IDX_MAX_LEN);
        if (f & (ERR_RECORD_OVERFLOW | ERR_CAPACITY)) {
            redo->push_back(c->batch);
            ctx->pool.push_back(c);
            continue;
        }
        c->byte_off.assign(hm, hm + P + 1);
        c->skm_off.assign(hm + P + 1, hm + 2 * P + 2);
        c->kmers.assign(hm + 2 * P + 2, hm + 3 * P + 2);
        c->nbytes = c->byte_off[P];
        c->nskm = c->skm_off[P];
        // profiled launches: the byte models' superkmer terms, now known
        // (records written by find; records, index, keys and bytes by scatter)
        if (c->pend_find >= 0 && (size_t)c->pend_find < ctx->pend.size())
            ctx->pend[c->pend_find].bytes += 16.0 * (double)c->nskm;
        if (c->pend_scatter >= 0 && (size_t)c->pend_scatter < ctx->pend.size())
            ctx->pend[c->pend_scatter].bytes = 28.0 * (double)c->nskm + 0.25 * (double)c->bases + (double)c->nbytes;
        c->pend_find = c->pend_scatter = -1;
        keep.push_back(c);
    }
    ctx->store.swap(keep);
    return rc;
}

// Device pointers of the superkmers of partitions [p0, p1) of chunk c, indexed
// by the chunk's own partition offsets (spilled chunks are staged into `arena`
// at *arena_used and the pointers rebased).
int chunk_range(gkc_ctx *ctx, StoreChunk *c, uint32_t p0, uint32_t p1, DevBuf &arena, uint64_t *arena_used,
                const uint8_t **bytes, const uint64_t **idx, const uint32_t **keys, cudaStream_t st = nullptr,
                int what = STAGE_BOTH) {
    if (!st) st = ctx->s;
    if (!c->on_host) {
        *bytes = c->bytes;
        *idx = c->idx;
        *keys = c->keys;
        return GKC_OK;
    }
    const uint64_t b0 = c->byte_off[p0], b1 = c->byte_off[p1], s0 = c->skm_off[p0], s1 = c->skm_off[p1];
    // bytes (+32 B of padding), index and keys, each 16-byte aligned so the
    // next chunk's index stays 8-byte aligned
    auto a16 = [](uint64_t x) { return (x + 15) / 16 * 16; };
    const uint64_t nbb = a16(b1 - b0 + 32), nib = a16((s1 - s0) * 8), nkb = a16((s1 - s0) * 4);
    const uint64_t need = nbb + nib + nkb;
    if (*arena_used + need > arena.cap) return ctx->fail(GKC_EINTERNAL, "staging arena too small");
    uint8_t *base = arena.as<uint8_t>() + *arena_used;
    uint8_t *pb = base;
    uint64_t *pi = reinterpret_cast<uint64_t *>(base + nbb);
    uint32_t *pk = reinterpret_cast<uint32_t *>(base + nbb + nib);
    RET(stage_spilled(ctx, c, p0, p1, pb, pi, pk, st, what));
    *arena_used += need;
    // the kernels index with the chunk's absolute offsets: rebase
    *bytes = pb - b0;
    *idx = pi - s0;
    *keys = pk - s0;
    return GKC_OK;
}

// Counts the sub-buckets listed in `ids` through the L2 hash table (the
// sub-buckets whose distinct k-mers outgrew shared memory).
int count_buckets_l2(gkc_ctx *ctx, const std::vector<uint32_t> &ids, const std::vector<uint64_t> &off,
                     uint32_t cmin, uint32_t cmax) {
    const double slots = ctx->opt.table_slots > 0 ? ctx->opt.table_slots : 0.35;
    auto *sc = ctx->scal.as<unsigned long long>();  // [0] cursor [1] distinct [2] err
    for (uint32_t b : ids) {
        const uint64_t e0 = off[b], e1 = off[b + 1];
        for (int scale = 1;; scale *= 4) {
            // ~12 k-mers per superkmer; an undersized table is retried larger
            uint64_t C = next_pow2(std::max<uint64_t>(4096, (uint64_t)((double)(e1 - e0) * 12.0 * slots) * scale));
            RET(ensure_table(ctx, C));
            CK(cudaMemsetAsync(ctx->part_err.p, 0, 4, ctx->s));
            {
                uint32_t g = (uint32_t)std::min<uint64_t>((e1 - e0 + 63) / 64, (uint64_t)ctx->sms * 8);
                KScope ks(ctx, GKC_K_HASH_INSERT, 16.0 * (e1 - e0));
                hash_insert_entries_kernel<<<std::max(g, 1u), H_THREADS, 0, ctx->s>>>(
                    ctx->bk_entries.as<BEntry>() + e0, e1 - e0, ctx->opt.k, ctx->table.as<HSlot>(), C - 1,
                    ctx->part_err.as<uint32_t>());
                LAUNCHED();
            }
            HCollectParams q;
            q.tab = ctx->table.as<HSlot>();
            q.cap = C;
            q.cmin = cmin;
            q.cmax = cmax;
            q.out_k = ctx->out_k.as<uint64_t>();
            q.out_c = ctx->out_c.as<uint32_t>();
            q.out_cursor = sc;
            q.out_cap = ctx->out_cap;
            q.distinct = sc + 1;
            q.err = reinterpret_cast<uint32_t *>(sc + 2);
            q.part_err = ctx->part_err.as<uint32_t>();
            {
                uint32_t g = (uint32_t)std::min<uint64_t>((C + H_THREADS * HC_ITEMS - 1) / (H_THREADS * HC_ITEMS),
                                                          (uint64_t)ctx->sms * 8);
                KScope ks(ctx, GKC_K_HASH_COLLECT, 32.0 * C);
                hash_collect_kernel<<<g, H_THREADS, 0, ctx->s>>>(q);
                LAUNCHED();
            }
            uint32_t perr = 0;
            CK(cudaMemcpyAsync(&perr, ctx->part_err.p, 4, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            if (!(perr & ERR_TABLE_FULL)) break;
            if (scale >= 256) return ctx->fail(GKC_EINTERNAL, "hash table retries exhausted");
        }
    }
    return GKC_OK;
}

constexpr int BC_TS = 8192;    // shared-memory table slots per CTA (96 KB)
constexpr int BC_TS2 = 16384;  // second pass over the sub-buckets that overflowed (192 KB, one CTA per SM)
// sub-buckets of more k-mer instances go to the record split (8x the 8k
// instances a sub-bucket is sized for: only a minimizer that dominates its
// sub-bucket, as in a low-complexity run, makes one this large)
constexpr uint64_t BC_HEAVY_KMERS = 65536;

// Counts the minimizer sub-buckets `ids` that overflowed shared memory or are
// heavy: their k-mers are re-split by k-mer hash into record sub-buckets of
// at most 4k instances, counted in shared memory; record sub-buckets that
// still overflow go through the L2 table.
int count_buckets_records_slice(gkc_ctx *ctx, const std::vector<uint32_t> &ids, const std::vector<uint64_t> &off,
                                const std::vector<uint64_t> &bk_kmers, uint32_t cmin, uint32_t cmax) {
    std::vector<RWork> work;
    uint64_t NR = 0, inst = 0, ents = 0;
    for (uint32_t b : ids) {
        const uint64_t kb = bk_kmers[b];
        // at least two record sub-buckets of at most 4k instances each, so a
        // table stays at most half full even when every k-mer is distinct
        uint32_t r_log = 1;
        while (r_log < (uint32_t)RS_MAX_LOG && kb / (1ull << r_log) > 4096) r_log++;
        for (uint64_t e = off[b]; e < off[b + 1]; e += RW_ENTRIES)
            work.push_back({e, std::min<uint64_t>(e + RW_ENTRIES, off[b + 1]), (uint32_t)NR, r_log});
        NR += 1ull << r_log;
        inst += kb;
        ents += off[b + 1] - off[b];
    }
    if (work.empty()) return GKC_OK;
    const uint32_t nw = (uint32_t)work.size();
    CK(ctx->r_work.ensure(nw * sizeof(RWork)));
    CK(ctx->r_count.ensure(NR * 4));
    CK(ctx->r_off.ensure((NR + 1) * 8));
    CK(ctx->r_cur.ensure(NR * 8));
    CK(ctx->r_recs.ensure(std::max<uint64_t>(inst, 1) * sizeof(KRec)));
    CK(ctx->r_stage.ensure(std::max<uint64_t>(inst, 1) * sizeof(KRec)));
    CK(ctx->r_winst.ensure(nw * 4));
    CK(ctx->r_woff.ensure((nw + 1) * 8));
    CK(ctx->r_wrec.ensure(nw * 4));
    CK(ctx->r_failed.ensure((NR + 1) * 4));
    // (a slice ends with a wait on the stream, so the pinned work list of the
    // slice before has been copied)
    CK(ctx->h_work.ensure(nw * sizeof(RWork)));
    std::memcpy(ctx->h_work.p, work.data(), nw * sizeof(RWork));
    CK(cudaMemcpyAsync(ctx->r_work.p, ctx->h_work.p, nw * sizeof(RWork), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemsetAsync(ctx->r_count.p, 0, NR * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->r_failed.p, 0, 4, ctx->s));
    auto *sc = ctx->scal.as<unsigned long long>();
    {
        KScope ks(ctx, GKC_K_HASH_RECORDS, 16.0 * (double)ents + 4.0 * nw);
        work_inst_kernel<<<(nw + 7) / 8, 256, 0, ctx->s>>>(ctx->bk_entries.as<BEntry>(), ctx->r_work.as<RWork>(),
                                                            nw, ctx->r_winst.as<uint32_t>());
        LAUNCHED();
    }
    RET(scan_u32(ctx, ctx->r_winst.as<uint32_t>(), nw, ctx->r_woff.as<uint64_t>(),
                 ctx->r_woff.as<unsigned long long>() + nw));
    {
        RAggParams ap;
        ap.entries = ctx->bk_entries.as<BEntry>();
        ap.work = ctx->r_work.as<RWork>();
        ap.woff = ctx->r_woff.as<uint64_t>();
        ap.k = ctx->opt.k;
        ap.stage = ctx->r_stage.as<KRec>();
        ap.wrec = ctx->r_wrec.as<uint32_t>();
        ap.rcount = ctx->r_count.as<uint32_t>();
        CK(cudaFuncSetAttribute(rec_agg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RA_SMEM));
        KScope ks(ctx, GKC_K_HASH_RECORDS, 16.0 * inst);
        rec_agg_kernel<<<nw, RSP_THREADS, RA_SMEM, ctx->s>>>(ap);
        LAUNCHED();
    }
    RET(scan_u32(ctx, ctx->r_count.as<uint32_t>(), NR, ctx->r_off.as<uint64_t>(),
                 ctx->r_off.as<unsigned long long>() + NR));
    CK(cudaMemcpyAsync(ctx->r_cur.p, ctx->r_off.p, NR * 8, cudaMemcpyDeviceToDevice, ctx->s));
    {
        RScatterParams rp;
        rp.work = ctx->r_work.as<RWork>();
        rp.woff = ctx->r_woff.as<uint64_t>();
        rp.wrec = ctx->r_wrec.as<uint32_t>();
        rp.stage = ctx->r_stage.as<KRec>();
        rp.rcursor = ctx->r_cur.as<unsigned long long>();
        rp.recs = ctx->r_recs.as<KRec>();
        KScope ks(ctx, GKC_K_HASH_RECORDS, 32.0 * inst);
        rec_scatter_kernel<<<nw, RSP_THREADS, 0, ctx->s>>>(rp);
        LAUNCHED();
    }
    // records after pre-aggregation: one counting CTA per RC_WINDOW of them
    uint64_t nrec = 0;
    CK(cudaMemcpyAsync(&nrec, ctx->r_off.as<uint64_t>() + NR, 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const uint64_t nwin = std::max<uint64_t>(1, (nrec + RC_WINDOW - 1) / RC_WINDOW);
    CK(ctx->r_failed.ensure((std::max<uint64_t>(NR, nwin) + 1) * 4));
    RCountParams cp;
    cp.recs = ctx->r_recs.as<KRec>();
    cp.roff = ctx->r_off.as<uint64_t>();
    cp.nr = NR;
    cp.cmin = cmin;
    cp.cmax = cmax;
    cp.out_k = ctx->out_k.as<uint64_t>();
    cp.out_c = ctx->out_c.as<uint32_t>();
    cp.out_cursor = sc;
    cp.out_cap = ctx->out_cap;
    cp.distinct = sc + 1;
    cp.failed = ctx->r_failed.as<uint32_t>();
    cp.err = reinterpret_cast<uint32_t *>(sc + 2);
    CK(cudaFuncSetAttribute(rec_count_kernel<BC_TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, BC_TS * 12));
    {
        KScope ks(ctx, GKC_K_HASH_RECORDS, 16.0 * nrec);
        rec_count_kernel<BC_TS><<<(unsigned)nwin, BC_THREADS, BC_TS * 12, ctx->s>>>(cp);
        LAUNCHED();
    }
    uint32_t nfail = 0;
    CK(cudaMemcpyAsync(&nfail, ctx->r_failed.p, 4, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    if (!nfail) return GKC_OK;
    CK(ctx->h_ids.ensure(nfail * 4ull));
    CK(ctx->h_off.ensure((NR + 1) * 8));
    CK(cudaMemcpyAsync(ctx->h_ids.p, ctx->r_failed.as<uint32_t>() + 1, nfail * 4, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(ctx->h_off.p, ctx->r_off.p, (NR + 1) * 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const std::vector<uint32_t> rids(ctx->h_ids.as<uint32_t>(), ctx->h_ids.as<uint32_t>() + nfail);
    const std::vector<uint64_t> roff(ctx->h_off.as<uint64_t>(), ctx->h_off.as<uint64_t>() + NR + 1);
    const double slots = ctx->opt.table_slots > 0 ? ctx->opt.table_slots : 0.35;
    for (uint32_t r : rids) {
        // the records of window r, as rec_count_kernel chose them
        const uint64_t lo = std::lower_bound(roff.begin(), roff.end(), r * RC_WINDOW) - roff.begin();
        const uint64_t hi = std::min<uint64_t>(
            std::lower_bound(roff.begin(), roff.end(), (r + 1) * RC_WINDOW) - roff.begin(), NR);
        if (lo >= hi) continue;
        const uint64_t e0 = roff[lo], e1 = roff[hi];
        for (int scale = 1;; scale *= 4) {
            uint64_t C = next_pow2(std::max<uint64_t>(4096, (uint64_t)((double)(e1 - e0) * 3.0 * slots) * scale));
            RET(ensure_table(ctx, C));
            CK(cudaMemsetAsync(ctx->part_err.p, 0, 4, ctx->s));
            {
                uint32_t g = (uint32_t)std::min<uint64_t>((e1 - e0 + H_THREADS - 1) / H_THREADS, (uint64_t)ctx->sms * 8);
                KScope ks(ctx, GKC_K_HASH_INSERT, 16.0 * (e1 - e0));
                hash_insert_records_kernel<<<std::max(g, 1u), H_THREADS, 0, ctx->s>>>(
                    ctx->r_recs.as<KRec>() + e0, e1 - e0, ctx->table.as<HSlot>(), C - 1, ctx->part_err.as<uint32_t>());
                LAUNCHED();
            }
            HCollectParams q;
            q.tab = ctx->table.as<HSlot>();
            q.cap = C;
            q.cmin = cmin;
            q.cmax = cmax;
            q.out_k = ctx->out_k.as<uint64_t>();
            q.out_c = ctx->out_c.as<uint32_t>();
            q.out_cursor = sc;
            q.out_cap = ctx->out_cap;
            q.distinct = sc + 1;
            q.err = reinterpret_cast<uint32_t *>(sc + 2);
            q.part_err = ctx->part_err.as<uint32_t>();
            {
                uint32_t g = (uint32_t)std::min<uint64_t>((C + H_THREADS * HC_ITEMS - 1) / (H_THREADS * HC_ITEMS),
                                                          (uint64_t)ctx->sms * 8);
                KScope ks(ctx, GKC_K_HASH_COLLECT, 32.0 * C);
                hash_collect_kernel<<<g, H_THREADS, 0, ctx->s>>>(q);
                LAUNCHED();
            }
            uint32_t perr = 0;
            CK(cudaMemcpyAsync(&perr, ctx->part_err.p, 4, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            if (!(perr & ERR_TABLE_FULL)) break;
            if (scale >= 256) return ctx->fail(GKC_EINTERNAL, "hash table retries exhausted");
        }
    }
    return GKC_OK;
}

// The record path holds two 16-byte records per k-mer instance of its
// sub-buckets (staged and sorted): heavy sub-buckets are counted in slices
// whose records fit the free device memory.  A sub-bucket's k-mers are all in
// that sub-bucket, so slices are independent.
int count_buckets_records(gkc_ctx *ctx, const std::vector<uint32_t> &ids, const std::vector<uint64_t> &off,
                          const std::vector<uint64_t> &bk_kmers, uint32_t cmin, uint32_t cmax) {
    uint64_t inst = 0;
    for (uint32_t b : ids) inst += bk_kmers[b];
    uint64_t cap_inst = ~0ull;
    if ((double)inst * 40 > 0.3 * (double)ctx->free_hint) {  // large: size the slices from the memory free now
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        const uint64_t avail = fr + ctx->r_recs.cap + ctx->r_stage.cap;  // the record buffers are reallocated
        cap_inst = std::max<uint64_t>(1ull << 22, (uint64_t)(avail * 0.6) / 40);
    }
    // GKC_RECORD_SLICE=n caps a slice at n instances, so that tests can make
    // small inputs take several slices
    if (const char *rs = getenv("GKC_RECORD_SLICE")) cap_inst = std::max<uint64_t>(1, strtoull(rs, nullptr, 10));
    std::vector<uint32_t> slice;
    uint64_t acc = 0;
    for (uint32_t b : ids) {
        if (!slice.empty() && acc + bk_kmers[b] > cap_inst) {
            RET(count_buckets_records_slice(ctx, slice, off, bk_kmers, cmin, cmax));
            slice.clear();
            acc = 0;
        }
        slice.push_back(b);
        acc += bk_kmers[b];
    }
    if (!slice.empty()) RET(count_buckets_records_slice(ctx, slice, off, bk_kmers, cmin, cmax));
    return GKC_OK;
}

// ---------------------------------------------------------------------------
// phase 2, hash counter: shared-memory counting of minimizer sub-buckets, with
// the L2 table for sub-buckets that overflow shared memory.  Device-resident
// stores are counted in one group; a spilled store in groups of partitions
// whose superkmers fit the device staging budget.

// want: the partitions to count (null: all)
int count_hash(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, const std::vector<char> *want) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    std::vector<uint64_t> np(P, 0), nbp(P, 0), nsp(P, 0);
    bool spilled = false;
    for (auto *c : ctx->store) {
        spilled |= c->on_host;
        for (uint32_t p = 0; p < P; p++) {
            np[p] += c->kmers[p];
            nbp[p] += c->byte_off[p + 1] - c->byte_off[p];
            nsp[p] += c->skm_off[p + 1] - c->skm_off[p];
        }
    }
    uint64_t N = 0, NS = 0;
    for (uint32_t p = 0; p < P; p++) N += np[p], NS += nsp[p];
    // sub-buckets of partition p: 2^s_p of about 8k k-mer instances each (4k
    // to 8k), so that a sub-bucket's distinct k-mers (a fraction of its
    // instances) fit the table.  A sub-bucket that outgrows it goes to the
    // record path, which costs several times its decode: halving the target
    // from 16k cut phase 2 by a third on bacterial_100m (60 -> 40 ms per
    // 3 Gbp) and by 3% on skewed_200m, where doubling it cost 26%.
    constexpr uint64_t SUB_BUCKET_KMERS = 8192;
    std::vector<uint32_t> slog(2 * P);  // [0, P) s_p, [P, 2P) first sub-bucket of p
    uint64_t NB = 0;
    for (uint32_t p = 0; p < P; p++) {
        uint32_t sl = 0;
        while (!ctx->opt.hash_l2_only && sl < (uint32_t)BS_LOG_LIMIT && np[p] > (SUB_BUCKET_KMERS << sl)) sl++;
        slog[p] = sl;
        slog[P + p] = (uint32_t)NB;
        NB += 1ull << sl;
    }
    auto bbase = [&](uint32_t p) -> uint64_t { return p < P ? slog[P + p] : NB; };
    ctx->times[4] = (double)NB;
    ctx->times[5] = 0;
    ctx->times[8] = 0;
    float stage_ms = 0;  // host-to-device staging of spilled chunks
    uint64_t groups = 0;
    // output capacity, grown per group from the kept k-mers per instance of
    // the groups before (at first the bound 1/cmin), at most 25% of free
    // device memory; a group whose output overflows is counted again with
    // the capacity its cursor asked for
    size_t free0 = 0;
    {
        size_t tot = 0;
        CK(cudaMemGetInfo(&free0, &tot));
    }
    ctx->free_hint = free0;
    const uint64_t out_budget = std::max<uint64_t>(1ull << 24, (uint64_t)(free0 * 0.25) / 12);
    double kept_ratio = 1.0 / std::max<uint32_t>(cmin, 1);
    // GKC_OUT_ESTIMATE=n sets each group's first output estimate to n - 1
    // entries, so that tests can make every group overflow and be redone
    const char *oe = getenv("GKC_OUT_ESTIMATE");
    const uint64_t out_est_override = oe ? strtoull(oe, nullptr, 10) : 0;
    uint64_t out_used = ctx->n_out;  // entries written before this group
    uint64_t distinct_used = 0;      // distinct k-mers of the groups before
    int redo = 0;                    // times the current group was counted again
    CK(ctx->bk_skms.ensure(NB * 4));
    CK(ctx->bk_kmers.ensure(NB * 8));
    CK(ctx->bk_off.ensure((NB + 1) * 8));
    CK(ctx->bk_cur.ensure(NB * 8));
    CK(ctx->bk_failed.ensure((NB + 1) * 4));
    CK(ctx->bk_part.ensure(2ull * P * 4));
    CK(cudaMemcpyAsync(ctx->bk_part.p, slog.data(), 2ull * P * 4, cudaMemcpyHostToDevice, ctx->s));
    CK(ctx->part_err.ensure(std::max<uint32_t>(P, 16) * 4));
    CK(ctx->scal.ensure(64));
    CK(ctx->h_scal.ensure(64));
    CK(cudaMemsetAsync(ctx->scal.p, 0, 64, ctx->s));
    auto *sc = ctx->scal.as<unsigned long long>();
    CK(cudaMemcpyAsync(sc, &ctx->n_out, 8, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaFuncSetAttribute(bucket_count_persistent_kernel<BC_TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            BC_TS * 14));
    CK(cudaFuncSetAttribute(bucket_count_persistent_kernel<BC_TS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared));
    int bc_per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bc_per_sm, bucket_count_persistent_kernel<BC_TS>, BC_THREADS,
                                                     BC_TS * 14));
    CK(ctx->bk_next.ensure(8));
    CK(cudaFuncSetAttribute(bucket_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BS_SMEM));
    // groups of partitions
    // a spilled store holds two staging arenas (this group's and the next's)
    uint64_t budget = spilled ? std::max<uint64_t>(1ull << 26, (uint64_t)(free0 * 0.1)) : ~0ull;
    // streamed output: groups of 1/2, 1/4, 1/8 and 1/16 of the store, then
    // the rest, so that each group's output is copied to the host while the
    // next one counts (a group's copy takes about 0.4 of its counting time)
    // and only the last, small group's copy is exposed
    const bool stream_out = ctx->stream_k && ctx->stream_c;
    uint64_t stream_tot = 0;
    if (stream_out)
        for (uint32_t p = 0; p < P; p++) stream_tot += nbp[p] + 12 * nsp[p];  // as a group's gb counts
    auto group_budget = [&](size_t g) -> uint64_t {
        if (!stream_out) return budget;
        return std::min<uint64_t>(budget, (stream_tot >> (std::min<size_t>(g, 3) + 1)) + 1);
    };
    float acc_ms = 0;
    // the groups of partitions, formed up front
    struct Grp {
        uint32_t p0, p1;
        uint64_t gb, gs;  // staged bytes, superkmers
    };
    std::vector<Grp> grps;
    for (uint32_t q0 = 0; q0 < P;) {
        if (want && !(*want)[q0]) {
            q0++;
            continue;
        }
        uint32_t q1 = q0;
        uint64_t gb = 0, gs = 0;
        const uint64_t gbud = group_budget(grps.size());
        while (q1 < P && (!want || (*want)[q1]) &&
               (q1 == q0 || gb + nbp[q1] + 12 * nsp[q1] + 16 * nsp[q1] <= gbud)) {
            gb += nbp[q1] + 12 * nsp[q1];
            gs += nsp[q1];
            q1++;
        }
        if (gs) grps.push_back({q0, q1, gb, gs});
        q0 = q1;
    }
    // Spilled store: group g's chunk ranges are staged into arena g % 2 on the
    // copy stream, and group g + 1's are staged while group g counts.  The
    // counting waits for its staging; the staging into an arena waits for the
    // end of the group that used it before.
    const size_t nst = ctx->store.size();
    DevBuf *arena[2] = {&ctx->bk_arena, &ctx->bk_arena2};
    std::vector<const uint8_t *> cbs[2];
    std::vector<const uint64_t *> cis[2];
    std::vector<const uint32_t *> cks[2];
    cudaEvent_t staged[2] = {nullptr, nullptr}, freed[2] = {nullptr, nullptr}, st0[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    long staged_g[2] = {-1, -1};
    struct EvBack {  // the events go back to the pool on every exit
        gkc_ctx *c;
        cudaEvent_t *e[4];
        ~EvBack() {
            for (auto *a : e)
                for (int i = 0; i < 2; i++)
                    if (a[i]) c->evpool.push_back(a[i]);
        }
    } evback{ctx, {staged, freed, st0, copied}};
    if (spilled) {
        uint64_t mx = 0;
        for (const auto &g : grps) mx = std::max<uint64_t>(mx, g.gb);
        uint64_t mn = 0, ms = 0;  // largest staged range of one chunk
        uint32_t mp = 0;
        for (const auto &g : grps)
            for (auto *c : ctx->store) {
                mn = std::max<uint64_t>(mn, c->byte_off[g.p1] - c->byte_off[g.p0]);
                ms = std::max<uint64_t>(ms, c->skm_off[g.p1] - c->skm_off[g.p0]);
                mp = std::max<uint32_t>(mp, g.p1 - g.p0);
            }
        RET(stage_scratch(ctx, mn, ms, mp));
        for (int i = 0; i < 2; i++) {
            // each chunk's range adds at most 32 + 3 x 15 bytes of padding
            CK(arena[i]->ensure(mx + 96 * nst + 64));
            cbs[i].resize(nst);
            cis[i].resize(nst);
            cks[i].resize(nst);
            staged[i] = ctx->take_event();
            freed[i] = ctx->take_event();
            st0[i] = ctx->take_event();
            copied[i] = ctx->take_event();
            CK(cudaEventRecord(freed[i], ctx->s));
        }
    }
    // a group's copies go back to back on the copy stream; its index
    // rebuilds follow on the rebuild stream, beside the next group's copies
    auto stage = [&](size_t gi) -> int {
        const int sl = (int)(gi & 1);
        uint64_t used = 0;
        CK(cudaStreamWaitEvent(ctx->cs, freed[sl], 0));
        CK(cudaEventRecord(st0[sl], ctx->cs));
        for (size_t j = 0; j < nst; j++)
            RET(chunk_range(ctx, ctx->store[j], grps[gi].p0, grps[gi].p1, *arena[sl], &used, &cbs[sl][j],
                            &cis[sl][j], &cks[sl][j], ctx->cs, STAGE_COPY));
        CK(cudaEventRecord(copied[sl], ctx->cs));
        CK(cudaStreamWaitEvent(ctx->rs, copied[sl], 0));
        used = 0;
        for (size_t j = 0; j < nst; j++)
            RET(chunk_range(ctx, ctx->store[j], grps[gi].p0, grps[gi].p1, *arena[sl], &used, &cbs[sl][j],
                            &cis[sl][j], &cks[sl][j], ctx->rs, STAGE_REBUILD));
        CK(cudaEventRecord(staged[sl], ctx->rs));
        staged_g[sl] = (long)gi;
        return GKC_OK;
    };
    // host copies of the sub-bucket offsets and k-mer counts, filled group by
    // group over each group's own range of sub-buckets
    std::vector<uint64_t> off(NB + 1), km(NB);
    for (size_t gi = 0; gi < grps.size();) {
        const uint32_t p0 = grps[gi].p0, p1 = grps[gi].p1;
        const uint64_t gs = grps[gi].gs;
        uint64_t gN = 0;
        for (uint32_t p = p0; p < p1; p++) gN += np[p];
        uint64_t est = std::min<uint64_t>(gN / std::max<uint32_t>(cmin, 1),
                                          (uint64_t)((double)gN * kept_ratio * 1.25) + 65536);
        if (out_est_override) est = out_est_override - 1;
        const uint64_t out_need = out_used + std::min<uint64_t>(est, out_budget) + 1024;
        if (stream_out && out_need > ctx->out_cap) CK(cudaStreamSynchronize(ctx->cs));  // copies read the old buffer
        RET(ensure_out(ctx, out_need, out_used));
        CK(ctx->bk_entries.ensure(gs * sizeof(BEntry)));
        CK(cudaMemsetAsync(ctx->bk_skms.p, 0, NB * 4, ctx->s));
        CK(cudaMemsetAsync(ctx->bk_kmers.p, 0, NB * 8, ctx->s));
        std::vector<const uint8_t *> cb(nst);
        std::vector<const uint64_t *> ci(nst);
        std::vector<const uint32_t *> ck(nst);
        if (spilled) {
            const int sl = (int)(gi & 1);
            if (staged_g[sl] != (long)gi) RET(stage(gi));
            if (gi + 1 < grps.size() && staged_g[(gi + 1) & 1] != (long)(gi + 1)) RET(stage(gi + 1));
            CK(cudaStreamWaitEvent(ctx->s, staged[sl], 0));
            cb = cbs[sl];
            ci = cis[sl];
            ck = cks[sl];
        } else {  // device chunks: their own pointers, no copies
            uint64_t unused = 0;
            for (size_t j = 0; j < nst; j++)
                RET(chunk_range(ctx, ctx->store[j], p0, p1, ctx->bk_arena, &unused, &cb[j], &ci[j], &ck[j]));
        }
        CK(cudaEventRecord(ctx->e2, ctx->s));
        // the split of every chunk's part of the group, one launch per pass
        std::vector<BSChunk> bsc;
        uint32_t ncta = 0;
        for (size_t j = 0; j < ctx->store.size(); j++) {
            StoreChunk *c = ctx->store[j];
            const uint64_t i0 = c->skm_off[p0], i1 = c->skm_off[p1];
            if (i1 == i0) continue;
            bsc.push_back({ci[j], ck[j], cb[j], i0, i1, c->d_skm_off.as<unsigned long long>(),
                           c->d_byte_off.as<unsigned long long>(), ncta});
            ncta += (uint32_t)((i1 - i0 + BS_PER_CTA - 1) / BS_PER_CTA);
        }
        if (!bsc.empty()) {
            CK(ctx->h_desc.ensure(bsc.size() * sizeof(BSChunk)));
            CK(ctx->bk_desc.ensure(bsc.size() * sizeof(BSChunk)));
            std::memcpy(ctx->h_desc.p, bsc.data(), bsc.size() * sizeof(BSChunk));
            CK(cudaMemcpyAsync(ctx->bk_desc.p, ctx->h_desc.p, bsc.size() * sizeof(BSChunk), cudaMemcpyHostToDevice,
                               ctx->s));
        }
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 1) {
                RET(scan_u32(ctx, ctx->bk_skms.as<uint32_t>(), NB, ctx->bk_off.as<uint64_t>(),
                             ctx->bk_off.as<unsigned long long>() + NB));
                CK(cudaMemcpyAsync(ctx->bk_cur.p, ctx->bk_off.p, NB * 8, cudaMemcpyDeviceToDevice, ctx->s));
            }
            if (!ncta) continue;
            BSplitParams sp;
            sp.chunks = ctx->bk_desc.as<BSChunk>();
            sp.nchunks = (uint32_t)bsc.size();
            sp.P = P;
            sp.part_slog = ctx->bk_part.as<uint32_t>();
            sp.part_bbase = ctx->bk_part.as<uint32_t>() + P;
            sp.bucket_skms = ctx->bk_skms.as<uint32_t>();
            sp.bucket_kmers = ctx->bk_kmers.as<unsigned long long>();
            sp.bucket_cursor = ctx->bk_cur.as<unsigned long long>();
            sp.entries = ctx->bk_entries.as<BEntry>();
            sp.pass = pass;
            KScope ks(ctx, GKC_K_BUCKET_SPLIT, pass ? 28.0 * gs : 12.0 * gs);
            bucket_split_kernel<<<ncta, BS_THREADS, BS_SMEM, ctx->s>>>(sp);
            LAUNCHED();
        }
        CK(cudaMemsetAsync(ctx->bk_failed.p, 0, 4, ctx->s));
        BCountParams bp;
        bp.entries = ctx->bk_entries.as<BEntry>();
        bp.bucket_off = ctx->bk_off.as<uint64_t>();
        bp.bucket_kmers = ctx->bk_kmers.as<unsigned long long>();
        bp.heavy_kmers = BC_HEAVY_KMERS;
        bp.b0 = (uint32_t)bbase(p0);
        bp.ids = nullptr;
        bp.k = ctx->opt.k;
        bp.cmin = cmin;
        bp.cmax = cmax;
        bp.out_k = ctx->out_k.as<uint64_t>();
        bp.out_c = ctx->out_c.as<uint32_t>();
        bp.out_cursor = sc;
        bp.out_cap = ctx->out_cap;
        bp.distinct = sc + 1;
        bp.failed = ctx->bk_failed.as<uint32_t>();
        bp.err = reinterpret_cast<uint32_t *>(sc + 2);
        if (!ctx->opt.hash_l2_only) {
            uint64_t gbytes = 0;
            for (uint32_t p = p0; p < p1; p++) gbytes += nbp[p];
            const uint32_t nbg = (uint32_t)(bbase(p1) - bbase(p0));
            const uint32_t grid =
                std::max<uint32_t>(1, std::min<uint32_t>(nbg, (uint32_t)(ctx->sms * std::max(bc_per_sm, 1))));
            CK(cudaMemsetAsync(ctx->bk_next.p, 0, 4, ctx->s));
            KScope ks(ctx, GKC_K_HASH_INSERT, (double)gbytes + 16.0 * gs);
            bucket_count_persistent_kernel<BC_TS><<<grid, BC_THREADS, BC_TS * 14, ctx->s>>>(bp, nbg,
                                                                                           ctx->bk_next.as<uint32_t>());
            LAUNCHED();
        }
        CK(cudaEventRecord(ctx->e3, ctx->s));
        // one host round trip: the failed sub-buckets, the sub-bucket offsets and
        // k-mer counts the record path needs for them (this group's range of
        // sub-buckets only), and the output cursor (pinned buffers: pageable
        // copies stage through the driver and stall with the host's load;
        // every wait is a chance to catch such a stall)
        const uint64_t gb0 = bbase(p0), gb1 = bbase(p1);
        CK(ctx->h_ids.ensure((NB + 1) * 4));
        CK(ctx->h_off.ensure((NB + 1) * 8));
        CK(ctx->h_km.ensure(NB * 8));
        CK(ctx->h_cur.ensure(32));
        CK(cudaMemcpyAsync(ctx->h_ids.p, ctx->bk_failed.p, (gb1 - gb0 + 1) * 4, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaMemcpyAsync(ctx->h_off.as<uint64_t>() + gb0, ctx->bk_off.as<uint64_t>() + gb0, (gb1 - gb0 + 1) * 8,
                           cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaMemcpyAsync(ctx->h_km.as<uint64_t>() + gb0, ctx->bk_kmers.as<uint64_t>() + gb0, (gb1 - gb0) * 8,
                           cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaMemcpyAsync(ctx->h_cur.p, sc, 24, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        const uint32_t nfail = std::min<uint32_t>(ctx->h_ids.as<uint32_t>()[0], (uint32_t)(gb1 - gb0));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->e2, ctx->e3));
        acc_ms += ms;
        groups++;
        std::vector<uint32_t> ids;
        if (nfail || ctx->opt.hash_l2_only) {  // this group's sub-bucket offsets: off[gb0 .. gb1]
            std::copy(ctx->h_off.as<uint64_t>() + gb0, ctx->h_off.as<uint64_t>() + gb1 + 1, off.begin() + gb0);
            if (nfail) ids.assign(ctx->h_ids.as<uint32_t>() + 1, ctx->h_ids.as<uint32_t>() + 1 + nfail);
        }
        if (ctx->opt.hash_l2_only)  // every non-empty sub-bucket (one per partition)
            for (uint64_t b = bbase(p0); b < bbase(p1); b++)
                if (off[b + 1] > off[b]) ids.push_back(b);
        if (!ids.empty() && !ctx->opt.hash_l2_only) {
            // Second pass: a sub-bucket that outgrew the 8192-slot table (not a
            // heavy one) is counted again with 16384 slots; only heavy
            // sub-buckets and those that overflow again take the record path,
            // whose records cost several times the decode.  (A first pass of
            // 6144 slots at three CTAs per SM inserted 14% faster, but sent so
            // many more sub-buckets of high-error reads to the later passes
            // that mixed long reads lost 25%.)
            std::vector<uint32_t> heavy, over;
            for (uint32_t b : ids) (ctx->h_km.as<uint64_t>()[b] > BC_HEAVY_KMERS ? heavy : over).push_back(b);
            if (!over.empty()) {
                const uint32_t no = (uint32_t)over.size();
                CK(ctx->h_ids2.ensure((no + 1) * 4ull));
                CK(ctx->bk_ids2.ensure(no * 4ull));
                CK(ctx->bk_failed2.ensure((no + 1) * 4ull));
                std::memcpy(ctx->h_ids2.p, over.data(), no * 4ull);
                CK(cudaMemcpyAsync(ctx->bk_ids2.p, ctx->h_ids2.p, no * 4ull, cudaMemcpyHostToDevice, ctx->s));
                CK(cudaMemsetAsync(ctx->bk_failed2.p, 0, 4, ctx->s));
                CK(cudaFuncSetAttribute(bucket_count_kernel<BC_TS2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        BC_TS2 * 12));
                bp.ids = ctx->bk_ids2.as<uint32_t>();
                bp.failed = ctx->bk_failed2.as<uint32_t>();
                bp.out_cap = ctx->out_cap;
                {
                    uint64_t ob = 0;
                    for (uint32_t b : over) ob += 16 * (off[b + 1] - off[b]);
                    KScope ks(ctx, GKC_K_HASH_RECORDS, (double)ob);
                    bucket_count_kernel<BC_TS2><<<no, BC_THREADS, BC_TS2 * 12, ctx->s>>>(bp);
                    LAUNCHED();
                }
                CK(cudaMemcpyAsync(ctx->h_ids2.p, ctx->bk_failed2.p, (no + 1) * 4ull, cudaMemcpyDeviceToHost, ctx->s));
                CK(cudaStreamSynchronize(ctx->s));
                const uint32_t nf2 = std::min<uint32_t>(ctx->h_ids2.as<uint32_t>()[0], no);
                ctx->times[8] += (double)(no - nf2);
                over.assign(ctx->h_ids2.as<uint32_t>() + 1, ctx->h_ids2.as<uint32_t>() + 1 + nf2);
            }
            heavy.insert(heavy.end(), over.begin(), over.end());
            ids.swap(heavy);
        }
        if (!ids.empty()) {
            if (ctx->opt.hash_l2_only) {
                RET(count_buckets_l2(ctx, ids, off, cmin, cmax));
            } else {
                ctx->fallback_buckets += ids.size();
                ctx->times[5] += (double)ids.size();
                std::copy(ctx->h_km.as<uint64_t>() + gb0, ctx->h_km.as<uint64_t>() + gb1, km.begin() + gb0);
                RET(count_buckets_records(ctx, ids, off, km, cmin, cmax));
            }
        }
        // entries written so far: the next group's capacity starts there (read
        // again only if the record path or the L2 table wrote more)
        unsigned long long hg[3];
        if (ids.empty()) {
            std::memcpy(hg, ctx->h_cur.p, 24);
        } else {
            CK(cudaMemcpyAsync(ctx->h_cur.p, sc, 24, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            std::memcpy(hg, ctx->h_cur.p, 24);
        }
        if ((uint32_t)hg[2] & ERR_OUTPUT_FULL) {  // count the group again with room for all of it
            if (++redo > 2) return ctx->fail(GKC_EINTERNAL, "output capacity exceeded");
            const uint64_t need = hg[0];
            if (stream_out) CK(cudaStreamSynchronize(ctx->cs));
            RET(ensure_out(ctx, need + need / 16 + 1024, out_used));
            hg[0] = out_used;
            hg[1] = distinct_used;
            hg[2] &= ~(unsigned long long)ERR_OUTPUT_FULL;
            CK(cudaMemcpyAsync(sc, hg, 24, cudaMemcpyHostToDevice, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            continue;
        }
        if (gN) kept_ratio = std::min(1.0 / std::max<uint32_t>(cmin, 1), (double)(hg[0] - out_used) / (double)gN + 1e-3);
        // the group's output is complete (the stream was synchronised above):
        // copy it out on the copy stream while the next group counts
        if (stream_out && ctx->streamed == out_used && hg[0] <= ctx->stream_cap && hg[0] > out_used) {
            const uint64_t a = out_used, n = hg[0] - out_used;
            CK(cudaMemcpyAsync(ctx->stream_k + a, ctx->out_k.as<uint64_t>() + a, n * 8, cudaMemcpyDeviceToHost,
                               ctx->cs));
            CK(cudaMemcpyAsync(ctx->stream_c + a, ctx->out_c.as<uint32_t>() + a, n * 4, cudaMemcpyDeviceToHost,
                               ctx->cs));
            ctx->streamed = hg[0];
        }
        out_used = hg[0];
        distinct_used = hg[1];
        redo = 0;
        if (spilled) {  // the arena is free once this group's work (waited for above) is done
            const int sl = (int)(gi & 1);
            float sms = 0;
            if (cudaEventElapsedTime(&sms, st0[sl], staged[sl]) == cudaSuccess) stage_ms += sms;
            CK(cudaEventRecord(freed[sl], ctx->s));
        }
        gi++;
    }
    CK(cudaMemcpyAsync(ctx->h_scal.p, sc, 24, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    auto *hs = ctx->h_scal.as<unsigned long long>();
    if ((uint32_t)hs[2] & ERR_OUTPUT_FULL) return ctx->fail(GKC_EINTERNAL, "output capacity exceeded");
    ctx->n_out = hs[0];
    ctx->n_distinct += hs[1];
    ctx->times[3] = acc_ms;
    ctx->times[6] = stage_ms;
    ctx->times[7] = (double)groups;
    if (stream_out) CK(cudaStreamSynchronize(ctx->cs));
    return GKC_OK;
}

// Run-length count + threshold of the sorted keys `src` (n), appending to the
// output; adds the sort's time (events e2..e3, recorded by the caller) to
// *sort_ms.
// RLE + threshold of n sorted keys, appended to the output.  sort_err: the
// radix sort's device error words (onesweep_sort, read here at the first
// synchronisation), or null.
template <class KT>
int reduce_sorted(gkc_ctx *ctx, const KT *src, uint64_t n, uint32_t cmin, uint32_t cmax, float *sort_ms,
                  const uint32_t *sort_err = nullptr) {
    constexpr double KB = sizeof(KT);
    // ---- RLE ----
    const uint64_t rt = (n + RL_TILE - 1) / RL_TILE;
    CK(ctx->tilecnt.ensure(std::max<uint64_t>(rt, 1) * 4));
    CK(ctx->tileoff.ensure(std::max<uint64_t>(rt, 1) * 8));
    CK(ctx->scal.ensure(64));
    CK(ctx->h_scal.ensure(64));
    auto *sc = ctx->scal.as<unsigned long long>();
    uint64_t d = 0;
    if (rt) {
        {
            KScope ks(ctx, GKC_K_RLE, KB * n);
            rle_count_kernel<KT><<<(unsigned)rt, RL_THREADS, 0, ctx->s>>>(src, n, ctx->tilecnt.as<uint32_t>());
            LAUNCHED();
        }
        RET(scan_u32(ctx, ctx->tilecnt.as<uint32_t>(), rt, ctx->tileoff.as<uint64_t>(), sc));
        CK(cudaMemcpyAsync(ctx->h_scal.p, sc, 8, cudaMemcpyDeviceToHost, ctx->s));
        if (sort_err) CK(cudaMemcpyAsync(ctx->h_scal.as<uint32_t>() + 8, sort_err, 16, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        if (sort_err) {
            const uint32_t *e = ctx->h_scal.as<uint32_t>() + 8;
            if (e[0] & ERR_LOOKBACK)
                return ctx->fail(GKC_EINTERNAL, "radix sort: a look-back wait ran out (tile %u, %u of its segment, "
                                                "digit slot %u)", e[1], e[3], e[2]);
        }
        d = ctx->h_scal.as<unsigned long long>()[0];
        CK(ctx->heads_pos.ensure(std::max<uint64_t>(d, 1) * 8));
        CK(ctx->heads_key.ensure(std::max<uint64_t>(d, 1) * sizeof(KT)));
        KScope ks(ctx, GKC_K_RLE, KB * n + (8 + KB) * d);
        rle_write_kernel<KT><<<(unsigned)rt, RL_THREADS, 0, ctx->s>>>(src, n, ctx->tileoff.as<uint64_t>(),
                                                                       ctx->heads_pos.as<uint64_t>(),
                                                                       ctx->heads_key.as<KT>());
        LAUNCHED();
    }
    uint64_t kept = 0;
    const uint64_t kt = (d + RL_TILE - 1) / RL_TILE;
    if (kt) {
        CK(ctx->tilecnt.ensure(kt * 4));
        CK(ctx->tileoff.ensure(kt * 8));
        {
            KScope ks(ctx, GKC_K_RLE, 8.0 * d);
            keep_count_kernel<<<(unsigned)kt, RL_THREADS, 0, ctx->s>>>(ctx->heads_pos.as<uint64_t>(), d, n, cmin,
                                                                         cmax, ctx->tilecnt.as<uint32_t>());
            LAUNCHED();
        }
        RET(scan_u32(ctx, ctx->tilecnt.as<uint32_t>(), kt, ctx->tileoff.as<uint64_t>(), sc));
        CK(cudaMemcpyAsync(ctx->h_scal.p, sc, 8, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        kept = ctx->h_scal.as<unsigned long long>()[0];
        RET(ensure_out(ctx, ctx->n_out + kept, ctx->n_out));
        KScope ks(ctx, GKC_K_RLE, (8 + KB) * d + (4 + KB) * kept);
        keep_write_kernel<KT><<<(unsigned)kt, RL_THREADS, 0, ctx->s>>>(
            ctx->heads_pos.as<uint64_t>(), ctx->heads_key.as<KT>(), d, n, cmin, cmax,
            ctx->tileoff.as<uint64_t>(), ctx->out_k.as<KT>() + ctx->n_out, ctx->out_c.as<uint32_t>() + ctx->n_out);
        LAUNCHED();
    }
    float ms = 0;
    CK(cudaEventSynchronize(ctx->e3));
    CK(cudaEventElapsedTime(&ms, ctx->e2, ctx->e3));
    *sort_ms += ms;
    ctx->n_out += kept;
    ctx->n_distinct += d;
    return GKC_OK;
}


// ---------------------------------------------------------------------------
// phase 2, sort counter: the radix sort of count_onesweep.cu over segments
// `segs` of the n keys in keysA (every segment < 2^30 keys).  Digits of at
// most RB bits, spread evenly over nbits; *sorted receives the buffer that
// holds the result (keysA or keysB).  Nothing here waits for the device: the
// look-back error flags (part_err) are read at the reduction's first
// synchronisation (reduce_sorted).
template <int RB, class KT>
int onesweep_sort(gkc_ctx *ctx, const std::vector<uint64_t> &segs, uint64_t n, int nbits, KT **sorted) {
    constexpr double KB = sizeof(KT);
    constexpr uint64_t T = os_tile<KT>();
    constexpr int NB = 1 << RB;
    OsPasses ps{};
    ps.n = (nbits + RB - 1) / RB;
    if (ps.n > OS_MAX_PASSES) return ctx->fail(GKC_EINTERNAL, "too many radix passes");
    for (int p = 0, sh = 0; p < ps.n; p++) {  // widths differ by at most one bit
        ps.width[p] = nbits / ps.n + (p < nbits % ps.n ? 1 : 0);
        ps.shift[p] = sh;
        sh += ps.width[p];
    }
    // segment tables: first key, first tile and first histogram chunk of
    // each segment (a few KB, through a pinned buffer: the previous sort's
    // copy finished at its reduction's synchronisation)
    const uint32_t nseg = (uint32_t)segs.size();
    const size_t tab = (nseg + 1) * (8ull + 4 + 4);
    CK(ctx->h_segs.ensure(tab));
    CK(ctx->os_segs.ensure(tab));
    auto *key0 = ctx->h_segs.as<unsigned long long>();
    auto *tile0 = reinterpret_cast<uint32_t *>(key0 + nseg + 1);
    uint32_t *chunk0 = tile0 + nseg + 1;
    uint64_t ntiles = 0, nchunks = 0, start = 0;
    for (uint32_t i = 0; i <= nseg; i++) {
        key0[i] = start;
        tile0[i] = (uint32_t)ntiles;
        chunk0[i] = (uint32_t)nchunks;
        if (i == nseg) break;
        ntiles += (segs[i] + T - 1) / T;
        nchunks += (segs[i] + OS_HCHUNK - 1) / OS_HCHUNK;
        start += segs[i];
    }
    KT *src = ctx->keysA.as<KT>(), *dst = ctx->keysB.as<KT>();
    *sorted = src;
    if (!ntiles) return GKC_OK;
    if (ntiles > UINT32_MAX || nchunks > INT32_MAX) return ctx->fail(GKC_ELIMIT, "radix sort: too many tiles");
    const uint64_t nhist = segs.size() * (uint64_t)ps.n * NB;
    CK(ctx->os_hist.ensure(nhist * 4));
    CK(ctx->os_status.ensure(ntiles * NB * 4));
    CK(ctx->tiles.ensure(ntiles * sizeof(OsTile)));
    CK(ctx->os_ctr.ensure(64 * 4));
    CK(ctx->part_err.ensure(64));
    CK(cudaMemcpyAsync(ctx->os_segs.p, ctx->h_segs.p, tab, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemsetAsync(ctx->os_hist.p, 0, nhist * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->os_status.p, 0, ntiles * NB * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->os_ctr.p, 0, 64 * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->part_err.p, 0, 16, ctx->s));
    OsSegs sg;
    sg.key0 = ctx->os_segs.as<unsigned long long>();
    sg.tile0 = reinterpret_cast<const uint32_t *>(sg.key0 + nseg + 1);
    sg.chunk0 = sg.tile0 + nseg + 1;
    sg.nseg = nseg;
    const size_t hsm = (size_t)ps.n * NB * 4;
    {
        static bool attr = false;  // per template instance
        if (!attr) {
            CK(cudaFuncSetAttribute(os_hist_kernel<RB, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)((size_t)((8 * sizeof(KT) + RB - 1) / RB) * NB * 4)));
            CK(cudaFuncSetAttribute(os_pass_kernel<RB, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)os_pass_smem<RB, KT>()));
            // all of the unified L1 that may be shared memory: several CTAs per SM
            CK(cudaFuncSetAttribute(os_pass_kernel<RB, KT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
            attr = true;
        }
    }
    {
        KScope ks(ctx, GKC_K_RADIX_HIST, KB * n + 4.0 * nhist);
        os_hist_kernel<RB, KT><<<(unsigned)nchunks, OS_THREADS, hsm, ctx->s>>>(src, sg, ps,
                                                                              ctx->os_hist.as<uint32_t>());
        LAUNCHED();
    }
    {
        KScope ks(ctx, GKC_K_SCAN, 8.0 * nhist + 32.0 * ntiles);
        os_scan_kernel<RB><<<(unsigned)(segs.size() * ps.n), 1024, 0, ctx->s>>>(ctx->os_hist.as<uint32_t>());
        LAUNCHED();
        os_tiles_kernel<(int)T><<<(unsigned)((ntiles + 255) / 256), 256, 0, ctx->s>>>(sg, (uint32_t)ntiles,
                                                                                     ctx->tiles.as<OsTile>());
        LAUNCHED();
    }
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, os_pass_kernel<RB, KT>, OS_THREADS,
                                                     os_pass_smem<RB, KT>()));
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)ctx->sms * std::max(per_sm, 1));
    static const uint32_t flags[3][2] = {{1u << 30, 2u << 30}, {3u << 30, 1u << 30}, {2u << 30, 3u << 30}};
    for (int p = 0; p < ps.n; p++) {
        OsPassParams q;
        q.in = src;
        q.out = dst;
        q.tiles = ctx->tiles.as<OsTile>();
        q.ntiles = (uint32_t)ntiles;
        q.status = ctx->os_status.as<uint32_t>();
        q.gbase = ctx->os_hist.as<uint32_t>();
        q.npass = ps.n;
        q.pass = p;
        q.shift = ps.shift[p];
        q.width = ps.width[p];
        q.agg = flags[p % 3][0];
        q.inc = flags[p % 3][1];
        q.tile_ctr = ctx->os_ctr.as<uint32_t>() + p;
        q.err = ctx->part_err.as<uint32_t>();
        {
            KScope ks(ctx, GKC_K_RADIX_SCATTER, 2 * KB * n + 8.0 * ntiles * NB);
            os_pass_kernel<RB, KT><<<grid, OS_THREADS, os_pass_smem<RB, KT>(), ctx->s>>>(q);
            LAUNCHED();
        }
        std::swap(src, dst);
    }
    *sorted = src;
    return GKC_OK;
}

// ---------------------------------------------------------------------------
// phase 2, sort counter: sorts `n` keys (KT: u64, or u128 for k > 32) already
// in keysA split into segments segs (sizes), then RLE + threshold, appending
// to the output.  Digits of RB bits; segments of 2^30 keys or more take the
// three-kernel sort (a histogram, a scan and a scatter per digit).
template <int RB, class KT>
int sort_and_reduce_rb(gkc_ctx *ctx, const std::vector<uint64_t> &segs, uint64_t n, int nbits, uint32_t cmin,
                       uint32_t cmax, float *sort_ms) {
    constexpr double KB = sizeof(KT);
    const uint64_t seg_max = ctx->opt.sort_seg_max && ctx->opt.sort_seg_max < OS_SEG_MAX ? ctx->opt.sort_seg_max
                                                                                          : OS_SEG_MAX;
    bool small_segs = true;
    for (uint64_t sz : segs) small_segs &= sz <= seg_max;
    if (small_segs) {
        KT *sorted = nullptr;
        CK(cudaEventRecord(ctx->e2, ctx->s));
        const int rc = onesweep_sort<RB, KT>(ctx, segs, n, nbits, &sorted);
        if (rc != GKC_OK) return rc;
        CK(cudaEventRecord(ctx->e3, ctx->s));
        return reduce_sorted<KT>(ctx, sorted, n, cmin, cmax, sort_ms, n ? ctx->part_err.as<uint32_t>() : nullptr);
    }
    constexpr int RB8 = RB > 8 ? 8 : RB;  // the three-kernel sort keeps per-warp u32 counters of 2^RB digits
    // tiles
    std::vector<TileDesc> td;
    uint64_t start = 0, cnt_base = 0;
    for (uint64_t sz : segs) {
        constexpr uint64_t RS_TILE = rs_tile<KT>();
        uint32_t nt = (uint32_t)((sz + RS_TILE - 1) / RS_TILE);
        for (uint32_t t = 0; t < nt; t++) {
            TileDesc d;
            d.start = start + (uint64_t)t * RS_TILE;
            d.cnt_base = cnt_base;
            d.n = (uint32_t)std::min<uint64_t>(RS_TILE, sz - (uint64_t)t * RS_TILE);
            d.t = t;
            d.nt = nt;
            d.pad = 0;
            td.push_back(d);
        }
        start += sz;
        cnt_base += (uint64_t)nt << RB8;
    }
    const uint64_t ntiles = td.size();
    const uint64_t ncounts = cnt_base;
    if (ntiles) {
        CK(ctx->tiles.ensure(ntiles * sizeof(TileDesc)));
        CK(ctx->counts.ensure(ncounts * 4));
        CK(ctx->offsets.ensure(ncounts * 8));
        CK(cudaMemcpyAsync(ctx->tiles.p, td.data(), ntiles * sizeof(TileDesc), cudaMemcpyHostToDevice, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));  // td is host memory about to go out of scope
    }
    KT *src = ctx->keysA.as<KT>(), *dst = ctx->keysB.as<KT>();
    CK(cudaEventRecord(ctx->e2, ctx->s));
    for (int shift = 0; shift < nbits && ntiles; shift += RB8) {
        {
            KScope ks(ctx, GKC_K_RADIX_HIST, KB * n + 4.0 * ncounts);
            radix_hist_kernel<RB8, KT><<<(unsigned)ntiles, RS_THREADS, 0, ctx->s>>>(
                src, ctx->tiles.as<TileDesc>(), shift, ctx->counts.as<uint32_t>());
            LAUNCHED();
        }
        RET(scan_u32(ctx, ctx->counts.as<uint32_t>(), ncounts, ctx->offsets.as<uint64_t>(), nullptr));
        {
            KScope ks(ctx, GKC_K_RADIX_SCATTER, 2 * KB * n + 8.0 * ncounts);
            radix_scatter_kernel<RB8, KT><<<(unsigned)ntiles, RS_THREADS, 0, ctx->s>>>(
                src, dst, ctx->tiles.as<TileDesc>(), shift, ctx->offsets.as<uint64_t>());
            LAUNCHED();
        }
        std::swap(src, dst);
    }
    CK(cudaEventRecord(ctx->e3, ctx->s));
    return reduce_sorted<KT>(ctx, src, n, cmin, cmax, sort_ms);
}

template <class KT = uint64_t>
int sort_and_reduce(gkc_ctx *ctx, const std::vector<uint64_t> &segs, uint64_t n, int nbits, uint32_t cmin,
                    uint32_t cmax, float *sort_ms) {
    switch (ctx->opt.radix_bits) {
        case 4: return sort_and_reduce_rb<4, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 5: return sort_and_reduce_rb<5, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 6: return sort_and_reduce_rb<6, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 7: return sort_and_reduce_rb<7, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 8: return sort_and_reduce_rb<8, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 9: return sort_and_reduce_rb<9, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        case 10: return sort_and_reduce_rb<10, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
        default: return sort_and_reduce_rb<11, KT>(ctx, segs, n, nbits, cmin, cmax, sort_ms);
    }
}

// Sort counter over the store's partitions (all, or those in `want`), in
// groups of partitions whose keys fit the memory budget.  KT = u128 counts
// k-mers of 33 to 64 bases.
template <class KT>
int count_sort(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, const std::vector<char> *want) {
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    std::vector<uint64_t> np(P, 0);
    for (auto *c : ctx->store)
        for (uint32_t p = 0; p < P; p++) np[p] += c->kmers[p];
    uint64_t budget = ctx->opt.group_keys;
    if (!budget) {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        // per key of a group: two key buffers, the look-back statuses, and at
        // worst (every key distinct) a run head and an output entry each
        budget = std::max<uint64_t>(1ull << 20, (uint64_t)(fr * 0.8) / (4 * sizeof(KT) + 16));
    }
    CK(ctx->segoff.ensure(P * 8));
    CK(ctx->segcur.ensure(P * 8));
    float sort_ms = 0;
    uint32_t p0 = 0;
    while (p0 < P) {
        if (want && !(*want)[p0]) {
            p0++;
            continue;
        }
        uint32_t p1 = p0;
        uint64_t n = 0;
        while (p1 < P && (!want || (*want)[p1]) && (p1 == p0 || n + np[p1] <= budget)) n += np[p1++];
        std::vector<uint64_t> segoff(P, 0), segs;
        uint64_t o = 0;
        for (uint32_t p = p0; p < p1; p++) { segoff[p] = o; o += np[p]; segs.push_back(np[p]); }
        if (n) {
            CK(ctx->keysA.ensure(n * sizeof(KT)));
            CK(ctx->keysB.ensure(n * sizeof(KT)));
            CK(cudaMemcpyAsync(ctx->segoff.p, segoff.data(), P * 8, cudaMemcpyHostToDevice, ctx->s));
            CK(cudaMemsetAsync(ctx->segcur.p, 0, P * 8, ctx->s));
            for (auto *c : ctx->store) {
                uint64_t i0 = c->skm_off[p0], i1 = c->skm_off[p1];
                if (i1 == i0) continue;
                const uint8_t *bytes = c->bytes;
                const uint64_t *idx = c->idx;
                if (c->on_host) {  // stage the group's part of a spilled chunk
                    uint64_t b0 = c->byte_off[p0], b1 = c->byte_off[p1];
                    CK(cudaStreamSynchronize(ctx->s));
                    CK(ctx->stage_bytes.ensure(b1 - b0 + 32));
                    CK(ctx->stage_idx.ensure((i1 - i0) * 8 + 8));
                    CK(ctx->stage_keys.ensure((i1 - i0) * 4 + 4));
                    RET(stage_spilled(ctx, c, p0, p1, ctx->stage_bytes.as<uint8_t>(), ctx->stage_idx.as<uint64_t>(),
                                      ctx->stage_keys.as<uint32_t>(), ctx->s));
                    // kernel indexes bytes by partition offsets: rebase the pointers
                    bytes = ctx->stage_bytes.as<uint8_t>() - b0;
                    idx = ctx->stage_idx.as<uint64_t>() - i0;
                }
                SExtractParams x;
                x.bytes = bytes;
                x.idx = idx;
                x.n_skm = i1;
                x.part_skm_off = c->d_skm_off.as<unsigned long long>();
                x.part_byte_off = c->d_byte_off.as<unsigned long long>();
                x.P = P;
                x.k = ctx->opt.k;
                x.canonical = 1;
                x.keys = ctx->keysA.p;
                x.seg_off = ctx->segoff.as<unsigned long long>();
                x.seg_cursor = ctx->segcur.as<unsigned long long>();
                x.i_begin = i0;
                uint32_t g = (uint32_t)std::min<uint64_t>((i1 - i0 + SX_THREADS - 1) / SX_THREADS, (uint64_t)ctx->sms * 8);
                uint64_t kx = 0;
                for (uint32_t p = p0; p < p1; p++) kx += c->kmers[p];
                KScope ks(ctx, GKC_K_SORT_EXTRACT,
                          (double)(c->byte_off[p1] - c->byte_off[p0]) + 8.0 * (i1 - i0) + (double)sizeof(KT) * kx);
                sort_extract_kernel<KT><<<g, SX_THREADS, 0, ctx->s>>>(x);
                LAUNCHED();
            }
            RET(sort_and_reduce<KT>(ctx, segs, n, 2 * ctx->opt.k, cmin, cmax, &sort_ms));
        }
        p0 = p1;
    }
    ctx->times[3] = sort_ms;
    return GKC_OK;
}

// Hash counter for k of 33 to 64 (u128 keys, count_wide.cu) over the
// partitions `want` (null: all) of a device-resident store, in groups of
// partitions whose sub-bucket entries fit a fifth of free memory.  Per group:
// the split (count_bucket.cu, key-independent), a 4096-slot count per
// sub-bucket of about 4k instances, a second pass with 8192 slots over the
// sub-buckets that overflowed, and the radix sort for the rest (heavy
// sub-buckets and those that overflowed twice), whose k-mer instances are
// extracted into the key buffer.  A spilled store is counted by the sort
// counter.
int count_hash_wide(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, const std::vector<char> *want) {
    for (auto *c : ctx->store)
        if (c->on_host) return count_sort<u128>(ctx, cmin, cmax, want);
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    const int k = ctx->opt.k;
    std::vector<uint64_t> np(P, 0), nsp(P, 0);
    for (auto *c : ctx->store)
        for (uint32_t p = 0; p < P; p++) {
            np[p] += c->kmers[p];
            nsp[p] += c->skm_off[p + 1] - c->skm_off[p];
        }
    // sub-buckets of about 4k instances (2k to 4k): the table holds 4096 keys
    constexpr uint64_t SUB_BUCKET_KMERS_WIDE = 4096;
    constexpr uint64_t HEAVY_WIDE = 32768;  // larger sub-buckets go to the radix sort at once
    constexpr int TS1 = 4096, TS2 = 8192;
    // pieces of a failed sub-bucket: each sized for WIDE_PIECE_KEYS distinct
    // keys at 0.3 distinct per instance, at most WIDE_MAX_PIECES of them and
    // WIDE_PIECE_WORK instances decoded over all of them (each piece decodes
    // the whole sub-bucket); beyond that, and for sub-buckets of more than
    // WIDE_SPLIT_MAX instances, the radix sort
    constexpr uint64_t WIDE_PIECE_KEYS = 6144, WIDE_MAX_PIECES = 64, WIDE_PIECE_WORK = 1ull << 22,
                       WIDE_SPLIT_MAX = 1ull << 20;
    constexpr uint64_t WIDE_EXTRACT_KMERS = 1ull << 16;  // instances per extraction work item
    std::vector<uint32_t> slog(2 * P);
    uint64_t NB = 0;
    for (uint32_t p = 0; p < P; p++) {
        uint32_t sl = 0;
        while (sl < (uint32_t)BS_LOG_LIMIT && np[p] > (SUB_BUCKET_KMERS_WIDE << sl)) sl++;
        slog[p] = sl;
        slog[P + p] = (uint32_t)NB;
        NB += 1ull << sl;
    }
    auto bbase = [&](uint32_t p) -> uint64_t { return p < P ? slog[P + p] : NB; };
    ctx->times[4] = (double)NB;
    ctx->times[5] = 0;
    ctx->times[6] = 0;
    ctx->times[8] = 0;
    size_t free0 = 0, tot0 = 0;
    CK(cudaMemGetInfo(&free0, &tot0));
    ctx->free_hint = free0;
    CK(ctx->bk_skms.ensure(NB * 4));
    CK(ctx->bk_kmers.ensure(NB * 8));
    CK(ctx->bk_off.ensure((NB + 1) * 8));
    CK(ctx->bk_cur.ensure(NB * 8));
    CK(ctx->bk_failed.ensure((NB + 1) * 4));
    CK(ctx->bk_part.ensure(2ull * P * 4));
    CK(cudaMemcpyAsync(ctx->bk_part.p, slog.data(), 2ull * P * 4, cudaMemcpyHostToDevice, ctx->s));
    CK(ctx->scal.ensure(64));
    CK(ctx->h_scal.ensure(64));
    CK(ctx->h_ids.ensure((NB + 1) * 4));
    CK(ctx->h_off.ensure((NB + 1) * 8));
    CK(ctx->h_km.ensure(NB * 8));
    auto *sc = ctx->scal.as<unsigned long long>();  // [0] output cursor, [1] distinct, [2] errors
    CK(cudaFuncSetAttribute(bucket_count_wide_kernel<TS1>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS1 * 24));
    CK(cudaFuncSetAttribute(bucket_count_wide_kernel<TS2>, cudaFuncAttributeMaxDynamicSharedMemorySize, TS2 * 24));
    CK(cudaFuncSetAttribute(bucket_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BS_SMEM));
    const uint64_t budget = std::max<uint64_t>(1ull << 26, (uint64_t)(free0 * 0.2));  // entry bytes per group
    uint64_t distinct_dev = 0;
    float acc_ms = 0;
    uint64_t groups = 0;
    for (uint32_t p0 = 0; p0 < P;) {
        if (want && !(*want)[p0]) {
            p0++;
            continue;
        }
        uint32_t p1 = p0;
        uint64_t gs = 0, gN = 0;
        while (p1 < P && (!want || (*want)[p1]) && (p1 == p0 || 16 * (gs + nsp[p1]) <= budget)) {
            gs += nsp[p1];
            gN += np[p1];
            p1++;
        }
        if (!gs) {
            p0 = p1;
            continue;
        }
        groups++;
        const uint64_t out_used = ctx->n_out;
        // room for every k-mer of the group that can pass the threshold
        RET(ensure_out(ctx, out_used + gN / std::max<uint32_t>(cmin, 1) + 1024, out_used));
        for (int attempt = 0;; attempt++) {
            CK(ctx->bk_entries.ensure(gs * sizeof(BEntry)));
            CK(cudaMemsetAsync(ctx->bk_skms.p, 0, NB * 4, ctx->s));
            CK(cudaMemsetAsync(ctx->bk_kmers.p, 0, NB * 8, ctx->s));
            // the device cursor starts at this group's output; the stream is idle here
            // (the previous group ended with a wait), so the pinned words are free
            const unsigned long long start[3] = {out_used, 0, 0};
            std::memcpy(ctx->h_scal.p, start, 24);
            CK(cudaMemcpyAsync(sc, ctx->h_scal.p, 24, cudaMemcpyHostToDevice, ctx->s));
            CK(cudaEventRecord(ctx->e2, ctx->s));
            // the split of every chunk's part of the group (device chunks: their own pointers)
            std::vector<BSChunk> bsc;
            uint32_t ncta = 0;
            for (StoreChunk *c : ctx->store) {
                const uint64_t i0 = c->skm_off[p0], i1 = c->skm_off[p1];
                if (i1 == i0) continue;
                bsc.push_back({c->idx, c->keys, c->bytes, i0, i1, c->d_skm_off.as<unsigned long long>(),
                               c->d_byte_off.as<unsigned long long>(), ncta});
                ncta += (uint32_t)((i1 - i0 + BS_PER_CTA - 1) / BS_PER_CTA);
            }
            CK(ctx->h_desc.ensure(bsc.size() * sizeof(BSChunk)));
            CK(ctx->bk_desc.ensure(bsc.size() * sizeof(BSChunk)));
            std::memcpy(ctx->h_desc.p, bsc.data(), bsc.size() * sizeof(BSChunk));
            CK(cudaMemcpyAsync(ctx->bk_desc.p, ctx->h_desc.p, bsc.size() * sizeof(BSChunk), cudaMemcpyHostToDevice,
                               ctx->s));
            for (int pass = 0; pass < 2; pass++) {
                if (pass == 1) {
                    RET(scan_u32(ctx, ctx->bk_skms.as<uint32_t>(), NB, ctx->bk_off.as<uint64_t>(),
                                 ctx->bk_off.as<unsigned long long>() + NB));
                    CK(cudaMemcpyAsync(ctx->bk_cur.p, ctx->bk_off.p, NB * 8, cudaMemcpyDeviceToDevice, ctx->s));
                }
                BSplitParams sp;
                sp.chunks = ctx->bk_desc.as<BSChunk>();
                sp.nchunks = (uint32_t)bsc.size();
                sp.P = P;
                sp.part_slog = ctx->bk_part.as<uint32_t>();
                sp.part_bbase = ctx->bk_part.as<uint32_t>() + P;
                sp.bucket_skms = ctx->bk_skms.as<uint32_t>();
                sp.bucket_kmers = ctx->bk_kmers.as<unsigned long long>();
                sp.bucket_cursor = ctx->bk_cur.as<unsigned long long>();
                sp.entries = ctx->bk_entries.as<BEntry>();
                sp.pass = pass;
                KScope ks(ctx, GKC_K_BUCKET_SPLIT, pass ? 28.0 * gs : 12.0 * gs);
                bucket_split_kernel<<<ncta, BS_THREADS, BS_SMEM, ctx->s>>>(sp);
                LAUNCHED();
            }
            BCountParams bp;
            bp.entries = ctx->bk_entries.as<BEntry>();
            bp.bucket_off = ctx->bk_off.as<uint64_t>();
            bp.bucket_kmers = ctx->bk_kmers.as<unsigned long long>();
            bp.heavy_kmers = HEAVY_WIDE;
            bp.b0 = (uint32_t)bbase(p0);
            bp.ids = nullptr;
            bp.k = k;
            bp.cmin = cmin;
            bp.cmax = cmax;
            bp.out_k = ctx->out_k.as<uint64_t>();
            bp.out_c = ctx->out_c.as<uint32_t>();
            bp.out_cursor = sc;
            bp.out_cap = ctx->out_cap;
            bp.distinct = sc + 1;
            bp.failed = ctx->bk_failed.as<uint32_t>();
            bp.err = reinterpret_cast<uint32_t *>(sc + 2);
            CK(cudaMemsetAsync(ctx->bk_failed.p, 0, 4, ctx->s));
            {
                uint64_t gbytes = 0;
                for (StoreChunk *c : ctx->store) gbytes += c->byte_off[p1] - c->byte_off[p0];
                KScope ks(ctx, GKC_K_HASH_INSERT, (double)gbytes + 16.0 * gs);
                bucket_count_wide_kernel<TS1><<<(unsigned)(bbase(p1) - bbase(p0)), BC_THREADS, TS1 * 24, ctx->s>>>(bp);
                LAUNCHED();
            }
            CK(cudaMemcpyAsync(ctx->h_ids.p, ctx->bk_failed.p, (NB + 1) * 4, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaMemcpyAsync(ctx->h_off.p, ctx->bk_off.p, (NB + 1) * 8, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaMemcpyAsync(ctx->h_km.p, ctx->bk_kmers.p, NB * 8, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            const uint32_t nfail = std::min<uint32_t>(ctx->h_ids.as<uint32_t>()[0], (uint32_t)NB);
            const uint64_t *hkm = ctx->h_km.as<uint64_t>(), *hoff = ctx->h_off.as<uint64_t>();
            // the failed sub-buckets in pieces by key hash (wide_piece): pb the
            // sub-bucket, pp its (piece, pieces); pieces that stay too large go
            // to the radix sort (sb, sp)
            std::vector<uint32_t> pb, pp, sb, sp;
            for (uint32_t i = 0; i < nfail; i++) {
                const uint32_t b = ctx->h_ids.as<uint32_t>()[1 + i];
                const uint64_t m = hkm[b];
                const uint64_t n0 = std::max<uint64_t>(1, (m * 3 / 10 + WIDE_PIECE_KEYS - 1) / WIDE_PIECE_KEYS);
                const bool split = m <= WIDE_SPLIT_MAX && n0 <= WIDE_MAX_PIECES && n0 * m <= WIDE_PIECE_WORK;
                for (uint32_t r = 0; r < (split ? n0 : 1u); r++) {
                    (split ? pb : sb).push_back(b);
                    (split ? pp : sp).push_back(r);
                    (split ? pp : sp).push_back(split ? (uint32_t)n0 : 1u);
                }
            }
            auto put_pieces = [&](const std::vector<uint32_t> &ib, const std::vector<uint32_t> &ip) -> int {
                const size_t np = ib.size();
                CK(ctx->h_ids2.ensure(np * 12 + 8 * (np + 1)));
                CK(ctx->bk_ids2.ensure(np * 4));
                CK(ctx->bk_piece.ensure(np * 8));
                std::memcpy(ctx->h_ids2.p, ib.data(), np * 4);
                std::memcpy(ctx->h_ids2.as<uint8_t>() + np * 4, ip.data(), np * 8);
                CK(cudaMemcpyAsync(ctx->bk_ids2.p, ctx->h_ids2.p, np * 4, cudaMemcpyHostToDevice, ctx->s));
                CK(cudaMemcpyAsync(ctx->bk_piece.p, ctx->h_ids2.as<uint8_t>() + np * 4, np * 8, cudaMemcpyHostToDevice,
                                   ctx->s));
                return GKC_OK;
            };
            // second pass, level by level: 8192 slots, one CTA per SM; a piece
            // that overflows splits in two at the next level
            while (!pb.empty()) {
                const uint32_t np = (uint32_t)pb.size();
                RET(put_pieces(pb, pp));
                CK(ctx->bk_failed2.ensure((np + 1) * 4ull));
                CK(cudaMemsetAsync(ctx->bk_failed2.p, 0, 4, ctx->s));
                bp.ids = ctx->bk_ids2.as<uint32_t>();
                bp.piece = ctx->bk_piece.as<uint32_t>();
                bp.failed = ctx->bk_failed2.as<uint32_t>();
                bp.heavy_kmers = UINT64_MAX;
                {
                    uint64_t ob = 0;
                    for (uint32_t b : pb) ob += 16 * (hoff[b + 1] - hoff[b]);
                    KScope ks(ctx, GKC_K_HASH_RECORDS, (double)ob);
                    bucket_count_wide_kernel<TS2><<<np, BC_THREADS, TS2 * 24, ctx->s>>>(bp);
                    LAUNCHED();
                }
                uint32_t *hf = reinterpret_cast<uint32_t *>(ctx->h_ids2.as<uint8_t>() + np * 12);
                CK(cudaMemcpyAsync(hf, ctx->bk_failed2.p, (np + 1) * 4ull, cudaMemcpyDeviceToHost, ctx->s));
                CK(cudaStreamSynchronize(ctx->s));
                const uint32_t nf2 = std::min<uint32_t>(hf[0], np);
                ctx->times[8] += (double)(np - nf2);
                std::vector<uint32_t> nb, npp;
                for (uint32_t i = 0; i < nf2; i++) {
                    const uint32_t j = hf[1 + i], b = pb[j], r = pp[2 * j], n = pp[2 * j + 1];
                    if (2ull * n <= WIDE_MAX_PIECES && 2ull * n * hkm[b] <= WIDE_PIECE_WORK) {
                        for (uint32_t h = 0; h < 2; h++) {
                            nb.push_back(b);
                            npp.push_back(2 * r + h);
                            npp.push_back(2 * n);
                        }
                    } else {
                        sb.push_back(b);
                        sp.push_back(r);
                        sp.push_back(n);
                    }
                }
                pb.swap(nb);
                pp.swap(npp);
            }
            bp.piece = nullptr;
            unsigned long long hg[3];
            CK(cudaMemcpyAsync(ctx->h_scal.p, sc, 24, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            std::memcpy(hg, ctx->h_scal.p, 24);
            if ((uint32_t)hg[2] & ERR_OUTPUT_FULL) {  // count the group again with room for all of it
                if (attempt >= 2) return ctx->fail(GKC_EINTERNAL, "output capacity exceeded");
                RET(ensure_out(ctx, hg[0] + hg[0] / 16 + 1024, out_used));
                continue;
            }
            ctx->n_out = hg[0];
            distinct_dev += hg[1];
            float ms = 0;
            CK(cudaEventRecord(ctx->e3, ctx->s));
            CK(cudaEventSynchronize(ctx->e3));
            CK(cudaEventElapsedTime(&ms, ctx->e2, ctx->e3));
            acc_ms += ms;
            // the rest by the radix sort: the k-mer instances of those pieces
            // counted, extracted, sorted, run-length reduced and thresholded
            // after this group's output
            if (!sb.empty()) {
                ctx->times[5] += (double)sb.size();
                // work items of about WIDE_EXTRACT_KMERS instances: entry ranges of one piece
                std::vector<unsigned long long> wr;
                std::vector<uint32_t> wp;
                uint64_t ib = 0;
                for (size_t j = 0; j < sb.size(); j++) {
                    const uint32_t b = sb[j];
                    const uint64_t ne = hoff[b + 1] - hoff[b];
                    const uint64_t per = std::max<uint64_t>(1, hkm[b] / std::max<uint64_t>(ne, 1));
                    const uint64_t w = std::max<uint64_t>(32, WIDE_EXTRACT_KMERS / per);
                    ib += 16 * ne;
                    for (uint64_t c = hoff[b]; c < hoff[b + 1]; c += w) {
                        wr.push_back(c);
                        wr.push_back(std::min<uint64_t>(c + w, hoff[b + 1]));
                        wp.push_back(sp[2 * j]);
                        wp.push_back(sp[2 * j + 1]);
                    }
                }
                const uint32_t nw = (uint32_t)(wr.size() / 2);
                // pinned: [ranges 16 B][pieces 8 B][counts, then offsets 8 B] per item
                CK(ctx->h_ids2.ensure(nw * 32ull));
                CK(ctx->bk_piece.ensure(nw * 8ull));
                CK(ctx->r_work.ensure(nw * 16ull));
                CK(ctx->r_off.ensure(nw * 8ull));
                uint8_t *hb = ctx->h_ids2.as<uint8_t>();
                std::memcpy(hb, wr.data(), nw * 16ull);
                std::memcpy(hb + nw * 16ull, wp.data(), nw * 8ull);
                CK(cudaMemcpyAsync(ctx->r_work.p, hb, nw * 16ull, cudaMemcpyHostToDevice, ctx->s));
                CK(cudaMemcpyAsync(ctx->bk_piece.p, hb + nw * 16ull, nw * 8ull, cudaMemcpyHostToDevice, ctx->s));
                BExtractParams xp;
                xp.entries = ctx->bk_entries.as<BEntry>();
                xp.range = ctx->r_work.as<unsigned long long>();
                xp.piece = ctx->bk_piece.as<uint32_t>();
                xp.key_off = nullptr;
                xp.k = k;
                xp.keys = nullptr;
                xp.counts = ctx->r_off.as<unsigned long long>();
                {
                    KScope ks(ctx, GKC_K_SORT_EXTRACT, (double)ib);
                    bucket_extract_wide_kernel<<<nw, BC_THREADS, 0, ctx->s>>>(xp);  // instances per item
                    LAUNCHED();
                }
                unsigned long long *hc = reinterpret_cast<unsigned long long *>(hb + nw * 24ull);
                CK(cudaMemcpyAsync(hc, ctx->r_off.p, nw * 8ull, cudaMemcpyDeviceToHost, ctx->s));
                CK(cudaStreamSynchronize(ctx->s));
                uint64_t n = 0;
                for (uint32_t i = 0; i < nw; i++) {
                    const unsigned long long c = hc[i];
                    hc[i] = n;
                    n += c;
                }
                CK(cudaMemcpyAsync(ctx->r_off.p, hc, nw * 8ull, cudaMemcpyHostToDevice, ctx->s));
                CK(ctx->keysA.ensure(n * sizeof(u128)));
                CK(ctx->keysB.ensure(n * sizeof(u128)));
                xp.key_off = ctx->r_off.as<unsigned long long>();
                xp.keys = ctx->keysA.as<u128>();
                {
                    KScope ks(ctx, GKC_K_SORT_EXTRACT, (double)ib + 16.0 * n);
                    bucket_extract_wide_kernel<<<nw, BC_THREADS, 0, ctx->s>>>(xp);
                    LAUNCHED();
                }
                float sort_ms = 0;  // appends at ctx->n_out, adds its distinct k-mers to ctx->n_distinct
                RET(sort_and_reduce<u128>(ctx, std::vector<uint64_t>{n}, n, 2 * k, cmin, cmax, &sort_ms));
                acc_ms += sort_ms;
            }
            break;
        }
        p0 = p1;
    }
    ctx->n_distinct += distinct_dev;
    ctx->times[3] = acc_ms;
    ctx->times[7] = (double)groups;
    return GKC_OK;
}


// Makes the rank table `ranks` (device, 4^p) the context's order: phase 1
// reads its canonical form.
int install_order(gkc_ctx *ctx, const uint32_t *ranks) {
    const int p = ctx->opt.p;
    const uint32_t n = 1u << (2 * p);
    CK(ctx->lut.ensure(n * 4ull));
    const uint32_t g = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sms * 8);
    canonical_table_kernel<<<g, 256, 0, ctx->s>>>(ranks, n, p, ctx->lut.as<uint32_t>());
    LAUNCHED();
    CK(cudaStreamSynchronize(ctx->s));
    ctx->has_lut = true;
    return GKC_OK;
}

int upload(gkc_ctx *ctx, DevBuf &buf, const void *src, uint64_t bytes, int mem, const void **dptr) {
    if (mem == GKC_MEM_DEVICE) {
        *dptr = src;
        return GKC_OK;
    }
    CK(buf.ensure(bytes + 16));
    CK(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, ctx->s));
    *dptr = buf.p;
    return GKC_OK;
}

}  // namespace

// ===========================================================================
// C ABI
extern "C" {

void gkc_default_options(gkc_options *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->k = 31;
    o->p = 11;
    o->partitions = 512;
    o->counter = GKC_COUNTER_HASH;
    o->radix_bits = 8;
    o->table_slots = 0.35;
    o->batch_bases = 1ull << 30;
    o->spill_host = 0;
    o->group_keys = 0;
    o->hash_l2_only = 0;
    o->hpc = 0;
    o->sort_seg_max = 0;
}

const char *gkc_strerror(int code) {
    switch (code) {
        case GKC_OK: return "ok";
        case GKC_EINVAL: return "invalid argument";
        case GKC_ECUDA: return "CUDA error";
        case GKC_ENOMEM: return "out of memory";
        case GKC_ESTATE: return "invalid call order";
        case GKC_EINTERNAL: return "internal error";
        case GKC_ELIMIT: return "larger than a fixed-size limit";
        default: return "unknown error";
    }
}

const char *gkc_last_error(const gkc_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

uint64_t gkc_kernel_launches(const gkc_ctx *ctx) { return ctx ? ctx->launches : 0; }

int gkc_create(int device, const gkc_options *opt, gkc_ctx **out) {
    if (!out) return GKC_EINVAL;
    *out = nullptr;
    gkc_options o;
    gkc_default_options(&o);
    if (opt) o = *opt;
    if (o.p < 3 || o.p > 16 || o.k < o.p || o.k > 64 || o.partitions < 1 || o.partitions > 4096 ||
        (o.counter != GKC_COUNTER_SORT && o.counter != GKC_COUNTER_HASH) || o.radix_bits < 0 || o.radix_bits > 11 ||
        (o.radix_bits != 0 && o.radix_bits < 4))
        return GKC_EINVAL;
    if (!o.radix_bits) o.radix_bits = 8;
    if (!o.batch_bases) o.batch_bases = 1ull << 30;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return GKC_ECUDA;
    auto *ctx = new gkc_ctx();
    ctx->device = device;
    ctx->opt = o;
    auto cleanup = [&](int code) { delete ctx; return code; };
    if (cudaSetDevice(device) != cudaSuccess) return cleanup(GKC_ECUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return cleanup(GKC_ECUDA);
    ctx->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->own_s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->cs, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->ss, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->rs, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(GKC_ECUDA);
    cudaEvent_t *sevs[] = {&ctx->spill_ready, &ctx->spill_done[0], &ctx->spill_done[1]};
    for (auto *e : sevs)
        if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return cleanup(GKC_ECUDA);
    ctx->s = ctx->own_s;
    cudaEvent_t *evs[] = {&ctx->e0, &ctx->e1, &ctx->e2, &ctx->e3};
    for (auto *e : evs)
        if (cudaEventCreate(e) != cudaSuccess) return cleanup(GKC_ECUDA);
    for (int i = 0; i < gkc_ctx::NSLOT; i++)
        if (cudaEventCreateWithFlags(&ctx->buf_free[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->buf_ready[i], cudaEventDisableTiming) != cudaSuccess)
            return cleanup(GKC_ECUDA);
    for (int i = 0; i < 2; i++)
        if (cudaEventCreateWithFlags(&ctx->pk_copied[i], cudaEventDisableTiming) != cudaSuccess)
            return cleanup(GKC_ECUDA);
    *out = ctx;
    return GKC_OK;
}

int gkc_destroy(gkc_ctx *ctx) {
    if (!ctx) return GKC_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->s) cudaStreamSynchronize(ctx->s);
    if (ctx->cs) cudaStreamSynchronize(ctx->cs);
    delete ctx;
    return GKC_OK;
}

int gkc_set_order(gkc_ctx *ctx, const uint32_t *lut, uint64_t n, int mem) {
    if (!ctx) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    if (!lut) {
        ctx->has_lut = false;
        return GKC_OK;
    }
    uint64_t need = 1ull << (2 * ctx->opt.p);
    if (n != need) return ctx->fail(GKC_EINVAL, "order table needs 4^p = %llu entries", (unsigned long long)need);
    CK(ctx->ord_stage.ensure(n * 4));
    CK(cudaMemcpyAsync(ctx->ord_stage.p, lut, n * 4,
                       mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->s));
    RET(install_order(ctx, ctx->ord_stage.as<uint32_t>()));
    return GKC_OK;
}

}  // extern "C"

namespace {

struct ReadBatch {
    uint64_t r0, r1;  // reads [r0, r1) of the caller's CSR
};

// Homopolymer compression of a device batch (read r at offs[r] - base) into
// ctx->hpc_reads / hpc_offs (offsets from 0); *kept = the compressed bases.
int hpc_batch(gkc_ctx *ctx, const uint8_t *d_reads, const uint64_t *d_offs, uint64_t n_reads, uint64_t base,
              uint64_t total, uint64_t *kept) {
    const uint64_t ntiles = std::max<uint64_t>((total + gkc::HPC_TILE - 1) / gkc::HPC_TILE, 1);
    CK(ctx->hpc_tiles.ensure(ntiles * 4));
    CK(ctx->hpc_tbase.ensure((ntiles + 1) * 8));
    CK(ctx->hpc_reads.ensure(total + 64));
    CK(ctx->hpc_offs.ensure((n_reads + 1) * 8));
    gkc::HpcParams a;
    a.reads = d_reads;
    a.offs = d_offs;
    a.n_reads = n_reads;
    a.base = base;
    a.n = total;
    a.tile_kept = ctx->hpc_tiles.as<uint32_t>();
    a.tile_base = ctx->hpc_tbase.as<uint64_t>();
    a.out = ctx->hpc_reads.as<uint8_t>();
    a.out_offs = ctx->hpc_offs.as<uint64_t>();
    unsigned long long *dtot = ctx->hpc_tbase.as<unsigned long long>() + ntiles;
    if (total) {
        gkc::hpc_count_kernel<<<(uint32_t)ntiles, gkc::HPC_THREADS, 0, ctx->s>>>(a);
        LAUNCHED();
        RET(scan_u32(ctx, a.tile_kept, ntiles, ctx->hpc_tbase.as<uint64_t>(), dtot));
        gkc::hpc_write_kernel<<<(uint32_t)ntiles, gkc::HPC_THREADS, 0, ctx->s>>>(a);
        LAUNCHED();
    } else {
        CK(cudaMemsetAsync(dtot, 0, 8, ctx->s));
    }
    const uint32_t g = (uint32_t)std::min<uint64_t>((n_reads + 256) / 256, (uint64_t)ctx->sms * 8);
    gkc::hpc_tail_offsets_kernel<<<g, 256, 0, ctx->s>>>(d_offs, n_reads, base, total, dtot, a.out_offs);
    LAUNCHED();
    CK(ctx->h_scal.ensure(64));
    CK(cudaMemcpyAsync(ctx->h_scal.p, dtot, 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    *kept = *ctx->h_scal.as<uint64_t>();
    return GKC_OK;
}

// Phase 1 over host batches: the copy of batch i+1 (copy stream, three device
// slots) overlaps phase 1 of batch i; no batch waits for the host (phase1_async)
// unless the store spills (phase1_exact).
// Host batches.  Every other batch crosses PCIe packed into 2-bit words (a
// quarter of the ASCII bytes; gkc_pack_bases, on the host's threads), the
// others as ASCII: the host's threads pack one batch while the copy engine
// moves the next, so both host-memory readers work at once (packing every
// batch left the copy engine idle and the threads the bound).  Packed
// batches alternate between two pinned buffers, so the host packs the next
// one while the last one's copy is still in flight.  With homopolymer
// compression every batch goes as ASCII (its kernels read it).  Batch i + 1
// is prepared and copied while phase 1 of batch i runs.
int add_host_batches(gkc_ctx *ctx, const char *reads, const uint64_t *offs, const std::vector<ReadBatch> &batches) {
    const bool exact = ctx->opt.spill_host;
    const bool pack = !ctx->opt.hpc;
    const size_t nbat = batches.size();
    uint64_t max_b = 0, max_r = 0;
    for (const auto &b : batches) {
        max_b = std::max<uint64_t>(max_b, offs[b.r1] - offs[b.r0]);
        max_r = std::max<uint64_t>(max_r, b.r1 - b.r0);
    }
    CK(cudaStreamSynchronize(ctx->s));  // the slots may be reallocated below
    // packed words of a batch, and 4 zero words after them (the scatter reads
    // a code window one word past a superkmer's last base)
    const uint64_t max_w = (max_b + 15) / 16 + 4;
    for (int slot = 0; slot < gkc_ctx::NSLOT; slot++) {
        CK(ctx->reads[slot].ensure(std::max<uint64_t>(max_b + 64, pack ? max_w * 4 : 0)));
        CK(ctx->offs[slot].ensure((max_r + 1) * 8));
    }
    if (pack)
        for (int pb = 0; pb < 2; pb++) CK(ctx->pk_host[pb].ensure(max_w * 4));
    while (ctx->batch_ev.size() < 2 * nbat) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        ctx->batch_ev.push_back(ev);
    }
    auto packed = [&](size_t bi) { return pack && (bi & 1); };
    auto stage = [&](size_t bi, cudaStream_t st) -> int {
        const int slot = (int)(bi % gkc_ctx::NSLOT);
        const ReadBatch &b = batches[bi];
        const uint64_t base = offs[b.r0], nb = offs[b.r1] - base, nr = b.r1 - b.r0;
        if (packed(bi)) {
            // pinned buffer pb's words are rewritten once their last copy is done
            const int pb = (int)((bi >> 1) & 1);
            CK(cudaEventSynchronize(ctx->pk_copied[pb]));
            const uint64_t nw = (nb + 15) / 16;
            uint32_t *hw = ctx->pk_host[pb].as<uint32_t>();
            gkc_host::pack_bases(reinterpret_cast<const uint8_t *>(reads) + base, nb, hw, nw);
            std::memset(hw + nw, 0, 16);
            CK(cudaStreamWaitEvent(st, ctx->buf_free[slot], 0));
            CK(cudaEventRecord(ctx->batch_ev[2 * bi], st));  // the batch starts with its copy
            CK(cudaMemcpyAsync(ctx->reads[slot].p, hw, (nw + 4) * 4, cudaMemcpyHostToDevice, st));
            CK(cudaEventRecord(ctx->pk_copied[pb], st));
            ctx->h2d_bytes += (nw + 4) * 4;
        } else {
            CK(cudaStreamWaitEvent(st, ctx->buf_free[slot], 0));
            CK(cudaEventRecord(ctx->batch_ev[2 * bi], st));  // the batch starts with its copy
            CK(cudaMemcpyAsync(ctx->reads[slot].p, reads + base, nb, cudaMemcpyHostToDevice, st));
            ctx->h2d_bytes += nb;
        }
        CK(cudaMemcpyAsync(ctx->offs[slot].p, offs + b.r0, (nr + 1) * 8, cudaMemcpyHostToDevice, st));
        ctx->h2d_bytes += (nr + 1) * 8;
        CK(cudaEventRecord(ctx->buf_ready[slot], st));
        return GKC_OK;
    };
    auto run = [&](size_t bi, bool sync_exact) -> int {
        const int slot = (int)(bi % gkc_ctx::NSLOT);
        const ReadBatch &b = batches[bi];
        const uint64_t base = offs[b.r0], nb = offs[b.r1] - base, nr = b.r1 - b.r0;
        CK(cudaStreamWaitEvent(ctx->s, ctx->buf_ready[slot], 0));
        int rc;
        if (ctx->opt.hpc) {  // phase 1 reads the compressed copy, offsets from 0
            uint64_t kept = 0;
            RET(hpc_batch(ctx, ctx->reads[slot].as<uint8_t>(), ctx->offs[slot].as<uint64_t>(), nr, base, nb, &kept));
            const uint8_t *hr = ctx->hpc_reads.as<uint8_t>();
            uint64_t *ho = ctx->hpc_offs.as<uint64_t>();
            rc = sync_exact ? phase1_exact(ctx, hr, ho, nr, kept) : phase1_async(ctx, hr, ho, nr, kept, 0, bi);
        } else {
            ctx->p1_packed = packed(bi) ? ctx->reads[slot].as<uint32_t>() : nullptr;
            if (sync_exact) {
                const uint32_t g = (uint32_t)std::min<uint64_t>((nr + 256) / 256, (uint64_t)ctx->sms * 8);
                rebase_offsets_kernel<<<g, 256, 0, ctx->s>>>(ctx->offs[slot].as<uint64_t>(), nr + 1, base);
                LAUNCHED();
                rc = phase1_exact(ctx, ctx->reads[slot].as<uint8_t>(), ctx->offs[slot].as<uint64_t>(), nr, nb);
            } else {
                rc = phase1_async(ctx, ctx->reads[slot].as<uint8_t>(), ctx->offs[slot].as<uint64_t>(), nr, nb,
                                  base, bi);
            }
            ctx->p1_packed = nullptr;
        }
        CK(cudaEventRecord(ctx->buf_free[slot], ctx->s));
        CK(cudaEventRecord(ctx->batch_ev[2 * bi + 1], ctx->s));
        return rc;
    };
    for (int slot = 0; slot < gkc_ctx::NSLOT; slot++) CK(cudaEventRecord(ctx->buf_free[slot], ctx->s));
    // batch i's phase 1 is queued before batch i + 1 is staged, so that the
    // device works while the host packs
    int rc = nbat ? stage(0, ctx->cs) : GKC_OK;
    for (size_t bi = 0; rc == GKC_OK && bi < nbat; bi++) {
        rc = run(bi, exact);
        if (rc == GKC_OK && bi + 1 < nbat) rc = stage(bi + 1, ctx->cs);
    }
    CK(cudaStreamSynchronize(ctx->s));
    if (rc != GKC_OK) return rc;
    std::vector<uint64_t> redo;
    RET(phase1_finish(ctx, &redo));
    ctx->batch_ms.assign(nbat, 0.0);
    for (size_t bi = 0; bi < nbat; bi++) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ctx->batch_ev[2 * bi], ctx->batch_ev[2 * bi + 1]) == cudaSuccess)
            ctx->batch_ms[bi] = ms;
    }
    for (uint64_t bi : redo) {  // capacity overflow: the batch again, with exact sizes
        RET(stage(bi, ctx->s));
        RET(run(bi, true));
        CK(cudaStreamSynchronize(ctx->s));
    }
    return GKC_OK;
}

// FASTQ (format 0) or FASTA (1) text -> the CSR in ctx->fx_out / fx_offs.
// state_in: FASTQ line phase at the text's start (0 at a file's start).
int parse_fastx(gkc_ctx *ctx, const char *text, uint64_t n, int mem, int format, int state_in, uint64_t *n_reads,
                uint64_t *n_bases, int *state_out) {
    if ((format != GKC_FASTQ && format != GKC_FASTA) || state_in < 0 || state_in > 3 || (!text && n))
        return ctx->fail(GKC_EINVAL, "fastx: format must be GKC_FASTQ or GKC_FASTA and the state 0..3");
    const bool fasta = format == GKC_FASTA;
    *n_reads = *n_bases = 0;
    *state_out = fasta ? 0 : state_in;
    if (n == 0) return GKC_OK;
    // staged into an aligned buffer: the tile kernels read 16-byte words
    CK(ctx->fx_text.ensure(n + 64));
    CK(cudaMemcpyAsync(ctx->fx_text.p, text, n, mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                                      : cudaMemcpyHostToDevice, ctx->s));
    const uint64_t ntiles = (n + FX_TILE - 1) / FX_TILE;
    CK(ctx->fx_tiles.ensure(ntiles * sizeof(FxT)));
    CK(ctx->fx_state.ensure(ntiles));
    CK(ctx->fx_kept.ensure(ntiles * 8));
    CK(ctx->fx_reads.ensure(ntiles * 8));
    CK(ctx->fx_res.ensure(64));
    CK(ctx->h_scal.ensure(64));
    // a read already open at the text's start: FASTQ phase 1, or FASTA text
    // that starts with sequence lines (a record continued from the text before)
    uint8_t first = 0;
    CK(cudaMemcpyAsync(&first, ctx->fx_text.p, 1, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const int virtual_read = fasta ? (first != '>') : (state_in == 1);
    FxParams a;
    a.text = ctx->fx_text.as<uint8_t>();
    a.n = n;
    a.tiles = ctx->fx_tiles.as<FxT>();
    a.ntiles = ntiles;
    a.tile_state = ctx->fx_state.as<uint8_t>();
    a.tile_kept = ctx->fx_kept.as<uint64_t>();
    a.tile_reads = ctx->fx_reads.as<uint64_t>();
    a.result = ctx->fx_res.as<uint64_t>();
    a.state_in = state_in;
    a.out = nullptr;
    a.offs = nullptr;
    if (fasta) fastx_tile_kernel<true><<<(uint32_t)ntiles, FX_THREADS, 0, ctx->s>>>(a);
    else fastx_tile_kernel<false><<<(uint32_t)ntiles, FX_THREADS, 0, ctx->s>>>(a);
    LAUNCHED();
    fastx_carry_kernel<<<1, FX_CARRY_THREADS, 0, ctx->s>>>(a, virtual_read);
    LAUNCHED();
    uint64_t *hr = ctx->h_scal.as<uint64_t>();
    CK(cudaMemcpyAsync(hr, ctx->fx_res.p, 24, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const uint64_t kept = hr[0], reads = hr[1];
    const int st = (int)hr[2];
    CK(ctx->fx_out.ensure(kept + 64));
    CK(ctx->fx_offs.ensure((reads + 1) * 8));
    a.out = ctx->fx_out.as<uint8_t>();
    a.offs = ctx->fx_offs.as<uint64_t>();
    if (virtual_read) CK(cudaMemsetAsync(a.offs, 0, 8, ctx->s));
    if (fasta) fastx_write_kernel<true><<<(uint32_t)ntiles, FX_THREADS, 0, ctx->s>>>(a);
    else fastx_write_kernel<false><<<(uint32_t)ntiles, FX_THREADS, 0, ctx->s>>>(a);
    LAUNCHED();
    hr[3] = kept;
    CK(cudaMemcpyAsync(a.offs + reads, hr + 3, 8, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    *n_reads = reads;
    *n_bases = kept;
    *state_out = fasta ? 0 : st;
    return GKC_OK;
}

// Device-resident reads in batches of about batch_bases bases: each batch's
// phase 1 reads the caller's bytes in place and a rebased copy of its
// offsets.  Smaller batches keep the scatter's partition slices in L2 (one
// 3 Gbp batch scatters about 40% slower than six 0.5 Gbp ones).
int add_device_batches(gkc_ctx *ctx, const uint8_t *dr, const uint64_t *offs, uint64_t n_reads, uint64_t total) {
    const uint64_t bb = std::max<uint64_t>(ctx->opt.batch_bases, 1);
    const uint32_t ncut = (uint32_t)((total + bb - 1) / bb);
    CK(ctx->tiles.ensure((ncut + 1) * 16ull));
    uint64_t *cut_idx = ctx->tiles.as<uint64_t>(), *cut_off = cut_idx + ncut + 1;
    batch_cuts_kernel<<<(ncut + 256) / 256, 256, 0, ctx->s>>>(offs, n_reads, bb, ncut, cut_idx, cut_off);
    LAUNCHED();
    std::vector<uint64_t> h(2 * (ncut + 1));
    CK(cudaMemcpyAsync(h.data(), cut_idx, h.size() * 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    // batch j ends at cut j + 1; empty ones (a read longer than a batch spans
    // several cuts) are dropped.  base / bend: offsets of the batch's bounds
    std::vector<ReadBatch> batches;
    std::vector<uint64_t> base, bend;
    uint64_t max_r = 0, r0 = 0, b0 = 0;
    for (uint32_t j = 0; j < ncut; j++) {
        const uint64_t r1 = h[j + 1], b1 = h[ncut + 1 + j + 1];
        if (r1 <= r0) continue;
        batches.push_back({r0, r1});
        base.push_back(b0);
        bend.push_back(b1);
        max_r = std::max<uint64_t>(max_r, r1 - r0);
        r0 = r1;
        b0 = b1;
    }
    CK(ctx->offs[0].ensure((max_r + 1) * 8));
    uint64_t *bo = ctx->offs[0].as<uint64_t>();
    while (ctx->batch_ev.size() < 2 * batches.size()) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        ctx->batch_ev.push_back(ev);
    }
    // everything on ctx->s: a batch's offsets copy waits for the batch before
    for (size_t bi = 0; bi < batches.size(); bi++) {
        const uint64_t r0 = batches[bi].r0, nr = batches[bi].r1 - r0, nb = bend[bi] - base[bi];
        CK(cudaEventRecord(ctx->batch_ev[2 * bi], ctx->s));
        CK(cudaMemcpyAsync(bo, offs + r0, (nr + 1) * 8, cudaMemcpyDeviceToDevice, ctx->s));
        RET(phase1_async(ctx, dr + base[bi], bo, nr, nb, base[bi], bi));
        CK(cudaEventRecord(ctx->batch_ev[2 * bi + 1], ctx->s));
    }
    CK(cudaStreamSynchronize(ctx->s));
    std::vector<uint64_t> redo;
    RET(phase1_finish(ctx, &redo));
    ctx->batch_ms.assign(batches.size(), 0.0);
    for (size_t bi = 0; bi < batches.size(); bi++) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ctx->batch_ev[2 * bi], ctx->batch_ev[2 * bi + 1]) == cudaSuccess)
            ctx->batch_ms[bi] = ms;
    }
    for (uint64_t bi : redo) {  // capacity overflow: the batch again, with exact sizes
        const uint64_t r0 = batches[bi].r0, nr = batches[bi].r1 - r0, nb = bend[bi] - base[bi];
        CK(cudaMemcpyAsync(bo, offs + r0, (nr + 1) * 8, cudaMemcpyDeviceToDevice, ctx->s));
        const uint32_t g = (uint32_t)std::min<uint64_t>((nr + 256) / 256, (uint64_t)ctx->sms * 8);
        rebase_offsets_kernel<<<g, 256, 0, ctx->s>>>(bo, nr + 1, base[bi]);
        LAUNCHED();
        RET(phase1_exact(ctx, dr + base[bi], bo, nr, nb));
        CK(cudaStreamSynchronize(ctx->s));
    }
    return GKC_OK;
}

}  // namespace

extern "C" {

int gkc_add_reads(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int mem) {
    if (!ctx || (!reads && n_reads) || !offs) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (char c : ctx->counted)
        if (c) return ctx->fail(GKC_ESTATE, "the store is partly counted; clear it before adding reads");
    ctx->times[0] = ctx->times[1] = 0;
    ctx->h2d_bytes = 0;
    ctx->batch_ms.clear();
    if (n_reads == 0) return GKC_OK;
    if (mem == GKC_MEM_DEVICE) {
        uint64_t first = 0, total = 0;
        CK(cudaMemcpyAsync(&first, offs, 8, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaMemcpyAsync(&total, offs + n_reads, 8, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        if (first != 0) return ctx->fail(GKC_EINVAL, "device input needs offs[0] == 0");
        CK(cudaEventRecord(ctx->e2, ctx->s));
        const uint8_t *dr = reinterpret_cast<const uint8_t *>(reads);
        if (ctx->opt.hpc) {  // phase 1 reads the compressed copy
            RET(hpc_batch(ctx, dr, offs, n_reads, 0, total, &total));
            dr = ctx->hpc_reads.as<uint8_t>();
            offs = ctx->hpc_offs.as<uint64_t>();
        }
        if (ctx->opt.spill_host) {
            RET(phase1_exact(ctx, dr, offs, n_reads, total));
        } else if (total > ctx->opt.batch_bases) {
            RET(add_device_batches(ctx, dr, offs, n_reads, total));
        } else {
            // no rebase: the caller's offsets are only read
            RET(phase1_async(ctx, dr, const_cast<uint64_t *>(offs), n_reads, total, 0, 0));
            CK(cudaStreamSynchronize(ctx->s));
            std::vector<uint64_t> redo;
            RET(phase1_finish(ctx, &redo));
            if (!redo.empty()) RET(phase1_exact(ctx, dr, offs, n_reads, total));
        }
        CK(cudaEventRecord(ctx->e3, ctx->s));
        CK(cudaEventSynchronize(ctx->e3));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->e2, ctx->e3));
        ctx->times[0] = ms;
        if (ctx->batch_ms.empty()) ctx->batch_ms.assign(1, ms);  // one batch
        return GKC_OK;
    }
    if (offs[0] > offs[n_reads]) return ctx->fail(GKC_EINVAL, "offsets are not ascending");
    // batches of whole reads of about batch_bases bases
    std::vector<ReadBatch> batches;
    uint64_t r = 0;
    while (r < n_reads) {
        uint64_t lim = offs[r] + ctx->opt.batch_bases;
        uint64_t lo = r + 1, hi = n_reads;  // the last read end within the budget
        while (lo < hi) {
            uint64_t mid = (lo + hi + 1) >> 1;
            if (offs[mid] <= lim) lo = mid; else hi = mid - 1;
        }
        batches.push_back({r, std::max<uint64_t>(r + 1, lo)});
        r = batches.back().r1;
    }
    CK(cudaEventRecord(ctx->e2, ctx->s));
    const int rc = add_host_batches(ctx, reads, offs, batches);
    CK(cudaEventRecord(ctx->e3, ctx->s));
    CK(cudaEventSynchronize(ctx->e3));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->e2, ctx->e3);
    ctx->times[0] = ms;
    return rc;
}

int gkc_add_reads_batches(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads,
                          const uint64_t *batch_reads, uint64_t n_batches) {
    if (!ctx || (!reads && n_reads) || !offs || (!batch_reads && n_batches)) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (char c : ctx->counted)
        if (c) return ctx->fail(GKC_ESTATE, "the store is partly counted; clear it before adding reads");
    ctx->times[0] = ctx->times[1] = 0;
    ctx->h2d_bytes = 0;
    ctx->batch_ms.clear();
    std::vector<ReadBatch> batches;
    uint64_t r = 0;
    for (uint64_t i = 0; i < n_batches; i++) {
        if (batch_reads[i] == 0) continue;
        batches.push_back({r, r + batch_reads[i]});
        r += batch_reads[i];
    }
    if (r != n_reads) return ctx->fail(GKC_EINVAL, "batch sizes add up to %llu reads, not %llu",
                                       (unsigned long long)r, (unsigned long long)n_reads);
    if (n_reads && offs[0] > offs[n_reads]) return ctx->fail(GKC_EINVAL, "offsets are not ascending");
    CK(cudaEventRecord(ctx->e2, ctx->s));
    const int rc = add_host_batches(ctx, reads, offs, batches);
    CK(cudaEventRecord(ctx->e3, ctx->s));
    CK(cudaEventSynchronize(ctx->e3));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->e2, ctx->e3);
    ctx->times[0] = ms;
    return rc;
}

int gkc_batch_timings(gkc_ctx *ctx, double *ms, uint64_t cap, uint64_t *n) {
    if (!ctx) return GKC_EINVAL;
    if (n) *n = ctx->batch_ms.size();
    for (uint64_t i = 0; ms && i < cap && i < ctx->batch_ms.size(); i++) ms[i] = ctx->batch_ms[i];
    return GKC_OK;
}

int gkc_parse_fastx(gkc_ctx *ctx, const char *text, uint64_t n, int mem, int format, int *state, char *reads,
                    uint64_t cap_bases, uint64_t *offs, uint64_t cap_reads, int out_mem, uint64_t *n_reads,
                    uint64_t *n_bases) {
    if (!ctx || !n_reads || !n_bases) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    int st = 0;
    RET(parse_fastx(ctx, text, n, mem, format, state ? *state : 0, n_reads, n_bases, &st));
    if (state) *state = st;
    if (!reads && !offs) return GKC_OK;  // sizes only
    if (!reads || !offs || cap_bases < *n_bases || cap_reads < *n_reads + 1) return GKC_ELIMIT;
    const cudaMemcpyKind kind = out_mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (*n_bases) CK(cudaMemcpyAsync(reads, ctx->fx_out.p, *n_bases, kind, ctx->s));
    if (*n_reads) CK(cudaMemcpyAsync(offs, ctx->fx_offs.p, (*n_reads + 1) * 8, kind, ctx->s));
    else if (out_mem == GKC_MEM_DEVICE) CK(cudaMemsetAsync(offs, 0, 8, ctx->s));
    else offs[0] = 0;
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_add_skm(gkc_ctx *ctx, const uint8_t *bytes, const uint64_t *part_off, int mem) {
    if (!ctx || !part_off) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (char cn : ctx->counted)
        if (cn) return ctx->fail(GKC_ESTATE, "the store is partly counted; clear it before appending");
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    if (part_off[0] != 0) return ctx->fail(GKC_EINVAL, "part_off[0] must be 0");
    for (uint32_t p = 0; p < P; p++)
        if (part_off[p + 1] < part_off[p]) return ctx->fail(GKC_EINVAL, "part_off is not ascending");
    const uint64_t n = part_off[P];
    if (n == 0) return GKC_OK;
    if (!bytes) return GKC_EINVAL;
    StoreChunk *c = ctx->take_chunk();
    auto fail = [&](int rc) {
        ctx->pool.push_back(c);
        return rc;
    };
    cudaError_t e = c->dbytes.ensure(n + 32);
    if (e == cudaSuccess) e = c->d_byte_off.ensure((P + 1) * 8);
    if (e == cudaSuccess) e = c->d_skm_off.ensure((P + 1) * 8);
    if (e == cudaSuccess) e = c->d_kmers.ensure(P * 8ull);
    if (e == cudaSuccess) e = c->h_meta.ensure((3ull * P + 3) * 8);
    if (e != cudaSuccess) return fail(ctx->fail(GKC_ENOMEM, "skm chunk allocation: %s", cudaGetErrorString(e)));
    c->byte_off.assign(part_off, part_off + P + 1);
    uint8_t *db = c->dbytes.as<uint8_t>();
    if (cudaMemcpyAsync(db, bytes, n, mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        ctx->s) != cudaSuccess ||
        cudaMemsetAsync(db + n, 0, 32, ctx->s) != cudaSuccess ||
        cudaMemcpyAsync(c->d_byte_off.p, c->byte_off.data(), (P + 1) * 8, cudaMemcpyHostToDevice, ctx->s) !=
            cudaSuccess)
        return fail(ctx->fail(GKC_ECUDA, "skm staging copy failed"));
    // superkmer bounds
    const uint64_t ntiles = (n + gkc::SL_TILE - 1) / gkc::SL_TILE;
    if (ctx->sk_tiles.ensure(ntiles * sizeof(gkc::SlT)) != cudaSuccess || ctx->sk_state.ensure(ntiles) != cudaSuccess ||
        ctx->sk_tstarts.ensure(ntiles * 8) != cudaSuccess || ctx->sk_res.ensure(64) != cudaSuccess ||
        ctx->h_scal.ensure(64) != cudaSuccess)
        return fail(ctx->fail(GKC_ENOMEM, "skm scan buffers"));
    gkc::SlParams a;
    a.bytes = db;
    a.n = n;
    a.part_off = c->d_byte_off.as<unsigned long long>();
    a.P = P;
    a.tiles = ctx->sk_tiles.as<gkc::SlT>();
    a.ntiles = ntiles;
    a.tile_state = ctx->sk_state.as<uint8_t>();
    a.tile_starts = ctx->sk_tstarts.as<uint64_t>();
    a.result = ctx->sk_res.as<uint64_t>();
    a.err = reinterpret_cast<uint32_t *>(ctx->sk_res.as<uint64_t>() + 1);
    a.starts = nullptr;
    CK(cudaMemsetAsync(ctx->sk_res.p, 0, 64, ctx->s));
    gkc::skm_tile_kernel<<<(uint32_t)ntiles, gkc::SL_THREADS, 0, ctx->s>>>(a);
    LAUNCHED();
    gkc::skm_carry_kernel<<<1, gkc::SL_CARRY_THREADS, 0, ctx->s>>>(a);
    LAUNCHED();
    uint64_t *hr = ctx->h_scal.as<uint64_t>();
    CK(cudaMemcpyAsync(hr, ctx->sk_res.p, 16, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const uint64_t nskm = hr[0];
    if (ctx->sk_starts.ensure(std::max<uint64_t>(nskm, 1) * 8) != cudaSuccess ||
        ctx->sk_k32.ensure(std::max<uint64_t>(nskm, 1) * 4) != cudaSuccess ||
        c->didx.ensure(std::max<uint64_t>(nskm, 1) * 8) != cudaSuccess ||
        c->dkeys.ensure(std::max<uint64_t>(nskm, 1) * 4) != cudaSuccess)
        return fail(ctx->fail(GKC_ENOMEM, "skm index allocation (%llu superkmers)", (unsigned long long)nskm));
    a.starts = ctx->sk_starts.as<uint64_t>();
    gkc::skm_starts_kernel<<<(uint32_t)ntiles, gkc::SL_THREADS, 0, ctx->s>>>(a);
    LAUNCHED();
    gkc::SiParams x;
    x.bytes = db;
    x.n = n;
    x.part_off = a.part_off;
    x.P = P;
    x.part0 = 0;
    x.P_store = P;
    x.pmod = gkc::fastmod_m(P);
    x.k = ctx->opt.k;
    x.p = ctx->opt.p;
    x.lut = ctx->has_lut ? ctx->lut.as<uint32_t>() : nullptr;
    x.starts = a.starts;
    x.nskm = nskm;
    x.idx = c->didx.as<uint64_t>();
    x.keys = c->dkeys.as<uint32_t>();
    x.part_kmers32 = ctx->sk_k32.as<uint32_t>();
    x.err = a.err;
    const uint32_t g = (uint32_t)std::min<uint64_t>((nskm + 255) / 256, (uint64_t)ctx->sms * 8);
    if (nskm) {
        if (x.lut) gkc::skm_index_kernel<true><<<g, 256, 0, ctx->s>>>(x);
        else gkc::skm_index_kernel<false><<<g, 256, 0, ctx->s>>>(x);
        LAUNCHED();
    }
    gkc::skm_part_totals_kernel<<<P, 256, 0, ctx->s>>>(a.part_off, P, a.starts, nskm, x.part_kmers32,
                                                        c->d_skm_off.as<unsigned long long>(),
                                                        c->d_kmers.as<unsigned long long>());
    LAUNCHED();
    auto *hm = c->h_meta.as<unsigned long long>();
    CK(cudaMemcpyAsync(hm, c->d_skm_off.p, (P + 1) * 8, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(hm + P + 1, c->d_kmers.p, P * 8ull, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaMemcpyAsync(hr, ctx->sk_res.p, 16, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    const uint32_t err = (uint32_t)hr[1];
    if (err & gkc::SKM_ERR_TRUNCATED) return fail(ctx->fail(GKC_EINVAL, "skm bytes: a partition ends inside a superkmer"));
    if (err & gkc::SKM_ERR_SHORT) return fail(ctx->fail(GKC_EINVAL, "skm bytes: a superkmer holds fewer than k bases"));
    if (err & gkc::SKM_ERR_PARTITION)
        return fail(ctx->fail(GKC_EINVAL, "skm bytes: superkmers whose minimizer maps to another partition "
                                          "(written with another minimizer order, partition count or p)"));
    c->skm_off.assign(hm, hm + P + 1);
    c->kmers.assign(hm + P + 1, hm + 2 * P + 1);
    c->nbytes = n;
    c->nskm = nskm;
    c->bytes = db;
    c->idx = c->didx.as<uint64_t>();
    c->keys = c->dkeys.as<uint32_t>();
    c->on_host = false;
    c->pending = false;
    if (ctx->opt.spill_host) {
        const int rc = spill_chunk(ctx, c);
        if (rc != GKC_OK) return fail(rc);
    }
    ctx->store.push_back(c);
    return GKC_OK;
}

int gkc_add_fastx(gkc_ctx *ctx, const char *text, uint64_t n, int mem, int format, int *state, uint64_t *n_reads,
                  uint64_t *n_bases) {
    if (!ctx) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (char c : ctx->counted)
        if (c) return ctx->fail(GKC_ESTATE, "the store is partly counted; clear it before adding reads");
    uint64_t nr = 0, nb = 0;
    int st = 0;
    RET(parse_fastx(ctx, text, n, mem, format, state ? *state : 0, &nr, &nb, &st));
    if (state) *state = st;
    if (n_reads) *n_reads = nr;
    if (n_bases) *n_bases = nb;
    if (!nr) return GKC_OK;
    return gkc_add_reads(ctx, ctx->fx_out.as<char>(), ctx->fx_offs.as<uint64_t>(), nr, GKC_MEM_DEVICE);
}

int gkc_store_stats(gkc_ctx *ctx, uint64_t *pb, uint64_t *ps, uint64_t *pk) {
    if (!ctx) return GKC_EINVAL;
    const int P = ctx->opt.partitions;
    for (int p = 0; p < P; p++) {
        uint64_t b = 0, s = 0, k = 0;
        for (auto *c : ctx->store) {
            b += c->byte_off[p + 1] - c->byte_off[p];
            s += c->skm_off[p + 1] - c->skm_off[p];
            k += c->kmers[p];
        }
        if (pb) pb[p] = b;
        if (ps) ps[p] = s;
        if (pk) pk[p] = k;
    }
    return GKC_OK;
}

int gkc_store_export(gkc_ctx *ctx, int part, uint8_t *out, uint64_t cap, uint64_t *n) {
    if (!ctx || part < 0 || part >= ctx->opt.partitions || !n) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    RET(spill_sync(ctx));
    uint64_t total = 0;
    for (auto *c : ctx->store) total += c->byte_off[part + 1] - c->byte_off[part];
    *n = total;
    if (!out) return GKC_OK;
    if (cap < total) return ctx->fail(GKC_EINVAL, "export buffer too small (%llu < %llu)",
                                      (unsigned long long)cap, (unsigned long long)total);
    CK(cudaStreamSynchronize(ctx->s));  // spill copies still in flight
    uint64_t o = 0;
    for (auto *c : ctx->store) {
        uint64_t b0 = c->byte_off[part], b1 = c->byte_off[part + 1];
        if (b1 > b0)
            CK(cudaMemcpyAsync(out + o, c->bytes + b0, b1 - b0, c->on_host ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost,
                               ctx->s));
        o += b1 - b0;
    }
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_store_pack(gkc_ctx *ctx, int p0, int p1, uint8_t *bytes, uint64_t cap_bytes, uint64_t *idx, uint32_t *keys,
                   uint64_t cap_skms, uint64_t *counts) {
    if (!ctx || p0 < 0 || p1 < p0 || p1 > ctx->opt.partitions || !counts) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    RET(spill_sync(ctx));
    const uint32_t n = (uint32_t)(p1 - p0);
    for (int p = p0; p < p1; p++)
        if (!ctx->counted.empty() && ctx->counted[p])
            return ctx->fail(GKC_ESTATE, "partition %d was counted already", p);
    // per-partition totals and packed offsets
    std::vector<uint64_t> boff(n + 1, 0), soff(n + 1, 0);
    for (uint32_t j = 0; j < n; j++) {
        uint64_t b = 0, sk = 0, km = 0;
        for (auto *c : ctx->store) {
            b += c->byte_off[p0 + j + 1] - c->byte_off[p0 + j];
            sk += c->skm_off[p0 + j + 1] - c->skm_off[p0 + j];
            km += c->kmers[p0 + j];
        }
        counts[j] = b;
        counts[n + j] = sk;
        counts[2 * n + j] = km;
        boff[j + 1] = boff[j] + b;
        soff[j + 1] = soff[j] + sk;
    }
    if (!bytes && !idx && !keys) return GKC_OK;  // sizes only
    if (!bytes || !idx || !keys) return ctx->fail(GKC_EINVAL, "pack needs bytes, index and keys buffers");
    if (cap_bytes < boff[n] || cap_skms < soff[n])
        return ctx->fail(GKC_EINVAL, "pack buffers too small (%llu < %llu bytes or %llu < %llu superkmers)",
                         (unsigned long long)cap_bytes, (unsigned long long)boff[n], (unsigned long long)cap_skms,
                         (unsigned long long)soff[n]);
    std::vector<uint64_t> within(n, 0), within_s(n, 0);  // bytes / superkmers of the chunks before
    std::vector<PackDesc> d;
    bool spilled = false;
    for (auto *c : ctx->store) spilled |= c->on_host;
    if (spilled) {  // the largest chunk range staged at a time
        uint64_t mx = 0;
        for (auto *c : ctx->store)
            if (c->on_host)
                mx = std::max<uint64_t>(mx, c->byte_off[p1] - c->byte_off[p0] +
                                                12 * (c->skm_off[p1] - c->skm_off[p0]));
        CK(ctx->bk_arena.ensure(mx + 96 + 64));
    }
    // device chunks are gathered in one launch; a spilled chunk is staged and
    // gathered on its own, since the staging buffer is reused
    auto flush = [&]() -> int {
        if (d.empty()) return GKC_OK;
        CK(ctx->tiles.ensure(d.size() * sizeof(PackDesc)));
        CK(cudaMemcpyAsync(ctx->tiles.p, d.data(), d.size() * sizeof(PackDesc), cudaMemcpyHostToDevice, ctx->s));
        pack_gather_kernel<<<(uint32_t)d.size(), PK_THREADS, 0, ctx->s>>>(ctx->tiles.as<PackDesc>(), bytes, idx, keys);
        LAUNCHED();
        CK(cudaStreamSynchronize(ctx->s));  // the descriptors (pageable) and the staging are reused
        d.clear();
        return GKC_OK;
    };
    for (auto *c : ctx->store) {
        const uint8_t *cb;
        const uint64_t *ci;
        const uint32_t *ck;
        uint64_t used = 0;
        if (c->on_host) RET(flush());
        RET(chunk_range(ctx, c, (uint32_t)p0, (uint32_t)p1, ctx->bk_arena, &used, &cb, &ci, &ck));
        for (uint32_t j = 0; j < n; j++) {
            const uint32_t p = p0 + j;
            const uint64_t nb = c->byte_off[p + 1] - c->byte_off[p], ns = c->skm_off[p + 1] - c->skm_off[p];
            if (!nb && !ns) continue;
            d.push_back({cb + c->byte_off[p], ci + c->skm_off[p], ck + c->skm_off[p], boff[j] + within[j],
                         soff[j] + within_s[j], nb, ns, within[j]});
            within[j] += nb;
            within_s[j] += ns;
        }
        if (c->on_host) RET(flush());
    }
    RET(flush());
    return GKC_OK;
}

int gkc_store_append(gkc_ctx *ctx, int p0, int p1, const uint8_t *bytes, const uint64_t *idx, const uint32_t *keys,
                     const uint64_t *counts) {
    if (!ctx || p0 < 0 || p1 < p0 || p1 > ctx->opt.partitions || !counts) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    for (int p = p0; p < p1 && !ctx->counted.empty(); p++)  // partitions not yet counted may still grow
        if (ctx->counted[p]) return ctx->fail(GKC_ESTATE, "partition %d was counted already", p);
    const uint32_t P = (uint32_t)ctx->opt.partitions, n = (uint32_t)(p1 - p0);
    uint64_t nb = 0, ns = 0;
    for (uint32_t j = 0; j < n; j++) nb += counts[j], ns += counts[n + j];
    if (!ns) return GKC_OK;
    if (!bytes || !idx || !keys) return GKC_EINVAL;
    StoreChunk *c = ctx->take_chunk();
    c->byte_off.assign(P + 1, 0);
    c->skm_off.assign(P + 1, 0);
    c->kmers.assign(P, 0);
    for (uint32_t p = 0; p < P; p++) {
        const bool in = p >= (uint32_t)p0 && p < (uint32_t)p1;
        c->byte_off[p + 1] = c->byte_off[p] + (in ? counts[p - p0] : 0);
        c->skm_off[p + 1] = c->skm_off[p] + (in ? counts[n + p - p0] : 0);
        c->kmers[p] = in ? counts[2 * n + p - p0] : 0;
    }
    c->nbytes = nb;
    c->nskm = ns;
    c->on_host = false;
    c->pending = false;
    DevBuf *db = &c->dbytes, *di = &c->didx, *dk = &c->dkeys;
    if (ctx->opt.spill_host) {
        const int rc = spill_slot(ctx, nb, ns, &db, &di, &dk);
        if (rc != GKC_OK) {
            ctx->pool.push_back(c);
            return rc;
        }
    }
    cudaError_t e = db->ensure(nb + 32);
    if (e == cudaSuccess) e = di->ensure(ns * 8);
    if (e == cudaSuccess) e = dk->ensure(ns * 4);
    if (e == cudaSuccess) e = c->d_byte_off.ensure((P + 1) * 8);
    if (e == cudaSuccess) e = c->d_skm_off.ensure((P + 1) * 8);
    if (e != cudaSuccess) {
        ctx->pool.push_back(c);
        return ctx->fail(GKC_ENOMEM, "appended chunk allocation (%llu bytes): %s", (unsigned long long)nb,
                         cudaGetErrorString(e));
    }
    c->bytes = db->as<uint8_t>();
    c->idx = di->as<uint64_t>();
    c->keys = dk->as<uint32_t>();
    // cudaMemcpyDefault: the packed range may be in device or host memory
    CK(cudaMemcpyAsync(c->bytes, bytes, nb, cudaMemcpyDefault, ctx->s));
    CK(cudaMemsetAsync(c->bytes + nb, 0, 32, ctx->s));
    CK(cudaMemcpyAsync(c->idx, idx, ns * 8, cudaMemcpyDefault, ctx->s));
    CK(cudaMemcpyAsync(c->keys, keys, ns * 4, cudaMemcpyDefault, ctx->s));
    CK(cudaMemcpyAsync(c->d_byte_off.p, c->byte_off.data(), (P + 1) * 8, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemcpyAsync(c->d_skm_off.p, c->skm_off.data(), (P + 1) * 8, cudaMemcpyHostToDevice, ctx->s));
    if (ctx->opt.spill_host) {
        const int rc = spill_chunk(ctx, c);
        if (rc != GKC_OK) {
            ctx->pool.push_back(c);
            return rc;
        }
    }
    ctx->store.push_back(c);
    // the caller may free or reuse its buffers when this returns
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_pack_bases(const char *bases, uint64_t n, uint32_t *words) {
    if ((!bases || !words) && n) return GKC_EINVAL;
    gkc_host::pack_bases(reinterpret_cast<const uint8_t *>(bases), n, words, (n + 15) / 16);
    return GKC_OK;
}

int gkc_reserve_host(gkc_ctx *ctx, uint64_t bytes, uint64_t *pinned) {
    if (!ctx) return GKC_EINVAL;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return GKC_ECUDA;
    const cudaError_t e = ctx->arena.reserve(bytes);
    if (pinned) *pinned = ctx->arena.pinned();
    // not ctx->fail: the error text belongs to the thread running batches
    return e == cudaSuccess ? GKC_OK : GKC_ENOMEM;
}

int gkc_store_clear(gkc_ctx *ctx) {
    if (!ctx) return GKC_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->s);
    spill_sync(ctx);     // the arena is rewound
    ctx->clear_store();  // buffers stay pooled for the next batch
    ctx->counted.assign(ctx->counted.size(), 0);
    return GKC_OK;
}

}  // extern "C"

namespace {

// Counts the partitions `want` (null: all) of the store; the result replaces
// the previous one.
int count_store(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, const std::vector<char> *want, uint64_t *n_out,
                uint64_t *n_distinct) {
    CK(cudaSetDevice(ctx->device));
    RET(spill_sync(ctx));
    ctx->n_out = 0;
    ctx->n_distinct = 0;
    ctx->has_result = false;
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, ctx->s));
    // k > 32: u128 keys (the hash counter's 128-bit tables, or the sort counter)
    ctx->res_kw = ctx->opt.k > 32 ? 2 : 1;
    int rc = ctx->opt.k > 32 ? (ctx->opt.counter == GKC_COUNTER_HASH ? count_hash_wide(ctx, cmin, cmax, want)
                                                                     : count_sort<u128>(ctx, cmin, cmax, want))
             : ctx->opt.counter == GKC_COUNTER_HASH ? count_hash(ctx, cmin, cmax, want)
                                                    : count_sort<uint64_t>(ctx, cmin, cmax, want);
    cudaEventRecord(t1, ctx->s);
    cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    ctx->times[2] = ms;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != GKC_OK) return rc;
    ctx->has_result = true;
    if (n_out) *n_out = ctx->n_out;
    if (n_distinct) *n_distinct = ctx->n_distinct;
    return GKC_OK;
}

}  // namespace

extern "C" {

int gkc_count(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, uint64_t *n_out, uint64_t *n_distinct) {
    if (!ctx || cmin > cmax) return GKC_EINVAL;
    for (char c : ctx->counted)
        if (c) return ctx->fail(GKC_ESTATE, "partitions of this store were counted already");
    const int rc = count_store(ctx, cmin, cmax, nullptr, n_out, n_distinct);
    gkc_store_clear(ctx);
    return rc;
}

int gkc_count_partitions(gkc_ctx *ctx, const int32_t *parts, uint64_t n, uint32_t cmin, uint32_t cmax,
                         uint64_t *n_out, uint64_t *n_distinct) {
    if (!ctx || cmin > cmax || (!parts && n)) return GKC_EINVAL;
    const uint32_t P = (uint32_t)ctx->opt.partitions;
    if (ctx->counted.size() != P) ctx->counted.assign(P, 0);
    std::vector<char> want(P, 0);
    for (uint64_t i = 0; i < n; i++) {
        if (parts[i] < 0 || (uint32_t)parts[i] >= P) return ctx->fail(GKC_EINVAL, "partition %d out of range", parts[i]);
        if (ctx->counted[parts[i]] || want[parts[i]])
            return ctx->fail(GKC_ESTATE, "partition %d counted twice", parts[i]);
        want[parts[i]] = 1;
    }
    const int rc = count_store(ctx, cmin, cmax, &want, n_out, n_distinct);
    if (rc != GKC_OK) return rc;
    bool all = true;
    for (uint32_t p = 0; p < P; p++) {
        ctx->counted[p] |= want[p];
        all &= ctx->counted[p] != 0;
    }
    if (all) gkc_store_clear(ctx);  // every partition is counted: release the store
    return GKC_OK;
}

// ---- the boundary in five calls (thin forms of the calls in this file) ----
int gkc_init(int device, const gkc_options *config, gkc_ctx **out) { return gkc_create(device, config, out); }

int gkc_skmgen_batch(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int k, int p, int P,
                     const uint32_t *order_lut, int mem, uint64_t *part_bytes, uint64_t *part_skms,
                     uint64_t *part_kmers) {
    if (!ctx) return GKC_EINVAL;
    if (k != ctx->opt.k || p != ctx->opt.p || P != ctx->opt.partitions)
        return ctx->fail(GKC_EINVAL, "k, p and P of a batch must be the context's (%d, %d, %d)", ctx->opt.k,
                         ctx->opt.p, ctx->opt.partitions);
    if (order_lut) {
        if (!ctx->store.empty()) return ctx->fail(GKC_ESTATE, "the order of a non-empty store cannot change");
        RET(gkc_set_order(ctx, order_lut, 1ull << (2 * p), GKC_MEM_HOST));
    }
    RET(gkc_add_reads(ctx, reads, offs, n_reads, mem));
    return gkc_store_stats(ctx, part_bytes, part_skms, part_kmers);
}

int gkc_count_partition(gkc_ctx *ctx, int part, uint32_t cmin, uint32_t cmax, uint64_t *kmers, uint32_t *counts,
                        uint64_t cap, int mem, uint64_t *n_out, uint64_t *n_distinct) {
    if (!ctx) return GKC_EINVAL;
    const int32_t id = part;
    uint64_t no = 0, nd = 0;
    RET(gkc_count_partitions(ctx, &id, 1, cmin, cmax, &no, &nd));
    if (n_out) *n_out = no;
    if (n_distinct) *n_distinct = nd;
    if (kmers || counts) {
        if (cap < no)
            return ctx->fail(GKC_EINVAL, "output buffer too small (%llu < %llu)", (unsigned long long)cap,
                             (unsigned long long)no);
        RET(gkc_result(ctx, kmers, counts, cap, mem));
    }
    return GKC_OK;
}

int gkc_set_order_lut(gkc_ctx *ctx, const uint32_t *lut) {
    if (!ctx) return GKC_EINVAL;
    return gkc_set_order(ctx, lut, 1ull << (2 * ctx->opt.p), GKC_MEM_HOST);
}

int gkc_shutdown(gkc_ctx *ctx) { return gkc_destroy(ctx); }

int gkc_result(gkc_ctx *ctx, uint64_t *kmers, uint32_t *counts, uint64_t cap, int mem) {
    if (!ctx) return GKC_EINVAL;
    if (!ctx->has_result) return ctx->fail(GKC_ESTATE, "no result: call gkc_count first");
    CK(cudaSetDevice(ctx->device));
    uint64_t n = std::min(cap, ctx->n_out);
    cudaMemcpyKind kind = mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (n && kmers) CK(cudaMemcpyAsync(kmers, ctx->out_k.p, n * 8 * ctx->res_kw, kind, ctx->s));
    if (n && counts) CK(cudaMemcpyAsync(counts, ctx->out_c.p, n * 4, kind, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_result_device(gkc_ctx *ctx, const uint64_t **kmers, const uint32_t **counts, uint64_t *n) {
    if (!ctx) return GKC_EINVAL;
    if (!ctx->has_result) return ctx->fail(GKC_ESTATE, "no result: call gkc_count first");
    if (kmers) *kmers = ctx->out_k.as<uint64_t>();
    if (counts) *counts = ctx->out_c.as<uint32_t>();
    if (n) *n = ctx->n_out;
    return GKC_OK;
}

int gkc_count_reads(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int mem,
                    uint32_t cmin, uint32_t cmax, uint64_t *kmers, uint32_t *counts, uint64_t cap, int out_mem,
                    uint64_t *n_out, uint64_t *n_distinct) {
    if (!ctx) return GKC_EINVAL;
    RET(gkc_store_clear(ctx));
    RET(gkc_add_reads(ctx, reads, offs, n_reads, mem));
    uint64_t no = 0, nd = 0;
    // host output with the hash counter: each group's k-mers are copied out
    // while the next group counts
    ctx->streamed = 0;
    if (kmers && counts && out_mem == GKC_MEM_HOST && ctx->opt.counter == GKC_COUNTER_HASH && ctx->opt.k <= 32) {
        ctx->stream_k = kmers;
        ctx->stream_c = counts;
        ctx->stream_cap = cap;
    }
    const int rc = gkc_count(ctx, cmin, cmax, &no, &nd);
    ctx->stream_k = nullptr;
    ctx->stream_c = nullptr;
    ctx->stream_cap = 0;
    RET(rc);
    if (n_out) *n_out = no;
    if (n_distinct) *n_distinct = nd;
    if (kmers || counts) {
        if (cap < no) return ctx->fail(GKC_EINVAL, "output buffer too small (%llu < %llu)",
                                       (unsigned long long)cap, (unsigned long long)no);
        if (ctx->streamed != no) RET(gkc_result(ctx, kmers, counts, cap, out_mem));
    }
    return GKC_OK;
}

int gkc_count_keys(gkc_ctx *ctx, const uint64_t *keys, uint64_t n, int mem, uint32_t cmin, uint32_t cmax,
                   uint64_t *n_out, uint64_t *n_distinct) {
    if (!ctx || (!keys && n) || cmin > cmax) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    ctx->n_out = 0;
    ctx->n_distinct = 0;
    ctx->has_result = false;
    ctx->res_kw = 1;  // the keys are u64 whatever the context's k
    if (ctx->opt.counter == GKC_COUNTER_HASH) {
        const double slots = ctx->opt.table_slots > 0 ? ctx->opt.table_slots : 0.35;
        const void *dk;
        RET(upload(ctx, ctx->keysA, keys, n * 8, mem, &dk));
        RET(ensure_out(ctx, n / std::max<uint32_t>(cmin, 1) + 1024, 0));
        CK(ctx->part_err.ensure(64));
        CK(ctx->scal.ensure(64));
        CK(ctx->h_scal.ensure(64));
        for (int scale = 1;; scale *= 4) {
            uint64_t C = next_pow2(std::max<uint64_t>(1024, (uint64_t)((double)n * slots) * scale));
            RET(ensure_table(ctx, C));
            CK(cudaMemsetAsync(ctx->part_err.p, 0, 64, ctx->s));
            CK(cudaMemsetAsync(ctx->scal.p, 0, 64, ctx->s));
            auto *sc = ctx->scal.as<unsigned long long>();
            if (n) {
                uint32_t g = (uint32_t)std::min<uint64_t>((n + H_THREADS - 1) / H_THREADS, (uint64_t)ctx->sms * 8);
                KScope ks(ctx, GKC_K_HASH_INSERT, 8.0 * n);
                hash_insert_keys_kernel<<<g, H_THREADS, 0, ctx->s>>>(
                    reinterpret_cast<const uint64_t *>(dk), n, ctx->table.as<HSlot>(), C - 1,
                    ctx->part_err.as<uint32_t>());
                LAUNCHED();
            }
            HCollectParams q;
            q.tab = ctx->table.as<HSlot>();
            q.cap = C;
            q.cmin = cmin;
            q.cmax = cmax;
            q.out_k = ctx->out_k.as<uint64_t>();
            q.out_c = ctx->out_c.as<uint32_t>();
            q.out_cursor = sc;
            q.out_cap = ctx->out_cap;
            q.distinct = sc + 1;
            q.err = reinterpret_cast<uint32_t *>(sc + 2);
            q.part_err = ctx->part_err.as<uint32_t>();
            uint32_t g = (uint32_t)std::min<uint64_t>((C + H_THREADS * HC_ITEMS - 1) / (H_THREADS * HC_ITEMS),
                                                      (uint64_t)ctx->sms * 8);
            {
                KScope ks(ctx, GKC_K_HASH_COLLECT, 24.0 * C);
                hash_collect_kernel<<<g, H_THREADS, 0, ctx->s>>>(q);
                LAUNCHED();
            }
            uint32_t perr = 0;
            CK(cudaMemcpyAsync(&perr, ctx->part_err.p, 4, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaMemcpyAsync(ctx->h_scal.p, sc, 24, cudaMemcpyDeviceToHost, ctx->s));
            CK(cudaStreamSynchronize(ctx->s));
            if (perr & ERR_DECODE) return ctx->fail(GKC_EINVAL, "key 2^64-1 is reserved");
            if (perr & ERR_TABLE_FULL) {
                if (scale >= 64) return ctx->fail(GKC_EINTERNAL, "hash table retries exhausted");
                continue;
            }
            auto *hs = ctx->h_scal.as<unsigned long long>();
            ctx->n_out = hs[0];
            ctx->n_distinct = hs[1];
            break;
        }
    } else {
        CK(ctx->keysA.ensure(n * 8 + 8));
        CK(ctx->keysB.ensure(n * 8 + 8));
        CK(cudaMemcpyAsync(ctx->keysA.p, keys, n * 8, mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           ctx->s));
        std::vector<uint64_t> segs{n};
        float ms = 0;
        RET(sort_and_reduce(ctx, segs, n, 64, cmin, cmax, &ms));
        ctx->times[3] = ms;
    }
    ctx->has_result = true;
    if (n_out) *n_out = ctx->n_out;
    if (n_distinct) *n_distinct = ctx->n_distinct;
    return GKC_OK;
}

int gkc_set_stream(gkc_ctx *ctx, void *stream) {
    if (!ctx) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->s));
    ctx->s = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->own_s;
    return GKC_OK;
}

int gkc_set_profiling(gkc_ctx *ctx, int on) {
    if (!ctx) return GKC_EINVAL;
    ctx->prof_flush();
    ctx->prof = on != 0;
    return GKC_OK;
}

int gkc_kernel_stats(gkc_ctx *ctx, double *ms, uint64_t *launches, double *bytes, int n, int reset) {
    if (!ctx || n < 0) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    ctx->prof_flush();
    for (int i = 0; i < n && i < GKC_K_CLASSES; i++) {
        if (ms) ms[i] = ctx->kms[i];
        if (launches) launches[i] = ctx->klaunch[i];
        if (bytes) bytes[i] = ctx->kbytes[i];
    }
    if (reset)
        for (int i = 0; i < GKC_K_CLASSES; i++) ctx->kms[i] = ctx->kbytes[i] = 0, ctx->klaunch[i] = 0;
    return GKC_OK;
}

int gkc_last_timings(gkc_ctx *ctx, double *t, int n) {
    if (!ctx || !t) return GKC_EINVAL;
    ctx->times[9] = (double)ctx->h2d_bytes;
    for (int i = 0; i < n && i < 10; i++) t[i] = ctx->times[i];
    return GKC_OK;
}

// ---------------------------------------------------------------------------
// learned minimizer order

uint64_t gkc_mlp_param_count(int p) {
    if (p < 1 || p > MLP_MAX_P) return 0;
    return mlp_layout(p).n;
}

int gkc_minimizer_loads(gkc_ctx *ctx, uint64_t *loads, uint64_t n, int mem) {
    if (!ctx || !loads) return GKC_EINVAL;
    CK(cudaSetDevice(ctx->device));
    RET(spill_sync(ctx));
    const uint64_t np = 1ull << (2 * ctx->opt.p);
    if (n != np) return ctx->fail(GKC_EINVAL, "minimizer loads need 4^p = %llu entries", (unsigned long long)np);
    CK(ctx->ord_loads.ensure(np * 8));
    CK(cudaMemsetAsync(ctx->ord_loads.p, 0, np * 8, ctx->s));
    for (StoreChunk *c : ctx->store) {
        if (!c->nskm) continue;
        const uint64_t *idx = c->idx;
        const uint32_t *keys = c->keys;
        if (c->on_host) {  // a spilled chunk: stage it, its index and keys rebuilt
            const uint64_t nbb = (c->nbytes + 32 + 15) / 16 * 16;
            CK(ctx->ord_stage.ensure(nbb + c->nskm * 12));
            uint8_t *sb = ctx->ord_stage.as<uint8_t>();
            RET(stage_spilled(ctx, c, 0, (uint32_t)ctx->opt.partitions, sb, reinterpret_cast<uint64_t *>(sb + nbb),
                              reinterpret_cast<uint32_t *>(sb + nbb + c->nskm * 8), ctx->s));
            idx = reinterpret_cast<const uint64_t *>(sb + nbb);
            keys = reinterpret_cast<const uint32_t *>(sb + nbb + c->nskm * 8);
        }
        const uint32_t g = (uint32_t)std::min<uint64_t>((c->nskm + 255) / 256, (uint64_t)ctx->sms * 8);
        minimizer_loads_kernel<<<g, 256, 0, ctx->s>>>(idx, keys, c->nskm, (uint32_t)(np - 1),
                                                      ctx->ord_loads.as<unsigned long long>());
        LAUNCHED();
        if (c->on_host) CK(cudaStreamSynchronize(ctx->s));  // the staging buffer is reused
    }
    CK(cudaMemcpyAsync(loads, ctx->ord_loads.p, np * 8,
                       mem == GKC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

namespace {

// Device copies of the network inputs; targets/weights are 4^p arrays.
int mlp_upload(gkc_ctx *ctx, const float *params, const float *targets, const float *weights) {
    const int p = ctx->opt.p;
    const MlpLayout L = mlp_layout(p);
    const uint64_t np = 1ull << (2 * p);
    CK(ctx->mlp_p.ensure(L.n * 4));
    CK(ctx->mlp_g.ensure(L.n * 4));
    CK(ctx->mlp_scalar.ensure(64));
    CK(cudaMemcpyAsync(ctx->mlp_p.p, params, L.n * 4, cudaMemcpyHostToDevice, ctx->s));
    if (targets) {
        CK(ctx->mlp_t.ensure(np * 4));
        CK(cudaMemcpyAsync(ctx->mlp_t.p, targets, np * 4, cudaMemcpyHostToDevice, ctx->s));
    }
    if (weights) {
        CK(ctx->mlp_w.ensure(np * 4));
        CK(cudaMemcpyAsync(ctx->mlp_w.p, weights, np * 4, cudaMemcpyHostToDevice, ctx->s));
    }
    return GKC_OK;
}

int mlp_launch(gkc_ctx *ctx, const uint32_t *pmers, uint64_t s0, uint64_t n, bool weights, float norm, bool train,
               float *scores) {
    const int p = ctx->opt.p;
    MlpParams a;
    a.params = ctx->mlp_p.as<float>();
    a.L = mlp_layout(p);
    a.pmers = pmers;
    a.s0 = s0;
    a.n = n;
    a.targets = train ? ctx->mlp_t.as<float>() : nullptr;
    a.weights = train && weights ? ctx->mlp_w.as<float>() : nullptr;
    a.norm = norm;
    a.grad = train ? ctx->mlp_g.as<float>() : nullptr;
    a.loss = train ? ctx->mlp_scalar.as<float>() : nullptr;
    a.scores = scores;
    const size_t sm = mlp_smem_floats(p) * 4;
    CK(cudaFuncSetAttribute(mlp_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    mlp_tile_kernel<<<(unsigned)((n + MLP_TILE - 1) / MLP_TILE), MLP_THREADS, sm, ctx->s>>>(a);
    LAUNCHED();
    return GKC_OK;
}

}  // namespace

int gkc_mlp_grad(gkc_ctx *ctx, const float *params, const uint32_t *pmers, uint64_t n, const float *targets,
                 const float *weights, float norm, float *grad, float *loss) {
    if (!ctx || !params || !pmers || !targets || !grad || n == 0) return GKC_EINVAL;
    const int p = ctx->opt.p;
    if (p > MLP_MAX_P) return ctx->fail(GKC_EINVAL, "the network supports p <= %d", MLP_MAX_P);
    CK(cudaSetDevice(ctx->device));
    const MlpLayout L = mlp_layout(p);
    const uint64_t np = 1ull << (2 * p);
    for (uint64_t i = 0; i < n; i++)
        if (pmers[i] >= np) return ctx->fail(GKC_EINVAL, "sample %llu is not a %d-mer", (unsigned long long)i, p);
    RET(mlp_upload(ctx, params, targets, weights));
    CK(ctx->mlp_s.ensure(n * 4));
    CK(cudaMemcpyAsync(ctx->mlp_s.p, pmers, n * 4, cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemsetAsync(ctx->mlp_g.p, 0, L.n * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->mlp_scalar.p, 0, 4, ctx->s));
    RET(mlp_launch(ctx, ctx->mlp_s.as<uint32_t>(), 0, n, weights != nullptr, norm, true, nullptr));
    CK(cudaMemcpyAsync(grad, ctx->mlp_g.p, L.n * 4, cudaMemcpyDeviceToHost, ctx->s));
    if (loss) CK(cudaMemcpyAsync(loss, ctx->mlp_scalar.p, 4, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_mlp_train(gkc_ctx *ctx, float *params, const float *targets, const float *weights, int epochs, int batch,
                  float lr, uint64_t seed, float *loss) {
    if (!ctx || !params || !targets || epochs < 0 || batch < 1 || !(lr > 0.f)) return GKC_EINVAL;
    const int p = ctx->opt.p;
    if (p > MLP_MAX_P) return ctx->fail(GKC_EINVAL, "the network supports p <= %d", MLP_MAX_P);
    CK(cudaSetDevice(ctx->device));
    const MlpLayout L = mlp_layout(p);
    const uint64_t np = 1ull << (2 * p);
    RET(mlp_upload(ctx, params, targets, weights));
    CK(ctx->mlp_m.ensure(L.n * 4));
    CK(ctx->mlp_v.ensure(L.n * 4));
    CK(ctx->mlp_s.ensure(np * 4));
    CK(cudaMemsetAsync(ctx->mlp_m.p, 0, L.n * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->mlp_v.p, 0, L.n * 4, ctx->s));
    CK(cudaMemsetAsync(ctx->mlp_g.p, 0, L.n * 4, ctx->s));
    // batch loss = sum_s w_s e_s^2 / (batch * mean weight)
    double wmean = 1.0;
    if (weights) {
        double sw = 0;
        for (uint64_t i = 0; i < np; i++) sw += weights[i];
        wmean = sw / (double)np;
        if (!(wmean > 0)) return ctx->fail(GKC_EINVAL, "weights sum to zero");
    }
    const float norm = (float)(1.0 / ((double)batch * wmean));
    AdamParams ap;
    ap.params = ctx->mlp_p.as<float>();
    ap.m = ctx->mlp_m.as<float>();
    ap.v = ctx->mlp_v.as<float>();
    ap.grad = ctx->mlp_g.as<float>();
    ap.n = L.n;
    ap.lr = lr;
    ap.beta1 = 0.9f;
    ap.beta2 = 0.999f;
    ap.eps = 1e-8f;
    uint64_t step = 0;
    float last = 0.f;
    for (int e = 0; e < epochs; e++) {
        const uint32_t key = (uint32_t)(seed * 0x9E3779B97F4A7C15ull >> 32) ^ (uint32_t)(e * 0x85EBCA6Bu);
        epoch_samples_kernel<<<(unsigned)std::min<uint64_t>((np + 255) / 256, (uint64_t)ctx->sms * 8), 256, 0,
                               ctx->s>>>(ctx->mlp_s.as<uint32_t>(), (uint32_t)np, 2 * p, key);
        LAUNCHED();
        CK(cudaMemsetAsync(ctx->mlp_scalar.p, 0, 4, ctx->s));
        for (uint64_t b0 = 0; b0 < np; b0 += (uint64_t)batch) {
            const uint64_t nb = std::min<uint64_t>((uint64_t)batch, np - b0);
            RET(mlp_launch(ctx, ctx->mlp_s.as<uint32_t>() + b0, 0, nb, weights != nullptr, norm, true, nullptr));
            step++;
            ap.c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)step)));
            ap.c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)step)));
            mlp_adam_kernel<<<(L.n + 255) / 256, 256, 0, ctx->s>>>(ap);
            LAUNCHED();
        }
        CK(cudaMemcpyAsync(&last, ctx->mlp_scalar.p, 4, cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
    }
    // mean per-batch loss of the last epoch
    if (loss) *loss = last / (float)((np + batch - 1) / batch);
    CK(cudaMemcpyAsync(params, ctx->mlp_p.p, L.n * 4, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_mlp_scores(gkc_ctx *ctx, const float *params, float *scores, int mem) {
    if (!ctx || !params || !scores) return GKC_EINVAL;
    const int p = ctx->opt.p;
    if (p > MLP_MAX_P) return ctx->fail(GKC_EINVAL, "the network supports p <= %d", MLP_MAX_P);
    CK(cudaSetDevice(ctx->device));
    const uint64_t np = 1ull << (2 * p);
    RET(mlp_upload(ctx, params, nullptr, nullptr));
    float *d = scores;
    if (mem != GKC_MEM_DEVICE) {
        CK(ctx->ord_stage.ensure(np * 4));
        d = ctx->ord_stage.as<float>();
    }
    RET(mlp_launch(ctx, nullptr, 0, np, false, 0.f, false, d));
    if (mem != GKC_MEM_DEVICE) CK(cudaMemcpyAsync(scores, d, np * 4, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return GKC_OK;
}

int gkc_mlp_order(gkc_ctx *ctx, const float *params, uint64_t heavy, uint32_t *lut_out) {
    if (!ctx || !params) return GKC_EINVAL;
    const int p = ctx->opt.p;
    if (p > ORDER_MAX_P) return ctx->fail(GKC_EINVAL, "the learned order supports p <= %d", ORDER_MAX_P);
    CK(cudaSetDevice(ctx->device));
    const uint32_t np = 1u << (2 * p);
    // scores of every p-mer
    std::vector<float> sc(np);
    RET(gkc_mlp_scores(ctx, params, sc.data(), GKC_MEM_HOST));
    // the `heavy` highest-scoring p-mers get levels 1 .. 2^(32-2p)-2 by score
    const uint32_t K = (uint32_t)std::min<uint64_t>(heavy ? heavy : np / 4, np);
    std::vector<uint32_t> ids(np);
    for (uint32_t v = 0; v < np; v++) ids[v] = v;
    auto higher = [&](uint32_t x, uint32_t y) { return sc[x] > sc[y] || (sc[x] == sc[y] && x < y); };
    std::nth_element(ids.begin(), ids.begin() + K, ids.end(), higher);
    ids.resize(K);
    const uint32_t lmax = (1u << (32 - 2 * p)) - 2;
    float lo = K ? sc[ids[0]] : 0.f, hi = lo;
    for (uint32_t v : ids) lo = std::min(lo, sc[v]), hi = std::max(hi, sc[v]);
    std::vector<uint32_t> vl(2 * (size_t)K);
    for (uint32_t i = 0; i < K; i++) {
        const float f = hi > lo ? (sc[ids[i]] - lo) / (hi - lo) : 0.f;
        vl[2 * i] = ids[i];
        vl[2 * i + 1] = 1 + std::min<uint32_t>(lmax - 1, (uint32_t)(f * (float)(lmax - 1)));
    }
    CK(ctx->ord_list.ensure(std::max<size_t>(vl.size(), 2) * 4));
    CK(cudaMemcpyAsync(ctx->ord_list.p, vl.data(), vl.size() * 4, cudaMemcpyHostToDevice, ctx->s));
    CK(ctx->ord_stage.ensure(np * 4ull));
    uint32_t *ranks = ctx->ord_stage.as<uint32_t>();
    const uint32_t g = (uint32_t)std::min<uint64_t>((np + 255) / 256, (uint64_t)ctx->sms * 8);
    order_mix_kernel<<<g, 256, 0, ctx->s>>>(np, p, ranks);
    LAUNCHED();
    order_levels_kernel<<<(K + 255) / 256 + 1, 256, 0, ctx->s>>>(ctx->ord_list.as<uint2>(), K, p, ranks);
    LAUNCHED();
    if (lut_out) CK(cudaMemcpyAsync(lut_out, ranks, np * 4ull, cudaMemcpyDeviceToHost, ctx->s));
    RET(install_order(ctx, ranks));
    return GKC_OK;
}

}  // extern "C"

#include "count_noalloc.cu"
