// gkc_b200_shim.cpp -- RapidGKC's GPU entry points on the B200 counter.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "gpu_skmgen.h"        // PinnedCSR, GenSuperkmerGPU, GPUReset, CountTask
#include "gpu_kmercounting.h"  // kmc_counting_GPU_streams
#include "skmstore.hpp"        // SKMStoreNoncon
#include "utilities.hpp"       // CUDAParams, T_kmc
#include "gkc_capi.h"          // this library

namespace {
struct Device {
    std::mutex mu;                      // a context is used by one thread at a time
    gkc_ctx *ctx = nullptr;
    std::vector<uint64_t> pb, ps, pk;   // store totals already added to the SKMStoreNoncon counters
};
Device g_dev[16];

void check(int rc, gkc_ctx *ctx) {      // the reference exits on CUDA errors (CUDA_CHECK)
    if (rc != GKC_OK) {
        std::fprintf(stderr, "B200 counter: %s (%s)\n", gkc_strerror(rc), ctx ? gkc_last_error(ctx) : "");
        std::exit(1);
    }
}

gkc_ctx *context(int did, int k, int p, int P) {
    Device &d = g_dev[did];
    if (!d.ctx) {
        gkc_options o;
        gkc_default_options(&o);
        o.k = k;
        o.p = p;
        o.partitions = P;
        o.counter = GKC_COUNTER_HASH;   // GKC_COUNTER_SORT for the reference's sort semantics (sorted output)
        check(gkc_create(did, &o, &d.ctx), nullptr);
        d.pb.assign(P, 0); d.ps.assign(P, 0); d.pk.assign(P, 0);
    }
    return d.ctx;
}
}  // namespace

// gpu_skmgen.cu defined PinnedCSR (gpu_skmgen.h:29-42); this file replaces it:
// the batch's reads concatenated into pinned host memory with u64 offsets.
PinnedCSR::PinnedCSR(std::vector<ReadPtr> &reads, bool /*keep_original*/) {
    n_reads = reads.size();
    size_capacity = 0;
    for (const ReadPtr &r : reads) size_capacity += r.len;
    if (cudaHostAlloc(reinterpret_cast<void **>(&reads_offs), (n_reads + 1) * sizeof(T_CSR_cap), cudaHostAllocDefault) ||
        cudaHostAlloc(reinterpret_cast<void **>(&reads_CSR), size_capacity + 1, cudaHostAllocDefault)) {
        std::fprintf(stderr, "B200 counter: pinned allocation of %llu bytes failed\n", (unsigned long long)size_capacity);
        std::exit(1);
    }
    T_CSR_cap o = 0;
    reads_offs[0] = 0;
    for (T_read_cnt i = 0; i < n_reads; i++) {
        std::memcpy(reads_CSR + o, reads[i].read, reads[i].len);
        o += reads[i].len;
        reads_offs[i + 1] = o;
    }
}

PinnedCSR::~PinnedCSR() {
    cudaFreeHost(reads_offs);
    cudaFreeHost(reads_CSR);
}

size_t GPUReset(int did) {
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(did);
    cudaMemGetInfo(&free_b, &total_b);
    return free_b;
}

void GenSuperkmerGPU(PinnedCSR &reads, const T_kvalue K, const T_kvalue P, bool /*HPC*/, CUDAParams &gpars,
                     CountTask /*task*/, const int SKM_partitions, std::vector<SKMStoreNoncon *> stores, int /*tid*/) {
    static_assert(sizeof(T_CSR_cap) == sizeof(uint64_t), "CSR offsets are 64-bit");
    const int did = 0;                                        // one GPU: see "Limits" below
    Device &d = g_dev[did];
    std::lock_guard<std::mutex> lock(d.mu);
    gkc_ctx *ctx = context(did, K, P, SKM_partitions);
    check(gkc_add_reads(ctx, reads.get_reads_CSR(), reinterpret_cast<const uint64_t *>(reads.get_reads_offs()),
                        reads.get_n_reads(), GKC_MEM_HOST), ctx);
    std::vector<uint64_t> pb(SKM_partitions), ps(SKM_partitions), pk(SKM_partitions);
    check(gkc_store_stats(ctx, pb.data(), ps.data(), pk.data()), ctx);
    for (int i = 0; i < SKM_partitions; i++) {               // the superkmers stay in device memory;
        stores[i]->tot_size_bytes += pb[i] - d.pb[i];        // the stores carry the reference's counters
        stores[i]->skm_cnt += ps[i] - d.ps[i];
        stores[i]->kmer_cnt += pk[i] - d.pk[i];
    }
    d.pb.swap(pb); d.ps.swap(ps); d.pk.swap(pk);
}

size_t kmc_counting_GPU_streams(T_kvalue k, std::vector<SKMStoreNoncon *> stores, CUDAParams &gpars,
                                T_kmer_cnt min_freq, T_kmer_cnt max_freq, std::vector<T_kmc> out[], int gpuid,
                                int tid) {
    Device &d = g_dev[0];
    std::lock_guard<std::mutex> lock(d.mu);
    std::vector<int32_t> parts;
    for (auto *s : stores) parts.push_back(s->id);
    uint64_t n_out = 0, n_distinct = 0;
    check(gkc_count_partitions(d.ctx, parts.data(), parts.size(), min_freq, max_freq, &n_out, &n_distinct), d.ctx);
    // The reference leaves out[] empty (gpu_kmercounting.cu:505-508).  To keep the
    // counted k-mers, copy them out with gkc_result:
    //   std::vector<T_kmer> km(n_out); std::vector<uint32_t> ct(n_out);
    //   gkc_result(d.ctx, reinterpret_cast<uint64_t *>(km.data()), ct.data(), n_out, GKC_MEM_HOST);
    // (T_kmer is u64, or unsigned __int128 in the LONGERKMER build: for k > 32
    // gkc_result writes two words per k-mer, low first, which is that layout.)
    for (auto *s : stores) delete s;                          // ownership as in gpu_kmercounting.cu:532-535
    return n_distinct;
}
