// gkc_b200_shim.cpp -- RapidGKC's GPU entry points on the B200 counter.
//
// Replaces gpu_skmgen.cu and gpu_kmercounting.cu in RapidGKC's build, keeping
// their signatures (gpu_skmgen.h:52-58, gpu_kmercounting.h:14-17).
//
// Devices.  The reference runs with -ngpu N devices: phase 1 takes the next
// device round-robin for every batch (gpars.device_id.fetch_add(1) % n_devices,
// gpu_skmgen.cu:515-516) and phase 2 counts a group of partitions on the
// device its worker thread names (gpuid, gkc_main.cpp:112-113).  Here each of
// the N devices has one counting context whose store holds the superkmers of
// the batches it took.  A partition's superkmers are therefore spread over
// the N stores: before a phase-2 call counts its partitions on device gpuid,
// every other device packs those partitions (gkc_store_pack) and they are
// appended to gpuid's store (gkc_store_append), so each partition is counted
// once, on one device, from all of its superkmers.  When -ngpu names more
// devices than the machine has, device d runs on GPU d % (GPUs present), each
// with its own context.
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
constexpr int MAX_DEVICES = 64;

struct Device {
    std::mutex mu;                      // a context is used by one thread at a time
    gkc_ctx *ctx = nullptr;
    std::vector<uint64_t> pb, ps, pk;   // store totals already added to the SKMStoreNoncon counters
};
Device g_dev[MAX_DEVICES];
std::mutex g_setup;
int g_k = 0, g_p = 0, g_parts = 0;      // the run's k, minimizer length and partitions (first phase-1 call)

void check(int rc, gkc_ctx *ctx) {      // the reference exits on CUDA errors (CUDA_CHECK)
    if (rc != GKC_OK) {
        std::fprintf(stderr, "B200 counter: %s (%s)\n", gkc_strerror(rc), ctx ? gkc_last_error(ctx) : "");
        std::exit(1);
    }
}

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "B200 counter: %s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

// The GPU that device d (0 <= d < -ngpu) runs on.
int physical(int d) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) n = 1;
    return d % n;
}

int logical_devices(const CUDAParams &gpars) {
    const int n = gpars.n_devices > 0 ? gpars.n_devices : 1;
    return n < MAX_DEVICES ? n : MAX_DEVICES;
}

// Device d's context (made on first use; the caller holds g_dev[d].mu).
gkc_ctx *context(int d) {
    Device &dv = g_dev[d];
    if (!dv.ctx) {
        gkc_options o;
        gkc_default_options(&o);
        {
            std::lock_guard<std::mutex> lock(g_setup);
            o.k = g_k;
            o.p = g_p;
            o.partitions = g_parts;
        }
        o.counter = GKC_COUNTER_HASH;   // GKC_COUNTER_SORT for the reference's sort semantics (sorted output)
        check(gkc_create(physical(d), &o, &dv.ctx), nullptr);
        dv.pb.assign(o.partitions, 0); dv.ps.assign(o.partitions, 0); dv.pk.assign(o.partitions, 0);
    }
    return dv.ctx;
}

// Moves partitions [p0, p1) of device src's store to device dst's store.
void pull(int src, int dst, int p0, int p1) {
    const int n = p1 - p0;
    std::vector<uint64_t> counts(3 * (size_t)n);
    uint8_t *h_bytes = nullptr;
    uint64_t *h_idx = nullptr;
    uint32_t *h_keys = nullptr;
    uint64_t nb = 0, ns = 0;
    {
        Device &s = g_dev[src];
        std::lock_guard<std::mutex> lock(s.mu);
        if (!s.ctx) return;
        check(gkc_store_pack(s.ctx, p0, p1, nullptr, 0, nullptr, nullptr, 0, counts.data()), s.ctx);
        for (int j = 0; j < n; j++) nb += counts[j], ns += counts[n + j];
        if (!ns) return;
        uint8_t *d_bytes = nullptr;
        uint64_t *d_idx = nullptr;
        uint32_t *d_keys = nullptr;
        check_cuda(cudaSetDevice(physical(src)), "cudaSetDevice");
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&d_bytes), nb + 16), "cudaMalloc");
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&d_idx), ns * 8), "cudaMalloc");
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&d_keys), ns * 4), "cudaMalloc");
        check(gkc_store_pack(s.ctx, p0, p1, d_bytes, nb + 16, d_idx, d_keys, ns, counts.data()), s.ctx);
        check_cuda(cudaMallocHost(reinterpret_cast<void **>(&h_bytes), nb + 16), "cudaMallocHost");
        check_cuda(cudaMallocHost(reinterpret_cast<void **>(&h_idx), ns * 8), "cudaMallocHost");
        check_cuda(cudaMallocHost(reinterpret_cast<void **>(&h_keys), ns * 4), "cudaMallocHost");
        check_cuda(cudaMemcpy(h_bytes, d_bytes, nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
        check_cuda(cudaMemcpy(h_idx, d_idx, ns * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
        check_cuda(cudaMemcpy(h_keys, d_keys, ns * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
        cudaFree(d_bytes);
        cudaFree(d_idx);
        cudaFree(d_keys);
    }
    {
        Device &t = g_dev[dst];
        std::lock_guard<std::mutex> lock(t.mu);
        check(gkc_store_append(context(dst), p0, p1, h_bytes, h_idx, h_keys, counts.data()), t.ctx);
    }
    cudaFreeHost(h_bytes);
    cudaFreeHost(h_idx);
    cudaFreeHost(h_keys);
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

// The reference resets device did and returns its free memory
// (gpu_skmgen.cu:487-497); the device is not reset here, so other users of
// the GPU are unaffected.
size_t GPUReset(int did) {
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(physical(did));
    cudaMemGetInfo(&free_b, &total_b);
    return free_b;
}

void GenSuperkmerGPU(PinnedCSR &reads, const T_kvalue K, const T_kvalue P, bool /*HPC*/, CUDAParams &gpars,
                     CountTask /*task*/, const int SKM_partitions, std::vector<SKMStoreNoncon *> stores, int /*tid*/) {
    static_assert(sizeof(T_CSR_cap) == sizeof(uint64_t), "CSR offsets are 64-bit");
    {
        std::lock_guard<std::mutex> lock(g_setup);
        if (!g_parts) g_k = K, g_p = P, g_parts = SKM_partitions;
    }
    const int did = gpars.device_id.fetch_add(1) % logical_devices(gpars);  // gpu_skmgen.cu:515-516
    Device &d = g_dev[did];
    std::lock_guard<std::mutex> lock(d.mu);
    gkc_ctx *ctx = context(did);
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
    const int nd = logical_devices(gpars);
    const int dst = (gpuid % nd + nd) % nd;
    std::vector<int32_t> parts;
    for (auto *s : stores) parts.push_back(s->id);
    // bring the partitions' superkmers from the other devices, run by run of
    // consecutive partition ids
    for (size_t a = 0; a < parts.size();) {
        size_t b = a + 1;
        while (b < parts.size() && parts[b] == parts[b - 1] + 1) b++;
        for (int src = 0; src < nd; src++)
            if (src != dst) pull(src, dst, parts[a], parts[a] + (int)(b - a));
        a = b;
    }
    Device &d = g_dev[dst];
    std::lock_guard<std::mutex> lock(d.mu);
    gkc_ctx *ctx = context(dst);
    uint64_t n_out = 0, n_distinct = 0;
    check(gkc_count_partitions(ctx, parts.data(), parts.size(), min_freq, max_freq, &n_out, &n_distinct), ctx);
    // The reference leaves out[] empty (gpu_kmercounting.cu:505-508).  To keep the
    // counted k-mers, copy them out with gkc_result:
    //   std::vector<T_kmer> km(n_out); std::vector<uint32_t> ct(n_out);
    //   gkc_result(ctx, reinterpret_cast<uint64_t *>(km.data()), ct.data(), n_out, GKC_MEM_HOST);
    // (T_kmer is u64, or unsigned __int128 in the LONGERKMER build: for k > 32
    // gkc_result writes two words per k-mer, low first, which is that layout.)
    for (auto *s : stores) delete s;                          // ownership as in gpu_kmercounting.cu:532-535
    return n_distinct;
}
