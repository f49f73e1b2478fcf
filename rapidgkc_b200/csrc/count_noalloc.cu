// count_noalloc.cu -- gkc_count_keys_noalloc: the raw-key hash count of
// gkc_count_keys without a context and without allocating.  Its scratch (the
// open-addressing table of count_hash.cu and four counters) is fixed device
// memory declared here; each call starts from a clear of that memory.
// Included by engine.cu after count_hash.cu.
#include <cuda.h>

#include <mutex>

namespace gkc {

constexpr uint64_t NA_SLOTS = 1ull << 20;  // 16 MiB of 16-byte slots; keys <= NA_SLOTS / 2
static __device__ __align__(256) HSlot na_table[NA_SLOTS];
// [0] output cursor, [1] distinct keys, [2] output errors, [3] insert errors
static __device__ __align__(256) unsigned long long na_scal[4];

}  // namespace gkc

namespace {

// The scratch's device addresses in one context of one device.  A context
// reset (cudaDeviceReset, which the reference's GPUReset calls) ends the
// context whose addresses were looked up; the next call on that device sees
// a new context id and looks them up again.
struct NaDevice {
    bool ready = false;
    unsigned long long ctx_id = 0;
    HSlot *table = nullptr;
    unsigned long long *scal = nullptr;
    int sms = 0;
};
constexpr int NA_MAX_DEVICES = 64;
NaDevice na_dev[NA_MAX_DEVICES];
std::mutex na_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context (0 when it cannot be
// read: then the addresses are looked up on every call).
unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
            get_id = reinterpret_cast<CtxGetIdFn>(g);
        }
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Addresses of the scratch on device `dev` (current), looked up once per
// context of the device.
int na_setup(int dev, NaDevice **out) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) return GKC_EINVAL;
    std::lock_guard<std::mutex> lock(na_mu);
    NaDevice &d = na_dev[dev];
    const unsigned long long id = current_ctx_id();
    if (!d.ready || !id || id != d.ctx_id) {
        d.ready = false;
        void *t = nullptr, *s = nullptr;
        if (cudaGetSymbolAddress(&t, na_table) != cudaSuccess) return GKC_ECUDA;
        if (cudaGetSymbolAddress(&s, na_scal) != cudaSuccess) return GKC_ECUDA;
        if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GKC_ECUDA;
        d.table = static_cast<HSlot *>(t);
        d.scal = static_cast<unsigned long long *>(s);
        d.ctx_id = current_ctx_id();  // the lookup made the context current if none was
        d.ready = d.ctx_id != 0;
    }
    *out = &d;
    return GKC_OK;
}

// Launches a kernel and returns its own launch status: cudaLaunchKernel
// reports the launch's error directly, and only that error is taken off the
// thread's error state (an earlier caller's pending error is left as it was).
template <class... Args>
cudaError_t na_launch(void (*kernel)(Args...), uint32_t grid, uint32_t block, cudaStream_t s, Args... args) {
    void *argv[] = {static_cast<void *>(&args)...};
    const cudaError_t e = cudaLaunchKernel(reinterpret_cast<const void *>(kernel), dim3(grid), dim3(block), argv, 0, s);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

}  // namespace

extern "C" int gkc_count_keys_noalloc(const uint64_t *keys, uint64_t n, uint32_t cmin, uint32_t cmax,
                                      uint64_t *out_kmers, uint32_t *out_counts, uint64_t out_cap, uint64_t *n_out,
                                      uint64_t *n_distinct, void *stream) {
    if (n > GKC_NOALLOC_MAX_KEYS) return GKC_ELIMIT;
    if ((!keys && n) || ((!out_kmers || !out_counts) && out_cap) || cmin > cmax) return GKC_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GKC_ECUDA;
    NaDevice *d = nullptr;
    const int rc = na_setup(dev, &d);
    if (rc != GKC_OK) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // what must start empty: every slot (key = all ones, count 0) and the counters
    const uint32_t gi = (uint32_t)std::min<uint64_t>((NA_SLOTS + 255) / 256, (uint64_t)d->sms * 8);
    if (na_launch(hash_init_kernel, gi, 256, s, d->table, (uint64_t)NA_SLOTS) != cudaSuccess) return GKC_ECUDA;
    if (cudaMemsetAsync(d->scal, 0, 4 * sizeof(unsigned long long), s) != cudaSuccess) return GKC_ECUDA;
    if (n) {
        const uint32_t g = (uint32_t)std::min<uint64_t>((n + H_THREADS - 1) / H_THREADS, (uint64_t)d->sms * 8);
        if (na_launch(hash_insert_keys_kernel, g, H_THREADS, s, keys, n, d->table, (uint64_t)(NA_SLOTS - 1),
                      reinterpret_cast<uint32_t *>(d->scal + 3)) != cudaSuccess)
            return GKC_ECUDA;
    }
    HCollectParams q;
    q.tab = d->table;
    q.cap = NA_SLOTS;
    q.cmin = cmin;
    q.cmax = cmax;
    q.out_k = out_kmers;
    q.out_c = out_counts;
    q.out_cursor = d->scal;
    q.out_cap = out_cap;
    q.distinct = d->scal + 1;
    q.err = reinterpret_cast<uint32_t *>(d->scal + 2);
    q.part_err = reinterpret_cast<const uint32_t *>(d->scal + 3);
    const uint32_t gc = (uint32_t)std::min<uint64_t>((NA_SLOTS + H_THREADS * HC_ITEMS - 1) / (H_THREADS * HC_ITEMS),
                                                     (uint64_t)d->sms * 8);
    if (na_launch(hash_collect_kernel, gc, H_THREADS, s, q) != cudaSuccess) return GKC_ECUDA;
    unsigned long long h[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(h, d->scal, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return GKC_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return GKC_ECUDA;
    if ((uint32_t)h[3] & ERR_DECODE) return GKC_EINVAL;  // a key was 2^64 - 1
    // More than H_MAX_PROBE keys whose hashes fall on one run of slots: a key
    // set can be built to do this (the hash is invertible); the table is
    // fixed, so the call fails and writes no output.
    if ((uint32_t)h[3] & ERR_TABLE_FULL) return GKC_ELIMIT;
    if (n_out) *n_out = h[0];
    if (n_distinct) *n_distinct = h[1];
    if ((uint32_t)h[2] & ERR_OUTPUT_FULL) return GKC_ELIMIT;  // *n_out holds the size needed
    return GKC_OK;
}
