// hpc.cu -- homopolymer compression of reads (opt.hpc).
//
// The reference's -hpc (GPU_HPCEncoding, gpu_skmgen.cu:145-173) collapses
// each run of equal bytes in a read to one byte before minimizers and
// superkmers are computed: a byte is kept when it starts its read or differs
// from the byte before it.  Here that is a compaction of the whole batch:
// hpc_count_kernel counts the kept bytes of each 16 KiB tile, a device scan
// orders the tiles, and hpc_write_kernel writes the kept bytes (staged in
// shared memory, stored coalesced) and each read's new offset.
#include "gkc_device.cuh"

namespace gkc {

constexpr int HPC_THREADS = 256, HPC_PER = 64, HPC_TILE = HPC_THREADS * HPC_PER;

struct HpcParams {
    const uint8_t *reads;   // batch bytes; read r is [offs[r] - base, offs[r + 1] - base)
    const uint64_t *offs;   // n_reads + 1 entries
    uint64_t n_reads, base, n;
    uint32_t *tile_kept;    // [ntiles] kept bytes of each tile (count pass)
    const uint64_t *tile_base;  // [ntiles] kept bytes before each tile (write pass)
    uint8_t *out;
    uint64_t *out_offs;     // offsets of the reads that start inside the batch's bytes
};

// first read r with offs[r] - base >= pos (n_reads when none)
__device__ __forceinline__ uint64_t hpc_next_read(const HpcParams &a, uint64_t pos) {
    uint64_t lo = 0, hi = a.n_reads;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a.offs[mid] - a.base >= pos) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// Walks bytes [pos, pos + len): calls f(q, r, false) for every read r that
// starts at q (empty reads included, in order), then f(q, -1, true) if byte q
// is kept.  Returns the kept bytes.
template <class F>
__device__ __forceinline__ uint32_t hpc_walk(const HpcParams &a, uint64_t pos, int len, F f) {
    uint64_t r = hpc_next_read(a, pos);
    uint64_t rs = r < a.n_reads ? a.offs[r] - a.base : ~0ull;
    uint8_t prev = pos ? a.reads[pos - 1] : 0;
    uint32_t kept = 0;
    for (int i = 0; i < len; i++) {
        const uint64_t q = pos + i;
        const uint8_t c = a.reads[q];
        bool start = false;
        while (rs == q) {
            f(q, (int64_t)r, false);
            start = true;
            ++r;
            rs = r < a.n_reads ? a.offs[r] - a.base : ~0ull;
        }
        if (start || c != prev) {
            f(q, (int64_t)-1, true);
            kept++;
        }
        prev = c;
    }
    return kept;
}

__global__ void __launch_bounds__(HPC_THREADS) hpc_count_kernel(HpcParams a) {
    __shared__ uint32_t ws[HPC_THREADS / 32];
    const uint64_t pos = blockIdx.x * (uint64_t)HPC_TILE + (uint64_t)threadIdx.x * HPC_PER;
    const int len = pos < a.n ? (int)(a.n - pos < (uint64_t)HPC_PER ? a.n - pos : HPC_PER) : 0;
    const uint32_t k = hpc_walk(a, pos, len, [](uint64_t, int64_t, bool) {});
    uint32_t tot;
    block_exclusive_scan<HPC_THREADS>(k, &tot, ws);
    if (threadIdx.x == 0) a.tile_kept[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(HPC_THREADS) hpc_write_kernel(HpcParams a) {
    __shared__ uint32_t ws[HPC_THREADS / 32];
    __shared__ uint8_t stage[HPC_TILE];
    const uint64_t pos = blockIdx.x * (uint64_t)HPC_TILE + (uint64_t)threadIdx.x * HPC_PER;
    const int len = pos < a.n ? (int)(a.n - pos < (uint64_t)HPC_PER ? a.n - pos : HPC_PER) : 0;
    const uint32_t mine = hpc_walk(a, pos, len, [](uint64_t, int64_t, bool) {});
    uint32_t tot;
    uint32_t k = block_exclusive_scan<HPC_THREADS>(mine, &tot, ws);
    const uint64_t tb = a.tile_base[blockIdx.x];
    hpc_walk(a, pos, len, [&](uint64_t q, int64_t r, bool kept) {
        if (kept) stage[k++] = a.reads[q];
        else a.out_offs[r] = tb + k;  // the read's first kept byte lands at tb + k
    });
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < tot; i += HPC_THREADS) a.out[tb + i] = stage[i];
}

// Offsets of the reads that start at the batch's end (empty reads at the end,
// and the final offset n_reads): the compressed total.
__global__ void hpc_tail_offsets_kernel(const uint64_t *offs, uint64_t n_reads, uint64_t base, uint64_t n,
                                        const unsigned long long *total, uint64_t *out_offs) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r <= n_reads;
         r += (uint64_t)gridDim.x * blockDim.x)
        if (r == n_reads || offs[r] - base >= n) out_offs[r] = *total;
}

}  // namespace gkc
