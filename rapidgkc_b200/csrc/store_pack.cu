// store_pack.cu -- the gather kernel behind gkc_store_pack.
//
// A store holds one chunk per phase-1 batch, each partition-major.  Packing
// a range of partitions lays every partition's slices from all chunks side by
// side (chunk order), so the range is one contiguous block of bytes, index and
// keys: what the multi-GPU exchange sends to the partition's owner.  An index
// entry's byte offset is relative to its partition's first byte in the chunk;
// a slice that lands `delta` bytes into the packed partition gets `delta`
// added, so the packed range needs no further rebasing wherever it goes.
#pragma once

#include "gkc_device.cuh"

// one (partition, chunk) slice
struct PackDesc {
    const uint8_t *sb;   // source bytes of the slice
    const uint64_t *si;  // source index entries
    const uint32_t *sk;  // source keys
    uint64_t db, ds;     // destination byte / superkmer offset
    uint64_t nb, ns;     // bytes, superkmers of the slice
    uint64_t delta;      // added to each index entry's byte offset
};

constexpr int PK_THREADS = 256;

// One CTA per slice.  Bytes move as aligned 4-byte destination words built
// from up to two source words (the slices start at arbitrary byte offsets);
// the ragged ends go byte by byte.
__global__ void __launch_bounds__(PK_THREADS) pack_gather_kernel(const PackDesc *__restrict__ d,
                                                                 uint8_t *__restrict__ ob,
                                                                 uint64_t *__restrict__ oi,
                                                                 uint32_t *__restrict__ ok) {
    const PackDesc q = d[blockIdx.x];
    uint8_t *dst = ob + q.db;
    // head bytes up to the destination's 4-byte boundary
    const uint64_t h4 = (4 - (reinterpret_cast<uintptr_t>(dst) & 3)) & 3;
    const uint64_t head = q.nb < h4 ? q.nb : h4;
    if (threadIdx.x < head) dst[threadIdx.x] = q.sb[threadIdx.x];
    const uint64_t nw = (q.nb - head) >> 2;
    const uint8_t *src = q.sb + head;
    uint32_t *dw = reinterpret_cast<uint32_t *>(dst + head);
    const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 3);
    const uint32_t *sw = reinterpret_cast<const uint32_t *>(src - sh);
    // sw[i + 1] is read only when sh != 0; its first byte is source byte
    // 4 i + 4 - sh < 4 nw <= nb - head, inside the slice, so the aligned
    // word lies in the source buffer
    for (uint64_t i = threadIdx.x; i < nw; i += PK_THREADS) {
        const uint32_t lo = __ldg(sw + i);
        dw[i] = sh ? __funnelshift_r(lo, __ldg(sw + i + 1), 8 * sh) : lo;
    }
    for (uint64_t i = head + nw * 4 + threadIdx.x; i < q.nb; i += PK_THREADS) dst[i] = q.sb[i];
    for (uint64_t i = threadIdx.x; i < q.ns; i += PK_THREADS) {
        oi[q.ds + i] = q.si[i] + q.delta;
        ok[q.ds + i] = q.sk[i];
    }
}
