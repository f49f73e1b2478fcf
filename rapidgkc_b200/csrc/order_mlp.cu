// order_mlp.cu -- the learned minimizer order: a small network scores every
// p-mer, and the scores are baked into the 4^p rank table that
// find_superkmers_kernel reads in place of the default value order.
//
// Network (FP32): one-hot p-mer (4p inputs) -> 64 ReLU -> 64 ReLU -> 1.  The
// parameter vector holds W1 [4p][64], b1, W2 [64][64] (row = input unit), b2,
// w3, b3.  Training minimises sum_s wt_s (y_s - t_s)^2 * norm, where the
// target t of a p-mer is log2(1 + its k-mer load as a minimizer) measured by
// the counter itself (minimizer_loads_kernel), so that heavy p-mers score high
// and are ranked last.
//
// Kernels:
//   mlp_tile_kernel      forward (and, when training, backward) of a tile of
//                        MLP_TILE samples per CTA: layer 1 is a row gather (the
//                        input is one-hot), layers 2-3 and all gradients are
//                        shared-memory FP32 products; each CTA adds its
//                        gradient to the global one with one atomic per
//                        parameter;
//   mlp_adam_kernel      one Adam step per parameter;
//   order_mix_kernel, order_levels_kernel
//                        the rank table of the learned order: the p-mers of
//                        highest score ranked last, by score, all others in a
//                        fixed pseudo-random order;
//   canonical_table_kernel  min over a p-mer and its reverse complement of the
//                        rank: the table phase 1 reads (one read per position);
//   minimizer_loads_kernel  k-mer instances per minimizer key of the store.
#include "gkc_device.cuh"

namespace gkc {

constexpr int MH = 64;           // hidden units
constexpr int MLP_TILE = 128;    // samples per CTA
constexpr int MLP_THREADS = 256;
constexpr int MLP_MAX_P = 16;
constexpr int ORDER_MAX_P = 15;  // rank levels need 32 - 2p >= 2 bits
constexpr int HS = MH + 1;       // padded row stride of activations and W2 in shared memory

struct MlpLayout {
    int p, in;                          // in = 4p inputs
    uint32_t oW1, ob1, oW2, ob2, ow3, ob3, n;
};

__host__ __device__ inline MlpLayout mlp_layout(int p) {
    MlpLayout l;
    l.p = p;
    l.in = 4 * p;
    l.oW1 = 0;
    l.ob1 = l.oW1 + (uint32_t)l.in * MH;
    l.oW2 = l.ob1 + MH;
    l.ob2 = l.oW2 + MH * MH;
    l.ow3 = l.ob2 + MH;
    l.ob3 = l.ow3 + MH;
    l.n = l.ob3 + 1;
    return l;
}

// shared memory of mlp_tile_kernel, in floats
__host__ __device__ inline size_t mlp_smem_floats(int p) {
    return (size_t)4 * p * MH + MH * HS + 3 * MH + 2 * (size_t)MLP_TILE * HS + 2 * MLP_TILE + 8;
}

struct MlpParams {
    const float *params;
    MlpLayout L;
    const uint32_t *pmers;     // samples: explicit p-mers, or null for p-mers s0 .. s0+n-1
    uint64_t s0, n;
    const float *targets;      // [4^p] by p-mer (training only)
    const float *weights;      // [4^p] by p-mer, or null for 1
    float norm;                // loss scale: 1 / (sum of the batch's weights)
    float *grad;               // [L.n], accumulated (null: forward only)
    float *loss;               // accumulated
    float *scores;             // [samples] forward outputs, or null
};

__global__ void __launch_bounds__(MLP_THREADS)
mlp_tile_kernel(MlpParams a) {
    extern __shared__ float msm[];
    const MlpLayout &L = a.L;
    const int p = L.p;
    float *W1 = msm;                           // [4p][64]
    float *W2 = W1 + 4 * p * MH;               // [64][HS]
    float *b1 = W2 + MH * HS;
    float *b2 = b1 + MH;
    float *w3 = b2 + MH;
    float *H1 = w3 + MH;                       // [TILE][HS]: h1, then dL/da1
    float *H2 = H1 + MLP_TILE * HS;            // [TILE][HS]: h2, then dL/da2
    float *dy = H2 + MLP_TILE * HS;            // [TILE]
    uint32_t *pm = reinterpret_cast<uint32_t *>(dy + MLP_TILE);  // [TILE]
    float *red = reinterpret_cast<float *>(pm + MLP_TILE);       // [8]
    const int tid = threadIdx.x;
    const uint64_t t0 = blockIdx.x * (uint64_t)MLP_TILE;
    const int nt = a.n - t0 < (uint64_t)MLP_TILE ? (int)(a.n - t0) : MLP_TILE;
    for (int i = tid; i < 4 * p * MH; i += MLP_THREADS) W1[i] = a.params[L.oW1 + i];
    for (int i = tid; i < MH * MH; i += MLP_THREADS) W2[(i >> 6) * HS + (i & 63)] = a.params[L.oW2 + i];
    if (tid < MH) {
        b1[tid] = a.params[L.ob1 + tid];
        b2[tid] = a.params[L.ob2 + tid];
        w3[tid] = a.params[L.ow3 + tid];
    }
    if (tid < MLP_TILE) pm[tid] = tid < nt ? (a.pmers ? a.pmers[t0 + tid] : (uint32_t)(a.s0 + t0 + tid)) : 0u;
    if (tid < 8) red[tid] = 0.f;
    __syncthreads();
    const float b3 = a.params[L.ob3];
    const int j = tid & 63, sg = tid >> 6;   // unit, sample group (4 groups of 32)
    // ---- layer 1: h1[s][j] = relu(b1 + sum_pos W1[4 pos + base][j])
    for (int s = sg; s < MLP_TILE; s += 4) {
        const uint32_t v = pm[s];
        float acc = b1[j];
        for (int pos = 0; pos < p; pos++) acc += W1[(4 * pos + ((v >> (2 * (p - 1 - pos))) & 3)) * MH + j];
        H1[s * HS + j] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    // ---- layer 2
    for (int s = sg; s < MLP_TILE; s += 4) {
        float acc = b2[j];
#pragma unroll 16
        for (int i = 0; i < MH; i++) acc = fmaf(H1[s * HS + i], W2[i * HS + j], acc);
        H2[s * HS + j] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    // ---- output, loss and dL/dy
    if (tid < MLP_TILE) {
        const int s = tid;
        float y = b3;
#pragma unroll 16
        for (int i = 0; i < MH; i++) y = fmaf(H2[s * HS + i], w3[i], y);
        float d = 0.f, l = 0.f;
        if (s < nt) {
            if (a.scores) a.scores[t0 + s] = y;
            if (a.grad) {
                const uint32_t v = pm[s];
                const float w = a.weights ? a.weights[v] : 1.f;
                const float e = y - a.targets[v];
                d = 2.f * w * e * a.norm;
                l = w * e * e * a.norm;
            }
        }
        dy[s] = d;
#pragma unroll
        for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(FULL, l, o);
        if ((tid & 31) == 0) atomicAdd(&red[0], l);
    }
    if (!a.grad) return;  // uniform: forward-only launches take no barrier below
    __syncthreads();
    if (tid == 0) atomicAdd(a.loss, red[0]);
    // ---- dw3[j] = sum_s dy[s] h2[s][j], db3 = sum_s dy[s]
    {
        float acc = 0.f;
        for (int s = sg; s < MLP_TILE; s += 4) acc = fmaf(dy[s], H2[s * HS + j], acc);
        atomicAdd(&a.grad[L.ow3 + j], acc);
        if (tid == 0) {
            float d3 = 0.f;
            for (int s = 0; s < MLP_TILE; s++) d3 += dy[s];
            atomicAdd(&a.grad[L.ob3], d3);
        }
    }
    __syncthreads();
    // ---- dL/da2[s][j] = dy[s] w3[j] [h2 > 0]   (in place over h2)
    for (int s = sg; s < MLP_TILE; s += 4) {
        const float h = H2[s * HS + j];
        H2[s * HS + j] = h > 0.f ? dy[s] * w3[j] : 0.f;
    }
    __syncthreads();
    // ---- dW2[i][j] = sum_s h1[s][i] da2[s][j]; db2[j] = sum_s da2[s][j]
    {
        float acc[16];
#pragma unroll
        for (int k = 0; k < 16; k++) acc[k] = 0.f;
        float accb = 0.f;
        for (int s = 0; s < MLP_TILE; s++) {
            const float g = H2[s * HS + j];
            accb += g;
#pragma unroll
            for (int k = 0; k < 16; k++) acc[k] = fmaf(H1[s * HS + sg + 4 * k], g, acc[k]);
        }
#pragma unroll
        for (int k = 0; k < 16; k++) atomicAdd(&a.grad[L.oW2 + (sg + 4 * k) * MH + j], acc[k]);
        if (sg == 0) atomicAdd(&a.grad[L.ob2 + j], accb);
    }
    __syncthreads();
    // ---- dL/da1[s][i] = (sum_j da2[s][j] W2[i][j]) [h1 > 0]   (in place over h1)
    {
        const int i = j;
        for (int s = sg; s < MLP_TILE; s += 4) {
            float acc = 0.f;
#pragma unroll 16
            for (int jj = 0; jj < MH; jj++) acc = fmaf(H2[s * HS + jj], W2[i * HS + jj], acc);
            const float h = H1[s * HS + i];
            H1[s * HS + i] = h > 0.f ? acc : 0.f;
        }
    }
    __syncthreads();
    // ---- dW1[4 pos + b][i] = sum_{s: base(s, pos) = b} da1[s][i]; db1[i] = sum_s da1[s][i]
    {
        const int i = j;
        for (int pos = sg; pos < p; pos += 4) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            const int sh = 2 * (p - 1 - pos);
            for (int s = 0; s < MLP_TILE; s++) {
                const float g = H1[s * HS + i];
                const uint32_t b = (pm[s] >> sh) & 3;
                acc[0] += b == 0 ? g : 0.f;
                acc[1] += b == 1 ? g : 0.f;
                acc[2] += b == 2 ? g : 0.f;
                acc[3] += b == 3 ? g : 0.f;
            }
#pragma unroll
            for (int b = 0; b < 4; b++) atomicAdd(&a.grad[L.oW1 + (4 * pos + b) * MH + i], acc[b]);
        }
        if (sg == 0) {
            float accb = 0.f;
            for (int s = 0; s < MLP_TILE; s++) accb += H1[s * HS + i];
            atomicAdd(&a.grad[L.ob1 + i], accb);
        }
    }
}

struct AdamParams {
    float *params, *m, *v, *grad;
    uint32_t n;
    float lr, beta1, beta2, eps;
    float c1, c2;  // 1 / (1 - beta^t) bias corrections
};

__global__ void mlp_adam_kernel(AdamParams a) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const float g = a.grad[i];
        const float m = a.beta1 * a.m[i] + (1.f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        a.params[i] -= a.lr * (m * a.c1) / (sqrtf(v * a.c2) + a.eps);
        a.grad[i] = 0.f;
    }
}

// Sample list of one epoch: a bijective mix of [0, 4^p) keyed by the epoch.
__global__ void epoch_samples_kernel(uint32_t *out, uint32_t n, int bits, uint32_t key) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = mix_bits(i, bits, key);
}

// The learned order's rank table: rank(v) = (level(v) << 2p) | mix(v).  mix
// is a bijection of 2p bits, so ranks are distinct and p-mers of one level
// are ordered pseudo-randomly rather than by value.  Level 0 for all p-mers
// (order_mix_kernel), then the heavy ones get their levels (order_levels_kernel).
__global__ void order_mix_kernel(uint32_t n, int p, uint32_t *lut) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        lut[v] = mix_bits(v, 2 * p, ORDER_MIX_KEY);
}

__global__ void order_levels_kernel(const uint2 *vl, uint32_t K, int p, uint32_t *lut) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < K; i += gridDim.x * blockDim.x)
        lut[vl[i].x] |= vl[i].y << (2 * p);
}

// The table phase 1 reads: the canonical key of a p-mer position,
// min(rank(v), rank(rc(v))), so one read replaces the two strands' reads.
__global__ void canonical_table_kernel(const uint32_t *lut, uint32_t n, int p, uint32_t *ctab) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t a = lut[v], b = lut[rc32(v, p)];
        ctab[v] = a < b ? a : b;
    }
}

// k-mer instances per minimizer key (its low 2p bits) of one store chunk
__global__ void minimizer_loads_kernel(const uint64_t *idx, const uint32_t *keys, uint64_t n, uint32_t kmask2p,
                                       unsigned long long *loads) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(loads + (keys[i] & kmask2p), (unsigned long long)idx_len(idx[i]));
}

}  // namespace gkc
