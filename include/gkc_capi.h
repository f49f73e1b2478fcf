/*
 * gkc_capi.h -- C ABI of the B200 k-mer counter (librapidgkc_b200.so).
 *
 * Plain pointers and sizes only.  Every function returns GKC_OK (0) or a
 * negative GKC_E* code and never exits the process; gkc_last_error() gives
 * the message.  A context is bound to one CUDA device and is not thread-safe:
 * use one context per host thread (the reference runs several host workers
 * per GPU, utilities.hpp:214; each would own a context here).
 *
 * The entry points replace the reference's GPU interface
 * (paths relative to the RapidGKC source tree):
 *   gkc_create       GPUReset                 gpu_skmgen.h:52, gpu_skmgen.cu:487-497
 *   gkc_add_reads    GenSuperkmerGPU          gpu_skmgen.h:54-58, gpu_skmgen.cu:504-718
 *   gkc_store_stats  SKMStoreNoncon counters  skmstore.hpp:85-87
 *   gkc_store_export SKMStoreNoncon bytes     skmstore.hpp:156-187, 222-236
 *   gkc_count        kmc_counting_GPU_streams gpu_kmercounting.h:14-17, gpu_kmercounting.cu:343-548
 *   gkc_count_partitions  the same, on the store subset one call is given
 *   gkc_result       the kmc_result vectors   gkc_main.cpp:294, gpu_kmercounting.cu:505-508
 *   gkc_store_clear  SKMStoreNoncon::clear_skm_data   skmstore.hpp:189-198
 *   gkc_add_skm      SKMStoreNoncon::load_from_file   skmstore.hpp:102-114
 *   gkc_add_fastx, gkc_parse_fastx  ReadLoader's record extraction  fileloader.hpp:201-232, 269-330
 *   gkc_set_order    the fixed minimizer order        minimizer_filter.h:20
 *   gkc_count_keys   the hash counter's insert_batch  gpu_hash_counter.cu:376-419 (its test, :693-708)
 *   gkc_init, gkc_skmgen_batch, gkc_count_partition, gkc_set_order_lut, gkc_shutdown
 *                    the same steps in five calls (end of this file)
 * and add what the reference declares but never does: the count threshold
 * [min, max] (utilities.hpp:190) and an output of the counted k-mers.
 * The other entry points have no counterpart in the reference: context
 * teardown (gkc_destroy), batching and its timings (gkc_add_reads_batches,
 * gkc_batch_timings), device results (gkc_result_device), the one-call
 * count (gkc_count_reads), the pinned spill arena (gkc_reserve_host), the
 * multi-GPU exchange (gkc_store_pack, gkc_store_append), instrumentation
 * (gkc_last_timings, gkc_kernel_launches, gkc_set_profiling,
 * gkc_kernel_stats), streams (gkc_set_stream), the learned order
 * (gkc_minimizer_loads, gkc_mlp_*) and gkc_count_keys_noalloc.
 */
#ifndef GKC_CAPI_H
#define GKC_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    GKC_OK = 0,
    GKC_EINVAL = -1,    /* bad argument */
    GKC_ECUDA = -2,     /* CUDA runtime error */
    GKC_ENOMEM = -3,    /* device or pinned memory exhausted */
    GKC_ESTATE = -4,    /* call out of order (e.g. result before count) */
    GKC_EINTERNAL = -5, /* retries exhausted or inconsistent internal state */
    GKC_ELIMIT = -6     /* input or output larger than a fixed-size limit */
};

enum { GKC_COUNTER_SORT = 0, GKC_COUNTER_HASH = 1 };
enum { GKC_MEM_HOST = 0, GKC_MEM_DEVICE = 1 };
enum { GKC_FASTQ = 0, GKC_FASTA = 1 };

typedef struct gkc_ctx gkc_ctx;

typedef struct gkc_options {
    int k;                  /* k-mer length, p <= k <= 64 (reference -k, utilities.hpp:187); k   */
                            /* > 32 is the reference's 128-bit LONGERKMER build (types.h:34-35,  */
                            /* utilities.hpp:280-281): k-mers take two words; either counter     */
                            /* counts them (hash: 16-byte keys in the sub-bucket tables)         */
    int p;                  /* minimizer length, 3 <= p <= 16 (reference -p, utilities.hpp:188)   */
    int partitions;         /* superkmer partitions, 1..4096 (reference -skm, utilities.hpp:189)  */
    int counter;            /* GKC_COUNTER_SORT or GKC_COUNTER_HASH                               */
    int radix_bits;         /* LSD digit width of the sort counter, 4..11 (0 = 8)                 */
    double table_slots;     /* hash slots per k-mer instance of a partition (0 = 0.35)            */
    uint64_t batch_bases;   /* bases per phase-1 batch, host and device input (0 = 1 GiB)         */
    int spill_host;         /* keep the partition store in pinned host memory (streamed input)    */
    uint64_t group_keys;    /* max k-mer instances per sort group (0 = from free device memory)   */
    int hash_l2_only;       /* hash counter: 0 = shared-memory sub-buckets with the L2 table for  */
                            /* the ones that overflow; 1 = every partition through the L2 table   */
    int hpc;                /* 1: homopolymer compression of every read before phase 1: a run of  */
                            /* equal bytes counts as one base (reference -hpc, gpu_skmgen.cu:145) */
    uint64_t sort_seg_max;  /* sort counter: partitions of more k-mer instances than this take    */
                            /* the three-kernel radix sort, the others the one-pass-per-digit     */
                            /* sort (0 = 2^30 - 1, its limit; lower values are for tests)         */
} gkc_options;

/* Fills defaults: k=31, p=11, partitions=512, hash counter. */
void gkc_default_options(gkc_options *opt);

/* Creates a context on CUDA device `device` (replaces GPUReset; the device
 * is not reset, other users of it are unaffected). */
int gkc_create(int device, const gkc_options *opt, gkc_ctx **out);
int gkc_destroy(gkc_ctx *ctx);
const char *gkc_last_error(const gkc_ctx *ctx);
const char *gkc_strerror(int code);

/* Minimizer order: `lut` holds 4^p ranks (uint32) indexed by the 2-bit p-mer
 * value; the canonical minimizer of a k-mer is the p-mer of least rank over
 * both strands (phase 1 reads a precomputed min(rank(v), rank(rc(v))) table,
 * one read per position).  NULL restores the reference's default order (value
 * order with the "rapidgkc" filter, minimizer_filter.h:20).  `mem` says where
 * lut lives. */
int gkc_set_order(gkc_ctx *ctx, const uint32_t *lut, uint64_t n, int mem);

/* Phase 1: splits a CSR batch of ASCII reads (reads[offs[i]..offs[i+1])) into
 * superkmers and appends them to the context's partition store.  Host input
 * is copied in batches of opt.batch_bases bases, overlapped with compute
 * (pinned host memory gives the overlap).  Device input requires offs[0]==0;
 * it is processed in place, in batches of the same size. 
 * Reads shorter than k contribute nothing. */
int gkc_add_reads(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int mem);

/* Phase 1 over caller-chosen batches of host reads: batch i holds the next
 * batch_reads[i] reads (batches of uneven size; they add up to n_reads).
 * Batch i+1 is copied while batch i is processed; each batch's kernels run as
 * one CUDA graph with no host round trip (a batch whose superkmers outgrow the
 * preallocated store chunk is redone with exact sizes).  gkc_add_reads on host
 * input does the same with batches of opt.batch_bases bases.  No reference
 * counterpart: the reference copies and splits 2000-read batches with a host
 * round trip each (gpu_skmgen.cu:504-718). */
int gkc_add_reads_batches(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads,
                          const uint64_t *batch_reads, uint64_t n_batches);

/* Latency of each batch of the last gkc_add_reads / gkc_add_reads_batches call
 * (milliseconds from the start of its host-to-device copy to the end of its
 * phase 1, CUDA events): ms[i] for i < min(cap, *n); *n = batches. */
int gkc_batch_timings(gkc_ctx *ctx, double *ms, uint64_t cap, uint64_t *n);

/* Phase 1 from FASTQ or FASTA text (host or device memory, n bytes): the
 * records are scanned on the GPU into reads, which gkc_add_reads then takes.
 * Replaces the reference loader's newline search and read extraction
 * (fileloader.hpp:201-232, 269-330).
 *   GKC_FASTQ: 4-line records; line 4i+1 of the text is a read, counting from
 *     *state = the line phase at the text's start (0 at a file's start; NULL
 *     means 0).  *state is set to the phase at its end, so a file can be fed
 *     in pieces cut after any newline, as the reference carries its phase
 *     across buffers.
 *   GKC_FASTA: a record is a '>' header line and the sequence lines up to the
 *     next header, concatenated (the reference's loader takes every second
 *     line instead, which reads multi-line FASTA wrongly).  Text that starts
 *     with sequence lines continues a record cut from the text before; its
 *     bases form a read of their own, so a cut record loses the k-mers that
 *     span the cut unless the caller repeats k-1 bases.  *state is unused.
 * '\n' and '\r' are never part of a read.  *n_reads / *n_bases (may be NULL)
 * = reads and bases found (reads shorter than k add no k-mers). */
int gkc_add_fastx(gkc_ctx *ctx, const char *text, uint64_t n, int mem, int format, int *state, uint64_t *n_reads,
                  uint64_t *n_bases);

/* The scan of gkc_add_fastx alone: the reads as a CSR, copied to `reads`
 * (cap_bases bytes) and `offs` (cap_reads entries, n_reads + 1 used) in host
 * or device memory (out_mem).  With reads and offs NULL only the sizes are
 * returned; buffers too small give GKC_ELIMIT with the sizes set. */
int gkc_parse_fastx(gkc_ctx *ctx, const char *text, uint64_t n, int mem, int format, int *state, char *reads,
                    uint64_t cap_bases, uint64_t *offs, uint64_t cap_reads, int out_mem, uint64_t *n_reads,
                    uint64_t *n_bases);

/* Per-partition totals of the store: superkmer bytes, superkmers, k-mers
 * (SKMStoreNoncon::tot_size_bytes / skm_cnt / kmer_cnt).  Arrays of
 * opt.partitions entries; any may be NULL. */
int gkc_store_stats(gkc_ctx *ctx, uint64_t *part_bytes, uint64_t *part_skms, uint64_t *part_kmers);

/* Copies partition `part`'s superkmer bytes (the reference's .skm format,
 * skmstore.hpp:129-141) to host memory `out` of `cap` bytes; *n = bytes. */
int gkc_store_export(gkc_ctx *ctx, int part, uint8_t *out, uint64_t cap, uint64_t *n);

/* Drops every superkmer in the store. */
int gkc_store_clear(gkc_ctx *ctx);

/* Packs partitions [p0, p1) of the store into one partition-major range:
 * each partition's superkmers from every chunk, in chunk order, into device
 * memory `bytes` (cap_bytes), `idx` (u64) and `keys` (u32) of cap_skms
 * entries.  counts (host, 3 x (p1 - p0)) = per partition bytes, superkmers,
 * k-mers; with all three buffers NULL only counts are written, to size them.
 * Index offsets stay relative to each partition's first byte, so a packed
 * range appends to any context unchanged.  The multi-GPU exchange packs
 * [0, P) and sends each owner its range: a step the reference does not have
 * (its stores never leave one process, skmstore.hpp:62-279). */
int gkc_store_pack(gkc_ctx *ctx, int p0, int p1, uint8_t *bytes, uint64_t cap_bytes, uint64_t *idx,
                   uint32_t *keys, uint64_t cap_skms, uint64_t *counts);

/* Appends a packed range of partitions [p0, p1) (gkc_store_pack's layout, in
 * device or host memory; counts in host memory) to the store as one chunk
 * (SKMStoreNoncon::add_skms, skmstore.hpp:189-198, for a received range).
 * None of [p0, p1) may have been counted yet (gkc_count_partitions); other
 * partitions of the store may have been.  The buffers may be reused when the
 * call returns. */
int gkc_store_append(gkc_ctx *ctx, int p0, int p1, const uint8_t *bytes, const uint64_t *idx,
                     const uint32_t *keys, const uint64_t *counts);

/* Appends superkmers given as the reference's .skm bytes (skmstore.hpp:
 * 129-141: a partition's superkmers in skm_3x format, concatenated; the bytes
 * gkc_store_export gives): partition p's bytes are bytes[part_off[p] ..
 * part_off[p+1]) (part_off: P+1 entries in host memory; bytes in host or
 * device memory, mem).  The superkmer bounds are found on the GPU, and each
 * superkmer's minimizer is recomputed under the context's order from its
 * first k-mer.  GKC_EINVAL, and nothing appended, if a partition ends inside a
 * superkmer, a superkmer holds fewer than k bases, or a minimizer maps to
 * another partition than the one its bytes came in (bytes written with
 * another order, p or partition count).  Lets this counter count a store the
 * reference wrote (its phase 1, .skm files), and the reference count ours. */
int gkc_add_skm(gkc_ctx *ctx, const uint8_t *bytes, const uint64_t *part_off, int mem);

/* Pins host memory for spilled chunks (opt.spill_host) until the context's
 * host arena holds `bytes` in all, used or free; *pinned (may be NULL) = bytes
 * pinned.  A stream of known size reserves ahead; this is the one call that
 * may run on another host thread while gkc_add_reads runs.  The arena never
 * pins past the point where an eighth of physical memory (at least 8 GiB)
 * would no longer be available: that fails with GKC_ENOMEM.
 * Replaces the reference's per-chunk host buffers of SKMStoreNoncon
 * (skmstore.hpp:62-279, add_skms). */
int gkc_reserve_host(gkc_ctx *ctx, uint64_t bytes, uint64_t *pinned);

/* Phase 2: counts every partition of the store and keeps the k-mers whose
 * count c satisfies cmin <= c <= cmax.  *n_out = k-mers kept; *n_distinct =
 * distinct k-mers before the threshold (the reference's return value).  The
 * store is consumed (the reference deletes its stores, gpu_kmercounting.cu:532).
 * Output order: partition by partition; ascending k-mer inside a partition
 * with the sort counter, unordered with the hash counter. */
int gkc_count(gkc_ctx *ctx, uint32_t cmin, uint32_t cmax, uint64_t *n_out, uint64_t *n_distinct);

/* Phase 2 on some partitions: counts partitions parts[0..n) of the store
 * (each at most once per store), as kmc_counting_GPU_streams counts the stores
 * it is given (gpu_kmercounting.h:14-17, called per store subset by
 * gkc_main.cpp:113).  The result replaces the previous one (gkc_result); the
 * store is released once every partition has been counted.  Adding reads to
 * a partly counted store, or counting a partition twice, is GKC_ESTATE. */
int gkc_count_partitions(gkc_ctx *ctx, const int32_t *parts, uint64_t n, uint32_t cmin, uint32_t cmax,
                         uint64_t *n_out, uint64_t *n_distinct);

/* Copies the last gkc_count result: kmers[i] (2-bit, first base in the most
 * significant position, canonical) and counts[i], i < min(cap, n_out).  For
 * k > 32 a k-mer takes two words, kmers[2i] (low) and kmers[2i+1] (high):
 * the memory layout of an unsigned __int128 on a little-endian host, the
 * reference's T_kmer under LONGERKMER (types.h:34-35); cap counts k-mers. */
int gkc_result(gkc_ctx *ctx, uint64_t *kmers, uint32_t *counts, uint64_t cap, int mem);

/* Device pointers to the last result (valid until the next call; two words
 * per k-mer for k > 32, as gkc_result). */
int gkc_result_device(gkc_ctx *ctx, const uint64_t **kmers, const uint32_t **counts, uint64_t *n);

/* One call: gkc_store_clear + gkc_add_reads + gkc_count + gkc_result (cap in
 * k-mers: 2 * cap words for k > 32). */
int gkc_count_reads(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int mem,
                    uint32_t cmin, uint32_t cmax, uint64_t *kmers, uint32_t *counts, uint64_t cap,
                    int out_mem, uint64_t *n_out, uint64_t *n_distinct);

/* Counts raw 64-bit keys (no superkmers, no canonical step) with the
 * configured counter; results as gkc_count, one word per key whatever the
 * context's k.  keys must not be 2^64-1. */
int gkc_count_keys(gkc_ctx *ctx, const uint64_t *keys, uint64_t n, int mem, uint32_t cmin, uint32_t cmax,
                   uint64_t *n_out, uint64_t *n_distinct);

/* Statistics of the last gkc_add_reads (phase 1) and gkc_count (phase 2)
 * calls (n <= 10 entries): times[0..3] = device milliseconds (CUDA events) of
 * phase 1, its superkmer search, phase 2, and phase 2's counting kernels;
 * times[4] = sub-buckets of the hash counter, times[5] = those re-split by
 * k-mer hash (they held more than 65536 k-mer instances, or their distinct
 * k-mers overflowed shared memory twice); hash counter only: times[6] =
 * device milliseconds of staging spilled chunks back, times[7] = partition
 * groups counted, times[8] = sub-buckets that overflowed the first table and
 * were counted by the second pass (16384 slots); times[9] = bytes the last
 * gkc_add_reads copied from host to device (host batches: read bases, half of
 * the batches packed to 2-bit words, and offsets). */
int gkc_last_timings(gkc_ctx *ctx, double *times, int n);

/* Number of kernels this context launched since creation. */
uint64_t gkc_kernel_launches(const gkc_ctx *ctx);

/* Runs the context's work on `stream` (a cudaStream_t of the context's
 * device; NULL restores the context's own stream). */
int gkc_set_stream(gkc_ctx *ctx, void *stream);

/* Kernel classes of gkc_kernel_stats. */
enum {
    GKC_K_FIND_SUPERKMERS = 0,  /* phase 1: minimizers + superkmer records */
    GKC_K_SCATTER = 1,          /* phase 1: records -> partition bytes     */
    GKC_K_HASH_INSERT = 2,      /* phase 2 hash: sub-bucket decode + count */
    GKC_K_HASH_COLLECT = 3,     /* phase 2 hash: threshold + clear table   */
    GKC_K_SORT_EXTRACT = 4,     /* phase 2 sort: decode -> key buffer      */
    GKC_K_RADIX_HIST = 5,       /* phase 2 sort: tile digit histograms     */
    GKC_K_RADIX_SCATTER = 6,    /* phase 2 sort: stable scatter            */
    GKC_K_SCAN = 7,             /* device-wide scans                       */
    GKC_K_RLE = 8,              /* run-length encoding + threshold         */
    GKC_K_BUCKET_SPLIT = 9,     /* phase 2 hash: superkmers -> sub-buckets */
    GKC_K_HASH_RECORDS = 10,    /* phase 2 hash: overflowed sub-buckets    */
                                /* (second pass, 16384 slots) and heavy    */
                                /* ones (k-mer records)                    */
    GKC_K_CLASSES = 11
};

/* With profiling on, every kernel launch is bracketed by CUDA events on the
 * launching stream; gkc_kernel_stats then returns, per class, the summed
 * device milliseconds, the number of launches and the algorithmic DRAM bytes
 * (compulsory reads + writes of the class's inputs and outputs) since the
 * last reset.  Phase 1 keeps its batches; each batch's kernels are launched
 * directly instead of as one CUDA graph, since timing events do not time
 * inside a graph.  Arrays of n <= GKC_K_CLASSES entries; any may be NULL. */
int gkc_set_profiling(gkc_ctx *ctx, int on);
int gkc_kernel_stats(gkc_ctx *ctx, double *ms, uint64_t *launches, double *bytes, int n, int reset);

/* No counterpart in the reference (its host passes ASCII to the device,
 * gpu_skmgen.cu:573-574).  Packs n ASCII bases into 2-bit codes, 16 to a
 * word, base 16w + t in bits 31-2t..30-2t of words[w], with the device's base
 * map (A/C/G/T in either case -> 0..3, every other byte -> 0); positions past
 * n in the last word are 0.  words holds (n + 15) / 16 entries.  Host memory
 * only; runs on the library's pool of host threads.  This is the form in which
 * gkc_add_reads and gkc_count_reads copy host batches to the device (a
 * quarter of the ASCII bytes), except with homopolymer compression on, whose
 * kernels read ASCII. */
int gkc_pack_bases(const char *bases, uint64_t n, uint32_t *words);

/* ---- learned minimizer order ------------------------------------------
 * No counterpart in the reference: its order is fixed (value order with the
 * "rapidgkc" filter, minimizer_filter.h:20, gpu_skmgen.cu:243-252).  A network
 * (one-hot p-mer, 4p inputs -> 64 ReLU -> 64 ReLU -> 1, FP32) scores every
 * p-mer; the order ranks p-mers by score, so p-mers with a high predicted
 * load are chosen as minimizers last.  Parameters: one float vector of
 * gkc_mlp_param_count(p) entries, W1 [4p][64] (input 4*pos + base, pos 0 = the
 * first base), b1 [64], W2 [64][64] (row = input unit), b2 [64], w3 [64], b3.
 * All use the context's p and device; p <= 16. */

/* Number of network parameters for minimizer length p (0 if p is out of range). */
uint64_t gkc_mlp_param_count(int p);

/* k-mer instances of the store per minimizer key: loads[key & (4^p - 1)], n =
 * 4^p.  With the default order the key is the minimizer's value (4^p - 1 also
 * stands for k-mers without a valid p-mer); with an order table it is the
 * minimizer's rank. */
int gkc_minimizer_loads(gkc_ctx *ctx, uint64_t *loads, uint64_t n, int mem);

/* One forward and backward pass over the n samples pmers[] (host memory):
 * loss = norm * sum_s w_s (y_s - t_s)^2 with t_s = targets[pmers[s]] and
 * w_s = weights[pmers[s]] (weights may be NULL: all 1); targets and weights
 * hold 4^p floats.  grad receives d loss / d params. */
int gkc_mlp_grad(gkc_ctx *ctx, const float *params, const uint32_t *pmers, uint64_t n, const float *targets,
                 const float *weights, float norm, float *grad, float *loss);

/* Trains params (host, in place) with Adam (lr, betas 0.9 / 0.999) on all 4^p
 * p-mers for `epochs` passes in shuffled batches of `batch`; *loss (optional)
 * = mean batch loss of the last pass.  Deterministic samples for a seed; the
 * gradient sums use atomics, so results vary in the last bits. */
int gkc_mlp_train(gkc_ctx *ctx, float *params, const float *targets, const float *weights, int epochs, int batch,
                  float lr, uint64_t seed, float *loss);

/* Scores of all 4^p p-mers (scores[v], host or device memory). */
int gkc_mlp_scores(gkc_ctx *ctx, const float *params, float *scores, int mem);

/* Makes the network's order the context's order (p <= 15).  rank(v) =
 * (level << 2p) | mix(v), mix = a fixed bijection of 2p bits: the `heavy`
 * p-mers of highest score (the ones predicted heavy as minimizers; 0 = 4^p / 4)
 * get levels 1 .. 2^(32-2p)-2 by score and are chosen last; every other p-mer
 * has level 0, so their order is pseudo-random instead of by value.  lut_out
 * (optional, host, 4^p entries) receives the rank table (what gkc_set_order
 * would take for the same order). */
int gkc_mlp_order(gkc_ctx *ctx, const float *params, uint64_t heavy, uint32_t *lut_out);

/* ---- counting without allocation ----------------------------------------
 * No counterpart in the reference.  gkc_count_keys_noalloc counts raw 64-bit
 * keys like gkc_count_keys with the hash counter, but needs no context and
 * allocates nothing: its scratch is a fixed table in the library's device
 * memory (16 MiB, GKC_NOALLOC_SLOTS slots), which limits it to n <=
 * GKC_NOALLOC_MAX_KEYS keys; larger n returns GKC_ELIMIT before any work.
 * For callers that must not allocate device memory, e.g. code that already
 * holds its own memory pool or runs where cudaMalloc / cudaFree would
 * synchronise the device mid-pipeline.
 *   keys         device memory, n keys, none equal to 2^64-1 (GKC_EINVAL)
 *   out_kmers / out_counts  device memory of out_cap entries: the keys whose
 *                count c satisfies cmin <= c <= cmax, unordered; if more than
 *                out_cap qualify, returns GKC_ELIMIT with *n_out = the number
 *   stream       a cudaStream_t of the current device (NULL: the default
 *                stream); the call copies its counters back to the host and
 *                waits for the stream before it returns
 * Runs on the current CUDA device.  The first call on a device (and the first
 * after the device's context is reset, e.g. by cudaDeviceReset) looks up the
 * scratch's address (cudaGetSymbolAddress).  All calls on one device share the one scratch
 * table and it keeps the last call's contents (each call clears it first),
 * so two calls in flight at the same time (other host threads, other
 * streams) race and give wrong results: the caller serialises them.
 * GKC_ELIMIT is also returned, with no output, when more than 4096 of the
 * keys hash onto one run of slots: the table is fixed, and the hash is
 * invertible, so a key set can be built to do this. */
enum { GKC_NOALLOC_SLOTS = 1 << 20, GKC_NOALLOC_MAX_KEYS = 1 << 19 };
int gkc_count_keys_noalloc(const uint64_t *keys, uint64_t n, uint32_t cmin, uint32_t cmax, uint64_t *out_kmers,
                           uint32_t *out_counts, uint64_t out_cap, uint64_t *n_out, uint64_t *n_distinct,
                           void *stream);

/* ---- the boundary in five calls ------------------------------------------
 * One call per step of the reference's GPU interface, each a thin form of the
 * calls above; every one returns a GKC_* status (the reference exits on
 * errors instead, CUDA_CHECK in utilities.hpp).
 *
 * gkc_init: device setup, in place of GPUReset (gpu_skmgen.h:52), which
 * resets the device; this one does not.  Same as gkc_create. */
int gkc_init(int device, const gkc_options *config, gkc_ctx **out);

/* gkc_skmgen_batch: one phase-1 batch, in place of GenSuperkmerGPU
 * (gpu_skmgen.h:54-58): the batch's superkmers are appended to the
 * context's partition store (gkc_add_reads), and part_bytes / part_skms /
 * part_kmers (P entries each, may be NULL) receive the store's totals per
 * partition, the counters GenSuperkmerGPU leaves in each SKMStoreNoncon
 * (tot_size_bytes, skm_cnt, kmer_cnt; skmstore.hpp:85-87).  k, p and P must
 * be the context's (GKC_EINVAL otherwise).  order_lut (4^p ranks, host
 * memory) installs a minimizer order as gkc_set_order does; only while the
 * store is empty (GKC_ESTATE otherwise), since one store holds one order. */
int gkc_skmgen_batch(gkc_ctx *ctx, const char *reads, const uint64_t *offs, uint64_t n_reads, int k, int p, int P,
                     const uint32_t *order_lut, int mem, uint64_t *part_bytes, uint64_t *part_skms,
                     uint64_t *part_kmers);

/* gkc_count_partition: phase 2 of one partition, the per-store step of
 * kmc_counting_GPU_streams (gpu_kmercounting.h:14-17): counts partition
 * `part` (gkc_count_partitions with one id), keeps counts in [cmin, cmax],
 * and copies its (k-mer, count) table to kmers / counts (cap entries, in
 * `mem`; two words per k-mer for k > 32) when they are given; a table larger
 * than cap is GKC_EINVAL with *n_out set.  *n_distinct = the partition's
 * distinct k-mers (the reference's return value). */
int gkc_count_partition(gkc_ctx *ctx, int part, uint32_t cmin, uint32_t cmax, uint64_t *kmers, uint32_t *counts,
                        uint64_t cap, int mem, uint64_t *n_out, uint64_t *n_distinct);

/* gkc_set_order_lut: gkc_set_order with a host table of 4^p ranks (NULL: the
 * default order, minimizer_filter.h:20). */
int gkc_set_order_lut(gkc_ctx *ctx, const uint32_t *lut);

/* gkc_shutdown: releases the context (gkc_destroy). */
int gkc_shutdown(gkc_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* GKC_CAPI_H */
