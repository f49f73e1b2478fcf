/*
 * gkc_oracle.c -- CPU restatement of RapidGKC's k-mer counting hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * entry point and bench.py's CPU-baseline leg load it to verify or time the
 * CUDA product path.  It is never linked into, imported by, or called from
 * the product library (rapidgkc_b200/), which has no CPU fallback.
 *
 * Every function restates the reference algorithm in plain C and cites the
 * reference file:line it follows (paths are relative to the RapidGKC tree).
 * Parity of this restatement is pinned twice: against the reference's own
 * golden vector (cpu_funcs.cpp:654-676, `#ifdef TEST` main) and against the
 * reference CPU path itself, compiled from its sources into oracle/_ref/ by
 * oracle/Makefile (see tests/test_oracle.py and tests/golden/).
 *
 * Deliberate, documented differences from the reference (both sides of the
 * comparison use them, and the parity tests only feed inputs where the
 * reference is well defined):
 *   - bytes outside {A,C,G,T,U,N} (either case) are read like 'N'; the
 *     reference maps them to 255 and produces malformed superkmer bytes;
 *   - superkmer byte sizes are kept in 32 bits (the reference's T_skm_len is
 *     16 bits and wraps beyond 65535 bytes, types.h:19).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ASCII -> 2-bit code, forward strand (cpu_funcs.cpp:20-54):
 * A/a=0 C/c=1 G/g=2 T/t=3, N/n=0 and U/u=0. */
static uint8_t fwd_code(uint8_t c) {
    switch (c) {
        case 'A': case 'a': return 0;
        case 'C': case 'c': return 1;
        case 'G': case 'g': return 2;
        case 'T': case 't': return 3;
        default: return 0;  /* N, U and (deviation) anything else */
    }
}
/* Complement code (cpu_funcs.cpp:55-88): A=3 C=2 G=1 T=0, N/n=3 and U/u=3. */
static uint8_t cmp_code(uint8_t c) { return (uint8_t)(3 - fwd_code(c)); }

/* Default minimizer filter "rapidgkc" (minimizer_filter.h:20): a p-mer is
 * invalid if its first three bases are AAA, ACA, CAA or CCA, or its last three
 * bases are AAA. */
int orc_filter_default(uint32_t v, int p) {
    return (((v >> ((p - 3) * 2)) & 0x2Bu) != 0) & ((v & 0x3Fu) != 0);
}

/* Ordering key of one p-mer.  Default order: the value itself, or the
 * sentinel mm_mask = 4^p-1 when filtered (cpu_funcs.cpp:109-123,
 * gpu_skmgen.cu:243-252).  Learned order: a 4^p lookup table of ranks. */
static uint32_t pmer_key(uint32_t v, int p, const uint32_t *lut) {
    uint32_t mask = 0xFFFFFFFFu >> (32 - 2 * p);
    if (lut) return lut[v];
    return orc_filter_default(v, p) ? v : mask;
}

/* Per k-mer canonical minimizer key: min over the k-p+1 p-mers of the k-mer,
 * forward and reverse complement both, compared by key
 * (gpu_skmgen.cu:218-274; cpu_funcs.cpp:124-146).  keys[i] for k-mer i,
 * i in [0, len-k].  Returns the number of k-mers (0 if len < k). */
int64_t orc_kmer_keys(const uint8_t *read, int64_t len, int k, int p,
                      const uint32_t *lut, uint32_t *keys) {
    if (len < k) return 0;
    int64_t npm = len - p + 1, nk = len - k + 1, i, j;
    uint32_t mask = 0xFFFFFFFFu >> (32 - 2 * p);
    uint32_t *pk = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)npm);
    uint32_t f = 0, r = 0;
    for (j = 0; j < len; j++) {
        f = ((f << 2) | fwd_code(read[j])) & mask;
        r = (r >> 2) | ((uint32_t)cmp_code(read[j]) << (2 * p - 2));
        if (j >= p - 1) {
            uint32_t a = pmer_key(f, p, lut), b = pmer_key(r, p, lut);
            pk[j - p + 1] = a < b ? a : b;
        }
    }
    for (i = 0; i < nk; i++) {
        uint32_t m = pk[i];
        for (j = 1; j <= k - p; j++) if (pk[i + j] < m) m = pk[i + j];
        keys[i] = m;
    }
    free(pk);
    return nk;
}

/* Superkmer split of one read (cpu_funcs.cpp:147-198, gpu_skmgen.cu:287-363):
 * a superkmer is a maximal run of consecutive k-mers with the same minimizer
 * key.  offs[0..n] are k-mer indices (offs[n] = len-k+1), mm[0..n-1] the
 * keys.  Returns n (0 if len < k).  offs needs len-k+2 entries. */
int64_t orc_skm_split(const uint8_t *read, int64_t len, int k, int p,
                      const uint32_t *lut, int64_t *offs, uint32_t *mm) {
    if (len < k) return 0;
    int64_t nk = len - k + 1, n = 0, i;
    uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nk);
    orc_kmer_keys(read, len, k, p, lut, keys);
    offs[0] = 0; mm[0] = keys[0];
    for (i = 1; i < nk; i++) {
        if (keys[i] != keys[i - 1]) { n++; offs[n] = i; mm[n] = keys[i]; }
    }
    n++;
    offs[n] = nk;
    free(keys);
    return n;
}

/* Partition of a superkmer (cpu_funcs.cpp:213-215, gpu_skmgen.cu:276-278). */
uint32_t orc_partition(uint32_t key, uint32_t P) { return (~key) % P; }

/* Bytes of a superkmer of k-mers [beg, end) in the 3-bases-per-byte format,
 * including the terminal non-full byte (cpu_funcs.cpp:216-218). */
uint64_t orc_skm_nbytes(int64_t beg, int64_t end, int k) {
    return (uint64_t)(((beg % 3) + end + (k - 1) - beg + 3) / 3);
}

/* Packed byte b of a read (cpu_funcs.cpp:200-211, gpu_skmgen.cu:383-426):
 * [7:6] = number of valid bases (3 for full bytes; len%3 for the last byte),
 * [5:0] = three 2-bit bases, first base in [5:4]; missing bases are 0. */
static uint8_t packed_byte(const uint8_t *read, int64_t len, int64_t b) {
    int64_t pos = 3 * b, t;
    int64_t cnt = len - pos; if (cnt > 3) cnt = 3; if (cnt < 0) cnt = 0;
    uint8_t v = (uint8_t)(cnt << 6);
    for (t = 0; t < cnt; t++) v |= (uint8_t)(fwd_code(read[pos + t]) << (4 - 2 * t));
    return v;
}

/* Writes the bytes of superkmer [beg, end) of a read to out and returns the
 * byte count (cpu_funcs.cpp:238-244, gpu_skmgen.cu:459-465): a copy of the
 * packed read whose first byte's header says 3-beg%3 bases (held in its low
 * bits) and whose last byte's header says (end-1+k)%3 bases (high bits). */
uint64_t orc_skm_write(const uint8_t *read, int64_t len, int64_t beg, int64_t end,
                       int k, uint8_t *out) {
    uint64_t nb = orc_skm_nbytes(beg, end, k), b;
    for (b = 0; b < nb; b++) out[b] = packed_byte(read, len, beg / 3 + (int64_t)b);
    out[0] = (uint8_t)((out[0] & 0x3F) | ((3 - beg % 3) << 6));
    out[nb - 1] = (uint8_t)((out[nb - 1] & 0x3F) | (((end - 1 + k) % 3) << 6));
    return nb;
}

/* Phase 1 over a CSR batch of ASCII reads (cpu_funcs.cpp:252-298).
 * Counting mode (out == NULL): accumulates per-partition bytes, superkmers and
 * k-mers into part_bytes/part_skms/part_kmers (caller zeroes them).
 * Writing mode (out != NULL): appends every superkmer, in read order, at
 * out[part_cursor[p]] and advances part_cursor[p].
 * Reads shorter than k are skipped (fileloader.hpp:304).  Returns the number
 * of superkmers. */
int64_t orc_skmgen(const uint8_t *reads, const uint64_t *offs, int64_t n_reads,
                   int k, int p, uint32_t P, const uint32_t *lut,
                   uint64_t *part_bytes, uint64_t *part_skms, uint64_t *part_kmers,
                   uint8_t *out, uint64_t *part_cursor) {
    int64_t r, i, total = 0, maxlen = 0;
    for (r = 0; r < n_reads; r++) {
        int64_t l = (int64_t)(offs[r + 1] - offs[r]);
        if (l > maxlen) maxlen = l;
    }
    int64_t *so = (int64_t *)malloc(sizeof(int64_t) * (size_t)(maxlen + 2));
    uint32_t *mm = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(maxlen + 1));
    for (r = 0; r < n_reads; r++) {
        const uint8_t *read = reads + offs[r];
        int64_t len = (int64_t)(offs[r + 1] - offs[r]);
        int64_t n = orc_skm_split(read, len, k, p, lut, so, mm);
        for (i = 0; i < n; i++) {
            uint32_t part = orc_partition(mm[i], P);
            uint64_t nb = orc_skm_nbytes(so[i], so[i + 1], k);
            if (out) {
                orc_skm_write(read, len, so[i], so[i + 1], k, out + part_cursor[part]);
                part_cursor[part] += nb;
            } else {
                part_bytes[part] += nb;
                part_skms[part] += 1;
                part_kmers[part] += (uint64_t)(so[i + 1] - so[i]);
            }
        }
        total += n;
    }
    free(so); free(mm);
    return total;
}

/* Reverse complement of a 2k-bit k-mer (cpu_funcs.cpp:427-436,
 * gpu_kmercounting.cu:63-74). */
uint64_t orc_revcomp(uint64_t x, int k) {
    uint64_t r = 0; int i;
    x = ~x;
    for (i = 0; i < k; i++) { r = (r << 2) | (x & 3u); x >>= 2; }
    return r;
}

/* Decodes a stream of superkmers into canonical k-mers min(x, rc(x))
 * (cpu_funcs.cpp:437-515, gpu_kmercounting.cu:90-165).  Each superkmer is a
 * first byte (its low [7:6] bases valid), full bytes, and a terminal non-full
 * byte (its high [7:6] bases valid).  Writes to kmers (may be NULL to count)
 * and returns the number of k-mers, or -1 on a malformed stream. */
int64_t orc_extract(const uint8_t *bytes, uint64_t nbytes, int k, uint64_t *kmers) {
    uint64_t i = 0, mask = (k == 32) ? ~0ull : ((1ull << (2 * k)) - 1);
    int64_t n = 0;
    while (i < nbytes) {
        /* first byte */
        int h = bytes[i] >> 6, have = 0, t;
        uint64_t x = 0;
        for (t = 3 - h; t < 3; t++) { x = ((x << 2) | ((bytes[i] >> (4 - 2 * t)) & 3u)) & mask; have++; }
        if (have >= k) { if (kmers) { uint64_t rc = orc_revcomp(x, k); kmers[n] = x < rc ? x : rc; } n++; }
        i++;
        for (;;) {
            if (i >= nbytes) return -1;
            int c = bytes[i] >> 6;
            for (t = 0; t < c; t++) {
                x = ((x << 2) | ((bytes[i] >> (4 - 2 * t)) & 3u)) & mask;
                if (++have >= k) {
                    if (kmers) { uint64_t rc = orc_revcomp(x, k); kmers[n] = x < rc ? x : rc; }
                    n++;
                }
            }
            i++;
            if (c != 3) break;  /* terminal byte ends the superkmer */
        }
    }
    return n;
}

/* LSD radix sort of u64 keys, 16-bit digits (a plain sort; any sort gives the
 * same multiset as the reference's MSD radix + std::sort, cpu_funcs.cpp:365). */
void orc_sort_u64(uint64_t *a, int64_t n) {
    if (n <= 1) return;
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    size_t *cnt = (size_t *)malloc(sizeof(size_t) * 65536);
    uint64_t *src = a, *dst = tmp;
    int pass;
    for (pass = 0; pass < 4; pass++) {
        int sh = pass * 16; int64_t i; size_t s = 0;
        memset(cnt, 0, sizeof(size_t) * 65536);
        for (i = 0; i < n; i++) cnt[(src[i] >> sh) & 0xFFFF]++;
        for (i = 0; i < 65536; i++) { size_t c = cnt[i]; cnt[i] = s; s += c; }
        for (i = 0; i < n; i++) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        uint64_t *t = src; src = dst; dst = t;
    }
    /* four passes: the result is back in a */
    free(tmp); free(cnt);
}

/* Sort + run-length encode + threshold (cpu_funcs.cpp:586-651,
 * gpu_kmercounting.cu:420-523).  Sorts keys in place, writes the distinct
 * keys whose count c satisfies cmin <= c <= cmax (the [min,max] inclusive
 * range declared at utilities.hpp:190) to out_k/out_c in ascending key order,
 * counts saturating at 2^32-1 (types.h:101-102).  Returns the number written;
 * *n_distinct receives the number of distinct keys before the threshold. */
int64_t orc_count(uint64_t *keys, int64_t n, uint32_t cmin, uint32_t cmax,
                  uint64_t *out_k, uint32_t *out_c, int64_t *n_distinct) {
    int64_t i = 0, w = 0, d = 0;
    orc_sort_u64(keys, n);
    while (i < n) {
        int64_t j = i + 1;
        while (j < n && keys[j] == keys[i]) j++;
        uint64_t run = (uint64_t)(j - i);
        uint32_t c = run > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)run;
        if (c >= cmin && c <= cmax) {
            if (out_k) out_k[w] = keys[i];
            if (out_c) out_c[w] = c;
            w++;
        }
        d++;
        i = j;
    }
    if (n_distinct) *n_distinct = d;
    return w;
}

/* ------------------------------------------------------------------------
 * k-mers longer than 32 bases (the reference's LONGERKMER build, k <= 64,
 * T_kmer = unsigned __int128, types.h:34-35; utilities.hpp:280-281).  Keys
 * are passed as two u64 words per k-mer, low word first: the memory layout of
 * an unsigned __int128 on a little-endian host. */
typedef unsigned __int128 orc_u128;

static orc_u128 orc_revcomp128(orc_u128 x, int k) {
    orc_u128 r = 0; int i;
    x = ~x;
    for (i = 0; i < k; i++) { r = (r << 2) | (x & 3u); x >>= 2; }
    return r;
}

static void orc_put128(uint64_t *out, int64_t n, orc_u128 x, int k) {
    orc_u128 rc = orc_revcomp128(x, k), m = x < rc ? x : rc;
    out[2 * n] = (uint64_t)m;
    out[2 * n + 1] = (uint64_t)(m >> 64);
}

/* orc_extract for k <= 64 (cpu_funcs.cpp:437-515 with a 128-bit T_kmer). */
int64_t orc_extract_wide(const uint8_t *bytes, uint64_t nbytes, int k, uint64_t *kmers2) {
    orc_u128 mask = k >= 64 ? ~(orc_u128)0 : (((orc_u128)1 << (2 * k)) - 1);
    uint64_t i = 0;
    int64_t n = 0;
    while (i < nbytes) {
        int h = bytes[i] >> 6, have = 0, t;
        orc_u128 x = 0;
        for (t = 3 - h; t < 3; t++) { x = ((x << 2) | ((bytes[i] >> (4 - 2 * t)) & 3u)) & mask; have++; }
        if (have >= k) { if (kmers2) orc_put128(kmers2, n, x, k); n++; }
        i++;
        for (;;) {
            if (i >= nbytes) return -1;
            int c = bytes[i] >> 6;
            for (t = 0; t < c; t++) {
                x = ((x << 2) | ((bytes[i] >> (4 - 2 * t)) & 3u)) & mask;
                if (++have >= k) { if (kmers2) orc_put128(kmers2, n, x, k); n++; }
            }
            i++;
            if (c != 3) break;
        }
    }
    return n;
}

static int orc_cmp128(const void *a, const void *b) {
    const uint64_t *x = (const uint64_t *)a, *y = (const uint64_t *)b;
    if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    return 0;
}

/* orc_count for k <= 64: sorts the (low, high) pairs ascending as 128-bit
 * values, run-length encodes and applies [cmin, cmax]. */
int64_t orc_count_wide(uint64_t *keys2, int64_t n, uint32_t cmin, uint32_t cmax,
                       uint64_t *out_k2, uint32_t *out_c, int64_t *n_distinct) {
    int64_t i = 0, w = 0, d = 0;
    if (n > 1) qsort(keys2, (size_t)n, 16, orc_cmp128);
    while (i < n) {
        int64_t j = i + 1;
        while (j < n && keys2[2 * j] == keys2[2 * i] && keys2[2 * j + 1] == keys2[2 * i + 1]) j++;
        uint64_t run = (uint64_t)(j - i);
        uint32_t c = run > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)run;
        if (c >= cmin && c <= cmax) {
            if (out_k2) { out_k2[2 * w] = keys2[2 * i]; out_k2[2 * w + 1] = keys2[2 * i + 1]; }
            if (out_c) out_c[w] = c;
            w++;
        }
        d++;
        i = j;
    }
    if (n_distinct) *n_distinct = d;
    return w;
}
