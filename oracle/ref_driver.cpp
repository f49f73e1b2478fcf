// ref_driver.cpp -- drives RapidGKC's own CPU k-mer counting path.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this driver together
// with the reference's cpu_funcs.cpp, taken from the reference source tree
// where it lies (never copied), into oracle/_ref/libgkc_ref.so.  Tests use it
// to pin the C restatement (oracle/gkc_oracle.c) and to generate golden
// fixtures; bench.py's reference arm uses ref_run() as the CPU baseline.
//
// Reference entry points called (external linkage in cpu_funcs.cpp):
//   GenSuperkmerCPU   cpu_funcs.cpp:252-298  (phase 1, one batch of reads)
//   gen_skm_offs      cpu_funcs.cpp:147-198  (superkmer split of one read)
//   _h_process_bytes  cpu_funcs.cpp:437-515  (superkmer bytes -> canonical k-mers)
//   sort_kmers        cpu_funcs.cpp:365-392  (in-tree MSD radix + std::sort)
//   KmerCountingCPU   cpu_funcs.cpp:586-651  (phase 2 of one partition)
//   ReadLoader        fileloader.hpp:51-545  (FASTQ / FASTA record extraction)
//
// oracle/Makefile builds it three times: libgkc_ref.so with the reference's
// default 64-bit T_kmer (k <= 32), libgkc_ref_long.so with -DLONGERKMER, the
// reference's own 128-bit build for k <= 64 (types.h:34-35, CMakeLists.txt
// target l_<name>), and libgkc_ref_short.so with -DSHORTERKMER, its 32-bit
// build for k <= 16 (types.h:36-37, target s_<name>).
#include "cpu_funcs.h"
#include "fileloader.hpp"
#include "utilities.hpp"

#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <thread>
#include <vector>

Logger *logger = new Logger(0, Logger::LV_WARNING, false);

void _h_process_bytes(size_t beg, size_t end, u_char *skms, T_kmer *kmers,
                      std::atomic<size_t> *kmer_store_pos, T_kvalue k);
void sort_kmers(T_kmer *kmers, const T_skm_partsize n_kmers, const T_kvalue K_kmer, int i_base);
T_read_len gen_skm_offs(u_char *read, T_read_len len, const T_kvalue K_kmer,
                        const T_kvalue P_minimizer, T_read_len *skm_offs, T_minimizer *minimizers);

namespace {

struct Phase1Result {
    std::vector<SKMStoreNoncon *> stores;
};

// Moves every queued chunk of a store into one contiguous buffer (the same
// dequeue loop the reference's extract_kmers_cpu uses, cpu_funcs.cpp:548-559).
std::vector<u_char> drain_store(SKMStoreNoncon *s) {
    std::vector<u_char> out(s->tot_size_bytes);
    size_t pos = 0, count;
    SKM bulk[1024];
    do {
        count = s->skms.try_dequeue_bulk(bulk, 1024);
        for (size_t i = 0; i < count; i++) {
            memcpy(out.data() + pos, bulk[i].skm_chunk, bulk[i].chunk_bytes);
            pos += bulk[i].chunk_bytes;
        }
    } while (count);
    out.resize(pos);
    return out;
}

// Runs GenSuperkmerCPU over batches of `batch` reads with `threads` workers,
// like the reference's -cpuonly phase 1 (gkc_main.cpp:77-81 called from the
// loader's thread pool, fileloader.hpp:492-525).  GenSuperkmerCPU packs each
// read in place, so it is given a private copy of the reads.
void run_phase1(std::vector<char> &buf, const uint64_t *offs, int64_t n_reads, int k, int p,
                int P, int threads, int batch, std::vector<SKMStoreNoncon *> &stores, bool hpc = false) {
    std::atomic<int64_t> next{0};
    auto worker = [&](int tid) {
        for (;;) {
            int64_t b = next.fetch_add(batch);
            if (b >= n_reads) break;
            int64_t e = std::min<int64_t>(n_reads, b + batch);
            std::vector<ReadPtr> reads;
            reads.reserve(e - b);
            for (int64_t r = b; r < e; r++) {
                T_read_len len = (T_read_len)(offs[r + 1] - offs[r]);
                if (len < k) continue;  // the loader drops reads shorter than k
                reads.push_back(ReadPtr{buf.data() + offs[r], len});
            }
            if (!reads.empty())
                GenSuperkmerCPU(reads, (T_kvalue)k, (T_kvalue)p, hpc, P, stores, tid);
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(worker, t);
    for (auto &t : ts) t.join();
}

}  // namespace

extern "C" {

// Superkmer split of one read by the reference (cpu_funcs.cpp:147).
// offs needs len+1 entries, mm len entries.  Returns the superkmer count.
int ref_gen_skm_offs(const char *read, int len, int k, int p, int *offs, unsigned *mm) {
    std::vector<u_char> r(read, read + len);
    return gen_skm_offs(r.data(), len, (T_kvalue)k, (T_kvalue)p, offs, mm);
}

// Phase 1 of the reference over a CSR batch.  Fills per-partition bytes,
// superkmer and k-mer counts, and returns an opaque handle holding the
// partition stores.
void *ref_phase1_hpc(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int P,
                     int threads, int hpc, uint64_t *part_bytes, uint64_t *part_skms, uint64_t *part_kmers);

void *ref_phase1(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int P,
                 int threads, uint64_t *part_bytes, uint64_t *part_skms, uint64_t *part_kmers) {
    return ref_phase1_hpc(reads, offs, n_reads, k, p, P, threads, 0, part_bytes, part_skms, part_kmers);
}

// ref_phase1 with the reference's CPU homopolymer compression on or off
// (GenSuperkmerCPU's HPC argument, cpu_funcs.cpp:253-275).  Every read must
// stay at least k + 1 bytes long after compression: the reference's
// _hpc_encoding returns the compressed length minus one (cpu_funcs.cpp:92-100),
// and a read left shorter than k is read past its end (cpu_funcs.cpp:124-146).
void *ref_phase1_hpc(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int P,
                     int threads, int hpc, uint64_t *part_bytes, uint64_t *part_skms, uint64_t *part_kmers) {
    std::vector<char> buf(reads, reads + offs[n_reads]);
    auto *res = new Phase1Result();
    for (int i = 0; i < P; i++) res->stores.push_back(new SKMStoreNoncon(i, false));
    run_phase1(buf, offs, n_reads, k, p, P, threads, 2000, res->stores, hpc != 0);
    for (int i = 0; i < P; i++) {
        part_bytes[i] = res->stores[i]->tot_size_bytes;
        part_skms[i] = res->stores[i]->skm_cnt;
        part_kmers[i] = res->stores[i]->kmer_cnt;
    }
    return res;
}

// Copies the bytes of one partition (superkmers in the store's queue order).
// May be called once per partition.  Returns the byte count.
int64_t ref_part_bytes(void *h, int part, uint8_t *out) {
    auto *res = (Phase1Result *)h;
    std::vector<u_char> b = drain_store(res->stores[part]);
    memcpy(out, b.data(), b.size());
    return (int64_t)b.size();
}

// Counts a partition's superkmer bytes with the reference's own extraction
// and sort, then run-length encodes and applies [cmin, cmax].  Keys are
// written in ascending order, two u64 words each (low first) in the
// LONGERKMER build.  Returns the number written.
int64_t ref_count_bytes(const uint8_t *bytes, uint64_t nbytes, uint64_t n_kmers, int k,
                        uint32_t cmin, uint32_t cmax, uint64_t *out_k, uint32_t *out_c,
                        int64_t *n_distinct) {
    *n_distinct = 0;
    if (n_kmers == 0) return 0;
    std::vector<u_char> b(bytes, bytes + nbytes);
    std::vector<T_kmer> kmers(n_kmers);
    std::atomic<size_t> pos{0};
    _h_process_bytes(0, nbytes, b.data(), kmers.data(), &pos, (T_kvalue)k);
    if (pos.load() != n_kmers) return -1;
    sort_kmers(kmers.data(), n_kmers, (T_kvalue)k, 0);
    int64_t w = 0, d = 0;
    size_t i = 0;
    while (i < n_kmers) {
        size_t j = i + 1;
        while (j < n_kmers && kmers[j] == kmers[i]) j++;
        size_t run = j - i;
        uint32_t c = run > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)run;
        if (c >= cmin && c <= cmax) {
#ifdef LONGERKMER
            // two words per k-mer, low word first
            if (out_k) {
                out_k[2 * w] = (uint64_t)kmers[i];
                out_k[2 * w + 1] = (uint64_t)(kmers[i] >> 64);
            }
#else
            if (out_k) out_k[w] = kmers[i];
#endif
            if (out_c) out_c[w] = c;
            w++;
        }
        d++;
        i = j;
    }
    *n_distinct = d;
    return w;
}

// The reads of a FASTQ or FASTA file (FASTA when the name ends in 'a') as
// the reference's loader extracts them (ReadLoader::work_while_loading,
// fileloader.hpp:492-525; no length filter, one worker, buffers of
// buffer_mb MB so that lines cross buffer boundaries).  The loader hands
// reads over in batches; they are returned in the order the worker received
// them.  Writes at most cap bytes to out and cap_reads + 1 offsets; returns
// the number of reads, or -1 when out or offs is too small.
int64_t ref_load_reads(const char *path, int buffer_mb, char *out, uint64_t cap, uint64_t *offs,
                       uint64_t cap_reads) {
    std::vector<std::string> files{path};
    std::vector<std::string> got;
    std::mutex mu;
    ReadLoader::work_while_loading(
        0,
        [&](std::vector<ReadPtr> &batch, int) {
            std::lock_guard<std::mutex> lk(mu);
            for (const ReadPtr &r : batch) got.emplace_back(r.read, r.len);
        },
        1, files, 4096, 64, buffer_mb);
    uint64_t o = 0;
    if (got.size() > cap_reads) return -1;
    offs[0] = 0;
    for (size_t i = 0; i < got.size(); i++) {
        if (o + got[i].size() > cap) return -1;
        memcpy(out + o, got[i].data(), got[i].size());
        o += got[i].size();
        offs[i + 1] = o;
    }
    return (int64_t)got.size();
}

// Bits of the reference's T_kmer in this build (64, or 128 under LONGERKMER).
int ref_kmer_bits() { return (int)(8 * sizeof(T_kmer)); }

// Order-independent digest of the reference's thresholded (k-mer, count)
// table for a CSR read set: the reference's phase 1 (GenSuperkmerCPU over
// 2000-read batches, `threads` workers), then per partition its own
// extraction (_h_process_bytes) and sort (sort_kmers), with the run-length
// count of KmerCountingCPU (cpu_funcs.cpp:614-640) and [cmin, cmax] applied.
// out[0] kept k-mers, out[1] distinct k-mers, out[2] XOR of the kept k-mers,
// out[3] sum of k-mer * count (mod 2^64), out[4] sum of kept counts,
// out[5] k-mer instances.  A 128-bit k-mer enters as low ^ high * 0x9E3779B97F4A7C15.
// Returns 0, or -1 when a partition's extraction disagrees with its count.
int ref_digest(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int P, int threads,
               uint32_t cmin, uint32_t cmax, uint64_t *out) {
    std::vector<char> buf(reads, reads + offs[n_reads]);
    std::vector<SKMStoreNoncon *> stores;
    for (int i = 0; i < P; i++) stores.push_back(new SKMStoreNoncon(i, false));
    run_phase1(buf, offs, n_reads, k, p, P, threads, 2000, stores);
    std::atomic<int> next{0};
    std::atomic<int> bad{0};
    std::vector<std::array<uint64_t, 6>> acc(threads, std::array<uint64_t, 6>{0, 0, 0, 0, 0, 0});
    auto worker = [&](int tid) {
        auto &a = acc[tid];
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= P) break;
            SKMStoreNoncon *s = stores[i];
            const size_t nk = s->kmer_cnt;
            std::vector<u_char> b = drain_store(s);
            s->clear_skm_data();
            delete s;
            if (nk == 0) continue;
            std::vector<T_kmer> kmers(nk);
            std::atomic<size_t> pos{0};
            _h_process_bytes(0, b.size(), b.data(), kmers.data(), &pos, (T_kvalue)k);
            if (pos.load() != nk) {
                bad = 1;
                continue;
            }
            sort_kmers(kmers.data(), nk, (T_kvalue)k, 0);
            a[5] += nk;
            size_t r = 0;
            while (r < nk) {
                size_t j = r + 1;
                while (j < nk && kmers[j] == kmers[r]) j++;
                const size_t run = j - r;
                const uint32_t c = run > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)run;
                a[1]++;
                if (c >= cmin && c <= cmax) {
#ifdef LONGERKMER
                    const uint64_t key = (uint64_t)kmers[r] ^ ((uint64_t)(kmers[r] >> 64) * 0x9E3779B97F4A7C15ull);
#else
                    const uint64_t key = (uint64_t)kmers[r];
#endif
                    a[0]++;
                    a[2] ^= key;
                    a[3] += key * (uint64_t)c;
                    a[4] += c;
                }
                r = j;
            }
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(worker, t);
    for (auto &t : ts) t.join();
    for (int f = 0; f < 6; f++) out[f] = 0;
    for (auto &a : acc) {
        out[0] += a[0];
        out[1] += a[1];
        out[2] ^= a[2];
        out[3] += a[3];
        out[4] += a[4];
        out[5] += a[5];
    }
    return bad.load() ? -1 : 0;
}

void ref_free(void *h) {
    auto *res = (Phase1Result *)h;
    for (auto *s : res->stores) {
        s->clear_skm_data();
        delete s;
    }
    delete res;
}

// The reference's CPU-only pipeline for timing: phase 1 with `threads`
// workers over 2000-read batches, then phase 2 with `threads` workers, one
// KmerCountingCPU call per partition and one sorter thread each (the
// reference's `-cpuonly -im -t T -t2 T -tsort 1`, gkc_main.cpp:96-127).
// Returns the total number of distinct k-mers (gkc_main.cpp:385); t1/t2
// receive the phase wall times in seconds.
int64_t ref_run(const char *reads, const uint64_t *offs, int64_t n_reads, int k, int p, int P,
                int threads, double *t1, double *t2) {
    std::vector<char> buf(reads, reads + offs[n_reads]);
    std::vector<SKMStoreNoncon *> stores;
    for (int i = 0; i < P; i++) stores.push_back(new SKMStoreNoncon(i, false));
    auto c0 = std::chrono::steady_clock::now();
    run_phase1(buf, offs, n_reads, k, p, P, threads, 2000, stores);
    auto c1 = std::chrono::steady_clock::now();
    std::atomic<int> next{0};
    std::atomic<int64_t> distinct{0};
    std::vector<std::vector<T_kmc>> results(P);
    auto worker = [&](int tid) {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= P) break;
            // KmerCountingCPU deletes the store (cpu_funcs.cpp:648); an empty
            // partition returns early without deleting it.
            SKMStoreNoncon *s = stores[i];
            bool empty = s->kmer_cnt == 0;
            distinct += (int64_t)KmerCountingCPU((T_kvalue)k, s, 1, 0xFFFFFFFFu, results[i], tid, 1);
            if (empty) delete s;
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++) ts.emplace_back(worker, t);
    for (auto &t : ts) t.join();
    auto c2 = std::chrono::steady_clock::now();
    *t1 = std::chrono::duration<double>(c1 - c0).count();
    *t2 = std::chrono::duration<double>(c2 - c1).count();
    return distinct.load();
}

}  // extern "C"
