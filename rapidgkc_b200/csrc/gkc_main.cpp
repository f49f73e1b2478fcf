// gkc_main.cpp -- command-line k-mer counter on the B200 library.
//
// Takes RapidGKC's own flags (gkc_main.cpp / utilities.hpp:222-270 of the
// reference): -k, -p, -skm, -read <files...>, and accepts its thread, launch
// and file-store flags (the library picks launch shapes itself and keeps the
// store in device memory).  Adds what the reference declares but never does:
// the count threshold (utilities.hpp:190) and an output of the counted
// k-mers.
//
//   gkc_main -k 31 -p 11 -skm 512 -ci 2 -o counts.bin -read reads.fq.gz [more files]
//
// Output (-o): binary (-of bin, default): "GKCB1\0\0\0", u32 k, u32 0, u64 n,
// then n records of u64 k-mer (2-bit, first base in the most significant
// position, canonical) and u32 count, little-endian, 12 bytes each (for
// k > 32: the k-mer's low then high u64, 20 bytes each); or text
// (-of txt): "<k-mer>\t<count>\n".  Order: the library's (per partition;
// ascending within a partition with -counter sort), or ascending k-mer with
// -sorted.
//
// Input: FASTA or FASTQ, plain or gzip (zlib reads both).  A reader thread
// fills pinned blocks of about -bb MB of decompressed text while the main
// thread hands the previous block to the GPU, which scans its records
// (gkc_add_fastx) and splits the reads into superkmers.
#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gkc_capi.h"

namespace {

// Defaults are the reference's (utilities.hpp:187-189): k=21, p=7, 31
// partitions.  Its count threshold [1, 1000] (utilities.hpp:190) is never
// applied by the reference, so the default here keeps every k-mer.
struct Args {
    int k = 21, p = 7, partitions = 31, device = 0;
    uint32_t cmin = 1, cmax = 0xFFFFFFFFu;
    std::string out, fmt = "bin", counter = "hash", order = "default";
    bool sorted = false, hpc = false;
    uint64_t batch_mb = 1024;
    std::vector<std::string> files;
};

[[noreturn]] void usage(const char *prog, const char *why) {
    std::fprintf(stderr,
                 "%s\nUsage: %s [-k <K> (21)] [-p <P> (7)] [-skm <partitions> (31)] [-ci <min count>] [-cx <max count>]\n"
                 "       [-o <output>] [-of bin|txt] [-sorted] [-counter hash|sort]\n"
                 "       [-order default|learned|<params.f32>] [-gpu <device>] [-bb <batch MB>] [-hpc 0|1]\n"
                 "       -read <files...>\n"
                 "       (-t -tgpu -t2 -tgz -tsort -tmp -im -fb -rb -grid -block -grid2 -block2 -ns1 -ns2 -rps\n"
                 "        -gpuonly -log -lv are accepted for compatibility and have no effect)\n",
                 why, prog);
    std::exit(2);
}

Args parse_args(int argc, char **argv) {
    Args a;
    auto need = [&](int &i) -> const char * {
        if (i + 1 >= argc) usage(argv[0], "missing value");
        return argv[++i];
    };
    for (int i = 1; i < argc; i++) {
        const std::string f = argv[i];
        if (f == "-k") a.k = std::atoi(need(i));
        else if (f == "-p") a.p = std::atoi(need(i));
        else if (f == "-skm") a.partitions = std::atoi(need(i));
        else if (f == "-ci") a.cmin = (uint32_t)std::strtoul(need(i), nullptr, 10);
        else if (f == "-cx") a.cmax = (uint32_t)std::strtoul(need(i), nullptr, 10);
        else if (f == "-o") a.out = need(i);
        else if (f == "-of") a.fmt = need(i);
        else if (f == "-sorted") a.sorted = true;
        else if (f == "-counter") a.counter = need(i);
        else if (f == "-order") a.order = need(i);
        else if (f == "-gpu") a.device = std::atoi(need(i));
        else if (f == "-bb") a.batch_mb = std::strtoull(need(i), nullptr, 10);
        else if (f == "-hpc") a.hpc = std::atoi(need(i)) != 0;
        else if (f == "-ngpu") {
            if (std::atoi(need(i)) > 1) usage(argv[0], "one GPU per process (-ngpu 1)");
        } else if (f == "-cpuonly") {
            usage(argv[0], "there is no CPU path (-cpuonly)");
        } else if (f == "-t" || f == "-tgpu" || f == "-t2" || f == "-tgz" || f == "-tsort" || f == "-tmp" ||
                   f == "-fb" || f == "-rb" || f == "-grid" || f == "-block" || f == "-grid2" || f == "-block2" ||
                   f == "-ns1" || f == "-ns2" || f == "-rps" || f == "-log" || f == "-lv") {
            need(i);
        } else if (f == "-im" || f == "-gpuonly") {
        } else if (f == "-read") {
            while (i + 1 < argc && argv[i + 1][0] != '-') a.files.push_back(argv[++i]);
        } else {
            usage(argv[0], ("unknown argument " + f).c_str());
        }
    }
    if (a.files.empty()) usage(argv[0], "no input (-read)");
    if (a.fmt != "bin" && a.fmt != "txt") usage(argv[0], "-of must be bin or txt");
    if (a.counter != "hash" && a.counter != "sort") usage(argv[0], "-counter must be hash or sort");
    if (a.cmin > a.cmax) usage(argv[0], "-ci is larger than -cx");
    return a;
}

void check(int rc, gkc_ctx *ctx, const char *what) {
    if (rc != GKC_OK) {
        std::fprintf(stderr, "gkc_main: %s: %s (%s)\n", what, gkc_strerror(rc), ctx ? gkc_last_error(ctx) : "");
        std::exit(1);
    }
}

// A block of FASTA / FASTQ text in pinned host memory, cut where the GPU
// scanner can pick up again (TextReader::next).
struct TextBlock {
    char *p = nullptr;
    uint64_t cap = 0, n = 0;
    int fmt = GKC_FASTQ;
    bool file_start = false;  // the first block of a file: the FASTQ phase restarts
    uint64_t repeated = 0;    // bases repeated from the block before (FASTA, see below)
    void reserve(uint64_t want) {
        if (want <= cap) return;
        char *q = nullptr;
        const uint64_t c = want + want / 4;
        if (cudaHostAlloc(reinterpret_cast<void **>(&q), c, cudaHostAllocDefault) != cudaSuccess) {
            std::fprintf(stderr, "gkc_main: pinned allocation of %llu bytes failed\n", (unsigned long long)c);
            std::exit(1);
        }
        if (n) std::memcpy(q, p, n);
        if (p) cudaFreeHost(p);
        p = q;
        cap = c;
    }
    ~TextBlock() {
        if (p) cudaFreeHost(p);
    }
};

// Decompressed text of one file (plain or gzip) in blocks of about `block`
// bytes.  FASTQ blocks end after a newline: the GPU scanner carries the line
// phase across them, as the reference loader does (fileloader.hpp:201-232).
// FASTA blocks end before a '>' header line, so records stay whole; a record
// longer than a block is cut after a newline, and its last k - 1 bases are
// repeated at the start of the next block, so every k-mer across the cut is
// counted once.
class TextReader {
public:
    TextReader(const std::string &path, uint64_t block, int k)
        : fp_(gzopen(path.c_str(), "rb")), path_(path), block_(block), k_(k) {
        if (!fp_) {
            std::fprintf(stderr, "gkc_main: cannot open %s\n", path.c_str());
            std::exit(1);
        }
        gzbuffer(fp_, 1 << 22);
    }
    ~TextReader() { gzclose(fp_); }
    // The next block; false at the end of the file.
    bool next(TextBlock &b) {
        b.n = 0;
        b.repeated = repeat_;
        b.file_start = first_;
        b.reserve(std::max<uint64_t>(block_, carry_.size()) + 64);
        std::memcpy(b.p, carry_.data(), carry_.size());
        b.n = carry_.size();
        carry_.clear();
        repeat_ = 0;
        for (;;) {  // fill the block; grow it while it holds no place to cut
            while (!eof_ && b.n < b.cap - 64) {
                const uint64_t want = std::min<uint64_t>(b.cap - 64 - b.n, 1u << 30);
                const int got = gzread(fp_, b.p + b.n, (unsigned)want);
                if (got < 0) {
                    std::fprintf(stderr, "gkc_main: read error in %s\n", path_.c_str());
                    std::exit(1);
                }
                if (got == 0) eof_ = true;
                b.n += (uint64_t)got;
                if (b.n >= block_) break;
            }
            if (first_) detect(b);
            first_ = false;
            if (eof_ || cut(b)) break;
            b.reserve(b.cap * 2);
        }
        b.fmt = fmt_;
        return b.n > 0;
    }

private:
    void detect(const TextBlock &b) {
        uint64_t i = 0;
        while (i < b.n && (b.p[i] == '\n' || b.p[i] == '\r' || b.p[i] == ' ')) i++;
        if (i == b.n) return;  // empty: either format gives no reads
        if (b.p[i] == '@') fmt_ = GKC_FASTQ;
        else if (b.p[i] == '>') fmt_ = GKC_FASTA;
        else {
            std::fprintf(stderr, "gkc_main: %s is not FASTA or FASTQ\n", path_.c_str());
            std::exit(1);
        }
    }
    // Cuts the block at a place the scanner can resume from and keeps the
    // rest for the next block; false if there is none yet.
    bool cut(TextBlock &b) {
        uint64_t c = b.n;
        if (fmt_ == GKC_FASTA) {  // before the last header line
            for (uint64_t i = b.n; i-- > 1;)
                if (b.p[i] == '>' && b.p[i - 1] == '\n') {
                    c = i;
                    break;
                }
            if (c < b.n) {
                carry_.assign(b.p + c, b.n - c);
                b.n = c;
                return true;
            }
        }
        uint64_t nl = b.n;  // after the last newline
        for (uint64_t i = b.n; i-- > 0;)
            if (b.p[i] == '\n') {
                nl = i + 1;
                break;
            }
        if (nl == b.n && (b.n == 0 || b.p[b.n - 1] != '\n')) return false;
        carry_.assign(b.p + nl, b.n - nl);
        b.n = nl;
        if (fmt_ == GKC_FASTA) {  // inside a record: repeat its last k - 1 bases
            // the block holds no header line but perhaps one at its start
            uint64_t s0 = 0;
            if (b.p[0] == '>') {
                s0 = nl;
                for (uint64_t i = 0; i < nl; i++)
                    if (b.p[i] == '\n') {
                        s0 = i + 1;
                        break;
                    }
            }
            std::string tail;
            for (uint64_t i = nl; i-- > s0 && (int)tail.size() < k_ - 1;)
                if (b.p[i] != '\n' && b.p[i] != '\r') tail.push_back(b.p[i]);
            std::reverse(tail.begin(), tail.end());
            repeat_ = tail.size();
            carry_.insert(0, tail + "\n");
        }
        return true;
    }
    gzFile fp_;
    std::string path_, carry_;
    uint64_t block_;
    int k_;
    int fmt_ = GKC_FASTQ;
    bool first_ = true, eof_ = false;
    uint64_t repeat_ = 0;
};

std::vector<float> load_params(const std::string &path, uint64_t n) {
    std::vector<float> v(n);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), 4, n, f) != n) {
        std::fprintf(stderr, "gkc_main: cannot read %llu parameters from %s\n", (unsigned long long)n, path.c_str());
        std::exit(1);
    }
    std::fclose(f);
    return v;
}

std::string exe_dir() {
    char buf[4096];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    if (n <= 0) return ".";
    std::string s(buf, (size_t)n);
    return s.substr(0, s.rfind('/'));
}

// km holds kw u64 words per k-mer (kw = 2 for k > 32: low word first).
void write_output(const Args &a, const uint64_t *km, int kw, const uint32_t *ct, uint64_t n) {
    FILE *f = std::fopen(a.out.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "gkc_main: cannot write %s\n", a.out.c_str());
        std::exit(1);
    }
    std::vector<char> buf;
    buf.reserve(1 << 24);
    auto flush = [&]() {
        if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) {
            std::fprintf(stderr, "gkc_main: write to %s failed\n", a.out.c_str());
            std::exit(1);
        }
        buf.clear();
    };
    if (a.fmt == "bin") {
        const char magic[8] = {'G', 'K', 'C', 'B', '1', 0, 0, 0};
        const uint32_t hk[2] = {(uint32_t)a.k, 0};
        buf.insert(buf.end(), magic, magic + 8);
        buf.insert(buf.end(), reinterpret_cast<const char *>(hk), reinterpret_cast<const char *>(hk) + 8);
        buf.insert(buf.end(), reinterpret_cast<const char *>(&n), reinterpret_cast<const char *>(&n) + 8);
        for (uint64_t i = 0; i < n; i++) {
            buf.insert(buf.end(), reinterpret_cast<const char *>(km + kw * i),
                       reinterpret_cast<const char *>(km + kw * (i + 1)));
            buf.insert(buf.end(), reinterpret_cast<const char *>(ct + i), reinterpret_cast<const char *>(ct + i) + 4);
            if (buf.size() > (1u << 24) - 64) flush();
        }
    } else {
        char rec[96];
        for (uint64_t i = 0; i < n; i++) {
            const unsigned __int128 x = kw == 2 ? ((unsigned __int128)km[2 * i + 1] << 64) | km[2 * i] : km[i];
            for (int j = 0; j < a.k; j++) rec[j] = "ACGT"[(int)(x >> (2 * (a.k - 1 - j))) & 3];
            const int m = std::snprintf(rec + a.k, sizeof(rec) - a.k, "\t%u\n", ct[i]);
            buf.insert(buf.end(), rec, rec + a.k + m);
            if (buf.size() > (1u << 24) - 64) flush();
        }
    }
    flush();
    std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) {
    const Args a = parse_args(argc, argv);
    const auto t_start = std::chrono::steady_clock::now();
    auto secs = [&]() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    };
    gkc_options opt;
    gkc_default_options(&opt);
    opt.k = a.k;
    opt.p = a.p;
    opt.partitions = a.partitions;
    opt.counter = a.counter == "sort" ? GKC_COUNTER_SORT : GKC_COUNTER_HASH;
    opt.hpc = a.hpc ? 1 : 0;
    gkc_ctx *ctx = nullptr;
    check(gkc_create(a.device, &opt, &ctx), nullptr, "create");
    if (a.order != "default") {
        const std::string path = a.order == "learned" ? exe_dir() + "/orders/skewed_m" + std::to_string(a.p) + ".f32"
                                                      : a.order;
        const std::vector<float> params = load_params(path, gkc_mlp_param_count(a.p));
        check(gkc_mlp_order(ctx, params.data(), 0, nullptr), ctx, "learned order");
    }
    // ---- phase 1: a reader thread fills one pinned text block while the GPU
    // scans and splits the other
    const uint64_t block = a.batch_mb << 20;
    TextBlock blocks[2];
    std::mutex mu;
    std::condition_variable cv;
    bool full[2] = {false, false}, eof = false;
    uint64_t produced = 0, consumed = 0;
    uint64_t n_reads = 0, n_bases = 0;
    std::thread parser([&]() {  // fills slots 0, 1, 0, ... in turn
        size_t fi = 0;
        TextReader *rd = new TextReader(a.files[0], block, a.k);
        for (int slot = 0;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&]() { return !full[slot]; });
            }
            if (!rd->next(blocks[slot])) {
                delete rd;
                rd = nullptr;
                if (++fi == a.files.size()) break;
                rd = new TextReader(a.files[fi], block, a.k);
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            full[slot] = true;
            produced++;
            cv.notify_all();
            slot ^= 1;
        }
        std::lock_guard<std::mutex> lk(mu);
        eof = true;
        cv.notify_all();
    });
    int state = 0;  // FASTQ line phase, carried from block to block
    for (int slot = 0;; slot ^= 1) {  // takes slots 0, 1, 0, ... in turn
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&]() { return full[slot] || (eof && consumed == produced); });
            if (!full[slot]) break;
        }
        TextBlock &b = blocks[slot];
        if (b.file_start) state = 0;
        uint64_t nr = 0, nb = 0;
        check(gkc_add_fastx(ctx, b.p, b.n, GKC_MEM_HOST, b.fmt, &state, &nr, &nb), ctx, "phase 1");
        n_reads += nr;
        n_bases += nb - b.repeated;
        std::lock_guard<std::mutex> lk(mu);
        full[slot] = false;
        consumed++;
        cv.notify_all();
    }
    parser.join();
    const double t1 = secs();
    // ---- phase 2
    uint64_t kmer_instances = 0;
    {
        std::vector<uint64_t> pb(a.partitions), ps(a.partitions), pk(a.partitions);
        check(gkc_store_stats(ctx, pb.data(), ps.data(), pk.data()), ctx, "store stats");
        for (uint64_t v : pk) kmer_instances += v;
    }
    uint64_t n_out = 0, n_distinct = 0;
    check(gkc_count(ctx, a.cmin, a.cmax, &n_out, &n_distinct), ctx, "phase 2");
    const double t2 = secs();
    if (!a.out.empty()) {
        const int kw = a.k > 32 ? 2 : 1;  // u64 words per k-mer
        uint64_t *km = nullptr;
        uint32_t *ct = nullptr;
        if (cudaHostAlloc(reinterpret_cast<void **>(&km), std::max<uint64_t>(n_out, 1) * 8 * kw, 0) != cudaSuccess ||
            cudaHostAlloc(reinterpret_cast<void **>(&ct), std::max<uint64_t>(n_out, 1) * 4, 0) != cudaSuccess) {
            std::fprintf(stderr, "gkc_main: pinned allocation for %llu results failed\n", (unsigned long long)n_out);
            return 1;
        }
        check(gkc_result(ctx, km, ct, n_out, GKC_MEM_HOST), ctx, "result");
        if (a.sorted) {
            std::vector<uint64_t> ix(n_out);
            for (uint64_t i = 0; i < n_out; i++) ix[i] = i;
            auto key = [&](uint64_t i) {
                return kw == 2 ? ((unsigned __int128)km[2 * i + 1] << 64) | km[2 * i] : (unsigned __int128)km[i];
            };
            std::sort(ix.begin(), ix.end(), [&](uint64_t x, uint64_t y) { return key(x) < key(y); });
            std::vector<uint64_t> k2(n_out * kw);
            std::vector<uint32_t> c2(n_out);
            for (uint64_t i = 0; i < n_out; i++) {
                for (int w = 0; w < kw; w++) k2[kw * i + w] = km[kw * ix[i] + w];
                c2[i] = ct[ix[i]];
            }
            write_output(a, k2.data(), kw, c2.data(), n_out);
        } else {
            write_output(a, km, kw, ct, n_out);
        }
        cudaFreeHost(km);
        cudaFreeHost(ct);
    }
    const double t3 = secs();
    // the reference's report: its log lines on stderr (gkc_main.cpp:385 and
    // the phase-1 k-mer total), the wall seconds alone on stdout (:433)
    std::fprintf(stderr, "P0 [INFO]\tKMER TOT CNT = %llu\n", (unsigned long long)kmer_instances);
    std::fprintf(stderr, "P0 [NOTICE]\tTotal number of distinct kmers: %llu\n", (unsigned long long)n_distinct);
    std::fprintf(stderr,
                 "reads %llu, bases %llu, distinct k-mers %llu, written %llu (count in [%u, %u])\n"
                 "phase 1 %.3f s, phase 2 %.3f s, output %.3f s, total %.3f s (%.2f Gbp/s)\n",
                 (unsigned long long)n_reads, (unsigned long long)n_bases, (unsigned long long)n_distinct,
                 (unsigned long long)n_out, a.cmin, a.cmax, t1, t2 - t1, t3 - t2, t3, n_bases / t3 / 1e9);
    std::printf("%g\n", t3);
    gkc_destroy(ctx);
    return 0;
}
