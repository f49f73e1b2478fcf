// synth.cpp -- seeded synthetic genomes and read sets for the k-mer counter.
//
// No public dataset is available to this project, so workloads are produced
// here with the shapes the counter is specified on: i.i.d. genomes at a given
// GC fraction, repeat families copied at a divergence, low-complexity runs
// (poly-A, (AT)n, (CAG)n), and reads sampled from both strands with uniform
// substitution errors, either fixed-length short reads or log-normal long
// reads.  Every random draw comes from a counter-based generator keyed by
// (seed, stream, index), so the output does not depend on the thread count.
//
// C ABI (all return 0 on success, negative on bad arguments):
//   gkc_synth_genome  fills a genome buffer
//   gkc_synth_reads   samples reads of one fixed length into a CSR buffer
//   gkc_synth_long_read_lengths  draws clipped log-normal read lengths
//   gkc_synth_reads_var  samples reads with given lengths into a CSR buffer
#include <algorithm>
#include <string>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Counter-based stream: draw i of stream s under seed.
struct Rng {
    uint64_t key, ctr = 0;
    Rng(uint64_t seed, uint64_t stream) : key(mix64(seed * 0x100000001B3ull ^ mix64(stream))) {}
    uint64_t next() { return mix64(key + 0x632BE59BD9B4E019ull * (++ctr)); }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? (uint64_t)(((unsigned __int128)next() * n) >> 64) : 0; }
    double normal() {  // Box-Muller
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

const char ACGT[4] = {'A', 'C', 'G', 'T'};

inline char comp(char c) {
    switch (c) { case 'A': return 'T'; case 'C': return 'G'; case 'G': return 'C'; default: return 'A'; }
}

inline char gc_base(Rng &r, double gc) {
    double u = r.uni();
    if (u < gc) return (u < gc * 0.5) ? 'C' : 'G';
    return (u < gc + (1.0 - gc) * 0.5) ? 'A' : 'T';
}

int nthreads_or_default(int t) {
    if (t > 0) return t;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

template <class F> void parallel_for(int64_t n, int threads, F f) {
    threads = (int)std::max<int64_t>(1, std::min<int64_t>(threads, n));
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
        ts.emplace_back([=]() {
            int64_t b = n * t / threads, e = n * (t + 1) / threads;
            for (int64_t i = b; i < e; i++) f(i);
        });
    for (auto &t : ts) t.join();
}

}  // namespace

extern "C" {

// Genome of `length` bases.  Background: i.i.d. with GC fraction `gc`.
// Then `n_families` repeat consensus sequences of uniform length in
// [fam_min, fam_max] are copied at uniform positions until `repeat_frac` of
// the genome has been written by copies; each copy gets substitutions at a
// rate drawn uniformly in [div_min, div_max].  Finally low-complexity runs of
// uniform length in [lc_min, lc_max], a third each poly-A, (AT)n and (CAG)n,
// are written until `lowcomp_frac` of the genome is covered.
int gkc_synth_genome(uint64_t seed, int64_t length, double gc, double repeat_frac,
                     int n_families, int fam_min, int fam_max, double div_min, double div_max,
                     double lowcomp_frac, int lc_min, int lc_max, char *out, int threads) {
    if (length <= 0 || !out || gc < 0 || gc > 1) return -1;
    threads = nthreads_or_default(threads);
    const int64_t CH = 1 << 20;
    int64_t nch = (length + CH - 1) / CH;
    parallel_for(nch, threads, [&](int64_t c) {
        Rng r(seed, 1000 + (uint64_t)c);
        int64_t b = c * CH, e = std::min(length, b + CH);
        for (int64_t i = b; i < e; i++) out[i] = gc_base(r, gc);
    });
    if (repeat_frac > 0 && n_families > 0 && fam_max >= fam_min && fam_min > 0) {
        Rng r(seed, 1);
        std::vector<std::string> fam(n_families);
        for (int f = 0; f < n_families; f++) {
            int64_t L = fam_min + (int64_t)r.below((uint64_t)(fam_max - fam_min + 1));
            fam[f].resize(L);
            for (int64_t i = 0; i < L; i++) fam[f][i] = gc_base(r, gc);
        }
        int64_t target = (int64_t)(repeat_frac * (double)length), written = 0;
        while (written < target) {
            const std::string &s = fam[r.below(n_families)];
            int64_t L = (int64_t)s.size();
            if (L >= length) break;
            int64_t pos = (int64_t)r.below((uint64_t)(length - L));
            double div = div_min + (div_max - div_min) * r.uni();
            bool rc = r.below(2);
            for (int64_t i = 0; i < L; i++) {
                char c = rc ? comp(s[L - 1 - i]) : s[i];
                if (r.uni() < div) c = ACGT[(std::find(ACGT, ACGT + 4, c) - ACGT + 1 + r.below(3)) & 3];
                out[pos + i] = c;
            }
            written += L;
        }
    }
    if (lowcomp_frac > 0 && lc_max >= lc_min && lc_min > 0) {
        Rng r(seed, 2);
        int64_t target = (int64_t)(lowcomp_frac * (double)length), written = 0;
        static const char *motif[3] = {"A", "AT", "CAG"};
        while (written < target) {
            int64_t L = lc_min + (int64_t)r.below((uint64_t)(lc_max - lc_min + 1));
            if (L >= length) break;
            int64_t pos = (int64_t)r.below((uint64_t)(length - L));
            int t = (int)r.below(3);
            const char *m = motif[t];
            int ml = (int)strlen(m);
            for (int64_t i = 0; i < L; i++) out[pos + i] = m[i % ml];
            written += L;
        }
    }
    return 0;
}

// `n_reads` reads of `read_len` bases at uniform positions, reverse
// complemented with probability 1/2 when both_strands is set, each base
// substituted with probability `err` by one of the three other bases.
// out_reads holds n_reads*read_len bytes; out_offs n_reads+1 offsets.
int gkc_synth_reads(const char *genome, int64_t glen, uint64_t seed, int64_t n_reads, int read_len,
                    double err, int both_strands, char *out_reads, uint64_t *out_offs, int threads) {
    if (!genome || glen < read_len || read_len <= 0 || n_reads < 0) return -1;
    threads = nthreads_or_default(threads);
    for (int64_t i = 0; i <= n_reads; i++) out_offs[i] = (uint64_t)i * (uint64_t)read_len;
    parallel_for(n_reads, threads, [&](int64_t i) {
        Rng r(seed, 0x1000000000ull + (uint64_t)i);
        int64_t pos = (int64_t)r.below((uint64_t)(glen - read_len + 1));
        bool rc = both_strands && r.below(2);
        char *o = out_reads + (uint64_t)i * read_len;
        for (int j = 0; j < read_len; j++) {
            char c = rc ? comp(genome[pos + read_len - 1 - j]) : genome[pos + j];
            if (err > 0 && r.uni() < err) {
                int idx = (int)(std::find(ACGT, ACGT + 4, c) - ACGT);
                c = ACGT[(idx + 1 + (int)r.below(3)) & 3];
            }
            o[j] = c;
        }
    });
    return 0;
}

// Log-normal lengths with the given median and log-space sigma, clipped to
// [lmin, lmax].
int gkc_synth_long_read_lengths(uint64_t seed, int64_t n, double median, double sigma, int64_t lmin,
                                int64_t lmax, int64_t *out) {
    if (n < 0 || median <= 0 || lmin > lmax) return -1;
    Rng r(seed, 3);
    double mu = std::log(median);
    for (int64_t i = 0; i < n; i++) {
        double v = std::exp(mu + sigma * r.normal());
        int64_t L = (int64_t)std::llround(v);
        out[i] = std::min(lmax, std::max(lmin, L));
    }
    return 0;
}

// Reads with per-read lengths `lens` (CSR offsets already in out_offs,
// n_reads+1 entries), otherwise like gkc_synth_reads.  `stream` separates
// read sets drawn from the same genome and seed.
int gkc_synth_reads_var(const char *genome, int64_t glen, uint64_t seed, uint64_t stream,
                        int64_t n_reads, const uint64_t *offs, double err, int both_strands,
                        char *out_reads, int threads) {
    if (!genome || n_reads < 0) return -1;
    threads = nthreads_or_default(threads);
    for (int64_t i = 0; i < n_reads; i++)
        if ((int64_t)(offs[i + 1] - offs[i]) > glen) return -2;
    parallel_for(n_reads, threads, [&](int64_t i) {
        Rng r(seed, (stream << 40) + 0x2000000000ull + (uint64_t)i);
        int64_t L = (int64_t)(offs[i + 1] - offs[i]);
        int64_t pos = (int64_t)r.below((uint64_t)(glen - L + 1));
        bool rc = both_strands && r.below(2);
        char *o = out_reads + offs[i];
        for (int64_t j = 0; j < L; j++) {
            char c = rc ? comp(genome[pos + L - 1 - j]) : genome[pos + j];
            if (err > 0 && r.uni() < err) {
                int idx = (int)(std::find(ACGT, ACGT + 4, c) - ACGT);
                c = ACGT[(idx + 1 + (int)r.below(3)) & 3];
            }
            o[j] = c;
        }
    });
    return 0;
}

}  // extern "C"
