// pack_host.cpp -- host-side packing of ASCII read bases into 2-bit codes.
//
// A host batch of reads crosses PCIe as 2-bit codes, 16 bases to a u32 word
// (base 16w + t in bits 31-2t..30-2t, first base highest), instead of one byte
// per base: a quarter of the bytes.  The words are exactly those that phase 1
// stages from ASCII on the device (find_superkmers_kernel), with the device's
// base map (gkc_device.cuh codes4): A/C/G/T in either case -> 0/1/2/3, every
// other byte (N, U, IUPAC codes, anything) -> 0.  Positions past the last base
// of the last word are 0.
//
// The packing runs on a pool of host threads; each thread takes a contiguous
// range of words.  On a CPU with AVX2 a thread packs 32 bases per step (byte
// codes by shifts and compares, then multiply-adds into 4-base bytes and one
// byte shuffle into words); elsewhere, and for the batch's last partial
// words, a scalar loop does the same.
#include <immintrin.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <thread>
#include <vector>

namespace gkc_host {

// The device's base map for one byte.
static inline uint32_t code_of(uint8_t b) {
    const uint8_t l = (uint8_t)(b | 0x20);
    const bool ok = l == 'a' || l == 'c' || l == 'g' || l == 't';
    return ok ? (uint32_t)(((b >> 1) ^ (b >> 2)) & 3) : 0u;
}

// Words [w0, w1) of the n bases at src (positions >= n read as 0).
static void pack_words_scalar(const uint8_t *src, uint64_t n, uint32_t *dst, uint64_t w0, uint64_t w1) {
    for (uint64_t w = w0; w < w1; w++) {
        const uint64_t q = w * 16;
        uint32_t word = 0;
        if (q + 16 <= n) {
            for (int t = 0; t < 16; t++) word |= code_of(src[q + t]) << (30 - 2 * t);
        } else {
            for (int t = 0; t < 16; t++)
                if (q + t < n) word |= code_of(src[q + t]) << (30 - 2 * t);
        }
        dst[w] = word;
    }
}

__attribute__((target("avx2"))) static void pack_words_avx2(const uint8_t *src, uint64_t n, uint32_t *dst,
                                                             uint64_t w0, uint64_t w1) {
    const __m256i three = _mm256_set1_epi8(3), lower = _mm256_set1_epi8(0x20);
    const __m256i ca = _mm256_set1_epi8('a'), cc = _mm256_set1_epi8('c'), cg = _mm256_set1_epi8('g'),
                  ct = _mm256_set1_epi8('t');
    const __m256i w4 = _mm256_set1_epi16(0x0104);      // byte pairs: first * 4 + second
    const __m256i w16 = _mm256_set1_epi32(0x00010010);  // 16-bit pairs: first * 16 + second
    // the low byte of each 32-bit lane (4 bases), last first: one u32 word per 128-bit half
    const __m256i gather = _mm256_setr_epi8(12, 8, 4, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                                            12, 8, 4, 0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1);
    uint64_t w = w0;
    for (; w + 2 <= w1 && (w + 2) * 16 <= n; w += 2) {
        const __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i *>(src + w * 16));
        __m256i c = _mm256_and_si256(_mm256_xor_si256(_mm256_srli_epi16(v, 1), _mm256_srli_epi16(v, 2)), three);
        const __m256i l = _mm256_or_si256(v, lower);
        const __m256i ok = _mm256_or_si256(_mm256_or_si256(_mm256_cmpeq_epi8(l, ca), _mm256_cmpeq_epi8(l, cc)),
                                           _mm256_or_si256(_mm256_cmpeq_epi8(l, cg), _mm256_cmpeq_epi8(l, ct)));
        c = _mm256_and_si256(c, ok);
        const __m256i p4 = _mm256_madd_epi16(_mm256_maddubs_epi16(c, w4), w16);
        const __m256i g = _mm256_shuffle_epi8(p4, gather);
        dst[w] = (uint32_t)_mm256_extract_epi32(g, 0);
        dst[w + 1] = (uint32_t)_mm256_extract_epi32(g, 4);
    }
    pack_words_scalar(src, n, dst, w, w1);
}

static void pack_words(const uint8_t *src, uint64_t n, uint32_t *dst, uint64_t w0, uint64_t w1) {
    static const bool avx2 = __builtin_cpu_supports("avx2");
    if (avx2) pack_words_avx2(src, n, dst, w0, w1);
    else pack_words_scalar(src, n, dst, w0, w1);
}

// A fixed pool of packing threads; one job at a time (callers serialise).
class PackPool {
  public:
    static PackPool &get() {
        static PackPool pool;
        return pool;
    }
    // Packs n bases into words[0, nwords); words past the bases are 0.
    void run(const uint8_t *src, uint64_t n, uint32_t *words, uint64_t nwords) {
        std::lock_guard<std::mutex> one(job_mu_);
        if (nwords < 4096 || threads_.empty()) {  // small: not worth waking the pool
            pack_words(src, n, words, 0, nwords);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            src_ = src;
            n_ = n;
            dst_ = words;
            nwords_ = nwords;
            left_ = (int)threads_.size();
            gen_++;
        }
        cv_.notify_all();
        part(0, (int)threads_.size() + 1);  // the calling thread takes a share too
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return left_ == 0; });
    }

  private:
    PackPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nt = (int)std::min(hw, 16u) - 1;  // workers besides the calling thread
        for (int t = 0; t < nt; t++) threads_.emplace_back([this, t] { loop(t + 1); });
    }
    ~PackPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : threads_) t.join();
    }
    void part(int i, int parts) {
        const uint64_t per = (nwords_ + parts - 1) / parts;
        const uint64_t w0 = std::min<uint64_t>(nwords_, per * i), w1 = std::min<uint64_t>(nwords_, w0 + per);
        if (w0 < w1) pack_words(src_, n_, dst_, w0, w1);
    }
    void loop(int i) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            part(i, (int)threads_.size() + 1);
            std::lock_guard<std::mutex> lk(mu_);
            if (--left_ == 0) done_cv_.notify_one();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex job_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    uint64_t gen_ = 0;
    int left_ = 0;
    bool stop_ = false;
    const uint8_t *src_ = nullptr;
    uint64_t n_ = 0, nwords_ = 0;
    uint32_t *dst_ = nullptr;
};

void pack_bases(const uint8_t *src, uint64_t n, uint32_t *words, uint64_t nwords) {
    PackPool::get().run(src, n, words, nwords);
}

}  // namespace gkc_host
