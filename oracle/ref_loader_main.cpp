// ref_loader_main.cpp -- the reference's FASTQ / FASTA loader as a program.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile links this with ref_driver.cpp
// and the reference's cpu_funcs.cpp into oracle/_ref/ref_load_reads.  The
// loader's threads run in a process of their own: called inside a Python
// test process through ctypes, the reference's loader crashed, while as a
// program it runs cleanly.
//
//   ref_load_reads <input.fq|input.fa> <buffer MB> <output>
//
// Output: u64 n, then n + 1 u64 offsets, then the reads' bytes
// (ref_load_reads in ref_driver.cpp: the reads as ReadLoader extracts them,
// fileloader.hpp:51-545).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

extern "C" int64_t ref_load_reads(const char *path, int buffer_mb, char *out, uint64_t cap, uint64_t *offs,
                                  uint64_t cap_reads);

int main(int argc, char **argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <input> <buffer MB> <output>\n", argv[0]);
        return 2;
    }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fclose(f);
    std::vector<char> out(size + 1);
    std::vector<uint64_t> offs(size + 2);
    const int64_t n = ref_load_reads(argv[1], std::atoi(argv[2]), out.data(), size + 1, offs.data(), size + 1);
    if (n < 0) return 1;
    FILE *o = std::fopen(argv[3], "wb");
    if (!o) return 2;
    const uint64_t nn = (uint64_t)n;
    std::fwrite(&nn, 8, 1, o);
    std::fwrite(offs.data(), 8, nn + 1, o);
    std::fwrite(out.data(), 1, offs[nn], o);
    std::fclose(o);
    return 0;
}
