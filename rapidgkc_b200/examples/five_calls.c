/* five_calls.c -- counts the k-mers of a few reads through the five calls:
 * gkc_init (GPUReset), gkc_skmgen_batch (GenSuperkmerGPU),
 * gkc_count_partition (kmc_counting_GPU_streams, per partition),
 * gkc_shutdown. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "gkc_capi.h"

int main(void) {
    static const char reads[] =
        "ACGTTGCAAGGCTTACCGATGCATGCAAGTCCGATTAGCCGATAGGCTAACGTTAGC"  /* read 0: 57 bases */
        "TTGACCGTAGGCATCGATCGGATCCAAGTTGCAGCATGCAACGTTGCAAGGCTTACCGATG";  /* read 1: 61 bases */
    const uint64_t offs[] = {0, 57, 118};
    enum { K = 31, P_MIN = 11, PARTS = 4, CAP = 256 };
    gkc_options o;
    gkc_default_options(&o);
    o.k = K;
    o.p = P_MIN;
    o.partitions = PARTS;
    gkc_ctx *ctx = NULL;
    int rc = gkc_init(0, &o, &ctx);
    if (rc != GKC_OK) {
        fprintf(stderr, "gkc_init: %s\n", gkc_strerror(rc));
        return 1;
    }
    uint64_t kmers_per_part[PARTS];
    rc = gkc_skmgen_batch(ctx, reads, offs, 2, K, P_MIN, PARTS, NULL, GKC_MEM_HOST, NULL, NULL, kmers_per_part);
    uint64_t distinct = 0, instances = 0;
    for (int part = 0; rc == GKC_OK && part < PARTS; part++) {
        uint64_t kmers[CAP];
        uint32_t counts[CAP];
        uint64_t n = 0, d = 0;
        rc = gkc_count_partition(ctx, part, 1, UINT32_MAX, kmers, counts, CAP, GKC_MEM_HOST, &n, &d);
        distinct += d;
        instances += kmers_per_part[part];
    }
    if (rc != GKC_OK) fprintf(stderr, "error: %s (%s)\n", gkc_strerror(rc), gkc_last_error(ctx));
    else printf("instances %llu distinct %llu\n", (unsigned long long)instances, (unsigned long long)distinct);
    gkc_shutdown(ctx);
    return rc == GKC_OK ? 0 : 1;
}
