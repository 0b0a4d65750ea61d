/* A GPU job driven from C through the ABI alone (gcc, no C++ runtime of the caller), the way
 * the reference's host drives its engine (src/service/gpu.rs:806-887): create a context
 * (Kernel::load), prepare a job (Engine::prepare), launch one iteration over indices from 0
 * (Engine::launch), read the candidate hits and confirm each needle's first key on the host.
 *
 *   abi_gpu <key hex> <needle>:<fold>:<mode> ...
 *
 * Prints "launch <found> <lowest>", then per needle k "hits <k> <index> ..." (its candidates
 * below 65536, in index order) and "first <k> <status> <index> <public key hex>". */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "meikey_b200.h"

static int hexval(char c) { return c <= '9' ? c - '0' : (c | 32) - 'a' + 10; }

static int report(mk_ctx* ctx, int st, const char* what) {
    char err[256] = "";
    mk_last_error(ctx, err, sizeof err);
    fprintf(stderr, "FAIL %s: status %d (%s)\n", what, st, err);
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 3 || strlen(argv[1]) != 64) return 2;
    uint8_t key[32];
    for (int i = 0; i < 32; i++) key[i] = (uint8_t)(hexval(argv[1][2 * i]) << 4 | hexval(argv[1][2 * i + 1]));
    const uint32_t n = (uint32_t)(argc - 2);
    mk_needle* needles = calloc(n, sizeof *needles);
    char** texts = calloc(n, sizeof *texts);
    for (uint32_t k = 0; k < n; k++) {
        texts[k] = strdup(argv[2 + k]);
        char* c1 = strchr(texts[k], ':');
        char* c2 = c1 ? strchr(c1 + 1, ':') : NULL;
        if (!c2) return 2;
        *c1 = 0;
        needles[k].bytes = (const uint8_t*)texts[k];
        needles[k].len = (uint32_t)strlen(texts[k]);
        needles[k].fold = (uint32_t)atoi(c1 + 1);
        needles[k].mode = (uint32_t)atoi(c2 + 1);
    }
    mk_options opt;
    memset(&opt, 0, sizeof opt);
    opt.table_rows = 12;
    opt.keys_per_thread = 8;
    opt.block = 512;
    opt.self_check = 1;
    opt.hit_capacity = 1u << 18;
    mk_ctx* ctx = NULL;
    int st = mk_ctx_create(0, &opt, &ctx);
    if (st != MK_OK) return report(ctx, st, "mk_ctx_create");
    mk_info info;
    if ((st = mk_ctx_info(ctx, &info)) != MK_OK) return report(ctx, st, "mk_ctx_info");
    if (info.keys_per_iter < 65536) return report(ctx, -1, "one iteration covers fewer than 65536 indices");
    mk_job* job = NULL;
    if ((st = mk_job_prepare(ctx, key, MK_SEED_CHACHA20, needles, n, 0, &job)) != MK_OK)
        return report(ctx, st, "mk_job_prepare");
    int found = 0;
    uint64_t lowest = 0;
    if ((st = mk_job_launch(job, 0, 1, &found, &lowest)) != MK_OK) return report(ctx, st, "mk_job_launch");
    printf("launch %d %llu\n", found, (unsigned long long)lowest);
    uint32_t written = 0;
    uint64_t total = 0;
    if ((st = mk_job_hits(job, NULL, 0, &written, &total)) != MK_OK) return report(ctx, st, "mk_job_hits (count)");
    mk_hit* hits = calloc(total ? total : 1, sizeof *hits);
    if ((st = mk_job_hits(job, hits, (uint32_t)total, &written, &total)) != MK_OK)
        return report(ctx, st, "mk_job_hits");
    for (uint32_t k = 0; k < n; k++) {
        printf("hits %u", k);
        for (uint32_t i = 0; i < written; i++)
            if (hits[i].needle == k && hits[i].index < 65536) printf(" %llu", (unsigned long long)hits[i].index);
        printf("\n");
    }
    mk_outcome* out = calloc(n, sizeof *out);
    if ((st = mk_job_first_matches(job, out, n)) != MK_OK) return report(ctx, st, "mk_job_first_matches");
    for (uint32_t k = 0; k < n; k++) {
        printf("first %u %d %llu ", k, out[k].status, (unsigned long long)out[k].index);
        for (int i = 0; i < 32; i++) printf("%02x", out[k].pk[i]);
        printf("\n");
    }
    mk_job_destroy(job);
    mk_ctx_destroy(ctx);
    for (uint32_t k = 0; k < n; k++) free(texts[k]);
    free(texts);
    free(needles);
    free(hits);
    free(out);
    return 0;
}
