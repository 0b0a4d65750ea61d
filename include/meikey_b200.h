/*
 * meikey_b200 — C ABI of the B200 (sm_100a) candidate-key search backend.
 *
 * Drop-in boundary for meikey's GPU search backend: the calls below take the place
 * of the reference's `Engine` trait and `Kernel` (src/service/gpu.rs:806-887), which
 * the `Gpu` searcher (src/service/gpu.rs:1162-1327) drives from one host thread per
 * device.  All entry points return an `int` status (MK_OK = 0) and never abort the
 * process; the text of the last error of a context is kept in that context.
 * Plain pointers and sizes only: every buffer named "host" is ordinary host memory,
 * read or written only during the call.  A context, and the jobs, graphs and server made
 * from it, are used from one host thread at a time (as the reference drives one Gpu per
 * thread, src/service/search.rs:129-170); mk_job_stop is the exception and may be called
 * from another thread while a launch of the job runs.
 *
 * Seeds (src/model/search.rs:27-50, src/service/gpu.rs:1330-1351):
 *   MK_SEED_CHACHA20  seed(i) = 32-byte half (i & 1) of ChaCha20 block i >> 1
 *                     (RFC 8439 block function, 64-bit counter, stream 0), key = `key`
 *   MK_SEED_COUNTER   seed(i) = key with i added to its last 8 bytes (little-endian)
 * The public key of a seed is the Ed25519 public key: compress(clamp(SHA-512(seed)[0..32])·B).
 *   MK_SEED_INCREMENTAL  the low-security incremental path: `key` is a little-endian scalar
 *                     s0 below 2^255 (e.g. a clamped SHA-512 of one seed) and index i stands
 *                     for the scalar s0 + i itself, public key compress((s0 + i)·B), so
 *                     consecutive keys are consecutive points P_i = P_0 + i·B.  The reference
 *                     has no GPU kernel for it; the host confirms a hit from s0 + i.
 */
#ifndef MEIKEY_B200_H
#define MEIKEY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MK_ABI_VERSION 2

#if defined(__GNUC__)
#define MK_API __attribute__((visibility("default")))
#else
#define MK_API
#endif

/* Status codes.  1..8 mirror the reference's GpuError (src/service/gpu.rs:444-499);
 * the rest are states the reference reported by panicking or not at all. */
enum mk_status {
    MK_OK = 0,
    MK_ERR_DRIVER_NOT_FOUND = 1, /* GpuError::DriverNotFound */
    MK_ERR_NO_DEVICE = 2,        /* GpuError::NoDevice */
    MK_ERR_OUT_OF_RANGE = 3,     /* GpuError::OutOfRange: an option outside its range */
    MK_ERR_SELF_CHECK = 4,       /* GpuError::SelfCheck: GPU keys differ from the host derivation */
    MK_ERR_NO_SETTINGS = 5,      /* GpuError::NoSettings: autotuner had nothing to measure */
    MK_ERR_CUDA = 6,             /* GpuError::Driver: a CUDA runtime call failed */
    MK_ERR_NOT_BUILT = 7,        /* GpuError::NotEmbedded: no kernel variant for these options */
    MK_ERR_BAD_ARG = 8,          /* null pointer, bad mode, needle too long, ... */
    MK_ERR_OUT_OF_MEMORY = 9,
    MK_ERR_STOPPED = 10,         /* the launch ended early on the job's stop word */
    MK_ERR_HIT_RING_FULL = 11,   /* more hits than the hit ring holds; hits beyond it are counted only */
    MK_ERR_PATTERN = 12          /* pattern text rejected (src/model/pattern.rs:21-52) */
};

/* seed sources (SeedSource, src/model/search.rs:27-36) */
enum mk_seed_source { MK_SEED_CHACHA20 = 0, MK_SEED_COUNTER = 1, MK_SEED_INCREMENTAL = 2 };

/* match modes (kernel.cu MODE_CONTAINS / MODE_SUFFIX / MODE_REGEX, src/service/gpu.rs:610-616) */
enum mk_mode { MK_MODE_CONTAINS = 0, MK_MODE_SUFFIX = 1, MK_MODE_REGEX = 2 };

/* Kernel options (GpuOptions, src/service/gpu.rs:189-199).  Zero means "default".
 * table_rows chooses the comb geometry (rows of the fixed-base table: fewer rows
 * means fewer point additions per key and a larger table in HBM). */
typedef struct mk_options {
    uint32_t table_rows;      /* 10..63; default 12 (rows 10-20 are HBM tables of 26 GB down to 11 MB, 32-63 the
                                 comb windows of 8 down to 4 bits) */
    uint32_t keys_per_thread; /* keys one thread derives before the pooled inversion (default 16) */
    uint32_t block;           /* threads per CTA (default 512): 256 or 512, keys per thread 4, 8 or 16;
                                 see inverter_rotates for who inverts */
    uint32_t blocks_per_sm;   /* resident CTAs per SM the grid is sized for (0 = occupancy maximum) */
    uint32_t self_check;      /* 1: derive keys at creation and compare with the host derivation */
    uint32_t hit_capacity;    /* hit-ring entries per job (0 = 65536) */
    uint32_t hash_warps;      /* 4: search with hashing warps (block 512, keys per thread 8 or 16): 11 comb
                                 warps, 1 inverter, 4 warps computing the SHA-512 scalars, so that hashing
                                 overlaps the comb multiplies; ChaCha20 and counter seeds only.  0: off */
    uint32_t inverter_rotates;/* 0: a search CTA's last warp only inverts the CTA's products; 1: every warp
                                 derives keys and the inversion rotates over four warps, one per SM
                                 sub-partition (pays with long iterations: many needles).  Not with hash_warps */
    uint32_t inversion_batch; /* keys sharing one field inversion (the batch of Montgomery's trick, the
                                 reference's MEIKEY_BATCH x 4 pooled threads, kernel.cu:2024-2028):
                                 keys_per_thread x compute threads / pools, for pools a divisor of the
                                 compute threads (480; 512 with inverter_rotates; 352 with hash_warps) of
                                 at most 32, e.g. 256 = 8 x 480 / 15.  0: 32 pools (keys_per_thread x 15,
                                 x 16 with inverter_rotates, x 11 with hash_warps); else
                                 MK_ERR_OUT_OF_RANGE when no pool count gives it */
    uint32_t table_in_smem;   /* 1: every search CTA copies the comb table into shared memory and reads its
                                 entries there instead of gathering them from HBM (96 bytes an entry: about
                                 40+ rows, e.g. 42 rows of 6-bit digits, 133 KB; block 512, keys per thread
                                 4 or 8, the dedicated inverter; regex tables then stay in global memory).
                                 MK_ERR_OUT_OF_RANGE when the table does not fit */
    uint32_t hash_interleave; /* 1: each thread hashes the next iteration's seeds inside the current
                                 iteration's comb rows, 8 SHA-512 rounds per row, so that the hashing
                                 (ALU pipe) issues between the field multiplies (IMAD pipe) of one
                                 warp; 12 rows, block 512, keys per thread 8 or 16, the dedicated
                                 inverter, the table in HBM.  ChaCha20 and counter seeds (the
                                 incremental source hashes nothing) */
} mk_options;

/* One pattern as the reference's GPU needle (Needle, src/service/gpu.rs:618-660):
 * text needles are base64 characters (lowercase when fold = 1), 1..43 bytes;
 * regex needles are a DFA table of `len` states × 65 little-endian u16
 * (src/model/pattern/dfa.rs:189-200: state 0 accepts, state 1 starts, column 64
 * flags acceptance at the end of input). */
typedef struct mk_needle {
    const uint8_t* bytes;
    uint32_t len;
    uint32_t fold;
    uint32_t mode;
} mk_needle;

/* A candidate hit: its index and the needle it may match.  The GPU tests the
 * character that depends on the x sign with both values, so a hit is a
 * candidate that the host confirms (src/service/gpu.rs:973-996). */
typedef struct mk_hit {
    uint64_t index;
    uint32_t needle;
    uint32_t reserved;
} mk_hit;

typedef struct mk_info {
    int device;
    uint32_t sms;
    uint32_t grid;            /* CTAs per launch */
    uint32_t block;           /* threads per CTA */
    uint32_t keys_per_thread;
    uint32_t table_rows;
    uint64_t table_bytes;
    uint64_t keys_per_iter;   /* grid · (block - 32; block with inverter_rotates; 352 with hash_warps) · keys_per_thread */
    char name[96];
    uint32_t inversion_batch; /* keys sharing one field inversion */
    uint32_t table_in_smem;   /* 1: search CTAs read the comb table from shared memory */
} mk_info;

/* One candidate of the autotuner and what it measured. */
typedef struct mk_tune_entry {
    mk_options options;   /* the candidate (self_check is forced on) */
    int status;           /* MK_OK, or why it was dropped (MK_ERR_SELF_CHECK, MK_ERR_OUT_OF_RANGE, ...) */
    uint32_t stage;       /* the last stage it ran in: 1, or 2 for a finalist */
    double keys_per_s;    /* its best measured secure-path rate */
} mk_tune_entry;

/* mk_search: where and how long one job searches. */
typedef struct mk_search_config {
    uint64_t first;          /* first index */
    uint64_t max_tries;      /* indices to search before giving up (0 = no limit) */
    double time_limit_s;     /* wall-clock limit checked between launches (0 = none) */
    uint32_t iters;          /* iterations per launch (keys_per_iter each) */
    uint32_t reserved;
} mk_search_config;

/* The outcome of mk_search: a host-verified key, or why there is none. */
typedef struct mk_outcome {
    int status;              /* MK_OK: key found; MK_ERR_STOPPED: budget, time limit or cancel */
    uint32_t needle;         /* the needle the key matches */
    uint64_t index;          /* its index */
    uint64_t tries;          /* indices searched (Stats::tries) */
    double elapsed_s;        /* Stats::elapsed */
    uint8_t secret[32];      /* seed, or the scalar s0 + index of the incremental source */
    uint8_t pk[32];          /* public key */
} mk_outcome;

/* Progress callback between launches (Progress, src/service/search.rs:33-40); nonzero cancels. */
typedef int (*mk_progress_fn)(void* user, uint64_t tries, double elapsed_s);

/* Continuous-batching server options. */
typedef struct mk_server_options {
    uint32_t max_jobs;       /* jobs admitted at once (needle slots, 1..128) */
    uint32_t iters_per_tick; /* iterations per tick (one launch of iters_per_tick·keys_per_iter indices) */
    uint64_t budget;         /* indices a job searches from its admission before it is censored */
    uint64_t hit_capacity;   /* hit-ring entries the admitted jobs may plan for (0 = no limit) */
    uint64_t device_bytes;   /* device memory the admitted jobs may hold (0 = no limit): per job its
                                reserved hit-ring records (16 bytes each; four times its expected
                                candidates per tick, plus 64), its DFA table and 64 bytes of state */
} mk_server_options;

/* A finished job of the server. */
typedef struct mk_job_result {
    uint64_t id;             /* the caller's id */
    int status;              /* MK_OK found; MK_ERR_STOPPED censored at the budget */
    uint32_t reserved;
    uint64_t admit_index;    /* stream index at admission: the job searched [admit, admit + budget) */
    uint64_t index;          /* the key's index (found) */
    uint64_t tries;          /* indices searched for the job */
    double expected_tries;   /* the estimate used for admission */
    uint8_t secret[32];
    uint8_t pk[32];
} mk_job_result;

typedef struct mk_ctx mk_ctx;
typedef struct mk_job mk_job;
typedef struct mk_graph mk_graph;
typedef struct mk_server mk_server;

/* Library ABI version (MK_ABI_VERSION). */
MK_API uint32_t mk_abi_version(void);

/* Number of CUDA devices (src/service/gpu.rs:1229-1236 device_count); 0 without a driver. */
MK_API int mk_device_count(void);

/* Gpu::new / Kernel::load (src/service/gpu.rs:678-706, 1162-1216): builds the comb table
 * on the device and, with self_check, compares derived keys with the host derivation.
 * On failure *out may still hold a context: read its error with mk_last_error, then
 * release it with mk_ctx_destroy. */
MK_API int mk_ctx_create(int device, const mk_options* options, mk_ctx** out);
MK_API void mk_ctx_destroy(mk_ctx* ctx);
/* text of the context's last error ("" when none); copies at most size-1 bytes */
MK_API int mk_last_error(const mk_ctx* ctx, char* buf, size_t size);
MK_API int mk_ctx_info(const mk_ctx* ctx, mk_info* out);
/* Engine::keys_per_iter (src/service/gpu.rs:832-834) */
MK_API uint64_t mk_keys_per_iter(const mk_ctx* ctx);

/* Engine::prepare (src/service/gpu.rs:836-857).  Multiple needles are matched in one
 * pass; hits carry the needle's position in `needles`. */
MK_API int mk_job_prepare(mk_ctx* ctx, const uint8_t key[32], int seed_source, const mk_needle* needles,
                   uint32_t n_needles, int stop_on_hit, mk_job** out);
MK_API void mk_job_destroy(mk_job* job);

/* Engine::launch (src/service/gpu.rs:859-887): searches indices base .. base +
 * keys_per_iter·iters - 1, waits, and reports whether any candidate hit was found
 * (*found = 1, *index = the lowest hit index).  Hits are kept for mk_job_hits. */
MK_API int mk_job_launch(mk_job* job, uint64_t base, uint32_t iters, int* found, uint64_t* index);
/* Candidate hits of the last launch in increasing index order: writes min(cap, kept)
 * records and sets *written to that number; *total is every hit found, which exceeds the
 * number kept when the device ring overflowed (then MK_ERR_HIT_RING_FULL is returned). */
MK_API int mk_job_hits(mk_job* job, mk_hit* out, uint32_t cap, uint32_t* written, uint64_t* total);

/* Replaces the job's needles between launches (same rules as mk_job_prepare; waits for the
 * job's queued launches first).  Text needles are re-packed into the existing device copy
 * without allocating; regex needles get fresh device tables.  Hits of later launches carry
 * positions in the new array.  The reference rebuilds a Launch instead (gpu.rs:836-857). */
MK_API int mk_job_update(mk_job* job, const mk_needle* needles, uint32_t n_needles);

/* CUDA graph of `launches` consecutive search launches of `iters` iterations each (the job
 * word is reset once at the start; hits of all launches accumulate in the job's ring).
 * mk_graph_launch replays it over base .. base + launches·iters·keys_per_iter - 1, waits and
 * reports like mk_job_launch (hits through mk_job_hits); mk_graph_enqueue only queues it.
 * The reference launches each range from the host loop instead (gpu.rs:917-971). */
MK_API int mk_job_graph_create(mk_job* job, uint32_t iters, uint32_t launches, mk_graph** out);
MK_API int mk_graph_launch(mk_graph* graph, uint64_t base, int* found, uint64_t* index);
MK_API int mk_graph_enqueue(mk_graph* graph, uint64_t base);
MK_API void mk_graph_destroy(mk_graph* graph);

/* Requests (on = 1) or withdraws (on = 0) a stop of the job's launches: the word is written
 * from a separate stream, so it reaches a launch that is running; that launch ends within two
 * iterations per CTA and reports MK_ERR_STOPPED, with the hits found until then.  The request
 * stays set for later launches until withdrawn (the reference cancels between launches only,
 * src/service/search.rs:33-40). */
MK_API int mk_job_stop(mk_job* job, int on);

/* For each needle k < n: the lowest candidate of the last launch (or graph replay) that the
 * host confirms (mk_job_confirm, in index order), in out[k] (status MK_OK with index, key and
 * secret; MK_ERR_STOPPED when none of its candidates matches with the real x sign).  Needles
 * are confirmed on up to 16 host threads of the call's own (fewer, down to the calling thread
 * alone, when the host starts no more); it returns when all are done.  When the launch found
 * more candidates than the hit ring holds, the outcomes are those of the kept candidates, which
 * need not include a needle's lowest one, and MK_ERR_HIT_RING_FULL is returned (as by
 * mk_job_hits; launch fewer iterations or raise mk_options.hit_capacity). */
MK_API int mk_job_first_matches(mk_job* job, mk_outcome* out, uint32_t n);

/* Validates needles as mk_job_prepare would (host only, no device). */
MK_API int mk_needles_check(const mk_needle* needles, uint32_t n_needles);
/* keys_per_iter of the job's context */
MK_API uint64_t mk_job_keys_per_iter(const mk_job* job);

/* Expected number of indices to search until a key matches the needle (1 / the probability
 * that a uniformly random key matches, computed exactly by propagating a uniform character
 * distribution through the needle's DFA); INFINITY when it cannot match.  Host only. */
MK_API double mk_expected_tries(const mk_needle* needle);

/* Searcher::run for one job (src/service/search.rs:33-40 over gpu.rs:917-996): launches of
 * cfg->iters iterations over cfg->first, first + keys_per_iter·iters, ...; after each launch
 * its candidates are confirmed on the host in index order (mk_job_confirm) and the first
 * that matches with its real x sign is returned: the lowest matching index of the range.
 * Stops with status MK_ERR_STOPPED when max_tries indices are searched, the time limit passes
 * or `progress` returns nonzero (checked between launches, so a cancel takes effect within
 * one launch).  A launch whose candidates overflow the job's hit ring is run again over the
 * same start in launches of half the iterations; MK_ERR_HIT_RING_FULL is returned only when
 * a single iteration overflows it (raise mk_options.hit_capacity).  The return value is an
 * error of the engine, else MK_OK. */
MK_API int mk_search(mk_job* job, const mk_search_config* cfg, mk_progress_fn progress, void* user,
                     mk_outcome* out);

/* Searcher::run over several jobs at once (the reference's All, src/service/search.rs:107-180,
 * one searcher per device): one host thread per job runs mk_search's loop over cfgs[k] (each
 * job on a context of its own, on one device or several; MK_ERR_BAD_ARG when two jobs share a
 * context).  The first host-verified key sets every other job's stop word (mk_job_stop), so
 * their running launches end within two iterations and no new launch starts.  `progress` runs
 * on the calling thread about every 100 ms with the tries summed over the jobs, and a nonzero
 * return cancels all; cfgs[0].time_limit_s limits the whole call.  *out is the winner's
 * outcome with tries summed over every job (Stats of All: completed launches and the winner's
 * range up to its key) and *winner its position, or status MK_ERR_STOPPED and *winner = n when
 * no job found a key.  The stop requests are withdrawn before the call returns. */
MK_API int mk_search_many(mk_job* const* jobs, uint32_t n, const mk_search_config* cfgs, mk_progress_fn progress,
                          void* user, mk_outcome* out, uint32_t* winner);

/* The GPU and the host cores searching together (the reference's Both, src/service/search.rs:
 * 86-103): mk_search's loop of `job` over cfg on one host thread, and cpu_threads host threads
 * that derive keys of the same key stream from index cpu_first upward (chunks of 64
 * consecutive indices, the host derivation and a full match against every needle of the job),
 * the reference's CPU Parallel worker in scalar form.  Pick cpu_first away from the GPU's
 * range.  The first key found by either side stops the other (the job's stop word on the GPU
 * side); *winner is 0 for the GPU, 1 for the host cores, 2 when none (status MK_ERR_STOPPED,
 * after cfg->max_tries on the GPU side together with the time limit or a cancel from
 * `progress`, which runs on the calling thread about every 100 ms; the host cores search
 * until a key, the time limit or a cancel).  Tries are summed over both sides. */
MK_API int mk_search_both(mk_job* job, const mk_search_config* cfg, uint32_t cpu_threads, uint64_t cpu_first,
                          mk_progress_fn progress, void* user, mk_outcome* out, uint32_t* winner);

/* Continuous batching of many jobs over one candidate stream (no counterpart in the
 * reference): every mk_server_tick is one launch over the next iters_per_tick·keys_per_iter
 * indices of the stream (key, seed source) that tests the needles of all admitted jobs.
 * Submitted jobs wait in a queue and are admitted at tick boundaries, shortest expected
 * search first, while needle slots, the matcher's capacity, the hit-ring plan and the
 * device-memory budget allow.  A job admitted at stream index a searches [a, a + budget):
 * its result is the lowest index there whose key matches (confirmed on the host) and that
 * no other job has received: one index, so one secret, goes to one job only; of two jobs
 * matching the same key the one admitted earlier gets it.  That is the key mk_search finds
 * for the needle alone from first = a once the indices delivered before it (in the order
 * mk_server_results returns them) are skipped; otherwise the job is censored at the budget.
 * The server keeps a job of its own on the context; ticks are synchronous. */
MK_API int mk_server_create(mk_ctx* ctx, const uint8_t key[32], int seed_source, const mk_server_options* options,
                            uint64_t first, mk_server** out);
MK_API int mk_server_submit(mk_server* server, const mk_needle* needle, uint64_t id);
MK_API int mk_server_tick(mk_server* server, uint32_t* active, uint32_t* queued);
/* Drains finished jobs (in completion order): writes up to cap results, *n = the number written. */
MK_API int mk_server_results(mk_server* server, mk_job_result* out, uint32_t cap, uint32_t* n);
MK_API uint64_t mk_server_position(const mk_server* server);
MK_API void mk_server_destroy(mk_server* server);

/* The host confirmation of a candidate (src/service/gpu.rs:973-996, confirm): re-derives
 * index `index` of the job's key stream on the CPU — the seed and its Ed25519 public key, or
 * for MK_SEED_INCREMENTAL the scalar s0 + index and (s0 + index)·B — and tests needle
 * `needle` against the full key (x sign known).  Writes the public key and the secret (the
 * 32-byte seed, or the 32-byte little-endian scalar) and sets *matched to 1 when the key
 * matches; a candidate that only matched through the other x sign gives *matched = 0. */
MK_API int mk_job_confirm(mk_job* job, uint64_t index, uint32_t needle, uint8_t pk[32], uint8_t secret[32],
                          int* matched);

/* Asynchronous form: enqueue one launch on the context's stream without waiting
 * (mk_ctx_sync waits for all queued work); mk_job_collect waits and then reads the job word
 * and hit ring like mk_job_launch does (hits of the last enqueued launch). */
MK_API int mk_job_enqueue(mk_job* job, uint64_t base, uint32_t iters);
MK_API int mk_job_collect(mk_job* job, int* found, uint64_t* index);
MK_API int mk_ctx_sync(mk_ctx* ctx);
/* CUDA events on the context's stream: record into slot (0..15); elapsed ms between two slots */
MK_API int mk_ctx_record(mk_ctx* ctx, int slot);
MK_API int mk_ctx_elapsed(mk_ctx* ctx, int from_slot, int to_slot, float* ms);

/* meikey_derive (src/service/gpu/kernel.cu:2062-2069, src/service/gpu.rs:783-804):
 * n full public keys (x sign included) of indices first..first+n-1 into host `out` (32·n bytes). */
MK_API int mk_derive(mk_ctx* ctx, const uint8_t key[32], int seed_source, uint64_t first, uint64_t n, uint8_t* out);

/* mk_derive that allocates nothing.  This entry point has no counterpart in the reference.
 * It is for callers that must not allocate device memory while they run: a serving process
 * that gave the device's memory to the comb table and job slots at start-up, or a host
 * framework whose device memory belongs to its own pool; and cudaMalloc/cudaFree would also
 * synchronize the device and stall every other job sharing it.  The device staging for the
 * keys is a fixed 2 MiB array inside the library (held by every GPU that loads it until the
 * process exits), so n is limited to 65536 keys; larger n returns MK_ERR_OUT_OF_RANGE.
 * Seed sources MK_SEED_CHACHA20 and MK_SEED_COUNTER only: MK_SEED_INCREMENTAL returns
 * MK_ERR_BAD_ARG (use mk_derive).  The array's device address is looked up by mk_ctx_create,
 * with the context's device current, and kept in the context; a cudaDeviceReset of that device
 * invalidates it together with the context's other device memory, so create a new context
 * after one.  All calls share the array: calls that overlap on the GPU, from any thread or
 * context on the same device, race on it. */
MK_API int mk_derive_noalloc(mk_ctx* ctx, const uint8_t key[32], int seed_source, uint64_t first, uint64_t n,
                             uint8_t* out);

/* Dfa::new + Dfa::gpu_table with the checks of Pattern::regex (src/model/pattern/dfa.rs:52-108,
 * 189-200; src/model/pattern.rs:135-165): compiles a regex into the DFA table of a
 * MK_MODE_REGEX needle (states × 65 little-endian u16, state 0 accepts, state 1 starts,
 * column 64 flags acceptance at the end), for an unanchored search over the 43 characters
 * after the key prefix, which form the whole haystack.  The dialect is the reference's:
 * regex-syntax in ASCII mode (literals, `.`, classes with ranges, negation, nesting, POSIX
 * names and the && -- ~~ operations, \d \D \w \W \s \S, ^ $ \A \z \b \B \< \> \b{start}
 * \b{end} \b{start-half} \b{end-half}, punctuation / control / hex escapes, groups incl. named
 * ones, flag groups (?imsUuxR-...) and (?flags:...), `|`, * + ? {m} {m,} {m,n} and their lazy
 * forms); case_sensitive = 0 starts with the i flag set.  Unicode classes (\p, \P) and a
 * Unicode word boundary (\b under the u flag) are rejected, as is every escape outside the
 * dialect.  `table` must hold max_states·130 bytes (the reference's limit is 16384 states).
 * Returns MK_ERR_PATTERN (text in `err`) for an empty pattern, a syntax error, a pattern
 * that matches the empty string, one that no public key can match (e.g. `^Q`: the first
 * searched character is A-P) or more than max_states states.  Needs no device. */
MK_API int mk_regex_compile(const char* pattern, int case_sensitive, uint32_t max_states, uint8_t* table,
                            uint32_t* states, char* err, size_t err_size);

/* mk_regex_compile with the subset construction (the part of Dfa::new whose cost grows with
 * the DFA) on the context's GPU: the host parses the pattern and builds its NFA and each NFA
 * state's epsilon closures, then one CTA walks the DFA breadth first, resolving the successors
 * of a frontier's (state, value) pairs in parallel and numbering new states in the host's
 * order.  The table, state count, status and error text are those of mk_regex_compile for the
 * same arguments.  NFAs of up to 2048 states (MK_ERR_PATTERN beyond).  Runs on the context's
 * stream and waits for it. */
MK_API int mk_regex_compile_device(mk_ctx* ctx, const char* pattern, int case_sensitive, uint32_t max_states,
                                   uint8_t* table, uint32_t* states, char* err, size_t err_size);

/* Staged autotuner (GpuOptions::fastest_staged, src/service/gpu.rs:302-393, 1016-1113):
 * stage 1 creates a self-checked context per candidate (a variant whose keys differ from the
 * host derivation is dropped) and times one launch of about trial_keys secure-path
 * candidates; stage 2 re-times the `finalists` fastest in three rounds of alternating order.
 * Writes every entry's status, stage and rate, and the index of the fastest to *best.
 * MK_ERR_NO_SETTINGS when no candidate ran. */
MK_API int mk_autotune(int device, mk_tune_entry* entries, uint32_t n, uint32_t finalists, uint64_t trial_keys,
                       uint32_t* best);

/* mk_autotune timed on the caller's own job instead of the fixed secure-path one: the key,
 * seed source and needles of mk_job_prepare (the best options depend on the matching work;
 * inverter_rotates pays with many needles).  A candidate whose job cannot be prepared (e.g.
 * hash_warps with the incremental source) is dropped with that status. */
MK_API int mk_autotune_job(int device, mk_tune_entry* entries, uint32_t n, uint32_t finalists, uint64_t trial_keys,
                           const uint8_t key[32], int seed_source, const mk_needle* needles, uint32_t n_needles,
                           uint32_t* best);

/* Field multiplications per second on the context's device in radix 2^32 (the search
 * kernel's eight-limb field), radix 2^25.5 (ten limbs, 100 mad.wide products) and radix
 * 2^51 held in FP64 registers (five limbs, products split exactly by fused multiply-adds,
 * the reference's F51 limbs, src/service/gpu/kernel.cu:1318-1441), four independent chains
 * per thread at full occupancy: the measurement behind the choice of limb radix (the search
 * kernel is built for radix 2^32 only).  The radix-2^51 chains are also run against radix
 * 2^32 from the same inputs; MK_ERR_SELF_CHECK if any result differs. */
MK_API int mk_measure_field_mul(mk_ctx* ctx, double* radix32_per_s, double* radix26_per_s,
                                double* radix51_fp64_per_s);

/* Field multiplications per second of the two radix-2^32 forms, measured like
 * mk_measure_field_mul: the schoolbook product (64 mad.lo + 64 mad.hi) and one level of
 * Karatsuba on the 128-bit halves (48 + 48, plus about 60 adds and logic operations), which
 * the secure path's comb additions and batches use.  Both forms run the same chains;
 * MK_ERR_SELF_CHECK if any result differs. */
MK_API int mk_measure_field_mul_forms(mk_ctx* ctx, double* schoolbook_per_s, double* karatsuba_per_s);

/* OpenSSH output of a found key.  mk_openssh_public writes the authorized_keys line
 * "ssh-ed25519 <base64 blob>[ comment]" (VanityKey::public_openssh, src/model/key.rs:132-139);
 * mk_openssh_private writes the unencrypted openssh-key-v1 private key file of a seed
 * (private_openssh, src/repository/key_file.rs:276-320; checkint is the file's random check
 * word, a parameter so that tests can fix it).  Both write a NUL-terminated string, set
 * *written to its length (without the NUL) and return MK_ERR_BAD_ARG when `cap` is too small
 * or the comment holds a line break.  Host only; the private writer wipes its buffers. */
MK_API int mk_openssh_public(const uint8_t pk[32], const char* comment, char* out, size_t cap, size_t* written);
MK_API int mk_openssh_private(const uint8_t seed[32], const char* comment, uint32_t checkint, char* out, size_t cap,
                              size_t* written);

/* Comb table entry (row, column) as 24 words (y+x, y-x, 2dxy; row 0 holds 2xy), for tests. */
MK_API int mk_table_entry(mk_ctx* ctx, uint32_t row, uint64_t col, uint32_t out[24]);

/* Field products on the device, for tests: for i < n (at most 2^20), a[8i..8i+8) times
 * b[8i..8i+8) mod 2^255 - 19, little-endian 32-bit words of any value below 2^256, in the
 * schoolbook form into schoolbook[8i..] and in the Karatsuba form the secure path uses into
 * karatsuba[8i..].  The results are the kernels' own words: below 2^256, congruent to the
 * product, not reduced to canonical.  Allocates device memory and waits for the context's
 * stream. */
MK_API int mk_field_mul_pairs(mk_ctx* ctx, const uint32_t* a, const uint32_t* b, uint32_t n, uint32_t* schoolbook,
                              uint32_t* karatsuba);

/* Bytes the job has copied host->device and device->host so far (kernel parameters,
 * compiled needles, job state and hit records), for end-to-end accounting. */
MK_API int mk_job_io_bytes(const mk_job* job, uint64_t* h2d, uint64_t* d2h);

/* Field multiplications and 32-bit integer multiply-adds per key of the configured search
 * kernel for a seed source (the algorithmic count: comb additions, or the incremental
 * source's point additions, batch-inversion share, compression). */
MK_API int mk_ctx_work_per_key(const mk_ctx* ctx, int seed_source, double* field_muls, double* int_mads);

/* Measured peaks of 32-bit integer multiply-adds on the context's device, in MADs/s, each
 * the best of three bounded runs of 10-30 ms at full occupancy with no memory traffic:
 *   *chain_per_s  rows of a schoolbook product as the field multiply issues them
 *                 (mad.lo.cc/madc.lo.cc then madc.hi.cc carry chains, 8 lo + 8 hi per row);
 *                 the denominator of the int-MAD roofline;
 *   *lo_per_s     plain mad.lo.u32 on independent registers (the low-half multiply rate).
 * The reference reports no roofline. */
MK_API int mk_measure_mad_peaks(mk_ctx* ctx, double* chain_per_s, double* lo_per_s);

/* The pieces of that instruction shape, each on 8 independent chains per thread at full
 * occupancy (multiply-adds per second): independent mad.hi.u32, independent mad.wide.u32
 * (a full 64-bit product into a 64-bit sum), and rows of 8 madc.lo.cc or 8 madc.hi.cc linked
 * through the carry flag.  Together with mk_measure_mad_peaks they separate the issue cost of
 * the high halves from the serialisation of the carry chains. */
MK_API int mk_measure_imad_rates(mk_ctx* ctx, double* hi_per_s, double* wide_per_s, double* lo_chain_per_s,
                                 double* hi_chain_per_s);

#ifdef __cplusplus
}
#endif

#endif /* MEIKEY_B200_H */
