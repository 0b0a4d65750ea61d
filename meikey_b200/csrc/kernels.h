// Launch interface between the host runtime (api.cpp) and the kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "types.h"

namespace mkre {
struct NfaTables;
}

namespace mkb {

struct KeyLaunch {
    const uint4* table;
    CombGeom geom;
    uint32_t key[8];
    uint32_t seed_src;     // 0 ChaCha20, 1 counter, 2 incremental
    uint32_t iters;
    uint64_t base;
    // search
    const MatchSet* match; // device copy
    HitRecord* hits;
    uint32_t hit_cap;
    uint32_t stop_on_hit;
    JobDevice* job;
    uint32_t* sink;
    // derive
    uint8_t* out;
    uint64_t count;
    // incremental source: index base + i stands for the point (s0 + base + i)·B
    const uint4* incr;     // INCR_WINDOWS·16 entries j·16^w·B, then INCR_STEPS entries j·B (table form)
    uint32_t start[32];    // (s0 + base)·B as x, y, 1, xy
    uint32_t delta[24];    // keys_per_iter·B: one search thread's jump between iterations
    // bytes of shared memory for the job's DFA tables (each 16-byte aligned; 0: read them
    // from global memory)
    uint32_t dfa_smem;
    // division of work inside a search CTA (LAYOUT_*)
    uint32_t layout;
    // field inversions per CTA and iteration (0: 32, one per lane of the inverting warp): each
    // pools the products of compute threads / inv_pools threads; a divisor of the compute
    // threads, at most 32
    uint32_t inv_pools;
    // bytes of the comb table in shared memory (search kernels; 0: gathered from HBM): every CTA
    // copies the table there at the start, entries 96 bytes apart
    uint32_t table_smem;
};

// LAYOUT_INVERTER_WARP: the last warp inverts, the others compute keys; LAYOUT_ROTATING: every
// warp computes keys and the inversion rotates over four warps; LAYOUT_INTERLEAVED: as
// LAYOUT_INVERTER_WARP, with each iteration's SHA-512 of the next iteration's seeds inside the
// comb rows (12 rows); LAYOUT_HASH_WARPS: 11 comb warps, 1 inverter, 4 hashing warps
// (k_search_hw; ChaCha20 / counter seeds)
constexpr uint32_t LAYOUT_INVERTER_WARP = 0, LAYOUT_ROTATING = 1, LAYOUT_INTERLEAVED = 2, LAYOUT_HASH_WARPS = 4;

// compute threads of a search CTA
inline uint32_t search_threads(uint32_t block, uint32_t layout) {
    return layout == LAYOUT_HASH_WARPS ? 352u : layout == LAYOUT_ROTATING ? block : block - 32u;
}

constexpr uint32_t DFA_SMEM_MAX = 48u * 1024u;

constexpr uint32_t SEED_INCREMENTAL = 2;
constexpr int INCR_WINDOWS = 8;   // 4-bit windows of a thread's offset (offsets below 2^32)
constexpr int INCR_STEPS = 16;    // j·B for j = 0 .. keys per thread - 1
constexpr int INCR_ENTRIES = INCR_WINDOWS * 16 + INCR_STEPS;

cudaError_t launch_keys(const KeyLaunch& L, bool derive, uint32_t kpt, uint32_t block, uint32_t grid, cudaStream_t st);
// Field multiplications per second in radix 2^32 (the search kernel's), radix 2^25.5 and
// radix 2^51 in FP64; *radix51_exact tells whether radix-2^51 chains matched radix 2^32.
cudaError_t measure_field_mul_rates(int sms, cudaStream_t st, double* radix32_per_s, double* radix26_per_s,
                                    double* radix51_per_s, bool* radix51_exact);
// Subset construction of a regex DFA on the device (dfa_build.cu) from the pattern's NFA
// tables: the table of mk_regex_compile (states x 65 u16, row 0 the accept state) in *table
// and its state count in *states, or *too_many when it has more than max_states states.
// Synchronizes `st`.  NFAs of up to 32·MAX_DFA_NFA_WORDS states.
constexpr uint32_t MAX_DFA_NFA_WORDS = 64;
cudaError_t build_dfa_device(const mkre::NfaTables& t, uint32_t max_states, cudaStream_t st,
                             std::vector<uint8_t>* table, uint32_t* states, bool* too_many);
// Field multiplications per second of the schoolbook and Karatsuba radix-2^32 forms;
// *same_words tells whether their chains ended in the same words.
cudaError_t measure_field_mul_forms(int sms, cudaStream_t st, double* schoolbook_per_s, double* karatsuba_per_s,
                                    bool* same_words);
// a[i]·b[i] mod p (8 words each, below 2^256) in the schoolbook and Karatsuba forms, for tests;
// synchronizes `st`.
cudaError_t field_mul_pairs(const uint32_t* a, const uint32_t* b, uint32_t n, uint32_t* out_s, uint32_t* out_k,
                            cudaStream_t st);
// Integer multiply-adds of one radix-2^32 field multiplication in each form (products and the
// fold by 38) and of a squaring; the secure path multiplies in the Karatsuba form.
constexpr double MADS_MUL_SCHOOLBOOK = 64 + 64 + 16;
constexpr double MADS_MUL_KARATSUBA = 48 + 48 + 16;
constexpr double MADS_SQUARE = 72 + 16;
// The kernel of a variant and its dynamic shared memory (for graph nodes); sets the
// kernel's shared-memory limit like launch_keys does.
cudaError_t keys_kernel(bool derive, bool incr, uint32_t kpt, uint32_t block, uint32_t layout, uint32_t dfa_smem,
                        uint32_t table_smem, const void** func, size_t* dyn);
cudaError_t keys_occupancy(bool derive, bool incr, uint32_t kpt, uint32_t block, uint32_t layout, uint32_t table_smem,
                           int* blocks_per_sm);
// multiply-adds per second of the carry-chain row microbenchmark and of plain mad.lo.u32
cudaError_t measure_mad_peaks(int sms, cudaStream_t st, double* chain_per_s, double* lo_per_s);
// multiply-adds per second of independent mad.hi.u32, independent mad.wide.u32, and rows of
// 8 madc.lo.cc / 8 madc.hi.cc linked through the carry flag
cudaError_t measure_imad_rates(int sms, cudaStream_t st, double rates[4]);

// Largest n of mk_derive_noalloc and the device address of its fixed staging array on the
// current device (looked up when a context is created).
constexpr uint64_t NOALLOC_MAX_KEYS = 1ull << 16;
cudaError_t noalloc_staging(uint8_t** ptr);
cudaError_t launch_build_table(uint4* table, const CombGeom& g, const uint32_t* points, uint64_t first,
                               uint64_t count, cudaStream_t st);

}  // namespace mkb
