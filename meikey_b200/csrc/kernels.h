// Launch interface between the host runtime (api.cpp) and the kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "types.h"

namespace mkb {

struct KeyLaunch {
    const uint4* table;
    CombGeom geom;
    uint32_t key[8];
    uint32_t seed_src;     // 0 ChaCha20, 1 counter
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
};

cudaError_t launch_keys(const KeyLaunch& L, bool derive, uint32_t kpt, uint32_t block, uint32_t grid, cudaStream_t st);
cudaError_t keys_occupancy(bool derive, uint32_t kpt, uint32_t block, int* blocks_per_sm);
cudaError_t measure_imad(int sms, cudaStream_t st, double* mads_per_s);

// Largest n of mk_derive_noalloc and the device address of its fixed staging array on
// `device` (looked up once per device; the device must be current).
constexpr uint64_t NOALLOC_MAX_KEYS = 1ull << 16;
cudaError_t noalloc_staging(int device, uint8_t** ptr);
cudaError_t launch_build_table(uint4* table, const CombGeom& g, const uint32_t* points, uint64_t first,
                               uint64_t count, cudaStream_t st);

}  // namespace mkb
