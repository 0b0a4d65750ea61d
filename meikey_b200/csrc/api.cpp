// C ABI of the B200 search backend (include/meikey_b200.h).
//
// The context owns the device, its stream and the comb table; a job owns the key,
// the compiled needles and its hit ring.  Every entry point returns a status and
// records the text of a failure in the context (no exceptions cross the ABI).
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <thread>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/meikey_b200.h"
#include "abi_guard.h"
#include "hitsort.h"
#include "host25519.h"
#include "jobs.h"
#include "kernels.h"
#include "regex.h"

using mkb::CombGeom;

struct mk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;     // stop requests, written while a launch runs on `stream`
    cudaMemPool_t pool = nullptr;    // job buffers (stream-ordered, kept across jobs)
    std::vector<mkhits::HitBuf> spare_hits;  // host hit buffers of released jobs
    cudaEvent_t ev[16] = {};
    mk_info info{};
    CombGeom geom{};
    uint4* table = nullptr;
    uint4* incr = nullptr;           // incremental source: window table then step table
    uint32_t delta[24] = {};         // keys_per_iter·B (table form)
    uint32_t kpt = 8, block = 256, grid = 0;
    uint32_t hash_warps = 0;  // 4: search kernel with hashing warps (ChaCha20 / counter seeds)
    uint32_t layout = mkb::LAYOUT_INVERTER_WARP;  // division of work inside a search CTA
    uint32_t inv_pools = 32;  // field inversions per search CTA and iteration
    uint32_t table_smem = 0;  // bytes of the comb table each search CTA keeps in shared memory (0: HBM)
    uint32_t hit_capacity = 1u << 16;
    uint8_t* noalloc = nullptr;  // device address of mk_derive_noalloc's fixed staging array
    std::string err;
};

struct mk_job {
    mk_ctx* ctx = nullptr;
    uint8_t key[32];
    int source = 0;
    int stop_on_hit = 0;
    std::vector<mkh25519::Needle> needles;
    mkb::MatchSet* d_match = nullptr;
    std::vector<uint8_t*> d_dfa;
    uint32_t* d_gram4 = nullptr;  // 4-gram prefilter bitmap (2 MB), allocated on first use
    mkb::HitRecord* d_hits = nullptr;
    uint32_t cap = 1u << 16;
    mkb::JobDevice* d_job = nullptr;
    uint32_t* d_sink = nullptr;
    mkhits::HitBuf last;     // hits of the last launch (ordered only when `sorted`)
    bool sorted = true;
    uint32_t last_total = 0;
    uint64_t h2d = 0, d2h = 0;  // bytes copied for this job
};

struct mk_graph {
    mk_job* job = nullptr;
    uint32_t iters = 0;
    uint64_t span = 0;  // keys of one launch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphNode_t> nodes;
    std::vector<mkb::KeyLaunch> params;
    const void* func = nullptr;
    size_t dyn = 0;
};

namespace {

// Job buffers come from the context's stream-ordered pool.  A released job's memory stays in
// the pool for the next job, so making and releasing a job neither maps nor unmaps device
// memory; cudaFree synchronizes the whole device and took tens of milliseconds per job.
// An allocation is ordered on the context's stream: callers synchronize that stream before
// another stream or a blocking copy touches the buffer.
template <class T>
bool pool_alloc(mk_ctx* c, T** p, size_t bytes) {
    void* q = nullptr;
    if (cudaMallocFromPoolAsync(&q, bytes, c->pool, c->stream) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return false;
    }
    *p = (T*)q;
    return true;
}

void pool_free(mk_ctx* c, void* p) {
    if (p) cudaFreeAsync(p, c->stream);
}

int fail(mk_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(mk_ctx* c, cudaError_t e, const char* what) {
    return fail(c, MK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define MK_CUDA(ctx, call)                                     \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

const char B64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

int b64_value(uint8_t c) {
    const char* p = c ? strchr(B64, c) : nullptr;
    return p ? (int)(p - B64) : -1;
}

// Comb geometry for `rows` rows: rows-1 signed rows of width w or w+1 and a top row
// of the remaining bits, chosen to minimise the number of entries.
bool make_geometry(uint32_t rows, CombGeom& g) {
    if (rows < 3 || rows > (uint32_t)mkb::MAX_ROWS) return false;
    const uint32_t n = rows - 1;
    double best = 1e300;
    uint32_t bw = 0, ba = 0, bt = 0;
    for (uint32_t w = 2; w <= 27; w++)
        for (uint32_t a = 0; a < n; a++) {
            uint32_t used = n * w + a;
            if (used >= 251) continue;
            uint32_t t = 251 - used;
            if (t > 27) continue;
            double entries = (double)a * ((1u << w) + 1) + (double)(n - a) * ((1u << (w - 1)) + 1) + (double)(1u << t) + 1;
            if (entries < best) {
                best = entries;
                bw = w;
                ba = a;
                bt = t;
            }
        }
    if (!bw) return false;
    memset(&g, 0, sizeof g);
    g.rows = rows;
    uint32_t off = 0;
    uint64_t base = 0;
    for (uint32_t i = 0; i < rows; i++) {
        uint32_t w = i + 1 == rows ? bt : (i < ba ? bw + 1 : bw);
        g.width[i] = w;
        g.offset[i] = off;
        g.row_base[i] = base;
        g.cols[i] = i + 1 == rows ? (1ull << w) + 1 : (1ull << (w - 1)) + 1;
        off += w;
        base += g.cols[i];
    }
    g.entries = base;
    return off == 251;
}

// Public key of index `index` of a job's key stream on the host (the confirmation path).
bool host_public_key(const uint8_t key[32], int source, uint64_t index, uint8_t pk[32]) {
    if (source == MK_SEED_INCREMENTAL) {
        uint8_t s[32];
        if (!mkh25519::incremental_scalar(key, index, s)) return false;
        mkh25519::scalar_public_key(s, pk);
        return true;
    }
    uint8_t seed[32];
    mkh25519::seed_of(key, source, index, seed);
    mkh25519::public_key(seed, pk);
    return true;
}

// KeyLaunch fields of the incremental source for a launch starting at index `base`.
void set_incremental(const mk_ctx* c, const uint8_t s0[32], uint64_t base, mkb::KeyLaunch& L) {
    uint8_t s[32];
    mkh25519::incremental_scalar(s0, base, s);
    mkh25519::scalar_point_words(s, L.start);
    memcpy(L.delta, c->delta, sizeof L.delta);
    L.incr = c->incr;
}

int self_check(mk_ctx* c) {
    // every seed source, an odd first index (seed from the second half of a block)
    const uint64_t n = 257;
    std::vector<uint8_t> got(32 * n);
    for (int src = 0; src < 3; src++) {
        uint8_t key[32];
        for (int i = 0; i < 32; i++) key[i] = (uint8_t)(0x5a ^ (i * 37 + src * 101));
        key[31] &= 0x7f;  // incremental scalars start below 2^255
        uint64_t first = 0x123456789abull | 1;
        int st = mk_derive(c, key, src, first, n, got.data());
        if (st) return st;
        for (uint64_t i = 0; i < n; i += (i < 8 ? 1 : 31)) {
            uint8_t pk[32];
            host_public_key(key, src, first + i, pk);
            if (memcmp(pk, &got[32 * i], 32) != 0)
                return fail(c, MK_ERR_SELF_CHECK, "GPU public keys differ from the host derivation");
        }
    }
    return MK_OK;
}

}  // namespace

namespace mkjobs {

mk_ctx* context_of(const mk_job* job) { return job ? job->ctx : nullptr; }

int host_match(const mk_job* j, uint64_t index, uint8_t pk[32], uint8_t secret[32], uint32_t* needle) {
    if (j->source == MK_SEED_INCREMENTAL) {
        if (!mkh25519::incremental_scalar(j->key, index, secret)) return -1;
        mkh25519::scalar_public_key(secret, pk);
    } else {
        mkh25519::seed_of(j->key, j->source, index, secret);
        mkh25519::public_key(secret, pk);
    }
    for (uint32_t k = 0; k < j->needles.size(); k++)
        if (mkh25519::matches(j->needles[k], pk)) {
            *needle = k;
            return 1;
        }
    return 0;
}

}  // namespace mkjobs

extern "C" {

uint32_t mk_abi_version(void) { return MK_ABI_VERSION; }

int mk_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int mk_last_error(const mk_ctx* ctx, char* buf, size_t size) {
    if (!buf || size == 0) return MK_ERR_BAD_ARG;
    const char* s = ctx ? ctx->err.c_str() : "";
    snprintf(buf, size, "%s", s);
    return MK_OK;
}

int mk_ctx_create(int device, const mk_options* options, mk_ctx** out) try {
    if (!out) return MK_ERR_BAD_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorInsufficientDriver || e == cudaErrorNoDevice) return e == cudaErrorNoDevice ? MK_ERR_NO_DEVICE : MK_ERR_DRIVER_NOT_FOUND;
    if (e != cudaSuccess) return MK_ERR_DRIVER_NOT_FOUND;
    if (device < 0 || device >= n) return MK_ERR_NO_DEVICE;
    mk_options o{};
    if (options) o = *options;
    if (!o.table_rows) o.table_rows = 12;
    if (!o.keys_per_thread) o.keys_per_thread = 16;
    if (!o.block) o.block = 512;
    const bool built = (o.block == 256 && (o.keys_per_thread == 4 || o.keys_per_thread == 8 || o.keys_per_thread == 16)) ||
                       (o.block == 512 && (o.keys_per_thread == 4 || o.keys_per_thread == 8 || o.keys_per_thread == 16));
    // the shared-memory table: built for the dedicated-inverter layout, block 512, 4 or 8 keys per thread
    const bool smem_ok = o.table_in_smem == 0 ||
                         (o.table_in_smem == 1 && o.block == 512 && (o.keys_per_thread == 4 || o.keys_per_thread == 8) &&
                          !o.hash_warps && !o.inverter_rotates);
    // hashing inside the comb rows: 12 rows (10 full rows carry the 80 rounds), block 512, 8 or 16
    // keys per thread, the dedicated inverter, the table in HBM
    const bool shai_ok = o.hash_interleave == 0 ||
                         (o.hash_interleave == 1 && o.table_rows == 12 && o.block == 512 &&
                          (o.keys_per_thread == 8 || o.keys_per_thread == 16) && !o.hash_warps &&
                          !o.inverter_rotates && !o.table_in_smem);
    const bool hw_ok = o.hash_warps == 0 || (o.hash_warps == 4 && o.block == 512 && (o.keys_per_thread == 8 || o.keys_per_thread == 16));
    const bool rot_ok = o.inverter_rotates <= 1 && !(o.inverter_rotates && o.hash_warps);
    if (o.table_rows < 10 || o.table_rows > (uint32_t)mkb::MAX_ROWS - 1 || !built || !hw_ok || !rot_ok || !smem_ok || !shai_ok ||
        o.blocks_per_sm > 16 || o.hit_capacity > (1u << 26))
        return MK_ERR_OUT_OF_RANGE;
    // inversion batch: keys per field inversion = keys per thread x compute threads / pools, with
    // the pools a divisor of the compute threads and at most 32 (one per lane of the inverting warp)
    const uint32_t layout = o.hash_warps         ? mkb::LAYOUT_HASH_WARPS
                            : o.inverter_rotates ? mkb::LAYOUT_ROTATING
                            : o.hash_interleave  ? mkb::LAYOUT_INTERLEAVED
                                                 : mkb::LAYOUT_INVERTER_WARP;
    const uint32_t ct = mkb::search_threads(o.block, layout);
    uint32_t pools = 32;
    if (o.inversion_batch) {
        const uint64_t keys = (uint64_t)ct * o.keys_per_thread;
        if (keys % o.inversion_batch) return MK_ERR_OUT_OF_RANGE;
        pools = (uint32_t)(keys / o.inversion_batch);
        if (pools == 0 || pools > 32 || ct % pools) return MK_ERR_OUT_OF_RANGE;
    } else if (ct % 32) {
        return MK_ERR_OUT_OF_RANGE;
    }
    mk_ctx* c = new (std::nothrow) mk_ctx;
    if (!c) return MK_ERR_OUT_OF_MEMORY;
    *out = c;
    c->device = device;
    c->kpt = o.keys_per_thread;
    c->block = o.block;
    c->hash_warps = o.hash_warps;
    c->layout = layout;
    c->inv_pools = pools;
    if (o.hit_capacity) c->hit_capacity = o.hit_capacity;
    MK_CUDA(c, cudaSetDevice(device));
    MK_CUDA(c, mkb::noalloc_staging(&c->noalloc));
    MK_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    MK_CUDA(c, cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    {
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        MK_CUDA(c, cudaMemPoolCreate(&c->pool, &pp));
        uint64_t keep = ~0ull;  // freed blocks stay in the pool until the context goes
        MK_CUDA(c, cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    for (auto& ev : c->ev) MK_CUDA(c, cudaEventCreate(&ev));
    cudaDeviceProp prop;
    MK_CUDA(c, cudaGetDeviceProperties(&prop, device));
    if (!make_geometry(o.table_rows, c->geom)) return fail(c, MK_ERR_OUT_OF_RANGE, "no comb geometry for this row count");
    if (o.table_in_smem) {
        const uint64_t bytes = c->geom.entries * (uint64_t)mkb::ENTRY_WORDS * 4;  // 96 bytes per entry
        if (bytes > (uint64_t)prop.sharedMemPerBlockOptin)
            return fail(c, MK_ERR_OUT_OF_RANGE, "the comb table does not fit in shared memory (use more rows)");
        c->table_smem = (uint32_t)bytes;
    }
    int occ = 0;
    cudaError_t oe = mkb::keys_occupancy(false, false, c->kpt, c->block, c->layout, c->table_smem, &occ);
    if (oe != cudaSuccess && c->table_smem) {
        cudaGetLastError();
        return fail(c, MK_ERR_OUT_OF_RANGE, "the comb table and the CTA's buffers do not fit in shared memory");
    }
    MK_CUDA(c, oe);
    if (occ < 1) return fail(c, MK_ERR_NOT_BUILT, "kernel does not fit on this device");
    uint32_t per_sm = o.blocks_per_sm ? std::min<uint32_t>(o.blocks_per_sm, (uint32_t)occ) : (uint32_t)occ;
    c->grid = (uint32_t)prop.multiProcessorCount * per_sm;
    // table
    size_t bytes = (size_t)c->geom.entries * mkb::COMB_STRIDE_WORDS * 4;
    e = cudaMalloc(&c->table, bytes);
    if (e != cudaSuccess) {
        c->table = nullptr;
        return fail(c, MK_ERR_OUT_OF_MEMORY, "comb table allocation failed");
    }
    std::vector<uint32_t> pts = mkh25519::comb_points(c->geom.rows, c->geom.offset);
    uint32_t* d_pts = nullptr;
    MK_CUDA(c, cudaMalloc(&d_pts, pts.size() * 4));
    MK_CUDA(c, cudaMemcpyAsync(d_pts, pts.data(), pts.size() * 4, cudaMemcpyHostToDevice, c->stream));
    const uint64_t chunk = 1ull << 22;
    for (uint64_t f = 0; f < c->geom.entries; f += chunk) {
        uint64_t cnt = std::min<uint64_t>(chunk, c->geom.entries - f);
        MK_CUDA(c, mkb::launch_build_table(c->table, c->geom, d_pts, f, cnt, c->stream));
    }
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_pts);
    // incremental source: j·16^w·B (w < 8, j < 16), then j·B (j < 16), in the table form
    {
        std::vector<uint32_t> words((size_t)mkb::INCR_ENTRIES * mkb::ENTRY_WORDS);
        for (int w = 0; w < mkb::INCR_WINDOWS; w++)
            for (int j = 0; j < 16; j++)
                mkh25519::niels_of_multiple((uint64_t)j << (4 * w), &words[(size_t)(w * 16 + j) * mkb::ENTRY_WORDS]);
        for (int j = 0; j < mkb::INCR_STEPS; j++)
            mkh25519::niels_of_multiple((uint64_t)j,
                                        &words[(size_t)(mkb::INCR_WINDOWS * 16 + j) * mkb::ENTRY_WORDS]);
        if (cudaMalloc(&c->incr, words.size() * 4) != cudaSuccess) {
            c->incr = nullptr;
            return fail(c, MK_ERR_OUT_OF_MEMORY, "incremental table allocation failed");
        }
        MK_CUDA(c, cudaMemcpy(c->incr, words.data(), words.size() * 4, cudaMemcpyHostToDevice));
        mkh25519::niels_of_multiple((uint64_t)c->grid * mkb::search_threads(c->block, c->layout) * c->kpt, c->delta);
    }
    // info
    mk_info& in = c->info;
    in.device = device;
    in.sms = (uint32_t)prop.multiProcessorCount;
    in.grid = c->grid;
    in.block = c->block;
    in.keys_per_thread = c->kpt;
    in.table_rows = c->geom.rows;
    in.table_bytes = bytes;
    // the threads of a search CTA that derive keys (all but a dedicated inverter warp, unless the
    // inversion rotates; 352 comb threads with hashing warps)
    in.keys_per_iter = (uint64_t)c->grid * mkb::search_threads(c->block, c->layout) * c->kpt;
    in.inversion_batch = mkb::search_threads(c->block, c->layout) * c->kpt / c->inv_pools;
    in.table_in_smem = c->table_smem ? 1 : 0;
    snprintf(in.name, sizeof in.name, "%.95s", prop.name);
    if (o.self_check) {
        int st = self_check(c);
        if (st) return st;
    }
    return MK_OK;
} MK_ABI_CATCH(out && *out ? &(*out)->err : nullptr)

void mk_ctx_destroy(mk_ctx* c) try {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->table) cudaFree(c->table);
    if (c->incr) cudaFree(c->incr);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->pool) cudaMemPoolDestroy(c->pool);
    delete c;
} MK_ABI_CATCH_VOID

int mk_ctx_info(const mk_ctx* c, mk_info* out) {
    if (!c || !out) return MK_ERR_BAD_ARG;
    *out = c->info;
    return MK_OK;
}

uint64_t mk_keys_per_iter(const mk_ctx* c) { return c ? c->info.keys_per_iter : 0; }

// Sources 0..2; the incremental source takes a scalar below 2^255 as its key.
static int check_source(mk_ctx* c, const uint8_t key[32], int seed_source) {
    if (seed_source < MK_SEED_CHACHA20 || seed_source > MK_SEED_INCREMENTAL) return fail(c, MK_ERR_BAD_ARG, "unknown seed source");
    if (seed_source == MK_SEED_INCREMENTAL && (key[31] & 0x80))
        return fail(c, MK_ERR_BAD_ARG, "incremental start scalar must be below 2^255");
    return MK_OK;
}

int mk_derive(mk_ctx* c, const uint8_t key[32], int seed_source, uint64_t first, uint64_t n, uint8_t* out) try {
    if (!c || !key || (!out && n)) return fail(c, MK_ERR_BAD_ARG, "bad argument");
    if (int st = check_source(c, key, seed_source)) return st;
    if (seed_source == MK_SEED_INCREMENTAL && n != 0 && n - 1 > ~0ull - first)  // last index first + n - 1
        return fail(c, MK_ERR_OUT_OF_RANGE, "incremental indices must not wrap past 2^64");
    if (n == 0) return MK_OK;
    MK_CUDA(c, cudaSetDevice(c->device));
    const uint64_t per_launch = 1ull << 22;
    uint8_t* d_out = nullptr;
    uint64_t cap = std::min(n, per_launch);
    MK_CUDA(c, cudaMalloc(&d_out, cap * 32));
    for (uint64_t done = 0; done < n; done += per_launch) {
        uint64_t cnt = std::min(per_launch, n - done);
        mkb::KeyLaunch L{};
        L.table = c->table;
        L.geom = c->geom;
        for (int i = 0; i < 8; i++) L.key[i] = (uint32_t)key[4 * i] | (uint32_t)key[4 * i + 1] << 8 | (uint32_t)key[4 * i + 2] << 16 | (uint32_t)key[4 * i + 3] << 24;
        L.seed_src = (uint32_t)seed_source;
        L.iters = 1;
        L.base = first + done;
        L.out = d_out;
        L.count = cnt;
        if (seed_source == MK_SEED_INCREMENTAL) set_incremental(c, key, L.base, L);
        uint64_t threads = (cnt + c->kpt - 1) / c->kpt;
        uint32_t grid = (uint32_t)((threads + c->block - 1) / c->block);
        cudaError_t e = mkb::launch_keys(L, true, c->kpt, c->block, grid, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out + 32 * done, d_out, cnt * 32, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            cudaFree(d_out);
            return cuda_fail(c, e, "derive");
        }
    }
    cudaFree(d_out);
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

// Same keys as mk_derive, with the device output staged in the library's fixed device
// array instead of a cudaMalloc'd buffer: this call allocates nothing.  Every slot of the
// staging that is copied back is written by the kernel first, so nothing has to be cleared.
int mk_derive_noalloc(mk_ctx* c, const uint8_t key[32], int seed_source, uint64_t first, uint64_t n, uint8_t* out) try {
    if (!c || !key || (!out && n)) return fail(c, MK_ERR_BAD_ARG, "bad argument");
    if (seed_source != MK_SEED_CHACHA20 && seed_source != MK_SEED_COUNTER)
        return fail(c, MK_ERR_BAD_ARG, "mk_derive_noalloc: ChaCha20 and counter seeds only (use mk_derive)");
    if (n > mkb::NOALLOC_MAX_KEYS)
        return fail(c, MK_ERR_OUT_OF_RANGE, "mk_derive_noalloc: n exceeds the fixed staging of 65536 keys");
    if (n == 0) return MK_OK;
    MK_CUDA(c, cudaSetDevice(c->device));
    uint8_t* staging = c->noalloc;
    mkb::KeyLaunch L{};
    L.table = c->table;
    L.geom = c->geom;
    for (int i = 0; i < 8; i++)
        L.key[i] = (uint32_t)key[4 * i] | (uint32_t)key[4 * i + 1] << 8 | (uint32_t)key[4 * i + 2] << 16 | (uint32_t)key[4 * i + 3] << 24;
    L.seed_src = (uint32_t)seed_source;
    L.iters = 1;
    L.base = first;
    L.out = staging;
    L.count = n;
    uint64_t threads = (n + c->kpt - 1) / c->kpt;
    uint32_t grid = (uint32_t)((threads + c->block - 1) / c->block);
    MK_CUDA(c, mkb::launch_keys(L, true, c->kpt, c->block, grid, c->stream));
    MK_CUDA(c, cudaMemcpyAsync(out, staging, n * 32, cudaMemcpyDeviceToHost, c->stream));
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_table_entry(mk_ctx* c, uint32_t row, uint64_t col, uint32_t out[24]) {
    if (!c || !out || row >= c->geom.rows || col >= c->geom.cols[row]) return fail(c, MK_ERR_BAD_ARG, "bad table entry");
    MK_CUDA(c, cudaSetDevice(c->device));
    MK_CUDA(c, cudaMemcpy(out, c->table + (c->geom.row_base[row] + col) * (mkb::COMB_STRIDE_WORDS / 4), 96,
                          cudaMemcpyDeviceToHost));
    return MK_OK;
}

// Compiles needles into a MatchSet on the host (src/service/gpu.rs:618-660 Needle::new,
// dfa.rs:189-200): text needles become bit ranges of the shift-and state (a needle never
// straddles a 64-bit word; fold lowercases the needle and accepts the uppercase value too),
// DFA tables are validated and kept for upload.  A job with GRAM4_MIN_NEEDLES or more text
// needles of 4+ characters also gets the 4-gram prefilter: needles shorter than 4 are packed
// first (the words every key scans), and `gram4` receives the bitmap of the long needles'
// first 4-grams in every case variant.  No device work.
static int pack_needles(mk_ctx* c, const mk_needle* needles, uint32_t n_needles, mkb::MatchSet& ms,
                        std::vector<mkh25519::Needle>& hosts, std::vector<uint32_t>* gram4) {
    if (n_needles && !needles) return fail(c, MK_ERR_BAD_ARG, "bad argument");
    if (n_needles > (uint32_t)mkb::MAX_NEEDLES) return fail(c, MK_ERR_BAD_ARG, "too many needles");
    memset(&ms, 0, sizeof ms);
    hosts.clear();
    hosts.resize(n_needles);
    // validate and normalise every needle first
    uint32_t long_text = 0;
    for (uint32_t i = 0; i < n_needles; i++) {
        const mk_needle& nd = needles[i];
        mkh25519::Needle& h = hosts[i];
        h.mode = nd.mode;
        h.fold = nd.fold != 0;
        h.len = nd.len;
        if (nd.mode == MK_MODE_REGEX) {
            if (nd.len == 0 || nd.len > 65535 || !nd.bytes) return fail(c, MK_ERR_BAD_ARG, "bad DFA table");
            size_t bytes = (size_t)nd.len * 65 * 2;
            h.bytes.assign(nd.bytes, nd.bytes + bytes);
            // every transition must name a state of the table
            for (size_t st = 0; st < nd.len; st++)
                for (int v = 0; v < 64; v++) {
                    uint32_t t = h.bytes[(st * 65 + v) * 2] | (uint32_t)h.bytes[(st * 65 + v) * 2 + 1] << 8;
                    if (t >= nd.len) return fail(c, MK_ERR_BAD_ARG, "DFA transition out of range");
                }
            if (ms.n_regex >= 16) return fail(c, MK_ERR_BAD_ARG, "at most 16 regex needles per job");
            ms.dfa_states[ms.n_regex] = nd.len;
            ms.regex_id[ms.n_regex] = (uint16_t)i;
            ms.n_regex++;
        } else if (nd.mode == MK_MODE_CONTAINS || nd.mode == MK_MODE_SUFFIX) {
            if (nd.len == 0 || nd.len > 43 || !nd.bytes) return fail(c, MK_ERR_BAD_ARG, "needle length must be 1..43");
            h.bytes.assign(nd.bytes, nd.bytes + nd.len);
            for (auto& ch : h.bytes) {
                if (b64_value(ch) < 0) return fail(c, MK_ERR_PATTERN, "needle character outside the base64 alphabet");
                if (h.fold && ch >= 'A' && ch <= 'Z') ch = (uint8_t)(ch + 32);
            }
            if (nd.len >= 4) long_text++;
        } else {
            return fail(c, MK_ERR_BAD_ARG, "unknown needle mode");
        }
    }
    // the packing is the same whether or not the bitmap is wanted (gram4 null: check only)
    const bool prefilter = long_text >= mkb::GRAM4_MIN_NEEDLES;
    uint32_t bit = 0;  // next free bit in the shift-and state
    auto place = [&](uint32_t i) -> int {
        const mkh25519::Needle& h = hosts[i];
        const uint32_t len = h.len;
        if ((bit & 63) + len > 64) bit = (bit + 63) & ~63u;
        if (bit + len > 64u * mkb::SA_WORDS) return fail(c, MK_ERR_BAD_ARG, "needles exceed the shift-and state");
        for (uint32_t k = 0; k < len; k++) {
            uint32_t b = bit + k;
            uint8_t ch = h.bytes[k];
            int v = b64_value(ch);
            ms.mask[b >> 6][v] |= 1ull << (b & 63);
            if (h.fold && ch >= 'a' && ch <= 'z') ms.mask[b >> 6][v - 26] |= 1ull << (b & 63);
        }
        ms.first_bit[bit >> 6] |= 1ull << (bit & 63);
        uint32_t last = bit + len - 1;
        if (h.mode == MK_MODE_SUFFIX) ms.suffix_bit[last >> 6] |= 1ull << (last & 63);
        else ms.last_bit[last >> 6] |= 1ull << (last & 63);
        ms.text_id[ms.n_text] = (uint16_t)i;
        ms.text_last[ms.n_text] = (uint16_t)last;
        ms.n_text++;
        bit += len;
        return MK_OK;
    };
    auto is_text = [&](uint32_t i) { return hosts[i].mode != MK_MODE_REGEX; };
    if (prefilter) {
        for (uint32_t i = 0; i < n_needles; i++)
            if (is_text(i) && hosts[i].len < 4)
                if (int st = place(i)) return st;
        bit = (bit + 63) & ~63u;
        ms.short_words = bit / 64;
        for (uint32_t i = 0; i < n_needles; i++)
            if (is_text(i) && hosts[i].len >= 4)
                if (int st = place(i)) return st;
        if (gram4) gram4->assign(mkb::GRAM4_WORDS, 0u);
        for (uint32_t i = 0; gram4 && i < n_needles; i++) {
            if (!is_text(i) || hosts[i].len < 4) continue;
            const mkh25519::Needle& h = hosts[i];
            // every case variant of the first four characters
            int vals[4][2], nv[4];
            for (int k = 0; k < 4; k++) {
                const uint8_t ch = h.bytes[k];
                vals[k][0] = b64_value(ch);
                nv[k] = (h.fold && ch >= 'a' && ch <= 'z') ? 2 : 1;
                vals[k][1] = vals[k][0] - 26;
            }
            for (int m = 0; m < 16; m++) {
                bool ok = true;
                uint32_t g = 0;
                for (int k = 0; k < 4; k++) {
                    const int pick = (m >> k) & 1;
                    if (pick >= nv[k]) ok = false;
                    g = g << 6 | (uint32_t)vals[k][pick];
                }
                if (ok) (*gram4)[g >> 5] |= 1u << (g & 31);
            }
        }
    } else {
        for (uint32_t i = 0; i < n_needles; i++)
            if (is_text(i))
                if (int st = place(i)) return st;
    }
    ms.sa_words = ms.n_text ? (bit + 63) / 64 : 0;
    if (!prefilter) ms.short_words = ms.sa_words;
    ms.narrow = ms.n_text && !prefilter && bit <= 32;
    return MK_OK;
}

// Uploads a packed MatchSet and its DFA tables to the job's device copy (after the job's
// previous launches have finished).  DFA tables get fresh device buffers; text needles
// need no allocation.
static int upload_needles(mk_job* j, mkb::MatchSet& ms, std::vector<mkh25519::Needle>& hosts,
                          const std::vector<uint32_t>& gram4) {
    mk_ctx* c = j->ctx;
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    ms.gram4 = nullptr;
    // all copies are ordered on the context's stream after the allocations; the stream is
    // drained before returning, while the host vectors are still alive
    if (!gram4.empty()) {
        if (!j->d_gram4 && !pool_alloc(c, &j->d_gram4, gram4.size() * 4))
            return fail(c, MK_ERR_OUT_OF_MEMORY, "prefilter allocation");
        MK_CUDA(c, cudaMemcpyAsync(j->d_gram4, gram4.data(), gram4.size() * 4, cudaMemcpyHostToDevice, c->stream));
        j->h2d += gram4.size() * 4;
        ms.gram4 = j->d_gram4;
    }
    for (auto d : j->d_dfa) pool_free(c, d);
    j->d_dfa.clear();
    for (uint32_t r = 0; r < ms.n_regex; r++) {
        const mkh25519::Needle& h = hosts[ms.regex_id[r]];
        uint8_t* d = nullptr;
        if (!pool_alloc(c, &d, h.bytes.size())) {
            cudaStreamSynchronize(c->stream);
            return fail(c, MK_ERR_OUT_OF_MEMORY, "DFA allocation");
        }
        j->d_dfa.push_back(d);
        MK_CUDA(c, cudaMemcpyAsync(d, h.bytes.data(), h.bytes.size(), cudaMemcpyHostToDevice, c->stream));
        j->h2d += h.bytes.size();
        ms.dfa[r] = d;
    }
    if (!j->d_match && !pool_alloc(c, &j->d_match, sizeof ms)) {
        cudaStreamSynchronize(c->stream);
        return fail(c, MK_ERR_OUT_OF_MEMORY, "match allocation");
    }
    MK_CUDA(c, cudaMemcpyAsync(j->d_match, &ms, sizeof ms, cudaMemcpyHostToDevice, c->stream));
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    j->h2d += sizeof ms;
    j->needles = std::move(hosts);
    return MK_OK;
}

int mk_job_prepare(mk_ctx* c, const uint8_t key[32], int seed_source, const mk_needle* needles, uint32_t n_needles,
                   int stop_on_hit, mk_job** out) try {
    if (!c || !key || !out || (n_needles && !needles)) return fail(c, MK_ERR_BAD_ARG, "bad argument");
    if (int st = check_source(c, key, seed_source)) return st;
    if (seed_source == MK_SEED_INCREMENTAL && c->hash_warps)
        return fail(c, MK_ERR_NOT_BUILT, "the hashing-warp search layout serves hashed seed sources only");
    *out = nullptr;
    MK_CUDA(c, cudaSetDevice(c->device));
    std::unique_ptr<mkb::MatchSet> ms(new (std::nothrow) mkb::MatchSet);
    if (!ms) return fail(c, MK_ERR_OUT_OF_MEMORY, "host allocation");
    std::vector<mkh25519::Needle> hosts;
    std::vector<uint32_t> gram4;
    if (int st = pack_needles(c, needles, n_needles, *ms, hosts, &gram4)) return st;
    mk_job* j = new (std::nothrow) mk_job;
    if (!j) return fail(c, MK_ERR_OUT_OF_MEMORY, "host allocation");
    j->ctx = c;
    if (!c->spare_hits.empty()) {
        j->last = std::move(c->spare_hits.back());
        c->spare_hits.pop_back();
    }
    memcpy(j->key, key, 32);
    j->source = seed_source;
    j->stop_on_hit = stop_on_hit;
    j->cap = c->hit_capacity;
    auto bail = [&](int code, const std::string& msg) {
        mk_job_destroy(j);
        return fail(c, code, msg);
    };
    if (int st = upload_needles(j, *ms, hosts, gram4)) {
        std::string keep = c->err;
        mk_job_destroy(j);
        return fail(c, st, keep);
    }
    if (!pool_alloc(c, &j->d_hits, sizeof(mkb::HitRecord) * j->cap)) return bail(MK_ERR_OUT_OF_MEMORY, "hit ring");
    if (!pool_alloc(c, &j->d_job, sizeof(mkb::JobDevice))) return bail(MK_ERR_OUT_OF_MEMORY, "job state");
    if (cudaMemsetAsync(j->d_job, 0, sizeof(mkb::JobDevice), c->stream) != cudaSuccess)
        return bail(MK_ERR_CUDA, "job state");
    if (!pool_alloc(c, &j->d_sink, sizeof(uint32_t) * (size_t)c->grid * c->block)) return bail(MK_ERR_OUT_OF_MEMORY, "sink");
    // the side stream (stop requests) and blocking copies may touch the buffers from here on
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(MK_ERR_CUDA, "job buffers");
    *out = j;
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_needles_check(const mk_needle* needles, uint32_t n_needles) try {
    std::unique_ptr<mkb::MatchSet> ms(new (std::nothrow) mkb::MatchSet);
    if (!ms) return MK_ERR_OUT_OF_MEMORY;
    std::vector<mkh25519::Needle> hosts;
    return pack_needles(nullptr, needles, n_needles, *ms, hosts, nullptr);
} MK_ABI_CATCH(nullptr)

uint64_t mk_job_keys_per_iter(const mk_job* j) { return j && j->ctx ? j->ctx->info.keys_per_iter : 0; }

int mk_job_update(mk_job* j, const mk_needle* needles, uint32_t n_needles) try {
    if (!j) return MK_ERR_BAD_ARG;
    mk_ctx* c = j->ctx;
    MK_CUDA(c, cudaSetDevice(c->device));
    std::unique_ptr<mkb::MatchSet> ms(new (std::nothrow) mkb::MatchSet);
    if (!ms) return fail(c, MK_ERR_OUT_OF_MEMORY, "host allocation");
    std::vector<mkh25519::Needle> hosts;
    std::vector<uint32_t> gram4;
    if (int st = pack_needles(c, needles, n_needles, *ms, hosts, &gram4)) return st;
    return upload_needles(j, *ms, hosts, gram4);
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

void mk_job_destroy(mk_job* j) try {
    if (!j) return;
    if (j->ctx) cudaSetDevice(j->ctx->device);
    if (j->ctx && j->ctx->stream) {
        mk_ctx* c = j->ctx;
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->side);  // a stop request still in flight writes d_job
        for (auto d : j->d_dfa) pool_free(c, d);
        pool_free(c, j->d_gram4);
        pool_free(c, j->d_match);
        pool_free(c, j->d_hits);
        pool_free(c, j->d_job);
        pool_free(c, j->d_sink);
        if (j->last.cap && c->spare_hits.size() < 4) {
            j->last.clear();
            c->spare_hits.push_back(std::move(j->last));
        }
    }
    delete j;
} MK_ABI_CATCH_VOID

// Shared memory for the job's DFA tables when they fit (the kernel then reads them there).
static uint32_t dfa_smem_bytes(const mk_job* j) {
    if (j->ctx->hash_warps) return 0;  // the hashing-warp kernel's scalar ring takes that shared memory
    if (j->ctx->table_smem) return 0;  // so does a comb table kept in shared memory
    uint64_t total = 0;
    for (const auto& h : j->needles)
        if (h.mode == MK_MODE_REGEX) total += ((uint64_t)h.len * 130 + 15) & ~15ull;
    return total <= mkb::DFA_SMEM_MAX ? (uint32_t)total : 0;
}

// Kernel parameters of one search launch of a job.
static mkb::KeyLaunch search_params(const mk_job* j, uint64_t base, uint32_t iters) {
    const mk_ctx* c = j->ctx;
    mkb::KeyLaunch L{};
    L.table = c->table;
    L.geom = c->geom;
    for (int i = 0; i < 8; i++)
        L.key[i] = (uint32_t)j->key[4 * i] | (uint32_t)j->key[4 * i + 1] << 8 | (uint32_t)j->key[4 * i + 2] << 16 | (uint32_t)j->key[4 * i + 3] << 24;
    L.seed_src = (uint32_t)j->source;
    L.iters = iters;
    L.base = base;
    L.match = j->d_match;
    L.hits = j->d_hits;
    L.hit_cap = j->cap;
    L.stop_on_hit = (uint32_t)j->stop_on_hit;
    L.job = j->d_job;
    L.sink = j->d_sink;
    if (j->source == MK_SEED_INCREMENTAL) set_incremental(c, j->key, base, L);
    L.dfa_smem = dfa_smem_bytes(j);
    L.layout = c->layout;
    L.inv_pools = c->inv_pools;
    L.table_smem = c->table_smem;
    return L;
}

static int enqueue(mk_job* j, uint64_t base, uint32_t iters) {
    mk_ctx* c = j->ctx;
    // an incremental index is the scalar offset itself: a range that wraps past 2^64 would
    // report indices whose keys are not the points the kernel stepped to
    if (j->source == MK_SEED_INCREMENTAL) {
        const unsigned __int128 end = (unsigned __int128)base + (unsigned __int128)c->info.keys_per_iter * iters;
        if (end > ((unsigned __int128)1 << 64)) return fail(c, MK_ERR_OUT_OF_RANGE, "incremental indices must not wrap past 2^64");
    }
    MK_CUDA(c, cudaSetDevice(c->device));
    MK_CUDA(c, cudaMemsetAsync(j->d_job, 0, 8, c->stream));  // hit_count and status; keep stop
    mkb::KeyLaunch L = search_params(j, base, iters);
    MK_CUDA(c, mkb::launch_keys(L, false, c->kpt, c->block, c->grid, c->stream));
    j->h2d += sizeof L;  // kernel parameters
    return MK_OK;
}

int mk_job_enqueue(mk_job* j, uint64_t base, uint32_t iters) try {
    if (!j) return MK_ERR_BAD_ARG;
    if (iters == 0) return MK_OK;
    return enqueue(j, base, iters);
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

// Waits for the job's queued work, then reads its state and hit ring (sorted by index).
static int collect(mk_job* j, int* found, uint64_t* index) {
    mk_ctx* c = j->ctx;
    mkb::JobDevice jd;
    MK_CUDA(c, cudaMemcpyAsync(&jd, j->d_job, sizeof jd, cudaMemcpyDeviceToHost, c->stream));
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    j->d2h += sizeof jd;
    j->last_total = jd.hit_count;
    uint32_t n = std::min(jd.hit_count, j->cap);
    if (n) {
        static_assert(sizeof(mkb::HitRecord) == sizeof(mk_hit) && offsetof(mkb::HitRecord, needle) == offsetof(mk_hit, needle),
                      "device hit records are read back as mk_hit");
        j->last.resize_uninit(n);
        MK_CUDA(c, cudaMemcpy(j->last.data(), j->d_hits, sizeof(mk_hit) * n, cudaMemcpyDeviceToHost));
        j->d2h += sizeof(mk_hit) * n;
        j->sorted = false;
        uint64_t lowest = ~0ull;
        mk_hit* h = j->last.data();
        for (uint32_t i = 0; i < n; i++) {
            h[i].reserved = 0;
            lowest = std::min(lowest, h[i].index);
        }
        if (found) *found = 1;
        if (index) *index = lowest;
    }
    if (jd.hit_count > j->cap) return fail(c, MK_ERR_HIT_RING_FULL, "hit ring overflow");
    if (jd.status & 1u) return MK_ERR_STOPPED;
    return MK_OK;
}

int mk_job_collect(mk_job* j, int* found, uint64_t* index) try {
    if (!j) return MK_ERR_BAD_ARG;
    j->last.clear();
    j->last_total = 0;
    if (found) *found = 0;
    MK_CUDA(j->ctx, cudaSetDevice(j->ctx->device));
    return collect(j, found, index);
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

int mk_job_launch(mk_job* j, uint64_t base, uint32_t iters, int* found, uint64_t* index) try {
    if (!j) return MK_ERR_BAD_ARG;
    j->last.clear();
    j->last_total = 0;
    if (found) *found = 0;
    if (iters == 0) return MK_OK;
    int st = enqueue(j, base, iters);
    if (st) return st;
    return collect(j, found, index);
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

int mk_job_hits(mk_job* j, mk_hit* out, uint32_t cap, uint32_t* written, uint64_t* total) try {
    if (!j || !written || !total || (cap && !out)) return MK_ERR_BAD_ARG;
    *total = j->last_total;
    uint32_t k = std::min<uint32_t>(cap, (uint32_t)j->last.n);
    if (k && !j->sorted) {
        mkhits::sort_hits(j->last.data(), j->last.n);
        j->sorted = true;
    }
    if (k) memcpy(out, j->last.data(), sizeof(mk_hit) * k);
    *written = k;
    return j->last_total > j->cap ? MK_ERR_HIT_RING_FULL : MK_OK;
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

// Re-derives a candidate on the host and tests its needle with the real x sign.  Touches no
// shared state (host threads confirm different needles at once); 1 / 2 for a bad needle or
// start scalar.
static int confirm_key(const mk_job* j, uint64_t index, uint32_t needle, uint8_t pk[32], uint8_t secret[32],
                       int* matched) {
    if (needle >= j->needles.size()) return 1;
    *matched = 0;
    if (j->source == MK_SEED_INCREMENTAL) {
        if (!mkh25519::incremental_scalar(j->key, index, secret)) return 2;
        mkh25519::scalar_public_key(secret, pk);
    } else {
        mkh25519::seed_of(j->key, j->source, index, secret);
        mkh25519::public_key(secret, pk);
    }
    *matched = mkh25519::matches(j->needles[needle], pk) ? 1 : 0;
    return 0;
}

static int confirm_fail(mk_job* j, int e) {
    return fail(j->ctx, MK_ERR_BAD_ARG,
                e == 1 ? "needle index out of range" : "incremental start scalar must be below 2^255");
}

int mk_job_confirm(mk_job* j, uint64_t index, uint32_t needle, uint8_t pk[32], uint8_t secret[32], int* matched) try {
    if (!j || !pk || !secret || !matched) return MK_ERR_BAD_ARG;
    if (int e = confirm_key(j, index, needle, pk, secret, matched)) return confirm_fail(j, e);
    return MK_OK;
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

int mk_job_stop(mk_job* j, int on) {
    if (!j) return MK_ERR_BAD_ARG;
    mk_ctx* c = j->ctx;
    MK_CUDA(c, cudaSetDevice(c->device));
    // the job word's stop field (nonzero = stop), set on the side stream so that it lands
    // while a launch of this job runs on the context's stream
    MK_CUDA(c, cudaMemsetAsync(&j->d_job->stop, on ? 1 : 0, sizeof(uint32_t), c->side));
    MK_CUDA(c, cudaStreamSynchronize(c->side));
    return MK_OK;
}

int mk_job_first_matches(mk_job* j, mk_outcome* out, uint32_t n) try {
    if (!j || (n && !out)) return MK_ERR_BAD_ARG;
    for (uint32_t k = 0; k < n; k++) {
        memset(&out[k], 0, sizeof out[k]);
        out[k].status = MK_ERR_STOPPED;
        out[k].needle = k;
    }
    // per needle, its candidates from the lowest index up until one matches with its real x
    // sign: the candidates are bucketed by needle and each bucket is a min-heap, so a needle
    // that confirms at once costs no ordering of the rest
    const mk_hit* h = j->last.data();
    const size_t m = j->last.n;
    std::vector<size_t> start(n + 1, 0);
    for (size_t i = 0; i < m; i++)
        if (h[i].needle < n) start[h[i].needle + 1]++;
    for (uint32_t k = 0; k < n; k++) start[k + 1] += start[k];
    std::vector<uint64_t>& idx = j->last.scratch;
    idx.resize(start[n]);
    {
        std::vector<size_t> next(start.begin(), start.end() - 1);
        for (size_t i = 0; i < m; i++)
            if (h[i].needle < n) idx[next[h[i].needle]++] = h[i].index;
    }
    // needles are independent: host threads take them in turn (a confirmation is a host
    // Ed25519 derivation, tens of microseconds)
    std::vector<int> errs(n, 0);
    std::atomic<uint32_t> next{0};
    auto work = [&]() {
        for (uint32_t k; (k = next.fetch_add(1)) < n;) {
            auto b = idx.begin() + start[k], e = idx.begin() + start[k + 1];
            std::make_heap(b, e, std::greater<uint64_t>());
            while (b != e) {
                std::pop_heap(b, e, std::greater<uint64_t>());
                --e;
                mk_outcome& o = out[k];
                int ok = 0;
                if ((errs[k] = confirm_key(j, *e, k, o.pk, o.secret, &ok)) != 0) break;
                if (ok) {
                    o.status = MK_OK;
                    o.index = *e;
                    break;
                }
            }
        }
    };
    uint32_t busy = 0;
    for (uint32_t k = 0; k < n; k++) busy += start[k + 1] > start[k];
    const uint32_t threads = std::min<uint32_t>(std::min<uint32_t>(busy, 16u), std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    try {
        pool.reserve(threads);
        for (uint32_t t = 1; t < threads; t++) pool.emplace_back(work);
    } catch (...) {
        // the host would not start another thread (e.g. a process limit): the threads that
        // did start and this one share the needles
    }
    work();
    for (auto& t : pool) t.join();
    for (uint32_t k = 0; k < n; k++)
        if (errs[k]) return confirm_fail(j, errs[k]);
    // candidates beyond the hit ring were counted but not kept: a needle's lowest candidate
    // may be among them, so the outcomes are those of the kept candidates only
    if (j->last_total > j->cap) return fail(j->ctx, MK_ERR_HIT_RING_FULL, "hit ring overflow: outcomes of the kept candidates only");
    return MK_OK;
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

int mk_job_io_bytes(const mk_job* j, uint64_t* h2d, uint64_t* d2h) {
    if (!j || !h2d || !d2h) return MK_ERR_BAD_ARG;
    *h2d = j->h2d;
    *d2h = j->d2h;
    return MK_OK;
}

int mk_ctx_work_per_key(const mk_ctx* c, int seed_source, double* field_muls, double* int_mads) {
    if (!c || !field_muls || !int_mads || seed_source < MK_SEED_CHACHA20 || seed_source > MK_SEED_INCREMENTAL)
        return MK_ERR_BAD_ARG;
    // radix-2^32 costs: a schoolbook multiplication is 64 mad.lo + 64 mad.hi (8x8 limbs) + 16
    // (fold by 38), the Karatsuba form 48 + 48 + 16, a squaring 28 cross products + 8 diagonal
    // ones (72) + 16.  The secure path's comb, batch and back-sweep multiply in the Karatsuba
    // form; the incremental path and the pooled inversions in the schoolbook one.
    const double MUL = mkb::MADS_MUL_SCHOOLBOOK, SQ = mkb::MADS_SQUARE;
    const double PATH_MUL = seed_source == MK_SEED_INCREMENTAL ? MUL : mkb::MADS_MUL_KARATSUBA;
    const double kpt = c->kpt, rows = c->geom.rows;
    const double ct = mkb::search_threads(c->block, c->layout);
    // comb: row 0 is free, full additions cost 7 multiplications, the last one 3
    double comb = 7.0 * (rows - 2) + 3.0;
    // Montgomery batch inside a thread: a_j and the running product (2 each for j > 0),
    // back-sweep y_j = a_j·inv and inv·den_j
    double batch = (4.0 * (kpt - 1) + 1.0) / kpt;
    if (seed_source == MK_SEED_INCREMENTAL) {
        // no comb: key j > 0 of a thread's run is the y of Q + j·B (3 multiplications), and Q
        // advances once per run by a full mixed addition (7); the thread's start point
        // (at most 8 additions per launch) is left out
        comb = (3.0 * (kpt - 1) + 7.0) / kpt;
    }
    // pooled inversion by the CTA's inverting warp: `pools` lanes, each over `groups` thread
    // products, 3(groups-1) multiplications and one inversion (254 squarings + 11 multiplications)
    const double pools = c->inv_pools, groups = ct / pools;
    double pool_mul = pools * (3.0 * (groups - 1) + 11.0) / (ct * kpt);
    double pool_sq = pools * 254.0 / (ct * kpt);
    *field_muls = comb + batch + pool_mul + pool_sq;
    *int_mads = (comb + batch) * PATH_MUL + pool_mul * MUL + pool_sq * SQ;
    return MK_OK;
}

int mk_measure_imad_rates(mk_ctx* c, double* hi_per_s, double* wide_per_s, double* lo_chain_per_s,
                          double* hi_chain_per_s) try {
    if (!c || !hi_per_s || !wide_per_s || !lo_chain_per_s || !hi_chain_per_s) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaSetDevice(c->device));
    double r[4] = {0, 0, 0, 0};
    MK_CUDA(c, mkb::measure_imad_rates((int)c->info.sms, c->stream, r));
    *hi_per_s = r[0];
    *wide_per_s = r[1];
    *lo_chain_per_s = r[2];
    *hi_chain_per_s = r[3];
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_measure_mad_peaks(mk_ctx* c, double* chain_per_s, double* lo_per_s) try {
    if (!c || !chain_per_s || !lo_per_s) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaSetDevice(c->device));
    MK_CUDA(c, mkb::measure_mad_peaks((int)c->info.sms, c->stream, chain_per_s, lo_per_s));
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

// ---- CUDA graph of a job's launches ----

int mk_job_graph_create(mk_job* j, uint32_t iters, uint32_t launches, mk_graph** out) try {
    if (!j || !out || iters == 0 || launches == 0 || launches > 4096) return MK_ERR_BAD_ARG;
    *out = nullptr;
    mk_ctx* c = j->ctx;
    MK_CUDA(c, cudaSetDevice(c->device));
    mk_graph* g = new (std::nothrow) mk_graph;
    if (!g) return fail(c, MK_ERR_OUT_OF_MEMORY, "host allocation");
    g->job = j;
    g->iters = iters;
    g->span = c->info.keys_per_iter * iters;
    g->params.resize(launches);
    g->nodes.resize(launches);
    auto bail = [&](cudaError_t e, const char* what) {
        mk_graph_destroy(g);
        return cuda_fail(c, e, what);
    };
    cudaError_t e = cudaGraphCreate(&g->graph, 0);
    if (e != cudaSuccess) return bail(e, "cudaGraphCreate");
    // reset hit count and status once; hits of all launches accumulate in the ring
    cudaMemsetParams ms{};
    ms.dst = j->d_job;
    ms.value = 0;
    ms.elementSize = 4;
    ms.width = 2;
    ms.height = 1;
    ms.pitch = 0;
    cudaGraphNode_t prev = nullptr;
    e = cudaGraphAddMemsetNode(&prev, g->graph, nullptr, 0, &ms);
    if (e != cudaSuccess) return bail(e, "cudaGraphAddMemsetNode");
    const void* func = nullptr;
    size_t dyn = 0;
    e = mkb::keys_kernel(false, j->source == MK_SEED_INCREMENTAL, c->kpt, c->block, c->layout, dfa_smem_bytes(j),
                         c->table_smem, &func, &dyn);
    if (e != cudaSuccess) return bail(e, "keys_kernel");
    for (uint32_t i = 0; i < launches; i++) {
        g->params[i] = search_params(j, g->span * i, iters);
        void* args[] = {&g->params[i]};
        cudaKernelNodeParams kp{};
        kp.func = const_cast<void*>(func);
        kp.gridDim = dim3(c->grid);
        kp.blockDim = dim3(c->block);
        kp.sharedMemBytes = (unsigned)dyn;
        kp.kernelParams = args;
        e = cudaGraphAddKernelNode(&g->nodes[i], g->graph, &prev, 1, &kp);
        if (e != cudaSuccess) return bail(e, "cudaGraphAddKernelNode");
        prev = g->nodes[i];
    }
    g->func = func;
    g->dyn = dyn;
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) return bail(e, "cudaGraphInstantiate");
    *out = g;
    return MK_OK;
} MK_ABI_CATCH(j && j->ctx ? &j->ctx->err : nullptr)

// Points every kernel node at its range of base .. base + launches·span and enqueues the graph.
static int graph_enqueue(mk_graph* g, uint64_t base) {
    mk_job* j = g->job;
    mk_ctx* c = j->ctx;
    MK_CUDA(c, cudaSetDevice(c->device));
    // the job's needles may have changed since the graph was made: size the DFA staging anew
    MK_CUDA(c, mkb::keys_kernel(false, j->source == MK_SEED_INCREMENTAL, c->kpt, c->block, c->layout, dfa_smem_bytes(j),
                                c->table_smem, &g->func,
                                &g->dyn));
    for (size_t i = 0; i < g->nodes.size(); i++) {
        g->params[i] = search_params(j, base + g->span * i, g->iters);
        void* args[] = {&g->params[i]};
        cudaKernelNodeParams kp{};
        kp.func = const_cast<void*>(g->func);
        kp.gridDim = dim3(c->grid);
        kp.blockDim = dim3(c->block);
        kp.sharedMemBytes = (unsigned)g->dyn;
        kp.kernelParams = args;
        MK_CUDA(c, cudaGraphExecKernelNodeSetParams(g->exec, g->nodes[i], &kp));
        j->h2d += sizeof(mkb::KeyLaunch);
    }
    MK_CUDA(c, cudaGraphLaunch(g->exec, c->stream));
    return MK_OK;
}

int mk_graph_enqueue(mk_graph* g, uint64_t base) try {
    if (!g) return MK_ERR_BAD_ARG;
    return graph_enqueue(g, base);
} MK_ABI_CATCH(g && g->job && g->job->ctx ? &g->job->ctx->err : nullptr)

int mk_graph_launch(mk_graph* g, uint64_t base, int* found, uint64_t* index) try {
    if (!g) return MK_ERR_BAD_ARG;
    mk_job* j = g->job;
    j->last.clear();
    j->last_total = 0;
    if (found) *found = 0;
    if (int st = graph_enqueue(g, base)) return st;
    return collect(j, found, index);
} MK_ABI_CATCH(g && g->job && g->job->ctx ? &g->job->ctx->err : nullptr)

void mk_graph_destroy(mk_graph* g) try {
    if (!g) return;
    if (g->job && g->job->ctx) {
        cudaSetDevice(g->job->ctx->device);
        cudaStreamSynchronize(g->job->ctx->stream);
    }
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
} MK_ABI_CATCH_VOID

int mk_measure_field_mul(mk_ctx* c, double* radix32_per_s, double* radix26_per_s, double* radix51_fp64_per_s) try {
    if (!c || !radix32_per_s || !radix26_per_s || !radix51_fp64_per_s) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaSetDevice(c->device));
    bool exact = false;
    MK_CUDA(c, mkb::measure_field_mul_rates((int)c->info.sms, c->stream, radix32_per_s, radix26_per_s,
                                            radix51_fp64_per_s, &exact));
    if (!exact) return fail(c, MK_ERR_SELF_CHECK, "radix-2^51 (FP64) products differ from radix 2^32");
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_regex_compile_device(mk_ctx* c, const char* pattern, int case_sensitive, uint32_t max_states, uint8_t* table,
                            uint32_t* states, char* err, size_t err_size) try {
    auto error = [&](const std::string& m, int code) {
        if (err && err_size) snprintf(err, err_size, "%s", m.c_str());
        return code;
    };
    if (err && err_size) err[0] = 0;
    if (!c || !pattern || !table || !states || max_states < 2 || max_states > 65535)
        return error("bad argument", MK_ERR_BAD_ARG);
    *states = 0;
    mkre::NfaTables t;
    std::string msg;
    int st = mkre::nfa_tables(pattern, case_sensitive, mkb::MAX_DFA_NFA_WORDS, &t, &msg);
    if (st != MK_OK) return error(msg, st);
    MK_CUDA(c, cudaSetDevice(c->device));
    std::vector<uint8_t> rows;
    uint32_t n = 0;
    bool too_many = false;
    MK_CUDA(c, mkb::build_dfa_device(t, max_states, c->stream, &rows, &n, &too_many));
    if (too_many) return error(mkre::too_complex(max_states), MK_ERR_PATTERN);
    st = mkre::check_table(rows.data(), n, &msg);
    if (st != MK_OK) return error(msg, st);
    memcpy(table, rows.data(), (size_t)n * 130);
    *states = n;
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_field_mul_pairs(mk_ctx* c, const uint32_t* a, const uint32_t* b, uint32_t n, uint32_t* schoolbook,
                       uint32_t* karatsuba) try {
    if (!c || !a || !b || !schoolbook || !karatsuba || n == 0 || n > (1u << 20)) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaSetDevice(c->device));
    MK_CUDA(c, mkb::field_mul_pairs(a, b, n, schoolbook, karatsuba, c->stream));
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_measure_field_mul_forms(mk_ctx* c, double* schoolbook_per_s, double* karatsuba_per_s) try {
    if (!c || !schoolbook_per_s || !karatsuba_per_s) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaSetDevice(c->device));
    bool same = false;
    MK_CUDA(c, mkb::measure_field_mul_forms((int)c->info.sms, c->stream, schoolbook_per_s, karatsuba_per_s, &same));
    if (!same) return fail(c, MK_ERR_SELF_CHECK, "Karatsuba field products differ from the schoolbook ones");
    return MK_OK;
} MK_ABI_CATCH(c ? &c->err : nullptr)

int mk_ctx_sync(mk_ctx* c) {
    if (!c) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaStreamSynchronize(c->stream));
    return MK_OK;
}

int mk_ctx_record(mk_ctx* c, int slot) {
    if (!c || slot < 0 || slot >= 16) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaEventRecord(c->ev[slot], c->stream));
    return MK_OK;
}

int mk_ctx_elapsed(mk_ctx* c, int a, int b, float* ms) {
    if (!c || !ms || a < 0 || a >= 16 || b < 0 || b >= 16) return MK_ERR_BAD_ARG;
    MK_CUDA(c, cudaEventSynchronize(c->ev[b]));
    MK_CUDA(c, cudaEventElapsedTime(ms, c->ev[a], c->ev[b]));
    return MK_OK;
}

}  // extern "C"
