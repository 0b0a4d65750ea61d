// Subset construction of a regex DFA on the device (Dfa::new, src/model/pattern/dfa.rs:52-108,
// the part whose cost grows with the DFA): one CTA walks the DFA breadth first, a frontier at
// a time.  The threads compute the successor sets of all (state, value) pairs of a chunk of
// the frontier in parallel and look them up in an open-addressing table of the states found so
// far; one thread then gives the new sets their numbers in (state, value) order, which is the
// order of discovery mk_regex_compile numbers states in on the host, so both build the same
// table.  Every loop is bounded by the table sizes; the CTA waits only at __syncthreads.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "kernels.h"
#include "regex.h"

namespace mkb {

namespace {

constexpr uint32_t DFA_BLOCK = 512;
constexpr uint32_t DFA_CHUNK = 4096;  // (state, value) pairs resolved between two barriers

struct DfaDev {
    uint32_t n, words, track_word, max_states, hash_mask;
    int32_t start, match;
    const uint32_t* plain;   // [n][words]
    const uint32_t* plainm;  // [words]
    const uint32_t* dec;     // [8][n][words]
    const uint32_t* decm;    // [8][words]
    const uint32_t* endm;    // [4][words]
    const int32_t* sym_to;   // [n]
    const uint64_t* sym;     // [n]
    uint32_t* keys;          // [max_states][words + 1]: DFA state j + 1 (word `words` holds its flags)
    uint32_t* cand;          // [DFA_CHUNK][words + 1]
    uint32_t* hash;          // [hash_mask + 1]: key index + 1, 0 when empty
    uint16_t* table;         // [max_states][65]
    uint32_t* result;        // [0] states including the accept state, [1] 1 when max_states was exceeded
};

__device__ __forceinline__ uint32_t key_hash(const uint32_t* k, uint32_t words) {
    uint32_t h = 0x811c9dc5u ^ k[words];
    for (uint32_t i = 0; i < words; i++) h = (h ^ k[i]) * 0x01000193u + (h >> 15);
    return h ^ (h >> 16);
}

__device__ __forceinline__ bool key_equal(const uint32_t* a, const uint32_t* b, uint32_t words) {
    for (uint32_t i = 0; i <= words; i++)
        if (a[i] != b[i]) return false;
    return true;
}

// DFA id (key index + 1) of the set `k`, or -1 when it is not in the table
__device__ int32_t dfa_find(const DfaDev& d, const uint32_t* k) {
    uint32_t h = key_hash(k, d.words) & d.hash_mask;
    for (uint32_t probe = 0; probe <= d.hash_mask; probe++) {
        const uint32_t e = d.hash[h];
        if (e == 0) return -1;
        if (key_equal(d.keys + (size_t)(e - 1) * (d.words + 1), k, d.words)) return (int32_t)e;
        h = (h + 1) & d.hash_mask;
    }
    return -1;
}

// Adds key index `idx` (its words already in d.keys) to the hash table; the table has more
// slots than states, so a free one is found.
__device__ void dfa_insert(const DfaDev& d, uint32_t idx) {
    const uint32_t* k = d.keys + (size_t)idx * (d.words + 1);
    uint32_t h = key_hash(k, d.words) & d.hash_mask;
    for (uint32_t probe = 0; probe <= d.hash_mask; probe++) {
        if (d.hash[h] == 0) {
            d.hash[h] = idx + 1;
            return;
        }
        h = (h + 1) & d.hash_mask;
    }
}

// Successor of DFA state `k` (key index) on base64 value v: 0 when the match state is reached
// (the accept state), else -1 with the successor's set and flags written to `out`.
__device__ int32_t dfa_step(const DfaDev& d, uint32_t k, uint32_t v, uint32_t* out) {
    const uint32_t W = d.words;
    const uint32_t* S = d.keys + (size_t)k * (W + 1);
    const bool first = k == 0, prev_word = (S[W] & 1u) != 0, word = v < 62;
    uint32_t C[MAX_DFA_NFA_WORDS], nx[MAX_DFA_NFA_WORDS];
    if (d.track_word) {
        // assertions between the previous character and this one
        const uint32_t c = (first ? 4u : 0u) | (prev_word ? 2u : 0u) | (word ? 1u : 0u);
        const uint32_t* m = d.decm + (size_t)c * W;
        for (uint32_t i = 0; i < W; i++)
            if (S[i] & m[i]) return 0;
        for (uint32_t i = 0; i < W; i++) C[i] = 0;
        for (uint32_t i = 0; i < W; i++)
            for (uint32_t b = S[i]; b; b &= b - 1) {
                const uint32_t* row = d.dec + ((size_t)c * d.n + i * 32 + __ffs(b) - 1) * W;
                for (uint32_t j = 0; j < W; j++) C[j] |= row[j];
            }
    } else {
        for (uint32_t i = 0; i < W; i++) C[i] = S[i];
        if ((C[d.match >> 5] >> (d.match & 31)) & 1u) return 0;
    }
    // the symbol edges on v, plus the start state (a match may start after this character)
    for (uint32_t i = 0; i < W; i++) nx[i] = 0;
    nx[d.start >> 5] |= 1u << (d.start & 31);
    for (uint32_t i = 0; i < W; i++)
        for (uint32_t b = C[i]; b; b &= b - 1) {
            const uint32_t s = i * 32 + __ffs(b) - 1;
            const int32_t to = d.sym_to[s];
            if (to >= 0 && ((d.sym[s] >> v) & 1ull)) nx[to >> 5] |= 1u << (to & 31);
        }
    for (uint32_t i = 0; i < W; i++)
        if (nx[i] & d.plainm[i]) return 0;
    for (uint32_t i = 0; i < W; i++) out[i] = 0;
    for (uint32_t i = 0; i < W; i++)
        for (uint32_t b = nx[i]; b; b &= b - 1) {
            const uint32_t* row = d.plain + (size_t)(i * 32 + __ffs(b) - 1) * W;
            for (uint32_t j = 0; j < W; j++) out[j] |= row[j];
        }
    out[W] = d.track_word && word ? 1u : 0u;
    return -1;
}

__global__ void __launch_bounds__(DFA_BLOCK) k_dfa_build(DfaDev d) {
    __shared__ uint32_t s_count;  // DFA states found, without the accept state
    __shared__ uint32_t s_over;
    __shared__ int32_t s_id[DFA_CHUNK];         // the chunk's successor ids, -1 while unnumbered
    __shared__ uint32_t s_new[DFA_CHUNK / 32];  // bit i: pair i of the chunk found no state
    const uint32_t tid = threadIdx.x, W = d.words;
    if (tid == 0) {
        s_count = 1;  // the start set, key index 0, written by the host
        s_over = 0;
        dfa_insert(d, 0);
    }
    __syncthreads();
    uint32_t lo = 0;
    // one frontier [lo, hi) a pass; the states found in a pass form the next frontier
    for (uint32_t pass = 0; pass < d.max_states && lo < s_count && !s_over; pass++) {
        const uint32_t hi = s_count;
        // acceptance at the end of the input
        for (uint32_t k = lo + tid; k < hi; k += DFA_BLOCK) {
            const uint32_t* S = d.keys + (size_t)k * (W + 1);
            const uint32_t c = (k == 0 ? 2u : 0u) | (S[W] & 1u);
            const uint32_t* m = d.endm + (size_t)c * W;
            bool eoi = false;
            for (uint32_t i = 0; i < W; i++) eoi |= (S[i] & m[i]) != 0;
            d.table[(size_t)(k + 1) * 65 + 64] = eoi ? 1 : 0;
        }
        const uint64_t pairs_end = (uint64_t)hi * 64;
        for (uint64_t base = (uint64_t)lo * 64; base < pairs_end && !s_over; base += DFA_CHUNK) {
            const uint32_t cnt = pairs_end - base < DFA_CHUNK ? (uint32_t)(pairs_end - base) : DFA_CHUNK;
            for (uint32_t w = tid; w < DFA_CHUNK / 32; w += DFA_BLOCK) s_new[w] = 0;
            __syncthreads();
            for (uint32_t i = tid; i < cnt; i += DFA_BLOCK) {
                const uint32_t k = (uint32_t)((base + i) >> 6), v = (uint32_t)((base + i) & 63);
                uint32_t* out = d.cand + (size_t)i * (W + 1);
                int32_t id = dfa_step(d, k, v, out);
                if (id < 0) id = dfa_find(d, out);
                s_id[i] = id;
                if (id < 0) atomicOr(&s_new[i >> 5], 1u << (i & 31));
            }
            __syncthreads();
            // new sets get their numbers in (state, value) order: the set bits of s_new, word by
            // word, lowest bit first
            if (tid == 0) {
                for (uint32_t wi = 0; wi < (cnt + 31) / 32 && !s_over; wi++) {
                    for (uint32_t bits = s_new[wi]; bits; bits &= bits - 1) {
                        const uint32_t i = wi * 32 + __ffs(bits) - 1;
                        const uint32_t* out = d.cand + (size_t)i * (W + 1);
                        int32_t id = dfa_find(d, out);
                        if (id < 0) {
                            if (s_count + 2 > d.max_states) {
                                s_over = 1;
                                break;
                            }
                            uint32_t* dst = d.keys + (size_t)s_count * (W + 1);
                            for (uint32_t j = 0; j <= W; j++) dst[j] = out[j];
                            dfa_insert(d, s_count);
                            s_count++;
                            id = (int32_t)s_count;
                        }
                        s_id[i] = id;
                    }
                }
            }
            __syncthreads();
            if (!s_over)
                for (uint32_t i = tid; i < cnt; i += DFA_BLOCK) {
                    const uint32_t k = (uint32_t)((base + i) >> 6), v = (uint32_t)((base + i) & 63);
                    d.table[(size_t)(k + 1) * 65 + v] = (uint16_t)s_id[i];
                }
            __syncthreads();
        }
        lo = hi;
        __syncthreads();
    }
    if (tid == 0) {
        d.result[0] = s_count + 1;
        d.result[1] = s_over;
    }
}

}  // namespace

cudaError_t build_dfa_device(const mkre::NfaTables& t, uint32_t max_states, cudaStream_t st,
                             std::vector<uint8_t>* table, uint32_t* states, bool* too_many) {
    *states = 0;
    *too_many = false;
    if (t.words == 0 || t.words > MAX_DFA_NFA_WORDS || max_states < 2) return cudaErrorInvalidValue;
    const size_t W = t.words, n = t.n;
    uint32_t hash_slots = 1;
    while (hash_slots < 2 * max_states) hash_slots <<= 1;
    // one device region: inputs, then the working arrays, each 16-byte aligned
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 15) & ~(size_t)15;
        return at;
    };
    const size_t o_plain = take(4 * n * W), o_plainm = take(4 * W), o_dec = take(t.track_word ? 4 * 8 * n * W : 0),
                 o_decm = take(4 * 8 * W), o_endm = take(4 * 4 * W), o_symto = take(4 * n), o_sym = take(8 * n);
    const size_t in_bytes = off;
    const size_t o_keys = take(4 * (size_t)max_states * (W + 1)), o_cand = take(4 * (size_t)DFA_CHUNK * (W + 1)),
                 o_hash = take(4 * (size_t)hash_slots),
                 o_table = take(2 * (size_t)max_states * 65), o_res = take(8);
    std::vector<uint8_t> in(in_bytes, 0);
    auto put = [&](size_t at, const void* src, size_t bytes) {
        if (bytes) memcpy(in.data() + at, src, bytes);
    };
    put(o_plain, t.plain.data(), 4 * n * W);
    put(o_plainm, t.plainm.data(), 4 * W);
    if (t.track_word) put(o_dec, t.dec.data(), 4 * 8 * n * W);
    put(o_decm, t.decm.data(), 4 * 8 * W);
    put(o_endm, t.endm.data(), 4 * 4 * W);
    put(o_symto, t.sym_to.data(), 4 * n);
    put(o_sym, t.sym.data(), 8 * n);
    std::vector<uint32_t> k0(W + 1);
    for (size_t i = 0; i < W; i++) k0[i] = t.k0[i];
    k0[W] = t.track_start ? 2u : 0u;

    uint8_t* base = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&base, off, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(base, in.data(), in_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + o_hash, 0, 4 * (size_t)hash_slots, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + o_table, 0, 2 * (size_t)max_states * 65, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + o_keys, k0.data(), 4 * (W + 1), cudaMemcpyHostToDevice, st);
    DfaDev d;
    d.n = t.n;
    d.words = t.words;
    d.track_word = t.track_word ? 1 : 0;
    d.max_states = max_states;
    d.hash_mask = hash_slots - 1;
    d.start = t.start;
    d.match = t.match;
    d.plain = (const uint32_t*)(base + o_plain);
    d.plainm = (const uint32_t*)(base + o_plainm);
    d.dec = (const uint32_t*)(base + o_dec);
    d.decm = (const uint32_t*)(base + o_decm);
    d.endm = (const uint32_t*)(base + o_endm);
    d.sym_to = (const int32_t*)(base + o_symto);
    d.sym = (const uint64_t*)(base + o_sym);
    d.keys = (uint32_t*)(base + o_keys);
    d.cand = (uint32_t*)(base + o_cand);
    d.hash = (uint32_t*)(base + o_hash);
    d.table = (uint16_t*)(base + o_table);
    d.result = (uint32_t*)(base + o_res);
    if (e == cudaSuccess) {
        k_dfa_build<<<1, DFA_BLOCK, 0, st>>>(d);
        e = cudaGetLastError();
    }
    uint32_t res[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(res, d.result, sizeof(res), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && !res[1] && res[0] >= 2 && res[0] <= max_states) {
        table->assign((size_t)res[0] * 130, 0);
        e = cudaMemcpyAsync(table->data(), d.table, (size_t)res[0] * 130, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) {
            // row 0: the absorbing accept state (every value stays, accepts at the end)
            for (int v = 0; v < 65; v++) {
                (*table)[v * 2] = v == 64 ? 1 : 0;
                (*table)[v * 2 + 1] = 0;
            }
            *states = res[0];
        }
    }
    *too_many = e == cudaSuccess && res[1] != 0;
    const cudaError_t ef = cudaFreeAsync(base, st);
    return e != cudaSuccess ? e : ef;
}

}  // namespace mkb
