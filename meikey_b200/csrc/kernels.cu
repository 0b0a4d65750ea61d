// sm_100a kernels of the candidate-key search path.
//
//   k_build_table  fills the comb table in HBM: entry (row, k) = k·2^(off_row)·8B
//                  (+ 2^254·B on the top row), affine (y+x, y-x, 2dxy), row 0 holds 2xy.
//   k_keys<…>      one fused pass per key: seed (ChaCha20 / counter) -> SHA-512 -> clamp
//                  -> comb multiply from the table -> y as a fraction -> per-thread
//                  Montgomery batch + per-CTA pooled inversion -> canonical y -> base64
//                  values -> shift-and / DFA match -> warp-ballot hit compaction.
//                  The DERIVE instantiation also computes x and writes full public keys.
//
// Reference behaviour: src/service/gpu/kernel.cu:1898-2069 (meikey_search / meikey_derive).
// The index layout matches it: index = base + ((it·nthreads + gid)·KPT + j).
#include <cuda_runtime.h>
#include <stdint.h>

#include "ge.cuh"
#include "hash.cuh"
#include "kernels.h"

namespace mkb {

using mk32::fe;
using mk32::ge;
using mk32::niels;
using mk32::u32;
using mk32::u64;

// ---------------------------------------------------------------------------
// shared helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ fe load_fe(const uint4* p) {
    uint4 a = __ldg(p), b = __ldg(p + 1);
    fe r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}

__device__ __forceinline__ niels load_entry(const uint4* table, u64 idx) {
    const uint4* e = table + idx * (ENTRY_WORDS / 4);
    niels n;
    n.ypx = load_fe(e);
    n.ymx = load_fe(e + 2);
    n.t2d = load_fe(e + 4);
    return n;
}

// bits [off, off+w) of the 256-bit value m (w <= 32)
__device__ __forceinline__ u32 bits_at(const u64 m[4], u32 off, u32 w) {
    u32 q = off >> 6, r = off & 63;
    u64 lo = q == 0 ? m[0] : q == 1 ? m[1] : q == 2 ? m[2] : m[3];
    u64 hi = q == 0 ? m[1] : q == 1 ? m[2] : q == 2 ? m[3] : 0ull;
    u64 v = lo >> r;
    if (r != 0) v |= hi << (64 - r);
    return (u32)(v & ((1ull << w) - 1ull));
}

// ---------------------------------------------------------------------------
// comb table build
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_build_table(uint4* table, const CombGeom g, const u32* __restrict__ points,
                                                     u64 first, u64 count) {
    u64 e = first + (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= first + count || e >= g.entries) return;
    u32 row = 0;
    for (u32 i = 1; i < g.rows; i++)
        if (e >= g.row_base[i]) row = i;
    u64 k = e - g.row_base[row];
    // points: per row R (X,Y,Z,T) then O (X,Y,Z,T), 8 words each; then 2d
    const u32* pr = points + (u64)row * 64;
    ge R, O;
    fe* rf[4] = {&R.X, &R.Y, &R.Z, &R.T};
    fe* of[4] = {&O.X, &O.Y, &O.Z, &O.T};
    for (int c = 0; c < 4; c++)
        for (int i = 0; i < 8; i++) {
            rf[c]->v[i] = pr[8 * c + i];
            of[c]->v[i] = pr[32 + 8 * c + i];
        }
    fe d2;
    for (int i = 0; i < 8; i++) d2.v[i] = points[(u64)g.rows * 64 + i];
    ge P = mk32::ge_identity();
    u32 nbits = 0;
    while (nbits < 63 && (g.cols[row] - 1) >> nbits) nbits++;
    for (int b = (int)nbits - 1; b >= 0; b--) {
        P = mk32::ge_add(P, P, d2);
        ge Q = mk32::ge_add(P, R, d2);
        if ((k >> b) & 1) P = Q;
    }
    P = mk32::ge_add(P, O, d2);
    fe zi = mk32::fe_invert(P.Z);
    fe x = mk32::fe_mul(P.X, zi), y = mk32::fe_mul(P.Y, zi);
    fe xy = mk32::fe_mul(x, y);
    fe t = row == 0 ? mk32::fe_add(xy, xy) : mk32::fe_mul(xy, d2);
    u32 w[24];
    mk32::fe_to_words(mk32::fe_add(y, x), w);
    mk32::fe_to_words(mk32::fe_sub(y, x), w + 8);
    mk32::fe_to_words(t, w + 16);
    uint4* out = table + e * (ENTRY_WORDS / 4);
#pragma unroll
    for (int q = 0; q < 6; q++) out[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

// ---------------------------------------------------------------------------
// the fused key kernel
// ---------------------------------------------------------------------------

// Comb multiply: s (clamped, 4 LE words) -> y = yn/yd (and x = xn/xd when wanted).
__device__ __forceinline__ void comb_mul(const uint4* __restrict__ table, const CombGeom& g, const u64 s[4], fe& yn,
                                         fe& yd, fe* xn, fe* xd) {
    // m = bits 3..253 of s
    u64 m[4];
    m[0] = s[0] >> 3 | s[1] << 61;
    m[1] = s[1] >> 3 | s[2] << 61;
    m[2] = s[2] >> 3 | s[3] << 61;
    m[3] = (s[3] >> 3) & ((1ull << (251 - 192)) - 1ull);
    const u32 rows = g.rows;
    int carry = 0;
    // row 0 -> extended coordinates (X = 2x, Y = 2y, Z = 2, T = 2xy)
    ge P;
    {
        u32 w = g.width[0];
        int v = (int)bits_at(m, g.offset[0], w) + carry;
        int half = 1 << (w - 1);
        carry = (v + half) >> w;
        int d = v - (carry << w);
        bool neg = d < 0;
        u32 ad = neg ? (u32)(-d) : (u32)d;
        niels n = load_entry(table, g.row_base[0] + ad);
        mk32::fe_cswap(n.ypx, n.ymx, neg);
        P.X = mk32::fe_sub(n.ypx, n.ymx);
        P.Y = mk32::fe_add(n.ypx, n.ymx);
        P.Z = mk32::fe_small(2);
        fe nt = mk32::fe_sub(mk32::fe_zero(), n.t2d);
#pragma unroll
        for (int i = 0; i < 8; i++) P.T.v[i] = neg ? nt.v[i] : n.t2d.v[i];
    }
#pragma unroll 1
    for (u32 row = 1; row + 1 < rows; row++) {
        u32 w = g.width[row];
        int v = (int)bits_at(m, g.offset[row], w) + carry;
        int half = 1 << (w - 1);
        carry = (v + half) >> w;
        int d = v - (carry << w);
        bool neg = d < 0;
        u32 ad = neg ? (u32)(-d) : (u32)d;
        niels n = load_entry(table, g.row_base[row] + ad);
        P = mk32::ge_add_niels(P, n, neg);
    }
    {
        u32 row = rows - 1;
        int d = (int)bits_at(m, g.offset[row], g.width[row]) + carry;  // in [0, 2^w_top]
        niels n = load_entry(table, g.row_base[row] + (u32)d);
        mk32::ge_add_niels_frac(P, n, yn, yd, xn, xd);
    }
}

// 6-bit values of the 44-character base64 tail of the key blob (0x20 then the key),
// from the key's 8 little-endian words; only positions 1..43 are searched.
__device__ __forceinline__ u32 tail_value(const u32 pk[8], int pos) {
    // group g covers bytes b0 = (g ? pk[3g-1] : 0x20), pk[3g], pk[3g+1]
    int g = pos >> 2, k = pos & 3;
    auto byte = [&](int i) -> u32 { return (pk[i >> 2] >> (8 * (i & 3))) & 0xffu; };
    u32 b0 = g == 0 ? 32u : byte(3 * g - 1);
    u32 b1 = byte(3 * g);
    u32 b2 = 3 * g + 1 < 32 ? byte(3 * g + 1) : 0u;
    u32 n = b0 << 16 | b1 << 8 | b2;
    return (n >> (18 - 6 * k)) & 63u;
}

#define MK_SIGN_POS 42

// Tests one key (y only; the character at position 42 is tried with both x signs, as
// kernel.cu:1804-1875 does) and sets bit `id` of hit_words for every needle that may match.
__device__ __forceinline__ void match_key(const MatchSet& ms, const u32 pk[8], u64 hit_words[2]) {
    hit_words[0] = hit_words[1] = 0;
    u32 vals[44];
#pragma unroll
    for (int pos = 1; pos < 44; pos++) vals[pos] = tail_value(pk, pos);
    // text needles: shift-and over sa_words words of state
    for (u32 wi = 0; wi < ms.sa_words; wi++) {
        u64 D = 0, acc = 0;
        u64 first = ms.first_bit[wi], last = ms.last_bit[wi];
#pragma unroll
        for (int pos = 1; pos < 44; pos++) {
            u64 mk = ms.mask[vals[pos]][wi];
            if (pos == MK_SIGN_POS) mk |= ms.mask[vals[pos] | 2u][wi];
            D = ((D << 1) | first) & mk;
            acc |= D & last;
        }
        acc |= D & ms.suffix_bit[wi];
        if (acc) {
            // map bits to needles
            for (u32 t = 0; t < ms.n_text; t++) {
                u32 b = ms.text_last[t];
                if ((b >> 6) == wi && ((acc >> (b & 63)) & 1)) {
                    u32 id = ms.text_id[t];
                    hit_words[id >> 6] |= 1ull << (id & 63);
                }
            }
        }
    }
    for (u32 r = 0; r < ms.n_regex; r++) {
        const uint8_t* t = ms.dfa[r];
        auto next = [&](u32 s, u32 i) -> u32 {
            u64 at = ((u64)s * 65u + i) * 2u;
            return (u32)__ldg(t + at) | (u32)__ldg(t + at + 1) << 8;
        };
        u32 s = 1, alt = 1;
#pragma unroll 1
        for (int pos = 1; pos < 44; pos++) {
            u32 v = vals[pos];
            if (pos == MK_SIGN_POS) alt = next(s, v | 2u);
            else if (pos > MK_SIGN_POS) alt = next(alt, v);
            s = next(s, v);
        }
        bool ok = s == 0 || next(s, 64) != 0 || alt == 0 || next(alt, 64) != 0;
        if (ok) {
            u32 id = ms.regex_id[r];
            hit_words[id >> 6] |= 1ull << (id & 63);
        }
    }
}

// Warp-compacted hit output: lanes with hits take consecutive ring slots with one
// atomicAdd per warp (inclusive scan of the per-lane hit counts).  Called by all 32 lanes.
__device__ __forceinline__ void report_hits(const u64 hw[2], u64 index, HitRecord* hits, u32 cap, JobDevice* jd) {
    const u32 lane = threadIdx.x & 31u;
    u32 cnt = (u32)(__popcll(hw[0]) + __popcll(hw[1]));
    u32 incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (u32)o) incl += y;
    }
    u32 total = __shfl_sync(0xffffffffu, incl, 31);
    u32 base = 0;
    if (lane == 31) base = atomicAdd(&jd->hit_count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    u32 slot = base + incl - cnt;
    for (int w = 0; w < 2; w++) {
        u64 bits = hw[w];
        while (bits) {
            int b = __ffsll((long long)bits) - 1;
            bits &= bits - 1;
            if (slot < cap) {
                hits[slot].index = index;
                hits[slot].needle = (u32)(w * 64 + b);
                hits[slot].reserved = 0;
            }
            slot++;
        }
    }
}

template <int KPT, int BLOCK, bool DERIVE>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK) k_keys(const KeyLaunch L) {
    constexpr int NUM = DERIVE ? 2 * KPT : KPT;
    constexpr int GROUPS = BLOCK / 32;
    __shared__ fe pool[2][BLOCK];
    __shared__ CombGeom g;
    __shared__ MatchSet ms;
    __shared__ u32 key[8];
    const u32 tid = threadIdx.x;
    const u64 gid = (u64)blockIdx.x * BLOCK + tid;
    const u64 nthreads = (u64)gridDim.x * BLOCK;
    // stage launch constants in shared memory
    {
        const u32* src = (const u32*)&L.geom;
        u32* dst = (u32*)&g;
        for (u32 i = tid; i < sizeof(CombGeom) / 4; i += BLOCK) dst[i] = src[i];
        if (!DERIVE) {
            const u32* s2 = (const u32*)L.match;
            u32* d2 = (u32*)&ms;
            for (u32 i = tid; i < sizeof(MatchSet) / 4; i += BLOCK) d2[i] = s2[i];
        }
        if (tid < 8) key[tid] = L.key[tid];
    }
    __syncthreads();
    mkh::CounterMid mid;
    if (L.seed_src == 1) mid = mkh::counter_mid(key);

    const u32 iters = DERIVE ? 1u : L.iters;
    u32 sink = 0;
    for (u32 it = 0; it < iters; it++) {
        if (!DERIVE) {
            bool stop = false;
            if (tid == 0) {
                volatile JobDevice* jd = L.job;
                stop = jd->stop != 0 || (L.stop_on_hit && jd->hit_count != 0);
            }
            if (__syncthreads_or(stop)) {
                if (tid == 0) atomicOr(&L.job->status, 1u);
                break;
            }
        }
        const u64 first = L.base + ((u64)it * nthreads + gid) * KPT;
        fe num[NUM], den[NUM], pre[NUM];
        u32 blk[16];
        u64 blk_id = ~0ull;
#pragma unroll 1
        for (int j = 0; j < KPT; j++) {
            const u64 idx = first + (u64)j;
            u64 s[4];
            if (L.seed_src == 1) {
                mkh::counter_scalar(mid, idx, s);
            } else {
                if ((idx >> 1) != blk_id) {
                    blk_id = idx >> 1;
                    mkh::chacha20_block(key, blk_id, blk);
                }
                u32 sw[8];
                const bool odd = idx & 1;
#pragma unroll
                for (int i = 0; i < 8; i++) sw[i] = odd ? blk[8 + i] : blk[i];
                mkh::seed_scalar(sw, s);
            }
            if (DERIVE) {
                comb_mul(L.table, g, s, num[2 * j], den[2 * j], &num[2 * j + 1], &den[2 * j + 1]);
                pre[2 * j] = j == 0 ? den[0] : mk32::fe_mul(pre[2 * j - 1], den[2 * j]);
                pre[2 * j + 1] = mk32::fe_mul(pre[2 * j], den[2 * j + 1]);
            } else {
                comb_mul(L.table, g, s, num[j], den[j], nullptr, nullptr);
                pre[j] = j == 0 ? den[0] : mk32::fe_mul(pre[j - 1], den[j]);
            }
        }
        // pooled inversion: lane L of warp 0 inverts the products of threads L, L+32, ...
        const int buf = it & 1;
        pool[buf][tid] = pre[NUM - 1];
        __syncthreads();
        if (tid < 32) {
            fe acc = pool[buf][tid];
            pool[buf ^ 1][tid] = acc;
#pragma unroll 1
            for (int k = 1; k < GROUPS; k++) {
                acc = mk32::fe_mul(acc, pool[buf][tid + 32 * k]);
                pool[buf ^ 1][tid + 32 * k] = acc;
            }
            fe inv = mk32::fe_invert(acc);
#pragma unroll 1
            for (int k = GROUPS - 1; k > 0; k--) {
                fe t = mk32::fe_mul(inv, pool[buf ^ 1][tid + 32 * (k - 1)]);
                inv = mk32::fe_mul(inv, pool[buf][tid + 32 * k]);
                pool[buf][tid + 32 * k] = t;
            }
            pool[buf][tid] = inv;
        }
        __syncthreads();
        fe inv = pool[buf][tid];
        // back-sweep: element e's inverse is inv·pre[e-1]; then inv·den[e] moves to e-1
#pragma unroll 1
        for (int j = KPT - 1; j >= 0; j--) {
            const u64 idx = first + (u64)j;
            u32 pk[8];
            if (DERIVE) {
                const int ex = 2 * j + 1, ey = 2 * j;
                fe xinv = mk32::fe_mul(inv, pre[ex - 1]);
                inv = mk32::fe_mul(inv, den[ex]);
                fe yinv = ey == 0 ? inv : mk32::fe_mul(inv, pre[ey - 1]);
                if (ey > 0) inv = mk32::fe_mul(inv, den[ey]);
                u32 xw[8];
                mk32::fe_to_words(mk32::fe_mul(num[ex], xinv), xw);
                mk32::fe_to_words(mk32::fe_mul(num[ey], yinv), pk);
                pk[7] |= (xw[0] & 1u) << 31;
                if (idx - L.base < L.count) {
                    uint4* o = (uint4*)(L.out + (idx - L.base) * 32);
                    o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
            } else {
                fe zinv = j == 0 ? inv : mk32::fe_mul(inv, pre[j - 1]);
                if (j > 0) inv = mk32::fe_mul(inv, den[j]);
                mk32::fe_to_words(mk32::fe_mul(num[j], zinv), pk);
                sink ^= pk[7];
                u64 hw[2];
                match_key(ms, pk, hw);
                const bool any = (hw[0] | hw[1]) != 0;
                // warp ballot: the (rare) warps with a hit compact their records into the ring
                if (__ballot_sync(0xffffffffu, any)) report_hits(hw, idx, L.hits, L.hit_cap, L.job);
            }
        }
    }
    if (!DERIVE && L.sink) L.sink[gid] = sink;
}

// ---------------------------------------------------------------------------
// host launch wrappers
// ---------------------------------------------------------------------------

template <int KPT, int BLOCK>
static cudaError_t launch_keys_t(const KeyLaunch& L, bool derive, uint32_t grid, cudaStream_t st) {
    if (derive) k_keys<KPT, BLOCK, true><<<grid, BLOCK, 0, st>>>(L);
    else k_keys<KPT, BLOCK, false><<<grid, BLOCK, 0, st>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_keys(const KeyLaunch& L, bool derive, uint32_t kpt, uint32_t block, uint32_t grid, cudaStream_t st) {
    if (block == 256) {
        switch (kpt) {
            case 4: return launch_keys_t<4, 256>(L, derive, grid, st);
            case 8: return launch_keys_t<8, 256>(L, derive, grid, st);
            case 16: return launch_keys_t<16, 256>(L, derive, grid, st);
        }
    } else if (block == 128) {
        switch (kpt) {
            case 4: return launch_keys_t<4, 128>(L, derive, grid, st);
            case 8: return launch_keys_t<8, 128>(L, derive, grid, st);
            case 16: return launch_keys_t<16, 128>(L, derive, grid, st);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t keys_occupancy(bool derive, uint32_t kpt, uint32_t block, int* blocks_per_sm) {
    const void* f = nullptr;
#define MK_OCC(K, B)                                                                       \
    if (kpt == K && block == B)                                                            \
        f = derive ? (const void*)k_keys<K, B, true> : (const void*)k_keys<K, B, false>;
    MK_OCC(4, 256) MK_OCC(8, 256) MK_OCC(16, 256) MK_OCC(4, 128) MK_OCC(8, 128) MK_OCC(16, 128)
#undef MK_OCC
    if (!f) return cudaErrorInvalidValue;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, (int)block, 0);
}

cudaError_t launch_build_table(uint4* table, const CombGeom& g, const uint32_t* points, uint64_t first,
                               uint64_t count, cudaStream_t st) {
    uint32_t blocks = (uint32_t)((count + 255) / 256);
    k_build_table<<<blocks, 256, 0, st>>>(table, g, points, first, count);
    return cudaGetLastError();
}

}  // namespace mkb
