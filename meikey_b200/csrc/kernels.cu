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

#include <algorithm>
#include <vector>

#include "ge.cuh"
#include "hash.cuh"
#include "kernels.h"

namespace mkb {

using mk32::fe;
using mk32::ge;
using mk32::niels;
using mk32::u32;
using mk32::u64;

// Field-multiply form of the secure path (comb additions, thread batches and back-sweep): one
// level of Karatsuba, 48 lo + 48 hi products a multiplication instead of 64 + 64, with the same
// results.  On B200 it is the faster form there; the incremental path, with few multiplies
// between its other work, runs faster with the schoolbook form and keeps it.
constexpr bool SECURE_KARATSUBA = true;

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
    uint4* out = table + e * (COMB_STRIDE_WORDS / 4);
#pragma unroll
    for (int q = 0; q < 6; q++) out[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
#pragma unroll
    for (int q = 6; q < COMB_STRIDE_WORDS / 4; q++) out[q] = make_uint4(0, 0, 0, 0);
}

// ---------------------------------------------------------------------------
// the fused key kernel
// ---------------------------------------------------------------------------

// Per-thread staging slots for the comb table: entry of row r is fetched with cp.async
// (16-byte LDGSTS, L2 only) into slot r & 1 one row ahead of its use.
struct EntrySlot {
    uint4 q[2][6];
};

__device__ __forceinline__ void fetch_entry(EntrySlot& slot, int which, const uint4* table, u64 idx) {
    const uint4* src = table + idx * (COMB_STRIDE_WORDS / 4);
    u32 dst = (u32)__cvta_generic_to_shared(&slot.q[which][0]);
#pragma unroll
    for (int q = 0; q < 6; q++)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16 * q), "l"(src + q) : "memory");
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void wait_entries() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ niels read_entry(const EntrySlot& slot, int which) {
    niels n;
    const uint4* q = slot.q[which];
    uint4 a;
    a = q[0]; n.ypx.v[0] = a.x; n.ypx.v[1] = a.y; n.ypx.v[2] = a.z; n.ypx.v[3] = a.w;
    a = q[1]; n.ypx.v[4] = a.x; n.ypx.v[5] = a.y; n.ypx.v[6] = a.z; n.ypx.v[7] = a.w;
    a = q[2]; n.ymx.v[0] = a.x; n.ymx.v[1] = a.y; n.ymx.v[2] = a.z; n.ymx.v[3] = a.w;
    a = q[3]; n.ymx.v[4] = a.x; n.ymx.v[5] = a.y; n.ymx.v[6] = a.z; n.ymx.v[7] = a.w;
    a = q[4]; n.t2d.v[0] = a.x; n.t2d.v[1] = a.y; n.t2d.v[2] = a.z; n.t2d.v[3] = a.w;
    a = q[5]; n.t2d.v[4] = a.x; n.t2d.v[5] = a.y; n.t2d.v[6] = a.z; n.t2d.v[7] = a.w;
    return n;
}

// signed digit of row `row` (rows before the top one), updating the carry
__device__ __forceinline__ int next_digit(const CombGeom& g, const u64 m[4], u32 row, int& carry) {
    u32 w = g.width[row];
    int v = (int)bits_at(m, g.offset[row], w) + carry;
    carry = (v + (1 << (w - 1))) >> w;
    return v - (carry << w);
}

__device__ __forceinline__ u64 entry_index(const CombGeom& g, u32 row, int d) {
    return g.row_base[row] + (u64)(d < 0 ? -d : d);
}

// bits 3..253 of a clamped scalar s: the number whose digits the comb rows take
__device__ __forceinline__ void comb_m(const u64 s[4], u64 m[4]) {
    m[0] = s[0] >> 3 | s[1] << 61;
    m[1] = s[1] >> 3 | s[2] << 61;
    m[2] = s[2] >> 3 | s[3] << 61;
    m[3] = (s[3] >> 3) & ((1ull << (251 - 192)) - 1ull);
}

// Row 0's entry (digit sign `neg`) in extended coordinates: X = 2x, Y = 2y, Z = 2, T = 2xy,
// without a multiplication (row 0 stores 2xy).
__device__ __forceinline__ ge comb_row0(niels n, bool neg) {
    ge P;
    mk32::fe_cswap(n.ypx, n.ymx, neg);
    P.X = mk32::fe_sub(n.ypx, n.ymx);
    P.Y = mk32::fe_add(n.ypx, n.ymx);
    P.Z = mk32::fe_small(2);
    fe nt = mk32::fe_sub(mk32::fe_zero(), n.t2d);
#pragma unroll
    for (int i = 0; i < 8; i++) P.T.v[i] = neg ? nt.v[i] : n.t2d.v[i];
    return P;
}

// Comb multiply: s (clamped, 4 LE words) -> y = yn/yd (and x = xn/xd when wanted).
// Row r's entry is fetched while row r-1 is being added.
__device__ __forceinline__ void comb_mul(const uint4* __restrict__ table, const CombGeom& g, const u64 s[4],
                                         EntrySlot& slot, fe& yn, fe& yd, fe* xn, fe* xd) {
    u64 m[4];
    comb_m(s, m);
    const u32 rows = g.rows;
    int carry = 0;
    int d0 = next_digit(g, m, 0, carry);
    fetch_entry(slot, 0, table, entry_index(g, 0, d0));
    int dn = next_digit(g, m, 1, carry);  // rows >= 3, so row 1 is not the top row
    fetch_entry(slot, 1, table, entry_index(g, 1, dn));
    wait_entries<1>();
    ge P = comb_row0(read_entry(slot, 0), d0 < 0);
#pragma unroll 1
    for (u32 row = 1; row + 1 < rows; row++) {
        const int d = dn;
        // prefetch row+1 (the top row's digit is unsigned: the carry lands in it unchanged)
        if (row + 2 < rows) dn = next_digit(g, m, row + 1, carry);
        else dn = (int)bits_at(m, g.offset[row + 1], g.width[row + 1]) + carry;
        fetch_entry(slot, (row + 1) & 1, table, entry_index(g, row + 1, dn));
        wait_entries<1>();
        niels n = read_entry(slot, row & 1);
        P = mk32::ge_add_niels<SECURE_KARATSUBA>(P, n, d < 0);
    }
    wait_entries<0>();
    niels n = read_entry(slot, (rows - 1) & 1);
    mk32::ge_add_niels_frac<SECURE_KARATSUBA>(P, n, yn, yd, xn, xd);
}

// comb_mul with one 8-round step of the SHA-512 `run` (the next iteration's seed) in every
// full-addition row, in the same straight-line block as the row's field multiplies, so that
// the hashing (ALU pipe) issues between the multiplies (IMAD pipe).  Built for 12 rows: the
// 10 full rows carry the 80 rounds.  y = yn/yd only.
__device__ __forceinline__ void comb_mul_sha(const uint4* __restrict__ table, const CombGeom& g, const u64 s[4],
                                             EntrySlot& slot, fe& yn, fe& yd, mkh::ShaRun& run) {
    u64 m[4];
    comb_m(s, m);
    const u32 rows = g.rows;
    int carry = 0;
    int d0 = next_digit(g, m, 0, carry);
    fetch_entry(slot, 0, table, entry_index(g, 0, d0));
    int dn = next_digit(g, m, 1, carry);
    fetch_entry(slot, 1, table, entry_index(g, 1, dn));
    wait_entries<1>();
    ge P = comb_row0(read_entry(slot, 0), d0 < 0);
#pragma unroll 1
    for (u32 row = 1; row + 1 < rows; row++) {
        const int d = dn;
        // the next row's digit without a branch (the top row's is unsigned: the carry lands
        // in it unchanged)
        int c2 = carry;
        const int sd = next_digit(g, m, row + 1, c2);
        const int td = (int)bits_at(m, g.offset[row + 1], g.width[row + 1]) + carry;
        const bool top = row + 2 >= rows;
        dn = top ? td : sd;
        carry = top ? carry : c2;
        fetch_entry(slot, (row + 1) & 1, table, entry_index(g, row + 1, dn));
        wait_entries<1>();
        niels n = read_entry(slot, row & 1);
        mkh::sha_run_step(run, 8u * (row - 1));
        P = mk32::ge_add_niels<SECURE_KARATSUBA>(P, n, d < 0);
    }
    wait_entries<0>();
    niels n = read_entry(slot, (rows - 1) & 1);
    mk32::ge_add_niels_frac<SECURE_KARATSUBA>(P, n, yn, yd, nullptr, nullptr);
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
// `lane_masks` (null: none) holds, for jobs whose text needles fit in 32 bits of state, the
// low half of mask word 0 once per lane (value v of lane l at v * 32 + l): every lane reads
// its own bank.
__device__ __forceinline__ void match_key(const MatchSet& ms, const u32* lane_masks, const u32 pk[8],
                                          u64 hit_words[2]) {
    hit_words[0] = hit_words[1] = 0;
    u32 vals[44];
#pragma unroll
    for (int pos = 1; pos < 44; pos++) vals[pos] = tail_value(pk, pos);
    // text needles: shift-and over sa_words words of state.  With the 4-gram prefilter, the
    // words of the needles of 4+ characters are scanned only when one of the key's 4-character
    // windows (position 42 with both values) is the start of such a needle.
    u32 words = ms.sa_words;
    if (ms.gram4) {
        u32 any = 0, gw = vals[1] << 12 | vals[2] << 6 | vals[3];
#pragma unroll
        for (int p = 1; p + 3 < 44; p++) {
            gw = (gw << 6 | vals[p + 3]) & 0xffffffu;
            any |= __ldg(ms.gram4 + (gw >> 5)) >> (gw & 31);
            if (p <= MK_SIGN_POS && MK_SIGN_POS <= p + 3) {
                const u32 g2 = gw | 2u << (6 * (p + 3 - MK_SIGN_POS));
                any |= __ldg(ms.gram4 + (g2 >> 5)) >> (g2 & 31);
            }
        }
        if (!(any & 1u)) words = ms.short_words;
    }
    if (lane_masks && words) {
        const u32* lm = lane_masks + (threadIdx.x & 31u);
        u32 D = 0, acc = 0;
        const u32 first = (u32)ms.first_bit[0], last = (u32)ms.last_bit[0];
#pragma unroll
        for (int pos = 1; pos < 44; pos++) {
            u32 mk = lm[vals[pos] * 32u];
            if (pos == MK_SIGN_POS) mk |= lm[(vals[pos] | 2u) * 32u];
            D = ((D << 1) | first) & mk;
            acc |= D & last;
        }
        acc |= D & (u32)ms.suffix_bit[0];
        for (u32 t = 0; acc && t < ms.n_text; t++) {
            const u32 b = ms.text_last[t];
            if ((acc >> b) & 1u) {
                const u32 id = ms.text_id[t];
                hit_words[id >> 6] |= 1ull << (id & 63);
            }
        }
        words = 0;
    }
    for (u32 wi = 0; wi < words; wi++) {
        u64 D = 0, acc = 0;
        u64 first = ms.first_bit[wi], last = ms.last_bit[wi];
#pragma unroll
        for (int pos = 1; pos < 44; pos++) {
            u64 mk = ms.mask[wi][vals[pos]];
            if (pos == MK_SIGN_POS) mk |= ms.mask[wi][vals[pos] | 2u];
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
    // regex needles: eight DFA walks side by side, so that their table lookups (shared
    // memory when the launch staged the tables there, else global) overlap
    for (u32 r0 = 0; r0 < ms.n_regex; r0 += 8) {
        const uint16_t* t[8];
        u32 s[8], alt[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            t[q] = reinterpret_cast<const uint16_t*>(ms.dfa[r0 + q < ms.n_regex ? r0 + q : r0]);
            s[q] = alt[q] = 1;
        }
#pragma unroll 1
        for (int pos = 1; pos < 44; pos++) {
            const u32 v = tail_value(pk, pos);
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (pos == MK_SIGN_POS) alt[q] = t[q][s[q] * 65u + (v | 2u)];
                else if (pos > MK_SIGN_POS) alt[q] = t[q][alt[q] * 65u + v];
                s[q] = t[q][s[q] * 65u + v];
            }
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const u32 r = r0 + q;
            if (r >= ms.n_regex) break;
            const bool ok = s[q] == 0 || t[q][s[q] * 65u + 64u] != 0 || alt[q] == 0 || t[q][alt[q] * 65u + 64u] != 0;
            if (!ok) continue;
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

// Seed of index `idx` -> clamped scalar.  `blk`/`blk_id` cache the ChaCha20 block
// shared by an even index and the next odd one.
__device__ __forceinline__ void scalar_of(u32 seed_src, const u32 key[8], const mkh::CounterMid& mid, u64 idx,
                                          u32 blk[16], u64& blk_id, u64 s[4]) {
    if (seed_src == 1) {
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
}

// Batch state of one iteration of one thread (Montgomery's trick with two field elements
// per key): a[j] = num_j · den_0 ··· den_(j-1) and den[j]; `prod` = den_0 ··· den_(KPT-1).
// With inv = 1/prod the back-sweep gives y_j = a[j] · inv_j, inv_(j-1) = inv_j · den[j].
template <int KPT>
struct Batch {
    fe a[KPT], den[KPT];
    fe prod;
};

// Seeds and clamped scalars of KPT consecutive indices (ALU work: ChaCha20, SHA-512).
template <int KPT>
__device__ __forceinline__ void scalars(const KeyLaunch& L, const u32 key[8], const mkh::CounterMid& mid, u64 first,
                                        u64 sc[KPT][4]) {
    u32 blk[16];
    u64 blk_id = ~0ull;
#pragma unroll 1
    for (int j = 0; j < KPT; j++) scalar_of(L.seed_src, key, mid, first + (u64)j, blk, blk_id, sc[j]);
}

__device__ __forceinline__ niels smem_niels(const uint4* q);

// Comb multiply with the whole table in shared memory (entries 96 bytes apart, `stab`): every
// row reads its entry there, with no staging; y = yn/yd only.
__device__ __forceinline__ void comb_mul_smem(const uint4* stab, const CombGeom& g, const u64 s[4], fe& yn, fe& yd) {
    u64 m[4];
    comb_m(s, m);
    const u32 rows = g.rows;
    int carry = 0;
    int d = next_digit(g, m, 0, carry);
    ge P = comb_row0(smem_niels(stab + entry_index(g, 0, d) * 6), d < 0);
#pragma unroll 1
    for (u32 row = 1; row + 1 < rows; row++) {
        d = next_digit(g, m, row, carry);
        P = mk32::ge_add_niels<SECURE_KARATSUBA>(P, smem_niels(stab + entry_index(g, row, d) * 6), d < 0);
    }
    // the top row's digit is unsigned: the carry lands in it unchanged
    d = (int)bits_at(m, g.offset[rows - 1], g.width[rows - 1]) + carry;
    mk32::ge_add_niels_frac<SECURE_KARATSUBA>(P, smem_niels(stab + entry_index(g, rows - 1, d) * 6), yn, yd, nullptr, nullptr);
}

// Comb multiplies of the KPT scalars (IMAD work) into the batch; STAB: from the table in
// shared memory.
template <int KPT, bool STAB = false>
__device__ __forceinline__ void combs(const KeyLaunch& L, const CombGeom& g, const u64 sc[KPT][4], EntrySlot& slot,
                                      const uint4* stab, Batch<KPT>& b) {
    fe run;
#pragma unroll 1
    for (int j = 0; j < KPT; j++) {
        fe num;
        if (STAB) comb_mul_smem(stab, g, sc[j], num, b.den[j]);
        else comb_mul(L.table, g, sc[j], slot, num, b.den[j], nullptr, nullptr);
        if (j == 0) {
            b.a[0] = num;
            run = b.den[0];
        } else {
            b.a[j] = mk32::fe_mul_as<SECURE_KARATSUBA>(num, run);
            run = mk32::fe_mul_as<SECURE_KARATSUBA>(run, b.den[j]);
        }
    }
    b.prod = run;
}

// Comb multiplies of this iteration's KPT scalars (sc) with the SHA-512 of the next
// iteration's seeds (indices next_first + j) carried through their rows: key j's comb reads
// sc[j] at its start and leaves the next iteration's scalar of key j there.  ChaCha20 blocks
// serve an even index and the next odd one (the other half is kept).
template <int KPT>
__device__ __forceinline__ void combs_sha(const KeyLaunch& L, const CombGeom& g, u64 sc[KPT][4], EntrySlot& slot,
                                          Batch<KPT>& b, const u32 key[8], const mkh::CounterMid& mid,
                                          u64 next_first) {
    fe run;
    u32 other[8];
    u64 other_id = ~0ull;
#pragma unroll 1
    for (int j = 0; j < KPT; j++) {
        const u64 idx = next_first + (u64)j;
        u64 w4[4];
        if (L.seed_src == 1) {
            mkh::counter_words(mid, idx, w4);
        } else {
            u32 sw[8];
            if ((idx >> 1) == other_id) {
#pragma unroll
                for (int i = 0; i < 8; i++) sw[i] = other[i];
            } else {
                u32 blk[16];
                mkh::chacha20_block(key, idx >> 1, blk);
                const bool odd = idx & 1;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    sw[i] = odd ? blk[8 + i] : blk[i];
                    other[i] = odd ? blk[i] : blk[8 + i];
                }
                other_id = idx >> 1;
            }
            mkh::seed_words(sw, w4);
        }
        mkh::ShaRun shr;
        mkh::sha_run_start(shr, w4);
        fe num;
        comb_mul_sha(L.table, g, sc[j], slot, num, b.den[j], shr);
        mkh::digest_scalar(shr.s[0], shr.s[1], shr.s[2], shr.s[3], sc[j]);
        if (j == 0) {
            b.a[0] = num;
            run = b.den[0];
        } else {
            b.a[j] = mk32::fe_mul_as<SECURE_KARATSUBA>(num, run);
            run = mk32::fe_mul_as<SECURE_KARATSUBA>(run, b.den[j]);
        }
    }
    b.prod = run;
}

// Backward pass: `inv` is 1/(product of the batch's denominators); yields each key's
// canonical y (sign bit 0), tests the needles and reports candidate hits.  K: Karatsuba
// multiplies.
template <int KPT, bool K = false>
__device__ __forceinline__ void backward(const KeyLaunch& L, const MatchSet& ms, const u32* lane_masks, u64 first,
                                         const Batch<KPT>& b, fe inv, u32& sink) {
#pragma unroll 1
    for (int j = KPT - 1; j >= 0; j--) {
        u32 pk[8];
        mk32::fe_to_words(mk32::fe_mul_as<K>(b.a[j], inv), pk);
        if (j > 0) inv = mk32::fe_mul_as<K>(inv, b.den[j]);
        sink ^= pk[7];
        u64 hw[2];
        match_key(ms, lane_masks, pk, hw);
        const bool any = (hw[0] | hw[1]) != 0;
        // warp ballot: the (rare) warps with a hit compact their records into the ring
        if (__ballot_sync(0xffffffffu, any)) report_hits(hw, first + (u64)j, L.hits, L.hit_cap, L.job);
    }
}

// Named barriers of the search pipeline: products of buffer b ready (1 + b), inverses of
// buffer b ready (3 + b).  Barrier 0 is __syncthreads.
__device__ __forceinline__ void bar_sync(int id, int count) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }
__device__ __forceinline__ void bar_arrive(int id, int count) { asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory"); }

// Inverts the `pools`·`groups` products prod[0 .. pools·groups) in place with one field
// inversion per pool: lane l < pools of the calling warp handles the strided pool l, l+pools,
// l+2·pools, ... (Montgomery's trick inside each pool); the other lanes idle.  With 32 pools
// every lane works; fewer pools share each inversion among more keys (the inversion batch of a
// pool is groups x the keys per thread).
__device__ __forceinline__ void invert_pools(fe* prod, fe* scratch, int groups, int pools = 32) {
    const int l = threadIdx.x & 31;
    if (l >= pools) return;
    fe acc = prod[l];
    scratch[l] = acc;
#pragma unroll 1
    for (int k = 1; k < groups; k++) {
        acc = mk32::fe_mul(acc, prod[l + pools * k]);
        scratch[l + pools * k] = acc;
    }
    fe inv = mk32::fe_invert(acc);
#pragma unroll 1
    for (int k = groups - 1; k > 0; k--) {
        fe t = mk32::fe_mul(inv, scratch[l + pools * (k - 1)]);
        inv = mk32::fe_mul(inv, prod[l + pools * k]);
        prod[l + pools * k] = t;
    }
    prod[l] = inv;
}

// ---------------------------------------------------------------------------
// incremental source: index base + i is the point (s0 + base + i)·B
// ---------------------------------------------------------------------------

__device__ __forceinline__ fe words_fe(const u32* w) {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = w[i];
    return r;
}

__device__ __forceinline__ niels words_niels(const u32* w) {
    niels n;
    n.ypx = words_fe(w);
    n.ymx = words_fe(w + 8);
    n.t2d = words_fe(w + 16);
    return n;
}

__device__ __forceinline__ niels smem_niels(const uint4* q) {
    niels n;
    uint4 a;
    a = q[0]; n.ypx.v[0] = a.x; n.ypx.v[1] = a.y; n.ypx.v[2] = a.z; n.ypx.v[3] = a.w;
    a = q[1]; n.ypx.v[4] = a.x; n.ypx.v[5] = a.y; n.ypx.v[6] = a.z; n.ypx.v[7] = a.w;
    a = q[2]; n.ymx.v[0] = a.x; n.ymx.v[1] = a.y; n.ymx.v[2] = a.z; n.ymx.v[3] = a.w;
    a = q[3]; n.ymx.v[4] = a.x; n.ymx.v[5] = a.y; n.ymx.v[6] = a.z; n.ymx.v[7] = a.w;
    a = q[4]; n.t2d.v[0] = a.x; n.t2d.v[1] = a.y; n.t2d.v[2] = a.z; n.t2d.v[3] = a.w;
    a = q[5]; n.t2d.v[4] = a.x; n.t2d.v[5] = a.y; n.t2d.v[6] = a.z; n.t2d.v[7] = a.w;
    return n;
}

// The launch's start point (s0 + base)·B plus offset·B from the 4-bit window table
// (offset < 2^32; one mixed addition per nonzero window).
__device__ __forceinline__ ge incr_start(const KeyLaunch& L, u64 offset) {
    ge P;
    P.X = words_fe(L.start);
    P.Y = words_fe(L.start + 8);
    P.Z = words_fe(L.start + 16);
    P.T = words_fe(L.start + 24);
#pragma unroll 1
    for (int w = 0; w < INCR_WINDOWS; w++) {
        const u32 d = (u32)(offset >> (4 * w)) & 15u;
        if (d) P = mk32::ge_add_niels(P, load_entry(L.incr, (u64)w * 16 + d), false);
    }
    return P;
}

// Copies the step table j·B (j = 0 .. INCR_STEPS-1) into shared memory.
__device__ __forceinline__ void load_steps(const KeyLaunch& L, uint4* steps, u32 tid, u32 nthr) {
    const uint4* src = L.incr + (u64)INCR_WINDOWS * 16 * (ENTRY_WORDS / 4);
    for (u32 i = tid; i < (u32)INCR_STEPS * (ENTRY_WORDS / 4); i += nthr) steps[i] = src[i];
}

// Batch of the KPT consecutive points Q + j·B (j = 0 .. KPT-1): key 0 is Q itself (y = Y/Z);
// key j > 0 takes y = (b + a)/(2Z - c) of the mixed addition with the step entry j·B,
// three multiplications, with Q's y+x, y-x and 2Z shared by all of them.
template <int KPT>
__device__ __forceinline__ void incr_fracs(const ge& Q, const uint4* steps, Batch<KPT>& b) {
    const fe ypx = mk32::fe_add(Q.Y, Q.X), ymx = mk32::fe_sub(Q.Y, Q.X), z2 = mk32::fe_add(Q.Z, Q.Z);
    b.a[0] = Q.Y;
    b.den[0] = Q.Z;
    fe run = Q.Z;
#pragma unroll 1
    for (int j = 1; j < KPT; j++) {
        const niels t = smem_niels(steps + j * (ENTRY_WORDS / 4));
        const fe A = mk32::fe_mul(ymx, t.ymx), B = mk32::fe_mul(ypx, t.ypx), C = mk32::fe_mul(Q.T, t.t2d);
        b.den[j] = mk32::fe_sub(z2, C);
        b.a[j] = mk32::fe_mul(mk32::fe_add(B, A), run);
        run = mk32::fe_mul(run, b.den[j]);
    }
    b.prod = run;
}

// Search kernel.  The compute threads each handle KPT consecutive indices per iteration
// (index = base + (it·nthreads + gid)·KPT + j, where gid and nthreads count the compute
// threads).  Iterations are pipelined two deep: a compute thread runs the forward pass of
// iteration it+1 before the backward pass of it, and the CTA's products of iteration it are
// turned into their inverses in between.  Who inverts:
//   ROT false: the CTA's last warp, which does nothing else (BLOCK-32 compute threads).  The
//     inversion's long dependent chain runs beside the other warps' work.  That warp's SM
//     sub-partition (warp w runs on sub-partition w % 4) then holds three compute warps
//     against four elsewhere;
//   ROT true: every thread computes keys, and the inversion of iteration it falls to warp
//     BLOCK/32 - 4 + it % 4, one warp per sub-partition in turn.  The sub-partitions carry
//     equal shares, but the inverting warp starts its next iteration only after the chain.
//     That pays when iterations are long (many needles) and costs when they are short.
// The CTA's CT products of an iteration are inverted in L.inv_pools pools (default 32: lane l
// of the inverting warp takes threads l, l+32, ...), one field inversion each, so one
// inversion serves KPT·CT/pools keys.
// Named barriers, all BLOCK threads: products of buffer b ready (1 + b): the inverting warp
// waits, the others arrive; inverses of buffer b ready (3 + b): the inverting warp arrives,
// the others wait.  Stop requests (host stop word, or a hit with stop_on_hit) are read by
// the inverting warp and take effect two iterations later, at a point every warp agrees on
// (tests/test_pipeline_protocol.py model-checks both forms).
// INCR: the incremental source.  A compute thread keeps the point Q of its first index in
// the current iteration; its keys are Q + j·B from the step table, and Q advances by
// keys_per_iter·B (one mixed addition) per iteration.  No comb table is read.
// STAB: the comb table lives in shared memory (copied by every CTA at the start, in place of
// the staging slots; tables of a few hundred to a few thousand entries, 40+ rows).
// SHAI: the SHA-512 of iteration it+1's seeds runs inside iteration it's comb rows (12 rows;
// the first iteration's scalars are hashed up front).
template <int KPT, int BLOCK, bool INCR, bool ROT, bool STAB = false, bool SHAI = false>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK) k_search(const KeyLaunch L) {
    constexpr int CT = ROT ? BLOCK : BLOCK - 32;  // compute threads
    constexpr int CW = CT / 32;                   // compute warps
    extern __shared__ uint4 dyn_smem[];
    fe (*prod)[CT] = reinterpret_cast<fe (*)[CT]>(dyn_smem);
    fe (*scratch)[CT] = prod + 2;
    EntrySlot* slots = reinterpret_cast<EntrySlot*>(scratch + 2);
    uint4* stab = reinterpret_cast<uint4*>(scratch + 2);  // STAB: the table in place of the slots
    __shared__ CombGeom g;
    __shared__ MatchSet ms;
    __shared__ u32 lane_masks[64 * 32];  // see match_key
    __shared__ u32 key[8];
    __shared__ mkh::CounterMid mid;
    __shared__ volatile u32 stop_iter;
    __shared__ uint4 steps[INCR ? INCR_STEPS * (ENTRY_WORDS / 4) : 1];
    const u32 tid = threadIdx.x;
    if (INCR) load_steps(L, steps, tid, BLOCK);
    {
        const u32* src = (const u32*)&L.geom;
        u32* dst = (u32*)&g;
        for (u32 i = tid; i < sizeof(CombGeom) / 4; i += BLOCK) dst[i] = src[i];
        const u32* s2 = (const u32*)L.match;
        u32* d2 = (u32*)&ms;
        for (u32 i = tid; i < sizeof(MatchSet) / 4; i += BLOCK) d2[i] = s2[i];
        if (tid < 8) key[tid] = L.key[tid];
        if (tid == 0) stop_iter = L.iters;
    }
    __syncthreads();
    if (STAB)  // entries 128 bytes apart in HBM, 96 here
        for (u32 e = tid; e < (u32)g.entries; e += BLOCK)
#pragma unroll
            for (int q = 0; q < 6; q++) stab[e * 6 + q] = L.table[(u64)e * (COMB_STRIDE_WORDS / 4) + q];
    u32 dfa_need = 0;
    for (u32 r = 0; r < ms.n_regex; r++) dfa_need += (ms.dfa_states[r] * 130u + 15u) & ~15u;
    if (L.dfa_smem && dfa_need <= L.dfa_smem) {
        // stage the job's DFA tables behind the other dynamic buffers (only when the launch
        // reserved room for all of them) and point the matcher at the copies (16-byte
        // aligned tables, copied in u16 units)
        uint8_t* area = reinterpret_cast<uint8_t*>(INCR ? (void*)slots : (void*)(slots + CT));
        u32 off = 0;
        for (u32 r = 0; r < ms.n_regex; r++) {
            const uint16_t* src = reinterpret_cast<const uint16_t*>(ms.dfa[r]);
            uint16_t* dst = reinterpret_cast<uint16_t*>(area + off);
            const u32 halves = ms.dfa_states[r] * 65u;
            for (u32 i = tid; i < halves; i += BLOCK) dst[i] = src[i];
            off += (halves * 2u + 15u) & ~15u;
        }
        __syncthreads();
        if (tid == 0) {
            off = 0;
            for (u32 r = 0; r < ms.n_regex; r++) {
                ms.dfa[r] = area + off;
                off += (ms.dfa_states[r] * 130u + 15u) & ~15u;
            }
        }
    }
    if (ms.narrow)
        for (u32 i = tid; i < 64u * 32u; i += BLOCK) lane_masks[i] = (u32)ms.mask[0][i >> 5];
    if (tid == 0 && L.seed_src == 1) mid = mkh::counter_mid(key);
    __syncthreads();
    const u32 iters = L.iters;
    if (iters == 0) return;
    // inversion pools of the CTA (a divisor of CT, at most 32; the host checks it)
    const int pools = L.inv_pools ? (int)L.inv_pools : 32;

    if (!ROT && tid >= (u32)CT) {
        // ---- dedicated inverter warp ----
        for (u32 it = 0;; it++) {
            const int b = it & 1;
            bar_sync(1 + b, BLOCK);
            if ((tid & 31) == 0) {
                const volatile JobDevice* jd = L.job;
                if (jd->stop != 0 || (L.stop_on_hit && jd->hit_count != 0)) {
                    u32 s = it + 2;
                    if (s < stop_iter) stop_iter = s;
                }
            }
            __syncwarp();
            invert_pools(prod[b], scratch[b], CT / pools, pools);
            __syncwarp();
            bar_arrive(3 + b, BLOCK);
            if (it + 1 >= iters || it + 1 >= stop_iter) break;
        }
        if ((tid & 31) == 0 && stop_iter < iters) atomicOr(&L.job->status, 1u);
        return;
    }

    // ---- compute warps ----
    const u32 warp = tid >> 5;
    auto inverts = [&](u32 it) { return ROT && warp == (u32)CW - 4u + (it & 3u); };
    const u64 gid = (u64)blockIdx.x * CT + tid;
    const u64 nthreads = (u64)gridDim.x * CT;
    EntrySlot& slot = slots[INCR || STAB ? 0 : tid];
    Batch<KPT> batch[2];
    u64 sc[KPT][4];
    u32 sink = 0;
    ge Q;
    if (INCR) Q = incr_start(L, gid * KPT);
    auto first_of = [&](u32 it) { return L.base + ((u64)it * nthreads + gid) * KPT; };
    auto produce = [&](u32 it) {
        const int b = it & 1;
        if (INCR) {
            incr_fracs<KPT>(Q, steps, batch[b]);
            Q = mk32::ge_add_niels(Q, words_niels(L.delta), false);
        } else if (SHAI) {
            if (it == 0) scalars<KPT>(L, key, mid, first_of(0), sc);
            combs_sha<KPT>(L, g, sc, slot, batch[b], key, mid, first_of(it + 1));
        } else {
            scalars<KPT>(L, key, mid, first_of(it), sc);
            combs<KPT, STAB>(L, g, sc, slot, stab, batch[b]);
        }
        prod[b][tid] = batch[b].prod;
        if (inverts(it)) {
            bar_sync(1 + b, BLOCK);
            if ((tid & 31) == 0) {
                const volatile JobDevice* jd = L.job;
                if (jd->stop != 0 || (L.stop_on_hit && jd->hit_count != 0)) {
                    u32 s = it + 2;
                    if (s < stop_iter) stop_iter = s;
                }
            }
            __syncwarp();
            invert_pools(prod[b], scratch[b], CT / pools, pools);
            __syncwarp();
            bar_arrive(3 + b, BLOCK);
        } else {
            bar_arrive(1 + b, BLOCK);
        }
    };
    produce(0);
    for (u32 it = 0;; it++) {
        const int b = it & 1;
        if (it + 1 < iters && it + 1 < stop_iter) produce(it + 1);
        if (!inverts(it)) bar_sync(3 + b, BLOCK);
        backward<KPT, !INCR && SECURE_KARATSUBA>(L, ms, ms.narrow ? lane_masks : nullptr, first_of(it), batch[b],
                                                 prod[b][tid], sink);
        if (it + 1 >= iters || it + 1 >= stop_iter) break;
    }
    // warp 0 never inverts, so with ROT the last stop decision is visible here
    if (ROT && tid == 0 && stop_iter < iters) atomicOr(&L.job->status, 1u);
    if (L.sink) L.sink[gid] = sink;
}

// Search kernel with hashing warps (ChaCha20 / counter seeds).  Warps 0..10 run the comb
// multiplies, warp 11 inverts, warps 12..15 (one per SM sub-partition) compute the seeds'
// SHA-512 scalars: hashing is ALU work and the comb is IMAD work, so the two pipes overlap
// instead of the compute warps alternating between them.  The index layout and results are
// those of k_search; only the division of work inside a CTA differs.
//
// Scalars go from the hashing warps to the comb warps through a two-slot shared ring of
// chunks (4 keys of every comb thread per chunk).  Named barriers:
//   1+b / 3+b  products / inverses of pipeline buffer b (comb warps and the inverter, 384)
//   5+s / 7+s  ring slot s full / empty (hashing and comb warps, 480)
//   9+(it&1)   the inverter's stop decision after iteration it (inverter and hashing warps, 160)
// Whether iteration X is computed is decided, by every role, from the stop word as it stands
// after the inverter's decision of iteration X-2; the inverter arrives on a decision barrier
// only when the hashing warps will wait on it, and the hashing warps drain the last two ring
// releases before they return, so no barrier phase is left open (model-checked in
// tests/test_pipeline_protocol.py).
template <int KPT, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) k_search_hw(const KeyLaunch L) {
    static_assert(BLOCK == 512 && KPT % 4 == 0 && KPT >= 8, "layout of 11 comb, 1 inverter, 4 hashing warps");
    constexpr int CW = 11, CT = CW * 32;     // comb warps / threads
    constexpr int INV_WARP = 11;
    constexpr int HT = 128;                  // hashing threads
    constexpr int CPI = KPT / 4;             // ring chunks per iteration
    constexpr int PAIRS = CT * 2;            // index pairs per chunk
    constexpr int B_PIPE = CT + 32, B_RING = CT + HT, B_STOP = 32 + HT;
    extern __shared__ uint4 dyn_smem[];
    fe (*prod)[CT] = reinterpret_cast<fe (*)[CT]>(dyn_smem);
    fe (*scratch)[CT] = prod + 2;
    EntrySlot* slots = reinterpret_cast<EntrySlot*>(scratch + 2);
    u64 (*ring)[4][CT][4] = reinterpret_cast<u64 (*)[4][CT][4]>(slots + CT);  // [slot][key][thread][word]
    __shared__ CombGeom g;
    __shared__ MatchSet ms;
    __shared__ u32 lane_masks[64 * 32];  // see match_key
    __shared__ u32 key[8];
    __shared__ mkh::CounterMid mid;
    __shared__ volatile u32 stop_iter;
    const u32 tid = threadIdx.x;
    const u32 warp = tid >> 5;
    {
        const u32* src = (const u32*)&L.geom;
        u32* dst = (u32*)&g;
        for (u32 i = tid; i < sizeof(CombGeom) / 4; i += BLOCK) dst[i] = src[i];
        const u32* s2 = (const u32*)L.match;
        u32* d2 = (u32*)&ms;
        for (u32 i = tid; i < sizeof(MatchSet) / 4; i += BLOCK) d2[i] = s2[i];
        if (tid < 8) key[tid] = L.key[tid];
        if (tid == 0) stop_iter = L.iters;
    }
    __syncthreads();
    if (ms.narrow)
        for (u32 i = tid; i < 64u * 32u; i += BLOCK) lane_masks[i] = (u32)ms.mask[0][i >> 5];
    if (tid == 0 && L.seed_src == 1) mid = mkh::counter_mid(key);
    __syncthreads();
    const u32 iters = L.iters;
    if (iters == 0) return;
    const u64 nthreads = (u64)gridDim.x * CT;
    auto first_of = [&](u32 it, u64 gid) { return L.base + ((u64)it * nthreads + gid) * KPT; };
    const int pools = L.inv_pools ? (int)L.inv_pools : 32;  // a divisor of CT, at most 32

    if (warp > (u32)INV_WARP) {
        // ---- hashing warps ----
        const u32 p = tid - (INV_WARP + 1) * 32;
        u32 X = 0;
        for (;; X++) {
            if (X >= iters) break;
            if (X >= 2) {
                bar_sync(9 + (X & 1), B_STOP);
                if (X >= stop_iter) break;
            }
#pragma unroll 1
            for (u32 c = 0; c < (u32)CPI; c++) {
                const u32 gc = X * CPI + c, slot = gc & 1;
                if (gc >= 2) bar_sync(7 + slot, B_RING);
#pragma unroll 1
                for (u32 v = p; v < (u32)PAIRS; v += HT) {
                    const u32 t = v >> 1, k0 = (v & 1) * 2;
                    const u64 idx = first_of(X, (u64)blockIdx.x * CT + t) + c * 4 + k0;
                    u32 blk[16];
                    u64 blk_id = ~0ull;
#pragma unroll 1
                    for (u32 q = 0; q < 2; q++) {
                        u64 sc[4];
                        scalar_of(L.seed_src, key, mid, idx + q, blk, blk_id, sc);
                        uint4* d = reinterpret_cast<uint4*>(ring[slot][k0 + q][t]);
                        d[0] = make_uint4((u32)sc[0], (u32)(sc[0] >> 32), (u32)sc[1], (u32)(sc[1] >> 32));
                        d[1] = make_uint4((u32)sc[2], (u32)(sc[2] >> 32), (u32)sc[3], (u32)(sc[3] >> 32));
                    }
                }
                bar_arrive(5 + slot, B_RING);
            }
        }
        // the comb warps release every chunk they take: wait for the last two releases
        const u32 G = X * CPI;
        bar_sync(7 + ((G - 2) & 1), B_RING);
        bar_sync(7 + ((G - 1) & 1), B_RING);
        return;
    }

    if (warp == (u32)INV_WARP) {
        // ---- inverter warp ----
        for (u32 it = 0;; it++) {
            const int b = it & 1;
            bar_sync(1 + b, B_PIPE);
            if ((tid & 31) == 0) {
                const volatile JobDevice* jd = L.job;
                if (jd->stop != 0 || (L.stop_on_hit && jd->hit_count != 0)) {
                    u32 s = it + 2;
                    if (s < stop_iter) stop_iter = s;
                }
            }
            __syncwarp();
            const bool more = it + 1 < iters && it + 1 < stop_iter;
            // the hashing warps wait on this decision only when they will consider iteration it+2
            if (it + 2 < iters && more) bar_arrive(9 + (it & 1), B_STOP);
            invert_pools(prod[b], scratch[b], CT / pools, pools);
            __syncwarp();
            bar_arrive(3 + b, B_PIPE);
            if (!more) break;
        }
        if ((tid & 31) == 0 && stop_iter < iters) atomicOr(&L.job->status, 1u);
        return;
    }

    // ---- comb warps ----
    const u64 gid = (u64)blockIdx.x * CT + tid;
    EntrySlot& slot = slots[tid];
    Batch<KPT> batch[2];
    u32 sink = 0;
    auto produce = [&](u32 it) {
        const int b = it & 1;
        Batch<KPT>& bt = batch[b];
        fe run;
#pragma unroll 1
        for (int j = 0; j < KPT; j++) {
            const u32 gc = it * CPI + (u32)(j >> 2), rs = gc & 1;
            if ((j & 3) == 0) bar_sync(5 + rs, B_RING);
            u64 sc[4];
            {
                const uint4* q = reinterpret_cast<const uint4*>(ring[rs][j & 3][tid]);
                const uint4 a = q[0], c = q[1];
                sc[0] = (u64)a.y << 32 | a.x;
                sc[1] = (u64)a.w << 32 | a.z;
                sc[2] = (u64)c.y << 32 | c.x;
                sc[3] = (u64)c.w << 32 | c.z;
            }
            if ((j & 3) == 3) bar_arrive(7 + rs, B_RING);
            fe num;
            comb_mul(L.table, g, sc, slot, num, bt.den[j], nullptr, nullptr);
            if (j == 0) {
                bt.a[0] = num;
                run = bt.den[0];
            } else {
                bt.a[j] = mk32::fe_mul_as<SECURE_KARATSUBA>(num, run);
                run = mk32::fe_mul_as<SECURE_KARATSUBA>(run, bt.den[j]);
            }
        }
        bt.prod = run;
        prod[b][tid] = bt.prod;
        bar_arrive(1 + b, B_PIPE);
    };
    produce(0);
    for (u32 it = 0;; it++) {
        const int b = it & 1;
        if (it + 1 < iters && it + 1 < stop_iter) produce(it + 1);
        bar_sync(3 + b, B_PIPE);
        backward<KPT, SECURE_KARATSUBA>(L, ms, ms.narrow ? lane_masks : nullptr, first_of(it, gid), batch[b],
                                        prod[b][tid], sink);
        if (it + 1 >= iters || it + 1 >= stop_iter) break;
    }
    if (L.sink) L.sink[gid] = sink;
}

// Derive kernel: full public keys (x sign included) of indices base .. base+count-1;
// one iteration, per-CTA pooled inversion of 2·KPT denominators per thread.  INCR: the
// thread's keys are Q + j·B with Q = (s0 + first)·B; key j gives y = (b+a)/(2Z-c) and
// x = (b-a)/(2Z+c) of the mixed addition with step entry j (entry 0 is the identity).
template <int KPT, int BLOCK, bool INCR>
__global__ void __launch_bounds__(BLOCK, 512 / BLOCK) k_derive(const KeyLaunch L) {
    constexpr int NUM = 2 * KPT;
    extern __shared__ uint4 dyn_smem[];
    fe* prod = reinterpret_cast<fe*>(dyn_smem);
    fe* scratch = prod + BLOCK;
    EntrySlot* slots = reinterpret_cast<EntrySlot*>(scratch + BLOCK);
    __shared__ CombGeom g;
    __shared__ u32 key[8];
    __shared__ uint4 steps[INCR ? INCR_STEPS * (ENTRY_WORDS / 4) : 1];
    const u32 tid = threadIdx.x;
    const u64 gid = (u64)blockIdx.x * BLOCK + tid;
    if (INCR) load_steps(L, steps, tid, BLOCK);
    {
        const u32* src = (const u32*)&L.geom;
        u32* dst = (u32*)&g;
        for (u32 i = tid; i < sizeof(CombGeom) / 4; i += BLOCK) dst[i] = src[i];
        if (tid < 8) key[tid] = L.key[tid];
    }
    __syncthreads();
    mkh::CounterMid mid;
    if (L.seed_src == 1) mid = mkh::counter_mid(key);
    const u64 first = L.base + gid * KPT;
    fe num[NUM], den[NUM], pre[NUM];
    u32 blk[16];
    u64 blk_id = ~0ull;
    ge Q;
    fe ypx, ymx, z2;
    if (INCR) {
        Q = incr_start(L, gid * KPT);
        ypx = mk32::fe_add(Q.Y, Q.X);
        ymx = mk32::fe_sub(Q.Y, Q.X);
        z2 = mk32::fe_add(Q.Z, Q.Z);
    }
#pragma unroll 1
    for (int j = 0; j < KPT; j++) {
        if (INCR) {
            const niels t = smem_niels(steps + j * (ENTRY_WORDS / 4));
            const fe A = mk32::fe_mul(ymx, t.ymx), B = mk32::fe_mul(ypx, t.ypx), C = mk32::fe_mul(Q.T, t.t2d);
            num[2 * j] = mk32::fe_add(B, A);
            den[2 * j] = mk32::fe_sub(z2, C);
            num[2 * j + 1] = mk32::fe_sub(B, A);
            den[2 * j + 1] = mk32::fe_add(z2, C);
        } else {
            u64 s[4];
            scalar_of(L.seed_src, key, mid, first + (u64)j, blk, blk_id, s);
            comb_mul(L.table, g, s, slots[tid], num[2 * j], den[2 * j], &num[2 * j + 1], &den[2 * j + 1]);
        }
        pre[2 * j] = j == 0 ? den[0] : mk32::fe_mul(pre[2 * j - 1], den[2 * j]);
        pre[2 * j + 1] = mk32::fe_mul(pre[2 * j], den[2 * j + 1]);
    }
    prod[tid] = pre[NUM - 1];
    __syncthreads();
    if (tid < 32) invert_pools(prod, scratch, BLOCK / 32);
    __syncthreads();
    fe inv = prod[tid];
#pragma unroll 1
    for (int j = KPT - 1; j >= 0; j--) {
        const u64 idx = first + (u64)j;
        const int ex = 2 * j + 1, ey = 2 * j;
        fe xinv = mk32::fe_mul(inv, pre[ex - 1]);
        inv = mk32::fe_mul(inv, den[ex]);
        fe yinv = ey == 0 ? inv : mk32::fe_mul(inv, pre[ey - 1]);
        if (ey > 0) inv = mk32::fe_mul(inv, den[ey]);
        u32 xw[8], pk[8];
        mk32::fe_to_words(mk32::fe_mul(num[ex], xinv), xw);
        mk32::fe_to_words(mk32::fe_mul(num[ey], yinv), pk);
        pk[7] |= (xw[0] & 1u) << 31;
        if (idx - L.base < L.count) {
            uint4* o = (uint4*)(L.out + (idx - L.base) * 32);
            o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
    }
}

// ---------------------------------------------------------------------------
// host launch wrappers
// ---------------------------------------------------------------------------

#define MK_VARIANTS(X) X(4, 256) X(8, 256) X(16, 256) X(4, 512) X(8, 512) X(16, 512)

// dynamic shared memory: products and inversion scratch (two buffers each for the
// search pipeline) and the per-thread table staging slots
// (the incremental source reads no comb table and needs no staging slots)
static size_t dyn_bytes(bool derive, bool incr, uint32_t block, uint32_t layout, uint32_t table_smem) {
    const size_t fe_bytes = 32;
    if (layout == LAYOUT_HASH_WARPS && !derive && !incr) {  // k_search_hw: 352 comb threads, plus the two-slot scalar ring
        const size_t ct = 352;
        return 4 * ct * fe_bytes + ct * sizeof(EntrySlot) + 2 * 4 * ct * 32;
    }
    const size_t threads = derive ? block : search_threads(block, layout == LAYOUT_HASH_WARPS ? LAYOUT_INVERTER_WARP : layout);
    // (the interleaved layout has the dedicated inverter's buffers)
    if (table_smem && !derive && !incr) return 4 * threads * fe_bytes + table_smem;  // the table in place of the slots
    return (derive ? 2 : 4) * threads * fe_bytes + (incr ? 0 : threads * sizeof(EntrySlot));
}

static const void* hw_kernel_of(uint32_t kpt, uint32_t block) {
    if (block != 512) return nullptr;
    if (kpt == 8) return (const void*)k_search_hw<8, 512>;
    if (kpt == 16) return (const void*)k_search_hw<16, 512>;
    return nullptr;
}

// search kernels with the comb table in shared memory: the dedicated-inverter layout, block
// 512, keys per thread 4 and 8
static const void* stab_kernel_of(uint32_t kpt, uint32_t block) {
    if (block != 512) return nullptr;
    if (kpt == 4) return (const void*)k_search<4, 512, false, false, true>;
    if (kpt == 8) return (const void*)k_search<8, 512, false, false, true>;
    return nullptr;
}

static const void* kernel_of(bool derive, bool incr, uint32_t kpt, uint32_t block, bool rot) {
#define MK_FN(K, B)                                                                                            \
    if (kpt == K && block == B) {                                                                              \
        if (derive) return incr ? (const void*)k_derive<K, B, true> : (const void*)k_derive<K, B, false>;      \
        if (rot) return incr ? (const void*)k_search<K, B, true, true> : (const void*)k_search<K, B, false, true>; \
        return incr ? (const void*)k_search<K, B, true, false> : (const void*)k_search<K, B, false, false>;    \
    }
    MK_VARIANTS(MK_FN)
#undef MK_FN
    return nullptr;
}

static cudaError_t prepare(const void* f, size_t dyn) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
}

// search kernels with the SHA-512 interleaved into the comb rows: the dedicated-inverter layout,
// block 512, keys per thread 8 and 16
static const void* shai_kernel_of(uint32_t kpt, uint32_t block) {
    if (block != 512) return nullptr;
    if (kpt == 8) return (const void*)k_search<8, 512, false, false, false, true>;
    if (kpt == 16) return (const void*)k_search<16, 512, false, false, false, true>;
    return nullptr;
}

// the kernel of a variant (the table-in-shared-memory search when table_smem > 0)
static const void* variant_kernel(bool derive, bool incr, uint32_t kpt, uint32_t block, uint32_t layout,
                                  uint32_t table_smem) {
    if (layout == LAYOUT_INTERLEAVED && !derive && !incr) return table_smem ? nullptr : shai_kernel_of(kpt, block);
    const bool hw = layout == LAYOUT_HASH_WARPS && !derive && !incr;
    if (table_smem && !derive && !incr) return layout == LAYOUT_INVERTER_WARP ? stab_kernel_of(kpt, block) : nullptr;
    return hw ? hw_kernel_of(kpt, block) : kernel_of(derive, incr, kpt, block, layout == LAYOUT_ROTATING);
}

cudaError_t launch_keys(const KeyLaunch& L, bool derive, uint32_t kpt, uint32_t block, uint32_t grid, cudaStream_t st) {
    const bool incr = L.seed_src == SEED_INCREMENTAL;
    if (incr && (kpt > (uint32_t)INCR_STEPS || !L.incr)) return cudaErrorInvalidValue;
    if (L.dfa_smem > DFA_SMEM_MAX || (derive && L.dfa_smem)) return cudaErrorInvalidValue;
    const bool hw = L.layout == LAYOUT_HASH_WARPS && !derive && !incr;
    if (hw && L.dfa_smem) return cudaErrorInvalidValue;  // the scalar ring takes that shared memory
    const uint32_t tsm = derive || incr ? 0 : L.table_smem;
    if (tsm && L.dfa_smem) return cudaErrorInvalidValue;  // the table takes that shared memory
    const void* f = variant_kernel(derive, incr, kpt, block, L.layout, tsm);
    if (!f) return cudaErrorInvalidValue;
    const size_t dyn = dyn_bytes(derive, incr, block, L.layout, tsm) + L.dfa_smem;
    cudaError_t e = prepare(f, dyn);
    if (e != cudaSuccess) return e;
    void* args[] = {const_cast<KeyLaunch*>(&L)};
    return cudaLaunchKernel(f, dim3(grid), dim3(block), args, dyn, st);
}

cudaError_t keys_kernel(bool derive, bool incr, uint32_t kpt, uint32_t block, uint32_t layout, uint32_t dfa_smem,
                        uint32_t table_smem, const void** func, size_t* dyn) {
    const bool hw = layout == LAYOUT_HASH_WARPS && !derive && !incr;
    const uint32_t tsm = derive || incr ? 0 : table_smem;
    const void* f = variant_kernel(derive, incr, kpt, block, layout, tsm);
    if (!f || dfa_smem > DFA_SMEM_MAX || ((hw || tsm) && dfa_smem)) return cudaErrorInvalidValue;
    *func = f;
    *dyn = dyn_bytes(derive, incr, block, layout, tsm) + dfa_smem;
    return prepare(f, *dyn);
}

cudaError_t keys_occupancy(bool derive, bool incr, uint32_t kpt, uint32_t block, uint32_t layout, uint32_t table_smem,
                           int* blocks_per_sm) {
    const uint32_t tsm = derive || incr ? 0 : table_smem;
    const void* f = variant_kernel(derive, incr, kpt, block, layout, tsm);
    if (!f) return cudaErrorInvalidValue;
    const size_t dyn = dyn_bytes(derive, incr, block, layout, tsm);
    cudaError_t e = prepare(f, dyn);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, (int)block, dyn);
}

cudaError_t launch_build_table(uint4* table, const CombGeom& g, const uint32_t* points, uint64_t first,
                               uint64_t count, cudaStream_t st) {
    uint32_t blocks = (uint32_t)((count + 255) / 256);
    k_build_table<<<blocks, 256, 0, st>>>(table, g, points, first, count);
    return cudaGetLastError();
}

}  // namespace mkb

namespace mkb {

// Peak of independent 32-bit multiply-adds: 8 chains per thread, no memory traffic.
__global__ void __launch_bounds__(256) k_mad_lo_peak(uint32_t iters, uint32_t x, uint32_t y, uint32_t* out) {
    uint32_t a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = threadIdx.x + i;
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[i]) : "r"(x), "r"(y));
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s ^= a[i];
    out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Peak of the field multiply's own instruction shape: one row of a schoolbook product,
// acc[0..8] += a·b[0..7] as a mad.lo.cc/madc.lo.cc chain followed by the madc.hi.cc chain
// one word up (16 multiply-adds and one addc), on four independent accumulators per thread.
// The multiplier a is the accumulator's top word plus the iteration, so no product can be
// hoisted out of the loop.
__global__ void __launch_bounds__(256) k_mad_chain_peak(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint32_t acc[4][9], b[8];
#pragma unroll
    for (int i = 0; i < 8; i++) b[i] = seed * (2 * i + 1) + threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int i = 0; i < 9; i++) acc[q][i] = threadIdx.x ^ (q * 9 + i);
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t* t = acc[q];
            const uint32_t a = t[8] + it;
            asm volatile(
                "mad.lo.cc.u32 %0, %9, %10, %0;\n\t"
                "madc.lo.cc.u32 %1, %9, %11, %1;\n\t"
                "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"
                "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"
                "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"
                "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"
                "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"
                "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"
                "addc.u32 %8, %8, 0;\n\t"
                "mad.hi.cc.u32 %1, %9, %10, %1;\n\t"
                "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"
                "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
                "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"
                "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"
                "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"
                "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"
                "madc.hi.u32 %8, %9, %17, %8;\n\t"
                : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
                  "+r"(t[8])
                : "r"(a), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int i = 0; i < 9; i++) s ^= acc[q][i];
    out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// The pieces of the field multiply's instruction mix, each on 8 chains per thread (so latency
// is hidden at full occupancy and the rate is what the pipe issues).  Every product has an
// operand that changes every iteration and differs between the chains, so no product can be
// hoisted out of the loop or shared between chains:
//   KIND 0  mad.hi.u32            the high half of a 32x32 product (independent chains)
//   KIND 1  mad.wide.u32          the full 64-bit product into a 64-bit sum (independent chains)
//   KIND 2  madc.lo.cc.u32 rows   8 low halves a_i·b linked through the carry flag
//   KIND 3  madc.hi.cc.u32 rows   8 high halves a_i·b linked through the carry flag
template <int KIND>
__global__ void __launch_bounds__(256) k_imad_rate(uint32_t iters, uint32_t x, uint32_t y, uint32_t* out) {
    uint32_t a[8], t[8];
    uint64_t w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        a[i] = (threadIdx.x * 8 + i) * 0x9e3779b9u + x;
        t[i] = threadIdx.x ^ (i * 0x01010101u);
        w[i] = (uint64_t)a[i] << 20;
    }
    for (uint32_t it = 0; it < iters; it++) {
        if (KIND == 0) {
#pragma unroll
            for (int i = 0; i < 8; i++) asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(t[i]) : "r"(a[i]), "r"(y));
        } else if (KIND == 1) {
#pragma unroll
            for (int i = 0; i < 8; i++)  // the multiplier is the sum's own low word
                asm volatile("{\n\t.reg .u32 m;\n\tcvt.u32.u64 m, %0;\n\tmad.wide.u32 %0, m, %1, %0;\n\t}"
                             : "+l"(w[i]) : "r"(a[i]));
        } else {
            const uint32_t b = t[7] + it;
            if (KIND == 2)
                asm volatile(
                    "mad.lo.cc.u32 %0, %8, %16, %0;\n\t"
                    "madc.lo.cc.u32 %1, %9, %16, %1;\n\t"
                    "madc.lo.cc.u32 %2, %10, %16, %2;\n\t"
                    "madc.lo.cc.u32 %3, %11, %16, %3;\n\t"
                    "madc.lo.cc.u32 %4, %12, %16, %4;\n\t"
                    "madc.lo.cc.u32 %5, %13, %16, %5;\n\t"
                    "madc.lo.cc.u32 %6, %14, %16, %6;\n\t"
                    "madc.lo.u32 %7, %15, %16, %7;\n\t"
                    : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7])
                    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b));
            else
                asm volatile(
                    "mad.hi.cc.u32 %0, %8, %16, %0;\n\t"
                    "madc.hi.cc.u32 %1, %9, %16, %1;\n\t"
                    "madc.hi.cc.u32 %2, %10, %16, %2;\n\t"
                    "madc.hi.cc.u32 %3, %11, %16, %3;\n\t"
                    "madc.hi.cc.u32 %4, %12, %16, %4;\n\t"
                    "madc.hi.cc.u32 %5, %13, %16, %5;\n\t"
                    "madc.hi.cc.u32 %6, %14, %16, %6;\n\t"
                    "madc.hi.u32 %7, %15, %16, %7;\n\t"
                    : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7])
                    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b));
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s ^= t[i] ^ (uint32_t)w[i] ^ (uint32_t)(w[i] >> 32);
    out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Rates of the four pieces (multiply-adds per second, best of three runs of 10-30 ms each).
cudaError_t measure_imad_rates(int sms, cudaStream_t st, double rates[4]) {
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256, iters = 1u << 16;
    uint32_t* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(uint32_t) * blocks * threads);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&](int kind, uint32_t it, uint32_t x) {
        if (kind == 0) k_imad_rate<0><<<blocks, threads, 0, st>>>(it, x, 0x9876u, out);
        else if (kind == 1) k_imad_rate<1><<<blocks, threads, 0, st>>>(it, x, 0x9876u, out);
        else if (kind == 2) k_imad_rate<2><<<blocks, threads, 0, st>>>(it, x, 0x9876u, out);
        else k_imad_rate<3><<<blocks, threads, 0, st>>>(it, x, 0x9876u, out);
    };
    for (int k = 0; k < 4; k++) {
        rates[k] = 0;
        launch(k, iters / 16, 0x1234u);
    }
    for (int rep = 0; rep < 12 && e == cudaSuccess; rep++) {
        const int k = rep % 4;
        cudaEventRecord(e0, st);
        launch(k, iters, 0x1234u + rep);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        const double mads = (double)blocks * threads * iters * 8;
        if (ms > 0 && mads / (ms * 1e-3) > rates[k]) rates[k] = mads / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e;
}

// Best of three timed runs (after a short warm-up) of both microbenchmarks, each about
// 10-30 ms at full occupancy: multiply-adds per second.
cudaError_t measure_mad_peaks(int sms, cudaStream_t st, double* chain_per_s, double* lo_per_s) {
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256;
    uint32_t* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(uint32_t) * blocks * threads);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best_chain = 0, best_lo = 0;
    const uint32_t lo_iters = 1u << 17, chain_iters = 1u << 14;
    k_mad_lo_peak<<<blocks, threads, 0, st>>>(lo_iters / 16, 0x12345u, 0x9876u, out);
    k_mad_chain_peak<<<blocks, threads, 0, st>>>(chain_iters / 16, 0x2468u, out);
    for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
        const bool chain = rep & 1;
        cudaEventRecord(e0, st);
        if (chain) k_mad_chain_peak<<<blocks, threads, 0, st>>>(chain_iters, 0x2468u + rep, out);
        else k_mad_lo_peak<<<blocks, threads, 0, st>>>(lo_iters, 0x12345u + rep, 0x9876u, out);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        if (ms <= 0) continue;
        const double mads = (double)blocks * threads * (chain ? (double)chain_iters * 4 * 16 : (double)lo_iters * 8);
        double& best = chain ? best_chain : best_lo;
        if (mads / (ms * 1e-3) > best) best = mads / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *chain_per_s = best_chain;
    *lo_per_s = best_lo;
    return e;
}

}  // namespace mkb

#include "fe26.cuh"
#include "fe51.cuh"

namespace mkb {

// Field-multiplication rate of three limb radices: four independent chains a <- a·b per
// thread, no memory traffic.  Radix 2^32 is the search kernel's field (fe32.cuh); radix
// 2^25.5 (fe26.cuh, ten limbs, 100 mad.wide products) and radix 2^51 in FP64 registers
// (fe51.cuh, five limbs, products split by fused multiply-adds) are the alternatives the
// search is not built for.  Radices 32 and 51 start from the same words and write the XOR
// of their chains' canonical words, so their outputs must agree.  RADIX 33 is radix 2^32 with
// the Karatsuba multiply (fe_mul_karatsuba), which must agree with the schoolbook form too.
template <int RADIX>
__global__ void __launch_bounds__(256) k_fe_mul_rate(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint32_t sum = 0;
    uint32_t wb[8], wa[4][8];
#pragma unroll
    for (int i = 0; i < 8; i++) wb[i] = seed * (i + 3) + threadIdx.x;
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int i = 0; i < 8; i++) wa[q][i] = threadIdx.x * 7 + q * 8 + i;
    if (RADIX == 32 || RADIX == 33) {
        mk32::fe a[4], b = mk32::fe_from_words(wb);
#pragma unroll
        for (int q = 0; q < 4; q++) a[q] = mk32::fe_from_words(wa[q]);
        for (uint32_t it = 0; it < iters; it++)
#pragma unroll
            for (int q = 0; q < 4; q++) a[q] = mk32::fe_mul_as<RADIX == 33>(a[q], b);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t w[8];
            mk32::fe_to_words(a[q], w);
#pragma unroll
            for (int i = 0; i < 8; i++) sum ^= w[i];
        }
    } else if (RADIX == 51) {
        mk51::fe a[4], b = mk51::fe_from_words(wb);
#pragma unroll
        for (int q = 0; q < 4; q++) a[q] = mk51::fe_from_words(wa[q]);
        for (uint32_t it = 0; it < iters; it++)
#pragma unroll
            for (int q = 0; q < 4; q++) a[q] = mk51::fe_mul(a[q], b);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint32_t w[8];
            mk51::fe_to_words(a[q], w);
#pragma unroll
            for (int i = 0; i < 8; i++) sum ^= w[i];
        }
    } else {
        mk::fe a[4], b;
#pragma unroll
        for (int i = 0; i < 10; i++) b.v[i] = (seed * (i + 3) + threadIdx.x) & 0x1ffffffu;
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int i = 0; i < 10; i++) a[q].v[i] = (threadIdx.x * 7 + q * 10 + i) & 0x1ffffffu;
        for (uint32_t it = 0; it < iters; it++)
#pragma unroll
            for (int q = 0; q < 4; q++) a[q] = mk::fe_mul(a[q], b);
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int i = 0; i < 10; i++) sum ^= a[q].v[i];
    }
    out[(uint64_t)blockIdx.x * blockDim.x + threadIdx.x] = sum;
}

cudaError_t measure_field_mul_rates(int sms, cudaStream_t st, double* radix32_per_s, double* radix26_per_s,
                                    double* radix51_per_s, bool* radix51_exact) {
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256, iters = 1u << 11;
    const size_t n = (size_t)blocks * threads;
    uint32_t* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(uint32_t) * n * 2);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best[3] = {0, 0, 0};
    auto launch = [&](int r, uint32_t it, uint32_t seed, uint32_t* o) {
        if (r == 0) k_fe_mul_rate<32><<<blocks, threads, 0, st>>>(it, seed, o);
        else if (r == 1) k_fe_mul_rate<26><<<blocks, threads, 0, st>>>(it, seed, o);
        else k_fe_mul_rate<51><<<blocks, threads, 0, st>>>(it, seed, o);
    };
    for (int r = 0; r < 3; r++) launch(r, iters / 16, 5u, out);
    for (int rep = 0; rep < 9 && e == cudaSuccess; rep++) {
        const int r = rep % 3;
        cudaEventRecord(e0, st);
        launch(r, iters, 9u + rep, out);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        const double muls = (double)n * iters * 4;
        if (ms > 0 && muls / (ms * 1e-3) > best[r]) best[r] = muls / (ms * 1e-3);
    }
    // exactness of radix 2^51: the same chains in radix 2^32 end in the same words
    bool same = false;
    if (e == cudaSuccess) {
        launch(0, 97, 3u, out);
        launch(2, 97, 3u, out + n);
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        std::vector<uint32_t> h(n * 2);
        e = cudaMemcpy(h.data(), out, sizeof(uint32_t) * n * 2, cudaMemcpyDeviceToHost);
        same = e == cudaSuccess && std::equal(h.begin(), h.begin() + n, h.begin() + n);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *radix32_per_s = best[0];
    *radix26_per_s = best[1];
    *radix51_per_s = best[2];
    *radix51_exact = same;
    return e;
}

// Products of operand pairs in both radix-2^32 forms: the words (below 2^256, not reduced
// to canonical) of a[i]·b[i] mod p, schoolbook into out_s and Karatsuba into out_k.
__global__ void k_fe_mul_pairs(const uint32_t* a, const uint32_t* b, uint32_t n, uint32_t* out_s, uint32_t* out_k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const mk32::fe x = mk32::fe_from_words(a + (size_t)i * 8), y = mk32::fe_from_words(b + (size_t)i * 8);
    const mk32::fe s = mk32::fe_mul_schoolbook(x, y), k = mk32::fe_mul_karatsuba(x, y);
#pragma unroll
    for (int w = 0; w < 8; w++) {
        out_s[(size_t)i * 8 + w] = s.v[w];
        out_k[(size_t)i * 8 + w] = k.v[w];
    }
}

cudaError_t field_mul_pairs(const uint32_t* a, const uint32_t* b, uint32_t n, uint32_t* out_s, uint32_t* out_k,
                            cudaStream_t st) {
    const size_t bytes = (size_t)n * 32;
    uint32_t* d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes * 4);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d, a, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d + (size_t)n * 8, b, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_fe_mul_pairs<<<(n + 255) / 256, 256, 0, st>>>(d, d + (size_t)n * 8, n, d + (size_t)n * 16,
                                                        d + (size_t)n * 24);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_s, d + (size_t)n * 16, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_k, d + (size_t)n * 24, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const cudaError_t ef = cudaFree(d);
    return e != cudaSuccess ? e : ef;
}

// Rates of the two radix-2^32 multiplication forms (schoolbook and Karatsuba), measured like
// measure_field_mul_rates, and whether their chains end in the same words.
cudaError_t measure_field_mul_forms(int sms, cudaStream_t st, double* schoolbook_per_s, double* karatsuba_per_s,
                                    bool* same_words) {
    const uint32_t blocks = (uint32_t)sms * 8, threads = 256, iters = 1u << 11;
    const size_t n = (size_t)blocks * threads;
    uint32_t* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(uint32_t) * n * 2);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best[2] = {0, 0};
    auto launch = [&](int k, uint32_t it, uint32_t seed, uint32_t* o) {
        if (k == 0) k_fe_mul_rate<32><<<blocks, threads, 0, st>>>(it, seed, o);
        else k_fe_mul_rate<33><<<blocks, threads, 0, st>>>(it, seed, o);
    };
    for (int k = 0; k < 2; k++) launch(k, iters / 16, 5u, out);
    for (int rep = 0; rep < 8 && e == cudaSuccess; rep++) {
        const int k = rep & 1;
        cudaEventRecord(e0, st);
        launch(k, iters, 9u + rep, out);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        const double muls = (double)n * iters * 4;
        if (ms > 0 && muls / (ms * 1e-3) > best[k]) best[k] = muls / (ms * 1e-3);
    }
    bool same = false;
    if (e == cudaSuccess) {
        launch(0, 97, 3u, out);
        launch(1, 97, 3u, out + n);
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        std::vector<uint32_t> h(n * 2);
        e = cudaMemcpy(h.data(), out, sizeof(uint32_t) * n * 2, cudaMemcpyDeviceToHost);
        same = e == cudaSuccess && std::equal(h.begin(), h.begin() + n, h.begin() + n);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *schoolbook_per_s = best[0];
    *karatsuba_per_s = best[1];
    *same_words = same;
    return e;
}

}  // namespace mkb

// ---------------------------------------------------------------------------
// Derive without allocation: fixed device staging for mk_derive_noalloc
// ---------------------------------------------------------------------------

namespace mkb {

// Device-side staging of the public keys written by mk_derive_noalloc: 65536 keys of 32
// bytes (2 MiB).  It is a file-scope device array, so every GPU that loads this library
// holds it until the process exits, and no call has to allocate device memory for it.
static __device__ __align__(256) uint8_t g_noalloc_pubkeys[NOALLOC_MAX_KEYS * 32];

// Device address of g_noalloc_pubkeys on the current device.  The name of the array in host
// code is only a host-side stand-in; its address on the device comes from
// cudaGetSymbolAddress, which the context looks up once when it is created (with its device
// current) and keeps, so it lives and dies with the context's other device memory.
cudaError_t noalloc_staging(uint8_t** ptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_pubkeys);
    if (e != cudaSuccess) return e;
    *ptr = static_cast<uint8_t*>(p);
    return cudaSuccess;
}

}  // namespace mkb
