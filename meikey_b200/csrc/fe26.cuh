// GF(2^255 - 19) in ten limbs of alternating 26 and 25 bits (radix 2^25.5).
//
// Products are 32x32->64-bit multiply-adds (mad.wide.u32, one IMAD.WIDE each),
// accumulated in 64-bit column sums, so a multiplication is 100 wide MADs,
// 9 small premultiplications by 19 and one carry pass.  Exact integer math, no FP.
//
// Limb bounds (let "1x" mean limbs below 2^26 / 2^25 for even / odd index):
//   fe_mul(f, g): f below 5x, g below 3.25x (19·g must fit 32 bits); result 1x (+tiny in limb 1)
//   fe_add: sums the bounds; fe_sub(a, b) = a + 2p - b needs b at most 1x + small
// These are the same bounds ref10-style 10-limb code uses; the 64-bit column sums of
// the unsigned form have a factor two more headroom than the signed form.
#pragma once
#include <stdint.h>

namespace mk {

typedef uint32_t u32;
typedef uint64_t u64;

struct fe {
    u32 v[10];
};

#define MK_M26 0x3ffffffu
#define MK_M25 0x1ffffffu

__device__ __forceinline__ fe fe_zero() {
    fe r;
#pragma unroll
    for (int i = 0; i < 10; i++) r.v[i] = 0;
    return r;
}

__device__ __forceinline__ fe fe_small(u32 x) {
    fe r = fe_zero();
    r.v[0] = x;
    return r;
}

__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
    fe r;
#pragma unroll
    for (int i = 0; i < 10; i++) r.v[i] = a.v[i] + b.v[i];
    return r;
}

// a + 2p - b  (b limbs must not exceed 2p's limbs)
__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
    fe r;
    r.v[0] = a.v[0] + 2u * (MK_M26 - 18u) - b.v[0];
#pragma unroll
    for (int i = 1; i < 10; i++) r.v[i] = a.v[i] + ((i & 1) ? 2u * MK_M25 : 2u * MK_M26) - b.v[i];
    return r;
}

// a + 4p - b (for b up to 3x)
__device__ __forceinline__ fe fe_sub4(const fe& a, const fe& b) {
    fe r;
    r.v[0] = a.v[0] + 4u * (MK_M26 - 18u) - b.v[0];
#pragma unroll
    for (int i = 1; i < 10; i++) r.v[i] = a.v[i] + ((i & 1) ? 4u * MK_M25 : 4u * MK_M26) - b.v[i];
    return r;
}

// carry a 64-bit column vector into 1x limbs
__device__ __forceinline__ fe fe_carry64(u64 h[10]) {
    u64 c;
    c = h[0] >> 26; h[1] += c; h[0] &= MK_M26;
    c = h[4] >> 26; h[5] += c; h[4] &= MK_M26;
    c = h[1] >> 25; h[2] += c; h[1] &= MK_M25;
    c = h[5] >> 25; h[6] += c; h[5] &= MK_M25;
    c = h[2] >> 26; h[3] += c; h[2] &= MK_M26;
    c = h[6] >> 26; h[7] += c; h[6] &= MK_M26;
    c = h[3] >> 25; h[4] += c; h[3] &= MK_M25;
    c = h[7] >> 25; h[8] += c; h[7] &= MK_M25;
    c = h[4] >> 26; h[5] += c; h[4] &= MK_M26;
    c = h[8] >> 26; h[9] += c; h[8] &= MK_M26;
    c = h[9] >> 25; h[0] += c * 19u; h[9] &= MK_M25;
    c = h[0] >> 26; h[1] += c; h[0] &= MK_M26;
    fe r;
#pragma unroll
    for (int i = 0; i < 10; i++) r.v[i] = (u32)h[i];
    return r;
}

// limbs back to 1x after additions (32-bit version)
__device__ __forceinline__ fe fe_carry(const fe& a) {
    u32 h[10];
#pragma unroll
    for (int i = 0; i < 10; i++) h[i] = a.v[i];
    u32 c;
    c = h[0] >> 26; h[1] += c; h[0] &= MK_M26;
    c = h[4] >> 26; h[5] += c; h[4] &= MK_M26;
    c = h[1] >> 25; h[2] += c; h[1] &= MK_M25;
    c = h[5] >> 25; h[6] += c; h[5] &= MK_M25;
    c = h[2] >> 26; h[3] += c; h[2] &= MK_M26;
    c = h[6] >> 26; h[7] += c; h[6] &= MK_M26;
    c = h[3] >> 25; h[4] += c; h[3] &= MK_M25;
    c = h[7] >> 25; h[8] += c; h[7] &= MK_M25;
    c = h[4] >> 26; h[5] += c; h[4] &= MK_M26;
    c = h[8] >> 26; h[9] += c; h[8] &= MK_M26;
    c = h[9] >> 25; h[0] += c * 19u; h[9] &= MK_M25;
    c = h[0] >> 26; h[1] += c; h[0] &= MK_M26;
    fe r;
#pragma unroll
    for (int i = 0; i < 10; i++) r.v[i] = h[i];
    return r;
}

__device__ __forceinline__ u64 wmad(u32 a, u32 b, u64 c) { return (u64)a * b + c; }

// h = f * g mod p
__device__ __forceinline__ fe fe_mul(const fe& f, const fe& g) {
    u32 g19[10];
#pragma unroll
    for (int j = 1; j < 10; j++) g19[j] = 19u * g.v[j];
    u32 f2[10];
#pragma unroll
    for (int i = 1; i < 10; i += 2) f2[i] = 2u * f.v[i];
    u64 h[10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        u64 acc = 0;
#pragma unroll
        for (int i = 0; i < 10; i++) {
            int j = k - i;
            bool wrap = j < 0;
            if (wrap) j += 10;
            // odd x odd limbs carry an extra factor 2 in radix 2^25.5
            u32 fi = ((i & 1) && (j & 1)) ? f2[i] : f.v[i];
            u32 gj = wrap ? g19[j] : g.v[j];
            acc = wmad(fi, gj, acc);
        }
        h[k] = acc;
    }
    return fe_carry64(h);
}

// f^2: symmetric products doubled (55 wide MADs)
__device__ __forceinline__ fe fe_sq(const fe& f) {
    u32 f2[10], f19[10], f38[10];
#pragma unroll
    for (int i = 0; i < 10; i++) {
        f2[i] = 2u * f.v[i];
        f19[i] = 19u * f.v[i];
        f38[i] = 38u * f.v[i];
    }
    u64 h[10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        u64 acc = 0;
#pragma unroll
        for (int i = 0; i < 10; i++) {
#pragma unroll
            for (int j = i; j < 10; j++) {
                int s = i + j;
                if (s != k && s != k + 10) continue;
                bool wrap = s >= 10;
                int m = ((i & 1) && (j & 1)) ? 2 : 1;   // radix factor
                int d = (i == j) ? 1 : 2;                // symmetric pair
                int fac = m * d;                         // 1, 2 or 4
                u32 a, b;
                if (fac == 1) { a = f.v[i]; b = wrap ? f19[j] : f.v[j]; }
                else if (fac == 2) { a = f2[i]; b = wrap ? f19[j] : f.v[j]; }
                else { a = f2[i]; b = wrap ? f38[j] : f2[j]; }
                acc = wmad(a, b, acc);
            }
        }
        h[k] = acc;
    }
    return fe_carry64(h);
}

// Canonical little-endian value as 8 words.  Exact for any limbs below 2^32:
// two sequential carry passes with the overflow above 2^255 folded back as 19,
// then one conditional subtraction of p.
__device__ __forceinline__ void fe_to_words(const fe& a, u32 out[8]) {
    u32 t[10];
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < 10; i++) {
        u64 x = (u64)a.v[i] + c;
        int bits = (i & 1) ? 25 : 26;
        t[i] = (u32)x & ((1u << bits) - 1u);
        c = x >> bits;
    }
    u64 x0 = (u64)t[0] + 19u * c;
    c = 0;
#pragma unroll
    for (int i = 0; i < 10; i++) {
        u64 x = (i == 0 ? x0 : (u64)t[i]) + c;
        int bits = (i & 1) ? 25 : 26;
        t[i] = (u32)x & ((1u << bits) - 1u);
        c = x >> bits;
    }
    t[0] += 19u * (u32)c;  // c is 0 or 1; when 1 the remaining value is tiny
    // now every limb is proper and the value is below 2^255; subtract p if value >= p
    u32 q = (t[0] + 19u) >> 26;
#pragma unroll
    for (int i = 1; i < 10; i++) q = (t[i] + q) >> ((i & 1) ? 25 : 26);
    t[0] += 19u * q;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        int bits = (i & 1) ? 25 : 26;
        u32 cc = t[i] >> bits;
        t[i] &= (1u << bits) - 1u;
        t[i + 1] += cc;
    }
    t[9] &= MK_M25;
    // pack: limb i starts at bit ceil(25.5 i)
    out[0] = t[0] | t[1] << 26;
    out[1] = t[1] >> 6 | t[2] << 19;
    out[2] = t[2] >> 13 | t[3] << 13;
    out[3] = t[3] >> 19 | t[4] << 6;
    out[4] = t[5] | t[6] << 25;
    out[5] = t[6] >> 7 | t[7] << 19;
    out[6] = t[7] >> 13 | t[8] << 12;
    out[7] = t[8] >> 20 | t[9] << 6;
}

// From 8 little-endian words of a value below 2^256 (bit 255 folded as 19).
__device__ __forceinline__ fe fe_from_words(const u32 w[8]) {
    fe r;
    r.v[0] = w[0] & MK_M26;
    r.v[1] = (w[0] >> 26 | w[1] << 6) & MK_M25;
    r.v[2] = (w[1] >> 19 | w[2] << 13) & MK_M26;
    r.v[3] = (w[2] >> 13 | w[3] << 19) & MK_M25;
    r.v[4] = (w[3] >> 6) & MK_M26;
    r.v[5] = w[4] & MK_M25;
    r.v[6] = (w[4] >> 25 | w[5] << 7) & MK_M26;
    r.v[7] = (w[5] >> 19 | w[6] << 13) & MK_M25;
    r.v[8] = (w[6] >> 12 | w[7] << 20) & MK_M26;
    r.v[9] = (w[7] >> 6) & MK_M25;
    r.v[0] += 19u * (w[7] >> 31);
    return r;
}

}  // namespace mk
