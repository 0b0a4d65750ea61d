// GF(2^255 - 19) in five signed limbs of radix 2^51 held in FP64 registers: the value is
// sum v[i] * 2^(51 i), each v[i] an integer.  B200 runs FP64 fused multiply-adds at the same
// rate as 32-bit integer multiply-adds, on a different pipe, so a multiply here leaves the
// IMAD pipe free.
//
// Limb products are split exactly into a high and a low half by two fused multiply-adds
// (the method of Emmart, Zheng and Weems, "Faster modular exponentiation using double
// precision floating point arithmetic on the GPU", ARITH 2018), here in a signed form: for
// integers a, b with |ab| < 2^103 and S = 1.5 * 2^104,
//   t = fma_rz(a, b, S)                 = S + floor(ab / 2^52) * 2^52       in [2^104, 2^105)
//   l = fma_rn(a, b, (S + 2^52) - t)     = 2^52 + (ab mod 2^52)              in [2^52, 2^53)
// Both results sit in a binade of fixed exponent, so their bit patterns, read as integers, are
// a constant plus floor(ab / 2^52) or (ab mod 2^52).  A column sums those patterns in 64-bit
// integers and takes the constants off once; the high halves weigh 2^52 = 2 * 2^51, i.e. twice
// a unit of the next column.  Exact integer arithmetic throughout, no rounding of values.
//
// Bounds kept by every caller:
//   - fe_mul / fe_mul_words: |a_i * b_j| < 2^103 for all limb pairs;
//   - fe_sq: |a_i| < 2^51;
//   - fe_carry: |limb| <= 2^53;  fe_to_words: carried input;
//   - results of fe_mul, fe_sq, fe_carry and fe_from_words have |limb| <= 2^50 + 64
//     ("carried"); a sum or difference of two carried values has |limb| <= 2^51 + 128, and a
//     product of two such sums stays below 2^103.
#pragma once
#include <stdint.h>

namespace mk51 {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

struct fe {
    double v[5];
};

constexpr double SPLIT = 0x1.8p+104;                // S = 1.5 * 2^104
constexpr double SPLIT_LO = 0x1.8p+104 + 0x1p+52;   // S + 2^52 (exact)
constexpr double ROUND51 = 0x1.8p+103;              // adding it rounds to a multiple of 2^51
constexpr double CENTER52 = 0x1.8p+52;              // |x| < 2^51 -> x + 1.5 * 2^52 in [2^52, 2^53)
constexpr double INV51 = 0x1p-51;
constexpr double FOLD51 = 19.0 * 0x1p-51;           // 2^255 = 19 (mod p), seen from limb 4
constexpr u64 SPLIT_BITS = 0x4678000000000000ull;   // bit pattern of S
constexpr u64 LO_BITS = 0x4330000000000000ull;      // bit pattern of 2^52
constexpr u64 CENTER_BITS = 0x4338000000000000ull;  // bit pattern of 1.5 * 2^52
constexpr u64 M51 = (1ull << 51) - 1;

__device__ __forceinline__ u64 dbits(double d) { return (u64)__double_as_longlong(d); }
__device__ __forceinline__ double bitsd(u64 b) { return __longlong_as_double((long long)b); }

// a signed integer |x| < 2^51 as a double, and back
__device__ __forceinline__ double i2d(i64 x) { return __dsub_rn(bitsd(CENTER_BITS + (u64)x), CENTER52); }
__device__ __forceinline__ i64 d2i(double x) { return (i64)(dbits(__dadd_rn(x, CENTER52)) - CENTER_BITS); }

__device__ __forceinline__ fe fe_zero() {
    fe r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = 0.0;
    return r;
}

__device__ __forceinline__ fe fe_small(u32 x) {
    fe r = fe_zero();
    r.v[0] = (double)x;
    return r;
}

__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
    fe r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = __dadd_rn(a.v[i], b.v[i]);
    return r;
}

__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
    fe r;
#pragma unroll
    for (int i = 0; i < 5; i++) r.v[i] = __dsub_rn(a.v[i], b.v[i]);
    return r;
}

// Limbs of |v| <= 2^53 brought to |limb| <= 2^50 + 64 in FP64: each limb is rounded to its
// nearest multiple of 2^51, which moves to the next limb (from limb 4: times 19 into limb 0).
__device__ __forceinline__ fe fe_carry(fe a) {
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const double m = __dsub_rn(__dadd_rn(a.v[i], ROUND51), ROUND51);
        a.v[i] = __dsub_rn(a.v[i], m);
        if (i < 4) a.v[i + 1] = __fma_rn(m, INV51, a.v[i + 1]);
        else a.v[0] = __fma_rn(m, FOLD51, a.v[0]);
    }
    return a;
}

// one limb product added to its column: lo += pattern of 2^52 + (ab mod 2^52),
// hi += pattern of S + floor(ab / 2^52) * 2^52
__device__ __forceinline__ void split_add(double a, double b, u64& lo, u64& hi) {
    const double t = __fma_rz(a, b, SPLIT);
    const double l = __fma_rn(a, b, __dsub_rn(SPLIT_LO, t));
    lo += dbits(l);
    hi += dbits(t);
}

// Columns to five centered 64-bit limbs.  n[k] is the number of products summed in column k.
// Column k is (lo[k] - n[k] LO_BITS) + 2 (hi[k-1] - n[k-1] SPLIT_BITS), all mod 2^64 (the
// true value is far inside the signed range); columns 5..9 fold down times 19.
template <int N0, int N1, int N2, int N3, int N4, int N5, int N6, int N7, int N8>
__device__ __forceinline__ void columns_to_limbs(const u64 lo[9], const u64 hi[9], i64 r[5]) {
    const u64 n[9] = {N0, N1, N2, N3, N4, N5, N6, N7, N8};
    i64 c[10];
#pragma unroll
    for (int k = 0; k < 10; k++) {
        u64 x = 0;
        if (k < 9) x += lo[k] - n[k] * LO_BITS;
        if (k >= 1) x += 2 * (hi[k - 1] - n[k - 1] * SPLIT_BITS);
        c[k] = (i64)x;
    }
#pragma unroll
    for (int k = 0; k < 5; k++) r[k] = c[k] + 19 * c[k + 5];
    // centered carries: limb k to [-2^50, 2^50), the excess to limb k + 1 (limb 4's times 19 to limb 0)
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const i64 q = (r[k] + (1ll << 50)) >> 51;
        r[k] -= q << 51;
        if (k < 4) r[k + 1] += q;
        else r[0] += 19 * q;
    }
    const i64 q = (r[0] + (1ll << 50)) >> 51;
    r[0] -= q << 51;
    r[1] += q;
}

__device__ __forceinline__ void mul_limbs(const fe& a, const fe& b, i64 r[5]) {
    u64 lo[9], hi[9];
#pragma unroll
    for (int k = 0; k < 9; k++) lo[k] = hi[k] = 0;
#pragma unroll
    for (int i = 0; i < 5; i++)
#pragma unroll
        for (int j = 0; j < 5; j++) split_add(a.v[i], b.v[j], lo[i + j], hi[i + j]);
    columns_to_limbs<1, 2, 3, 4, 5, 4, 3, 2, 1>(lo, hi, r);
}

__device__ __forceinline__ fe limbs_to_fe(const i64 r[5]) {
    fe o;
#pragma unroll
    for (int i = 0; i < 5; i++) o.v[i] = i2d(r[i]);
    return o;
}

__device__ __forceinline__ fe fe_mul(const fe& a, const fe& b) {
    i64 r[5];
    mul_limbs(a, b, r);
    return limbs_to_fe(r);
}

// a^2: ten cross products taken once with 2 a_i, five squares
__device__ __forceinline__ fe fe_sq(const fe& a) {
    u64 lo[9], hi[9];
#pragma unroll
    for (int k = 0; k < 9; k++) lo[k] = hi[k] = 0;
    double d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = __dadd_rn(a.v[i], a.v[i]);
#pragma unroll
    for (int i = 0; i < 5; i++) {
        split_add(a.v[i], a.v[i], lo[2 * i], hi[2 * i]);
#pragma unroll
        for (int j = i + 1; j < 5; j++) split_add(d[i], a.v[j], lo[i + j], hi[i + j]);
    }
    i64 r[5];
    columns_to_limbs<1, 1, 2, 2, 3, 2, 2, 1, 1>(lo, hi, r);
    return limbs_to_fe(r);
}

// Canonical value (mod p) of 64-bit limbs with |limb| < 2^53 as 8 little-endian words
__device__ __forceinline__ void limbs_to_words(const i64 in[5], u32 out[8]) {
    // + 8p, limb by limb (8 (2^51 - 19), then 8 (2^51 - 1)), makes every limb positive
    u64 r[5];
#pragma unroll
    for (int i = 0; i < 5; i++) r[i] = (u64)(in[i] + 8 * ((1ll << 51) - (i == 0 ? 19 : 1)));
    // two carry passes: the first leaves limb 0 below 2^51 + 19 * 10, the second below 2^51
    // (if its fold fires, the value was under 2^255 + 190, so every limb is already small)
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            r[i + 1] += r[i] >> 51;
            r[i] &= M51;
        }
        const u64 q = r[4] >> 51;
        r[4] &= M51;
        r[0] += 19 * q;
    }
    // x < 2^255: subtract p when x >= p, i.e. when x + 19 reaches 2^255
    u64 t[5];
    u64 c = 19;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        t[i] = r[i] + c;
        c = t[i] >> 51;
        t[i] &= M51;
    }
    const bool ge = c != 0;
#pragma unroll
    for (int i = 0; i < 5; i++) r[i] = ge ? t[i] : r[i];
    const u64 w[4] = {r[0] | r[1] << 51, r[1] >> 13 | r[2] << 38, r[2] >> 26 | r[3] << 25, r[3] >> 39 | r[4] << 12};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        out[2 * i] = (u32)w[i];
        out[2 * i + 1] = (u32)(w[i] >> 32);
    }
}

__device__ __forceinline__ void fe_to_words(const fe& a, u32 out[8]) {
    i64 r[5];
#pragma unroll
    for (int i = 0; i < 5; i++) r[i] = d2i(a.v[i]);
    limbs_to_words(r, out);
}

// y = a * b straight to canonical words (the product's limbs are not converted back to FP64)
__device__ __forceinline__ void fe_mul_words(const fe& a, const fe& b, u32 out[8]) {
    i64 r[5];
    mul_limbs(a, b, r);
    limbs_to_words(r, out);
}

// 8 little-endian words (any 256-bit value) to centered limbs
__device__ __forceinline__ fe fe_from_words(const u32 w[8]) {
    u64 q[4];
#pragma unroll
    for (int i = 0; i < 4; i++) q[i] = (u64)w[2 * i] | (u64)w[2 * i + 1] << 32;
    i64 r[5] = {(i64)(q[0] & M51), (i64)((q[0] >> 51 | q[1] << 13) & M51), (i64)((q[1] >> 38 | q[2] << 26) & M51),
                (i64)((q[2] >> 25 | q[3] << 39) & M51), (i64)(q[3] >> 12)};
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const i64 c = (r[k] + (1ll << 50)) >> 51;
        r[k] -= c << 51;
        if (k < 4) r[k + 1] += c;
        else r[0] += 19 * c;
    }
    return limbs_to_fe(r);
}

}  // namespace mk51
