// GF(2^255 - 19) in eight 32-bit limbs (radix 2^32), values kept below 2^256
// (congruent mod p, not canonical).  Products use hand-written mad.lo.cc /
// madc.hi.cc carry chains; 2^256 is folded back as 38.  Exact integer math, no FP.
#pragma once
#include <stdint.h>

namespace mk32 {

typedef uint32_t u32;
typedef uint64_t u64;

struct fe {
    u32 v[8];
};

__device__ __forceinline__ fe fe_zero() {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = 0;
    return r;
}

__device__ __forceinline__ fe fe_small(u32 x) {
    fe r = fe_zero();
    r.v[0] = x;
    return r;
}

// r = a + b mod 2^256 folded: a carry out of bit 256 adds 38
__device__ __forceinline__ fe fe_add(const fe& a, const fe& b) {
    fe r;
    u32 c;
    asm("add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(c)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // fold: r += 38·c; a second carry is impossible to miss: it leaves r < 38, and 38 more fits
    u32 add = 38u * c, c2;
    asm("add.cc.u32 %0, %0, %9;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, 0;\n\t"
        "addc.cc.u32 %6, %6, 0;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7]), "=r"(c2)
        : "r"(add));
    r.v[0] += 38u * c2;
    return r;
}

// r = a - b; a borrow subtracts 38 (2^256 ≡ 38)
__device__ __forceinline__ fe fe_sub(const fe& a, const fe& b) {
    fe r;
    u32 bw;
    asm("sub.cc.u32 %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32 %8, 0, 0;\n\t"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(bw)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]),
          "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // bw is 0 or 0xffffffff
    u32 sub = 38u & bw, b2;
    asm("sub.cc.u32 %0, %0, %9;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.cc.u32 %2, %2, 0;\n\t"
        "subc.cc.u32 %3, %3, 0;\n\t"
        "subc.cc.u32 %4, %4, 0;\n\t"
        "subc.cc.u32 %5, %5, 0;\n\t"
        "subc.cc.u32 %6, %6, 0;\n\t"
        "subc.cc.u32 %7, %7, 0;\n\t"
        "subc.u32 %8, 0, 0;\n\t"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7]), "=r"(b2)
        : "r"(sub));
    // a second borrow leaves r >= 2^256 - 38, so 38 less cannot borrow again
    r.v[0] -= 38u & b2;
    return r;
}

// Fold a 512-bit product t[0..15] to 8 words: t_lo + 38·t_hi, then the top word again.
__device__ __forceinline__ fe fe_reduce512(const u32 t[16]) {
    fe r;
    u32 top;
    // lo parts of 38·t[8+j] into words j, carries through
    asm("mad.lo.cc.u32 %0, %9, 38, %17;\n\t"
        "madc.lo.cc.u32 %1, %10, 38, %18;\n\t"
        "madc.lo.cc.u32 %2, %11, 38, %19;\n\t"
        "madc.lo.cc.u32 %3, %12, 38, %20;\n\t"
        "madc.lo.cc.u32 %4, %13, 38, %21;\n\t"
        "madc.lo.cc.u32 %5, %14, 38, %22;\n\t"
        "madc.lo.cc.u32 %6, %15, 38, %23;\n\t"
        "madc.lo.cc.u32 %7, %16, 38, %24;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]), "=r"(r.v[6]),
          "=r"(r.v[7]), "=r"(top)
        : "r"(t[8]), "r"(t[9]), "r"(t[10]), "r"(t[11]), "r"(t[12]), "r"(t[13]), "r"(t[14]), "r"(t[15]),
          "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]));
    // hi parts of 38·t[8+j] into words j+1
    asm("mad.hi.cc.u32 %1, %9, 38, %1;\n\t"
        "madc.hi.cc.u32 %2, %10, 38, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, 38, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, 38, %4;\n\t"
        "madc.hi.cc.u32 %5, %13, 38, %5;\n\t"
        "madc.hi.cc.u32 %6, %14, 38, %6;\n\t"
        "madc.hi.cc.u32 %7, %15, 38, %7;\n\t"
        "madc.hi.u32 %8, %16, 38, %8;\n\t"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7]), "+r"(top)
        : "r"(t[8]), "r"(t[9]), "r"(t[10]), "r"(t[11]), "r"(t[12]), "r"(t[13]), "r"(t[14]), "r"(t[15]));
    // top < 40: fold 38·top; one more carry is possible and is folded as 38 without further carry
    u32 add = 38u * top, c2;
    asm("add.cc.u32 %0, %0, %9;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\t"
        "addc.cc.u32 %3, %3, 0;\n\t"
        "addc.cc.u32 %4, %4, 0;\n\t"
        "addc.cc.u32 %5, %5, 0;\n\t"
        "addc.cc.u32 %6, %6, 0;\n\t"
        "addc.cc.u32 %7, %7, 0;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]), "+r"(r.v[6]),
          "+r"(r.v[7]), "=r"(c2)
        : "r"(add));
    r.v[0] += 38u * c2;
    return r;
}

// One row of the operand-scanning product: t[i..i+8] += a · b_i.
// Even-indexed a_j go in one carry chain (their lo/hi pairs tile words i..i+7),
// odd-indexed a_j in a second chain (words i+1..i+8).
#define MK32_ROW(I)                                                                                  \
    asm("mad.lo.cc.u32 %0, %9, %13, %0;\n\t"                                                        \
        "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"                                                       \
        "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"                                                      \
        "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"                                                      \
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"                                                      \
        "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"                                                      \
        "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"                                                      \
        "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"                                                      \
        "addc.u32 %8, %8, 0;\n\t"                                                                   \
        : "+r"(t[I]), "+r"(t[I + 1]), "+r"(t[I + 2]), "+r"(t[I + 3]), "+r"(t[I + 4]), "+r"(t[I + 5]), \
          "+r"(t[I + 6]), "+r"(t[I + 7]), "+r"(t[I + 8])                                            \
        : "r"(a.v[0]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]), "r"(b.v[I]));                         \
    asm("mad.lo.cc.u32 %0, %8, %12, %0;\n\t"                                                        \
        "madc.hi.cc.u32 %1, %8, %12, %1;\n\t"                                                       \
        "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"                                                       \
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"                                                       \
        "madc.lo.cc.u32 %4, %10, %12, %4;\n\t"                                                      \
        "madc.hi.cc.u32 %5, %10, %12, %5;\n\t"                                                      \
        "madc.lo.cc.u32 %6, %11, %12, %6;\n\t"                                                      \
        "madc.hi.u32 %7, %11, %12, %7;\n\t"                                                         \
        : "+r"(t[I + 1]), "+r"(t[I + 2]), "+r"(t[I + 3]), "+r"(t[I + 4]), "+r"(t[I + 5]),             \
          "+r"(t[I + 6]), "+r"(t[I + 7]), "+r"(t[I + 8])                                            \
        : "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]), "r"(b.v[I]));

// r = a·b mod p (as a value below 2^256), schoolbook: 64 lo + 64 hi products
__device__ __forceinline__ fe fe_mul_schoolbook(const fe& a, const fe& b) {
    u32 t[16];
#pragma unroll
    for (int i = 0; i < 16; i++) t[i] = 0;
    // after row I the partial sum is below 2^(32(I+9)), so word I+8 absorbs the final carry
    MK32_ROW(0) MK32_ROW(1) MK32_ROW(2) MK32_ROW(3) MK32_ROW(4) MK32_ROW(5) MK32_ROW(6) MK32_ROW(7)
    return fe_reduce512(t);
}

// One row of a 128 x 128-bit product: T[I..I+4] += X · Y_I, the even X limbs in one carry
// chain and the odd ones in a second; after row I the sum is below 2^(32(I+5)).
#define MK32_ROW4(T, X, Y, I)                                                                        \
    asm("mad.lo.cc.u32 %0, %5, %7, %0;\n\t"                                                          \
        "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"                                                         \
        "madc.lo.cc.u32 %2, %6, %7, %2;\n\t"                                                         \
        "madc.hi.cc.u32 %3, %6, %7, %3;\n\t"                                                         \
        "addc.u32 %4, %4, 0;\n\t"                                                                    \
        : "+r"(T[I]), "+r"(T[I + 1]), "+r"(T[I + 2]), "+r"(T[I + 3]), "+r"(T[I + 4])                 \
        : "r"(X[0]), "r"(X[2]), "r"(Y[I]));                                                          \
    asm("mad.lo.cc.u32 %0, %4, %6, %0;\n\t"                                                          \
        "madc.hi.cc.u32 %1, %4, %6, %1;\n\t"                                                         \
        "madc.lo.cc.u32 %2, %5, %6, %2;\n\t"                                                         \
        "madc.hi.u32 %3, %5, %6, %3;\n\t"                                                            \
        : "+r"(T[I + 1]), "+r"(T[I + 2]), "+r"(T[I + 3]), "+r"(T[I + 4])                             \
        : "r"(X[1]), "r"(X[3]), "r"(Y[I]));

// t[0..7] = x · y for 128-bit x, y (four limbs each): 16 lo + 16 hi products
__device__ __forceinline__ void mul128(const u32 x[4], const u32 y[4], u32 t[8]) {
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = 0;
    MK32_ROW4(t, x, y, 0) MK32_ROW4(t, x, y, 1) MK32_ROW4(t, x, y, 2) MK32_ROW4(t, x, y, 3)
}

// d = |x - y| for 128-bit x, y; returns all ones when x < y, else 0
__device__ __forceinline__ u32 absdiff128(const u32 x[4], const u32 y[4], u32 d[4]) {
    u32 s;
    asm("sub.cc.u32 %0, %5, %9;\n\t"
        "subc.cc.u32 %1, %6, %10;\n\t"
        "subc.cc.u32 %2, %7, %11;\n\t"
        "subc.cc.u32 %3, %8, %12;\n\t"
        "subc.u32 %4, 0, 0;\n\t"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(s)
        : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]));
    // negative: (d ^ s) - s = 2^128 - d, the magnitude
#pragma unroll
    for (int i = 0; i < 4; i++) d[i] ^= s;
    asm("sub.cc.u32 %0, %0, %4;\n\t"
        "subc.cc.u32 %1, %1, %4;\n\t"
        "subc.cc.u32 %2, %2, %4;\n\t"
        "subc.u32 %3, %3, %4;\n\t"
        : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
        : "r"(s));
    return s;
}

// r = a·b mod p by one level of subtractive Karatsuba on the 128-bit halves
// (a = A1·2^128 + A0): A0·B1 + A1·B0 = L + H - (A0 - A1)·(B0 - B1) with L = A0·B0 and
// H = A1·B1, so the 512-bit product takes 48 lo + 48 hi products and about 60 adds and
// logic operations instead of 64 + 64.  Both operands use the same difference X0 - X1, so an
// operand that enters several products (the point-addition outputs' E, F, G, H) has one
// |X0 - X1| the compiler can share.  The product t is the same 512-bit integer as the
// schoolbook's, and so is the folded result.
__device__ __forceinline__ fe fe_mul_karatsuba(const fe& a, const fe& b) {
    u32 da[4], db[4], mm[8], lo[8], hi[8], mid[9];
    const u32 sa = absdiff128(&a.v[0], &a.v[4], da);
    const u32 sb = absdiff128(&b.v[0], &b.v[4], db);
    // (A0 - A1)(B0 - B1) is subtracted, so |..|·|..| is subtracted when the signs agree
    const u32 s = ~(sa ^ sb);  // all ones: the middle product is subtracted
    mul128(da, db, mm);
    mul128(&a.v[0], &b.v[0], lo);
    mul128(&a.v[4], &b.v[4], hi);
    // mid = L + H, nine words
    asm("add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        : "=r"(mid[0]), "=r"(mid[1]), "=r"(mid[2]), "=r"(mid[3]), "=r"(mid[4]), "=r"(mid[5]), "=r"(mid[6]),
          "=r"(mid[7]), "=r"(mid[8])
        : "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]),
          "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]), "r"(hi[4]), "r"(hi[5]), "r"(hi[6]), "r"(hi[7]));
    // mid += ±M mod 2^288: (M ^ s) with a ninth word s, plus a carry-in of s & 1 (set by s + s);
    // the true value A0·B1 + A1·B0 lies in [0, 2^257)
#pragma unroll
    for (int i = 0; i < 8; i++) mm[i] ^= s;
    asm("{\n\t"
        ".reg .u32 cf;\n\t"
        "add.cc.u32 cf, %9, %9;\n\t"
        "addc.cc.u32 %0, %0, %10;\n\t"
        "addc.cc.u32 %1, %1, %11;\n\t"
        "addc.cc.u32 %2, %2, %12;\n\t"
        "addc.cc.u32 %3, %3, %13;\n\t"
        "addc.cc.u32 %4, %4, %14;\n\t"
        "addc.cc.u32 %5, %5, %15;\n\t"
        "addc.cc.u32 %6, %6, %16;\n\t"
        "addc.cc.u32 %7, %7, %17;\n\t"
        "addc.u32 %8, %8, %9;\n\t"
        "}"
        : "+r"(mid[0]), "+r"(mid[1]), "+r"(mid[2]), "+r"(mid[3]), "+r"(mid[4]), "+r"(mid[5]), "+r"(mid[6]),
          "+r"(mid[7]), "+r"(mid[8])
        : "r"(s), "r"(mm[0]), "r"(mm[1]), "r"(mm[2]), "r"(mm[3]), "r"(mm[4]), "r"(mm[5]), "r"(mm[6]), "r"(mm[7]));
    // t = L + mid·2^128 + H·2^256 (below 2^512: no carry out of word 15)
    u32 t[16];
    t[0] = lo[0];
    t[1] = lo[1];
    t[2] = lo[2];
    t[3] = lo[3];
    asm("add.cc.u32 %0, %12, %24;\n\t"
        "addc.cc.u32 %1, %13, %25;\n\t"
        "addc.cc.u32 %2, %14, %26;\n\t"
        "addc.cc.u32 %3, %15, %27;\n\t"
        "addc.cc.u32 %4, %16, %28;\n\t"
        "addc.cc.u32 %5, %17, %29;\n\t"
        "addc.cc.u32 %6, %18, %30;\n\t"
        "addc.cc.u32 %7, %19, %31;\n\t"
        "addc.cc.u32 %8, %20, %32;\n\t"
        "addc.cc.u32 %9, %21, 0;\n\t"
        "addc.cc.u32 %10, %22, 0;\n\t"
        "addc.u32 %11, %23, 0;\n\t"
        : "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(t[8]), "=r"(t[9]), "=r"(t[10]), "=r"(t[11]),
          "=r"(t[12]), "=r"(t[13]), "=r"(t[14]), "=r"(t[15])
        : "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]), "r"(hi[0]), "r"(hi[1]), "r"(hi[2]), "r"(hi[3]),
          "r"(hi[4]), "r"(hi[5]), "r"(hi[6]), "r"(hi[7]), "r"(mid[0]), "r"(mid[1]), "r"(mid[2]), "r"(mid[3]),
          "r"(mid[4]), "r"(mid[5]), "r"(mid[6]), "r"(mid[7]), "r"(mid[8]));
    return fe_reduce512(t);
}

// r = a·b mod p (as a value below 2^256)
__device__ __forceinline__ fe fe_mul(const fe& a, const fe& b) { return fe_mul_schoolbook(a, b); }

// r = a·b mod p in the form a kernel picks at compile time: Karatsuba when K.  Both forms
// return the same words for the same inputs.
template <bool K>
__device__ __forceinline__ fe fe_mul_as(const fe& a, const fe& b) {
    if constexpr (K) return fe_mul_karatsuba(a, b);
    else return fe_mul_schoolbook(a, b);
}

// r = a^2 mod p: the 28 cross products a_i·a_j (i < j) in per-row carry chains (row i
// adds a_i·a_(i+1..7) into t[2i+1 .. i+8]; the row's partial sum stays below 2^(32(i+9)),
// so word i+8 absorbs its carry), then doubled with funnel shifts, plus the 8 diagonal
// squares in one chain: 72 multiply-adds before the fold instead of 128.
__device__ __forceinline__ fe fe_sq(const fe& a) {
    u32 t[16];
#pragma unroll
    for (int i = 0; i < 16; i++) t[i] = 0;
    asm("mad.lo.cc.u32 %0, %7, %8, %0;\n\t"
        "madc.hi.cc.u32 %1, %7, %8, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
        "madc.lo.cc.u32 %4, %7, %10, %4;\n\t"
        "madc.hi.cc.u32 %5, %7, %10, %5;\n\t"
        "addc.u32 %6, %6, 0;\n\t"
        : "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
        : "r"(a.v[0]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %8, %9, %0;\n\t"
        "madc.hi.cc.u32 %1, %8, %9, %1;\n\t"
        "madc.lo.cc.u32 %2, %8, %10, %2;\n\t"
        "madc.hi.cc.u32 %3, %8, %10, %3;\n\t"
        "madc.lo.cc.u32 %4, %8, %11, %4;\n\t"
        "madc.hi.cc.u32 %5, %8, %11, %5;\n\t"
        "madc.lo.cc.u32 %6, %8, %12, %6;\n\t"
        "madc.hi.u32 %7, %8, %12, %7;\n\t"
        : "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %7, %8, %0;\n\t"
        "madc.hi.cc.u32 %1, %7, %8, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
        "madc.lo.cc.u32 %4, %7, %10, %4;\n\t"
        "madc.hi.cc.u32 %5, %7, %10, %5;\n\t"
        "addc.u32 %6, %6, 0;\n\t"
        : "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9])
        : "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %6, %7, %0;\n\t"
        "madc.hi.cc.u32 %1, %6, %7, %1;\n\t"
        "madc.lo.cc.u32 %2, %6, %8, %2;\n\t"
        "madc.hi.cc.u32 %3, %6, %8, %3;\n\t"
        "madc.lo.cc.u32 %4, %6, %9, %4;\n\t"
        "madc.hi.u32 %5, %6, %9, %5;\n\t"
        : "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9])
        : "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %5, %6, %0;\n\t"
        "madc.hi.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.cc.u32 %3, %5, %7, %3;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        : "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10])
        : "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %6, %7, %0;\n\t"
        "madc.hi.cc.u32 %1, %6, %7, %1;\n\t"
        "madc.lo.cc.u32 %2, %6, %8, %2;\n\t"
        "madc.hi.cc.u32 %3, %6, %8, %3;\n\t"
        "madc.lo.cc.u32 %4, %6, %9, %4;\n\t"
        "madc.hi.u32 %5, %6, %9, %5;\n\t"
        : "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10])
        : "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %5, %6, %0;\n\t"
        "madc.hi.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.cc.u32 %3, %5, %7, %3;\n\t"
        "addc.u32 %4, %4, 0;\n\t"
        : "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11])
        : "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
        "madc.hi.cc.u32 %1, %4, %5, %1;\n\t"
        "madc.lo.cc.u32 %2, %4, %6, %2;\n\t"
        "madc.hi.u32 %3, %4, %6, %3;\n\t"
        : "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11])
        : "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;\n\t"
        : "+r"(t[10]), "+r"(t[11]), "+r"(t[12])
        : "r"(a.v[4]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
        "madc.hi.cc.u32 %1, %4, %5, %1;\n\t"
        "madc.lo.cc.u32 %2, %4, %6, %2;\n\t"
        "madc.hi.u32 %3, %4, %6, %3;\n\t"
        : "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12])
        : "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;\n\t"
        : "+r"(t[11]), "+r"(t[12]), "+r"(t[13])
        : "r"(a.v[5]), "r"(a.v[6]));
    asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\t"
        "madc.hi.u32 %1, %2, %3, %1;\n\t"
        : "+r"(t[12]), "+r"(t[13])
        : "r"(a.v[5]), "r"(a.v[7]));
    asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\t"
        "madc.hi.u32 %1, %2, %3, %1;\n\t"
        : "+r"(t[13]), "+r"(t[14])
        : "r"(a.v[6]), "r"(a.v[7]));

    // t = 2·t (the cross sum is below 2^511)
#pragma unroll
    for (int k = 15; k > 0; k--) t[k] = __funnelshift_l(t[k - 1], t[k], 1);
    t[0] = 0;
    asm("mad.lo.cc.u32 %0, %16, %16, %0;\n\t"
        "madc.hi.cc.u32 %1, %16, %16, %1;\n\t"
        "madc.lo.cc.u32 %2, %17, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %17, %17, %3;\n\t"
        "madc.lo.cc.u32 %4, %18, %18, %4;\n\t"
        "madc.hi.cc.u32 %5, %18, %18, %5;\n\t"
        "madc.lo.cc.u32 %6, %19, %19, %6;\n\t"
        "madc.hi.cc.u32 %7, %19, %19, %7;\n\t"
        "madc.lo.cc.u32 %8, %20, %20, %8;\n\t"
        "madc.hi.cc.u32 %9, %20, %20, %9;\n\t"
        "madc.lo.cc.u32 %10, %21, %21, %10;\n\t"
        "madc.hi.cc.u32 %11, %21, %21, %11;\n\t"
        "madc.lo.cc.u32 %12, %22, %22, %12;\n\t"
        "madc.hi.cc.u32 %13, %22, %22, %13;\n\t"
        "madc.lo.cc.u32 %14, %23, %23, %14;\n\t"
        "madc.hi.u32 %15, %23, %23, %15;\n\t"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
          "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12]), "+r"(t[13]), "+r"(t[14]), "+r"(t[15])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]), "r"(a.v[7]));
    return fe_reduce512(t);
}

// Canonical value (mod p) as 8 words
__device__ __forceinline__ void fe_to_words(const fe& a, u32 out[8]) {
    // fold bit 255: x = lo255 + 19·bit255  (< 2^255 + 19)
    u32 w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = a.v[i];
    u32 hb = w[7] >> 31;
    w[7] &= 0x7fffffffu;
    u64 c = 19ull * hb;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        c += w[i];
        w[i] = (u32)c;
        c >>= 32;
    }
    // subtract p if x >= p: compute x + 19 and test bit 255
    u32 t[8];
    c = 19;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        c += w[i];
        t[i] = (u32)c;
        c >>= 32;
    }
    u32 ge = t[7] >> 31;
    t[7] &= 0x7fffffffu;
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = ge ? t[i] : w[i];
}

__device__ __forceinline__ fe fe_from_words(const u32 w[8]) {
    fe r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = w[i];
    return r;
}

}  // namespace mk32
