// edwards25519 point arithmetic over the radix-2^32 field (fe32.cuh).
//
// Points are extended (X:Y:Z:T), x = X/Z, y = Y/Z, xy = T/Z.  Table points are
// affine "Niels" triples (y+x, y-x, 2d·x·y) stored canonical as 8 LE words each.
// The mixed addition is the a = -1 complete formula (Hisil-Wong-Carter-Dawson 2008,
// also RFC 8032 5.1.4 with Z2 = 1): 7 multiplications, or 3 when only y = Y/Z of the
// sum is wanted (then y = (B+A)/(2Z-C) and x = (B-A)/(2Z+C)).
#pragma once
#include "fe32.cuh"

namespace mk32 {

struct ge {
    fe X, Y, Z, T;
};

struct niels {
    fe ypx, ymx, t2d;
};

__device__ __forceinline__ void fe_cswap(fe& a, fe& b, bool swap) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        u32 x = a.v[i], y = b.v[i];
        a.v[i] = swap ? y : x;
        b.v[i] = swap ? x : y;
    }
}

// P + Q for a table point Q given with its digit sign: a negative digit uses -Q,
// which swaps y+x / y-x and flips the sign of the 2dxy term (so F and G trade places).
// K: the field multiplies in Karatsuba form (same results).
template <bool K = false>
__device__ __forceinline__ ge ge_add_niels(const ge& p, niels q, bool neg) {
    fe_cswap(q.ypx, q.ymx, neg);
    fe a = fe_mul_as<K>(fe_sub(p.Y, p.X), q.ymx);
    fe b = fe_mul_as<K>(fe_add(p.Y, p.X), q.ypx);
    fe c = fe_mul_as<K>(p.T, q.t2d);
    fe d = fe_add(p.Z, p.Z);
    fe e = fe_sub(b, a), h = fe_add(b, a);
    fe f = fe_sub(d, c), g = fe_add(d, c);
    fe_cswap(f, g, neg);
    ge r;
    r.X = fe_mul_as<K>(e, f);
    r.Y = fe_mul_as<K>(g, h);
    r.Z = fe_mul_as<K>(f, g);
    r.T = fe_mul_as<K>(e, h);
    return r;
}

// Last addition (digit >= 0): the sum's y as a fraction yn/yd and, optionally, x as xn/xd.
template <bool K = false>
__device__ __forceinline__ void ge_add_niels_frac(const ge& p, const niels& q, fe& yn, fe& yd, fe* xn, fe* xd) {
    fe a = fe_mul_as<K>(fe_sub(p.Y, p.X), q.ymx);
    fe b = fe_mul_as<K>(fe_add(p.Y, p.X), q.ypx);
    fe c = fe_mul_as<K>(p.T, q.t2d);
    fe d = fe_add(p.Z, p.Z);
    yn = fe_add(b, a);
    yd = fe_sub(d, c);
    if (xn) {
        *xn = fe_sub(b, a);
        *xd = fe_add(d, c);
    }
}

// General addition P + Q of two extended points (9 multiplications; used for table building).
__device__ __forceinline__ ge ge_add(const ge& p, const ge& q, const fe& d2) {
    fe a = fe_mul(fe_sub(p.Y, p.X), fe_sub(q.Y, q.X));
    fe b = fe_mul(fe_add(p.Y, p.X), fe_add(q.Y, q.X));
    fe c = fe_mul(fe_mul(p.T, d2), q.T);
    fe zz = fe_mul(p.Z, q.Z);
    fe d = fe_add(zz, zz);
    fe e = fe_sub(b, a), h = fe_add(b, a);
    fe f = fe_sub(d, c), g = fe_add(d, c);
    ge r;
    r.X = fe_mul(e, f);
    r.Y = fe_mul(g, h);
    r.Z = fe_mul(f, g);
    r.T = fe_mul(e, h);
    return r;
}

__device__ __forceinline__ ge ge_identity() {
    ge r;
    r.X = fe_zero();
    r.Y = fe_small(1);
    r.Z = fe_small(1);
    r.T = fe_zero();
    return r;
}

// x^(p-2) by the standard addition chain for 2^255-21 (254 squarings, 11 multiplications)
__device__ __forceinline__ fe fe_pow2k(fe a, int k) {
#pragma unroll 1
    for (int i = 0; i < k; i++) a = fe_sq(a);
    return a;
}

__device__ __noinline__ fe fe_invert(const fe z) {
    fe z2 = fe_sq(z);                               // 2
    fe z9 = fe_mul(fe_sq(fe_sq(z2)), z);            // 9
    fe z11 = fe_mul(z9, z2);                        // 11
    fe z_5_0 = fe_mul(fe_sq(z11), z9);              // 2^5 - 1
    fe z_10_0 = fe_mul(fe_pow2k(z_5_0, 5), z_5_0);  // 2^10 - 1
    fe z_20_0 = fe_mul(fe_pow2k(z_10_0, 10), z_10_0);
    fe z_40_0 = fe_mul(fe_pow2k(z_20_0, 20), z_20_0);
    fe z_50_0 = fe_mul(fe_pow2k(z_40_0, 10), z_10_0);
    fe z_100_0 = fe_mul(fe_pow2k(z_50_0, 50), z_50_0);
    fe z_200_0 = fe_mul(fe_pow2k(z_100_0, 100), z_100_0);
    fe z_250_0 = fe_mul(fe_pow2k(z_200_0, 50), z_50_0);
    return fe_mul(fe_pow2k(z_250_0, 5), z11);       // 2^255 - 32 + 11 = p - 2
}

}  // namespace mk32
