// Seed expansion and hashing for the candidate-key path:
//   ChaCha20 block (RFC 8439; 64-bit block counter in words 12-13, stream 0) — one
//   block gives two 32-byte seeds (even index: first half, odd: second half),
//   the layout of src/service/gpu/kernel.cu:133-176 and src/service/gpu.rs:1344-1351;
//   SHA-512 of a single 32-byte message and the RFC 8032 clamp (kernel.cu:228-303).
// All 64-bit arithmetic; the compiler lowers rotates to funnel shifts.
#pragma once
#include <stdint.h>

namespace mkh {

typedef uint32_t u32;
typedef uint64_t u64;

#define MKH_ROTL32(x, n) (((x) << (n)) | ((x) >> (32 - (n))))
#define MKH_QR(a, b, c, d)                       \
    a += b; d ^= a; d = MKH_ROTL32(d, 16);       \
    c += d; b ^= c; b = MKH_ROTL32(b, 12);       \
    a += b; d ^= a; d = MKH_ROTL32(d, 8);        \
    c += d; b ^= c; b = MKH_ROTL32(b, 7);

// 64-byte keystream block `counter` for a 32-byte key given as 8 LE words
__device__ __forceinline__ void chacha20_block(const u32 key[8], u64 counter, u32 out[16]) {
    u32 x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                 key[4],      key[5],      key[6],      key[7],      (u32)counter, (u32)(counter >> 32), 0u, 0u};
#pragma unroll 1
    for (int r = 0; r < 10; r++) {
        MKH_QR(x[0], x[4], x[8], x[12]);
        MKH_QR(x[1], x[5], x[9], x[13]);
        MKH_QR(x[2], x[6], x[10], x[14]);
        MKH_QR(x[3], x[7], x[11], x[15]);
        MKH_QR(x[0], x[5], x[10], x[15]);
        MKH_QR(x[1], x[6], x[11], x[12]);
        MKH_QR(x[2], x[7], x[8], x[13]);
        MKH_QR(x[3], x[4], x[9], x[14]);
    }
    out[0] = x[0] + 0x61707865u;
    out[1] = x[1] + 0x3320646eu;
    out[2] = x[2] + 0x79622d32u;
    out[3] = x[3] + 0x6b206574u;
#pragma unroll
    for (int i = 0; i < 8; i++) out[4 + i] = x[4 + i] + key[i];
    out[12] = x[12] + (u32)counter;
    out[13] = x[13] + (u32)(counter >> 32);
    out[14] = x[14];
    out[15] = x[15];
}

__device__ __forceinline__ u32 bswap32(u32 x) { return __byte_perm(x, 0, 0x0123); }
__device__ __forceinline__ u64 rotr64(u64 x, int n) { return (x >> n) | (x << (64 - n)); }

__constant__ u64 SHA512_K[80] = {
    0x428a2f98d728ae22ull, 0x7137449123ef65cdull, 0xb5c0fbcfec4d3b2full, 0xe9b5dba58189dbbcull,
    0x3956c25bf348b538ull, 0x59f111f1b605d019ull, 0x923f82a4af194f9bull, 0xab1c5ed5da6d8118ull,
    0xd807aa98a3030242ull, 0x12835b0145706fbeull, 0x243185be4ee4b28cull, 0x550c7dc3d5ffb4e2ull,
    0x72be5d74f27b896full, 0x80deb1fe3b1696b1ull, 0x9bdc06a725c71235ull, 0xc19bf174cf692694ull,
    0xe49b69c19ef14ad2ull, 0xefbe4786384f25e3ull, 0x0fc19dc68b8cd5b5ull, 0x240ca1cc77ac9c65ull,
    0x2de92c6f592b0275ull, 0x4a7484aa6ea6e483ull, 0x5cb0a9dcbd41fbd4ull, 0x76f988da831153b5ull,
    0x983e5152ee66dfabull, 0xa831c66d2db43210ull, 0xb00327c898fb213full, 0xbf597fc7beef0ee4ull,
    0xc6e00bf33da88fc2ull, 0xd5a79147930aa725ull, 0x06ca6351e003826full, 0x142929670a0e6e70ull,
    0x27b70a8546d22ffcull, 0x2e1b21385c26c926ull, 0x4d2c6dfc5ac42aedull, 0x53380d139d95b3dfull,
    0x650a73548baf63deull, 0x766a0abb3c77b2a8ull, 0x81c2c92e47edaee6ull, 0x92722c851482353bull,
    0xa2bfe8a14cf10364ull, 0xa81a664bbc423001ull, 0xc24b8b70d0f89791ull, 0xc76c51a30654be30ull,
    0xd192e819d6ef5218ull, 0xd69906245565a910ull, 0xf40e35855771202aull, 0x106aa07032bbd1b8ull,
    0x19a4c116b8d2d0c8ull, 0x1e376c085141ab53ull, 0x2748774cdf8eeb99ull, 0x34b0bcb5e19b48a8ull,
    0x391c0cb3c5c95a63ull, 0x4ed8aa4ae3418acbull, 0x5b9cca4f7763e373ull, 0x682e6ff3d6b2b8a3ull,
    0x748f82ee5defb2fcull, 0x78a5636f43172f60ull, 0x84c87814a1f0ab72ull, 0x8cc702081a6439ecull,
    0x90befffa23631e28ull, 0xa4506cebde82bde9ull, 0xbef9a3f7b2c67915ull, 0xc67178f2e372532bull,
    0xca273eceea26619cull, 0xd186b8c721c0c207ull, 0xeada7dd6cde0eb1eull, 0xf57d4f7fee6ed178ull,
    0x06f067aa72176fbaull, 0x0a637dc5a2c898a6ull, 0x113f9804bef90daeull, 0x1b710b35131c471bull,
    0x28db77f523047d84ull, 0x32caab7b40c72493ull, 0x3c9ebe0a15c9bebcull, 0x431d67c49c100d4cull,
    0x4cc5d4becb3e42b6ull, 0x597f299cfc657e2aull, 0x5fcb6fab3ad6faecull, 0x6c44198c4a475817ull,
};

#define MKH_IV0 0x6a09e667f3bcc908ull
#define MKH_IV1 0xbb67ae8584caa73bull
#define MKH_IV2 0x3c6ef372fe94f82bull
#define MKH_IV3 0xa54ff53a5f1d36f1ull
#define MKH_IV4 0x510e527fade682d1ull
#define MKH_IV5 0x9b05688c2b3e6c1full
#define MKH_IV6 0x1f83d9abfb41bd6bull
#define MKH_IV7 0x5be0cd19137e2179ull

__device__ __forceinline__ void sha512_round(u64& a, u64& b, u64& c, u64& d, u64& e, u64& f, u64& g, u64& h,
                                             u64 w, u64 k) {
    u64 s1 = rotr64(e, 14) ^ rotr64(e, 18) ^ rotr64(e, 41);
    u64 ch = (e & f) ^ (~e & g);
    u64 t1 = h + s1 + ch + k + w;
    u64 s0 = rotr64(a, 28) ^ rotr64(a, 34) ^ rotr64(a, 39);
    u64 mj = (a & b) ^ (a & c) ^ (b & c);
    h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + s0 + mj;
}

// The clamped scalar from the final state words a..d: digest words h0..h3 = state + IV,
// read little-endian (the digest bytes are big-endian per word), then the RFC 8032 clamp
// (clear bits 0-2 and 255, set bit 254).
__device__ __forceinline__ void digest_scalar(u64 a, u64 b, u64 c, u64 d, u64 s_out[4]) {
    u64 hh[4] = {a + MKH_IV0, b + MKH_IV1, c + MKH_IV2, d + MKH_IV3};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        u32 hi = (u32)(hh[i] >> 32), lo = (u32)hh[i];
        s_out[i] = (u64)bswap32(lo) << 32 | bswap32(hi);
    }
    s_out[0] &= ~7ull;
    s_out[3] &= 0x7fffffffffffffffull;
    s_out[3] |= 0x4000000000000000ull;
}

// Rounds FROM..79 of the single padded block whose message words 0..3 are `w4`
// (words 4..15 are the fixed padding of a 32-byte message), from state `st` at the
// start of round FROM; writes the clamped scalar as 4 little-endian u64 words
// (s = h0..h3 + IV read little-endian).  Rounds 16..79 run as a rolled loop of
// 16-round blocks so the code stays small; schedule indices stay static inside a block.
template <int FROM>
__device__ __forceinline__ void sha512_scalar_from(const u64 st[8], const u64 w4[4], u64 s_out[4]) {
    u64 w[16];
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = w4[i];
    w[4] = 0x8000000000000000ull;
#pragma unroll
    for (int i = 5; i < 15; i++) w[i] = 0;
    w[15] = 256;
    u64 a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll
    for (int t = FROM; t < 16; t++) sha512_round(a, b, c, d, e, f, g, h, w[t], SHA512_K[t]);
#pragma unroll 1
    for (int blk = 16; blk < 80; blk += 16) {
#pragma unroll
        for (int i = 0; i < 16; i++) {
            u64 x15 = w[(i + 1) & 15], x2 = w[(i + 14) & 15];
            u64 s0 = rotr64(x15, 1) ^ rotr64(x15, 8) ^ (x15 >> 7);
            u64 s1 = rotr64(x2, 19) ^ rotr64(x2, 61) ^ (x2 >> 6);
            w[i] = w[i] + s0 + w[(i + 9) & 15] + s1;
            sha512_round(a, b, c, d, e, f, g, h, w[i], SHA512_K[blk + i]);
        }
    }
    digest_scalar(a, b, c, d, s_out);
}

// SHA-512 message words 0..3 (big-endian u64) of a seed given as 8 LE words
__device__ __forceinline__ void seed_words(const u32 sw[8], u64 w4[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) w4[i] = (u64)bswap32(sw[2 * i]) << 32 | bswap32(sw[2 * i + 1]);
}

// Clamped scalar of a seed given as 8 LE words (the ChaCha20 half-block)
__device__ __forceinline__ void seed_scalar(const u32 sw[8], u64 s_out[4]) {
    u64 w4[4];
    seed_words(sw, w4);
    u64 st[8] = {MKH_IV0, MKH_IV1, MKH_IV2, MKH_IV3, MKH_IV4, MKH_IV5, MKH_IV6, MKH_IV7};
    sha512_scalar_from<0>(st, w4, s_out);
}

// Low-security seeds (src/model/search.rs:45-50): bytes 0..23 of the base are shared,
// bytes 24..31 hold (LE tail of base) + index, so message words 0..2 and the first
// three rounds are the same for every index and are computed once per thread.
struct CounterMid {
    u64 st[8];   // state before round 3
    u64 w[3];    // message words 0..2
    u64 tail;    // LE u64 of base bytes 24..31
};

__device__ __forceinline__ CounterMid counter_mid(const u32 base[8]) {
    CounterMid m;
#pragma unroll
    for (int i = 0; i < 3; i++) m.w[i] = (u64)bswap32(base[2 * i]) << 32 | bswap32(base[2 * i + 1]);
    m.tail = (u64)base[7] << 32 | base[6];
    u64 a = MKH_IV0, b = MKH_IV1, c = MKH_IV2, d = MKH_IV3, e = MKH_IV4, f = MKH_IV5, g = MKH_IV6, h = MKH_IV7;
#pragma unroll
    for (int t = 0; t < 3; t++) sha512_round(a, b, c, d, e, f, g, h, m.w[t], SHA512_K[t]);
    m.st[0] = a; m.st[1] = b; m.st[2] = c; m.st[3] = d; m.st[4] = e; m.st[5] = f; m.st[6] = g; m.st[7] = h;
    return m;
}

// message words 0..3 of the counter seed of `index`
__device__ __forceinline__ void counter_words(const CounterMid& m, u64 index, u64 w4[4]) {
    u64 tail = m.tail + index;
    // seed bytes 24..31 = LE(tail); message word 3 reads them big-endian
    w4[0] = m.w[0];
    w4[1] = m.w[1];
    w4[2] = m.w[2];
    w4[3] = (u64)bswap32((u32)tail) << 32 | bswap32((u32)(tail >> 32));
}

__device__ __forceinline__ void counter_scalar(const CounterMid& m, u64 index, u64 s_out[4]) {
    u64 w4[4];
    counter_words(m, index, w4);
    sha512_scalar_from<3>(m.st, w4, s_out);
}

// SHA-512 of one padded 32-byte message advanced 8 rounds at a time with the same code for
// every step, so that a caller can interleave the steps with other work (the search kernel
// puts one step into each comb row).  The ring w[0..15] holds W[t0-16 .. t0-1] before the step
// of rounds t0..t0+7, t0 >= 16 (the first two steps take the message words, which start in
// the ring); each step writes W[t0..t0+7] into w[0..7] and swaps the halves.
struct ShaRun {
    u64 s[8];
    u64 w[16];
};

__device__ __forceinline__ void sha_run_start(ShaRun& r, const u64 w4[4]) {
    r.s[0] = MKH_IV0; r.s[1] = MKH_IV1; r.s[2] = MKH_IV2; r.s[3] = MKH_IV3;
    r.s[4] = MKH_IV4; r.s[5] = MKH_IV5; r.s[6] = MKH_IV6; r.s[7] = MKH_IV7;
#pragma unroll
    for (int i = 0; i < 4; i++) r.w[i] = w4[i];
    r.w[4] = 0x8000000000000000ull;
#pragma unroll
    for (int i = 5; i < 15; i++) r.w[i] = 0;
    r.w[15] = 256;
}

// rounds t0..t0+7 (t0 = 0, 8, ..., 72)
__device__ __forceinline__ void sha_run_step(ShaRun& r, u32 t0) {
    const bool sched = t0 >= 16;
    u64 a = r.s[0], b = r.s[1], c = r.s[2], d = r.s[3], e = r.s[4], f = r.s[5], g = r.s[6], h = r.s[7];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u64 x2 = i < 2 ? r.w[i + 14] : r.w[i - 2];   // W[t-2]
        const u64 x7 = i < 7 ? r.w[i + 9] : r.w[0];        // W[t-7]
        const u64 x15 = r.w[i + 1];                         // W[t-15]
        const u64 s0 = rotr64(x15, 1) ^ rotr64(x15, 8) ^ (x15 >> 7);
        const u64 s1 = rotr64(x2, 19) ^ rotr64(x2, 61) ^ (x2 >> 6);
        const u64 wt = sched ? r.w[i] + s0 + x7 + s1 : r.w[i];
        r.w[i] = wt;
        sha512_round(a, b, c, d, e, f, g, h, wt, SHA512_K[t0 + i]);
    }
    r.s[0] = a; r.s[1] = b; r.s[2] = c; r.s[3] = d; r.s[4] = e; r.s[5] = f; r.s[6] = g; r.s[7] = h;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u64 t = r.w[i];
        r.w[i] = r.w[i + 8];
        r.w[i + 8] = t;
    }
}

}  // namespace mkh
