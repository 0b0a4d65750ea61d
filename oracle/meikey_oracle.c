/*
 * meikey oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement, on the CPU, of the reference's candidate-key search
 * path (waxsd100/meikey).  It is the checker for the CUDA library: only the
 * tests, the smoke check and the benchmark's CPU-baseline leg may load it.
 * Nothing in the product links or calls this file.
 *
 * Every stage follows the reference's algorithm (citations are paths inside
 * the reference project):
 *   seed      ChaCha20 block with a 64-bit block counter and stream 0; index i
 *             takes half (i & 1) of block i >> 1
 *             (src/service/gpu/kernel.cu:133-176, src/service/gpu.rs:1344-1351);
 *             low-security seeds add the index to the last 8 bytes (LE)
 *             (src/model/search.rs:45-50, kernel.cu:179-189)
 *   scalar    clamp(SHA-512(seed)[0..32])  (kernel.cu:228-303, RFC 8032 5.1.5)
 *   point     s·B on edwards25519, compressed y with the x sign in bit 255
 *             (ed25519-dalek VerifyingKey, used by src/model/key.rs:98-101).
 *             The oracle uses its own 4-bit fixed-window table and 51-bit limbs;
 *             the public key depends only on the seed, not on the method.
 *   base64    tail of the OpenSSH blob: byte 32 then the key (kernel.cu:1707-1728,
 *             src/model/key.rs:43-52)
 *   match     contains / suffix / case folding and the sign-unknown candidate
 *             test (kernel.cu:1765-1835), the regex DFA walk (kernel.cu:1839-1875,
 *             src/model/pattern/dfa.rs:189-200)
 *   table     the reference's packed comb table, so that the reference kernel
 *             compiled for the CPU can be driven here (src/service/derive/comb.rs:285-392,
 *             src/service/gpu.rs:1416-1480)
 *
 * Parity of this oracle is pinned against the RFC 8032 section 7.1 vectors,
 * OpenSSL's Ed25519 (Python `cryptography`) and the reference kernel compiled
 * for the CPU (see tests/golden/make_golden.py).
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

typedef uint8_t u8;
typedef uint32_t u32;
typedef uint64_t u64;
typedef unsigned __int128 u128;

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* ChaCha20 (RFC 8439 block function, 64-bit counter in words 12-13)         */
/* ------------------------------------------------------------------------ */

static u32 rotl32(u32 x, int n) { return (x << n) | (x >> (32 - n)); }

#define QROUND(a, b, c, d)                 \
    a += b; d ^= a; d = rotl32(d, 16);     \
    c += d; b ^= c; b = rotl32(b, 12);     \
    a += b; d ^= a; d = rotl32(d, 8);      \
    c += d; b ^= c; b = rotl32(b, 7);

EXPORT void mko_chacha20_block(const u32 key[8], u64 counter, u32 out[16]) {
    u32 s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                 key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                 (u32)counter, (u32)(counter >> 32), 0u, 0u};
    u32 x[16];
    memcpy(x, s, sizeof x);
    for (int r = 0; r < 10; r++) {
        QROUND(x[0], x[4], x[8], x[12]);
        QROUND(x[1], x[5], x[9], x[13]);
        QROUND(x[2], x[6], x[10], x[14]);
        QROUND(x[3], x[7], x[11], x[15]);
        QROUND(x[0], x[5], x[10], x[15]);
        QROUND(x[1], x[6], x[11], x[12]);
        QROUND(x[2], x[7], x[8], x[13]);
        QROUND(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

static void key_words(const u8 key[32], u32 w[8]) {
    for (int i = 0; i < 8; i++)
        w[i] = (u32)key[4 * i] | (u32)key[4 * i + 1] << 8 | (u32)key[4 * i + 2] << 16 | (u32)key[4 * i + 3] << 24;
}

/* seed of index i from a 32-byte ChaCha20 key */
EXPORT void mko_chacha20_seed(const u8 key[32], u64 index, u8 seed[32]) {
    u32 kw[8], blk[16];
    key_words(key, kw);
    mko_chacha20_block(kw, index >> 1, blk);
    const u32* half = blk + ((index & 1) ? 8 : 0);
    for (int i = 0; i < 8; i++) {
        seed[4 * i] = (u8)half[i];
        seed[4 * i + 1] = (u8)(half[i] >> 8);
        seed[4 * i + 2] = (u8)(half[i] >> 16);
        seed[4 * i + 3] = (u8)(half[i] >> 24);
    }
}

/* low-security seed: base with index added to its last 8 bytes (LE, wrapping) */
EXPORT void mko_counter_seed(const u8 base[32], u64 index, u8 seed[32]) {
    memcpy(seed, base, 32);
    u64 tail = 0;
    for (int b = 7; b >= 0; b--) tail = tail << 8 | base[24 + b];
    tail += index;
    for (int b = 0; b < 8; b++) seed[24 + b] = (u8)(tail >> (8 * b));
}

/* ------------------------------------------------------------------------ */
/* SHA-512 (FIPS 180-4), any length                                           */
/* ------------------------------------------------------------------------ */

static const u64 K512[80] = {
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

static u64 rotr64(u64 x, int n) { return (x >> n) | (x << (64 - n)); }

static void sha512_compress(u64 h[8], const u8 blk[128]) {
    u64 w[80];
    for (int t = 0; t < 16; t++) {
        u64 v = 0;
        for (int b = 0; b < 8; b++) v = v << 8 | blk[8 * t + b];
        w[t] = v;
    }
    for (int t = 16; t < 80; t++) {
        u64 s0 = rotr64(w[t - 15], 1) ^ rotr64(w[t - 15], 8) ^ (w[t - 15] >> 7);
        u64 s1 = rotr64(w[t - 2], 19) ^ rotr64(w[t - 2], 61) ^ (w[t - 2] >> 6);
        w[t] = w[t - 16] + s0 + w[t - 7] + s1;
    }
    u64 a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int t = 0; t < 80; t++) {
        u64 S1 = rotr64(e, 14) ^ rotr64(e, 18) ^ rotr64(e, 41);
        u64 ch = (e & f) ^ (~e & g);
        u64 t1 = hh + S1 + ch + K512[t] + w[t];
        u64 S0 = rotr64(a, 28) ^ rotr64(a, 34) ^ rotr64(a, 39);
        u64 mj = (a & b) ^ (a & c) ^ (b & c);
        u64 t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

EXPORT void mko_sha512(const u8* msg, u64 len, u8 out[64]) {
    u64 h[8] = {0x6a09e667f3bcc908ull, 0xbb67ae8584caa73bull, 0x3c6ef372fe94f82bull, 0xa54ff53a5f1d36f1ull,
                0x510e527fade682d1ull, 0x9b05688c2b3e6c1full, 0x1f83d9abfb41bd6bull, 0x5be0cd19137e2179ull};
    u64 off = 0;
    while (len - off >= 128) {
        sha512_compress(h, msg + off);
        off += 128;
    }
    u8 tail[256];
    memset(tail, 0, sizeof tail);
    u64 rem = len - off;
    memcpy(tail, msg + off, rem);
    tail[rem] = 0x80;
    u64 total = rem + 1 + 16 <= 128 ? 128 : 256;
    u64 bits = len * 8;
    for (int b = 0; b < 8; b++) tail[total - 1 - b] = (u8)(bits >> (8 * b));
    sha512_compress(h, tail);
    if (total == 256) sha512_compress(h, tail + 128);
    for (int i = 0; i < 8; i++)
        for (int b = 0; b < 8; b++) out[8 * i + b] = (u8)(h[i] >> (56 - 8 * b));
}

/* clamp(SHA-512(seed)[0..32]) */
EXPORT void mko_secret_scalar(const u8 seed[32], u8 s[32]) {
    u8 hash[64];
    mko_sha512(seed, 32, hash);
    memcpy(s, hash, 32);
    s[0] &= 248;
    s[31] &= 127;
    s[31] |= 64;
}

/* ------------------------------------------------------------------------ */
/* GF(2^255 - 19), 5 limbs of 51 bits                                         */
/* ------------------------------------------------------------------------ */

typedef struct { u64 v[5]; } fe;
#define M51 ((1ull << 51) - 1)

static fe fe_zero(void) { fe r = {{0, 0, 0, 0, 0}}; return r; }
static fe fe_one(void) { fe r = {{1, 0, 0, 0, 0}}; return r; }
static fe fe_small(u64 x) { fe r = {{x, 0, 0, 0, 0}}; return r; }

static fe fe_carry(fe a) {
    for (int i = 0; i < 4; i++) { a.v[i + 1] += a.v[i] >> 51; a.v[i] &= M51; }
    a.v[0] += 19 * (a.v[4] >> 51); a.v[4] &= M51;
    a.v[1] += a.v[0] >> 51; a.v[0] &= M51;
    return a;
}
static fe fe_add(fe a, fe b) { fe r; for (int i = 0; i < 5; i++) r.v[i] = a.v[i] + b.v[i]; return fe_carry(r); }
/* a - b with 4p added (inputs carried, limbs < 2^52) */
static fe fe_sub(fe a, fe b) {
    fe r;
    r.v[0] = a.v[0] + 4 * (M51 - 18) - b.v[0];
    for (int i = 1; i < 5; i++) r.v[i] = a.v[i] + 4 * M51 - b.v[i];
    return fe_carry(r);
}
static fe fe_mul(fe a, fe b) {
    u128 t[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            u128 p = (u128)a.v[i] * b.v[j];
            if (i + j >= 5) t[i + j - 5] += p * 19; else t[i + j] += p;
        }
    fe r;
    u128 c = 0;
    for (int i = 0; i < 5; i++) { t[i] += c; r.v[i] = (u64)t[i] & M51; c = t[i] >> 51; }
    r.v[0] += (u64)c * 19;
    return fe_carry(r);
}
static fe fe_sq(fe a) { return fe_mul(a, a); }
static fe fe_neg(fe a) { return fe_sub(fe_zero(), a); }

/* canonical little-endian bytes */
static void fe_tobytes(fe a, u8 out[32]) {
    a = fe_carry(fe_carry(a));
    /* now a < 2^255 + small; subtract p if a >= p */
    u64 q = (a.v[0] + 19) >> 51;
    q = (a.v[1] + q) >> 51;
    q = (a.v[2] + q) >> 51;
    q = (a.v[3] + q) >> 51;
    q = (a.v[4] + q) >> 51;
    a.v[0] += 19 * q;
    for (int i = 0; i < 4; i++) { a.v[i + 1] += a.v[i] >> 51; a.v[i] &= M51; }
    a.v[4] &= M51;
    u64 w[4] = {a.v[0] | a.v[1] << 51, a.v[1] >> 13 | a.v[2] << 38, a.v[2] >> 26 | a.v[3] << 25,
                a.v[3] >> 39 | a.v[4] << 12};
    for (int i = 0; i < 4; i++)
        for (int b = 0; b < 8; b++) out[8 * i + b] = (u8)(w[i] >> (8 * b));
}
static fe fe_frombytes(const u8 in[32]) { /* ignores bit 255 */
    u64 w[4];
    for (int i = 0; i < 4; i++) {
        w[i] = 0;
        for (int b = 7; b >= 0; b--) w[i] = w[i] << 8 | in[8 * i + b];
    }
    fe r;
    r.v[0] = w[0] & M51;
    r.v[1] = (w[0] >> 51 | w[1] << 13) & M51;
    r.v[2] = (w[1] >> 38 | w[2] << 26) & M51;
    r.v[3] = (w[2] >> 25 | w[3] << 39) & M51;
    r.v[4] = (w[3] >> 12) & M51;
    return r;
}
/* a^e for e given as 32 little-endian bytes (square-and-multiply from the top bit) */
static fe fe_pow(fe a, const u8 e[32]) {
    fe r = fe_one();
    for (int bit = 255; bit >= 0; bit--) {
        r = fe_sq(r);
        if ((e[bit >> 3] >> (bit & 7)) & 1) r = fe_mul(r, a);
    }
    return r;
}
/* p - 2 and (p + 3) / 8, (p - 1) / 4 as LE bytes */
static void exp_p_minus(u8 e[32], int sub) { /* e = p - sub = (2^255 - 1) - (18 + sub), sub small */
    memset(e, 0xff, 32);
    e[31] = 0x7f;
    e[0] = (u8)(0xff - 18 - sub);
}
static fe fe_invert(fe a) { u8 e[32]; exp_p_minus(e, 2); return fe_pow(a, e); }
static int fe_iszero(fe a) { u8 b[32]; fe_tobytes(a, b); u8 acc = 0; for (int i = 0; i < 32; i++) acc |= b[i]; return acc == 0; }
static int fe_eq(fe a, fe b) { return fe_iszero(fe_sub(a, b)); }
static int fe_isodd(fe a) { u8 b[32]; fe_tobytes(a, b); return b[0] & 1; }

/* ------------------------------------------------------------------------ */
/* edwards25519: -x^2 + y^2 = 1 + d x^2 y^2                                   */
/* ------------------------------------------------------------------------ */

typedef struct { fe x, y, z, t; } ge;         /* extended coordinates */
typedef struct { fe ypx, ymx, t2d; } ge_niels; /* affine (y+x, y-x, 2dxy) */

static fe D, D2, SQRTM1;
static ge BASE;
static int inited;
/* WIN[i][j] = (j+1) * 16^i * B, i < 64, j < 15 */
static ge_niels WIN[64][15];

static ge ge_identity(void) { ge p = {fe_zero(), fe_one(), fe_one(), fe_zero()}; return p; }

/* unified addition (RFC 8032 5.1.4, a = -1) */
static ge ge_add(ge p, ge q) {
    fe a = fe_mul(fe_sub(p.y, p.x), fe_sub(q.y, q.x));
    fe b = fe_mul(fe_add(p.y, p.x), fe_add(q.y, q.x));
    fe c = fe_mul(fe_mul(p.t, D2), q.t);
    fe dd = fe_mul(fe_add(p.z, p.z), q.z);
    fe e = fe_sub(b, a), f = fe_sub(dd, c), g = fe_add(dd, c), h = fe_add(b, a);
    ge r = {fe_mul(e, f), fe_mul(g, h), fe_mul(f, g), fe_mul(e, h)};
    return r;
}
static ge ge_add_niels(ge p, ge_niels q) {
    fe a = fe_mul(fe_sub(p.y, p.x), q.ymx);
    fe b = fe_mul(fe_add(p.y, p.x), q.ypx);
    fe c = fe_mul(p.t, q.t2d);
    fe dd = fe_add(p.z, p.z);
    fe e = fe_sub(b, a), f = fe_sub(dd, c), g = fe_add(dd, c), h = fe_add(b, a);
    ge r = {fe_mul(e, f), fe_mul(g, h), fe_mul(f, g), fe_mul(e, h)};
    return r;
}
static ge ge_double(ge p) { return ge_add(p, p); }
static void ge_affine(ge p, fe* x, fe* y) {
    fe zi = fe_invert(p.z);
    *x = fe_mul(p.x, zi);
    *y = fe_mul(p.y, zi);
}
static ge_niels niels_from_affine(fe x, fe y) {
    ge_niels n = {fe_add(y, x), fe_sub(y, x), fe_mul(fe_mul(x, y), D2)};
    return n;
}
static void ge_compress(ge p, u8 out[32]) {
    fe x, y;
    ge_affine(p, &x, &y);
    fe_tobytes(y, out);
    out[31] |= (u8)(fe_isodd(x) << 7);
}

static void oracle_init(void) {
    if (inited) return;
    /* d = -121665 / 121666 */
    D = fe_mul(fe_neg(fe_small(121665)), fe_invert(fe_small(121666)));
    D2 = fe_add(D, D);
    /* sqrt(-1) = 2^((p-1)/4) */
    u8 e[32];
    memset(e, 0xff, 32);
    e[31] = 0x1f;
    e[0] = 0xfb; /* (p - 1) / 4 = 2^253 - 5 */
    SQRTM1 = fe_pow(fe_small(2), e);
    /* base point: y = 4/5, x even (RFC 8032 5.1) */
    fe by = fe_mul(fe_small(4), fe_invert(fe_small(5)));
    fe yy = fe_sq(by);
    fe u = fe_sub(yy, fe_one());
    fe v = fe_add(fe_mul(D, yy), fe_one());
    /* x = (u/v)^((p+3)/8) candidate via u v^3 (u v^7)^((p-5)/8) */
    fe v3 = fe_mul(fe_sq(v), v);
    fe v7 = fe_mul(fe_sq(v3), v);
    u8 e2[32];
    memset(e2, 0xff, 32);
    e2[31] = 0x0f;
    e2[0] = 0xfd; /* (p - 5) / 8 = 2^252 - 3 */
    fe x = fe_mul(fe_mul(u, v3), fe_pow(fe_mul(u, v7), e2));
    if (!fe_eq(fe_mul(v, fe_sq(x)), u)) x = fe_mul(x, SQRTM1);
    if (fe_isodd(x)) x = fe_neg(x);
    BASE.x = x; BASE.y = by; BASE.z = fe_one(); BASE.t = fe_mul(x, by);
    /* window table */
    ge row = BASE;
    for (int i = 0; i < 64; i++) {
        ge acc = row;
        for (int j = 0; j < 15; j++) {
            fe ax, ay;
            ge_affine(acc, &ax, &ay);
            WIN[i][j] = niels_from_affine(ax, ay);
            acc = ge_add(acc, row);
        }
        for (int k = 0; k < 4; k++) row = ge_double(row);
    }
    inited = 1;
}

EXPORT void mko_init(void) { oracle_init(); }

/* s·B for a 256-bit little-endian scalar (any value; no reduction mod L needed) */
static ge base_mul(const u8 s[32]) {
    ge acc = ge_identity();
    for (int i = 0; i < 64; i++) {
        int d = (s[i >> 1] >> ((i & 1) * 4)) & 15;
        if (d) acc = ge_add_niels(acc, WIN[i][d - 1]);
    }
    return acc;
}

EXPORT void mko_base_mul(const u8 s[32], u8 pk[32]) {
    oracle_init();
    ge_compress(base_mul(s), pk);
}

/* affine coordinates (canonical LE bytes) of s·B for a 256-bit little-endian scalar */
EXPORT void mko_point_affine(const u8 s[32], u8 x_out[32], u8 y_out[32]) {
    oracle_init();
    fe x, y;
    ge_affine(base_mul(s), &x, &y);
    fe_tobytes(x, x_out);
    fe_tobytes(y, y_out);
}

EXPORT void mko_pubkey_from_seed(const u8 seed[32], u8 pk[32]) {
    u8 s[32];
    oracle_init();
    mko_secret_scalar(seed, s);
    ge_compress(base_mul(s), pk);
}

/* src 0: ChaCha20 seeds, 1: counter seeds */
EXPORT void mko_seed(const u8 key[32], u32 src, u64 index, u8 seed[32]) {
    if (src == 1) mko_counter_seed(key, index, seed);
    else mko_chacha20_seed(key, index, seed);
}

/* incremental path: compressed (s0 + k)·B = s0·B + k·B for k = first .. first+n-1.
 * s0 is a 256-bit little-endian scalar below 2^255 (the caller's contract), so s0 + k
 * never wraps.  There is no reference kernel for this path: the definition is the
 * point sequence P_k = P_0 + k·B of the incremental (low-security) configuration. */
static void incremental_pubkey(const u8 s0[32], u64 k, u8 pk[32]) {
    u8 s[32];
    u64 c = 0;
    for (int b = 0; b < 32; b++) {
        u64 add = b < 8 ? (k >> (8 * b)) & 0xff : 0;
        c += (u64)s0[b] + add;
        s[b] = (u8)c;
        c >>= 8;
    }
    ge_compress(base_mul(s), pk);
}

EXPORT void mko_incremental(const u8 s0[32], u64 first, u64 n, u8* out) {
    oracle_init();
    for (u64 i = 0; i < n; i++) incremental_pubkey(s0, first + i, out + 32 * i);
}

/* public key of one index of source src (0 ChaCha20, 1 counter: Ed25519 key of the seed;
 * 2 incremental: (key + index)·B with key the start scalar) */
static void index_pubkey(const u8 key[32], u32 src, u64 index, u8 pk[32]) {
    if (src == 2) {
        incremental_pubkey(key, index, pk);
        return;
    }
    u8 seed[32];
    mko_seed(key, src, index, seed);
    mko_pubkey_from_seed(seed, pk);
}

/* public keys of indices first .. first+n-1 (full sign bit) */
EXPORT void mko_derive(const u8 key[32], u32 src, u64 first, u64 n, u8* out) {
    oracle_init();
    for (u64 i = 0; i < n; i++) index_pubkey(key, src, first + i, out + 32 * i);
}

/* ------------------------------------------------------------------------ */
/* base64 tail and matching                                                    */
/* ------------------------------------------------------------------------ */

static const char B64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
#define TAIL 44
#define SIGN_POS 42

/* 6-bit values of the 44-character tail (blob bytes 18..51: 0x20 then the key) */
static void tail_values(const u8 pk[32], u8 v[TAIL]) {
    for (int g = 0; g < 11; g++) {
        u32 b0 = g == 0 ? 32u : pk[3 * g - 1];
        u32 n = b0 << 16 | (u32)pk[3 * g] << 8 | pk[3 * g + 1];
        for (int k = 0; k < 4; k++) v[4 * g + k] = (u8)((n >> (18 - 6 * k)) & 63);
    }
}

/* full 68-character OpenSSH base64 of the key blob (no NUL) */
EXPORT void mko_public_b64(const u8 pk[32], char out[68]) {
    static const char HEAD[] = "AAAAC3NzaC1lZDI1NTE5AAAA";
    memcpy(out, HEAD, 24);
    u8 v[TAIL];
    tail_values(pk, v);
    for (int i = 0; i < TAIL; i++) out[24 + i] = B64[v[i]];
}

static int b64_value(u8 c) {
    for (int i = 0; i < 64; i++) if ((u8)B64[i] == c) return i;
    return 64;
}

/* does value v match needle character c (c lowercase when fold) */
static int value_matches(u8 v, u8 c, int fold) {
    u8 ch = (u8)B64[v];
    if (ch == c) return 1;
    if (fold && ch >= 'A' && ch <= 'Z' && (u8)(ch + 32) == c) return 1;
    return 0;
}

/*
 * Contains / suffix test over tail positions 1..43.
 * sign_unknown: pk has its sign bit cleared and the character at position 42
 * also matches with value bit 1 set (either sign), as kernel.cu:1804-1835.
 * mode 0 contains, 1 suffix.
 */
static int match_text(const u8 pk[32], const u8* needle, u32 len, int fold, u32 mode, int sign_unknown) {
    if (len == 0 || len > TAIL - 1) return 0;
    u8 v[TAIL];
    tail_values(pk, v);
    u32 lo = mode == 1 ? TAIL - len : 1;
    for (u32 s = lo; s + len <= TAIL; s++) {
        u32 k = 0;
        for (; k < len; k++) {
            u32 pos = s + k;
            int ok = value_matches(v[pos], needle[k], fold);
            if (!ok && sign_unknown && pos == SIGN_POS) ok = value_matches(v[pos] | 2, needle[k], fold);
            if (!ok) break;
        }
        if (k == len) return 1;
    }
    return 0;
}

/* DFA table as in src/model/pattern/dfa.rs:189-200: states x 65 u16 LE, ACCEPT 0, START 1 */
static u32 dfa_next(const u8* t, u32 s, u32 i) { u32 at = (s * 65u + i) * 2u; return (u32)t[at] | (u32)t[at + 1] << 8; }
static int dfa_done(const u8* t, u32 s) { return s == 0 || dfa_next(t, s, 64) != 0; }

static int match_dfa(const u8 pk[32], const u8* table, int sign_unknown) {
    u8 v[TAIL];
    tail_values(pk, v);
    u32 s = 1, alt = 1;
    for (int pos = 1; pos < TAIL; pos++) {
        if (pos == SIGN_POS) alt = dfa_next(table, s, sign_unknown ? (v[pos] | 2u) : v[pos]);
        else if (pos > SIGN_POS) alt = dfa_next(table, alt, v[pos]);
        s = dfa_next(table, s, v[pos]);
    }
    return dfa_done(table, s) || dfa_done(table, alt);
}

/* mode 0 contains, 1 suffix, 2 regex (needle = DFA table, len = states) */
EXPORT int mko_match(const u8 pk[32], const u8* needle, u32 len, u32 fold, u32 mode, u32 sign_unknown) {
    if (mode == 2) return match_dfa(pk, needle, sign_unknown != 0);
    return match_text(pk, needle, len, fold != 0, mode, sign_unknown != 0);
}

/*
 * Search indices first .. first+n-1: writes the indices whose key (y only,
 * sign bit cleared) may match with either sign, in increasing order.
 * Returns the number of such indices (hits beyond cap are counted, not written).
 */
EXPORT u64 mko_search(const u8 key[32], u32 src, u64 first, u64 n, const u8* needle, u32 len, u32 fold,
                      u32 mode, u64* hits, u64 cap) {
    oracle_init();
    u64 count = 0;
    for (u64 i = 0; i < n; i++) {
        u8 pk[32];
        index_pubkey(key, src, first + i, pk);
        pk[31] &= 0x7f;
        if (mko_match(pk, needle, len, fold, mode, 1)) {
            if (count < cap) hits[count] = first + i;
            count++;
        }
    }
    return count;
}

/* Candidate scan of n precomputed public keys pks (indices first .. first+n-1): the same
 * sign-unknown test as mko_search, for checking many needles against one key range. */
EXPORT u64 mko_match_keys(const u8* pks, u64 n, u64 first, const u8* needle, u32 len, u32 fold, u32 mode,
                          u64* hits, u64 cap) {
    u64 count = 0;
    for (u64 i = 0; i < n; i++) {
        u8 pk[32];
        memcpy(pk, pks + 32 * i, 32);
        pk[31] &= 0x7f;
        if (mko_match(pk, needle, len, fold, mode, 1)) {
            if (count < cap) hits[count] = first + i;
            count++;
        }
    }
    return count;
}

/* ------------------------------------------------------------------------ */
/* the reference's packed comb table (for the reference kernel built on CPU)  */
/* ------------------------------------------------------------------------ */

/* rows = ceil(251 / w), cols = 2^(w-1) + 1 (src/service/derive/comb.rs:285-287) */
EXPORT u64 mko_ref_table_words(u32 w) {
    u64 rows = (251 + w - 1) / w, cols = (1ull << (w - 1)) + 1;
    return rows * cols * 24;
}

static void put_fe_words(fe a, u32* out) {
    u8 b[32];
    fe_tobytes(a, b);
    for (int j = 0; j < 8; j++)
        out[j] = (u32)b[4 * j] | (u32)b[4 * j + 1] << 8 | (u32)b[4 * j + 2] << 16 | (u32)b[4 * j + 3] << 24;
}

/*
 * Row i, column k holds k · 2^(w·i) · 8B as (y+x, y-x, 2dxy), each canonical
 * and packed as 8 LE words; the top row is offset by 2^254·B and row 0 holds
 * 2xy in place of 2dxy (comb.rs:353-392, gpu.rs:1459-1480).  One row into
 * `out` (cols x 24 words), so that rows can be built on separate threads
 * (call mko_init first).
 */
EXPORT void mko_ref_table_row(u32 w, u32 i, u32* out) {
    oracle_init();
    u64 rows = (251 + w - 1) / w, cols = (1ull << (w - 1)) + 1;
    ge rowbase = BASE;
    for (u64 c = 0; c < 3 + (u64)w * i; c++) rowbase = ge_double(rowbase);
    fe* zs = (fe*)malloc(sizeof(fe) * cols);
    fe* pre = (fe*)malloc(sizeof(fe) * cols);
    ge* pts = (ge*)malloc(sizeof(ge) * cols);
    ge acc = ge_identity();
    if (i == rows - 1) {
        ge top = rowbase;
        for (u64 c = 0; c < 251 - w * (rows - 1); c++) top = ge_double(top);
        acc = top;
    }
    for (u64 k = 0; k < cols; k++) {
        pts[k] = acc;
        acc = ge_add(acc, rowbase);
    }
    /* batch inversion of the z coordinates */
    fe run = fe_one();
    for (u64 k = 0; k < cols; k++) { pre[k] = run; run = fe_mul(run, pts[k].z); }
    fe inv = fe_invert(run);
    for (u64 k = cols; k-- > 0;) { zs[k] = fe_mul(inv, pre[k]); inv = fe_mul(inv, pts[k].z); }
    for (u64 k = 0; k < cols; k++) {
        fe x = fe_mul(pts[k].x, zs[k]), y = fe_mul(pts[k].y, zs[k]);
        u32* e = out + k * 24;
        put_fe_words(fe_add(y, x), e);
        put_fe_words(fe_sub(y, x), e + 8);
        fe xy = fe_mul(x, y);
        put_fe_words(i == 0 ? fe_add(xy, xy) : fe_mul(xy, D2), e + 16);
    }
    free(zs);
    free(pre);
    free(pts);
}

EXPORT void mko_ref_table(u32 w, u32* out) {
    u64 rows = (251 + w - 1) / w, cols = (1ull << (w - 1)) + 1;
    for (u64 i = 0; i < rows; i++) mko_ref_table_row(w, (u32)i, out + i * cols * 24);
}

/* signed radix-2^w digits of m = bits 3..253 of a clamped scalar (comb.rs:414-445) */
EXPORT void mko_digits(const u8 s[32], u32 w, int32_t* out) {
    u64 words[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++)
        for (int b = 7; b >= 0; b--) words[i] = words[i] << 8 | s[8 * i + b];
    for (int i = 0; i < 4; i++) words[i] = words[i] >> 3 | words[i + 1] << 61;
    words[3] &= (1ull << (251 - 192)) - 1;
    u32 rows = (251 + w - 1) / w;
    int32_t half = 1 << (w - 1), carry = 0;
    for (u32 i = 0; i < rows; i++) {
        u32 off = i * w, q = off / 64, r = off % 64;
        u64 bits = words[q] >> r;
        if (r + w > 64 && q + 1 < 5) bits |= words[q + 1] << (64 - r);
        int32_t v = (int32_t)(bits & ((1ull << w) - 1)) + carry;
        if (i == rows - 1) out[i] = v;
        else {
            carry = (v + half) >> w;
            out[i] = v - (carry << w);
        }
    }
}
