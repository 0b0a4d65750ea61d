// Host-side Ed25519 (see host25519.h).  GF(2^255-19) in five 51-bit limbs with
// 128-bit products; points in extended coordinates; a fixed-base multiply with a
// 4-bit window table built once.  Used only for set-up and for hit confirmation.
#include "host25519.h"

#include <string.h>

#include <mutex>

namespace mkh25519 {

namespace {

typedef unsigned __int128 u128;
typedef uint64_t u64;
typedef uint32_t u32;
constexpr u64 MASK51 = (1ull << 51) - 1;

struct Fe {
    u64 l[5];
};

Fe fe(u64 x) { return Fe{{x, 0, 0, 0, 0}}; }

Fe carry(Fe a) {
    for (int i = 0; i < 4; i++) {
        a.l[i + 1] += a.l[i] >> 51;
        a.l[i] &= MASK51;
    }
    a.l[0] += 19 * (a.l[4] >> 51);
    a.l[4] &= MASK51;
    a.l[1] += a.l[0] >> 51;
    a.l[0] &= MASK51;
    return a;
}

Fe operator+(Fe a, const Fe& b) {
    for (int i = 0; i < 5; i++) a.l[i] += b.l[i];
    return carry(a);
}

// a - b + 4p
Fe operator-(Fe a, const Fe& b) {
    a.l[0] += 4 * (MASK51 - 18) - b.l[0];
    for (int i = 1; i < 5; i++) a.l[i] += 4 * MASK51 - b.l[i];
    return carry(a);
}

Fe operator*(const Fe& a, const Fe& b) {
    u128 t[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            u128 p = (u128)a.l[i] * b.l[j];
            if (i + j >= 5) t[i + j - 5] += p * 19;
            else t[i + j] += p;
        }
    Fe r;
    u128 c = 0;
    for (int i = 0; i < 5; i++) {
        t[i] += c;
        r.l[i] = (u64)t[i] & MASK51;
        c = t[i] >> 51;
    }
    r.l[0] += (u64)c * 19;
    return carry(r);
}

Fe neg(const Fe& a) { return fe(0) - a; }

void to_bytes(Fe a, uint8_t out[32]) {
    a = carry(carry(a));
    u64 q = (a.l[0] + 19) >> 51;
    for (int i = 1; i < 5; i++) q = (a.l[i] + q) >> 51;
    a.l[0] += 19 * q;
    for (int i = 0; i < 4; i++) {
        a.l[i + 1] += a.l[i] >> 51;
        a.l[i] &= MASK51;
    }
    a.l[4] &= MASK51;
    u64 w[4] = {a.l[0] | a.l[1] << 51, a.l[1] >> 13 | a.l[2] << 38, a.l[2] >> 26 | a.l[3] << 25,
                a.l[3] >> 39 | a.l[4] << 12};
    for (int i = 0; i < 32; i++) out[i] = (uint8_t)(w[i / 8] >> (8 * (i % 8)));
}

void to_words(const Fe& a, u32 out[8]) {
    uint8_t b[32];
    to_bytes(a, b);
    for (int j = 0; j < 8; j++) out[j] = (u32)b[4 * j] | (u32)b[4 * j + 1] << 8 | (u32)b[4 * j + 2] << 16 | (u32)b[4 * j + 3] << 24;
}

// a^e, e as 256-bit little-endian bytes
Fe pow(const Fe& a, const uint8_t e[32]) {
    Fe r = fe(1);
    for (int bit = 255; bit >= 0; bit--) {
        r = r * r;
        if ((e[bit >> 3] >> (bit & 7)) & 1) r = r * a;
    }
    return r;
}

// exponent 2^255 - 19 - sub as bytes
void exp_bytes(uint8_t e[32], int sub, int top, int low) {
    memset(e, 0xff, 32);
    e[31] = (uint8_t)top;
    e[0] = (uint8_t)low;
    (void)sub;
}

Fe invert(const Fe& a) {
    uint8_t e[32];
    exp_bytes(e, 2, 0x7f, 0xeb);  // p - 2
    return pow(a, e);
}

bool is_odd(const Fe& a) {
    uint8_t b[32];
    to_bytes(a, b);
    return b[0] & 1;
}

bool equal(const Fe& a, const Fe& b) {
    uint8_t x[32], y[32];
    to_bytes(a, x);
    to_bytes(b, y);
    return memcmp(x, y, 32) == 0;
}

struct Pt {
    Fe X, Y, Z, T;
};

struct Consts {
    Fe d, d2, sqrtm1;
    Pt B;
    Pt win[64][16];  // win[i][j] = j·16^i·B (j = 0..15), extended, Z = 1
};

Pt add(const Pt& p, const Pt& q, const Fe& d2) {
    Fe a = (p.Y - p.X) * (q.Y - q.X);
    Fe b = (p.Y + p.X) * (q.Y + q.X);
    Fe c = p.T * d2 * q.T;
    Fe zz = p.Z * q.Z;
    Fe d = zz + zz;
    Fe e = b - a, f = d - c, g = d + c, h = b + a;
    return Pt{e * f, g * h, f * g, e * h};
}

Pt identity() { return Pt{fe(0), fe(1), fe(1), fe(0)}; }

Pt affine(const Pt& p) {
    Fe zi = invert(p.Z);
    Fe x = p.X * zi, y = p.Y * zi;
    return Pt{x, y, fe(1), x * y};
}

const Consts& consts() {
    static Consts C;
    static std::once_flag once;
    std::call_once(once, [] {
        C.d = neg(fe(121665)) * invert(fe(121666));
        C.d2 = C.d + C.d;
        uint8_t e[32];
        exp_bytes(e, 0, 0x1f, 0xfb);  // (p - 1) / 4
        C.sqrtm1 = pow(fe(2), e);
        // base point: y = 4/5, x even (RFC 8032 5.1)
        Fe y = fe(4) * invert(fe(5));
        Fe yy = y * y;
        Fe u = yy - fe(1), v = C.d * yy + fe(1);
        Fe v3 = v * v * v;
        Fe v7 = v3 * v3 * v;
        exp_bytes(e, 0, 0x0f, 0xfd);  // (p - 5) / 8
        Fe x = u * v3 * pow(u * v7, e);
        if (!equal(v * x * x, u)) x = x * C.sqrtm1;
        if (is_odd(x)) x = neg(x);
        C.B = Pt{x, y, fe(1), x * y};
        Pt row = C.B;
        for (int i = 0; i < 64; i++) {
            Pt acc = identity();
            for (int j = 0; j < 16; j++) {
                C.win[i][j] = affine(acc);
                acc = add(acc, row, C.d2);
            }
            for (int k = 0; k < 4; k++) row = add(row, row, C.d2);
        }
    });
    return C;
}

Pt base_mul(const uint8_t s[32]) {
    const Consts& C = consts();
    Pt acc = identity();
    for (int i = 0; i < 64; i++) {
        int dgt = (s[i >> 1] >> ((i & 1) * 4)) & 15;
        if (dgt) acc = add(acc, C.win[i][dgt], C.d2);
    }
    return acc;
}

void compress(const Pt& p, uint8_t out[32]) {
    Pt a = affine(p);
    to_bytes(a.Y, out);
    out[31] |= (uint8_t)(is_odd(a.X) << 7);
}

// ---- ChaCha20 / SHA-512 ----

u32 rotl(u32 x, int n) { return (x << n) | (x >> (32 - n)); }

void chacha_block(const u32 k[8], u64 ctr, u32 out[16]) {
    u32 s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, k[0], k[1], k[2], k[3],
                 k[4], k[5], k[6], k[7], (u32)ctr, (u32)(ctr >> 32), 0, 0};
    u32 x[16];
    memcpy(x, s, sizeof x);
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 16);
        x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 12);
        x[a] += x[b]; x[d] = rotl(x[d] ^ x[a], 8);
        x[c] += x[d]; x[b] = rotl(x[b] ^ x[c], 7);
    };
    for (int r = 0; r < 10; r++) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

const u64 K[80] = {
    0x428a2f98d728ae22ull, 0x7137449123ef65cdull, 0xb5c0fbcfec4d3b2full, 0xe9b5dba58189dbbcull, 0x3956c25bf348b538ull,
    0x59f111f1b605d019ull, 0x923f82a4af194f9bull, 0xab1c5ed5da6d8118ull, 0xd807aa98a3030242ull, 0x12835b0145706fbeull,
    0x243185be4ee4b28cull, 0x550c7dc3d5ffb4e2ull, 0x72be5d74f27b896full, 0x80deb1fe3b1696b1ull, 0x9bdc06a725c71235ull,
    0xc19bf174cf692694ull, 0xe49b69c19ef14ad2ull, 0xefbe4786384f25e3ull, 0x0fc19dc68b8cd5b5ull, 0x240ca1cc77ac9c65ull,
    0x2de92c6f592b0275ull, 0x4a7484aa6ea6e483ull, 0x5cb0a9dcbd41fbd4ull, 0x76f988da831153b5ull, 0x983e5152ee66dfabull,
    0xa831c66d2db43210ull, 0xb00327c898fb213full, 0xbf597fc7beef0ee4ull, 0xc6e00bf33da88fc2ull, 0xd5a79147930aa725ull,
    0x06ca6351e003826full, 0x142929670a0e6e70ull, 0x27b70a8546d22ffcull, 0x2e1b21385c26c926ull, 0x4d2c6dfc5ac42aedull,
    0x53380d139d95b3dfull, 0x650a73548baf63deull, 0x766a0abb3c77b2a8ull, 0x81c2c92e47edaee6ull, 0x92722c851482353bull,
    0xa2bfe8a14cf10364ull, 0xa81a664bbc423001ull, 0xc24b8b70d0f89791ull, 0xc76c51a30654be30ull, 0xd192e819d6ef5218ull,
    0xd69906245565a910ull, 0xf40e35855771202aull, 0x106aa07032bbd1b8ull, 0x19a4c116b8d2d0c8ull, 0x1e376c085141ab53ull,
    0x2748774cdf8eeb99ull, 0x34b0bcb5e19b48a8ull, 0x391c0cb3c5c95a63ull, 0x4ed8aa4ae3418acbull, 0x5b9cca4f7763e373ull,
    0x682e6ff3d6b2b8a3ull, 0x748f82ee5defb2fcull, 0x78a5636f43172f60ull, 0x84c87814a1f0ab72ull, 0x8cc702081a6439ecull,
    0x90befffa23631e28ull, 0xa4506cebde82bde9ull, 0xbef9a3f7b2c67915ull, 0xc67178f2e372532bull, 0xca273eceea26619cull,
    0xd186b8c721c0c207ull, 0xeada7dd6cde0eb1eull, 0xf57d4f7fee6ed178ull, 0x06f067aa72176fbaull, 0x0a637dc5a2c898a6ull,
    0x113f9804bef90daeull, 0x1b710b35131c471bull, 0x28db77f523047d84ull, 0x32caab7b40c72493ull, 0x3c9ebe0a15c9bebcull,
    0x431d67c49c100d4cull, 0x4cc5d4becb3e42b6ull, 0x597f299cfc657e2aull, 0x5fcb6fab3ad6faecull, 0x6c44198c4a475817ull,
};

u64 rotr(u64 x, int n) { return (x >> n) | (x << (64 - n)); }

void compress_block(u64 h[8], const uint8_t* p) {
    u64 w[80];
    for (int t = 0; t < 16; t++) {
        w[t] = 0;
        for (int b = 0; b < 8; b++) w[t] = w[t] << 8 | p[8 * t + b];
    }
    for (int t = 16; t < 80; t++)
        w[t] = w[t - 16] + (rotr(w[t - 15], 1) ^ rotr(w[t - 15], 8) ^ (w[t - 15] >> 7)) + w[t - 7] +
               (rotr(w[t - 2], 19) ^ rotr(w[t - 2], 61) ^ (w[t - 2] >> 6));
    u64 v[8];
    memcpy(v, h, sizeof v);
    for (int t = 0; t < 80; t++) {
        u64 t1 = v[7] + (rotr(v[4], 14) ^ rotr(v[4], 18) ^ rotr(v[4], 41)) + ((v[4] & v[5]) ^ (~v[4] & v[6])) + K[t] + w[t];
        u64 t2 = (rotr(v[0], 28) ^ rotr(v[0], 34) ^ rotr(v[0], 39)) + ((v[0] & v[1]) ^ (v[0] & v[2]) ^ (v[1] & v[2]));
        memmove(v + 1, v, 7 * sizeof(u64));
        v[4] += t1;
        v[0] = t1 + t2;
    }
    for (int i = 0; i < 8; i++) h[i] += v[i];
}

const char B64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

}  // namespace

void sha512(const uint8_t* msg, size_t len, uint8_t out[64]) {
    u64 h[8] = {0x6a09e667f3bcc908ull, 0xbb67ae8584caa73bull, 0x3c6ef372fe94f82bull, 0xa54ff53a5f1d36f1ull,
                0x510e527fade682d1ull, 0x9b05688c2b3e6c1full, 0x1f83d9abfb41bd6bull, 0x5be0cd19137e2179ull};
    size_t off = 0;
    for (; len - off >= 128; off += 128) compress_block(h, msg + off);
    uint8_t tail[256] = {0};
    size_t rem = len - off;
    memcpy(tail, msg + off, rem);
    tail[rem] = 0x80;
    size_t total = rem + 17 <= 128 ? 128 : 256;
    u64 bits = (u64)len * 8;
    for (int b = 0; b < 8; b++) tail[total - 1 - b] = (uint8_t)(bits >> (8 * b));
    compress_block(h, tail);
    if (total == 256) compress_block(h, tail + 128);
    for (int i = 0; i < 64; i++) out[i] = (uint8_t)(h[i / 8] >> (56 - 8 * (i % 8)));
}

void chacha20_seed(const uint8_t key[32], uint64_t index, uint8_t seed[32]) {
    u32 k[8], blk[16];
    for (int i = 0; i < 8; i++) k[i] = (u32)key[4 * i] | (u32)key[4 * i + 1] << 8 | (u32)key[4 * i + 2] << 16 | (u32)key[4 * i + 3] << 24;
    chacha_block(k, index >> 1, blk);
    const u32* half = blk + ((index & 1) ? 8 : 0);
    for (int i = 0; i < 32; i++) seed[i] = (uint8_t)(half[i / 4] >> (8 * (i % 4)));
}

void counter_seed(const uint8_t base[32], uint64_t index, uint8_t seed[32]) {
    memcpy(seed, base, 32);
    u64 tail = 0;
    for (int b = 7; b >= 0; b--) tail = tail << 8 | base[24 + b];
    tail += index;
    for (int b = 0; b < 8; b++) seed[24 + b] = (uint8_t)(tail >> (8 * b));
}

void seed_of(const uint8_t key[32], int source, uint64_t index, uint8_t seed[32]) {
    if (source == 1) counter_seed(key, index, seed);
    else chacha20_seed(key, index, seed);
}

void public_key(const uint8_t seed[32], uint8_t pk[32]) {
    uint8_t h[64];
    sha512(seed, 32, h);
    h[0] &= 248;
    h[31] &= 127;
    h[31] |= 64;
    compress(base_mul(h), pk);
}

void scalar_public_key(const uint8_t s[32], uint8_t pk[32]) { compress(base_mul(s), pk); }

bool incremental_scalar(const uint8_t s0[32], uint64_t k, uint8_t s[32]) {
    if (s0[31] & 0x80) return false;
    u64 c = 0;
    for (int b = 0; b < 32; b++) {
        c += (u64)s0[b] + (b < 8 ? (k >> (8 * b)) & 0xff : 0);
        s[b] = (uint8_t)c;
        c >>= 8;
    }
    return true;
}

void scalar_point_words(const uint8_t s[32], uint32_t out[32]) {
    Pt a = affine(base_mul(s));
    to_words(a.X, out);
    to_words(a.Y, out + 8);
    to_words(a.Z, out + 16);
    to_words(a.T, out + 24);
}

void niels_of_multiple(uint64_t k, uint32_t out[24]) {
    const Consts& C = consts();
    uint8_t s[32] = {};
    for (int b = 0; b < 8; b++) s[b] = (uint8_t)(k >> (8 * b));
    Pt a = affine(base_mul(s));
    to_words(a.Y + a.X, out);
    to_words(a.Y - a.X, out + 8);
    to_words(a.T * C.d2, out + 16);
}

void public_b64(const uint8_t pk[32], char out[68]) {
    static const char HEAD[] = "AAAAC3NzaC1lZDI1NTE5AAAA";
    memcpy(out, HEAD, 24);
    uint8_t tail[33];
    tail[0] = 32;
    memcpy(tail + 1, pk, 32);
    for (int g = 0; g < 11; g++) {
        u32 n = (u32)tail[3 * g] << 16 | (u32)tail[3 * g + 1] << 8 | tail[3 * g + 2];
        for (int k = 0; k < 4; k++) out[24 + 4 * g + k] = B64[(n >> (18 - 6 * k)) & 63];
    }
}

bool matches(const Needle& n, const uint8_t pk[32]) {
    char b64[68];
    public_b64(pk, b64);
    const char* hay = b64 + 25;  // after the fixed prefix
    const int hay_len = 43;
    if (n.mode == 2) {
        auto next = [&](u32 s, u32 i) -> u32 {
            size_t at = ((size_t)s * 65 + i) * 2;
            return (u32)n.bytes[at] | (u32)n.bytes[at + 1] << 8;
        };
        u32 s = 1;
        for (int i = 0; i < hay_len; i++) {
            const char* p = strchr(B64, hay[i]);
            s = next(s, (u32)(p - B64));
            if (s == 0) return true;
        }
        return next(s, 64) != 0;
    }
    const int len = (int)n.len;
    if (len == 0 || len > hay_len) return false;
    auto same = [&](const char* w) {
        for (int k = 0; k < len; k++) {
            char c = w[k];
            if (n.fold && c >= 'A' && c <= 'Z') c = (char)(c + 32);
            if ((uint8_t)c != n.bytes[k]) return false;
        }
        return true;
    };
    if (n.mode == 1) return same(hay + hay_len - len);
    for (int s = 0; s + len <= hay_len; s++)
        if (same(hay + s)) return true;
    return false;
}

std::vector<uint32_t> comb_points(uint32_t rows, const uint32_t* offsets) {
    const Consts& C = consts();
    std::vector<uint32_t> out((size_t)rows * 64 + 8);
    // 8B then doublings up to each row's offset
    Pt b8 = C.B;
    for (int i = 0; i < 3; i++) b8 = add(b8, b8, C.d2);
    Pt cur = b8;
    uint32_t at = 0;
    for (uint32_t r = 0; r < rows; r++) {
        while (at < offsets[r]) {
            cur = add(cur, cur, C.d2);
            at++;
        }
        Pt R = affine(cur);
        Pt O = identity();
        if (r == rows - 1) {
            Pt t = C.B;
            for (int i = 0; i < 254; i++) t = add(t, t, C.d2);
            O = affine(t);
        }
        const Fe* rc[4] = {&R.X, &R.Y, &R.Z, &R.T};
        const Fe* oc[4] = {&O.X, &O.Y, &O.Z, &O.T};
        for (int c = 0; c < 4; c++) {
            to_words(*rc[c], &out[(size_t)r * 64 + 8 * c]);
            to_words(*oc[c], &out[(size_t)r * 64 + 32 + 8 * c]);
        }
    }
    to_words(C.d2, &out[(size_t)rows * 64]);
    return out;
}

}  // namespace mkh25519
