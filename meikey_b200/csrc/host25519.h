// Host-side (CPU) Ed25519 pieces the runtime needs around the GPU path:
//   - the comb table's row base points (2^k·8B) and curve constants for the device;
//   - confirmation of every GPU hit: the hit's seed is re-derived and its public key
//     computed here before anything is reported or written (src/service/gpu.rs:973-996);
//   - the OpenSSH base64 form and the pattern test used by that confirmation
//     (src/model/key.rs:43-52, src/model/pattern.rs:186-226, src/model/pattern/dfa.rs:114-125).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace mkh25519 {

// seeds (src/model/search.rs:45-50, src/service/gpu.rs:1344-1351)
void chacha20_seed(const uint8_t key[32], uint64_t index, uint8_t seed[32]);
void counter_seed(const uint8_t base[32], uint64_t index, uint8_t seed[32]);
void seed_of(const uint8_t key[32], int source, uint64_t index, uint8_t seed[32]);

void sha512(const uint8_t* msg, size_t len, uint8_t out[64]);

// compressed public key of a 32-byte seed (RFC 8032 5.1.5)
void public_key(const uint8_t seed[32], uint8_t pk[32]);

// Incremental (low-security) path: index k stands for the scalar s0 + k itself (no hashing,
// no clamping), so its public key is (s0 + k)·B.  s0 must be below 2^255 (false otherwise),
// which keeps s0 + k below 2^256 for every 64-bit k.
bool incremental_scalar(const uint8_t s0[32], uint64_t k, uint8_t s[32]);
// compressed public key of the 256-bit little-endian scalar s
void scalar_public_key(const uint8_t s[32], uint8_t pk[32]);
// s·B as extended coordinates with Z = 1: x, y, 1, xy (8 canonical LE words each)
void scalar_point_words(const uint8_t s[32], uint32_t out[32]);
// k·B in the table form (y+x, y-x, 2d·xy), 8 canonical LE words each; k = 0 gives (1, 1, 0)
void niels_of_multiple(uint64_t k, uint32_t out[24]);

// 68 base64 characters of the OpenSSH key blob (no terminator)
void public_b64(const uint8_t pk[32], char out[68]);

// A needle as the GPU receives it; `matches` tests the full key (x sign known).
struct Needle {
    std::vector<uint8_t> bytes;
    uint32_t len = 0;
    bool fold = false;
    uint32_t mode = 0;  // 0 contains, 1 suffix, 2 regex (bytes = DFA table)
};
bool matches(const Needle& n, const uint8_t pk[32]);

// Device constants: canonical little-endian words.
// rows_points: for every comb row, R = 2^(3+offset)·B then O (identity, or 2^254·B on the
// top row), each as extended (X, Y, Z, T) with 8 words per coordinate; then 2d.
std::vector<uint32_t> comb_points(uint32_t rows, const uint32_t* offsets);

}  // namespace mkh25519
