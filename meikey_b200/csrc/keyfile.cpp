// OpenSSH output of a found key (VanityKey::public_openssh, src/model/key.rs:132-139, and
// private_openssh, src/repository/key_file.rs:276-320): the authorized_keys line and the
// unencrypted "openssh-key-v1" private key file (OpenSSH PROTOCOL.key), built from the
// RFC 4251 wire forms (uint32 big-endian, string = uint32 length + bytes).
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/meikey_b200.h"
#include "abi_guard.h"
#include "host25519.h"

namespace {

const char B64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

std::string base64(const std::vector<uint8_t>& in) {
    std::string out;
    size_t i = 0;
    for (; i + 3 <= in.size(); i += 3) {
        uint32_t n = (uint32_t)in[i] << 16 | (uint32_t)in[i + 1] << 8 | in[i + 2];
        for (int k = 0; k < 4; k++) out += B64[(n >> (18 - 6 * k)) & 63];
    }
    if (i < in.size()) {
        uint32_t n = (uint32_t)in[i] << 16 | (i + 1 < in.size() ? (uint32_t)in[i + 1] << 8 : 0u);
        out += B64[(n >> 18) & 63];
        out += B64[(n >> 12) & 63];
        out += i + 1 < in.size() ? B64[(n >> 6) & 63] : '=';
        out += '=';
    }
    return out;
}

void put_u32(std::vector<uint8_t>& b, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}

void put_string(std::vector<uint8_t>& b, const uint8_t* p, size_t n) {
    put_u32(b, (uint32_t)n);
    b.insert(b.end(), p, p + n);
}

void put_string(std::vector<uint8_t>& b, const char* s) { put_string(b, (const uint8_t*)s, strlen(s)); }

// "string ssh-ed25519, string key" (RFC 8709 section 4)
std::vector<uint8_t> public_blob(const uint8_t pk[32]) {
    std::vector<uint8_t> b;
    put_string(b, "ssh-ed25519");
    put_string(b, pk, 32);
    return b;
}

bool comment_ok(const char* c) { return !strchr(c, '\n') && !strchr(c, '\r'); }

void wipe(std::vector<uint8_t>& v) {
    volatile uint8_t* p = v.data();
    for (size_t i = 0; i < v.size(); i++) p[i] = 0;
}

void wipe(std::string& s) {
    volatile char* p = &s[0];
    for (size_t i = 0; i < s.size(); i++) p[i] = 0;
}

int emit(const std::string& s, char* out, size_t cap, size_t* written) {
    if (written) *written = s.size();
    if (!out || cap < s.size() + 1) return MK_ERR_BAD_ARG;
    memcpy(out, s.c_str(), s.size() + 1);
    return MK_OK;
}

}  // namespace

extern "C" int mk_openssh_public(const uint8_t pk[32], const char* comment, char* out, size_t cap, size_t* written) try {
    if (!pk || !comment || !comment_ok(comment)) return MK_ERR_BAD_ARG;
    std::string line = "ssh-ed25519 " + base64(public_blob(pk));
    if (*comment) line += std::string(" ") + comment;
    return emit(line, out, cap, written);
} MK_ABI_CATCH(nullptr)

extern "C" int mk_openssh_private(const uint8_t seed[32], const char* comment, uint32_t checkint, char* out,
                                  size_t cap, size_t* written) try {
    if (!seed || !comment || !comment_ok(comment)) return MK_ERR_BAD_ARG;
    uint8_t pk[32];
    mkh25519::public_key(seed, pk);
    std::vector<uint8_t> keypair(seed, seed + 32);
    keypair.insert(keypair.end(), pk, pk + 32);
    std::vector<uint8_t> priv;
    put_u32(priv, checkint);
    put_u32(priv, checkint);
    put_string(priv, "ssh-ed25519");
    put_string(priv, pk, 32);
    put_string(priv, keypair.data(), keypair.size());
    put_string(priv, comment);
    for (uint8_t pad = 1; priv.size() % 8; pad++) priv.push_back(pad);  // 1, 2, 3, ... to a multiple of 8
    std::vector<uint8_t> body((const uint8_t*)"openssh-key-v1", (const uint8_t*)"openssh-key-v1" + 15);  // with its NUL
    put_string(body, "none");  // cipher
    put_string(body, "none");  // kdf
    put_string(body, "");      // kdf options
    put_u32(body, 1);          // number of keys
    std::vector<uint8_t> blob = public_blob(pk);
    put_string(body, blob.data(), blob.size());
    put_string(body, priv.data(), priv.size());
    std::string b64 = base64(body);
    std::string pem = "-----BEGIN OPENSSH PRIVATE KEY-----\n";
    for (size_t i = 0; i < b64.size(); i += 70) pem += b64.substr(i, 70) + "\n";
    pem += "-----END OPENSSH PRIVATE KEY-----\n";
    int st = emit(pem, out, cap, written);
    wipe(keypair);
    wipe(priv);
    wipe(body);
    wipe(b64);
    wipe(pem);
    return st;
} MK_ABI_CATCH(nullptr)
