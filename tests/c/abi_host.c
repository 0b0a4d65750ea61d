/* The C ABI used from C (gcc, no C++ runtime of the caller): the entry points that need no
 * device.  Prints one line per check; exits non-zero on the first failure. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "meikey_b200.h"

#define CHECK(cond, what)                                  \
    do {                                                   \
        if (!(cond)) {                                     \
            fprintf(stderr, "FAIL %s\n", what);            \
            return 1;                                      \
        }                                                  \
        printf("ok %s\n", what);                           \
    } while (0)

static int hexval(char c) { return c <= '9' ? c - '0' : (c | 32) - 'a' + 10; }

int main(int argc, char** argv) {
    /* argv[1]: RFC 8032 TEST 1 public key, hex */
    if (argc < 2 || strlen(argv[1]) != 64) return 2;
    uint8_t pk[32];
    for (int i = 0; i < 32; i++) pk[i] = (uint8_t)(hexval(argv[1][2 * i]) << 4 | hexval(argv[1][2 * i + 1]));

    CHECK(mk_abi_version() == MK_ABI_VERSION, "abi version");

    static uint8_t table[64 * 130];
    uint32_t states = 0;
    char err[128];
    CHECK(mk_regex_compile("x.{2}y$", 1, 64, table, &states, err, sizeof err) == MK_OK && states > 2, "regex compile");
    CHECK(mk_regex_compile("(ab", 1, 64, table, &states, err, sizeof err) == MK_ERR_PATTERN && err[0], "regex error text");

    mk_needle suffix = {(const uint8_t*)"Ab", 2, 0, MK_MODE_SUFFIX};
    CHECK(fabs(mk_expected_tries(&suffix) - 4096.0) < 1e-6, "expected tries of a 2-character suffix");
    mk_needle bad = {(const uint8_t*)"a-b", 3, 0, MK_MODE_CONTAINS};
    CHECK(mk_needles_check(&bad, 1) == MK_ERR_PATTERN, "needle outside the base64 alphabet");

    char line[256];
    size_t n = 0;
    CHECK(mk_openssh_public(pk, "", line, sizeof line, &n) == MK_OK &&
              strcmp(line, "ssh-ed25519 AAAAC3NzaC1lZDI1NTE5AAAAINdamAGCsQq31Uv+08lkBzoO4XLz2qYjJa8CGmj3B1Ea") == 0 &&
              n == strlen(line),
          "openssh public line");
    CHECK(mk_openssh_public(pk, "a\nb", line, sizeof line, &n) == MK_ERR_BAD_ARG, "comment with a line break");
    char small[8];
    CHECK(mk_openssh_public(pk, "", small, sizeof small, &n) == MK_ERR_BAD_ARG && n > sizeof small, "buffer too small");
    return 0;
}
