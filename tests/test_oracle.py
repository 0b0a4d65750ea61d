"""The CPU oracle against the golden vectors (no GPU).

The oracle is the checker of every GPU parity test, so it is pinned here against:
RFC 8032 section 7.1, OpenSSL (via the committed fixtures), the reference's own
kernel compiled for the CPU (fixtures, and live when oracle/_ref exists)."""
import hashlib
import json
import os
import random

import pytest

from conftest import GOLDEN, chacha_key


def test_rfc8032_vectors(oracle):
    """src/service/derive.rs:625-657 checks the same secret -> public pairs."""
    vec = json.load(open(os.path.join(GOLDEN, "rfc8032.json")))
    assert len(vec) >= 5
    for v in vec:
        assert oracle.pubkey(bytes.fromhex(v["secret"])).hex() == v["public"], v["name"]


def test_seed_streams(oracle):
    """ChaCha20 halves per index (gpu.rs:1344-1351) and counter seeds (model/search.rs:45-50)."""
    s = json.load(open(os.path.join(GOLDEN, "seeds.json")))
    key = bytes.fromhex(s["key"])
    assert key == chacha_key(1)
    for i, hexseed in s["chacha20"].items():
        assert oracle.seed(key, 0, int(i)).hex() == hexseed, i
    for i, hexseed in s["counter"].items():
        assert oracle.seed(key, 1, int(i)).hex() == hexseed, i
    # consecutive indices are consecutive 32-byte pieces of one keystream
    a, b = oracle.seed(key, 0, 6), oracle.seed(key, 0, 7)
    assert a != b


def test_pubkey_fixtures(oracle, golden_pubkeys):
    cha, cnt = golden_pubkeys
    key = chacha_key(1)
    assert oracle.derive(key, 0, 0, 4096) == cha
    assert oracle.derive(key, 1, 0, 1024) == cnt


def test_high_index_fixture(oracle, golden):
    key = bytes.fromhex(golden["chacha_key"])
    first = golden["pubkeys_high_first"]
    want = oracle.derive(key, 0, first, 16).hex()
    for variant, got in golden["pubkeys_high_by_reference_variant"].items():
        assert got == want, variant


def test_checksum_of_small_secure_workload(oracle, golden):
    """All 2^20 public keys of the small secure-path workload hash to the fixture."""
    key = bytes.fromhex(golden["chacha_key"])
    full = oracle.derive(key, 0, 0, 1 << 20)
    assert hashlib.sha256(full).hexdigest() == golden["sha256_of_pubkeys_0_2pow20"]


def test_search_fixtures(oracle, golden):
    """Candidate sets of the reference matcher (kernel.cu:1804-1875, sign unknown)."""
    key = bytes.fromhex(golden["chacha_key"])
    lo, hi = golden["search_range"]
    dfas = {d["regex"]: d for d in golden["dfas"]}
    for case in golden["search"][:6]:
        if case["mode"] == 2:
            d = dfas[case["regex"]]
            needle, length, fold = bytes.fromhex(d["table"]), d["states"], False
        else:
            fold = case["fold"]
            needle = case["needle"].lower().encode() if fold else case["needle"].encode()
            length = len(needle)
        assert oracle.search(key, 0, lo, hi - lo, needle, length, fold, case["mode"]) == case["hits"]


def test_sign_unknown_never_misses(oracle):
    """contains_unsigned_never_misses (src/service/gpu.rs:2113-2152): if the y-only key is not
    a candidate, neither sign of x gives a match.  Half the needles are cut from the key's own
    text across the sign-dependent character (tail position 42)."""
    rng = random.Random(11)
    alphabet = b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/"
    for trial in range(3000):
        pk = bytearray(rng.getrandbits(8) for _ in range(32))
        n = rng.randint(1, 4)
        if trial % 2:
            hay = oracle.public_b64(bytes(pk))[25:]  # tail positions 1..43
            sign_at = 41  # tail position 42
            start = max(0, min(43 - n, sign_at - rng.randint(0, n - 1)))
            needle = hay[start:start + n].encode()
        else:
            needle = bytes(rng.choice(alphabet) for _ in range(n))
        for mode in (0, 1):
            for fold in (False, True):
                nb = needle.lower() if fold else needle
                y = bytearray(pk)
                y[31] &= 0x7F
                maybe = oracle.match(bytes(y), nb, len(nb), fold, mode, True)
                for sign in (0, 0x80):
                    k = bytearray(y)
                    k[31] |= sign
                    if oracle.match(bytes(k), nb, len(nb), fold, mode, False):
                        assert maybe, (bytes(k).hex(), nb, mode, fold)


def test_full_match_agrees_with_text_search(oracle):
    """match (sign known) is a plain substring / suffix test on the 43 characters after the prefix."""
    rng = random.Random(3)
    for _ in range(2000):
        pk = bytes(rng.getrandbits(8) for _ in range(32))
        text = oracle.public_b64(pk)
        hay = text[25:]
        start = rng.randrange(0, 43)
        n = rng.randint(1, 43 - start)
        needle = hay[start:start + n]
        assert oracle.match(pk, needle.encode(), n, False, 0, False)
        assert oracle.match(pk, needle.lower().encode(), n, True, 0, False)
        assert oracle.match(pk, needle.encode(), n, False, 1, False) == hay.endswith(needle)


@pytest.mark.skipif(not os.path.isdir(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref")),
                    reason="reference CPU build (oracle/_ref) not present")
def test_oracle_matches_reference_cpu_build(oracle):
    """Live cross-check with the reference's kernel.cu compiled as C++ (every variant)."""
    variants = oracle.ref_variants()
    if not variants:
        pytest.skip("no reference variant built")
    table = oracle.ref_table(9)
    key = chacha_key(42)
    for path in variants:
        rk = oracle.RefKernel(path)
        for counter in (False, True):
            for first in (0, 1, 2**32 - 3, 2**40 + 17):
                got = rk.derive(table, 9, key, counter, first)
                assert got == oracle.derive(key, 1 if counter else 0, first, rk.batch), (path, counter, first)


def test_reference_table_digits(oracle):
    """Signed radix-2^w digits reassemble m = bits 3..253 of a clamped scalar (comb.rs:414-445)."""
    import ctypes
    rng = random.Random(9)
    for w in (2, 9, 12, 16, 20):
        rows = (251 + w - 1) // w
        for _ in range(50):
            s = bytearray(rng.getrandbits(8) for _ in range(32))
            s[0] &= 248
            s[31] &= 127
            s[31] |= 64
            out = (ctypes.c_int32 * rows)()
            oracle.lib().mko_digits(bytes(s), w, out)
            m = (int.from_bytes(bytes(s), "little") >> 3) & ((1 << 251) - 1)
            assert sum(d << (w * i) for i, d in enumerate(out)) == m
            half = 1 << (w - 1)
            assert all(-half <= d < half for d in out[:-1])
            assert 0 <= out[-1] <= half


def _clamp(h: bytes) -> bytes:
    s = bytearray(h[:32])
    s[0] &= 248
    s[31] &= 127
    s[31] |= 64
    return bytes(s)


def test_incremental_oracle_pins(oracle):
    """Incremental path (P_k = P_0 + k·B): key 0 of the start scalar clamp(SHA-512(seed)) is the
    seed's Ed25519 public key, and P_0 + B + ... + B built with plain Python affine Edwards
    additions gives the oracle's keys k = 0..40 (an independent restatement of the point sum)."""
    p = 2**255 - 19
    d = (-121665 * pow(121666, p - 2, p)) % p
    inv = lambda v: pow(v, p - 2, p)  # noqa: E731

    def add(P, Q):
        (x1, y1), (x2, y2) = P, Q
        t = d * x1 * x2 * y1 * y2 % p
        return ((x1 * y2 + y1 * x2) * inv(1 + t) % p, (y1 * y2 + x1 * x2) * inv(1 - t) % p)

    def compress(P):
        x, y = P
        return (y | (x & 1) << 255).to_bytes(32, "little")

    key = chacha_key(11)
    for index in (0, 1, 977):
        seed = oracle.seed(key, 0, index)
        s0 = _clamp(hashlib.sha512(seed).digest())
        assert oracle.derive(s0, 2, 0, 1) == oracle.pubkey(seed)
        B = oracle.point_affine(1)
        P = oracle.point_affine(int.from_bytes(s0, "little"))
        got = oracle.derive(s0, 2, 0, 41)
        for k in range(41):
            assert got[32 * k:32 * k + 32] == compress(P), (index, k)
            P = add(P, B)
    # far indices: key k of s0 is key 0 of s0 + k
    s0 = _clamp(hashlib.sha512(oracle.seed(key, 0, 0)).digest())
    for k in (2**32 - 1, 2**40 + 3, 2**64 - 1):
        sk = (int.from_bytes(s0, "little") + k).to_bytes(32, "little")
        assert oracle.derive(s0, 2, k, 1) == oracle.derive(sk, 2, 0, 1) == oracle.base_mul(sk)
