"""Generates the golden fixtures in this directory (run in a container where the
reference tree and Python `cryptography` are available):

    python tests/golden/make_golden.py

Sources of truth, cross-checked against each other before anything is written:
  * the RFC 8032 section 7.1 vectors from the reference's tests/data/rfc8032-ed25519.txt;
  * OpenSSL's Ed25519 and ChaCha20 through Python `cryptography`;
  * the reference's own kernel source compiled for the CPU (oracle/_ref, built by
    `make -C oracle ref`), driven with the reference's comb table (restated in the oracle);
  * the C oracle (oracle/liboracle.so).
Outputs are small: they are what the GPU tests compare against on a box without the reference.
"""
import hashlib
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import pyoracle as po  # noqa: E402
import dfa_builder  # noqa: E402

REF = os.environ.get("REF", os.path.join(os.path.dirname(ROOT), "reference"))


def chacha_key(seed: int) -> bytes:
    """ChaCha20 key of a workload: SHA-256 of the u64 seed in little-endian."""
    return hashlib.sha256(seed.to_bytes(8, "little")).digest()


def openssl_pub(seed: bytes) -> bytes:
    from cryptography.hazmat.primitives.asymmetric.ed25519 import Ed25519PrivateKey
    from cryptography.hazmat.primitives import serialization
    k = Ed25519PrivateKey.from_private_bytes(seed)
    return k.public_key().public_bytes(serialization.Encoding.Raw, serialization.PublicFormat.Raw)


def openssl_chacha(key: bytes, nbytes: int) -> bytes:
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    return Cipher(algorithms.ChaCha20(key, bytes(16)), mode=None).encryptor().update(bytes(nbytes))


def rfc_vectors():
    path = os.path.join(REF, "tests/data/rfc8032-ed25519.txt")
    out = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        name, sk, pk = line.strip().split(":")[:3]
        out.append({"name": name, "secret": sk, "public": pk})
    return out


REGEXES = [
    ("ab", True), ("[0-9]$", True), ("^[A-P]a", True), ("wa.o", False), ("(ab){2,}", True),
    ("zzzz|ofX", True), ("[0-9][A-F]x", False), ("a+b/c?", True), ("^[^A]", True), ("9$", True),
]


def main():
    refs = [po.RefKernel(p) for p in po.ref_variants()]
    if not refs:
        sys.exit("build the reference CPU kernel first: make -C oracle ref")
    ref = refs[0]
    lib = po.lib()

    # 1. RFC 8032 vectors: oracle and OpenSSL agree
    vec = rfc_vectors()
    for v in vec:
        sk = bytes.fromhex(v["secret"])
        assert po.pubkey(sk).hex() == v["public"], v["name"]
        assert openssl_pub(sk).hex() == v["public"], v["name"]
    json.dump(vec, open(os.path.join(HERE, "rfc8032.json"), "w"), indent=1)

    # 2. seeds: reference kernel, oracle and OpenSSL ChaCha20 agree
    key1 = chacha_key(1)
    ks = openssl_chacha(key1, 64 * 64)
    seeds = {}
    for i in list(range(16)) + [2**32 - 1, 2**32, 2**32 + 1, 2**33 + 5, 2**40 + 3, 2**63 + 9]:
        s_ref = ref.seed(key1, i)
        assert s_ref == po.seed(key1, 0, i), i
        if 32 * i + 32 <= len(ks):
            assert s_ref == ks[32 * i:32 * i + 32], i
        seeds[str(i)] = s_ref.hex()
    # counter seeds (src/model/search.rs:45-50): base with index added to the LE tail
    base = key1
    cseeds = {str(i): po.seed(base, 1, i).hex() for i in [0, 1, 255, 2**32, 2**64 - 1]}
    json.dump({"key": key1.hex(), "chacha20": seeds, "counter": cseeds},
              open(os.path.join(HERE, "seeds.json"), "w"), indent=1)

    # 3. public keys of indices 0..4095 (ChaCha20, key SHA-256(u64 1)) and 0..1023 (counter)
    width = 12
    table = po.ref_table(width)
    n_cha, n_cnt = 4096, 1024
    pk_ref = b"".join(ref.derive(table, width, key1, False, f) for f in range(0, n_cha, ref.batch))
    assert pk_ref == po.derive(key1, 0, 0, n_cha)
    for i in range(0, n_cha, 97):
        assert pk_ref[32 * i:32 * i + 32] == openssl_pub(ref.seed(key1, i))
    open(os.path.join(HERE, "pubkeys_chacha_key1_0_4096.bin"), "wb").write(pk_ref)
    pk_cnt = b"".join(ref.derive(table, width, key1, True, f) for f in range(0, n_cnt, ref.batch))
    assert pk_cnt == po.derive(key1, 1, 0, n_cnt)
    open(os.path.join(HERE, "pubkeys_counter_key1_0_1024.bin"), "wb").write(pk_cnt)
    # every variant of the reference build gives the same keys at high indices
    hi_first = 2**33 - 64
    hi = {}
    for r in refs:
        got = r.derive(table, width, key1, False, hi_first)[:32 * 16]
        assert got == po.derive(key1, 0, hi_first, 16)
        hi[os.path.basename(r.path)] = got.hex()
    # the small secure-path workload: all 2^20 keys from the reference build itself, equal to
    # the oracle's key for key; the GPU tests compare against the checksum of all of them
    from concurrent.futures import ThreadPoolExecutor
    n_full = 1 << 20
    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:  # ctypes releases the GIL
        full_ref = b"".join(ex.map(lambda f: ref.derive(table, width, key1, False, f), range(0, n_full, ref.batch)))
    full = po.derive(key1, 0, 0, n_full)
    assert full_ref == full
    digest = hashlib.sha256(full).hexdigest()
    assert full[:32 * n_cha] == pk_ref

    # 4. DFA tables: the builder agrees with Python `re` on random 43-character strings
    rng = random.Random(5)
    dfas = []
    for rx, cs in REGEXES:
        table_bytes, states = dfa_builder.build(rx, cs)
        pyre = dfa_builder.python_regex(rx, cs)
        for _ in range(3000):
            first = rng.randrange(16)
            vals = [first] + [rng.randrange(64) for _ in range(42)]
            text = bytes(dfa_builder.ALPHABET[v] for v in vals).decode()
            assert dfa_builder.run(table_bytes, states, vals) == bool(pyre.search(text)), (rx, text)
        dfas.append({"regex": rx, "case_sensitive": cs, "states": states, "table": table_bytes.hex()})

    # 5. candidate sets (y only, sign unknown) over indices 0..65535 from the reference's
    #    own matcher (contains_unsigned, kernel.cu:1804-1875) applied to its own keys
    n_search = 1 << 16
    pks = po.derive(key1, 0, 0, n_search)
    text_cases = [("ab", True, 0), ("Ab", False, 0), ("xyz", False, 0), ("a", True, 1), ("Q9", True, 1),
                  ("ke", False, 1), ("09", True, 0), ("+/", True, 0), ("wO", False, 0), ("K", False, 1)]
    search = []
    for needle, fold, mode in text_cases:
        nb = needle.lower().encode() if fold else needle.encode()
        hits = []
        for i in range(n_search):
            y = bytearray(pks[32 * i:32 * i + 32])
            y[31] &= 0x7F
            if ref.contains_unsigned(bytes(y), nb, len(nb), fold, mode):
                hits.append(i)
        want = po.search(key1, 0, 0, n_search, nb, len(nb), fold, mode)
        assert hits == want, needle
        search.append({"needle": needle, "fold": fold, "mode": mode, "hits": hits})
    for d in [dfas[k] for k in (0, 2, 3, 4, 5, 9)]:
        tb = bytes.fromhex(d["table"])
        hits = []
        for i in range(n_search):
            y = bytearray(pks[32 * i:32 * i + 32])
            y[31] &= 0x7F
            if ref.contains_unsigned(bytes(y), tb, d["states"], False, 2):
                hits.append(i)
        assert hits == po.search(key1, 0, 0, n_search, tb, d["states"], False, 2), d["regex"]
        search.append({"regex": d["regex"], "case_sensitive": d["case_sensitive"], "mode": 2, "hits": hits})

    meta = {
        "chacha_key_seed": 1,
        "chacha_key": key1.hex(),
        "sha256_of_pubkeys_0_2pow20": digest,
        "pubkeys_0_2pow20_from": os.path.basename(ref.path) + " (every key equal to the oracle's)",
        "pubkeys_high_first": hi_first,
        "pubkeys_high_by_reference_variant": hi,
        "search_range": [0, n_search],
        "search": search,
        "dfas": dfas,
        "reference_variants": [os.path.basename(r.path) for r in refs],
    }
    json.dump(meta, open(os.path.join(HERE, "golden.json"), "w"), indent=1)
    print("golden fixtures written; sha256(2^20 keys) =", digest)


if __name__ == "__main__":
    main()
