"""mk_derive_noalloc: public keys through the entry point that allocates no device memory.

It exists for callers that cannot allocate device memory while they run (a serving
process that committed the device's memory to the comb table and job slots at start-up,
or a host framework whose own pool owns the device memory; cudaMalloc would also stall
every job sharing the GPU).  Its keys must equal mk_derive's bit for bit, including on a
second call that reuses the library's fixed device staging.  This file is collected last
so that a run stopping at the first failure has already run every other test."""
import hashlib

import pytest

import meikey_b200 as mk
from meikey_b200 import _lib

pytestmark = pytest.mark.gpu


def key_of(seed: int) -> bytes:
    return hashlib.sha256(seed.to_bytes(8, "little")).digest()


@pytest.fixture(scope="module")
def ctx():
    c = mk.Context(device=0, table_rows=16, keys_per_thread=16, block=512)
    yield c
    c.close()


def test_two_calls_in_a_row_match_derive(ctx):
    cases = [(key_of(1), mk.SEED_CHACHA20, 0, 4096),
             (key_of(2), mk.SEED_COUNTER, 2**33 + 1, 1000)]
    for key, source, first, n in cases:  # two calls in a row, on the same staging
        got = ctx.derive_noalloc(key, source, first, n)
        assert got == ctx.derive(key, source, first, n)


def test_largest_size_and_reuse(ctx):
    n = _lib.NOALLOC_MAX_KEYS
    a = ctx.derive_noalloc(key_of(3), mk.SEED_CHACHA20, 77, n)
    b = ctx.derive_noalloc(key_of(4), mk.SEED_CHACHA20, 5, 3)  # shorter call after a full one
    assert a == ctx.derive(key_of(3), mk.SEED_CHACHA20, 77, n)
    assert b == ctx.derive(key_of(4), mk.SEED_CHACHA20, 5, 3)


def test_matches_golden_keys_and_oracle(ctx, golden_pubkeys, oracle):
    """Against fixtures and the oracle, not only mk_derive: the golden ChaCha20 keys 0..4095
    (pinned by OpenSSL and the reference build), then counter seeds whose indices run past
    the top of the 64-bit index space (the seed tail wraps), twice in a row."""
    cha, cnt = golden_pubkeys
    assert ctx.derive_noalloc(key_of(1), mk.SEED_CHACHA20, 0, 4096) == cha
    assert ctx.derive_noalloc(key_of(1), mk.SEED_COUNTER, 0, 1024) == cnt
    first, n = 2**64 - 100, 200
    for _ in range(2):
        got = ctx.derive_noalloc(key_of(5), mk.SEED_COUNTER, first, n)
        assert got == oracle.derive(key_of(5), mk.SEED_COUNTER, first, n)


def test_incremental_source_is_rejected(ctx):
    with pytest.raises(mk.GpuError) as e:
        ctx.derive_noalloc(bytes(31) + b"\x40", mk.SEED_INCREMENTAL, 0, 16)
    assert e.value.status == _lib.ERR_BAD_ARG


def test_oversize_is_rejected(ctx):
    with pytest.raises(mk.GpuError) as e:
        ctx.derive_noalloc(key_of(1), mk.SEED_CHACHA20, 0, _lib.NOALLOC_MAX_KEYS + 1)
    assert e.value.status == _lib.ERR_OUT_OF_RANGE
