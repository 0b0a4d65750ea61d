import hashlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def chacha_key(seed: int) -> bytes:
    """ChaCha20 key of the synthetic workloads: SHA-256 of the u64 seed, little-endian."""
    return hashlib.sha256(seed.to_bytes(8, "little")).digest()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_pubkeys():
    with open(os.path.join(GOLDEN, "pubkeys_chacha_key1_0_4096.bin"), "rb") as f:
        cha = f.read()
    with open(os.path.join(GOLDEN, "pubkeys_counter_key1_0_1024.bin"), "rb") as f:
        cnt = f.read()
    return cha, cnt


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_ctx():
    """A context with the default comb geometry on cuda:0 (built once per session)."""
    import meikey_b200 as mk
    ctx = mk.Context(device=0, table_rows=12, keys_per_thread=8, self_check=True, hit_capacity=1 << 18)
    yield ctx
    ctx.close()
