"""ctypes wrapper of the C oracle (liboracle.so) and of the reference kernel built for the CPU.

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's CPU-baseline
leg use this module as the checker; the product never imports it.
"""
import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    """Compile liboracle.so (and the reference CPU build when its sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    ref_src = os.environ.get("REF", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    if os.path.exists(os.path.join(ref_src, "src/service/gpu/kernel.cu")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_src}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        u8p, u32p, u64 = ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64
        sig = {
            "mko_init": (None, []),
            "mko_chacha20_block": (None, [u32p, u64, u32p]),
            "mko_chacha20_seed": (None, [u8p, u64, ctypes.c_void_p]),
            "mko_counter_seed": (None, [u8p, u64, ctypes.c_void_p]),
            "mko_seed": (None, [u8p, ctypes.c_uint32, u64, ctypes.c_void_p]),
            "mko_sha512": (None, [u8p, u64, ctypes.c_void_p]),
            "mko_secret_scalar": (None, [u8p, ctypes.c_void_p]),
            "mko_base_mul": (None, [u8p, ctypes.c_void_p]),
            "mko_pubkey_from_seed": (None, [u8p, ctypes.c_void_p]),
            "mko_point_affine": (None, [u8p, ctypes.c_void_p, ctypes.c_void_p]),
            "mko_derive": (None, [u8p, ctypes.c_uint32, u64, u64, ctypes.c_void_p]),
            "mko_incremental": (None, [u8p, u64, u64, ctypes.c_void_p]),
            "mko_public_b64": (None, [u8p, ctypes.c_void_p]),
            "mko_match": (ctypes.c_int, [u8p, u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
            "mko_search": (u64, [u8p, ctypes.c_uint32, u64, u64, u8p, ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_void_p, u64]),
            "mko_match_keys": (u64, [ctypes.c_void_p, u64, u64, u8p, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint32, ctypes.c_void_p, u64]),
            "mko_ref_table_words": (u64, [ctypes.c_uint32]),
            "mko_ref_table": (None, [ctypes.c_uint32, ctypes.c_void_p]),
            "mko_digits": (None, [u8p, ctypes.c_uint32, ctypes.c_void_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L.mko_init()
        _lib = L
    return _lib


def seed(key: bytes, source: int, index: int) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().mko_seed(key, source, index, out)
    return out.raw


def secret_scalar(seed_bytes: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().mko_secret_scalar(seed_bytes, out)
    return out.raw


def pubkey(seed_bytes: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().mko_pubkey_from_seed(seed_bytes, out)
    return out.raw


def base_mul(scalar: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().mko_base_mul(scalar, out)
    return out.raw


def point_affine(scalar: int):
    """(x, y) of scalar·B as integers (any 256-bit scalar)."""
    x = ctypes.create_string_buffer(32)
    y = ctypes.create_string_buffer(32)
    lib().mko_point_affine(scalar.to_bytes(32, "little"), x, y)
    return int.from_bytes(x.raw, "little"), int.from_bytes(y.raw, "little")


def public_b64(pk: bytes) -> str:
    out = ctypes.create_string_buffer(68)
    lib().mko_public_b64(pk, out)
    return out.raw.decode()


def match(pk: bytes, needle: bytes, length: int, fold: bool, mode: int, sign_unknown: bool) -> bool:
    return bool(lib().mko_match(pk, needle, length, int(fold), mode, int(sign_unknown)))


def _chunks(first, n, parts):
    step = max(1, (n + parts - 1) // parts)
    return [(first + i, min(step, n - i)) for i in range(0, n, step)]


def derive(key: bytes, source: int, first: int, n: int, threads: int = 0) -> bytes:
    """n full public keys; splits the range over threads (ctypes releases the GIL)."""
    threads = threads or os.cpu_count() or 1
    L = lib()
    out = ctypes.create_string_buffer(32 * n)
    base = ctypes.addressof(out)

    def run(a):
        f, cnt = a
        L.mko_derive(key, source, f, cnt, ctypes.c_void_p(base + 32 * (f - first)))

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, _chunks(first, n, threads * 4)))
    return out.raw


def search(key: bytes, source: int, first: int, n: int, needle: bytes, length: int, fold: bool, mode: int,
           threads: int = 0):
    """Sorted indices whose y-only key may match with either x sign (the GPU candidate set)."""
    threads = threads or os.cpu_count() or 1
    L = lib()

    def run(a):
        f, cnt = a
        cap = 1 << 16
        hits = (ctypes.c_uint64 * cap)()
        k = L.mko_search(key, source, f, cnt, needle, length, int(fold), mode, hits, cap)
        return [hits[i] for i in range(min(k, cap))]

    with ThreadPoolExecutor(threads) as ex:
        parts = list(ex.map(run, _chunks(first, n, threads * 4)))
    return sorted(i for p in parts for i in p)


def match_keys(pks: bytes, first: int, needle: bytes, length: int, fold: bool, mode: int):
    """Candidate indices among precomputed keys pks (index first + i for key i), sign unknown."""
    n = len(pks) // 32
    cap = n
    hits = (ctypes.c_uint64 * max(1, cap))()
    buf = ctypes.create_string_buffer(pks, len(pks))
    k = lib().mko_match_keys(buf, n, first, needle, length, int(fold), mode, hits, cap)
    return [hits[i] for i in range(min(k, cap))]


def ref_table(width: int):
    """The reference's packed comb table of width `width` (a ctypes u32 array)."""
    L = lib()
    words = L.mko_ref_table_words(width)
    buf = (ctypes.c_uint32 * words)()
    L.mko_ref_table(width, buf)
    return buf


def ref_variants():
    """Paths of the reference kernel compiled for the CPU (empty when it was not built)."""
    if not os.path.isdir(REF_DIR):
        return []
    return sorted(os.path.join(REF_DIR, f) for f in os.listdir(REF_DIR) if f.endswith(".so"))


class RefKernel:
    """The reference's own kernel source compiled as C++ (oracle/_ref), driven through
    its CPU test exports (src/service/gpu/kernel.cu:2083-2208)."""

    def __init__(self, path: str):
        self.path = path
        L = ctypes.CDLL(path)
        p = "meikey_test_"
        self.batch = getattr(L, p + "batch")()
        self.field = getattr(L, p + "field")()
        self._derive = getattr(L, p + "derive_batch")
        self._derive.restype = None
        self._derive.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                 ctypes.c_void_p]
        self._search = getattr(L, p + "search")
        self._search.restype = None
        self._search.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32,
                                 ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
        self._contains = getattr(L, p + "contains_unsigned")
        self._contains.restype = ctypes.c_int
        self._contains.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        self._seed = getattr(L, p + "seed")
        self._seed.restype = None
        self._seed.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        self._lib = L

    @staticmethod
    def key_words(key: bytes):
        return (ctypes.c_uint32 * 8)(*[int.from_bytes(key[4 * i:4 * i + 4], "little") for i in range(8)])

    def derive(self, table, width: int, key: bytes, counter: bool, first: int) -> bytes:
        """`batch` public keys starting at index `first`."""
        out = ctypes.create_string_buffer(32 * self.batch)
        self._derive(table, width, self.key_words(key), int(counter), first, out)
        return out.raw

    def seed(self, key: bytes, index: int) -> bytes:
        out = ctypes.create_string_buffer(32)
        self._seed(self.key_words(key), index, out)
        return out.raw

    def contains_unsigned(self, pk: bytes, needle: bytes, length: int, fold: bool, mode: int) -> bool:
        return bool(self._contains(pk, needle, length, int(fold), mode))

    def search(self, nthreads, table, width, key: bytes, counter: bool, needle: bytes, length: int, fold: bool,
               mode: int, base: int, iters: int, stop_on_hit: bool):
        """The reference's kernel emulated on the CPU: returns result[0..2] (flag, index)."""
        result = (ctypes.c_uint64 * 2)(0, 0)
        padded = needle + bytes(64)
        self._search(nthreads, table, width, self.key_words(key), int(counter), padded, length, int(fold), mode,
                     base, iters, int(stop_on_hit), result)
        return int(result[0]), int(result[1])
