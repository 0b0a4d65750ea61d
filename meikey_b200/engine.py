"""Host-side mirror of the reference's GPU engine (src/service/gpu.rs:806-887).

``Context`` corresponds to a loaded ``Kernel`` (comb table on the device, launch grid),
``Job`` to the ``Launch`` returned by ``Engine::prepare``; ``Job.launch`` is
``Engine::launch``.  Everything runs through the C ABI of libmeikey_b200.so.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

from . import _lib as L


class GpuError(RuntimeError):
    """A non-OK status from the library (the reference's GpuError, src/service/gpu.rs:444-499)."""

    def __init__(self, status: int, message: str = ""):
        self.status = status
        name = L.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {message}" if message else name)


@dataclass(frozen=True)
class Needle:
    """One pattern as the GPU receives it (src/service/gpu.rs:618-660).

    ``mode`` 0 contains, 1 suffix (``text`` are base64 characters; lowercase when
    ``fold``), 2 regex (``text`` is a DFA table of ``states`` × 65 little-endian u16).
    """
    text: bytes
    mode: int = L.MODE_CONTAINS
    fold: bool = False
    states: int = 0

    @staticmethod
    def contains(s: str, case_sensitive: bool = True) -> "Needle":
        return Needle(s.encode() if case_sensitive else s.lower().encode(), L.MODE_CONTAINS, not case_sensitive)

    @staticmethod
    def suffix(s: str, case_sensitive: bool = True) -> "Needle":
        return Needle(s.encode() if case_sensitive else s.lower().encode(), L.MODE_SUFFIX, not case_sensitive)

    @staticmethod
    def dfa(table: bytes, states: int) -> "Needle":
        return Needle(bytes(table), L.MODE_REGEX, False, states)

    def c_len(self) -> int:
        return self.states if self.mode == L.MODE_REGEX else len(self.text)


def _check(lib, ctx_ptr, status: int):
    if status != L.OK:
        buf = ctypes.create_string_buffer(512)
        lib.mk_last_error(ctx_ptr, buf, 512)
        raise GpuError(status, buf.value.decode(errors="replace"))


class Context:
    """A device with the comb table built on it (Gpu::new / Kernel::load)."""

    def __init__(self, device: int = 0, table_rows: int = 12, keys_per_thread: int = 16, block: int = 512,
                 blocks_per_sm: int = 0, self_check: bool = False, hit_capacity: int = 0):
        self._lib = L.load()
        opts = L.Options(table_rows, keys_per_thread, block, blocks_per_sm, 1 if self_check else 0, hit_capacity)
        ptr = ctypes.c_void_p()
        st = self._lib.mk_ctx_create(device, ctypes.byref(opts), ctypes.byref(ptr))
        self._ptr = ptr
        if st != L.OK:
            buf = ctypes.create_string_buffer(512)
            self._lib.mk_last_error(ptr, buf, 512)
            if ptr:
                self._lib.mk_ctx_destroy(ptr)
            self._ptr = ctypes.c_void_p()
            raise GpuError(st, buf.value.decode(errors="replace"))
        info = L.InfoC()
        _check(self._lib, self._ptr, self._lib.mk_ctx_info(self._ptr, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in L.InfoC._fields_}
        self.info["name"] = info.name.decode(errors="replace")

    @property
    def keys_per_iter(self) -> int:
        return int(self._lib.mk_keys_per_iter(self._ptr))

    def derive(self, key: bytes, source: int, first: int, n: int) -> bytes:
        """n full public keys (32 bytes each) of indices first..first+n-1."""
        out = ctypes.create_string_buffer(32 * n)
        _check(self._lib, self._ptr, self._lib.mk_derive(self._ptr, bytes(key), source, first, n, out))
        return out.raw

    def derive_noalloc(self, key: bytes, source: int, first: int, n: int) -> bytes:
        """As derive, through the entry point that allocates no device memory (n <= 65536).

        For callers that must not allocate device memory mid-run (a serving process whose
        device memory is committed at start-up, or one whose memory a host framework's pool
        owns); the first call on a device should come before any stream capture, and calls
        that overlap on the GPU share, and race on, the library's fixed staging array."""
        out = ctypes.create_string_buffer(32 * n)
        _check(self._lib, self._ptr, self._lib.mk_derive_noalloc(self._ptr, bytes(key), source, first, n, out))
        return out.raw

    def table_entry(self, row: int, col: int) -> List[int]:
        out = (ctypes.c_uint32 * 24)()
        _check(self._lib, self._ptr, self._lib.mk_table_entry(self._ptr, row, col, out))
        return list(out)

    def job(self, key: bytes, source: int, needles: Sequence[Needle], stop_on_hit: bool = False) -> "Job":
        return Job(self, key, source, needles, stop_on_hit)

    def work_per_key(self, source: int = L.SEED_CHACHA20):
        """(field multiplications, 32-bit integer MADs) per key of the search kernel for a seed source."""
        fm, im = ctypes.c_double(), ctypes.c_double()
        _check(self._lib, self._ptr, self._lib.mk_ctx_work_per_key(self._ptr, source, ctypes.byref(fm),
                                                                   ctypes.byref(im)))
        return fm.value, im.value

    def measure_mad_peaks(self):
        """(carry-chain row MADs/s, plain mad.lo MADs/s) of the device (bounded microbenchmarks)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(self._lib, self._ptr, self._lib.mk_measure_mad_peaks(self._ptr, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def sync(self):
        _check(self._lib, self._ptr, self._lib.mk_ctx_sync(self._ptr))

    def record(self, slot: int):
        _check(self._lib, self._ptr, self._lib.mk_ctx_record(self._ptr, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        _check(self._lib, self._ptr, self._lib.mk_ctx_elapsed(self._ptr, a, b, ctypes.byref(ms)))
        return float(ms.value)

    def close(self):
        if self._ptr:
            self._lib.mk_ctx_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _needle_array(needles: Sequence[Needle]):
    """(mk_needle array, buffers to keep alive) for a list of needles."""
    arr = (L.NeedleC * max(1, len(needles)))()
    keep = []
    for i, n in enumerate(needles):
        buf = (ctypes.c_uint8 * max(1, len(n.text))).from_buffer_copy(n.text if n.text else b"\0")
        keep.append(buf)
        arr[i] = L.NeedleC(ctypes.cast(buf, ctypes.POINTER(ctypes.c_uint8)), n.c_len(), int(n.fold), n.mode)
    return arr, keep


class Job:
    """Key + needles + hit ring on the device (the reference's ``Launch``)."""

    def __init__(self, ctx: Context, key: bytes, source: int, needles: Sequence[Needle], stop_on_hit: bool = False):
        if len(key) != 32:
            raise ValueError("key must be 32 bytes")
        self.ctx = ctx
        self._lib = ctx._lib
        self.needles = list(needles)
        arr, self._keep = _needle_array(self.needles)
        ptr = ctypes.c_void_p()
        _check(self._lib, ctx._ptr, self._lib.mk_job_prepare(ctx._ptr, bytes(key), source, arr, len(self.needles),
                                                             1 if stop_on_hit else 0, ctypes.byref(ptr)))
        self._ptr = ptr

    def launch(self, base: int, iters: int) -> Optional[int]:
        """Engine::launch: the lowest candidate index of base .. base+keys_per_iter·iters-1, or None."""
        found = ctypes.c_int()
        idx = ctypes.c_uint64()
        st = self._lib.mk_job_launch(self._ptr, base, iters, ctypes.byref(found), ctypes.byref(idx))
        if st not in (L.OK, L.ERR_STOPPED):
            _check(self._lib, self.ctx._ptr, st)
        return int(idx.value) if found.value else None

    def hits(self, cap: int = 1 << 16) -> Tuple[List[Tuple[int, int]], int]:
        """Candidate hits (index, needle) of the last launch, sorted, and the total count."""
        out = (L.HitC * cap)()
        written, total = ctypes.c_uint32(), ctypes.c_uint64()
        st = self._lib.mk_job_hits(self._ptr, out, cap, ctypes.byref(written), ctypes.byref(total))
        if st not in (L.OK, L.ERR_HIT_RING_FULL):
            _check(self._lib, self.ctx._ptr, st)
        return [(int(out[i].index), int(out[i].needle)) for i in range(written.value)], int(total.value)

    def update(self, needles: Sequence[Needle]):
        """Replace the needles between launches (hits then carry positions in the new list)."""
        self.needles = list(needles)
        arr, self._keep = _needle_array(self.needles)
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_update(self._ptr, arr, len(self.needles)))

    def graph(self, iters: int, launches: int) -> "Graph":
        """A CUDA graph of `launches` launches of `iters` iterations each (mk_job_graph_create)."""
        return Graph(self, iters, launches)

    def confirm(self, index: int, needle: int):
        """Host confirmation of a candidate: (matched, public key, secret).  The secret is the
        seed (ChaCha20 / counter sources) or the scalar s0 + index (incremental source)."""
        pk = ctypes.create_string_buffer(32)
        secret = ctypes.create_string_buffer(32)
        ok = ctypes.c_int()
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_confirm(self._ptr, index, needle, pk, secret,
                                                                  ctypes.byref(ok)))
        return bool(ok.value), pk.raw, secret.raw

    def io_bytes(self):
        """(host->device, device->host) bytes this job has copied so far."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_io_bytes(self._ptr, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def enqueue(self, base: int, iters: int):
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_enqueue(self._ptr, base, iters))

    def close(self):
        if self._ptr:
            self._lib.mk_job_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A job's consecutive launches captured as one CUDA graph (mk_job_graph_create)."""

    def __init__(self, job: Job, iters: int, launches: int):
        self.job = job
        self._lib = job._lib
        self.span = job.ctx.keys_per_iter * iters * launches
        ptr = ctypes.c_void_p()
        _check(self._lib, job.ctx._ptr, self._lib.mk_job_graph_create(job._ptr, iters, launches, ctypes.byref(ptr)))
        self._ptr = ptr

    def launch(self, base: int) -> Optional[int]:
        """Replays the graph over base .. base + span - 1; the lowest candidate index or None."""
        found = ctypes.c_int()
        idx = ctypes.c_uint64()
        st = self._lib.mk_graph_launch(self._ptr, base, ctypes.byref(found), ctypes.byref(idx))
        if st not in (L.OK, L.ERR_STOPPED):
            _check(self._lib, self.job.ctx._ptr, st)
        return int(idx.value) if found.value else None

    def enqueue(self, base: int):
        _check(self._lib, self.job.ctx._ptr, self._lib.mk_graph_enqueue(self._ptr, base))

    def close(self):
        if self._ptr:
            self._lib.mk_graph_destroy(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
