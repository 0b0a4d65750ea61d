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

    @staticmethod
    def regex(pattern: str, case_sensitive: bool = True, max_states: int = 16384, device: "Context" = None) -> "Needle":
        """A regex needle compiled by the library (mk_regex_compile); max_states defaults to the
        reference's limit (MAX_STATES, src/model/pattern/dfa.rs:18).  With a context as `device`
        the subset construction runs on its GPU (mk_regex_compile_device, the same table)."""
        lib = L.load()
        table = ctypes.create_string_buffer(max_states * 130)
        states = ctypes.c_uint32()
        err = ctypes.create_string_buffer(256)
        if device is None:
            st = lib.mk_regex_compile(pattern.encode(), 1 if case_sensitive else 0, max_states, table,
                                      ctypes.byref(states), err, 256)
        else:
            st = lib.mk_regex_compile_device(device._ptr, pattern.encode(), 1 if case_sensitive else 0, max_states,
                                             table, ctypes.byref(states), err, 256)
        if st != L.OK:
            msg = err.value.decode(errors="replace")
            if not msg and device is not None:
                buf = ctypes.create_string_buffer(512)
                lib.mk_last_error(device._ptr, buf, 512)
                msg = buf.value.decode(errors="replace")
            raise GpuError(st, msg)
        return Needle.dfa(table.raw[:states.value * 130], states.value)

    def c_len(self) -> int:
        return self.states if self.mode == L.MODE_REGEX else len(self.text)

    def expected_tries(self) -> float:
        """1 / probability that a random key matches (mk_expected_tries)."""
        arr, keep = _needle_array([self])
        return float(L.load().mk_expected_tries(arr))


def _outcome(out) -> dict:
    return {"status": out.status, "found": out.status == L.OK, "index": int(out.index), "needle": int(out.needle),
            "tries": int(out.tries), "elapsed_s": float(out.elapsed_s), "secret": bytes(out.secret),
            "pk": bytes(out.pk)}


def _progress_fn(progress):
    return L.PROGRESS_FN((lambda user, tries, el: 1 if progress(int(tries), float(el)) else 0)
                         if progress else (lambda user, tries, el: 0))


def search_many(jobs, first, max_tries=0, iters=16, time_limit_s=0.0, progress=None) -> dict:
    """Searcher::run over several jobs, one host thread each (mk_search_many, the reference's
    All): `first` and `max_tries` are one value for all jobs or one per job; the first key
    found stops the others.  Returns the winner's outcome with `winner` (len(jobs): none)."""
    n = len(jobs)
    firsts = first if isinstance(first, (list, tuple)) else [first] * n
    budgets = max_tries if isinstance(max_tries, (list, tuple)) else [max_tries] * n
    cfgs = (L.SearchConfigC * n)(*[L.SearchConfigC(f, m, time_limit_s, iters, 0) for f, m in zip(firsts, budgets)])
    ptrs = (ctypes.c_void_p * n)(*[j._ptr.value for j in jobs])
    out = L.OutcomeC()
    who = ctypes.c_uint32()
    lib = jobs[0]._lib
    _check(lib, jobs[0].ctx._ptr, lib.mk_search_many(ptrs, n, cfgs, _progress_fn(progress), None, ctypes.byref(out),
                                                     ctypes.byref(who)))
    return dict(_outcome(out), winner=int(who.value))


def _check(lib, ctx_ptr, status: int):
    if status != L.OK:
        buf = ctypes.create_string_buffer(512)
        lib.mk_last_error(ctx_ptr, buf, 512)
        raise GpuError(status, buf.value.decode(errors="replace"))


class Context:
    """A device with the comb table built on it (Gpu::new / Kernel::load)."""

    def __init__(self, device: int = 0, table_rows: int = 12, keys_per_thread: int = 16, block: int = 512,
                 blocks_per_sm: int = 0, self_check: bool = False, hit_capacity: int = 0, hash_warps: int = 0,
                 inverter_rotates: bool = False, inversion_batch: int = 0, table_in_smem: bool = False,
                 hash_interleave: bool = False):
        self._lib = L.load()
        opts = L.Options(table_rows, keys_per_thread, block, blocks_per_sm, 1 if self_check else 0, hit_capacity,
                         hash_warps, 1 if inverter_rotates else 0, inversion_batch, 1 if table_in_smem else 0,
                         1 if hash_interleave else 0)
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

    def measure_imad_rates(self) -> dict:
        """MADs/s of the field multiply's instruction pieces on independent chains (mad.hi,
        mad.wide) and in carry-linked rows (madc.lo.cc, madc.hi.cc): mk_measure_imad_rates."""
        v = [ctypes.c_double() for _ in range(4)]
        _check(self._lib, self._ptr, self._lib.mk_measure_imad_rates(self._ptr, *[ctypes.byref(x) for x in v]))
        return {"mad_hi": v[0].value, "mad_wide": v[1].value, "madc_lo_chain": v[2].value, "madc_hi_chain": v[3].value}

    def measure_field_mul(self):
        """(radix-2^32, radix-2^25.5, radix-2^51 FP64) field multiplications per second of the
        device; raises if the FP64 radix's products differ from radix 2^32's."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self._lib, self._ptr,
               self._lib.mk_measure_field_mul(self._ptr, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def field_mul_pairs(self, a: Sequence[int], b: Sequence[int]):
        """(schoolbook, karatsuba) lists of the device's a[i]·b[i] mod p for integers below 2^256,
        as the kernels leave them (below 2^256, congruent, not canonical): mk_field_mul_pairs."""
        n = len(a)
        assert n == len(b) and n > 0
        ina = (ctypes.c_uint32 * (8 * n))(*[(x >> (32 * w)) & 0xffffffff for x in a for w in range(8)])
        inb = (ctypes.c_uint32 * (8 * n))(*[(x >> (32 * w)) & 0xffffffff for x in b for w in range(8)])
        outs, outk = (ctypes.c_uint32 * (8 * n))(), (ctypes.c_uint32 * (8 * n))()
        _check(self._lib, self._ptr, self._lib.mk_field_mul_pairs(self._ptr, ina, inb, n, outs, outk))
        val = lambda arr, i: sum(arr[8 * i + w] << (32 * w) for w in range(8))
        return [val(outs, i) for i in range(n)], [val(outk, i) for i in range(n)]

    def measure_field_mul_forms(self):
        """{"schoolbook": ..., "karatsuba": ...} radix-2^32 field multiplications per second;
        raises if the two forms' products differ."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(self._lib, self._ptr, self._lib.mk_measure_field_mul_forms(self._ptr, ctypes.byref(a), ctypes.byref(b)))
        return {"schoolbook": a.value, "karatsuba": b.value}

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

    def search(self, first: int = 0, max_tries: int = 0, iters: int = 16, time_limit_s: float = 0.0,
               progress=None) -> dict:
        """Searcher::run (mk_search): the lowest host-confirmed match from `first`, or status
        STOPPED after max_tries indices, the time limit, or `progress(tries, elapsed)` returning
        True (checked between launches)."""
        cfg = L.SearchConfigC(first, max_tries, time_limit_s, iters, 0)
        out = L.OutcomeC()
        cb = L.PROGRESS_FN((lambda user, tries, el: 1 if progress(int(tries), float(el)) else 0)
                           if progress else (lambda user, tries, el: 0))
        _check(self._lib, self.ctx._ptr, self._lib.mk_search(self._ptr, ctypes.byref(cfg), cb, None, ctypes.byref(out)))
        return {"status": out.status, "found": out.status == L.OK, "index": int(out.index), "needle": int(out.needle),
                "tries": int(out.tries), "elapsed_s": float(out.elapsed_s), "secret": bytes(out.secret),
                "pk": bytes(out.pk)}

    def search_both(self, first: int = 0, max_tries: int = 0, iters: int = 16, time_limit_s: float = 0.0,
                    cpu_threads: int = 1, cpu_first: int = 1 << 62, progress=None) -> dict:
        """The GPU and `cpu_threads` host threads searching together (mk_search_both, the
        reference's Both): the first key either side finds; `winner` 0 GPU, 1 host, 2 none."""
        cfg = L.SearchConfigC(first, max_tries, time_limit_s, iters, 0)
        out = L.OutcomeC()
        who = ctypes.c_uint32()
        cb = _progress_fn(progress)
        _check(self._lib, self.ctx._ptr, self._lib.mk_search_both(self._ptr, ctypes.byref(cfg), cpu_threads, cpu_first,
                                                                  cb, None, ctypes.byref(out), ctypes.byref(who)))
        return dict(_outcome(out), winner=int(who.value))

    def stop(self, on: bool = True):
        """Request (or withdraw) a stop of this job's launches, also of one that is running."""
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_stop(self._ptr, 1 if on else 0))

    def collect(self) -> Optional[int]:
        """Waits for the job's queued launches and reads their hits (like launch, without launching)."""
        found = ctypes.c_int()
        idx = ctypes.c_uint64()
        st = self._lib.mk_job_collect(self._ptr, ctypes.byref(found), ctypes.byref(idx))
        if st not in (L.OK, L.ERR_STOPPED, L.ERR_HIT_RING_FULL):
            _check(self._lib, self.ctx._ptr, st)
        return int(idx.value) if found.value else None

    def first_matches(self) -> List[Optional[dict]]:
        """Per needle, the lowest host-confirmed key among the last launch's candidates, or None."""
        n = len(self.needles)
        out = (L.OutcomeC * max(1, n))()
        _check(self._lib, self.ctx._ptr, self._lib.mk_job_first_matches(self._ptr, out, n))
        return [{"index": int(out[k].index), "pk": bytes(out[k].pk), "secret": bytes(out[k].secret)}
                if out[k].status == L.OK else None for k in range(n)]

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


# keys/thread x block variants the library is built for
BUILT_VARIANTS = [(4, 256), (8, 256), (16, 256), (4, 512), (8, 512), (16, 512)]


def compute_threads(block: int, hash_warps: int = 0, inverter_rotates: int = 0) -> int:
    """Threads of a search CTA that derive keys."""
    return 352 if hash_warps else block if inverter_rotates else block - 32


def inversion_batches(keys_per_thread: int, block: int, hash_warps: int = 0, inverter_rotates: int = 0,
                      lo: int = 64, hi: int = 512):
    """The inversion batches in [lo, hi] a layout can run: keys per thread x compute threads /
    pools, for pool counts that divide the compute threads and are at most 32."""
    ct = compute_threads(block, hash_warps, inverter_rotates)
    return sorted({keys_per_thread * ct // p for p in range(1, 33)
                   if ct % p == 0 and lo <= keys_per_thread * ct // p <= hi})


def tune_space(rows=(11, 12, 13, 14, 16), variants=BUILT_VARIANTS, blocks_per_sm=(0,), hash_warps=(0, 4),
               inverter_rotates=(0,), inversion_batch=(0,), table_in_smem=(0,)):
    """Candidate options: comb rows (table size against multiplications per key) x keys per
    thread and block x CTAs per SM x the hashing-warp layout (built for block 512, keys per
    thread 8 and 16) x who inverts (a dedicated warp, or a duty rotating over four key warps;
    not with hashing warps) x the inversion batch (keys per field inversion; 0 = 32 pools,
    "all" = every batch of 64..512 the layout can run)."""
    out = []
    for r in rows:
        for (k, b) in variants:
            for s in blocks_per_sm:
                for h in hash_warps:
                    for v in inverter_rotates:
                        if not (h == 0 or (b == 512 and k in (8, 16))) or (h and v):
                            continue
                        batches = inversion_batches(k, b, h, v) if inversion_batch == "all" else inversion_batch
                        for ib in batches:
                            for t in table_in_smem:
                                # the shared-memory table: dedicated inverter, block 512, 4 or 8 keys
                                if t and (h or v or b != 512 or k not in (4, 8)):
                                    continue
                                out.append(dict(table_rows=r, keys_per_thread=k, block=b, blocks_per_sm=s,
                                                hash_warps=h, inverter_rotates=v, inversion_batch=ib,
                                                table_in_smem=t))
    return out


def autotune(device: int = 0, candidates=None, finalists: int = 3, trial_keys: int = 1 << 27,
             job: Optional[Tuple[bytes, int, Sequence[Needle]]] = None):
    """Runs mk_autotune, or mk_autotune_job when `job` = (key, seed source, needles) gives the
    workload to time; returns (best options dict, per-candidate results)."""
    lib = L.load()
    cands = candidates or tune_space()
    arr = (L.TuneEntryC * len(cands))()
    for i, c in enumerate(cands):
        arr[i].options = L.Options(c["table_rows"], c["keys_per_thread"], c["block"], c.get("blocks_per_sm", 0), 1, 0,
                                   c.get("hash_warps", 0), c.get("inverter_rotates", 0), c.get("inversion_batch", 0),
                                   c.get("table_in_smem", 0), c.get("hash_interleave", 0))
    best = ctypes.c_uint32()
    if job is None:
        st = lib.mk_autotune(device, arr, len(cands), finalists, trial_keys, ctypes.byref(best))
    else:
        key, source, needles = job
        narr, keep = _needle_array(list(needles))
        st = lib.mk_autotune_job(device, arr, len(cands), finalists, trial_keys, bytes(key), source, narr,
                                 len(needles), ctypes.byref(best))
    if st != L.OK:
        raise GpuError(st, "autotune")
    results = [dict(cands[i], status=arr[i].status, stage=arr[i].stage, keys_per_s=arr[i].keys_per_s)
               for i in range(len(cands))]
    return dict(cands[best.value]), results


class Server:
    """Continuous batching of many jobs over one candidate stream (mk_server_*)."""

    def __init__(self, ctx: Context, key: bytes, source: int = L.SEED_CHACHA20, max_jobs: int = 64,
                 iters_per_tick: int = 8, budget: int = 1 << 26, hit_capacity: int = 0, first: int = 0,
                 device_bytes: int = 0):
        self.ctx = ctx
        self._lib = ctx._lib
        opts = L.ServerOptionsC(max_jobs, iters_per_tick, budget, hit_capacity, device_bytes)
        ptr = ctypes.c_void_p()
        _check(self._lib, ctx._ptr, self._lib.mk_server_create(ctx._ptr, bytes(key), source, ctypes.byref(opts), first,
                                                               ctypes.byref(ptr)))
        self._ptr = ptr

    def submit(self, needle: Needle, job_id: int):
        arr, keep = _needle_array([needle])
        _check(self._lib, self.ctx._ptr, self._lib.mk_server_submit(self._ptr, arr, job_id))

    def tick(self):
        """One launch for all admitted jobs; returns (active, queued) after it."""
        a, q = ctypes.c_uint32(), ctypes.c_uint32()
        _check(self._lib, self.ctx._ptr, self._lib.mk_server_tick(self._ptr, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def results(self) -> List[dict]:
        out = (L.JobResultC * 256)()
        n = ctypes.c_uint32()
        res = []
        while True:
            _check(self._lib, self.ctx._ptr, self._lib.mk_server_results(self._ptr, out, 256, ctypes.byref(n)))
            for i in range(n.value):
                r = out[i]
                res.append({"id": int(r.id), "found": r.status == L.OK, "status": r.status,
                            "admit_index": int(r.admit_index), "index": int(r.index), "tries": int(r.tries),
                            "expected_tries": float(r.expected_tries), "secret": bytes(r.secret), "pk": bytes(r.pk)})
            if n.value < 256:
                return res

    @property
    def position(self) -> int:
        return int(self._lib.mk_server_position(self._ptr))

    def close(self):
        if self._ptr:
            self._lib.mk_server_destroy(self._ptr)
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


def openssh_public(pk: bytes, comment: str = "") -> str:
    """authorized_keys line of a public key (mk_openssh_public)."""
    lib = L.load()
    buf = ctypes.create_string_buffer(256 + 4 * len(comment.encode()))
    n = ctypes.c_size_t()
    st = lib.mk_openssh_public(bytes(pk), comment.encode(), buf, len(buf), ctypes.byref(n))
    if st != L.OK:
        raise GpuError(st, "openssh public line")
    return buf.value.decode()


def openssh_private(seed: bytes, comment: str = "", checkint: int = 0) -> str:
    """Unencrypted openssh-key-v1 private key file of a seed (mk_openssh_private)."""
    lib = L.load()
    buf = ctypes.create_string_buffer(1024 + 4 * len(comment.encode()))
    n = ctypes.c_size_t()
    st = lib.mk_openssh_private(bytes(seed), comment.encode(), checkint, buf, len(buf), ctypes.byref(n))
    if st != L.OK:
        raise GpuError(st, "openssh private key")
    return buf.value.decode()
