"""Benchmark of the candidate-key search path (one JSON line on rank 0).

Headline (the reference's throughput configuration, synthetic inputs): secure-path seeds
from ChaCha20 with key SHA-256(u64 7 little-endian), a case-sensitive 7-character contains
needle drawn uniformly from the base64 alphabet with numpy.random.default_rng(7), inversion
batched over 256 keys, 2^34 candidates in total.  A step is one launch over >= 2^30
consecutive candidate indices; the default 16 steps cover 2^34.

On one GPU the same line carries `workloads`, one record each (value, clocks, roofline, e2e)
for the other configurations:
  counter      the reference's published GPU mode: low-security counter seeds, needle TARGET
               case-insensitive (8 steps of 2^30);
  incremental  P_k = P_0 + k·B from s0 = clamp(SHA-512(ChaCha20 seed 0 of key SHA-256(u64
               11))), a case-sensitive 6-character suffix (numpy.random.default_rng(11)),
               2^32 candidates (16 steps of 2^28);
  multi        64 text patterns and 8 regexes in one job, each step a CUDA-graph replay of 4
               launches, 2^34 candidates;
  serving      1000 Poisson-arriving jobs through continuous batching against one job at a
               time (p50/p99 time to key).
--workload <name> measures one of them as the headline; --headline-only skips the others.

Multi-GPU: one process per GPU (torchrun), each rank searches its own index range
(rank·2^56 ...), so the work is weakly scaled with no data-path collective; timing is the
max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload secure|counter|incremental|multi|serving] [--headline-only]
"""
import argparse
import hashlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "keys/s on 1 B200 (bit-exact pubkeys), % int-MAD peak; multi-job p50/p99"
UNIT = "keys/s"
ALPHABET = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/"
# per workload: total candidates, candidates per step, seed source, generator seed, needle length, mode
WORKLOADS = {
    "secure": {"total": 1 << 34, "step": 1 << 30, "source": 0, "seed": 7, "length": 7, "mode": "contains",
               "inversion_batch": 256},
    # the reference's published GPU mode (docs/benchmark.md): low-security counter seeds, the
    # needle TARGET case-insensitive
    "counter": {"total": 1 << 33, "step": 1 << 30, "source": 1, "seed": 7, "length": 0, "mode": "contains_ci",
                "needle": "TARGET", "kpt": 8},
    "incremental": {"total": 1 << 32, "step": 1 << 28, "source": 2, "seed": 11, "length": 6, "mode": "suffix"},
    "multi": {"total": 1 << 34, "step": 1 << 30, "source": 0, "seed": 23, "length": 0, "mode": "mixed",
              "launches": 4, "inverter_rotates": True, "kpt": 16, "inversion_batch": 256},
    "serving": {"total": 0, "step": 0, "source": 0, "seed": 31, "length": 0, "mode": "mixed", "jobs": 1000,
                "rate": 50.0, "budget": 1 << 26, "iters_per_tick": 8, "device_bytes": 32 << 20},
}


def serving_jobs(n=1000, rate=50.0, seed=31):
    """Poisson arrivals (exponential gaps, mean 1/rate s) from numpy.random.default_rng(seed);
    pattern length uniform in 4..8 over the base64 alphabet; mode uniform over case-sensitive
    contains, case-sensitive suffix and case-insensitive contains."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        length = int(rng.integers(4, 9))
        text = "".join(ALPHABET[int(v)] for v in rng.integers(0, 64, length))
        out.append((t, text, ("contains", "suffix", "contains_ci")[int(rng.integers(0, 3))]))
    return out

# the multi-pattern workload's regexes: DFAs of 6..57 states (mk_regex_compile), each matching
# a random key with probability 2e-7 .. 1.4e-4 (exact, by propagating a uniform character
# distribution through the DFA), 4.1e-4 together
MULTI_REGEXES = ["(ab|cd|ef)[+/]x", "(?:aa|bb)(?:cc|dd)$", "x.{2}y.{2}z", "(?:ab|ba).{2}[0-9]{2}$",
                 "z[0-9]{3}z", "(?:xyz|XYZ)$", "(?:AA|BB|CC)[0-9]{3}", "[ab].{4}[cd]z[0-9]"]


def multi_patterns():
    """64 text patterns: length uniform in 3..9 and characters uniform over the base64 alphabet
    from numpy.random.default_rng(23); mode uniform over case-sensitive contains,
    case-sensitive suffix and case-insensitive contains."""
    import numpy as np
    rng = np.random.default_rng(23)
    out = []
    for _ in range(64):
        n = int(rng.integers(3, 10))
        text = "".join(ALPHABET[int(v)] for v in rng.integers(0, 64, n))
        out.append((text, ("contains", "suffix", "contains_ci")[int(rng.integers(0, 3))]))
    return out


def chacha20_seed0(key: bytes) -> bytes:
    """The first 32 bytes of the ChaCha20 keystream (RFC 8439 block 0, nonce 0)."""
    def rotl(x, n):
        return ((x << n) | (x >> (32 - n))) & 0xFFFFFFFF

    def qr(s, a, b, c, d):
        s[a] = (s[a] + s[b]) & 0xFFFFFFFF; s[d] = rotl(s[d] ^ s[a], 16)
        s[c] = (s[c] + s[d]) & 0xFFFFFFFF; s[b] = rotl(s[b] ^ s[c], 12)
        s[a] = (s[a] + s[b]) & 0xFFFFFFFF; s[d] = rotl(s[d] ^ s[a], 8)
        s[c] = (s[c] + s[d]) & 0xFFFFFFFF; s[b] = rotl(s[b] ^ s[c], 7)
    init = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574]
    init += [int.from_bytes(key[4 * i:4 * i + 4], "little") for i in range(8)] + [0, 0, 0, 0]
    s = list(init)
    for _ in range(10):
        qr(s, 0, 4, 8, 12); qr(s, 1, 5, 9, 13); qr(s, 2, 6, 10, 14); qr(s, 3, 7, 11, 15)
        qr(s, 0, 5, 10, 15); qr(s, 1, 6, 11, 12); qr(s, 2, 7, 8, 13); qr(s, 3, 4, 9, 14)
    return b"".join(((s[i] + init[i]) & 0xFFFFFFFF).to_bytes(4, "little") for i in range(8))


def workload_key(name: str = "secure") -> bytes:
    """ChaCha20 key SHA-256(u64 seed); the incremental workload's key is its start scalar
    clamp(SHA-512(ChaCha20 seed 0 of that key))."""
    w = WORKLOADS[name]
    key = hashlib.sha256(w["seed"].to_bytes(8, "little")).digest()
    if w["source"] != 2:
        return key
    h = bytearray(hashlib.sha512(chacha20_seed0(key)).digest()[:32])
    h[0] &= 248
    h[31] &= 127
    h[31] |= 64
    return bytes(h)


# which part of the multi-pattern workload a run searches: "all" (the workload), or only its
# "text" patterns or its "regex" patterns (to split the matching cost)
MULTI_SET = "all"


def workload_needle(name: str = "secure") -> str:
    import numpy as np
    w = WORKLOADS[name]
    if "needle" in w:
        return w["needle"]
    if name == "multi":
        text = [] if MULTI_SET == "regex" else [t for t, _ in multi_patterns()]
        rx = [] if MULTI_SET == "text" else list(MULTI_REGEXES)
        return ",".join(text + rx)
    rng = np.random.default_rng(w["seed"])
    return "".join(ALPHABET[int(i)] for i in rng.integers(0, 64, w["length"]))


def workload_needles(name: str = "secure"):
    import meikey_b200 as mk
    if name == "multi":
        out = []
        for text, mode in (multi_patterns() if MULTI_SET != "regex" else []):
            if mode == "suffix":
                out.append(mk.Needle.suffix(text))
            else:
                out.append(mk.Needle.contains(text, case_sensitive=mode == "contains"))
        return out + ([mk.Needle.regex(r, max_states=64) for r in MULTI_REGEXES] if MULTI_SET != "text" else [])
    n, mode = workload_needle(name), WORKLOADS[name]["mode"]
    if mode == "suffix":
        return [mk.Needle.suffix(n)]
    return [mk.Needle.contains(n, case_sensitive=mode != "contains_ci")]


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


RANK_SHIFT = 56  # rank r searches indices r·2^56 ...: disjoint for any run shorter than 2^56 candidates


def rank_first(rank: int, warmup: int, step_keys: int) -> int:
    """First timed index of a rank: its own 2^56-wide range, after its warm-up steps."""
    return (rank << RANK_SHIFT) + warmup * step_keys


class Dist:
    """Barrier and max-over-ranks for the torchrun case (NCCL on GPUs, gloo for CPU tests);
    no-ops for one process.  The data path has no collective: ranks search disjoint ranges."""

    def __init__(self, world, local, backend="nccl"):
        self.world = world
        self.pg = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.torch, self.dist = torch, dist
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU baseline: the reference's kernel compiled for the CPU (oracle/_ref) or the oracle port
# ---------------------------------------------------------------------------

class CpuBaseline:
    """The reference's kernel built for the CPU (secure path), else the C oracle port (and
    always the port for the incremental path, which has no reference implementation)."""

    def __init__(self, workload: str = "secure"):
        from oracle import pyoracle
        self.po = pyoracle
        self.threads = os.cpu_count() or 1
        self.source = WORKLOADS[workload]["source"]
        self.mode = 1 if WORKLOADS[workload]["mode"] == "suffix" else 0
        self.fold = WORKLOADS[workload]["mode"] == "contains_ci"
        variants = [p for p in pyoracle.ref_variants() if "f8_b32" in p] or pyoracle.ref_variants()
        if variants and self.source in (0, 1):
            self.kind = "reference"
            self.ref = pyoracle.RefKernel(variants[0])
            self.width = 16
            self.table = pyoracle.ref_table(self.width)
            self.what = (f"reference kernel.cu compiled as C++ ({os.path.basename(variants[0])}, comb width 16), "
                         f"its CPU search emulation on {self.threads} threads")
        else:
            self.kind = "port"
            self.ref = None
            self.what = f"C oracle restatement of the path (one base-point multiply per key) on {self.threads} threads"

    def run(self, key: bytes, needle: str, seconds: float, base: int = 0):
        """keys/s over a sample of about `seconds` of work on all threads."""
        from concurrent.futures import ThreadPoolExecutor
        nb = needle.lower().encode() if self.fold else needle.encode()
        if self.ref is not None:
            per_call = 128 * self.ref.batch  # one block of the emulated kernel per iteration

            def job(t, iters):
                self.ref.search(128, self.table, self.width, key, self.source == 1, nb, len(nb), self.fold, self.mode,
                                base + t * (1 << 40), iters, False)
            # calibrate
            t0 = time.perf_counter()
            job(0, 1)
            one = max(time.perf_counter() - t0, 1e-4)
            iters = max(1, int(seconds / one))
            t0 = time.perf_counter()
            with ThreadPoolExecutor(self.threads) as ex:
                list(ex.map(lambda t: job(t, iters), range(self.threads)))
            dt = time.perf_counter() - t0
            keys = self.threads * per_call * iters
        else:
            def job(t, n):
                self.po.search(key, self.source, base + t * (1 << 40), n, nb, len(nb), self.fold, self.mode, threads=1)
            t0 = time.perf_counter()
            job(0, 2000)
            per_key = max((time.perf_counter() - t0) / 2000, 1e-7)
            n = max(1000, int(seconds / per_key))
            t0 = time.perf_counter()
            with ThreadPoolExecutor(self.threads) as ex:
                list(ex.map(lambda t: job(t, n), range(self.threads)))
            dt = time.perf_counter() - t0
            keys = self.threads * n
        return keys / dt, keys


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    key, needle = workload_key(args.workload), workload_needle(args.workload)
    if args.workload in ("multi", "serving"):
        # the reference's search takes one needle: its keys/s on the secure workload's needle
        # stands for the CPU rate of these workloads
        key, needle = workload_key("secure"), workload_needle("secure")
    cpu = CpuBaseline(args.workload)
    per_step = args.ref_step_seconds
    for _ in range(args.warmup):
        cpu.run(key, needle, per_step / 4)
    rates, keys = [], 0
    t0 = time.perf_counter()
    for s in range(args.steps):
        r, k = cpu.run(key, needle, per_step, base=(s + 1) << 44)
        rates.append(r)
        keys += k
    dt = time.perf_counter() - t0
    value = keys / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(args.workload, None),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu.threads, "kind": cpu.kind,
                         "sample": f"{keys} candidates over {args.steps} steps; {cpu.what}"
                                   + ("; one needle ('" + needle + "'): the reference searches one pattern at a time"
                                      if args.workload in ("multi", "serving") else "")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.workload == "secure" and not args.headline_only:
        # the reference's published mode (counter seeds, TARGET case-insensitive) on the same cores
        ccpu = CpuBaseline("counter")
        rate, ckeys = ccpu.run(workload_key("counter"), workload_needle("counter"), 4 * per_step)
        line["workloads"] = {"counter": {
            "value": rate, "unit": UNIT, "config": workload_config("counter", None),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": ccpu.threads, "kind": ccpu.kind,
                             "sample": f"{ckeys} candidates; {ccpu.what}"}}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(workload, ctx, step_candidates=None, steps=None):
    if workload == "multi":
        cfg = {
            "workload": "batched multi-pattern: secure-path ChaCha20 seeds (key SHA-256(u64 23)), 64 text "
                        "patterns of length U{3..9} (numpy default_rng(23); case-sensitive contains, suffix, "
                        "case-insensitive contains) + 8 regexes as DFAs of <= 64 states, one job, each step "
                        "one CUDA-graph replay of 4 persistent launches; 2^34 candidates",
            "candidates_total": WORKLOADS[workload]["total"],
            "regexes": MULTI_REGEXES,
        }
    elif workload == "counter":
        cfg = {
            "workload": "the reference's published GPU mode: low-security counter seeds (key SHA-256(u64 7) with "
                        "the index added to its last 8 bytes), SHA-512 with the per-launch midstate, clamp, comb "
                        "multiply, pooled inversion, base64, needle 'TARGET' case-insensitive contains; 2^33 "
                        "candidates",
            "candidates_total": WORKLOADS[workload]["total"],
        }
    elif workload == "incremental":
        cfg = {
            "workload": "incremental (low-security) path: s0 = clamp(SHA-512(ChaCha20 seed 0 of key "
                        "SHA-256(u64 11))), P_k = P_0 + k*B by mixed additions, pooled inversion, base64, "
                        f"case-sensitive 6-char suffix '{workload_needle(workload)}' (numpy default_rng(11)); "
                        "2^32 candidates",
            "candidates_total": WORKLOADS[workload]["total"],
        }
    else:
        cfg = {
            "workload": "secure-path throughput: ChaCha20 seeds (key SHA-256(u64 7)), SHA-512, clamp, "
                        "comb multiply, pooled inversion, base64, case-sensitive 7-char contains "
                        f"'{workload_needle(workload)}' (numpy default_rng(7)); 2^34 candidates",
            "candidates_total": WORKLOADS[workload]["total"],
        }
    if ctx is not None:
        info = ctx.info
        cfg.update({
            "step_candidates": step_candidates,
            "steps_cover": step_candidates * steps if steps else None,
            "table_rows": info["table_rows"],
            "table_bytes": info["table_bytes"],
            "keys_per_thread": info["keys_per_thread"],
            "block": info["block"],
            "grid": info["grid"],
            # keys sharing one field inversion (mk_options.inversion_batch)
            "inversion_batch": info["inversion_batch"],
            "l2": ("no memory-resident inputs: each thread steps its own point, the 14 KB step tables "
                   "stay on chip" if workload == "incremental" else
                   "inputs larger than L2: random gathers from the comb table in HBM"),
            "parallelism": "one process per GPU, disjoint index ranges (rank * 2^56), no collective",
        })
    return cfg


def traffic_per_key(workload):
    """DRAM bytes per key of the search kernel from the committed ncu summary of this workload."""
    path = os.path.join(ROOT, "profiles", "k_search_dram.json" if workload == "secure" else
                        f"k_search_{workload}_dram.json")
    try:
        with open(path) as f:
            return json.load(f).get("dram_bytes_per_key")
    except (OSError, ValueError):
        return None


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    return xs[min(len(xs) - 1, int(math.ceil(q * len(xs))) - 1)]


def run_serving(args):
    print(json.dumps(serving(args)), flush=True)
    return 0


def serving(args):
    """Continuous batching against one job at a time on the same GPU, same jobs, same keys:
    the JSON record of the serving workload."""
    import meikey_b200 as mk
    wl = WORKLOADS["serving"]
    n_jobs = args.serve_jobs or wl["jobs"]
    jobs = serving_jobs(n_jobs, wl["rate"], wl["seed"])

    def needle(text, mode):
        return mk.Needle.suffix(text) if mode == "suffix" else mk.Needle.contains(text, case_sensitive=mode == "contains")
    needles = [needle(t, m) for _, t, m in jobs]
    key = hashlib.sha256(wl["seed"].to_bytes(8, "little")).digest()
    ctx = mk.Context(device=0, table_rows=args.rows, keys_per_thread=args.kpt or 8, block=args.block, self_check=True,
                     hit_capacity=1 << 22, inverter_rotates=bool(args.inverter_rotates))
    budget, iters, device_bytes = wl["budget"], wl["iters_per_tick"], wl["device_bytes"]
    # warm-up: a few ticks of a throw-away server
    with mk.Server(ctx, key, max_jobs=4, iters_per_tick=iters, budget=budget, first=1 << 60) as warm:
        for k in range(3):
            warm.submit(needles[k], k)
        for _ in range(args.warmup):
            warm.tick()
    clocks = ClockSampler(0)
    clocks.start()
    # serving: arrivals in real time, one tick after another while anything is admitted or queued
    res, done_at, order = {}, {}, []
    ticks = 0
    with mk.Server(ctx, key, max_jobs=128, iters_per_tick=iters, budget=budget, hit_capacity=1 << 21,
                   device_bytes=device_bytes) as srv:
        t0 = time.perf_counter()
        i = 0
        busy = False
        deadline = jobs[-1][0] + 600.0
        while len(res) < n_jobs:
            now = time.perf_counter() - t0
            if now > deadline:
                raise RuntimeError(f"serving run did not finish: {len(res)} of {n_jobs} jobs")
            while i < n_jobs and jobs[i][0] <= now:
                srv.submit(needles[i], i)
                i += 1
                busy = True
            if not busy:
                if i >= n_jobs:
                    raise RuntimeError(f"serving run lost jobs: {len(res)} of {n_jobs}")
                time.sleep(max(0.0, min(jobs[i][0] - now, 0.01)))
                continue
            active, queued = srv.tick()
            ticks += 1
            t_done = time.perf_counter() - t0
            for r in srv.results():
                res[r["id"]] = r
                done_at[r["id"]] = t_done
                order.append(r["id"])
            busy = active + queued > 0
        serve_span = time.perf_counter() - t0
        stream = srv.position
    clk = clocks.stop()
    # one job at a time: FIFO in arrival order, each job searched alone from its admission
    # index with the same budget, skipping the indices the server delivered to jobs that
    # finished before it (one key goes to one job), so the keys must be the same
    rank_of = {j: r for r, j in enumerate(order)}
    delivered = sorted((rank_of[j], res[j]["index"]) for j in res if res[j]["found"])
    base_res, base_done = {}, {}
    limit = min(n_jobs, args.serve_baseline_jobs or n_jobs)
    single = ctx.job(key, mk.SEED_CHACHA20, [needles[0]])  # one job, its needle replaced per request
    t0 = time.perf_counter()
    for k in range(limit):
        arrival = jobs[k][0]
        now = time.perf_counter() - t0
        if now < arrival:
            time.sleep(arrival - now)
        single.update([needles[k]])
        taken = {idx for r, idx in delivered if r < rank_of[k]}
        first, end = res[k]["admit_index"], res[k]["admit_index"] + budget
        while True:
            out = single.search(first=first, max_tries=end - first, iters=iters)
            if not out["found"] or out["index"] not in taken:
                break
            first = out["index"] + 1
        out["tries"] = (out["index"] + 1 if out["found"] else end) - res[k]["admit_index"]
        base_res[k] = out
        base_done[k] = time.perf_counter() - t0
    base_span = time.perf_counter() - t0
    single.close()
    ctx.close()
    identical = sum(1 for k in range(limit)
                    if base_res[k]["found"] == res[k]["found"]
                    and (not res[k]["found"] or (base_res[k]["index"], base_res[k]["pk"]) == (res[k]["index"], res[k]["pk"])))
    ttk = [done_at[k] - jobs[k][0] for k in range(n_jobs) if res[k]["found"]]
    ttk_all = [done_at[k] - jobs[k][0] for k in range(n_jobs)]
    b_ttk = [base_done[k] - jobs[k][0] for k in range(limit) if base_res[k]["found"]]
    b_all = [base_done[k] - jobs[k][0] for k in range(limit)]
    tries = sum(r["tries"] for r in res.values())
    b_tries = sum(base_res[k]["tries"] for k in range(limit))
    value = tries / serve_span
    b_value = b_tries / base_span
    line = {
        "metric": METRIC, "value": value, "unit": "keys/s", "n_gpus": 1, "steps": ticks, "warmup": args.warmup,
        "ms_per_step": 1000 * serve_span / max(1, ticks), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {
            "workload": f"serving: {n_jobs} vanity jobs, Poisson arrivals at {wl['rate']:g}/s (numpy default_rng(31)), "
                        "pattern length U{4..8}, mode uniform over case-sensitive contains / suffix / case-insensitive "
                        "contains; continuous batching over one ChaCha20 candidate stream (key SHA-256(u64 31)), "
                        f"per-job budget {budget} candidates, admission shortest-expected-first by needle slots, "
                        f"hit-ring plan and a device-memory budget of {device_bytes} bytes; each found index goes to "
                        "one job",
            "value_is": "aggregate job-keys/s: candidates searched for each job, summed over jobs, per second of the "
                        "serving run (one candidate tested for n admitted jobs counts n times)",
            "iters_per_tick": iters, "max_jobs": 128, "budget": budget,
        },
        "clocks": clk,
        "gpu_launches": ticks,
        "serving": {
            "jobs": n_jobs, "found": len(ttk), "censored": n_jobs - len(ttk),
            "p50_time_to_key_s": _pct(ttk, 0.5), "p99_time_to_key_s": _pct(ttk, 0.99),
            "p50_time_to_result_s": _pct(ttk_all, 0.5), "p99_time_to_result_s": _pct(ttk_all, 0.99),
            "jobs_per_s": n_jobs / serve_span, "span_s": serve_span,
            "stream_candidates_per_s": stream / serve_span,
        },
        "one_at_a_time": {
            "jobs": limit, "value": b_value, "unit": "keys/s", "found": len(b_ttk),
            "p50_time_to_key_s": _pct(b_ttk, 0.5), "p99_time_to_key_s": _pct(b_ttk, 0.99),
            "p50_time_to_result_s": _pct(b_all, 0.5), "p99_time_to_result_s": _pct(b_all, 0.99),
            "jobs_per_s": limit / base_span, "span_s": base_span,
        },
        "identical_results": f"{identical}/{limit}",
        "speedup_keys_per_s": value / b_value if b_value else None,
        "speedup_jobs_per_s": (n_jobs / serve_span) / (limit / base_span),
        "e2e": {"value": value, "unit": "keys/s", "note": "host wall clock around submit/tick/results, the public API"},
        "distinct_keys": len({res[k]["index"] for k in res if res[k]["found"]}) == len(ttk),
    }
    return line


def measure(args, workload, steps, e2e_steps, dist, world, rank, local, cpu_seconds=0.0):
    """One workload on this rank: `steps` device-timed steps (barrier and synchronize on both
    sides, max over ranks), then `e2e_steps` end-to-end steps through the public API; on rank 0
    the JSON record of the workload (None on the other ranks)."""
    import meikey_b200 as mk
    wl = WORKLOADS[workload]
    key, source = workload_key(workload), wl["source"]
    # the multi-pattern workload's 3-character patterns alone give ~1e-3 candidates per key
    # keys per thread: the workload's (the tuner's pick, profiles/autotune_sweep.md), else 16 for
    # the incremental source and 8 for the hashed ones
    kpt = args.kpt or wl.get("kpt") or (16 if source == 2 else 8)
    rotates = args.inverter_rotates if args.inverter_rotates is not None else bool(wl.get("inverter_rotates", False))
    hash_warps = args.hash_warps if source != 2 else 0
    inv_batch = args.inversion_batch
    if inv_batch is None:
        # the workload's batch where this layout can run it (256 = 8 keys x 480 threads / 15 pools)
        inv_batch = wl.get("inversion_batch", 0)
        if inv_batch not in mk.engine.inversion_batches(kpt, args.block, hash_warps, int(rotates), 1, 1 << 20):
            inv_batch = 0
    interleave = bool(args.hash_interleave) and source != 2
    ctx = mk.Context(device=local, table_rows=args.rows, keys_per_thread=kpt, block=args.block,
                     self_check=True, hit_capacity=(1 << 22) if workload == "multi" else 0,
                     hash_warps=hash_warps, inverter_rotates=rotates, inversion_batch=inv_batch,
                     hash_interleave=interleave, table_in_smem=bool(args.table_in_smem))
    kpi = ctx.keys_per_iter
    launches = wl.get("launches", 1)  # > 1: a step is one replay of a CUDA graph of that many launches
    iters = math.ceil((args.step_candidates or wl["step"]) / (kpi * launches))
    step_keys = kpi * iters * launches
    rank_base = rank_first(rank, 0, step_keys)
    peak, peak_lo = ctx.measure_mad_peaks()
    pieces = ctx.measure_imad_rates() if workload == args.workload else None
    field_muls, mads_per_key = ctx.work_per_key(source)
    needles = workload_needles(workload)
    job = ctx.job(key, source, needles)
    graph = job.graph(iters, launches) if launches > 1 else None

    def enqueue_step(base):
        if graph is not None:
            graph.enqueue(base)
        else:
            job.enqueue(base, iters)
    # warm-up
    for w in range(args.warmup):
        enqueue_step(rank_base + w * step_keys)
    ctx.sync()
    # timed region: device-resident inputs, K launches back to back
    clocks = ClockSampler(local)
    clocks.start()
    dist.barrier()
    ctx.sync()
    ctx.record(0)
    first = rank_first(rank, args.warmup, step_keys)
    for s in range(steps):
        enqueue_step(first + s * step_keys)
    ctx.record(1)
    ctx.sync()
    dist.barrier()
    ms_local = ctx.elapsed_ms(0, 1)
    clk = clocks.stop()
    ms = dist.max(ms_local)
    keys_all = step_keys * steps * world
    value = keys_all / (ms / 1000.0)
    per_gpu = step_keys * steps / (ms_local / 1000.0)
    # end to end through the public API: prepare (H2D of key + compiled needle), launch,
    # read the job state and hits back (D2H), confirm every needle's first key on the host
    h2d = d2h = 0
    found = confirmed = 0
    phases = {"prepare": 0.0, "launch_and_wait": 0.0, "read_hits": 0.0, "confirm": 0.0, "release": 0.0}
    e2e_clocks = ClockSampler(local)
    e2e_clocks.start()
    dist.barrier()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        tp = time.perf_counter()
        j = ctx.job(key, source, workload_needles(workload))
        g = j.graph(iters, launches) if launches > 1 else None
        tl = time.perf_counter()
        e2e_base = first + (steps + s) * step_keys
        if g is not None:
            g.launch(e2e_base)
        else:
            j.launch(e2e_base, iters)
        tr = time.perf_counter()
        found += j.hits(cap=0)[1]
        tc = time.perf_counter()
        # one key per needle is written: each needle's candidates are confirmed on the host
        # in index order until one matches with its real x sign (mk_job_first_matches)
        confirmed += sum(m is not None for m in j.first_matches())
        a, b = j.io_bytes()
        h2d += a
        d2h += b
        tx = time.perf_counter()
        if g is not None:
            g.close()
        j.close()
        te = time.perf_counter()
        for name, (x, y) in zip(phases, ((tp, tl), (tl, tr), (tr, tc), (tc, tx), (tx, te))):
            phases[name] += y - x
    dt_e2e = time.perf_counter() - t0
    e2e_clk = e2e_clocks.stop()
    dt_e2e = dist.max(dt_e2e)
    e2e = step_keys * e2e_steps * world / dt_e2e
    if graph is not None:
        graph.close()
    job.close()
    line = None
    if rank == 0:
        achieved = mads_per_key * per_gpu / 1e12
        tpk = traffic_per_key(workload)
        roofline = {
            "bound": "int_mad", "achieved": achieved, "peak": peak / 1e12, "unit": "Tmad/s",
            "frac": achieved / (peak / 1e12) if peak else None,
            "traffic": tpk * step_keys if tpk else None,
            "peak_source": "measured live: rows of mad.lo.cc/madc.hi.cc carry chains shaped like the field "
                           "multiply, independent accumulators, full occupancy (mk_measure_mad_peaks)",
            "peak_mad_lo": peak_lo / 1e12,
            "frac_of_mad_lo": achieved / (peak_lo / 1e12) if peak_lo else None,
            "work_per_key": {"field_muls": field_muls, "int_mads": mads_per_key,
                             "mul_form": ("schoolbook: 144 MADs a multiplication" if source == 2 else
                                          "Karatsuba: 112 MADs a multiplication (comb, batch, back-sweep); "
                                          "pooled inversions schoolbook (144), squarings 88")},
            # the peak's pieces, each on independent chains or carry-linked rows (Tmad/s)
            "imad_pieces": {k: v / 1e12 for k, v in pieces.items()} if pieces else None,
            "kernel_ms_per_launch": ms_local / (steps * launches),
        }
        cfg = workload_config(workload, ctx, step_keys, steps)
        cfg["launches_per_step"] = launches
        cfg["options_from"] = ("mk_autotune_job sweeps (profiles/autotune_sweep.md); the secure headline keeps 8 keys "
                               "per thread, the layout that forms the configuration's inversion batch of 256")
        cfg["hash_warps"] = hash_warps
        cfg["hash_interleave"] = int(interleave)
        cfg["table_in_smem"] = int(bool(args.table_in_smem))
        cfg["inverter_rotates"] = int(rotates)
        cfg["needles"] = len(needles)
        if workload == "multi" and MULTI_SET != "all":
            cfg["needle_set"] = MULTI_SET + " patterns only"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": cfg, "clocks": clk,
            "gpu_launches": steps * launches,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d // max(1, e2e_steps),
                    "d2h_bytes_per_step": d2h // max(1, e2e_steps), "steps": e2e_steps, "candidates": found,
                    "needles_confirmed_on_host": confirmed,
                    "ms_per_step_by_phase": {k: round(1000 * v / max(1, e2e_steps), 3) for k, v in phases.items()},
                    "clocks": e2e_clk},
            "roofline": roofline,
            "device": ctx.info["name"],
        }
    ctx.close()
    if rank == 0 and world == 1 and cpu_seconds > 0:
        cpu = CpuBaseline(workload)
        cpu_key, cpu_needle, what = key, workload_needle(workload), "the same workload"
        if workload == "multi":  # the reference searches one pattern at a time
            cpu_key, cpu_needle = workload_key("secure"), workload_needle("secure")
            what = f"the secure workload's needle '{cpu_needle}' (the reference searches one pattern at a time)"
        rate, keys = cpu.run(cpu_key, cpu_needle, cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cpu.threads, "kind": cpu.kind,
                                "sample": f"{keys} candidates of {what}; {cpu.what}"}
    return line


# the default run measures the headline workload and, on one GPU, these beside it (steps,
# end-to-end steps): every configuration the benchmark is quoted on, in one line
SUB_WORKLOADS = {"counter": (8, 2), "incremental": (16, 4), "multi": (16, 2)}


def run_ours(args):
    world, rank, local = dist_env()
    dist = Dist(world, local)
    line = measure(args, args.workload, args.steps, args.e2e_steps or args.steps, dist, world, rank, local,
                   0.0 if args.no_cpu_baseline else args.cpu_seconds)
    if world == 1 and args.workload == "secure" and not args.headline_only:
        # the sub-records of the other configurations (one GPU only: the scaling runs time the
        # headline alone)
        line["workloads"] = {}
        for name, (steps, e2e_steps) in SUB_WORKLOADS.items():
            line["workloads"][name] = measure(args, name, steps, e2e_steps, dist, world, rank, local)
        line["workloads"]["serving"] = serving(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def tune_candidates(workload):
    """The tuning space the multi-pattern configuration names, in three groups around the
    default point (12 rows, 8 keys per thread, block 512): comb windows (rows 10-20 from HBM,
    32 rows = 8-bit digits from HBM, 42 / 45 / 63 rows = 6-, 5-, 4-bit digits from shared
    memory), keys per thread x block x who inverts, and the inversion batch (64-512)."""
    from meikey_b200.engine import inversion_batches
    rot = int(WORKLOADS[workload].get("inverter_rotates", False))
    base = dict(table_rows=12, keys_per_thread=8, block=512, inverter_rotates=rot)
    out = []
    for rows in (10, 11, 12, 13, 14, 16, 20, 32):
        out.append(dict(base, table_rows=rows))
    for rows, kpt in ((42, 8), (45, 8), (63, 8), (42, 4)):
        out.append(dict(base, table_rows=rows, keys_per_thread=kpt, inverter_rotates=0, table_in_smem=1))
    for kpt, block in ((4, 256), (8, 256), (16, 256), (4, 512), (16, 512)):
        for r in (0, 1):
            out.append(dict(base, keys_per_thread=kpt, block=block, inverter_rotates=r))
    for kpt in (8, 16):
        for r in (0, 1):
            for ib in inversion_batches(kpt, 512, 0, r, 64, 512):
                out.append(dict(base, keys_per_thread=kpt, inverter_rotates=r, inversion_batch=ib))
    out.append(dict(base, inverter_rotates=0, hash_interleave=1))
    out.append(dict(base, inverter_rotates=0, hash_warps=4))
    return out


def run_autotune(args):
    """mk_autotune_job over tune_candidates() on the workload's own job; one JSON line per
    candidate, then the pick."""
    import meikey_b200 as mk
    from meikey_b200.engine import autotune
    wl = WORKLOADS[args.workload]
    cands = tune_candidates(args.workload)
    # the field radix: the search kernel is built for radix 2^32; the others are timed here
    with mk.Context(device=0, table_rows=16, keys_per_thread=8) as c:
        r32, r26, r51 = c.measure_field_mul()
        forms = c.measure_field_mul_forms()
    best, results = autotune(0, cands, finalists=4, trial_keys=args.tune_keys,
                             job=(workload_key(args.workload), wl["source"], workload_needles(args.workload)))
    for r in results:
        print(json.dumps(r), flush=True)
    print(json.dumps({"workload": args.workload, "best": best, "candidates": len(cands),
                      "field_mul_per_s": {"radix_2^32": r32, "radix_2^25.5": r26, "radix_2^51_fp64": r51,
                                          "radix_2^32_schoolbook": forms["schoolbook"],
                                          "radix_2^32_karatsuba": forms["karatsuba"]}}),
          flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=12, help="comb table rows")
    ap.add_argument("--kpt", type=int, default=0,
                    help="keys per thread (default: 8 for the hashed workloads, the mk_autotune winner on B200 in "
                         "profiles/autotune_sweep.md; 16 for the incremental workload, whose per-iteration jump "
                         "and inversion amortise over more keys)")
    ap.add_argument("--block", type=int, default=512)
    ap.add_argument("--hash-warps", type=int, default=0, choices=[0, 4],
                    help="4: search kernel with hashing warps (secure and multi workloads)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (default: --steps)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="secure")
    ap.add_argument("--serve-jobs", type=int, default=0, help="serving: number of jobs (default 1000)")
    ap.add_argument("--serve-baseline-jobs", type=int, default=0,
                    help="serving: jobs run one at a time for the comparison (default: all)")
    ap.add_argument("--step-candidates", type=int, default=0,
                    help="candidates per step (default 2^30 secure, 2^28 incremental; smaller only for "
                         "profiling captures)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--ref-step-seconds", type=float, default=2.0, help="reference arm: seconds per step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--inverter-rotates", action=argparse.BooleanOptionalAction, default=None,
                    help="every warp derives keys and the inversion rotates over four warps "
                         "(mk_options.inverter_rotates; default: on for the multi-pattern workload, "
                         "the layout mk_autotune_job picks for it, off otherwise)")
    ap.add_argument("--hash-interleave", type=int, default=0, choices=[0, 1],
                    help="1: hash the next iteration's seeds inside the comb rows (mk_options.hash_interleave; "
                         "ChaCha20 and counter workloads, 12 rows)")
    ap.add_argument("--autotune", action="store_true",
                    help="instead of the benchmark: mk_autotune_job over the tuning space on the workload's job "
                         "(comb windows, keys per thread, layouts, inversion batches); prints every candidate")
    ap.add_argument("--tune-keys", type=int, default=1 << 27, help="autotune: candidates per trial launch")
    ap.add_argument("--table-in-smem", action="store_true",
                    help="every CTA keeps the comb table in shared memory (mk_options.table_in_smem; 40+ rows, "
                         "e.g. --rows 42 --kpt 8)")
    ap.add_argument("--inversion-batch", type=int, default=None,
                    help="keys per field inversion (mk_options.inversion_batch; default: the workload's, 256 for the "
                         "secure and counter workloads where the layout can run it, else 32 pools)")
    ap.add_argument("--headline-only", action="store_true",
                    help="measure the --workload alone (by default the secure headline also carries the counter, "
                         "incremental, multi-pattern and serving workloads on one GPU)")
    ap.add_argument("--multi-set", choices=["all", "text", "regex"], default="all",
                    help="multi-pattern workload: search all its patterns, or only the text or regex ones")
    args = ap.parse_args()
    global MULTI_SET
    MULTI_SET = args.multi_set
    if args.autotune:
        return run_autotune(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
