"""CPU model of the search kernel's barrier protocol (csrc/kernels.cu, k_search), in both of
its layouts.  Rotating (ROT): every warp of a CTA derives keys, and the inversion of
iteration it is done by warp W-4+(it mod 4), one warp per SM sub-partition in turn.
Dedicated (the default): warp W-1 only inverts, every iteration, and the other warps derive
keys.  Named barriers 1+b (products of pipeline buffer b ready) and 3+b (their inverses
ready), b = it mod 2, count all W warps:
  - produce(it): a warp writes its product, then arrives on 1+b, except the iteration's
    inverting warp, which syncs on 1+b, inverts, may lower the shared stop iteration to
    it+2, and arrives on 3+b;
  - main loop: produce(it+1) when it+1 is below both the launch's iterations and the stop
    iteration, then sync on 3+b (all but the inverting warp), the backward pass of it, and
    stop after it when it+1 reaches either bound.
The model runs the warps' control flow under random schedules with PTX named-barrier
semantics (a phase completes when all W warps have arrived; bar.arrive does not wait) and
random stop requests, and checks that no schedule deadlocks, that no barrier phase mixes two
iterations, and that every warp runs the same iterations 0..L-1."""
import random

import pytest


def inv_warp(it, warps):
    return warps - 4 + (it & 3)


def inverter_program(w, warps, iters, state, stop_at, log):
    """The dedicated inverter warp: sync on the products, decide on stopping, invert, arrive."""
    it = 0
    while True:
        b = it & 1
        yield ("sync", 1 + b, it)
        if it in stop_at:
            yield ("point",)
            state["stop"] = min(state["stop"], it + 2)
        yield ("point",)
        yield ("arrive", 3 + b, it)
        log["produced"].append(it)
        log["done"].append(it)
        yield ("point",)
        if it + 1 >= iters or it + 1 >= state["stop"]:
            return
        it += 1


def compute_program(w, warps, iters, state, stop_at, log):
    """A key warp of the dedicated layout: arrive on the products, wait for the inverses."""
    def produce(it):
        yield ("point",)
        yield ("arrive", 1 + (it & 1), it)
        log["produced"].append(it)

    yield from produce(0)
    it = 0
    while True:
        yield ("point",)
        if it + 1 < iters and it + 1 < state["stop"]:
            yield from produce(it + 1)
        yield ("sync", 3 + (it & 1), it)
        log["done"].append(it)
        yield ("point",)
        if it + 1 >= iters or it + 1 >= state["stop"]:
            return
        it += 1


def warp_program(w, warps, iters, state, stop_at, log):
    def produce(it):
        b = it & 1
        yield ("point",)
        if w == inv_warp(it, warps):
            yield ("sync", 1 + b, it)
            if it in stop_at:  # the inverter reads the host stop word or the hit count
                yield ("point",)
                state["stop"] = min(state["stop"], it + 2)
            yield ("point",)
            yield ("arrive", 3 + b, it)
        else:
            yield ("arrive", 1 + b, it)
        log["produced"].append(it)

    yield from produce(0)
    it = 0
    while True:
        b = it & 1
        yield ("point",)
        if it + 1 < iters and it + 1 < state["stop"]:
            yield from produce(it + 1)
        if w != inv_warp(it, warps):
            yield ("sync", 3 + b, it)
        log["done"].append(it)
        yield ("point",)
        if it + 1 >= iters or it + 1 >= state["stop"]:
            return
        it += 1


def run_programs(progs, counts, rng):
    """Runs warp programs under a random schedule; counts[bar] = warps that complete a phase."""
    warps = len(progs)
    blocked = [None] * warps  # barrier a warp waits on
    finished = [False] * warps
    bars = {k: {"n": 0, "tag": None, "waiting": []} for k in counts}

    def arrive(w, bar, tag, wait):
        s = bars[bar]
        assert s["tag"] in (None, tag), f"barrier {bar} mixes phases {s['tag']} and {tag}"
        s["tag"] = tag
        s["n"] += 1
        if wait:
            s["waiting"].append(w)
            blocked[w] = bar
        if s["n"] == counts[bar]:
            for x in s["waiting"]:
                blocked[x] = None
            bars[bar] = {"n": 0, "tag": None, "waiting": []}

    steps = 0
    while not all(finished):
        ready = [w for w in range(warps) if not finished[w] and blocked[w] is None]
        assert ready, f"deadlock: blocked on {blocked}, barriers {bars}"
        w = rng.choice(ready)
        try:
            op = next(progs[w])
        except StopIteration:
            finished[w] = True
            continue
        if op[0] == "arrive":
            arrive(w, op[1], op[2], wait=False)
        elif op[0] == "sync":
            arrive(w, op[1], op[2], wait=True)
        steps += 1
        assert steps < 10**6
    for k, s in bars.items():
        assert s["n"] == 0, f"barrier {k} left with {s['n']} arrivals"


def run_schedule(warps, iters, stop_at, rng, dedicated=False):
    state = {"stop": iters}
    logs = [{"produced": [], "done": []} for _ in range(warps)]
    if dedicated:
        progs = [(inverter_program if w == warps - 1 else compute_program)(w, warps, iters, state, stop_at, logs[w])
                 for w in range(warps)]
    else:
        progs = [warp_program(w, warps, iters, state, stop_at, logs[w]) for w in range(warps)]
    run_programs(progs, {k: warps for k in (1, 2, 3, 4)}, rng)
    length = len(logs[0]["done"])
    for lg in logs:
        assert lg["done"] == list(range(length)) and lg["produced"] == list(range(length))
    assert 1 <= length <= iters
    return length


@pytest.mark.parametrize("dedicated", [False, True], ids=["rotating", "dedicated"])
@pytest.mark.parametrize("warps", [16, 8])
def test_inverter_protocol(warps, dedicated):
    rng = random.Random(warps + 100 * dedicated)
    for trial in range(400):
        iters = rng.choice([1, 2, 3, 4, 5, 7, 9])
        stop_at = {i for i in range(iters) if rng.random() < 0.15}
        length = run_schedule(warps, iters, stop_at, rng, dedicated)
        first_stop = min(stop_at) if stop_at else None
        want = iters if first_stop is None else min(iters, first_stop + 2)
        assert length == want, (trial, iters, sorted(stop_at), length)


# ---- k_search_hw: 11 comb warps, 1 inverter, 4 hashing warps ----
# Barriers (warp counts): 1+b / 3+b products / inverses (comb + inverter, 12); 5+s / 7+s ring
# slot s full / empty (comb + hashing, 15); 9+(it mod 2) the inverter's stop decision after
# iteration it (inverter + hashing, 5).  A ring chunk holds 4 keys of every comb thread; an
# iteration has KPT/4 chunks, chunk gc uses slot gc mod 2.

def hw_hash_program(iters, cpi, state, log):
    x = 0
    while True:
        if x >= iters:
            break
        if x >= 2:
            yield ("sync", 9 + (x & 1), x - 2)
            yield ("point",)
            if x >= state["stop"]:
                break
        for c in range(cpi):
            gc = x * cpi + c
            if gc >= 2:
                yield ("sync", 7 + (gc & 1), gc - 2)
            yield ("point",)
            yield ("arrive", 5 + (gc & 1), gc)
        log["filled"].append(x)
        x += 1
    g = x * cpi
    yield ("sync", 7 + ((g - 2) & 1), g - 2)
    yield ("sync", 7 + ((g - 1) & 1), g - 1)


def hw_inverter_program(iters, state, stop_at, log):
    it = 0
    while True:
        b = it & 1
        yield ("sync", 1 + b, it)
        if it in stop_at:
            yield ("point",)
            state["stop"] = min(state["stop"], it + 2)
        yield ("point",)
        more = it + 1 < iters and it + 1 < state["stop"]
        if it + 2 < iters and more:
            yield ("arrive", 9 + (it & 1), it)
        yield ("arrive", 3 + b, it)
        log["done"].append(it)
        if not more:
            return
        it += 1


def hw_comb_program(iters, kpt, cpi, state, log):
    def produce(it):
        for j in range(kpt):
            gc = it * cpi + j // 4
            if j % 4 == 0:
                yield ("sync", 5 + (gc & 1), gc)
            yield ("point",)
            if j % 4 == 3:
                yield ("arrive", 7 + (gc & 1), gc)
        yield ("arrive", 1 + (it & 1), it)
        log["produced"].append(it)

    yield from produce(0)
    it = 0
    while True:
        yield ("point",)
        if it + 1 < iters and it + 1 < state["stop"]:
            yield from produce(it + 1)
        yield ("sync", 3 + (it & 1), it)
        log["done"].append(it)
        yield ("point",)
        if it + 1 >= iters or it + 1 >= state["stop"]:
            return
        it += 1


@pytest.mark.parametrize("kpt", [8, 16])
def test_hashing_warp_protocol(kpt):
    """k_search_hw's barrier protocol (csrc/kernels.cu): no deadlock, no phase mixing two
    chunks or iterations, the hashing warps fill exactly the iterations the comb warps and
    the inverter run, and every ring release is drained before the hashing warps return."""
    rng = random.Random(kpt)
    cpi = kpt // 4
    for trial in range(300):
        iters = rng.choice([1, 2, 3, 4, 6, 9])
        stop_at = {i for i in range(iters) if rng.random() < 0.15}
        state = {"stop": iters}
        combs = [{"produced": [], "done": []} for _ in range(11)]
        inv = {"done": []}
        hashes = [{"filled": []} for _ in range(4)]
        progs = ([hw_comb_program(iters, kpt, cpi, state, lg) for lg in combs] +
                 [hw_inverter_program(iters, state, stop_at, inv)] +
                 [hw_hash_program(iters, cpi, state, lg) for lg in hashes])
        counts = {1: 12, 2: 12, 3: 12, 4: 12, 5: 15, 6: 15, 7: 15, 8: 15, 9: 5, 10: 5}
        run_programs(progs, counts, rng)
        first_stop = min(stop_at) if stop_at else None
        want = list(range(iters if first_stop is None else min(iters, first_stop + 2)))
        assert inv["done"] == want, (trial, iters, sorted(stop_at))
        for lg in combs:
            assert lg["produced"] == want and lg["done"] == want
        for lg in hashes:
            assert lg["filled"] == want
