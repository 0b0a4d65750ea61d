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


def run_schedule(warps, iters, stop_at, rng, dedicated=False):
    state = {"stop": iters}
    logs = [{"produced": [], "done": []} for _ in range(warps)]
    if dedicated:
        progs = [(inverter_program if w == warps - 1 else compute_program)(w, warps, iters, state, stop_at, logs[w])
                 for w in range(warps)]
    else:
        progs = [warp_program(w, warps, iters, state, stop_at, logs[w]) for w in range(warps)]
    blocked = [None] * warps  # barrier a warp waits on
    finished = [False] * warps
    bars = {k: {"n": 0, "tag": None, "waiting": []} for k in (1, 2, 3, 4)}

    def arrive(w, bar, tag, wait):
        s = bars[bar]
        assert s["tag"] in (None, tag), f"barrier {bar} mixes iterations {s['tag']} and {tag}"
        s["tag"] = tag
        s["n"] += 1
        if wait:
            s["waiting"].append(w)
            blocked[w] = bar
        if s["n"] == warps:
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
