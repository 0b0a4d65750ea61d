"""The device DFA builder (mk_regex_compile_device) against the host compiler (mk_regex_compile).

The subset construction runs on the GPU and numbers new states in the host's order, so for
every pattern the two must return the same status, the same error text, the same number of
states and the same table bytes.  The corpus is the host compiler's own test patterns (the
reference's cases and the dialect tests), the multi-pattern workload's regexes, word-boundary
and anchor forms, the errors (syntax, empty, empty-matching, no key can match, too many
states) and random patterns."""
import random
import time

import pytest

import meikey_b200 as mk
import test_regex
import test_regex_reference

pytestmark = pytest.mark.gpu

MULTI_REGEXES = ['(ab|cd|ef)[+/]x', '(?:aa|bb)(?:cc|dd)$', 'x.{2}y.{2}z', '(?:ab|ba).{2}[0-9]{2}$', 'z[0-9]{3}z',
                 '(?:xyz|XYZ)$', '(?:AA|BB|CC)[0-9]{3}', '[ab].{4}[cd]z[0-9]']
EXTRA = [r"\b9", r"(?i)ab$", r"\B[0-9]\b", r"(?i)x[[:digit:]]{2}\>", r"^A.{3}b", r"\AKb", r"a.{10}b",
         r"(a|b).{8}(c|d)", r"[0-9]{3}.{5}[a-f]{2}", r"x\by", r"(?i)\bab\B", r"\b{start}ab\b{end}",
         r"\b{start-half}Q\b{end-half}", r"(?m)^ab$", r"[[:alpha:]&&[^a-m]]{3}", r"(?x) a b \d"]
ERRORS = ["^Q", "", "a**", r"\p{L}", "a|", "(", "x{2,1}", "[z-a]"]


def _corpus():
    pats = [(p, cs) for p, cs in test_regex.PATTERNS]
    pats += [(p, cs) for p, cs, _ in test_regex_reference.SAMPLE_CASES]
    pats += [(p, cs) for p in MULTI_REGEXES + EXTRA + ERRORS for cs in (True, False)]
    rng = random.Random(3)
    atoms = ["a", "b", "Z", "9", "+", "/", ".", "[a-c]", "[0-9]", r"\d", r"\w", r"\b", r"\B", "^", "$", "(?i)q", "[^a]"]
    for _ in range(200):
        s = "".join(rng.choice(atoms) + rng.choice(["", "", "", "?", "{2}", "*", "+", "{1,3}"])
                    for _ in range(rng.randint(1, 6)))
        if rng.random() < 0.3:
            s = "(" + s + ")|" + rng.choice(atoms) * 2
        pats.append((s, rng.random() < 0.7))
    out, seen = [], set()
    for p in pats:
        if p not in seen:
            seen.add(p)
            out.append(p)
    return out


def _both(ctx, pattern, cs, max_states=16384):
    res = []
    for dev in (None, ctx):
        try:
            n = mk.Needle.regex(pattern, cs, max_states, device=dev)
            res.append((0, n.states, n.text))
        except mk.GpuError as e:
            res.append((e.status, str(e), None))
    return res


def test_device_tables_equal_host_tables(gpu_ctx):
    corpus = _corpus()
    assert len(corpus) > 250
    compiled = 0
    for pattern, cs in corpus:
        host, dev = _both(gpu_ctx, pattern, cs)
        assert dev == host, (pattern, cs)
        compiled += host[0] == 0
    assert compiled > 150


def test_device_state_limit(gpu_ctx):
    """The too-many-states error at the same limit, and the same table just under it."""
    pattern = r"[ab].{4}[cd]z[0-9]"
    states = mk.Needle.regex(pattern).states
    for limit in (states - 1, states, states + 1, 2, 3):
        host, dev = _both(gpu_ctx, pattern, True, limit)
        assert dev == host, limit
    assert _both(gpu_ctx, pattern, True, states)[1][0] == 0
    assert _both(gpu_ctx, pattern, True, states - 1)[1][0] == mk._lib.ERR_PATTERN


def test_device_large_dfa(gpu_ctx):
    """A DFA of thousands of states (several frontiers of several chunks each)."""
    pattern = r"a.{9}b.{2}[0-9]"
    host, dev = _both(gpu_ctx, pattern, True)
    assert host[0] == 0 and host[1] > 3000
    assert dev == host


def test_device_nfa_limit(gpu_ctx):
    """An NFA beyond 2048 states is refused by the device builder, with the reason."""
    with pytest.raises(mk.GpuError) as e:
        mk.Needle.regex("(?:ab|cd){700}", device=gpu_ctx)
    assert e.value.status == mk._lib.ERR_PATTERN and "device DFA builder" in str(e.value)


def test_device_needle_searches_like_host(gpu_ctx):
    """A job with the device-built needle reports the same candidates as with the host-built one."""
    from conftest import chacha_key
    a = mk.Needle.regex(r"\b9[a-f]", True)
    b = mk.Needle.regex(r"\b9[a-f]", True, device=gpu_ctx)
    assert a == b
    key = chacha_key(5)
    found = []
    for n in (a, b):
        with gpu_ctx.job(key, mk.SEED_CHACHA20, [n]) as job:
            job.launch(0, 2)
            hits, total = job.hits()
            assert total == len(hits)
            found.append(hits)
    assert found[0] == found[1] and len(found[0]) > 0


def test_device_build_time_reported(gpu_ctx):
    """Times both builders on the workload regexes (printed for the profile; no bound asserted
    beyond finishing)."""
    for dev in (None, gpu_ctx):
        t0 = time.perf_counter()
        for p in MULTI_REGEXES:
            mk.Needle.regex(p, device=dev)
        print("device" if dev is not None else "host", (time.perf_counter() - t0) / len(MULTI_REGEXES) * 1e3, "ms per regex")
