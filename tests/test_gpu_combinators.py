"""GPU tests of the searcher combinators: several jobs searching at once with first-hit cancel
(mk_search_many, the reference's All, src/service/search.rs:107-180) and the GPU with host
threads (mk_search_both, the reference's Both, search.rs:86-103).  Two contexts share the one
GPU of a test; their kernels never wait on each other (each job's stop word is written by the
host)."""
import time

import pytest

import meikey_b200 as mk
from conftest import chacha_key

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def two_ctx():
    a = mk.Context(device=0, table_rows=16, keys_per_thread=8, self_check=True, hit_capacity=1 << 18)
    b = mk.Context(device=0, table_rows=16, keys_per_thread=8, self_check=True, hit_capacity=1 << 18)
    yield a, b
    a.close()
    b.close()


def _lowest_full_match(oracle, key, source, first, n, text, fold=False, mode=0):
    nb = text.lower().encode() if fold else text.encode()
    for i in oracle.search(key, source, first, n, nb, len(nb), fold, mode):
        if oracle.match(oracle.derive(key, source, i, 1, threads=1), nb, len(nb), fold, mode, False):
            return i
    return None


def test_first_key_cancels_the_other_job(two_ctx, oracle):
    """Job 0 has a needle that matches within a few launches, job 1 one that practically never
    matches and no budget: the call returns job 0's key (the key mk_search finds alone) and job
    1's search ends with it; job 1's stop request is withdrawn afterwards."""
    a, b = two_ctx
    key = chacha_key(51)
    with a.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Xy9")]) as ja, \
            b.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Zq9xYw7Vu")]) as jb:
        t0 = time.perf_counter()
        out = mk.search_many([ja, jb], first=[1000, 1 << 50], iters=2)
        assert time.perf_counter() - t0 < 60
        assert out["found"] and out["winner"] == 0
        alone = ja.search(first=1000, iters=4)
        assert (out["index"], out["pk"], out["secret"]) == (alone["index"], alone["pk"], alone["secret"])
        assert out["pk"] == oracle.derive(key, 0, out["index"], 1)
        assert out["tries"] >= out["index"] - 1000 + 1
        # the stop request is gone: a launch of 6 iterations of job 1 runs them all (a stopped
        # one ends after two), with the hits of a fresh job
        jb.update([mk.Needle.contains("ab")])
        jb.launch(1 << 30, 6)
        after, _ = jb.hits(cap=1 << 18)
    with b.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("ab")]) as fresh:
        fresh.launch(1 << 30, 6)
        want, _ = fresh.hits(cap=1 << 18)
    assert after == want and after[-1][0] >= (1 << 30) + 5 * b.keys_per_iter


def test_no_key_in_the_budgets(two_ctx):
    a, b = two_ctx
    key = chacha_key(52)
    kpi = a.keys_per_iter
    with a.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Zq9xYw7Vu")]) as ja, \
            b.job(key, mk.SEED_COUNTER, [mk.Needle.contains("Wq8xYw7Vu")]) as jb:
        out = mk.search_many([ja, jb], first=0, max_tries=[2 * kpi + 3, 3 * kpi], iters=1)
    assert not out["found"] and out["winner"] == 2 and out["status"] == mk._lib.ERR_STOPPED
    assert out["tries"] == 5 * kpi + 3


def test_progress_cancels_all(two_ctx):
    a, b = two_ctx
    key = chacha_key(53)
    calls = []
    with a.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Zq9xYw7Vu")]) as ja, \
            b.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Wq8xYw7Vu")]) as jb:
        t0 = time.perf_counter()
        out = mk.search_many([ja, jb], first=[0, 1 << 40], iters=2,
                             progress=lambda tries, el: calls.append(tries) or el > 0.5)
        assert time.perf_counter() - t0 < 30
    assert not out["found"] and out["winner"] == 2 and calls


def test_jobs_of_one_context_are_refused(two_ctx):
    a, _ = two_ctx
    key = chacha_key(54)
    with a.job(key, 0, [mk.Needle.contains("ab")]) as j1, a.job(key, 0, [mk.Needle.contains("cd")]) as j2:
        with pytest.raises(mk.GpuError) as e:
            mk.search_many([j1, j2], first=0)
    assert e.value.status == mk._lib.ERR_BAD_ARG


def test_both_gpu_finds_the_key(two_ctx, oracle):
    a, _ = two_ctx
    key = chacha_key(55)
    with a.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Ab9")]) as j:
        out = j.search_both(first=7, iters=2, cpu_threads=2)
        alone = j.search(first=7, iters=2)
    assert out["found"] and out["winner"] in (0, 1)
    if out["winner"] == 0:
        assert (out["index"], out["pk"]) == (alone["index"], alone["pk"])
    assert out["pk"] == oracle.derive(key, 0, out["index"], 1)


@pytest.mark.parametrize("source", [mk.SEED_CHACHA20, mk.SEED_COUNTER])
def test_both_host_threads_find_the_key(two_ctx, oracle, source):
    """The GPU side spends its budget of one index without a key; one host thread then finds
    the lowest index from cpu_first whose full key matches (the oracle's)."""
    a, _ = two_ctx
    key = chacha_key(56 + source)
    needle = mk.Needle.contains("ab", case_sensitive=False)
    # a GPU index whose key does not match
    gpu_first = next(i for i in range(100) if _lowest_full_match(oracle, key, source, i, 1, "ab", True) is None)
    cpu_first = 1 << 40
    want = _lowest_full_match(oracle, key, source, cpu_first, 4000, "ab", True)
    with a.job(key, source, [needle]) as j:
        out = j.search_both(first=gpu_first, max_tries=1, iters=1, cpu_threads=1, cpu_first=cpu_first)
    assert out["found"] and out["winner"] == 1
    assert out["index"] == want
    assert out["pk"] == oracle.derive(key, source, want, 1)
    assert out["secret"] == oracle.seed(key, source, want)
