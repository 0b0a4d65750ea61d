"""GPU tests of the host loops: the single-job searcher (mk_search, the reference's
Searcher::run over the engine, src/service/search.rs:33-40, gpu.rs:917-996) and the
continuous-batching server (mk_server_*).  Keys are checked against the oracle; every
server result must equal the same job searched alone from its admission index."""
import random

import pytest

import meikey_b200 as mk
from conftest import chacha_key

pytestmark = pytest.mark.gpu

ALPHABET = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/"


def _first_full_match(oracle, key, source, first, last, needle):
    """Lowest index in [first, last] whose full key (x sign known) matches, by the oracle."""
    nb, n, fold, mode = needle.text, len(needle.text), needle.fold, needle.mode
    for i in oracle.search(key, source, first, last - first + 1, nb, n, fold, mode):
        if oracle.match(oracle.derive(key, source, i, 1), nb, n, fold, mode, False):
            return i
    return None


@pytest.mark.parametrize("source", [mk.SEED_CHACHA20, mk.SEED_COUNTER])
def test_search_returns_lowest_confirmed_key(gpu_ctx, oracle, source):
    key = chacha_key(31 + source)
    nd = mk.Needle.contains("Ab9")
    with gpu_ctx.job(key, source, [nd]) as job:
        out = job.search(first=12345, iters=1)
    assert out["found"]
    assert out["pk"] == oracle.derive(key, source, out["index"], 1)
    assert out["secret"] == oracle.seed(key, source, out["index"])
    assert out["tries"] == out["index"] - 12345 + 1
    assert _first_full_match(oracle, key, source, 12345, out["index"], nd) == out["index"]


def test_search_budget_and_cancel(gpu_ctx):
    key = chacha_key(40)
    kpi = gpu_ctx.keys_per_iter
    nd = mk.Needle.contains("zzzzzzzzz")  # practically never matches
    with gpu_ctx.job(key, mk.SEED_CHACHA20, [nd]) as job:
        out = job.search(first=0, max_tries=3 * kpi + 5, iters=2)
        assert not out["found"] and out["status"] == mk._lib.ERR_STOPPED
        assert out["tries"] == 3 * kpi + 5
        calls = []
        out = job.search(first=0, iters=1, progress=lambda tries, el: calls.append(tries) or True)
        assert not out["found"] and calls == [kpi] and out["tries"] == kpi


def _random_needles(n, seed):
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        length = rng.randint(3, 4)
        text = "".join(rng.choice(ALPHABET) for _ in range(length))
        mode = rng.randrange(3)
        if mode == 1:
            out.append(mk.Needle.suffix(text[:2]))
        else:
            out.append(mk.Needle.contains(text, case_sensitive=mode == 0))
    return out


def _serve(gpu_ctx, key, needles, budget, **kw):
    """Runs the jobs through a server; returns their results and the order they finished in."""
    results, order = {}, []
    with mk.Server(gpu_ctx, key, budget=budget, **kw) as srv:
        for i, nd in enumerate(needles):
            srv.submit(nd, i)
        for _ in range(400):
            srv.tick()
            for r in srv.results():
                results[r["id"]] = r
                order.append(r["id"])
            if len(results) == len(needles):
                break
    assert len(results) == len(needles)
    return results, order


def _alone(gpu_ctx, key, nd, admit, budget, consumed):
    """The job searched alone from its admission index (a different launch size), skipping the
    indices already delivered to jobs that finished before it."""
    first, end = admit, admit + budget
    with gpu_ctx.job(key, mk.SEED_CHACHA20, [nd]) as job:
        while True:
            out = job.search(first=first, max_tries=end - first, iters=3)
            if not out["found"] or out["index"] not in consumed:
                return out
            first = out["index"] + 1


def _check_against_alone(gpu_ctx, oracle, key, needles, budget, results, order):
    consumed = set()
    for i in order:
        r = results[i]
        alone = _alone(gpu_ctx, key, needles[i], r["admit_index"], budget, consumed)
        assert alone["found"] == r["found"], i
        if r["found"]:
            assert (alone["index"], alone["pk"], alone["secret"]) == (r["index"], r["pk"], r["secret"]), i
            assert r["pk"] == oracle.derive(key, 0, r["index"], 1)
            consumed.add(r["index"])
        else:
            assert r["tries"] == budget


def test_server_results_equal_jobs_alone(gpu_ctx, oracle):
    """24 jobs (two of them practically unmatchable) through 16 slots: each job's result (found key or censoring) is the
    result of the same needle searched alone from its admission index with a different launch
    size (skipping the indices delivered before it), and found keys are the oracle's."""
    key = chacha_key(31)
    kpi = gpu_ctx.keys_per_iter
    budget = 24 * kpi + 7
    needles = _random_needles(22, 5) + [mk.Needle.contains("Zq9xYw7"), mk.Needle.suffix("Qz81a")]
    results, order = _serve(gpu_ctx, key, needles, budget, max_jobs=16, iters_per_tick=2)
    assert any(r["found"] for r in results.values()) and any(not r["found"] for r in results.values())
    admits = sorted({r["admit_index"] for r in results.values()})
    assert len(admits) > 1  # some jobs waited for a slot
    _check_against_alone(gpu_ctx, oracle, key, needles, budget, results, order)


def test_server_gives_each_key_to_one_job(gpu_ctx, oracle):
    """The same needle submitted three times, and needles that match the same keys ('abcd' and
    'bcd', a folded and an exact copy): every found job gets its own index and secret, the one
    admitted first the lowest; each result is still the job alone with the indices delivered
    before it skipped."""
    key = chacha_key(34)
    kpi = gpu_ctx.keys_per_iter
    budget = 64 * kpi
    needles = [mk.Needle.contains("xY"), mk.Needle.contains("xY"), mk.Needle.contains("xY"),
               mk.Needle.contains("abc"), mk.Needle.contains("bc"), mk.Needle.contains("Bc", case_sensitive=False),
               mk.Needle.contains("bc")]
    results, order = _serve(gpu_ctx, key, needles, budget, max_jobs=8, iters_per_tick=1)
    found = [r for r in results.values() if r["found"]]
    assert len(found) == len(needles)
    assert len({r["index"] for r in found}) == len(found)
    assert len({r["secret"] for r in found}) == len(found)
    # the three copies of one needle: admitted together, they take its first three keys in slot order
    assert results[0]["index"] < results[1]["index"] < results[2]["index"]
    _check_against_alone(gpu_ctx, oracle, key, needles, budget, results, order)


def test_server_admits_by_device_memory(gpu_ctx):
    """With a device-memory budget for about one job's reservation, the second job waits for the
    first one's memory (admitted at a later stream index); without it both start together."""
    key = chacha_key(35)
    kpi = gpu_ctx.keys_per_iter
    needles = [mk.Needle.contains("Zq9xY"), mk.Needle.contains("Wv8uT")]
    # one job holds 16 * (4 * expected candidates per tick + 64) + 64 bytes: about 1.1 KB here
    res_tight, _ = _serve(gpu_ctx, key, needles, 2 * kpi, max_jobs=8, iters_per_tick=1, device_bytes=1500)
    res_free, _ = _serve(gpu_ctx, key, needles, 2 * kpi, max_jobs=8, iters_per_tick=1)
    assert res_free[0]["admit_index"] == res_free[1]["admit_index"]
    assert res_tight[1]["admit_index"] > res_tight[0]["admit_index"]


def test_server_admits_shortest_expected_first(gpu_ctx):
    """With one slot, the queued job with the smaller expected search is admitted first."""
    key = chacha_key(32)
    long_job = mk.Needle.contains("Zq9x")
    short_job = mk.Needle.contains("ab", case_sensitive=False)
    assert short_job.expected_tries() < long_job.expected_tries()
    with mk.Server(gpu_ctx, key, max_jobs=1, iters_per_tick=1, budget=gpu_ctx.keys_per_iter) as srv:
        srv.submit(long_job, 1)
        srv.submit(short_job, 2)
        srv.tick()
        first = srv.results()
        srv.tick()
        second = srv.results()
    assert [r["id"] for r in first] == [2] and [r["id"] for r in second] == [1]


def test_server_keeps_open_jobs_when_a_later_slot_finishes(gpu_ctx):
    """A long job in slot 0 stays open while a short job admitted after it (slot 1) finishes;
    later ticks still carry the long job's needle and censor it at its budget."""
    key = chacha_key(33)
    kpi = gpu_ctx.keys_per_iter
    long_job = mk.Needle.contains("Zq9xYw7")
    short_job = mk.Needle.contains("ab", case_sensitive=False)
    with mk.Server(gpu_ctx, key, max_jobs=4, iters_per_tick=1, budget=4 * kpi) as srv:
        srv.submit(long_job, 1)
        srv.tick()
        assert srv.results() == []
        srv.submit(short_job, 2)
        srv.tick()
        assert [r["id"] for r in srv.results()] == [2]
        srv.tick()
        srv.tick()
        last = srv.results()
    assert [(r["id"], r["found"], r["tries"]) for r in last] == [(1, False, 4 * kpi)]


def test_found_key_writes_openssh_files(gpu_ctx):
    """End to end: mk_search finds and confirms a key, mk_openssh_* write it, the files load
    in Python `cryptography` and the public line holds the pattern after the fixed prefix."""
    from cryptography.hazmat.primitives import serialization
    from meikey_b200.engine import openssh_private, openssh_public
    key = chacha_key(34)
    with gpu_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Q9z", case_sensitive=True)]) as job:
        out = job.search(first=0, iters=4, time_limit_s=60)
    assert out["found"]
    pub = openssh_public(out["pk"], "vanity")
    assert "Q9z" in pub.split()[1][25:]
    priv = serialization.load_ssh_private_key(openssh_private(out["secret"], "vanity", 1).encode(), password=None)
    raw = priv.public_key().public_bytes(serialization.Encoding.Raw, serialization.PublicFormat.Raw)
    assert raw == out["pk"]


def test_search_reruns_overflowing_launches(gpu_ctx, oracle):
    """A launch of 16 iterations with a frequent needle overflows the hit ring (2^18 records);
    mk_search searches the range again in shorter launches and still returns the lowest
    confirmed key, the same as a search of one iteration per launch."""
    key = chacha_key(35)
    nd = mk.Needle.contains("ab", case_sensitive=False)  # about 4 % of keys are candidates
    with gpu_ctx.job(key, mk.SEED_CHACHA20, [nd]) as job:
        wide = job.search(first=7, iters=16)
        narrow = job.search(first=7, iters=1)
    assert wide["found"] and (wide["index"], wide["pk"]) == (narrow["index"], narrow["pk"])
    assert _first_full_match(oracle, key, 0, 7, wide["index"], nd) == wide["index"]


def test_first_matches_are_lowest_confirmed_per_needle(gpu_ctx, oracle):
    """mk_job_first_matches (confirmed on several host threads): for every needle, the lowest
    candidate of the launch whose key matches with its real x sign, with the oracle's key and
    seed; needles without a confirmed candidate report STOPPED."""
    key = chacha_key(37)
    rng = random.Random(37)
    needles = [mk.Needle.contains("".join(rng.choice(ALPHABET) for _ in range(3))) for _ in range(24)]
    needles += [mk.Needle.suffix("Zq9xYw7"), mk.Needle.contains("ab", case_sensitive=False)]
    with gpu_ctx.job(key, mk.SEED_CHACHA20, needles) as job:
        job.launch(4242, 1)
        hits, total = job.hits(cap=1 << 18)
        outs = job.first_matches()
    assert total == len(hits) and len(outs) == len(needles)
    for k, nd in enumerate(needles):
        cands = [i for i, j in hits if j == k]
        want = None
        for i in cands:
            if oracle.match(oracle.derive(key, 0, i, 1), nd.text, len(nd.text), nd.fold, nd.mode, False):
                want = i
                break
        if want is None:
            assert outs[k] is None, k
        else:
            assert outs[k]["index"] == want, k
            assert outs[k]["pk"] == oracle.derive(key, 0, want, 1)
            assert outs[k]["secret"] == oracle.seed(key, 0, want)
