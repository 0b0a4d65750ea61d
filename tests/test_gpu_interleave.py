"""GPU parity of the search kernel that hashes the next iteration's seeds inside the current
iteration's comb rows (mk_options.hash_interleave): the candidate sets and keys are the
oracle's for both hashed seed sources, odd bases, many-iteration launches (every iteration
but the first takes scalars hashed during the one before), graph replays and early stops."""
import pytest

import meikey_b200 as mk
from conftest import chacha_key

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[8, 16], ids=["kpt8", "kpt16"])
def shai_ctx(request):
    ctx = mk.Context(device=0, table_rows=12, keys_per_thread=request.param, block=512, self_check=True,
                     hit_capacity=1 << 18, hash_interleave=True, inversion_batch=256)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("source", [mk.SEED_CHACHA20, mk.SEED_COUNTER])
@pytest.mark.parametrize("base,iters", [(0, 1), (1_000_003, 3), (2**40 + 1, 2)])
def test_search_matches_oracle(shai_ctx, oracle, source, base, iters):
    key = chacha_key(7 + source)
    n = shai_ctx.keys_per_iter * iters
    with shai_ctx.job(key, source, [mk.Needle.contains("abc", case_sensitive=False)]) as job:
        lowest = job.launch(base, iters)
        hits, total = job.hits(cap=1 << 18)
    want = oracle.search(key, source, base, n, b"abc", 3, True, 0)
    assert [i for i, _ in hits] == want and total == len(want)
    assert lowest == (want[0] if want else None)


def test_many_iterations_equal_single_launches(shai_ctx):
    key = chacha_key(3)
    kpi = shai_ctx.keys_per_iter
    nd = [mk.Needle.contains("Ab9")]
    with shai_ctx.job(key, mk.SEED_CHACHA20, nd) as job:
        job.launch(77, 6)
        together, _ = job.hits(cap=1 << 18)
        apart = []
        for r in range(6):
            job.launch(77 + r * kpi, 1)
            apart += job.hits(cap=1 << 18)[0]
    assert together == sorted(apart)


def test_graph_replays_and_search(shai_ctx, oracle):
    key = chacha_key(31)
    with shai_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("xY", case_sensitive=True)]) as job:
        g = job.graph(2, 3)
        g.launch(5)
        hits, _ = job.hits(cap=1 << 18)
        g.close()
        want = oracle.search(key, 0, 5, 6 * shai_ctx.keys_per_iter, b"xY", 2, False, 0)
        assert [i for i, _ in hits] == want
        out = job.search(first=12345, iters=2)
    assert out["found"] and out["pk"] == oracle.derive(key, 0, out["index"], 1)


def test_stop_request_ends_a_long_launch(shai_ctx):
    key = chacha_key(40)
    with shai_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("zzzzzzzzz")]) as job:
        job.stop(True)
        job.launch(0, 50)  # ends within two iterations per CTA
        job.stop(False)


def test_other_geometries_are_refused():
    for opts in [dict(table_rows=11), dict(table_rows=12, block=256), dict(table_rows=12, keys_per_thread=4),
                 dict(table_rows=12, inverter_rotates=True), dict(table_rows=12, hash_warps=4)]:
        kw = dict(keys_per_thread=8, block=512)
        kw.update(opts)
        with pytest.raises(mk.GpuError) as e:
            mk.Context(device=0, hash_interleave=True, **kw)
        assert e.value.status == mk._lib.ERR_OUT_OF_RANGE, opts
