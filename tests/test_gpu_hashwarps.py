"""GPU parity of the search kernel with hashing warps (mk_options.hash_warps = 4): the same
candidate sets as the oracle, across odd bases (ChaCha20 blocks split between chunks),
counter seeds, multi-iteration launches and early stops."""
import pytest

import meikey_b200 as mk
from conftest import chacha_key

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[8, 16], ids=["kpt8", "kpt16"])
def hw_ctx(request):
    ctx = mk.Context(device=0, table_rows=12, keys_per_thread=request.param, block=512, self_check=True,
                     hit_capacity=1 << 18, hash_warps=4)
    yield ctx
    ctx.close()


def test_layout(hw_ctx):
    info = hw_ctx.info
    assert hw_ctx.keys_per_iter == info["grid"] * 352 * info["keys_per_thread"]


@pytest.mark.parametrize("base", [0, 1_000_003, 2**40 + 1])
def test_full_launch_matches_oracle(hw_ctx, oracle, base):
    key = chacha_key(7)
    n = hw_ctx.keys_per_iter
    with hw_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)]) as job:
        lowest = job.launch(base, 1)
        hits, total = job.hits(cap=1 << 18)
    want = oracle.search(key, 0, base, n, b"abc", 3, True, 0)
    assert [i for i, _ in hits] == want and total == len(want)
    assert lowest == (want[0] if want else None)


def test_counter_seeds(hw_ctx, oracle):
    key = chacha_key(11)
    with hw_ctx.job(key, mk.SEED_COUNTER, [mk.Needle.suffix("Zq", case_sensitive=True)]) as job:
        job.launch(2**40 + 5, 1)
        hits, _ = job.hits(cap=1 << 18)
    assert [i for i, _ in hits] == oracle.search(key, 1, 2**40 + 5, hw_ctx.keys_per_iter, b"Zq", 2, False, 1)


@pytest.mark.parametrize("iters", [2, 3, 5])
def test_iterations_equal_single_launches(hw_ctx, iters):
    """A launch of several iterations runs the ring and the decision barriers through several
    rounds; its hits are those of one-iteration launches over the same ranges."""
    key = chacha_key(3)
    kpi = hw_ctx.keys_per_iter
    nd = [mk.Needle.contains("Ab9")]
    with hw_ctx.job(key, mk.SEED_CHACHA20, nd) as job:
        job.launch(77, iters)
        together, _ = job.hits(cap=1 << 18)
        apart = []
        for r in range(iters):
            job.launch(77 + r * kpi, 1)
            apart += job.hits(cap=1 << 18)[0]
    assert together == apart


def test_stop_on_hit(hw_ctx):
    """A frequent needle with stop_on_hit ends a long launch early; every role stops together."""
    key = chacha_key(4)
    kpi = hw_ctx.keys_per_iter
    with hw_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)],
                    stop_on_hit=True) as job:
        lowest = job.launch(0, 64)
        hits, total = job.hits(cap=1 << 18)
        assert lowest is not None
        assert all(i < 64 * kpi for i, _ in hits)
        p = 41 * (2 / 64) ** 3
        assert total < p * kpi * 64 / 4
        # the job runs again normally after a stopped launch
        job.launch(5 * kpi, 1)
        again, _ = job.hits(cap=1 << 18)
    assert again and all(5 * kpi <= i < 6 * kpi for i, _ in again)


def test_graph_and_multi_pattern(hw_ctx, oracle):
    """Graph replays and a job with text and regex needles (DFAs read from global memory in
    this layout) on the hashing-warp kernel."""
    key = chacha_key(23)
    kpi = hw_ctx.keys_per_iter
    needles = [mk.Needle.contains("xyz", case_sensitive=False), mk.Needle.regex("(ab|cd)[0-9]$")]
    with hw_ctx.job(key, mk.SEED_CHACHA20, needles) as job:
        with job.graph(1, 2) as g:
            g.launch(10)
            got, _ = job.hits(cap=1 << 18)
    pks = oracle.derive(key, 0, 10, 2 * kpi)
    want0 = oracle.match_keys(pks, 10, b"xyz", 3, True, 0)
    want1 = oracle.match_keys(pks, 10, needles[1].text, needles[1].states, False, 2)
    assert [i for i, k in got if k == 0] == want0
    assert [i for i, k in got if k == 1] == want1


def test_incremental_source_rejected(hw_ctx):
    with pytest.raises(mk.GpuError) as e:
        hw_ctx.job(bytes(32), mk.SEED_INCREMENTAL, [mk.Needle.contains("ab")])
    assert e.value.status == mk._lib.ERR_NOT_BUILT
