"""GPU parity of the search kernel with the rotating inversion (mk_options.inverter_rotates
= 1: every warp derives keys, and the inversion of iteration it falls to one of the last four
warps in turn): the same candidate sets as the oracle, for 512- and 256-thread CTAs, odd
bases, counter and incremental seeds, multi-iteration launches, early stops, graphs and
DFA needles."""
import pytest

import meikey_b200 as mk
from conftest import chacha_key
from test_gpu_parity import _start_scalar

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(8, 512), (4, 256)], ids=["kpt8-512", "kpt4-256"])
def rot_ctx(request):
    kpt, block = request.param
    ctx = mk.Context(device=0, table_rows=12, keys_per_thread=kpt, block=block, self_check=True,
                     hit_capacity=1 << 18, inverter_rotates=True)
    yield ctx
    ctx.close()


def test_layout(rot_ctx):
    info = rot_ctx.info
    assert rot_ctx.keys_per_iter == info["grid"] * info["block"] * info["keys_per_thread"]


@pytest.mark.parametrize("base", [0, 1_000_003, 2**40 + 1])
def test_full_launch_matches_oracle(rot_ctx, oracle, base):
    key = chacha_key(7)
    n = rot_ctx.keys_per_iter
    with rot_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)]) as job:
        lowest = job.launch(base, 1)
        hits, total = job.hits(cap=1 << 18)
    want = oracle.search(key, 0, base, n, b"abc", 3, True, 0)
    assert [i for i, _ in hits] == want and total == len(want)
    assert lowest == (want[0] if want else None)


def test_counter_seeds(rot_ctx, oracle):
    key = chacha_key(11)
    with rot_ctx.job(key, mk.SEED_COUNTER, [mk.Needle.suffix("Zq", case_sensitive=True)]) as job:
        job.launch(2**40 + 5, 1)
        hits, _ = job.hits(cap=1 << 18)
    assert [i for i, _ in hits] == oracle.search(key, 1, 2**40 + 5, rot_ctx.keys_per_iter, b"Zq", 2, False, 1)


@pytest.mark.parametrize("iters", [2, 3, 5, 9])
def test_iterations_equal_single_launches(rot_ctx, iters):
    """Launches of several iterations hand the inversion to every one of the four warps
    (and back); their hits are those of one-iteration launches over the same ranges."""
    key = chacha_key(3)
    kpi = rot_ctx.keys_per_iter
    nd = [mk.Needle.contains("Ab9")]
    with rot_ctx.job(key, mk.SEED_CHACHA20, nd) as job:
        job.launch(77, iters)
        together, _ = job.hits(cap=1 << 18)
        apart = []
        for r in range(iters):
            job.launch(77 + r * kpi, 1)
            apart += job.hits(cap=1 << 18)[0]
    assert together == apart


def test_stop_on_hit(rot_ctx):
    """A frequent needle with stop_on_hit ends a long launch early; every warp stops at the
    same iteration and the job runs normally afterwards."""
    key = chacha_key(4)
    kpi = rot_ctx.keys_per_iter
    with rot_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)],
                     stop_on_hit=True) as job:
        lowest = job.launch(0, 64)
        hits, total = job.hits(cap=1 << 18)
        assert lowest is not None
        assert all(i < 64 * kpi for i, _ in hits)
        assert total < 41 * (2 / 64) ** 3 * kpi * 64 / 4
        job.launch(5 * kpi, 1)
        again, _ = job.hits(cap=1 << 18)
    assert again and all(5 * kpi <= i < 6 * kpi for i, _ in again)


def test_graph_and_multi_pattern(rot_ctx, oracle):
    """Graph replays and a job with text and regex needles (DFAs staged in shared memory)."""
    key = chacha_key(23)
    kpi = rot_ctx.keys_per_iter
    needles = [mk.Needle.contains("xyz", case_sensitive=False), mk.Needle.regex("(ab|cd)[0-9]$")]
    with rot_ctx.job(key, mk.SEED_CHACHA20, needles) as job:
        with job.graph(1, 2) as g:
            g.launch(10)
            got, _ = job.hits(cap=1 << 18)
    pks = oracle.derive(key, 0, 10, 2 * kpi)
    assert [i for i, k in got if k == 0] == oracle.match_keys(pks, 10, b"xyz", 3, True, 0)
    assert [i for i, k in got if k == 1] == oracle.match_keys(pks, 10, needles[1].text, needles[1].states, False, 2)


def test_incremental_search_matches_oracle(rot_ctx, oracle):
    """Two iterations of the incremental source (per-thread start points and the jump of
    keys_per_iter·B follow the all-warps index layout)."""
    s0 = _start_scalar(0)
    kpi = rot_ctx.keys_per_iter
    base = 2**33 + 77
    needles = [mk.Needle.contains("ab", case_sensitive=False), mk.Needle.suffix("Q", case_sensitive=True)]
    with rot_ctx.job(s0, mk.SEED_INCREMENTAL, needles) as job:
        job.launch(base, 2)
        hits, total = job.hits(cap=1 << 18)
    assert total == len(hits)
    assert [i for i, k in hits if k == 0] == oracle.search(s0, 2, base, 2 * kpi, b"ab", 2, True, 0)
    assert [i for i, k in hits if k == 1] == oracle.search(s0, 2, base, 2 * kpi, b"Q", 1, False, 1)


def test_not_with_hashing_warps():
    with pytest.raises(mk.GpuError) as e:
        mk.Context(device=0, table_rows=12, keys_per_thread=8, block=512, hash_warps=4, inverter_rotates=True)
    assert e.value.status == mk._lib.ERR_OUT_OF_RANGE
