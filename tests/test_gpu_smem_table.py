"""GPU parity of the search kernel that keeps the whole comb table in shared memory
(mk_options.table_in_smem: every CTA copies the table of a 40+-row comb, e.g. 42 rows of 6-bit
digits in 133 KB, and reads its entries there instead of gathering them from HBM).  The
candidate sets are the oracle's; only where the entries come from differs."""
import pytest

import meikey_b200 as mk
from conftest import chacha_key

pytestmark = pytest.mark.gpu

CASES = [(42, 8), (45, 4), (63, 8)]


@pytest.fixture(scope="module", params=CASES, ids=[f"rows{r}-kpt{k}" for r, k in CASES])
def smem_ctx(request):
    rows, kpt = request.param
    ctx = mk.Context(device=0, table_rows=rows, keys_per_thread=kpt, block=512, self_check=True,
                     hit_capacity=1 << 18, table_in_smem=True)
    yield ctx
    ctx.close()


def test_info(smem_ctx):
    assert smem_ctx.info["table_in_smem"] == 1


@pytest.mark.parametrize("base,iters", [(0, 1), (1_000_003, 2)])
def test_search_matches_oracle(smem_ctx, oracle, base, iters):
    key = chacha_key(7)
    n = smem_ctx.keys_per_iter * iters
    with smem_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)]) as job:
        lowest = job.launch(base, iters)
        hits, total = job.hits(cap=1 << 18)
    want = oracle.search(key, 0, base, n, b"abc", 3, True, 0)
    assert [i for i, _ in hits] == want and total == len(want)
    assert lowest == (want[0] if want else None)


def test_counter_seeds_and_regex(smem_ctx, oracle, golden):
    key = chacha_key(11)
    with smem_ctx.job(key, mk.SEED_COUNTER, [mk.Needle.suffix("Zq")]) as job:
        job.launch(2**40 + 5, 1)
        hits, _ = job.hits(cap=1 << 18)
    assert [i for i, _ in hits] == oracle.search(key, 1, 2**40 + 5, smem_ctx.keys_per_iter, b"Zq", 2, False, 1)
    # a DFA needle (its table stays in global memory) over the golden range
    gkey = bytes.fromhex(golden["chacha_key"])
    lo, hi = golden["search_range"]
    d = {x["regex"]: x for x in golden["dfas"]}
    case = [c for c in golden["search"] if c["mode"] == 2][0]
    nd = mk.Needle.dfa(bytes.fromhex(d[case["regex"]]["table"]), d[case["regex"]]["states"])
    with smem_ctx.job(gkey, mk.SEED_CHACHA20, [nd]) as job:
        job.launch(lo, 1)
        got, _ = job.hits(cap=1 << 18)
    assert [i for i, _ in got if lo <= i < hi] == case["hits"]


def test_search_returns_the_oracles_key(smem_ctx, oracle):
    key = chacha_key(31)
    with smem_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("Ab9")]) as job:
        out = job.search(first=12345, iters=1)
    assert out["found"] and out["pk"] == oracle.derive(key, 0, out["index"], 1)


def test_tables_that_do_not_fit_are_refused():
    for rows, kpt, block in [(32, 8, 512), (20, 8, 512), (42, 16, 512), (42, 8, 256)]:
        with pytest.raises(mk.GpuError) as e:
            mk.Context(device=0, table_rows=rows, keys_per_thread=kpt, block=block, table_in_smem=True)
        assert e.value.status == mk._lib.ERR_OUT_OF_RANGE, (rows, kpt, block)
