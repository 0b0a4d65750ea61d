"""GPU parity of the search kernels with the inversion batch as an option (mk_options.
inversion_batch: keys sharing one field inversion = keys per thread x compute threads / pools).
Every batch gives the oracle's candidate sets and public keys: pooling decides only how the
denominators are inverted, never the keys."""
import pytest

import meikey_b200 as mk
from conftest import chacha_key
from test_gpu_parity import _start_scalar

pytestmark = pytest.mark.gpu

# (keys per thread, block, hash warps, rotating, inversion batch): the secure configuration's
# 256 (8 x 480 / 15), the largest and smallest pools, and each layout
LAYOUTS = [(8, 512, 0, 0, 256), (8, 512, 0, 0, 480), (8, 512, 0, 0, 160), (16, 512, 0, 0, 512),
           (16, 512, 0, 1, 256), (4, 256, 0, 0, 64), (8, 512, 4, 0, 256), (16, 512, 4, 0, 352)]


@pytest.fixture(scope="module", params=LAYOUTS, ids=[f"kpt{k}-b{b}-hw{h}-rot{r}-batch{i}" for k, b, h, r, i in LAYOUTS])
def batch_ctx(request):
    kpt, block, hw, rot, batch = request.param
    ctx = mk.Context(device=0, table_rows=16, keys_per_thread=kpt, block=block, self_check=True,
                     hit_capacity=1 << 18, hash_warps=hw, inverter_rotates=bool(rot), inversion_batch=batch)
    yield ctx
    ctx.close()


def test_info_reports_the_batch(batch_ctx):
    assert batch_ctx.info["inversion_batch"] in {b for *_, b in LAYOUTS}


@pytest.mark.parametrize("base,iters", [(0, 1), (1_000_003, 3)])
def test_search_matches_oracle(batch_ctx, oracle, base, iters):
    key = chacha_key(7)
    n = batch_ctx.keys_per_iter * iters
    with batch_ctx.job(key, mk.SEED_CHACHA20, [mk.Needle.contains("abc", case_sensitive=False)]) as job:
        lowest = job.launch(base, iters)
        hits, total = job.hits(cap=1 << 18)
    want = oracle.search(key, 0, base, n, b"abc", 3, True, 0)
    assert [i for i, _ in hits] == want and total == len(want)
    assert lowest == (want[0] if want else None)


def test_counter_and_incremental_seeds(batch_ctx, oracle):
    key = chacha_key(11)
    with batch_ctx.job(key, mk.SEED_COUNTER, [mk.Needle.suffix("Zq")]) as job:
        job.launch(2**40 + 5, 1)
        hits, _ = job.hits(cap=1 << 18)
    assert [i for i, _ in hits] == oracle.search(key, 1, 2**40 + 5, batch_ctx.keys_per_iter, b"Zq", 2, False, 1)
    if not uses_hash_warps(batch_ctx):  # the hashing-warp layout serves hashed seeds only
        s0 = _start_scalar(11)
        with batch_ctx.job(s0, mk.SEED_INCREMENTAL, [mk.Needle.suffix("Q9")]) as job:
            job.launch(1 << 20, 2)
            hits, _ = job.hits(cap=1 << 18)
        assert [i for i, _ in hits] == oracle.search(s0, 2, 1 << 20, 2 * batch_ctx.keys_per_iter, b"Q9", 2, False, 1)


def uses_hash_warps(ctx) -> bool:
    info = ctx.info
    return ctx.keys_per_iter == info["grid"] * 352 * info["keys_per_thread"]


def test_unrunnable_batches_are_refused():
    # not a whole number of pools, more than 32 pools, a batch larger than the CTA's keys
    for kpt, block, batch in [(8, 512, 100), (8, 512, 64), (8, 512, 7680), (16, 256, 100)]:
        with pytest.raises(mk.GpuError) as e:
            mk.Context(device=0, table_rows=16, keys_per_thread=kpt, block=block, inversion_batch=batch)
        assert e.value.status == mk._lib.ERR_OUT_OF_RANGE
