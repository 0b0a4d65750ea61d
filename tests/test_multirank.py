"""The multi-GPU plan on CPU: two gloo ranks on 127.0.0.1 run bench.py's Dist (barrier,
max over ranks) and its per-rank index plan; the ranges the ranks search (warm-up and timed
steps, and the end-to-end steps after them) are disjoint and each rank's are contiguous."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    d = bench.Dist(world, rank, backend="gloo")
    step_keys, warmup, steps, e2e = 3 * 1137 * 16, 3, 16, 16
    d.barrier()
    ranges = [(bench.rank_first(rank, 0, step_keys) + w * step_keys, step_keys) for w in range(warmup)]
    first = bench.rank_first(rank, warmup, step_keys)
    ranges += [(first + s * step_keys, step_keys) for s in range(steps + e2e)]
    slowest = d.max(float(10 + rank))  # each rank's "time"; all must see the maximum
    d.barrier()
    d.close()
    q.put((rank, ranges, slowest))


def test_two_ranks_plan_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (ranges, slowest) for r, ranges, slowest in out}
    assert by_rank[0][1] == by_rank[1][1] == 11.0
    spans = []
    for r in (0, 1):
        ranges = by_rank[r][0]
        for (a, n), (b, _) in zip(ranges, ranges[1:]):
            assert b == a + n  # contiguous within a rank
        spans.append((ranges[0][0], ranges[-1][0] + ranges[-1][1]))
    (a0, e0), (a1, e1) = sorted(spans)
    assert e0 <= a1  # disjoint across ranks
