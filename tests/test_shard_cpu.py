"""Multi-rank host logic of the lambda sharding on CPU (gloo, world size 2):
the ranks' lambda pieces tile the domain exactly and the report reduction sums
counts and takes the maximum time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import circlepacking_b200 as cp

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    lo, hi = cp.lambda_shard(rank, world)
    rep = {"evaluated": 10 + rank, "unresolved": rank, "clipped": 0, "fp32_decided": 0, "handles_evaluated": 3,
           "verdicts": [1, 2 + rank, 0, 0, 0], "device_ms": 1.0 + rank, "wall_ms": 2.0 * (1 + rank),
           "launches": 2 + rank, "per_depth": [4, 5 + rank] + [1] * rank, "max_depth_seen": 1 + rank}
    tot = cp.reduce_report(rep)
    out[rank] = (lo, hi, tot)
    dist.destroy_process_group()


def test_lambda_shards_tile_the_domain():
    import circlepacking_b200 as cp

    for world in (1, 2, 3, 7, 8):
        pieces = [cp.lambda_shard(r, world) for r in range(world)]
        assert pieces[0][0] == cp.LAMBDA_MIN and pieces[-1][1] == cp.LAMBDA_MAX
        for (a, b), (c, d) in zip(pieces, pieces[1:]):
            assert b == c and a < b
    with pytest.raises(ValueError):
        cp.lambda_shard(2, 2)


def test_two_rank_reduction_gloo():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (lo0, hi0, t0), (lo1, hi1, t1) = res[0], res[1]
    assert hi0 == lo1
    for t in (t0, t1):
        assert t["evaluated"] == 21 and t["unresolved"] == 1 and t["verdicts"][1] == 5
        assert t["device_ms"] == 2.0 and t["wall_ms"] == 4.0
        # per-depth histograms are summed bin by bin; the deepest bin of any rank counts
        assert t["per_depth"] == [8, 11, 1] and t["max_depth_seen"] == 2 and t["launches"] == 5
