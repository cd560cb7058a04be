"""Multi-rank host logic on CPU (gloo, world size 2): the lambda shards tile the
domain (equal widths or equal estimated work), the interleaved seed pieces of a
real lattice are disjoint and cover it, and the report reduction sums counts,
per-depth histograms and per-box digests so that the ranks' pieces add up to
the single-rank result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests import boxgen


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    return dist


def _worker(rank, world, port, out):
    import circlepacking_b200 as cp

    dist = _init(rank, world, port)
    lo, hi = cp.lambda_shard(rank, world)
    rep = {"evaluated": 10 + rank, "unresolved": rank, "clipped": 0, "fp32_decided": 0, "handles_evaluated": 3,
           "verdicts": [1, 2 + rank, 0, 0, 0], "device_ms": 1.0 + rank, "wall_ms": 2.0 * (1 + rank),
           "launches": 2 + rank, "per_depth": [4, 5 + rank] + [1] * rank, "max_depth_seen": 1 + rank,
           "digest": ((1 << 64) - 1 - rank, 0xF0 >> rank)}
    tot = cp.reduce_report(rep)
    out[rank] = (lo, hi, tot)
    dist.destroy_process_group()


def _seed_worker(rank, world, port, family, sizes, out):
    """One rank's piece of a real lattice seed: its boxes (CPU restatement of
    the lattice), their verdicts (CPU restatement), a report of them, reduced."""
    import circlepacking_b200 as cp
    from oracle import oracle as O

    dist = _init(rank, world, port)
    total = int(np.prod(sizes))
    idx = cp.seed_partition(total, rank, world)
    lo, hi = O.lattice_boxes(family, boxgen.LAMBDA, sizes, idx)
    v, _ = O.eval_boxes(family, lo, hi)
    rep = {"evaluated": int(idx.size), "unresolved": 0, "clipped": 0, "fp32_decided": 0, "handles_evaluated": 0,
           "verdicts": np.bincount(v, minlength=5).tolist(), "device_ms": 0.0, "wall_ms": 0.0, "launches": 1,
           "per_depth": [int(idx.size)], "max_depth_seen": 0, "digest": boxgen.host_digest(lo, hi, v)}
    gathered = [None] * world
    dist.all_gather_object(gathered, idx.tolist())
    out[rank] = (cp.reduce_report(rep), gathered)
    dist.destroy_process_group()


@pytest.mark.parametrize("balance", ["work", "width"])
def test_lambda_shards_tile_the_domain(balance):
    import circlepacking_b200 as cp

    for world in (1, 2, 3, 7, 8):
        pieces = [cp.lambda_shard(r, world, balance=balance) for r in range(world)]
        assert pieces[0][0] == cp.LAMBDA_MIN and pieces[-1][1] == cp.LAMBDA_MAX
        for (a, b), (c, d) in zip(pieces, pieces[1:]):
            assert b == c and a < b
    with pytest.raises(ValueError):
        cp.lambda_shard(2, 2)


def test_work_balanced_shards_equalise_the_work_model():
    """Equal integrals of (1 - lambda)^-2 per piece; the pieces narrow toward 0.99."""
    import circlepacking_b200 as cp

    world = 8
    pieces = [cp.lambda_shard(r, world) for r in range(world)]
    work = [1 / (1 - b) - 1 / (1 - a) for a, b in pieces]
    assert max(work) / min(work) < 1 + 1e-9
    widths = [b - a for a, b in pieces]
    assert all(w1 > w2 for w1, w2 in zip(widths, widths[1:]))


def test_seed_partition_covers_the_seed():
    import circlepacking_b200 as cp

    for total, world in ((100, 3), (7, 8), (4096, 8), (1, 1)):
        parts = [cp.seed_partition(total, r, world) for r in range(world)]
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(total))


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
        # digests: sum mod 2^64 and xor
        assert t["digest"] == (((1 << 64) - 1 + (1 << 64) - 2) & ((1 << 64) - 1), 0xF0 ^ 0x78)


@pytest.mark.parametrize("family,sizes", [(3, [16, 8, 8, 4]), (4, [32, 16, 8])])
def test_two_rank_seed_pieces_add_up_gloo(oracle, family, sizes):
    """A real lattice seed split between two gloo ranks: the pieces are disjoint,
    cover the seed, and the reduced report (counts and per-box digest) equals the
    single-rank report of the whole seed."""
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_seed_worker, args=(world, port, family, sizes, out), nprocs=world, join=True)
        res = dict(out)
    total = int(np.prod(sizes))
    idx = np.arange(total)
    lo, hi = oracle.lattice_boxes(family, boxgen.LAMBDA, sizes, idx)
    v, _ = oracle.eval_boxes(family, lo, hi)
    whole = boxgen.host_digest(lo, hi, v)
    for r in range(world):
        rep, gathered = res[r]
        union = np.concatenate([np.asarray(g) for g in gathered])
        assert union.size == total and np.array_equal(np.sort(union), idx)
        assert rep["evaluated"] == total
        assert rep["verdicts"] == np.bincount(v, minlength=5).tolist()
        assert rep["digest"] == whole
