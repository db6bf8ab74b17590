"""The N > 1 path on CPU: two gloo ranks, as bench.py runs one process per GPU.

Each rank assembles its own contiguous cell range (camellia2_b200.shard.shard_range)
with the oracle; rank 0 gathers the per-cell results and compares them with one
process assembling every cell: they are identical, because cells exchange nothing.
The max-over-ranks reduction used for the step time is checked on the same group."""
import os
import socket
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from camellia2_b200.shard import max_over_ranks, shard_range  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle import oracle as om
    from tests.helpers import coeffs_for, poisson2d
    form, bucket, nodes, par = poisson2d(2, 2, 4, 3, 0.2)
    P = om.OraclePlan(bucket)
    C = nodes.shape[0]
    co = coeffs_for(bucket, P.info, C)
    lo, hi = shard_range(C, rank, world)
    o = P.assemble(nodes[lo:hi], par[lo:hi], co[lo:hi])
    parts = [None] * world
    dist.all_gather_object(parts, {"lo": lo, "K": o["K"], "S": o["S"]})
    tmax = max_over_ranks(1.5 + rank)
    if rank == 0:
        K = np.concatenate([p["K"] for p in sorted(parts, key=lambda p: p["lo"])])
        S = np.concatenate([p["S"] for p in sorted(parts, key=lambda p: p["lo"])])
        np.savez(os.path.join(outdir, "r.npz"), K=K, S=S, tmax=tmax)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_cells_match_single_process(oracle_mod):
    from tests.helpers import coeffs_for, poisson2d
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        r = np.load(os.path.join(d, "r.npz"))
        form, bucket, nodes, par = poisson2d(2, 2, 4, 3, 0.2)
        P = oracle_mod.OraclePlan(bucket)
        ref = P.assemble(nodes, par, coeffs_for(bucket, P.info, nodes.shape[0]))
        assert np.array_equal(r["K"], ref["K"]) and np.array_equal(r["S"], ref["S"])
        assert float(r["tmax"]) == 2.5


def test_shard_range_covers_every_cell_once():
    for C in (0, 1, 7, 110592):
        for world in (1, 2, 3, 8):
            ranges = [shard_range(C, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == C
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            assert max(h - l for l, h in ranges) - min(h - l for l, h in ranges) <= 1
