"""Source sharding over ranks, on the CPU: world size 2 over gloo.

Each rank takes its shard of one global source list, computes the per-map
results of its sources (the oracle stands in for the GPU path here: no GPU on
this machine), and the shards are all-gathered back into global order; the
result must equal the single-process computation.  Also the shard balance."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from xtsrcmaps_b200.shard import shard_sources


def test_shards_cover_every_source_once():
    for n, world in ((50, 1), (50, 2), (7, 4), (3, 8), (0, 2)):
        parts = shard_sources(n, world)
        assert len(parts) == world
        allidx = np.concatenate(parts) if n else np.zeros(0, int)
        assert np.array_equal(np.sort(allidx), np.arange(n))
        sizes = [len(p) for p in parts]
        assert max(sizes) - min(sizes) <= 1


def test_longest_processing_time_balance():
    rng = np.random.default_rng(3)
    cost = rng.uniform(1.0, 100.0, 200)  # uneven cutouts
    parts = shard_sources(200, 4, cost)
    assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(200))
    loads = [cost[p].sum() for p in parts]
    # LPT is within 4/3 of optimal; the mean load is a lower bound of the optimum
    assert max(loads) <= 4.0 / 3.0 * max(np.mean(loads), cost.max()) + 1e-9


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import torch.distributed as dist

    from helpers import oracle_pipeline
    from xtsrcmaps_b200.shard import gather_rows, shard_sources
    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        job = make_job("c1", seed=9, n_sources=5)
        job.wcs = Wcs(30, 30, 15.5, 15.5, job.wcs.crval1, job.wcs.crval2, -0.5, 0.5, proj="CAR")
        mine = shard_sources(job.S, world)[rank]
        all_src = job.src_sph
        job.src_sph = all_src[mine]
        r = oracle_pipeline(job)
        local = np.concatenate([r["map"].sum(axis=(1, 2)), r["inv_integ"], r["factor"]], axis=1)
        g = gather_rows(local, mine, len(all_src))
        dist.barrier()
        q.put((rank, g))
    finally:
        dist.destroy_process_group()


def test_sharded_results_equal_single_process():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from helpers import oracle_pipeline
    from xtsrcmaps_b200.synth import make_job
    from xtsrcmaps_b200.wcs import Wcs

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    job = make_job("c1", seed=9, n_sources=5)
    job.wcs = Wcs(30, 30, 15.5, 15.5, job.wcs.crval1, job.wcs.crval2, -0.5, 0.5, proj="CAR")
    r = oracle_pipeline(job)
    want = np.concatenate([r["map"].sum(axis=(1, 2)), r["inv_integ"], r["factor"]], axis=1)
    for rank in range(world):
        assert np.array_equal(got[rank], want), rank
