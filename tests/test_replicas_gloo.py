"""CPU tests of the multi-GPU host logic with world_size-2 `gloo` process groups:
the batch sharding (every transform on exactly one rank, balanced bytes), the
max-over-ranks timing and whole-job rate of the replica bench, and a sharded batch
computed rank by rank with the FP64 oracle, gathered and compared with the
unsharded result.  The ranks are spawned processes; rendezvous on 127.0.0.1."""
import json
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, outdir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import time

    import oracle as O
    from fftm_b200 import replicas
    from fftm_b200.batch import draw_shapes, transform_bytes
    dist = replicas.init_group("gloo", timeout_s=60)
    assert replicas.env_rank() == (rank, world, rank)
    shapes = draw_shapes(24, seed=2, sizes=(4, 6, 8, 12))
    mine = replicas.shard(shapes, rank, world)
    rng = np.random.default_rng(100)
    fields = [rng.uniform(-1, 1, s) for s in shapes]
    t0 = time.perf_counter()
    res = {i: O.poisson3d_solve(fields[i], -1.0) for i in mine}
    local_ms = (time.perf_counter() - t0) * 1e3 + 5.0 * rank   # rank 1 is the slow one
    max_ms = replicas.max_over_ranks(dist, local_ms)
    gathered = [None] * world
    dist.all_gather_object(gathered, {"idx": mine, "ms": local_ms,
                                      "sums": {int(i): float(np.sum(np.abs(r))) for i, r in res.items()},
                                      "bytes": sum(transform_bytes(shapes[i]) for i in mine)})
    if rank == 0:
        with open(os.path.join(outdir, "out.json"), "w") as fh:
            json.dump({"max_ms": max_ms, "ranks": gathered,
                       "rate": replicas.whole_job_rate(1000.0, 3, world, max_ms),
                       "full": {i: float(np.sum(np.abs(O.poisson3d_solve(fields[i], -1.0))))
                                for i in range(len(shapes))}}, fh)
    dist.barrier()
    dist.destroy_process_group()


@pytest.fixture(scope="module")
def gloo_run(tmp_path_factory):
    import torch.multiprocessing as mp
    from oracle import build as ob
    ob.build()
    out = tmp_path_factory.mktemp("gloo")
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    with open(out / "out.json") as fh:
        return json.load(fh)


def test_shards_cover_batch_once(gloo_run):
    idx = [i for r in gloo_run["ranks"] for i in r["idx"]]
    assert sorted(idx) == list(range(24))
    b = [r["bytes"] for r in gloo_run["ranks"]]
    assert max(b) / min(b) < 1.25


def test_max_over_ranks_is_the_slowest_rank(gloo_run):
    ms = [r["ms"] for r in gloo_run["ranks"]]
    assert gloo_run["max_ms"] == pytest.approx(max(ms))
    assert gloo_run["rate"] == pytest.approx(1000.0 * 3 * 2 / (gloo_run["max_ms"] * 1e-3))


def test_sharded_results_equal_unsharded(gloo_run):
    got = {}
    for r in gloo_run["ranks"]:
        got.update({int(k): v for k, v in r["sums"].items()})
    for i, v in gloo_run["full"].items():
        assert got[int(i)] == v


def test_partition_lpt_balances():
    import fftm_b200.batch as B
    shapes = B.draw_shapes(512, seed=2)
    for n in (2, 4, 8):
        parts = B.partition_lpt(shapes, n)
        assert sorted(i for p in parts for i in p) == list(range(512))
        loads = [sum(B.transform_bytes(shapes[i]) for i in p) for p in parts]
        assert max(loads) / min(loads) < 1.01


def test_single_rank_defaults(monkeypatch):
    from fftm_b200 import replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.env_rank() == (0, 1, 0)
    assert replicas.init_group("gloo") is None
    assert replicas.max_over_ranks(None, 3.5) == 3.5
    assert replicas.shard([(4, 4, 4)] * 3, 0, 1) == [0, 1, 2]
