"""The N>1 path of bench.py on CPU: world_size-2 ranks over gloo.

bench.py --gpus N runs N independent replicas (one per GPU, no data-path
collective): rank 0 generates the R-MAT graph once into a cache every rank
loads after a barrier, every rank times its own runs, and the job's time is
the maximum over ranks (one MAX all-reduce), so `value` = N x the work of one
replica / the slowest rank's time. These tests run that host logic with two
gloo ranks, no GPU. The reference arm prints from rank 0 only."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, cache, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench.dist_env()
        assert (r, w, local) == (rank, world, rank)
        # Rank 0 generates, everyone loads the same graph after the barrier.
        csr = bench.make_graph(8, cache, rank, dist.barrier)
        digest = torch.tensor([float(csr.in_col.astype(np.int64).sum()), float(csr.arcs)],
                              dtype=torch.float64)
        gathered = [torch.zeros(2, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, digest)
        # The job's time is the slowest rank's.
        mine = 10.0 + 5.0 * rank
        slowest = bench.max_over_ranks(mine, "cpu")
        value = bench.replica_gteps(world, csr.arcs, 100, slowest)
        out[rank] = (torch.stack(gathered).numpy().tolist(), slowest, value, csr.arcs)
    finally:
        dist.destroy_process_group()


def test_replicas_share_graph_and_reduce_max(tmp_path):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), out), nprocs=world,
                       join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    g0, s0, v0, arcs = out[0]
    g1, s1, v1, _ = out[1]
    assert g0 == g1 and g0[0] == g0[1]  # both ranks loaded the identical graph
    assert s0 == s1 == 15.0             # max over ranks
    assert v0 == v1 == pytest.approx(2 * arcs * 100 / 15e-3 / 1e9)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    bench.run_reference_arm(bench.parse_args())
    assert capsys.readouterr().out == ""


def test_single_rank_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.replica_gteps(1, 1_000_000_000, 2, 1000.0) == pytest.approx(2.0)
