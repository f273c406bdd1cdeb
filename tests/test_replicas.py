"""CPU tests of the multi-GPU bookkeeping (replicas over query rows) with gloo, world size 2:
per-rank query sets, the barrier, the maximum of the step time over ranks and the whole-job
throughput the bench reports."""
import os
import socket

import numpy as np
import pytest

from rnn_b200 import replicas as RP


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q = RP.replica_queries(rank, world, 10000, 500)
        RP.barrier()
        ms = 10.0 + 5.0 * rank          # rank 1 is the slower one
        mx = RP.max_over_ranks(ms)
        thr = RP.job_throughput(1e9, world, mx)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), q=q, mx=mx, thr=thr)
        RP.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "r0.npz")
    r1 = np.load(tmp_path / "r1.npz")
    # both ranks see the slowest rank's time and the same whole-job throughput
    assert float(r0["mx"]) == 15.0 and float(r1["mx"]) == 15.0
    assert float(r0["thr"]) == pytest.approx(2e9 / 15e-3)
    assert float(r0["thr"]) == float(r1["thr"])
    # independent, deterministic query sets per rank
    assert not np.array_equal(r0["q"], r1["q"])
    assert np.array_equal(r0["q"], RP.replica_queries(0, 2, 10000, 500))
    assert np.unique(r0["q"]).size == 500


def test_single_process_uses_the_workload_queries():
    base = np.arange(100, 0, -1, dtype=np.int32)
    q = RP.replica_queries(0, 1, 1000, 40, default=base)
    assert np.array_equal(q, base[:40])
    assert RP.max_over_ranks(3.5) == 3.5
    assert RP.job_throughput(2e9, 1, 10.0) == pytest.approx(2e11)
