"""Multi-process replica plumbing on CPU (gloo, world size 2).

`bench.py --gpus N` runs N independent replicas of one placement; the only
cross-rank traffic is timing: a barrier around the timed region, the maximum of
the per-rank device times and the sum of iterations.  These tests run that
plumbing as two gloo ranks on the host.
"""
from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from myplacement_b200 import replicas
from myplacement_b200.design import workload


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, size: int, port: int, out) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(size), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    try:
        assert replicas.world() == (rank, size, rank)
        assert replicas.init(backend="gloo", timeout_s=60.0)
        replicas.barrier()
        slowest = replicas.reduce_max(10.0 + rank)
        total = replicas.reduce_sum(3 + rank)
        seed = replicas.replica_seed(2026, rank)
        design, _ = workload("small_5k", seed=seed, scale=0.05)
        # each replica places its own instance: the seeds (and so the designs) differ
        digest = float(design.module_x.sum())
        peers = replicas.reduce_sum(digest)
        replicas.barrier()
        replicas.shutdown()
        out.put((rank, slowest, total, seed, digest, peers))
    except Exception as exc:  # reported to the parent, which fails the test
        out.put((rank, repr(exc)))


@pytest.mark.timeout(180)
def test_two_rank_replica_plumbing():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in procs:
        item = queue.get(timeout=150)
        results[item[0]] = item
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert len(results[rank]) == 6, results[rank]
    for rank in (0, 1):
        _, slowest, total, seed, _, peers = results[rank]
        assert slowest == 11.0  # the job time is the slowest rank's
        assert total == 7.0
        assert seed == 2026 + rank
        assert peers == pytest.approx(results[0][4] + results[1][4])
    assert results[0][4] != results[1][4]


def test_single_process_helpers_are_identity(monkeypatch):
    for key in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(key, raising=False)
    assert replicas.world() == (0, 1, 0)
    assert replicas.init() is False
    replicas.barrier()
    assert replicas.reduce_max(2.5) == 2.5
    assert replicas.reduce_sum(4) == 4.0
    replicas.shutdown()


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
