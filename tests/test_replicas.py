"""Multi-rank replica runs on the CPU (gloo, world size 2): the helpers bench.py uses under torchrun
for N GPUs -- distinct replica seeds, max-over-ranks timing, whole-job throughput, teardown -- run
in two processes, and two replicas of a small VMC built from their rank seeds start from different
chains.  No GPU and no data-path collective: the VMC step does not shard across GPUs."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from pyqusolver_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, lr = replicas.rank_env()
    dist = replicas.init_group(w, backend="gloo", timeout_s=60)
    # a per-rank "timed region" of different length: the job's time is the slowest rank's
    my_ms = 10.0 + 5.0 * r
    total = replicas.max_over_ranks(my_ms, dist)
    value = replicas.job_throughput(16384, 4, total, w)
    # replicas draw different chains: the oracle's random initial states from the rank seed
    rng = np.random.default_rng(replicas.replica_seed(1234, r))
    chains = (rng.random((8, 16)) < 0.5).astype(np.int64)
    got = torch.tensor(chains.reshape(-1), dtype=torch.int64)
    gathered = [torch.zeros_like(got) for _ in range(w)]
    dist.all_gather(gathered, got)
    replicas.finish(dist)
    out[r] = (r, w, lr, total, value, [g.numpy().tolist() for g in gathered])


def test_two_gloo_ranks_max_timing_and_distinct_replicas():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        codes = [p.exitcode for p in procs]
        res = dict(out)
    assert codes == [0, 0], codes
    for r in range(world):
        rank, w, lr, total, value, gathered = res[r]
        assert (rank, w, lr) == (r, world, r)
        assert total == 15.0                                    # max over ranks, on every rank
        assert value == pytest.approx(world * 16384 * 4 / 0.015)
    g0, g1 = res[0][5]
    assert g0 != g1                                             # independent replicas
    assert res[0][5] == res[1][5]


def test_single_process_needs_no_group():
    assert replicas.init_group(1) is None
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_throughput(100, 10, 1000.0, 1) == 1000.0
    assert replicas.replica_seed(7, 0) != replicas.replica_seed(7, 1)
    with pytest.raises(ValueError):
        replicas.job_throughput(1, 1, 0.0, 1)
    replicas.finish(None)
