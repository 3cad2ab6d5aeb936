"""The replica (multi-GPU) host logic over gloo with two CPU ranks: timing is
the maximum over ranks, the whole-job rate counts every rank's units, and a
batch of independent cases is split round robin and gathered in case order."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT  # noqa: F401  (puts the repo on sys.path)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    from flite3d_b200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        rate, ms = replicas.replica_rate(100.0 * (rank + 1), steps=50)
        mine = replicas.cases_for_rank(7, rank, ws)
        res = replicas.gather_case_results({i: float(i * i) for i in mine}, 7, rank, ws)
        q.put((rank, rate, ms, mine, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_over_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, rate, ms, mine, res in out:
        assert ms == 200.0  # the slower rank sets the time
        assert rate == pytest.approx(2 * 50 / 0.2)
        assert mine == list(range(rank, 7, 2))
        assert res == [float(i * i) for i in range(7)]


def test_cases_for_rank_partitions():
    from flite3d_b200.replicas import cases_for_rank
    for ws in (1, 2, 3, 8):
        got = sorted(i for r in range(ws) for i in cases_for_rank(48, r, ws))
        assert got == list(range(48))
    with pytest.raises(ValueError):
        cases_for_rank(4, 2, 2)
