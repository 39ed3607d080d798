"""Multi-GPU runs are replicas: every rank advances its own board, with no
collective on the data path; the bench times the slowest rank. The replica
plumbing (bench.Ranks) is exercised here with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    from courant_b200 import scenes
    from courant_b200.api import Courant
    ranks = bench.Ranks(world, backend="gloo", device="cpu")
    # each replica builds its own board plan on the host; nothing is exchanged
    s, meta = scenes.parity_scene(Courant())
    cells = s.nx * s.ny * s.nz
    s.destroy()
    ranks.barrier()
    ms = 10.0 * (rank + 1)                 # the per-rank device time of a run
    worst = ranks.max(ms)
    ranks.barrier()
    out.put((rank, worst, bench.replica_rate(world, cells, 1000, worst)))
    ranks.close()


def test_two_gloo_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cells = 24 * 18 * 14
    assert [g[1] for g in got] == [20.0, 20.0]          # both ranks see the slowest time
    assert got[0][2] == pytest.approx(2 * cells * 1000 / 0.020)


def test_replica_rate_is_whole_job():
    import bench
    assert bench.replica_rate(1, 1000, 500, 1.0) == pytest.approx(5e8)
    assert bench.replica_rate(4, 1000, 500, 2.0) == pytest.approx(1e9)


def test_spawned_replicas_report_the_job(tmp_path):
    """bench.spawn_replicas, the path `bench.py --gpus N` takes outside
    torchrun: N ranks with RANK/LOCAL_RANK/WORLD_SIZE/MASTER_* set, here two
    gloo ranks on the CPU; rank 0 reports n_gpus 2 and the slowest rank."""
    import json
    import bench
    out = tmp_path / "line.json"
    rc = bench.spawn_replicas(2, [sys.executable, str(ROOT / "tests" / "replica_rank.py"), str(out)], timeout=180)
    assert rc == 0
    line = json.loads(out.read_text())
    assert line["n_gpus"] == 2 and line["max_ms"] == 20.0
    assert line["value"] == pytest.approx(2 * 24 * 18 * 14 * 1000 / 0.020)
