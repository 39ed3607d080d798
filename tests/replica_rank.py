"""One rank of the replica-plumbing test (tests/test_replicas.py), started by
bench.spawn_replicas: joins the job over gloo on the CPU, builds its own
board plan on the host, and reports the slowest rank's time and the job's
rank count, as bench.py's GPU arm does."""
import json
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
from courant_b200 import scenes  # noqa: E402
from courant_b200.api import Courant  # noqa: E402

world, rank = int(os.environ["WORLD_SIZE"]), int(os.environ["RANK"])
ranks = bench.Ranks(world, backend="gloo", device="cpu")
s, meta = scenes.parity_scene(Courant())
cells = s.nx * s.ny * s.nz
s.destroy()
ranks.barrier()
worst = ranks.max(10.0 * (rank + 1))       # the per-rank device time of a run
ranks.barrier()
if rank == 0:
    Path(sys.argv[1]).write_text(json.dumps({"n_gpus": world, "max_ms": worst,
                                             "value": bench.replica_rate(world, cells, 1000, worst)}))
ranks.close()
