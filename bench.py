#!/usr/bin/env python
"""Throughput benchmark of the FDTD time-stepping path (courant.h cem_step).

Workload (default `c3`, the large configuration): a seeded 4-layer board from
this package's generator (courant_b200/boards.py): three cores 0.2-1.0 mm
thick with eps_r 3.0-4.5, each a 4-pole Djordjevic-Sarkar Debye fit; 20
microstrip/stripline traces 0.1-0.5 mm wide with 45-degree jogs, 30
through-vias, a ground plane with clearances; 2D eigenmode ports on the port
trace; the reference's rule-based non-uniform mesh (restated in
courant_b200/mesher.py) sized to about 1500 x 1000 x 64 cells (97 M); 8-cell
CPML on five faces; 201 DFT frequencies to 20 GHz. Synthetic geometry from a
recorded seed; fields start at zero. `c1` and `c2` are the GCPW lines of
courant_b200/scenes.CONFIGS, `c3s` the generator at 500 x 349 x 64 (profiling).

One benchmark step = `chunk` FDTD time steps (default 500, the run-control
interval of the reference's board runner). `value` = cell-updates per second
(cells nx*ny*nz x time steps x ranks / max-over-ranks device time), timed
with CUDA events on the engine's stream. The state (about 12 GB for c3)
exceeds L2, so no flush is needed between steps. `e2e` = the same metric
through the C ABI for 10 000 steps with the plan and state uploaded from host
memory inside the timed region and the spectra and energy read back to the
host after every chunk.

On one GPU the line also carries `batching` (the 96-board mix, bounded: both
excitations of 12 boards of 5e4-8e6 cells, one run at a time against the
batching server) and `serving` (Poisson request streams at 0.5 and 2 req/s,
bounded to 24 requests each: the plain FIFO loop against the continuously
batching server, p50/p95/p99 time-to-S-parameters and solves/hour); each
names its bound.

--impl reference times the reference's own CPU core (oracle/_ref, OpenMP on
all host cores) on the same workload, a bounded sample of steps per
benchmark step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

def _workloads() -> dict:
    from courant_b200 import scenes
    w = {k: dict(desc=v["desc"], kw=v["kw"], ref_chunk=200 if k == "c1" else 20) for k, v in scenes.CONFIGS.items()}
    w["c3"] = dict(desc="seeded 4-layer board, 4-pole Debye cores, 20 traces, 30 vias, mode ports, "
                        "non-uniform mesh of about 1500x1000x64 cells",
                   board=dict(seed=2026, cells=96e6, ports="mode", nf=201, fmax=20e9, steps=30000,
                              target=(1500, 1000, 64)),
                   ref_chunk=1, e2e_steps=10000)
    # the same generator at 8 M cells: a case of the large board's kernels small enough to profile
    w["c3s"] = dict(desc="seeded 4-layer board as c3 at 500x330x64 cells",
                    board=dict(w["c3"]["board"], cells=10.6e6, target=(500, 330, 64), steps=30000), ref_chunk=5,
                    e2e_steps=10000)
    return w


WORKLOADS = _workloads()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            self.p.wait()
        self.f.flush()

    def summary(self) -> dict:
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            v = [x.strip() for x in line.split(",")]
            if len(v) >= 9:
                rows.append(v)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(z: dict) -> dict:
    """Compulsory DRAM bytes per time step (FP32 state): each field component,
    CPML auxiliary, Debye current and SIBC state read once and written once;
    coefficients, material indices and probe traffic excluded."""
    P = z["npole"]
    return {
        # whole step, all state read once + written once (the H/E-fused minimum)
        "step": 48 * z["cells"] + 8 * (z["psiE"] + z["psiH"]) + 8 * P * z["ndisp"] + 8 * z["sibc_terms"] * z["nsibc"],
        # E update as a kernel of its own: E read+write, H read, psi_E, Debye J
        "update_e": 36 * z["cells"] + 8 * z["psiE"] + 8 * P * z["ndisp"],
        # H update: H read+write, E read, psi_H
        "update_h": 36 * z["cells"] + 8 * z["psiH"],
    }


def _oracle():
    """The oracle package's ctypes module (oracle/oracle.py): the reference core's location for the CPU legs."""
    p = str(ROOT / "oracle")
    if p not in sys.path:
        sys.path.insert(1, p)
    import oracle
    return oracle


def build_sim(lib, workload: str):
    from courant_b200 import boards, scenes
    t = time.time()
    w = WORKLOADS[workload]
    if "board" in w:
        s, meta = boards.seeded_board(lib, **w["board"])
    else:
        s, meta = scenes.gcpw_line(lib, **w["kw"])
    meta["setup_s"] = time.time() - t
    return s, meta


def cpu_baseline(workload: str, steps_per_sample: int, samples: int) -> dict:
    """The reference core on the host cores, a bounded sample of the workload."""
    oracle = _oracle()
    from courant_b200.api import Courant
    ref = Courant(oracle.REF_LIB)
    s, meta = build_sim(ref, workload)
    s.step(2)   # warm caches / thread pool
    t = time.perf_counter()
    for _ in range(samples):
        s.step(steps_per_sample)
    dt = time.perf_counter() - t
    cells = meta["cells"]
    return {"value": cells * steps_per_sample * samples / dt, "unit": "cell-updates/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())), "kind": "reference",
            "sample": f"{samples} x cem_step({steps_per_sample}) of the {meta['dims']} workload "
                      f"({dt:.1f} s), setup excluded",
            "setup_s": meta["setup_s"]}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    oracle = _oracle()
    if not oracle.REF_LIB.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcourant_ref.so was not built"}))
        return
    from courant_b200.api import Courant
    ref = Courant(oracle.REF_LIB)
    s, meta = build_sim(ref, args.workload)
    per = args.ref_chunk or WORKLOADS[args.workload]["ref_chunk"]
    for _ in range(args.warmup):
        s.step(per)
    t = time.perf_counter()
    for _ in range(args.steps):
        s.step(per)
    dt = time.perf_counter() - t
    v = meta["cells"] * per * args.steps / dt
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "dims": meta["dims"], "cells": meta["cells"],
                       "time_steps_per_step": per, "setup_s": meta["setup_s"], "threads": cores},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} x cem_step({per}) after {args.warmup} warm-up"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _mix_requests(spec, nf):
    """serve.Request objects for (seed, cells, steps, excite[, nports]) tuples:
    seeded boards of the large configuration's generator with 2D mode ports
    (2 unless the tuple names a count)."""
    from courant_b200 import boards, serve
    return [serve.Request(boards.SeededBoard(t[0], t[1], ports="mode", nf=nf, excite=t[3],
                                             nports=t[4] if len(t) > 4 else 2), int(t[2]), tag=(t[0], t[3]))
            for t in spec]


def _same(a: dict | None, b: dict | None) -> bool:
    """Two request results hold the same S-parameters, bit for bit."""
    import numpy as np
    if a is None or b is None:
        return a is None and b is None
    keys = [k for k in a if k.startswith("S")]
    return keys == [k for k in b if k.startswith("S")] and all(np.array_equal(a[k], b[k]) for k in keys)


def _compare(lib, spec, arrivals, nf) -> dict:
    """The same requests through the plain FIFO loop (set-up, steps and
    S-parameters one request at a time, each waiting for its arrival) and
    through the continuously batching server; solves/hour, latencies and mean
    stage times of both, and whether every result is the same."""
    from courant_b200 import serve
    t0 = time.perf_counter()
    plain = serve.plain_loop(lib, _mix_requests(spec, nf), list(arrivals))
    sp = serve.summary(plain, t0, time.perf_counter())
    srv = serve.Server(lib, chunk=512, builders=8, finishers=8, planners=8)
    t0 = time.perf_counter()
    got = serve.serve_all(srv, _mix_requests(spec, nf), list(arrivals))
    t1 = time.perf_counter()
    srv.close()
    ss = serve.summary(got, t0, t1)
    same = all(_same(a.result, g.result) for a, g in zip(plain, got))
    return {"requests": len(spec), "same_results": same, "plain_fifo": sp, "served": ss,
            "gpu_busy_s": srv.gpu_ms / 1e3,
            "solves_per_hour_vs_plain": ss["solves_per_hour"] / sp["solves_per_hour"] if sp["solves_per_hour"] else None}


def batch_compare(lib, boards_n: int, seed: int = 2026) -> dict:
    """Batched uneven instances, the 96-board configuration bounded to
    `boards_n` boards: seeded boards of the large configuration's generator
    (2D mode ports, 16 frequencies) with cells log-uniform in 5e4-8e6, both
    excitations each, steps uniform in 1 000-4 000 (a tenth of the
    configuration's 10k-40k, so that the comparison takes minutes). All runs
    are there at the start. Plain: one run at a time (set-up, steps,
    S-parameters); batched: the server (host set-up on builder threads, device
    state on loader threads, all runs advancing together in batched launches,
    S-parameters on finisher threads). Results must be bit-identical."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    cells = np.exp(rng.uniform(np.log(5e4), np.log(8e6), boards_n))
    steps = rng.integers(1000, 4000, boards_n)
    spec = [(1000 + q, float(cells[q]), int(steps[q]), ex) for q in range(boards_n) for ex in (1, 2)]
    out = _compare(lib, spec, [0.0] * len(spec), nf=16)
    out["bound"] = (f"{boards_n} of 96 boards x 2 excitations, steps 1k-4k instead of 10k-40k, 16 frequencies; "
                    "solves/hour over the whole job (set-up, steps, S-parameters)")
    return out


def serve_compare(lib, n: int, rates: list, seed: int = 7) -> dict:
    """Serving, the Poisson request stream bounded to `n` requests per rate:
    seeded boards of the large configuration's generator with cells
    log-uniform in 1e5-2e7, 1-4 mode ports (uniform; port 1 driven), 16 frequencies,
    steps uniform in 1 000-5 000 (a tenth of 10k-50k), arriving as a Poisson
    stream at each rate of the sweep; the plain FIFO loop against the
    continuously batching server under a 160 GB HBM budget. Times are wall
    clock from arrival to S-parameters."""
    import numpy as np
    out = {"bound": f"{n} requests per rate, rates {rates} of the 0.05-2 req/s sweep, steps 1k-5k instead of "
                    "10k-50k, 16 frequencies", "rates": {}}
    for rate in rates:
        rng = np.random.Generator(np.random.PCG64(seed + int(rate * 1000)))
        cells = np.exp(rng.uniform(np.log(1e5), np.log(2e7), n))
        steps = rng.integers(1000, 5000, n)
        arr = np.cumsum(rng.exponential(1 / rate, n))
        arr -= arr[0]
        nports = rng.integers(1, 5, n)
        spec = [(500 + q, float(cells[q]), int(steps[q]), 1, int(nports[q])) for q in range(n)]
        out["rates"][str(rate)] = _compare(lib, spec, list(arr), nf=16)
    return out


class Ranks:
    """Replica plumbing of a multi-GPU run: one process per GPU, no collective
    on the data path; a barrier around the timed region and the maximum of a
    per-rank time (nccl on GPUs; gloo works the same way on CPU)."""

    def __init__(self, world: int, backend: str = "nccl", device: str = "cuda"):
        import torch.distributed as dist
        self.world, self.device, self.dist = world, device, dist
        if world > 1 and not dist.is_initialized():
            import datetime
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def spawn_replicas(n: int, cmd: list, env: dict | None = None, timeout: float | None = None) -> int:
    """Start `cmd` as n ranks of one job on this node (RANK, LOCAL_RANK,
    WORLD_SIZE, MASTER_ADDR 127.0.0.1 and a free MASTER_PORT set per rank),
    wait for all of them, and return the worst exit code. Rank 0's output
    is the job's; the others' stdout is discarded."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        e = dict(os.environ if env is None else env, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n),
                 LOCAL_WORLD_SIZE=str(n), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(cmd, env=e, stdout=None if r == 0 else subprocess.DEVNULL))
    rc = 0
    for p in procs:
        try:
            rc = max(rc, abs(p.wait(timeout=timeout)))
        except subprocess.TimeoutExpired:
            p.kill()
            rc = max(rc, 124)
    return rc


def replica_rate(world: int, cells: int, time_steps: int, max_ms: float) -> float:
    """Whole-job cell-updates/s of `world` replicas that each advanced `cells`
    cells by `time_steps` steps, timed by the slowest rank."""
    return world * cells * time_steps / (max_ms / 1e3)


def run_b200(args) -> None:
    import torch
    from courant_b200.api import Courant

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks(world)
    barrier, max_over_ranks = ranks.barrier, ranks.max
    wl = WORKLOADS[args.workload]
    ref_chunk = args.ref_chunk or wl["ref_chunk"]

    lib = Courant()
    lib.selectDevice(local)
    s, meta = build_sim(lib, args.workload)
    log(f"rank {rank}: setup {meta['setup_s']:.1f} s, grid {meta['dims']}")
    chunk = args.chunk
    for _ in range(args.warmup):
        s.step(chunk)
    s.synchronize()
    z = s.sizes()
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        gpu_ms = s.stepTimed(args.steps * chunk)
        torch.cuda.synchronize()
        barrier()
    gpu_ms = max_over_ranks(gpu_ms)
    cells = meta["cells"]
    value = replica_rate(world, cells, chunk * args.steps, gpu_ms)

    # per-kernel device time (event pair per launch) for the roofline
    prof = s.profileSteps(max(args.profile_steps, 1))
    ab = algorithmic_bytes(z)
    kern = {k: v for k, v in prof.items() if v["launches"]}
    dominant = max(kern, key=lambda k: kern[k]["ms"])
    tot = sum(v["ms"] for v in kern.values())
    peak, peak_kind = measured_peaks()
    dom_ms = kern[dominant]["ms"] / kern[dominant]["launches"]
    dom_bytes = ab.get(dominant)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9 if dom_bytes else None
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            t = json.loads(tf.read_text()).get(f"{args.workload}:{dominant}")
            traffic = t["dram_bytes_per_launch"] if t else None
        except Exception:
            traffic = None

    # end to end through the C ABI: upload plan + state, one whole excitation, spectra read every chunk
    e2e = None
    if not args.no_e2e:
        s.releaseDevice()
        e2e_steps = args.e2e_steps or min(meta["steps"], wl.get("e2e_steps", meta["steps"]))
        n_chunks = max(1, e2e_steps // chunk)
        ex = s.c.ex
        nvp, nip, nport = ex.cem_plan_nvprobe(s.h), ex.cem_plan_niprobe(s.h), ex.cem_plan_nport(s.h)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d2h = 0
        for _ in range(n_chunks):
            s.step(chunk)
            specs = [s.vprobe(p) for p in range(nvp)] + [s.iprobe(p) for p in range(nip)]
            specs += [s.portV(p) for p in range(nport)] + [s.portI(p) for p in range(nport)]
            specs.append(s.sourceSpectrum())
            s.energy()   # run control, as the reference's board runner checks after every chunk
            d2h += sum(a.size * 16 for a in specs) + 8
        torch.cuda.synchronize()
        wall = max_over_ranks(time.perf_counter() - t0)
        barrier()
        z2 = s.sizes()
        e2e = {"value": world * cells * chunk * n_chunks / wall, "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(z2["device_bytes"] / n_chunks), "d2h_bytes_per_step": int(d2h / n_chunks),
               "steps": n_chunks, "time_steps": n_chunks * chunk,
               "note": "first step uploads plan and state (device_bytes); spectra and energy read after every step"}

    batching = serving = None
    if rank == 0 and world == 1 and args.batch_runs > 0:
        log("batching comparison ...")
        batching = batch_compare(lib, args.batch_runs)
    if rank == 0 and world == 1 and args.serve_requests > 0:
        log("serving comparison ...")
        serving = serve_compare(lib, args.serve_requests, [float(r) for r in args.serve_rates.split(",")])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        oracle = _oracle()
        if oracle.REF_LIB.exists():
            s.destroy()   # the reference builds its own host state next (tens of GB for the largest board)
            cpu = cpu_baseline(args.workload, ref_chunk, args.ref_samples)

    if rank == 0:
        launches = z["launches_per_step"] * args.steps * chunk + math.ceil(args.steps * chunk / 1024)
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": gpu_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 DFT)",
            "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "dims": meta["dims"], "cells": cells,
                       "time_steps_per_step": chunk, "nf": len(meta["freqs"]), "ndisp": z["ndisp"],
                       "npole": z["npole"], "nsibc": z["nsibc"], "psi": z["psiE"] + z["psiH"],
                       "parallelism": f"replicas x{world}", "l2": "state (>1 GB) exceeds L2; no flush",
                       "setup_s": round(meta["setup_s"], 1)},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic, "bytes_per_launch": dom_bytes, "ms_per_launch": dom_ms,
                         "share": kern[dominant]["ms"] / tot,
                         "step_bytes": ab["step"], "step_frac": ab["step"] / (gpu_ms / 1e3 / (args.steps * chunk)) / 1e9 / peak},
            "kernels": {k: {"ms_per_launch": v["ms"] / v["launches"], "share": v["ms"] / tot} for k, v in kern.items()},
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "batching": batching,
            "serving": serving,
        }
        print(json.dumps(line))
    ranks.close()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3")
    ap.add_argument("--chunk", type=int, default=500, help="FDTD time steps per benchmark step")
    ap.add_argument("--ref-chunk", type=int, default=None,
                    help="time steps per step of the CPU reference (default per workload: c1 200, c2 20, c3 1)")
    ap.add_argument("--ref-samples", type=int, default=10, help="CPU-baseline samples in the b200 arm")
    ap.add_argument("--profile-steps", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-runs", type=int, default=12,
                    help="boards (two excitations each) in the batched-vs-plain comparison (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests per rate in the serving comparison (0: skip)")
    ap.add_argument("--serve-rates", default="0.5,2", help="Poisson arrival rates of the serving comparison, 1/s")
    args = ap.parse_args()
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    if args.impl == "reference":
        run_reference(args)
    elif args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_replicas(args.gpus, [sys.executable, str(Path(__file__).resolve()), *sys.argv[1:]]))
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
