"""Serving board simulations on one GPU with continuous batching.

A `Server` accepts requests (a builder returning a finalized simulation, a
step count) as they arrive. Builder threads do the host set-up (plan, mode
solves) in parallel; the GPU thread admits built simulations while their
estimated device footprint fits the HBM budget, loader threads create their
device state (tables, uploads), and the GPU thread adds them to one
`cemx_batch`, runs the batch in chunks, and hands every simulation that
reached its step count to finisher threads, which extract its S-parameters
and free it, while the batch goes on with the others. Requests that arrive while others are on the
GPU join at the next chunk boundary, so their work overlaps on the device.
Each simulation computes the same bits as when it runs alone.

`plain_loop` is the baseline: the same requests one at a time, set-up, steps
and results in order, on the same GPU.

Times are wall clock; `summary()` gives p50/p95/p99 time-to-S-parameters
(arrival to result) and solves per hour.
"""
from __future__ import annotations

import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .api import Courant, Sim


def footprint(sim: Sim) -> int:
    """Device bytes a simulation will hold, from its sizes before its device
    state exists: padded FP32 fields (6), u16 material indices (3), CPML
    auxiliaries (padded layout, about 1.5x the compact count), Debye currents,
    surface-impedance states, and a 10% margin for tables and probes."""
    z = sim.sizes()
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    sj = (nz + 1 + 7) // 8 * 8
    npts = (nx + 1) * (ny + 1) * sj
    b = npts * (6 * 4 + 3 * 2)
    b += int(1.5 * 4 * (z["psiE"] + 2 * z["psiH"]))
    b += int(1.3 * 4 * z["npole"] * z["ndisp"])
    b += 4 * z["sibc_terms"] * z["nsibc"] + 48 * z["nsibc"]
    return int(b * 1.1)


def results(sim: Sim, meta: dict) -> dict:
    """The S-matrix column of the driven port e (meta["excite"]): "S<q>" =
    S_qe for every port q, from the modal waves of mode ports or from the port
    spectra of lumped ports (50 ohm)."""
    from .scenes import s_column
    col = s_column(sim, meta)
    out = {f"S{q + 1}": b for q, b in enumerate(col["b"])}
    out["excite"] = meta.get("excite", 1)
    return out


@dataclass
class Request:
    build: object                 # callable(Courant) -> (Sim, meta)
    steps: int
    tag: object = None
    arrival: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    result: dict | None = None
    error: str | None = None
    cells: int = 0
    event: threading.Event = field(default_factory=threading.Event)
    # stage ends (perf_counter): host set-up, device state, last step on the GPU
    built: float = 0.0
    loaded: float = 0.0
    stepped: float = 0.0


class Server:
    def __init__(self, lib: Courant, budget_bytes: float = 160e9, chunk: int = 512, builders: int = 4,
                 finishers: int = 4, device: int = -1, tune: bool = True, planners: int = 0):
        self.lib = lib
        self.budget = int(budget_bytes)
        self.chunk = chunk
        self.tune = tune
        self.batch = lib.createBatch(device)
        self.batch.tune(tune)
        self.incoming: queue.Queue = queue.Queue()
        self.built: list = []          # (request, sim, meta, bytes) ready for admission, in arrival order
        self.lock = threading.Lock()
        self.wake = threading.Event()
        self.members: dict = {}        # sim handle -> (request, sim, meta, bytes)
        self.used = 0
        self.finished: list[Request] = []
        self.build_pool = ThreadPoolExecutor(builders)
        # library-free board planning (requests whose build has .plan and
        # .realize, boards.SeededBoard) in processes of their own, beside the
        # builder threads: the mesher's Python work needs no library and
        # would otherwise hold the interpreter lock the builders share
        self.planners = None
        if planners:
            import multiprocessing
            from concurrent.futures import ProcessPoolExecutor
            self.planners = ProcessPoolExecutor(planners, mp_context=multiprocessing.get_context("spawn"))
        self.load_pool = ThreadPoolExecutor(2)
        self.finish_pool = ThreadPoolExecutor(finishers)
        self.loaded: list = []         # admitted and on the device, waiting to join the batch
        self.device = device
        self.stop = False
        self.gpu_ms = 0.0
        self.thread = threading.Thread(target=self._gpu_loop, daemon=True)
        self.thread.start()

    # ---- requests
    def submit(self, build, steps: int, tag=None) -> Request:
        r = Request(build, int(steps), tag, arrival=time.perf_counter())
        self.build_pool.submit(self._build, r)
        return r

    def _build(self, r: Request):
        try:
            if self.planners is not None and hasattr(r.build, "plan") and hasattr(r.build, "realize"):
                sim, meta = r.build.realize(self.lib, self.planners.submit(r.build.plan).result())
            else:
                sim, meta = r.build(self.lib)
            r.built = time.perf_counter()
            r.cells = meta.get("cells", sim.nx * sim.ny * sim.nz)
            nbytes = footprint(sim)
            if nbytes > self.budget:
                raise RuntimeError(f"needs {nbytes / 1e9:.1f} GB, above the {self.budget / 1e9:.1f} GB budget")
            with self.lock:
                self.built.append((r, sim, meta, nbytes))
        except Exception as e:   # reported on the request
            r.error = str(e)
            r.done = time.perf_counter()
            r.event.set()
        self.wake.set()

    # ---- the GPU thread
    def _load(self, item):
        r, sim, meta, nbytes = item
        try:
            sim.prepareDevice(self.device)
            r.loaded = time.perf_counter()
            with self.lock:
                self.loaded.append(item)
        except Exception as e:
            r.error = str(e)
            sim.destroy()
            with self.lock:
                self.used -= nbytes
            r.done = time.perf_counter()
            r.event.set()
        self.wake.set()

    def _admit(self):
        with self.lock:
            keep = []
            for item in self.built:
                r, sim, meta, nbytes = item
                if self.used + nbytes <= self.budget:
                    self.used += nbytes
                    r.admitted = time.perf_counter()
                    self.load_pool.submit(self._load, item)
                else:
                    keep.append(item)
            self.built = keep
            ready, self.loaded = self.loaded, []
        for item in ready:
            r, sim, meta, nbytes = item
            self.batch.add(sim, r.steps)
            self.members[sim.h] = item

    def _finish(self, item):
        r, sim, meta, nbytes = item
        try:
            r.result = results(sim, meta)
        except Exception as e:
            r.error = str(e)
        sim.destroy()
        with self.lock:
            self.used -= nbytes
        r.done = time.perf_counter()
        self.finished.append(r)
        r.event.set()
        self.wake.set()

    def _gpu_loop(self):
        while not self.stop:
            try:
                self._gpu_iteration()
            except Exception as e:   # a failed batched launch or device error: fail its requests, start afresh
                self._fail_all(f"batch failed: {e}")

    def _gpu_iteration(self):
        self._admit()
        if not self.members:
            self.wake.wait(0.01)
            self.wake.clear()
            return
        self.batch.run(self.chunk)
        self.gpu_ms += self.batch.stats()["ms"]
        for h, item in list(self.members.items()):
            sim = item[1]
            if self.batch.left(sim) == 0:
                item[0].stepped = time.perf_counter()
                self.batch.remove(sim)
                del self.members[h]
                self.finish_pool.submit(self._finish, item)

    def _fail_all(self, why: str):
        """Every request on the GPU side (batch members and loaded, not yet
        added) gets the error; their simulations are freed and their bytes
        returned to the budget, and the batch is replaced by a new one, so
        requests still building or queued are served afterwards."""
        with self.lock:
            items = list(self.members.values()) + self.loaded
            self.members, self.loaded = {}, []
        try:
            self.batch.destroy()
        except Exception:
            pass
        for r, sim, meta, nbytes in items:
            r.error = why
            try:
                sim.destroy()
            except Exception:
                pass
            with self.lock:
                self.used -= nbytes
            r.done = time.perf_counter()
            r.event.set()
        try:
            self.batch = self.lib.createBatch(self.device)
            self.batch.tune(self.tune)
        except Exception as e:   # no batch can be made: stop serving, fail what is left
            self.stop = True
            with self.lock:
                rest, self.built = self.built, []
            for r, sim, meta, nbytes in rest:
                r.error = f"server stopped: {e}"
                r.done = time.perf_counter()
                r.event.set()

    def close(self):
        self.stop = True
        self.wake.set()
        self.thread.join()
        self.build_pool.shutdown(wait=True)
        self.load_pool.shutdown(wait=True)
        self.finish_pool.shutdown(wait=True)
        if self.planners is not None:
            self.planners.shutdown(wait=True)
        self.batch.destroy()


def plain_loop(lib: Courant, requests: list[Request], arrivals: list[float]) -> list[Request]:
    """The baseline: each request alone, in arrival order (set-up, steps,
    results), waiting for its arrival time; arrivals relative to the start."""
    t0 = time.perf_counter()
    for r, at in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        r.arrival = t0 + at
        try:
            sim, meta = r.build(lib)
            r.built = time.perf_counter()
            r.cells = meta.get("cells", sim.nx * sim.ny * sim.nz)
            sim.prepareDevice()
            r.loaded = time.perf_counter()
            sim.step(r.steps)
            sim.synchronize()
            r.stepped = time.perf_counter()
            r.result = results(sim, meta)
            sim.destroy()
        except Exception as e:
            r.error = str(e)
        r.done = time.perf_counter()
    return requests


def serve_all(server: Server, requests: list[Request], arrivals: list[float]) -> list[Request]:
    """Submit the requests at their arrival times (relative to now) and wait for all."""
    t0 = time.perf_counter()
    out = []
    for r, at in zip(requests, arrivals):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        out.append(server.submit(r.build, r.steps, r.tag))
    for r in out:
        while not r.event.wait(0.5):
            if not server.thread.is_alive() and not r.event.is_set():   # the GPU thread has stopped
                r.error = r.error or "server stopped"
                r.done = time.perf_counter()
                r.event.set()
    return out


def summary(reqs: list[Request], t_start: float, t_end: float) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs if r.error is None])
    cells = sum(r.cells * r.steps for r in reqs if r.error is None)
    wall = t_end - t_start
    return {"solves": int(len(lat)), "errors": sum(r.error is not None for r in reqs), "wall_s": wall,
            "solves_per_hour": len(lat) / wall * 3600 if wall > 0 else None,
            "cell_updates_per_s": cells / wall if wall > 0 else None,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p95_s": float(np.percentile(lat, 95)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "stage_means_s": stage_means(reqs)}


def stage_means(reqs: list[Request]) -> dict:
    """Mean seconds per stage of the finished requests: waiting and host
    set-up (arrival to built), device state (to loaded), steps including the
    wait for the GPU (to the last step), results (S-parameters and freeing)."""
    ok = [r for r in reqs if r.error is None and r.built and r.loaded and r.stepped]
    if not ok:
        return {}
    mean = lambda v: float(np.mean(v))
    return {"setup": mean([r.built - r.arrival for r in ok]), "device": mean([r.loaded - r.built for r in ok]),
            "steps": mean([r.stepped - r.loaded for r in ok]), "results": mean([r.done - r.stepped for r in ok])}
