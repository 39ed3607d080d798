"""Serving with continuous batching (courant_b200/serve.py): requests that
arrive while others run are admitted as memory frees up, their work overlaps
on the GPU, and each result equals the result of the same request run alone
(bit for bit: the batched kernels compute exactly the per-simulation
arithmetic)."""
import functools

import numpy as np
import pytest

from courant_b200 import boards, scenes, serve

MIX = [  # (builder, steps)
    (functools.partial(boards.seeded_board, seed=1, cells=5e4, ports="lumped", nf=6), 1200),
    (functools.partial(boards.seeded_board, seed=2, cells=1.2e5, ports="lumped", nf=6, nports=3, excite=2), 800),
    (functools.partial(boards.seeded_board, seed=3, cells=6e4, ports="mode", nf=4, nports=4, excite=3), 1000),
    (lambda c: scenes.lossy_scene(c), 900),
]


def test_footprint_grows_with_the_grid(lib):
    a, _ = boards.seeded_board(lib, 1, 5e4, ports="lumped", nf=2)
    b, _ = boards.seeded_board(lib, 1, 4e5, ports="lumped", nf=2)
    fa, fb = serve.footprint(a), serve.footprint(b)
    assert 5e4 * 30 < fa < fb
    a.destroy()
    b.destroy()


@pytest.mark.gpu
def test_served_results_equal_alone(lib):
    alone = serve.plain_loop(lib, [serve.Request(b, n) for b, n in MIX], [0.0] * len(MIX))
    assert all(r.error is None for r in alone)
    # room for about two of these at a time: later requests wait for memory
    srv = serve.Server(lib, budget_bytes=2.5 * max(serve.footprint(b(lib)[0]) for b, _ in MIX), chunk=256)
    try:
        got = serve.serve_all(srv, [serve.Request(b, n) for b, n in MIX], [0.0, 0.02, 0.05, 0.08])
    finally:
        srv.close()
    for a, g in zip(alone, got):
        assert g.error is None, g.error
        keys = [k for k in a.result if k.startswith("S")]
        assert keys == [k for k in g.result if k.startswith("S")] and len(keys) >= 2
        for k in keys:
            assert np.array_equal(a.result[k], g.result[k]), k
    s = serve.summary(got, min(r.arrival for r in got), max(r.done for r in got))
    assert s["solves"] == len(MIX) and s["p50_s"] <= s["p99_s"]


@pytest.mark.gpu
def test_request_above_budget_is_refused(lib):
    srv = serve.Server(lib, budget_bytes=1e6)
    try:
        r = srv.submit(lambda c: boards.seeded_board(c, 1, 5e4, ports="lumped", nf=2), 10)
        r.event.wait(60)
        assert r.error and "budget" in r.error
    finally:
        srv.close()


class _FakeSim:
    """Host stand-in of a finalized simulation (what footprint and the server read)."""
    _next = 0

    def __init__(self):
        _FakeSim._next += 1
        self.h, self.nx, self.ny, self.nz = _FakeSim._next, 8, 8, 8
        self.destroyed = False

    def sizes(self):
        return {"psiE": 0, "psiH": 0, "npole": 0, "ndisp": 0, "sibc_terms": 0, "nsibc": 0}

    def prepareDevice(self, device=-1):
        pass

    def destroy(self):
        self.destroyed = True


class _FakeBatch:
    """The first batch fails on its first run (as a failed batched launch
    does); later batches finish every member in one run."""
    made = 0

    def __init__(self):
        _FakeBatch.made += 1
        self.fail = _FakeBatch.made == 1
        self.left_ = {}

    def tune(self, on=True):
        return True

    def add(self, sim, steps):
        self.left_[sim.h] = steps

    def run(self, n):
        if self.fail:
            from courant_b200.api import CourantError
            raise CourantError("batch: a batched launch failed")
        for h in self.left_:
            self.left_[h] = 0
        return 0

    def stats(self):
        return {"ms": 0.0}

    def left(self, sim):
        return self.left_[sim.h]

    def remove(self, sim):
        del self.left_[sim.h]

    def destroy(self):
        pass


class _FakeLib:
    def createBatch(self, device=-1):
        return _FakeBatch()


def test_failed_batch_fails_its_requests_and_serving_goes_on(monkeypatch):
    """A batched launch that raises fails the requests on the GPU with the
    error (their events set, bytes released); the server replaces the batch
    and serves the next request. Host-only: fake simulations and batches."""
    sims = []

    def build(c):
        s = _FakeSim()
        sims.append(s)
        return s, {"cells": 512}

    monkeypatch.setattr(serve, "results", lambda sim, meta: {"S1": np.zeros(1), "S2": np.zeros(1)})
    _FakeBatch.made = 0
    srv = serve.Server(_FakeLib(), budget_bytes=1e9, chunk=16, builders=1, finishers=1)
    try:
        first = srv.submit(build, 10)
        assert first.event.wait(10)
        assert first.error and "batched launch failed" in first.error
        assert sims[0].destroyed
        second = srv.submit(build, 10)
        assert second.event.wait(10)
        assert second.error is None and second.result is not None
        assert srv.thread.is_alive() and srv.used == 0
    finally:
        srv.close()


def test_board_plan_in_a_process_gives_the_same_board(lib):
    """A seeded board planned in a spawned process (the server's planners)
    and realized here has the plan of one built in one go."""
    import multiprocessing
    from concurrent.futures import ProcessPoolExecutor
    from tests_util import cmp_plans
    req = boards.SeededBoard(21, 8e4, ports="mode", nf=4)
    with ProcessPoolExecutor(1, mp_context=multiprocessing.get_context("spawn")) as pool:
        plan = pool.submit(req.plan).result()
    a, ma = req.realize(lib, plan)
    b, mb = req(lib)
    assert ma["dims"] == mb["dims"] and cmp_plans(a.plan(), b.plan()) == []
    a.destroy()
    b.destroy()
