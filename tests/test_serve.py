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
    (functools.partial(boards.seeded_board, seed=2, cells=1.2e5, ports="lumped", nf=6), 800),
    (functools.partial(boards.seeded_board, seed=3, cells=6e4, ports="mode", nf=4), 1000),
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
        for k in ("S11", "S21"):
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
