"""Batches (cemx_batch_*): simulations of different sizes, pole counts and
step budgets advanced together must give exactly what each gives alone with
cem_step, stop at their own budgets, and keep doing so when members leave,
join between runs, or the batch tunes its graph length and work order."""
import numpy as np
import pytest

from courant_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = [scenes.parity_scene, scenes.lossy_scene, scenes.modeport_scene]


def results(s, meta):
    out = {f"f{c}": s.field(c) for c in range(6)}
    for p in meta.get("ports", []):
        out[f"V{p}"], out[f"I{p}"] = s.portV(p), s.portI(p)
    for p in meta.get("vprobes", []):
        out[f"vp{p}"] = s.vprobe(p)
    for p in meta.get("iprobes", []):
        out[f"ip{p}"] = s.iprobe(p)
    out["src"] = s.sourceSpectrum()
    out["energy"] = np.array([s.energy()])
    return out


def assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def alone(lib, fn, n):
    s, meta = fn(lib)
    s.step(n)
    r = results(s, meta)
    s.destroy()
    return r


@pytest.mark.parametrize("tune", [False, True], ids=["fixed", "tuned"])
def test_batch_matches_alone(lib, tune):
    budgets = [700, 450, 1100]
    ref = [alone(lib, fn, n) for fn, n in zip(SCENES, budgets)]
    b = lib.createBatch()
    b.tune(tune)
    sims = [fn(lib) for fn in SCENES]
    for (s, _), n in zip(sims, budgets):
        b.add(s, n)
    left = b.run(300)                   # every member advances 300 steps
    assert left == 3
    assert [s.steps for s, _ in sims] == [300, 300, 300]
    while b.run(10_000):                # each stops at its own budget
        pass
    assert [s.steps for s, _ in sims] == budgets
    assert [b.left(s) for s, _ in sims] == [0, 0, 0]
    for (s, meta), r in zip(sims, ref):
        assert_same(results(s, meta), r)
    st = b.stats()
    assert st["members"] == 3
    b.destroy()
    for s, _ in sims:
        s.destroy()


def test_batch_members_join_and_leave(lib):
    """A member added after others ran, and one removed part-way, still match."""
    ref_par = alone(lib, scenes.parity_scene, 900)
    ref_lossy = alone(lib, scenes.lossy_scene, 500)
    b = lib.createBatch()
    p, pm = scenes.parity_scene(lib)
    q, qm = scenes.lossy_scene(lib)
    x, _ = scenes.parity_scene(lib)
    b.add(p, 900)
    b.add(x, 900)
    b.run(256)
    b.add(q, 500)                        # joins at a chunk boundary
    b.run(100)
    b.remove(x)                          # leaves; stepping it alone afterwards still works
    x.step(3)
    while b.run(1000):
        pass
    assert p.steps == 900 and q.steps == 500 and x.steps == 359
    assert_same(results(p, pm), ref_par)
    assert_same(results(q, qm), ref_lossy)
    b.destroy()
    for s in (p, q, x):
        s.destroy()


def test_batch_rejects_misuse(lib):
    from courant_b200.api import CourantError
    b = lib.createBatch()
    s, _ = scenes.parity_scene(lib)
    b.add(s, 10)
    with pytest.raises(CourantError, match="already a member"):
        b.add(s, 10)
    with pytest.raises(CourantError, match="negative"):
        t, _ = scenes.parity_scene(lib)
        b.add(t, -1)
    assert b.run(5) == 1 and s.steps == 5
    assert b.run(100) == 0 and s.steps == 10
    b.destroy()
    s.destroy()


@pytest.mark.gpu
def test_launch_shape_tuner_chooses_caches_and_keeps_the_bits(lib, tmp_path, monkeypatch):
    """cemx_tune: the first long cem_step call times the launch-shape choices
    on the simulation's own steps and writes the choice for the grid shape to
    the cache file; a second simulation of the same shape takes it from the
    file; fields are the bits of an untuned run."""
    cache = tmp_path / "shapes.txt"
    monkeypatch.setenv("CEM_B200_TUNE_CACHE", str(cache))
    from courant_b200 import boards
    kw = dict(seed=77, cells=3e5, ports="lumped", nf=4, steps=3000)
    plain, _ = boards.seeded_board(lib, **kw)
    a, _ = boards.seeded_board(lib, **kw)
    b, _ = boards.seeded_board(lib, **kw)
    a.tune(True)
    b.tune(True)
    for x in (plain, a):
        x.step(3000)
    st = a.tuneState()
    assert st["tuned"] and not st["from_cache"] and st["thin"] in (8, 16, 32) and st["graph_steps"] in (16, 32, 64)
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].split()[0].startswith(f"{a.nx}x{a.ny}x{a.nz}/")
    b.step(3000)
    sb = b.tuneState()
    assert sb["tuned"] and sb["from_cache"]
    assert (sb["thin"], sb["graph_steps"], sb["z_tails"]) == (st["thin"], st["graph_steps"], st["z_tails"])
    for c in range(6):
        assert np.array_equal(a.field(c), plain.field(c)) and np.array_equal(b.field(c), plain.field(c)), c
    for x in (plain, a, b):
        x.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["board", "lossy"])
def test_z_tails_give_the_bits_of_general_blocks(lib, monkeypatch, which):
    """The z CPML slab run inside the lean kernels' rows (z tails,
    CEM_B200_ZTAIL=1), as rectangles of their own in the lean space
    (CEM_B200_ZTAIL=2, the form of the default from 2 M cells), as separate
    general blocks (CEM_B200_ZTAIL=0), and inside whole E rows of the Debye
    space (CEM_B200_ROWS=1) give the same fields and spectra bit for bit, on a
    seeded board (z-high CPML above air, Debye cores below) and on the lossy
    scene."""
    from courant_b200 import boards

    def make():
        if which == "board":
            return boards.seeded_board(lib, seed=78, cells=3e5, ports="mode", nf=4, steps=1200)
        return scenes.lossy_scene(lib)
    runs = []
    for zt, rows in (("1", "0"), ("0", "0"), ("1", "1"), ("2", "0")):
        monkeypatch.setenv("CEM_B200_ZTAIL", zt)
        monkeypatch.setenv("CEM_B200_ROWS", rows)
        s, meta = make()
        s.step(1200)
        runs.append((s, meta))
    (a, ma), (b, _), (w, _), (t, _) = runs
    za, zb = a.sizes(), b.sizes()
    assert za["h_general_pts"] < zb["h_general_pts"]
    if which == "board":
        assert za["e_general_pts"] < zb["e_general_pts"]
        assert w.sizes()["e_fast_pts"] < za["e_fast_pts"]     # whole rows: the air above the cores in the Debye space
    assert t.sizes()["e_general_pts"] == za["e_general_pts"]
    for x in (b, w, t):
        for c in range(6):
            assert np.array_equal(a.field(c), x.field(c)), c
        if "modeports" in ma:
            for p in ma["modeports"]:
                assert np.array_equal(a.modePortWaves(p)["b"], x.modePortWaves(p)["b"])
        for p in ma.get("ports", []):
            assert np.array_equal(a.portV(p), x.portV(p))
    for x in (a, b, w, t):
        x.destroy()
