"""The rule-based mesher (courant_b200/mesher.py, restating the reference's
web/src/mesh/mesher.ts) and the seeded boards built on it."""
import numpy as np
import pytest

from courant_b200 import boards, mesher


def test_fixed_lines_thirds_rule_and_grading():
    """Planes lie on the grid; a zero-thickness edge gets a line h/3 inside
    the metal and 2h/3 outside (mesher.ts :66-70); cells stay within the
    caps and grow by about the ratio away from refinement points."""
    h = 30e-6
    f = mesher.AxisFeatures(lo=0.0, hi=3e-3, sheet_edges=[(1e-3, "hi"), (1.5e-3, "lo")], planes=[2e-3])
    x = mesher.mesh_axis(f, h, 200e-6)
    for v in (0.0, 2e-3, 3e-3, 1e-3 + h / 3, 1e-3 - 2 * h / 3, 1.5e-3 - h / 3, 1.5e-3 + 2 * h / 3):
        assert np.min(np.abs(x - v)) < 1e-12, v
    c = np.diff(x)
    assert c.min() > 0 and c.max() <= 200e-6 * (1 + 1e-9)
    r = np.maximum(c[1:] / c[:-1], c[:-1] / c[1:])
    assert r.max() < 1.6


def test_spans_and_max_cells():
    f = mesher.AxisFeatures(lo=0.0, hi=2e-3, planes=[0.5e-3, 0.7e-3], spans=[(0.5e-3, 0.7e-3, 4)],
                            max_cell=[(0.0, 2e-3, 80e-6)])
    x = mesher.mesh_axis(f, 20e-6, 200e-6)
    inside = np.sum((x > 0.5e-3 + 1e-12) & (x < 0.7e-3 - 1e-12)) + 1
    assert inside >= 4
    assert np.diff(x).max() <= 80e-6 * (1 + 1e-9)


def test_close_lines_merge_keeping_priority():
    """Lines closer than hmin/4 merge; a plane (priority 2) wins over a thirds-rule line (1)."""
    h = 40e-6
    f = mesher.AxisFeatures(lo=0.0, hi=1e-3, planes=[0.5e-3], sheet_edges=[(0.5e-3 - h / 3 + 2e-6, "lo")])
    x = mesher.mesh_axis(f, h, 200e-6)
    assert np.min(np.abs(x - 0.5e-3)) < 1e-15
    assert np.sum(np.abs(x - 0.5e-3) < h / 4) == 1


def test_with_pml():
    x = mesher.with_pml(np.array([0.0, 1.0, 3.0]), 2, 0.5)
    assert np.allclose(x, [-1.0, -0.5, 0.0, 1.0, 3.0, 3.5, 4.0])
    z = mesher.with_pml(np.array([0.0, 1.0]), 2, 0.5, lo=False)
    assert np.allclose(z, [0.0, 1.0, 1.5, 2.0])


@pytest.mark.parametrize("cells", [6e4, 5e5])
def test_board_sizes_and_nonuniform_mesh(lib, cells):
    """A seeded board comes out near the requested size on a graded, non-uniform grid."""
    s, m = boards.seeded_board(lib, 3, cells, ports="mode", nf=2)
    try:
        assert 0.6 * cells < m["cells"] < 1.6 * cells
        for a in ("x", "y", "z"):
            r = m["mesh"][a]
            assert r["max_cell"] > 1.3 * r["min_cell"], a   # graded, not uniform
    finally:
        s.destroy()


def test_large_board_layout_is_the_large_configuration():
    """The 96 M-cell board's mesh (without building the simulation): 1500 x
    ~1000 x 64 cells, 20 traces and 30 vias, every cell positive."""
    lay = boards.draw_layout(2026, 20, 120)
    geo, hmin, x, y, z = boards.plan_mesh(lay, 96e6, 20e9, 8, 30, 4e-3, (1500, 1000, 64))
    nx, ny, nz = len(x) - 1, len(y) - 1, len(z) - 1
    assert abs(nx - 1500) <= 15 and nz == 64 and abs(ny - 1000) < 30
    assert len(geo.traces) == 20 and len(geo.vias) == 30
    for v in (x, y, z):
        assert np.all(np.diff(v) > 0)


def test_board_port_counts_and_windows():
    """1 to 4 ports: ports 1 and 2 on trace 0 (L4) with the whole cross-section, ports 3 and 4 on the
    second port trace (L3), whose window stops short of trace 0; an excitation outside the ports is refused."""
    one = boards.plan_board(41, 2e5, ports="mode", nf=2, nports=1)
    four = boards.plan_board(41, 2e5, ports="mode", nf=2, nports=4, excite=3)
    ny = len(four.y) - 1
    assert len(one.port) == 1 and len(four.port) == 4
    assert [p["end"] for p in four.port] == [0, 1, 0, 1]
    for p in four.port[:2]:
        assert (p["j0"], p["j1"]) == (0, ny) and p["vk1"] == four.kl[3]
    p3 = four.port[2]
    assert p3["vk1"] == four.kl[2] and (p3["j0"] > 0) != (p3["j1"] < ny)      # one wall, on trace 0's side
    assert not p3["j0"] <= four.port[0]["vj"] < p3["j1"]                     # trace 0 outside the window
    assert p3["neff0"] > four.port[0]["neff0"]                               # the covered line is slower
    for bad in (dict(nports=0), dict(nports=5), dict(nports=2, excite=3)):
        with pytest.raises(ValueError):
            boards.plan_board(41, 2e5, ports="mode", nf=2, **bad)


def test_s_column_takes_every_port():
    """The excited column of the S-matrix holds one wave per port (lumped ports at 50 ohm)."""
    from courant_b200 import scenes

    class Fake:
        def portV(self, p):
            return np.array([1.0 + p, 2.0])

        def portI(self, p):
            return np.array([0.01 * (p + 1), 0.02])
    for n in (1, 3, 4):
        col = scenes.s_column(Fake(), {"ports": list(range(n)), "excite": 1})
        assert len(col["b"]) == n
        a = (1.0 + 50 * 0.01) / (2 * np.sqrt(50))
        assert np.isclose(col["b"][0][0], (1.0 - 50 * 0.01) / (2 * np.sqrt(50)) / a)
