"""The FP64 plan built on the host by libcourant_b200 equals the reference
plan to the bit: every cem_plan_* array and the fits (golden digests from
tests/golden/make_golden.py, and live against the reference library when it
is built). The 2D mode solver is this library's own (closed-form assembly,
PEC unknowns eliminated, its own band LU), so the mode-port source weights,
propagation constants and impedances it feeds into the plan agree with the
reference's to rounding: within 1e-9 relative (the reference's own platform
agreement is about 1e-6, docs/design/0003-mode-ports.md:61)."""
import numpy as np
import pytest

from courant_b200 import scenes
from tests_util import cmp_plans, mode_source_diff, plan_digest

MODE_TOL = 1e-9


@pytest.mark.parametrize("name,fn", [("parity", scenes.parity_scene), ("lossy", scenes.lossy_scene)])
def test_plan_digest_matches_reference(lib, golden, name, fn):
    s, _ = fn(lib)
    assert plan_digest(s.plan()) == golden[name]["plan"]
    assert s.dt == golden[name]["dt"]


@pytest.mark.parametrize("fn", [scenes.parity_scene, scenes.lossy_scene])
def test_plan_live_against_reference(lib, ref_lib, fn):
    a, _ = fn(ref_lib)
    b, _ = fn(lib)
    assert cmp_plans(a.plan(), b.plan()) == []


def test_gcpw_plan_live_against_reference(lib, ref_lib):
    kw = dict(length=2e-3, hmin=100e-6, hmax=400e-6, dx=200e-6, yair=0.6e-3, zair=0.8e-3, npml=6, nf=5,
              tcu=35e-6, mask=20e-6, debye_poles=4, sigma_cu=5.8e7, huray=(0.5e-6, 2.0e11))
    a, _ = scenes.gcpw_line(ref_lib, **kw)
    b, _ = scenes.gcpw_line(lib, **kw)
    assert cmp_plans(a.plan(), b.plan()) == []
    assert a.conductorFitError() == b.conductorFitError()


@pytest.mark.parametrize("ports,nports,excite", [("mode", 2, 1), ("lumped", 2, 1), ("mode", 1, 1),
                                                  ("mode", 3, 3), ("mode", 4, 2), ("lumped", 4, 4)])
def test_seeded_board_plan_live_against_reference(lib, ref_lib, ports, nports, excite):
    """The seeded board generator builds the same plan on both libraries
    (4-pole Debye stackup, ground plane with clearances, staircased traces,
    vias, 1 to 4 mode or lumped ports, any of them driven)."""
    from courant_b200 import boards
    kw = dict(ports=ports, nf=4, nports=nports, excite=excite)
    a, ma = boards.seeded_board(ref_lib, 11, 6e4, **kw)
    b, mb = boards.seeded_board(lib, 11, 6e4, **kw)
    assert ma["dims"] == mb["dims"] and ma["steps"] == mb["steps"]
    assert len(mb["modeports" if ports == "mode" else "ports"]) == nports
    pa, pb = a.plan(), b.plan()
    assert cmp_plans(pa, pb, skip=("modeSource",)) == []
    assert mode_source_diff(pa["modeSource"], pb["modeSource"]) < MODE_TOL


def test_seeded_board_is_deterministic(lib):
    from courant_b200 import boards
    a, _ = boards.seeded_board(lib, 5, 5e4, ports="lumped", nf=2)
    b, _ = boards.seeded_board(lib, 5, 5e4, ports="lumped", nf=2)
    c, _ = boards.seeded_board(lib, 6, 5e4, ports="lumped", nf=2)
    assert cmp_plans(a.plan(), b.plan()) == []
    assert cmp_plans(a.plan(), c.plan()) != []


def test_djordjevic_sarkar_fit(lib, golden):
    g = golden["ds_fit"]
    m = lib.fitDjordjevicSarkar(*g["args"])
    assert m.eps_inf == g["eps_inf"] and m.fp == g["fp"] and m.deps == g["deps"] and m.tan_delta_error == g["err"]


def test_mode2d_wr28(lib, golden):
    import ctypes as C
    g = golden["mode2d_wr28"]
    a, b, NY, NZ = 7.112e-3, 3.556e-3, 48, 24
    y = np.array([a * j / NY for j in range(NY + 1)])
    z = np.array([b * k / NZ for k in range(NZ + 1)])
    dp = C.POINTER(C.c_double)
    m = lib.ex.cem_mode2d_create(NY, NZ, y.ctypes.data_as(dp), z.ctypes.data_as(dp))
    f = 35e9
    k0 = 2 * np.pi * f / 299792458.0
    beta = np.sqrt(k0 ** 2 - (np.pi / a) ** 2)
    assert lib.ex.cem_mode2d_solve(m, f, beta / k0, None, 300, 1e-13) == g["rc"] == 0
    Rs = np.sqrt(2 * np.pi * f * 1.25663706212e-6 / (2 * 5.8e7))
    assert abs(lib.ex.cem_mode2d_beta(m) - g["beta"]) < 1e-11 * g["beta"]
    assert abs(lib.ex.cem_mode2d_conductor_alpha(m, Rs) - g["alpha_c"]) < 1e-9 * g["alpha_c"]
    assert abs(lib.ex.cem_mode2d_power(m) - g["power"]) < 1e-9 * g["power"]
    # the reference test's own acceptance: discrete-dispersion beta to 1e-8 (test_mode2d.c:22-31)
    dy = a / NY
    kcd = 2 / dy * np.sin(np.pi / a * dy / 2)
    assert abs(g["beta"] - np.sqrt(k0 ** 2 - kcd ** 2)) / g["beta"] < 1e-8
    lib.ex.cem_mode2d_destroy(m)


def test_mode_port_source_and_port_modes(lib, ref_lib, golden):
    """Source weights (live against the reference) and the port's Z0 and beta
    at every output frequency (golden) of a small GCPW between mode ports."""
    g = golden["modeport_small"]
    kw = dict(length=2e-3, hmin=100e-6, hmax=400e-6, dx=200e-6, yair=0.6e-3, zair=0.8e-3,
              npml=6, feed=2e-3, mon=0.8e-3, nf=4, modeports=True, steps=300)
    s, meta = scenes.gcpw_line(lib, **kw)
    r, _ = scenes.gcpw_line(ref_lib, **kw)
    assert len(s.plan()["modeSource"]["idx"]) > 0
    assert mode_source_diff(r.plan()["modeSource"], s.plan()["modeSource"]) < MODE_TOL
    w = s.modePortWaves(meta["modeports"][0])   # port modes solved on the host, no stepping needed
    assert np.max(np.abs(w["z0"] - np.array(g["z0"])) / np.abs(g["z0"])) < MODE_TOL
    assert np.max(np.abs(w["beta"] - np.array(g["beta"])) / np.abs(g["beta"])) < MODE_TOL


def test_s2_renormalize(lib, ref_lib):
    rng = np.random.default_rng(7)
    for _ in range(20):
        S = list(rng.normal(size=4) * 0.4 + 1j * rng.normal(size=4) * 0.4)
        z1, z2 = rng.uniform(20, 80, size=2)
        assert lib.renormalize2(S, z1, z2, 50.0) == ref_lib.renormalize2(S, z1, z2, 50.0)


@pytest.mark.parametrize("case", ["board4", "modeport"])
def test_mode_port_walks_against_reference(lib, ref_lib, case):
    """Port impedance and propagation constant at every output frequency (the
    walk outward from f0, each solve seeded with the previous mode; this
    library solves the starting frequency once for both walks and takes
    finalize's solve there when f0 is an output frequency) agree with the
    reference's to rounding. No time steps are needed."""
    from courant_b200 import boards

    def make(c):
        if case == "board4":
            return boards.seeded_board(c, 32, 2.5e5, ports="mode", nf=8, nports=4, excite=3)
        return scenes.modeport_scene(c)
    (a, ma), (b, _) = make(lib), make(ref_lib)
    for p in ma["modeports"]:
        wa, wb = a.modePortWaves(p), b.modePortWaves(p)
        for k in ("z0", "beta"):
            assert np.max(np.abs(wa[k] - wb[k]) / np.abs(wb[k])) < 1e-8, (p, k)
    a.destroy()
    b.destroy()
