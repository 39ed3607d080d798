"""The benchmark configurations at their full step counts, against the f64
reference core.

The fixtures tests/golden/sparams_<config>.json hold the reference's own
S-parameters after the whole run (tests/golden/make_sparams.py, both
excitations). The gate on every S-parameter column, f >= 1 GHz:

* transmission (S21 driven at port 1, S12 driven at port 2): within 1e-3 dB
  in magnitude and 0.01 degree in phase;
* reflection (S11, S22): the same dB/degree gate where |S| is above -30 dB
  (the reference's own S11 rule applies only above -30 dB,
  tools/compare_s2p.py:7), and everywhere an absolute complex difference
  below 1e-4 of the incident wave, which is the dB gate's size at -30 dB.

Each test prints its worst errors, the figures quoted for the configuration.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from courant_b200 import scenes
from tests_util import db_deg, rel_l2

pytestmark = pytest.mark.gpu

DB_TOL, DEG_TOL, ABS_TOL = 1e-3, 0.01, 1e-4


def golden_sparams(name):
    p = GOLDEN / f"sparams_{name}.json"
    if not p.exists():
        pytest.skip(f"{p.name} not generated")
    return json.loads(p.read_text())


def _c(pairs):
    return np.array([complex(a, b) for a, b in pairs])


def column_errors(col, ref_run, excite):
    """Worst dB / degree / absolute errors of one S-matrix column against the reference's."""
    f = np.asarray(ref_run["freqs"])
    sel = f >= 1e9
    out = {}
    for q in range(len(ref_run["S"])):
        g, r = np.asarray(col["b"][q])[sel], _c(ref_run["S"][q])[sel]
        name = f"S{q + 1}{excite}"
        transmit = q + 1 != excite
        keep = np.ones(len(r), bool) if transmit else np.abs(r) > 10 ** (-30 / 20)
        ddb, ddeg = db_deg(g[keep], r[keep]) if keep.any() else (np.zeros(1), np.zeros(1))
        out[name] = {"db": float(ddb.max()), "deg": float(ddeg.max()), "abs": float(np.abs(g - r).max()),
                     "transmission": transmit}
    return out


def check(errs):
    for name, e in errs.items():
        assert e["db"] < DB_TOL and e["deg"] < DEG_TOL, (name, e)
        if not e["transmission"]:
            assert e["abs"] < ABS_TOL, (name, e)


@pytest.mark.parametrize("excite", [1, 2])
def test_c1_full_run_sparams(lib, excite):
    """Lossless GCPW, lumped ports, 121 x 62 x 40 cells, 20 000 steps, 401
    frequencies: both S-matrix columns against the reference core's."""
    gold = golden_sparams("c1")
    ref = gold["runs"][excite - 1]
    s, meta = scenes.config_line(lib, "c1", excite=excite)
    assert list(meta["dims"]) == ref["dims"] and s.dt == ref["dt"]
    s.step(meta["steps"])
    errs = column_errors(scenes.two_port_s(s, meta), ref, excite)
    print("c1 excite", excite, errs)
    check(errs)


def test_c1_fields_against_reference_live(lib, ref_lib):
    """C1 fields against the reference core run beside it: after 1 000 steps
    (the pulse on the line, fields near their peak) every component within
    relative L2 1e-5; after 3 000 steps, when the pulse has reached the
    ports and the fields decay, within 1e-5 of the largest norm the
    component's family (E or H) reached, the measure of the other scene
    tests (FP32 rounding scales with the peak field, not the decayed one)."""
    s, meta = scenes.config_line(lib, "c1")
    r, _ = scenes.config_line(ref_lib, "c1")
    peak = np.zeros(6)
    done = 0
    for upto in (500, 1000, 1500, 2000, 2500, 3000):
        s.step(upto - done)
        r.step(upto - done)
        done = upto
        peak = np.maximum(peak, [np.linalg.norm(r.field(c)) for c in range(6)])
        if upto == 1000:
            errs = [rel_l2(s.field(c), r.field(c)) for c in range(6)]
            print("c1 fields rel L2 at 1000 steps", errs)
            assert max(errs) < 1e-5, errs
    fam = np.repeat([peak[:3].max(), peak[3:].max()], 3)
    errs = [float(np.linalg.norm(s.field(c) - r.field(c)) / fam[c]) for c in range(6)]
    print("c1 fields at 3000 steps, relative to the family peak", errs)
    assert max(errs) < 1e-5, errs
    for p in meta["ports"]:
        v, vr = s.portV(p), r.portV(p)
        assert np.max(np.abs(v - vr)) / np.max(np.abs(vr)) < 1e-5


@pytest.mark.parametrize("excite", [1, 2])
def test_c2_full_run_sparams(lib, excite):
    """Lossy GCPW between 2D mode ports (6-pole Debye substrate, Huray SIBC,
    mask), 416 x 161 x 86 cells, 40 000 steps, 400 frequencies: both modal
    S-matrix columns against the reference core's, and the port impedances of
    the mode solves at every frequency (within 1e-6 relative, the reference's
    own agreement across platforms, docs/design/0003-mode-ports.md:61; this
    library's solver differs from the reference's by up to 2.4e-8 at 5 GHz)."""
    gold = golden_sparams("c2")
    ref = gold["runs"][excite - 1]
    s, meta = scenes.config_line(lib, "c2", excite=excite)
    assert list(meta["dims"]) == ref["dims"] and s.dt == ref["dt"]
    s.step(meta["steps"])
    col = scenes.two_port_s(s, meta)
    for q in range(2):
        z, zr = np.asarray(col["z0"][q]), np.asarray(ref["z0"][q])
        assert np.max(np.abs(z - zr) / np.abs(zr)) < 1e-6
    errs = column_errors(col, ref, excite)
    print("c2 excite", excite, errs)
    check(errs)


@pytest.mark.parametrize("seed,nports,excite", [(31, 2, 1), (31, 2, 2), (32, 4, 3), (31, 1, 1)])
def test_large_board_generator_scaled_against_reference(lib, ref_lib, seed, nports, excite):
    """A board from the large configuration's generator (4-layer stackup with
    4-pole Debye cores, traces with 45-degree jogs, vias, plane clearances,
    rule-based non-uniform mesh, 2D mode ports) at 2.5e5 cells, 5 000 steps,
    16 frequencies: both excitations of the 2-port board, the second trace
    driven on a 4-port one, and a 1-port one; the modal S-matrix columns
    against the reference core run on the same plan beside it, within the
    gate. (The 4-port board is seed 32: on seed 31 the reference's own mode
    solver does not converge for the second trace's port at one of the 16
    frequencies within its 300 iterations, and this library's, which refines
    its shift when an iteration stalls, does.)"""
    from courant_b200 import boards
    kw = dict(seed=seed, cells=2.5e5, ports="mode", nf=16, steps=5000, excite=excite, nports=nports)
    s, meta = boards.seeded_board(lib, **kw)
    r, mr = boards.seeded_board(ref_lib, **kw)
    assert meta["dims"] == mr["dims"] and meta["cells"] >= 2e5
    assert meta["mesh"]["y"]["max_cell"] > 1.3 * meta["mesh"]["y"]["min_cell"]   # non-uniform
    s.step(meta["steps"])
    r.step(meta["steps"])
    col, rcol = scenes.two_port_s(s, meta), scenes.two_port_s(r, mr)
    ref = {"freqs": list(meta["freqs"]),
           "S": [[[complex(v).real, complex(v).imag] for v in b] for b in rcol["b"]]}
    errs = column_errors(col, ref, excite)
    print("board ports", nports, "excite", excite, meta["dims"], errs)
    check(errs)
