"""Pins the oracle restatement (oracle/fdtd_oracle.c) to the reference core.

Driven by the plan the reference library exports, the restatement must give
the reference's cem_step results bit for bit: every field component, every
port/probe/source spectrum and the energy, on the every-feature lossless
parity scene (reference solver/apps/parity.c) and the lossy checkpoint scene
(Debye poles + copper surface impedance, solver/tests/test_checkpoint.c), and
on a small lossy GCPW between 2D mode ports (modal source plane). It must
also reproduce the committed reference results in tests/golden/golden.json
(spectra, energy and field checksums made by tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from courant_b200 import scenes


def _same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


def _spectra(x, meta):
    out = []
    for p in meta.get("ports", []):
        out += [x.portV(p), x.portI(p)]
    for p in meta.get("vprobes", []):
        out.append(x.vprobe(p))
    for p in meta.get("iprobes", []):
        out.append(x.iprobe(p))
    out.append(x.sourceSpectrum())
    return out


def small_modeport(c):
    return scenes.gcpw_line(c, length=2e-3, hmin=100e-6, hmax=400e-6, dx=200e-6, yair=0.6e-3, zair=0.8e-3,
                            npml=6, feed=2e-3, mon=0.8e-3, nf=4, tcu=35e-6, mask=20e-6, debye_poles=4,
                            sigma_cu=5.8e7, huray=(0.5e-6, 2.0e11), modeports=True, probes=True, steps=500)


@pytest.mark.parametrize("fn", [scenes.parity_scene, scenes.lossy_scene, small_modeport],
                         ids=["parity", "lossy", "modeport"])
def test_restatement_equals_reference_bit_for_bit(ref_lib, oracle_lib, fn):
    r, meta = fn(ref_lib)
    n = meta["steps"]
    o = oracle_lib.OracleSim.from_sim(r, meta["freqs"], n)
    for chunk in (n // 3, n - n // 3):
        r.step(chunk)
        o.step(chunk)
        for c in range(6):
            assert _same_bits(o.field(c), r.field(c)), c
    assert o.steps == r.steps == n
    for a, b in zip(_spectra(o, meta), _spectra(r, meta)):
        assert _same_bits(a.view(np.float64), b.view(np.float64))
    assert o.energy() == r.energy()


@pytest.mark.parametrize("name,fn", [("parity", scenes.parity_scene), ("lossy", scenes.lossy_scene)])
def test_restatement_reproduces_golden_results(ref_lib, oracle_lib, golden, name, fn):
    """Spectra, energy and field checksums of the reference run recorded in
    golden.json, reproduced by the restatement over the reference plan."""
    g = golden[name]
    r, meta = fn(ref_lib)
    assert r.dt == g["dt"]
    o = oracle_lib.OracleSim.from_sim(r, meta["freqs"], g["steps"])
    o.step(g["steps"])
    assert o.energy() == g["energy"]

    def cpx(pairs):
        return np.array([complex(a, b) for a, b in pairs])

    for q, p in enumerate(meta["ports"]):
        assert np.array_equal(o.portV(p), cpx(g["portV"][q]))
        assert np.array_equal(o.portI(p), cpx(g["portI"][q]))
    assert np.array_equal(o.vprobe(meta["vprobes"][0]), cpx(g["vprobe"][0]))
    assert np.array_equal(o.iprobe(meta["iprobes"][0]), cpx(g["iprobe"][0]))
    assert np.array_equal(o.sourceSpectrum(), cpx(g["source"]))
    for c in range(6):
        f = o.field(c)
        ref = g["fields"][c]
        assert float(np.abs(f).max()) == ref["maxabs"]
        assert abs(float((f * f).sum()) - ref["sumsq"]) <= 1e-12 * ref["sumsq"]
        assert abs(float(f.sum()) - ref["sum"]) <= 1e-9 * max(abs(ref["sum"]), ref["maxabs"])


def test_parity_printout_matches_restatement(ref_lib, oracle_lib):
    """The reference's known-answer printout (solver/apps/parity.c output,
    tests/golden/parity_scene.txt, 17 significant digits) from the restatement."""
    from conftest import GOLDEN
    ref = {}
    for line in (GOLDEN / "parity_scene.txt").read_text().splitlines():
        k, *v = line.split()
        ref[k] = [float(x) for x in v]
    r, meta = scenes.parity_scene(ref_lib)
    o = oracle_lib.OracleSim.from_sim(r, meta["freqs"], 1500)
    o.step(1500)
    assert float(f"{o.energy():.17g}") == ref["energy"][0]
    arrs = {"V1": o.portV(0), "V2": o.portV(1), "Vp": o.vprobe(0), "Ip": o.iprobe(0)}
    for name, a in arrs.items():
        for q in range(3):
            assert [float(f"{a[q].real:.17g}"), float(f"{a[q].imag:.17g}")] == ref[f"{name}[{q}]"], (name, q)
