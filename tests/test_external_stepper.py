"""The reference's external-stepper contract (solver/src/export.c): the
sample feed cem_push_samples (:115-149) and the writable state arrays
cem_state_array / cem_state_len (:244-268).

An engine that keeps its own copy of the fields records, per step, the
current-probe values at H time, the port voltages before and after the E
update and the voltage-probe values at E time, and pushes them into the core,
which folds them into exactly the DFTs cem_step would accumulate. The samples
here are recorded from the reference core itself, stepped phase by phase
(cem_mt_pre/H/mid/E/post), with the plan's edge indices and weights.
"""
import ctypes as C

import numpy as np
import pytest

from courant_b200 import scenes
from tests_util import rel_l2


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _weighted(fields, idx, w):
    """sum_e w_e * field[idx_e] over global indices comp * N + q."""
    idx = idx.astype(np.int64)
    N = fields[0].size
    return float(sum(fields[int(g // N)][int(g % N)] * wt for g, wt in zip(idx, w)))


def record_samples(sim, n):
    """Step the reference core `n` steps phase by phase and record the
    external-stepper samples of every step (step-major layout)."""
    plan = sim.plan()
    ex, h = sim.c.ex, sim.h
    views = [sim.fieldView(c) for c in range(6)]
    ip, vold, vnew, vp = [], [], [], []
    for _ in range(n):
        ex.cem_mt_pre(h)
        ex.cem_mt_H(h, 0, sim.nx + 1)
        ip += [_weighted(views[3:], q["idx"], q["w"]) for q in plan["iprobes"]]   # H indices (comp - 3) * N + q
        vold += [_weighted(views, q["idx"], q["vw"]) for q in plan["ports"]]
        ex.cem_mt_mid(h)
        ex.cem_mt_E(h, 0, sim.nx)
        ex.cem_mt_post(h)
        vnew += [_weighted(views, q["idx"], q["vw"]) for q in plan["ports"]]
        vp += [_weighted(views, q["idx"], q["w"]) for q in plan["vprobes"]]
    return [np.array(a, dtype=np.float64) for a in (ip, vold, vnew, vp)]


def _spectra(s, meta):
    out = [s.portV(p) for p in meta["ports"]] + [s.portI(p) for p in meta["ports"]]
    out += [s.vprobe(p) for p in meta["vprobes"]] + [s.iprobe(p) for p in meta["iprobes"]]
    return out + [s.sourceSpectrum()]


@pytest.mark.parametrize("fn", [scenes.parity_scene, scenes.lossy_scene], ids=["parity", "lossy"])
def test_push_samples_gives_the_reference_dfts(ref_lib, lib, fn):
    """Samples recorded from the reference, pushed into a fresh simulation of
    each library: both libraries accumulate the same bits, and the spectra
    match the reference's own stepped DFTs (which advance their phasors by
    rotation, so they agree to rounding, not bits)."""
    n = 240
    R, meta = fn(ref_lib)
    samples = record_samples(R, n)
    got = []
    for c in (ref_lib, lib):
        s, _ = fn(c)
        s.c.ex.cem_push_samples(s.h, n, *[_ptr(a) for a in samples])
        assert s.steps == n
        got.append(_spectra(s, meta))
    for a, b in zip(*got):
        assert np.array_equal(a, b)
    for a, r in zip(got[1], _spectra(R, meta)):
        assert np.max(np.abs(a - r)) <= 1e-9 * max(np.max(np.abs(r)), 1e-300)


def test_state_lengths_match_the_reference(ref_lib, lib):
    """cem_state_len of every state array (compact CPML layout, Debye J and
    E_old, SIBC states) is the reference's on the lossy scene."""
    R, _ = scenes.lossy_scene(ref_lib)
    B, _ = scenes.lossy_scene(lib)
    for which in range(5):
        for comp in range(3):
            for w in range(2):
                assert B.stateLen(which, comp, w) == R.stateLen(which, comp, w), (which, comp, w)
    assert B.stateLen(2) > 0 and B.stateLen(4) > 0 and B.stateLen(0, 0, 0) > 0


def _state(sim, which, comp=0, w=0):
    n = sim.stateLen(which, comp, w)
    p = sim.c.ex.cem_state_array(sim.h, which, comp, w)
    return np.ctypeslib.as_array(p, shape=(n,)) if n else np.zeros(0)


@pytest.mark.gpu
def test_state_arrays_round_trip_on_device(lib, ref_lib):
    """After 600 steps the GPU engine's state arrays, read through
    cem_state_array in the reference's compact layout, match the reference
    core's (FP32 state against f64: relative L2 <= 2e-4; the CPML and Debye
    recursions are driven by differences of nearly equal field values -
    neighbouring points, or one point before and after its update - so their
    FP32 rounding is larger than the fields'). The reference's arrays and
    fields written into the engine through the same pointers are taken up:
    150 steps later the E and H fields are within relative L2 1e-5 of the
    reference, and no further from it than a second engine run that never
    took the reference's state."""
    G, _ = scenes.lossy_scene(lib)
    G2, _ = scenes.lossy_scene(lib)
    R, _ = scenes.lossy_scene(ref_lib)
    for x in (G, G2, R):
        x.step(600)
    keys = [(0, c, w) for c in range(3) for w in range(2)] + [(1, c, w) for c in range(3) for w in range(2)]
    keys += [(2, 0, 0), (4, 0, 0)]
    for k in keys:
        g, r = _state(G, *k), _state(R, *k)
        assert g.shape == r.shape, k
        if np.linalg.norm(r) > 0:
            assert rel_l2(g, r) < 2e-4, k
    # write the reference's state (and fields) into the engine through the live pointers
    for k in keys:
        _state(G, *k)[:] = _state(R, *k)
    for c in range(6):
        G.fieldView(c)[:] = R.field(c)
    for x in (G, G2, R):
        x.step(150)
    for fam in (range(3), range(3, 6)):
        den = np.sqrt(sum(np.linalg.norm(R.field(c)) ** 2 for c in fam))
        err = np.sqrt(sum(np.linalg.norm(G.field(c) - R.field(c)) ** 2 for c in fam)) / den
        err2 = np.sqrt(sum(np.linalg.norm(G2.field(c) - R.field(c)) ** 2 for c in fam)) / den
        assert err < 1e-5 and err <= err2, (list(fam), err, err2)
