"""cemx_energy_noalloc: the energy reduction with its scratch in a static
device array instead of the simulation's buffers. It must return what
cem_energy returns, bit for bit, on consecutive calls, and refuse what it
cannot do without allocating. Named to be collected last, so it runs after
the other GPU tests in the same process as well as alone."""
import math

import numpy as np
import pytest

from courant_b200 import scenes
from courant_b200.api import CourantError


def test_noalloc_needs_device_state(lib):
    """Before the first step there is no device state, and this call never
    creates any (runs without a GPU: it fails before touching CUDA)."""
    s, _ = scenes.parity_scene(lib)
    try:
        with pytest.raises(CourantError, match="no device state"):
            s.energyNoAlloc()
    finally:
        s.destroy()


@pytest.mark.gpu
def test_noalloc_energy_matches_cem_energy(lib):
    s, _ = scenes.lossy_scene(lib)
    t, _ = scenes.parity_scene(lib)
    try:
        for steps in (120, 37):
            s.step(steps)
            t.step(steps)
            for sim in (s, t):
                ref = sim.energy()
                first, second = sim.energyNoAlloc(), sim.energyNoAlloc()
                assert ref > 0 and math.isfinite(ref)
                assert first == ref and second == ref
                assert sim.energy() == ref
    finally:
        s.destroy()
        t.destroy()


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_the_scratch(lib):
    """70001 x-planes of a 2x2 cross-section need 70001 block partials, above
    the 65536 of the static array: refused with a message, cem_energy works."""
    nx = 70000
    x = np.arange(nx + 1) * 1e-4
    y = np.arange(3) * 1e-4
    s = lib.createSim(x, y, y)
    try:
        s.finalize()
        s.step(1)
        with pytest.raises(CourantError, match="block partials"):
            s.energyNoAlloc()
        assert s.energy() == 0.0   # NaN if the device had failed
        s.step(1)
        assert s.steps == 2
    finally:
        s.destroy()


@pytest.mark.gpu
def test_noalloc_at_the_exact_capacity(lib):
    """65535 x-cells of a 2x2 cross-section need exactly 65536 block partials,
    the size of the static array, and two energy launches (grid y is split at
    65535 planes): accepted, and bit-equal to cem_energy on two calls in a row."""
    nx = 65535
    x = np.arange(nx + 1) * 1e-4
    y = np.arange(3) * 1e-4
    s = lib.createSim(x, y, y)
    try:
        p = s.addLumpedPort(2, 100, 1, 0, 2, -1, 50.0)
        s.setGaussian(p, 1.0, 8e-12, 2e-12)
        s.finalize()
        s.step(60)
        ref = s.energy()
        assert ref > 0 and math.isfinite(ref)
        assert s.energyNoAlloc() == ref and s.energyNoAlloc() == ref
    finally:
        s.destroy()
