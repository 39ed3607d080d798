"""The C ABI surface: every function of include/courant.h is exported by
libcourant_b200.so, and the setup calls keep the reference's error behaviour
(return -1 and set cem_last_error)."""
import re
import subprocess

import numpy as np
import pytest

from conftest import HAS_CUDA, ROOT


def declared_functions(header="courant.h"):
    text = (ROOT / "include" / header).read_text()
    return sorted(set(re.findall(r"CEM_API[^;(]*?\b(cemx?_\w+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) == 91
    ext = declared_functions("courant_b200.h")
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib.path)], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines()}
    missing = [n for n in names + ext if n not in exported]
    assert not missing, missing
    extra = sorted(exported - set(names) - set(ext))
    assert not extra, extra


def test_python_binding_covers_abi(lib):
    from courant_b200.api import API_NAMES
    assert sorted(API_NAMES) == declared_functions()


def test_version(lib):
    assert lib.version().startswith("20261017.0")


def test_setup_errors_match_reference(lib):
    x = np.linspace(0, 1e-3, 11)
    assert not lib.ex.cem_create(1, 10, 10, None, None, None)
    assert lib.last_error() == "grid needs at least 2 cells per axis"
    bad = x.copy()
    bad[3] = bad[2]
    from courant_b200.api import CourantError
    with pytest.raises(CourantError, match="strictly increasing"):
        lib.createSim(bad, x, x)
    s = lib.createSim(x, x, x)
    with pytest.raises(CourantError, match="bad CPML thickness"):
        s.setBoundary(0, 1, 5)
    with pytest.raises(CourantError, match="bad face"):
        s.setBoundary(7, 0, 0)
    with pytest.raises(CourantError, match="bad port definition"):
        s.addLumpedPort(2, 3, 3, 0, 11, 1, 50.0)
    with pytest.raises(CourantError, match="bad current probe"):
        s.addIProbe(0, 3, 5, 5, 1, 2)
    with pytest.raises(CourantError, match="set Debye poles first"):
        from courant_b200.api import DebyeModel
        s.materialBoxDebye(0, 1, 0, 1, 0, 1, DebyeModel(1.0, [], [0.1], 0))
    s.setFrequencies([1e9])
    s.finalize(0.99)
    with pytest.raises(CourantError, match="already finalized"):
        s.pecBox(0, 1, 0, 1, 0, 1)
    with pytest.raises(CourantError, match="already finalized"):
        s.finalize(0.99)


def test_port_on_pec_edge_rejected(lib):
    x = np.linspace(0, 1e-3, 11)
    s = lib.createSim(x, x, x)
    s.pecBox(-1, 1, -1, 1, -1, 1)
    s.addLumpedPort(2, 5, 5, 2, 4, 1, 50.0)
    from courant_b200.api import CourantError
    with pytest.raises(CourantError, match="port edge is PEC"):
        s.finalize(0.99)


@pytest.mark.skipif(HAS_CUDA, reason="checks the failure path of a host without a GPU")
def test_step_without_gpu_fails_loudly(lib, capfd):
    from courant_b200 import scenes
    from courant_b200.api import CourantError
    s, _ = scenes.parity_scene(lib)
    with pytest.raises(CourantError, match="no CUDA device"):
        s.step(3)
    assert s.steps == 0
    assert "no CUDA device" in capfd.readouterr().err


@pytest.mark.skipif(HAS_CUDA, reason="checks the no-GPU path")
def test_batch_without_gpu_fails_loudly(lib):
    from courant_b200.api import CourantError
    with pytest.raises(CourantError, match="no CUDA device"):
        lib.createBatch()


def test_field_pointer_before_finalize_is_writable(lib):
    x = np.linspace(0, 1e-3, 5)
    s = lib.createSim(x, x, x)
    v = s.fieldView(1)
    v[:] = 2.0
    assert np.all(s.field(1) == 2.0)
    assert s.index(1, 2, 3) == 1 * 25 + 2 * 5 + 3
