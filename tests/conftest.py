"""Shared fixtures. Tests marked `gpu` need a CUDA device (a B200); the rest
run on CPU: the C ABI surface, the FP64 host plan against the reference's, the
oracle restatement against the reference's own results, and host logic."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_CUDA = _has_cuda()


@pytest.fixture(scope="session")
def lib():
    from courant_b200 import build
    from courant_b200.api import Courant
    if build.needs_build():
        build.build()
    return Courant()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    if not oracle.LIB.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "restatement"], check=True, capture_output=True)
    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def ref_lib():
    from courant_b200.api import Courant
    import oracle
    if not oracle.REF_LIB.exists():
        pytest.skip("reference library oracle/_ref/libcourant_ref.so not built")
    return Courant(oracle.REF_LIB)


@pytest.fixture(scope="session")
def golden():
    return json.loads((GOLDEN / "golden.json").read_text())
