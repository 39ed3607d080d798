"""Generate the golden fixtures in tests/golden/ from the reference core.

Run here, where the reference sources exist and oracle/_ref has been built
(`make -C oracle ref`):

    python tests/golden/make_golden.py

Outputs (committed):
  parity_scene.txt  stdout of the reference's own known-answer program
                    (solver/apps/parity.c) built against the reference library
  golden.json       reference results for the parity and lossy (Debye + SIBC)
                    scenes after their step counts (dt, energy, spectra, field
                    checksums), SHA-256 of every exported plan array, the
                    Djordjevic-Sarkar fit, the WR-28 mode solve, and a small
                    mode-port GCPW's source weights and port modes.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

from courant_b200 import scenes  # noqa: E402
from courant_b200.api import Courant  # noqa: E402
from oracle import REF_LIB  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def plan_digest(plan: dict) -> dict:
    out = {}
    for k, v in plan.items():
        if isinstance(v, list) and v and isinstance(v[0], np.ndarray):
            out[k] = [digest(a) for a in v]
        elif isinstance(v, list) and v and isinstance(v[0], dict):
            out[k] = [{kk: digest(vv) if isinstance(vv, np.ndarray) else vv for kk, vv in d.items()} for d in v]
        elif isinstance(v, dict):
            out[k] = {kk: digest(vv) for kk, vv in v.items()}
        elif isinstance(v, np.ndarray):
            out[k] = digest(v)
        else:
            out[k] = v
    return out


def cpx(a) -> list:
    return [[float(x.real), float(x.imag)] for x in np.asarray(a)]


def run_scene(c: Courant, fn) -> dict:
    s, meta = fn(c)
    plan = s.plan()
    s.step(meta["steps"])
    res = {
        "steps": meta["steps"], "dt": s.dt, "energy": s.energy(), "plan": plan_digest(plan),
        "portV": [cpx(s.portV(p)) for p in meta["ports"]], "portI": [cpx(s.portI(p)) for p in meta["ports"]],
        "vprobe": [cpx(s.vprobe(p)) for p in meta["vprobes"]], "iprobe": [cpx(s.iprobe(p)) for p in meta["iprobes"]],
        "source": cpx(s.sourceSpectrum()),
        "fields": [{"sum": float(f.sum()), "sumsq": float((f * f).sum()), "maxabs": float(np.abs(f).max())}
                   for f in (s.field(q) for q in range(6))],
        "ndisp": plan["ndisp"], "nsibc": plan["nsibc"],
    }
    if plan.get("sibc"):
        res["sibc_c"] = plan["sibc"]["c"].tolist()
        res["sibc_e"] = plan["sibc"]["e"].tolist()
    return res


def mode2d_wr28(c: Courant) -> dict:
    import ctypes as C
    a, b, NY, NZ = 7.112e-3, 3.556e-3, 48, 24
    y = np.array([a * j / NY for j in range(NY + 1)])
    z = np.array([b * k / NZ for k in range(NZ + 1)])
    dp = C.POINTER(C.c_double)
    m = c.ex.cem_mode2d_create(NY, NZ, y.ctypes.data_as(dp), z.ctypes.data_as(dp))
    f = 35e9
    k0 = 2 * np.pi * f / 299792458.0
    beta = np.sqrt(k0 ** 2 - (np.pi / a) ** 2)
    rc = c.ex.cem_mode2d_solve(m, f, beta / k0, None, 300, 1e-13)
    Rs = np.sqrt(2 * np.pi * f * 1.25663706212e-6 / (2 * 5.8e7))
    out = {"rc": rc, "beta": c.ex.cem_mode2d_beta(m), "alpha_c": c.ex.cem_mode2d_conductor_alpha(m, Rs),
           "power": c.ex.cem_mode2d_power(m)}
    c.ex.cem_mode2d_destroy(m)
    return out


def small_modeport(c: Courant) -> dict:
    s, meta = scenes.gcpw_line(c, length=2e-3, hmin=100e-6, hmax=400e-6, dx=200e-6, yair=0.6e-3, zair=0.8e-3,
                               npml=6, feed=2e-3, mon=0.8e-3, nf=4, modeports=True, steps=300)
    plan = s.plan()
    out = {"dims": meta["dims"], "dt": s.dt, "mode_source": {k: digest(v) for k, v in plan["modeSource"].items()},
           "n_mode_source": len(plan["modeSource"]["idx"])}
    s.step(meta["steps"])
    w = s.modePortWaves(meta["modeports"][0])
    out.update({"freqs": list(meta["freqs"]), "z0": w["z0"].tolist(), "beta": w["beta"].tolist(),
                "a": cpx(w["a"]), "b": cpx(w["b"]), "steps": meta["steps"]})
    return out


def main() -> None:
    exe = ROOT / "oracle" / "_ref" / "ref_parity"
    txt = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    (OUT / "parity_scene.txt").write_text(txt)
    c = Courant(REF_LIB)
    ds = c.fitDjordjevicSarkar(4.3, 0.02, 1e9, 1e8, 40e9, 6)
    gold = {
        "source": "skyhoffert/CourantEM 20261017.0 solver core, built by oracle/Makefile",
        "parity": run_scene(c, scenes.parity_scene),
        "lossy": run_scene(c, scenes.lossy_scene),
        "ds_fit": {"args": [4.3, 0.02, 1e9, 1e8, 40e9, 6], "eps_inf": ds.eps_inf, "fp": ds.fp, "deps": ds.deps,
                   "err": ds.tan_delta_error},
        "mode2d_wr28": mode2d_wr28(c),
        "modeport_small": small_modeport(c),
    }
    (OUT / "golden.json").write_text(json.dumps(gold, indent=1))
    print("wrote", OUT / "parity_scene.txt", OUT / "golden.json")


if __name__ == "__main__":
    main()
