"""Generate full-length S-parameter fixtures of the benchmark GCPW lines from
the reference core.

Run here, where oracle/_ref has been built from the reference sources
(`make -C oracle ref`):

    python tests/golden/make_sparams.py c1            # ~1 min on 8 threads
    python tests/golden/make_sparams.py c2            # ~3 h on 8 threads (or --excite 1/2 in parallel, then --merge)

For each excitation (port 1 driven, then port 2) the reference steps the
configuration for its full step count (c1: 20 000, c2: 40 000) and the excited
column of the S-matrix is recorded: for lumped ports the waves from V and I at
50 ohm (the reference's courant.ts sParams), for mode ports the modal waves of
cem_mode_port_waves (reference solver/src/modeport.c:203-227) with each port's
Z0 and beta, and the 50-ohm renormalised matrix from cem_s2_renormalize
(modeport.c:242-264). A field checksum after the run is kept as well.

Output: tests/golden/sparams_<config>.json (committed).
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

from courant_b200 import scenes  # noqa: E402
from courant_b200.api import Courant  # noqa: E402
from oracle import REF_LIB  # noqa: E402

OUT = Path(__file__).resolve().parent


def cpx(a) -> list:
    return [[float(x.real), float(x.imag)] for x in np.asarray(a)]


def run(c: Courant, name: str, excite: int) -> dict:
    t0 = time.time()
    s, meta = scenes.config_line(c, name, excite=excite)
    t1 = time.time()
    s.step(meta["steps"])
    t2 = time.time()
    col = scenes.two_port_s(s, meta)
    t3 = time.time()
    out = {"excite": excite, "steps": meta["steps"], "dims": list(meta["dims"]), "dt": s.dt,
           "freqs": [float(f) for f in meta["freqs"]], "energy": s.energy(),
           "S": [cpx(b) for b in col["b"]],
           "fields": [{"sumsq": float((f * f).sum()), "maxabs": float(np.abs(f).max())}
                      for f in (s.field(q) for q in range(6))],
           "seconds": {"setup": t1 - t0, "steps": t2 - t1, "waves": t3 - t2}}
    if "z0" in col:
        out["z0"] = [z.tolist() for z in col["z0"]]
        out["beta"] = [b.tolist() for b in col["beta"]]
    print(f"{name} excite {excite}: setup {t1 - t0:.0f} s, {meta['steps']} steps {t2 - t1:.0f} s, "
          f"waves {t3 - t2:.0f} s", flush=True)
    s.destroy()
    return out


def main() -> None:
    """make_sparams.py NAME            both excitations, then the fixture
    make_sparams.py NAME --excite E    one excitation into sparams_NAME.eE.json (to run the two in parallel)
    make_sparams.py NAME --merge       the fixture from the two one-excitation files"""
    name = sys.argv[1]
    c = Courant(REF_LIB)
    if "--excite" in sys.argv:
        e = int(sys.argv[sys.argv.index("--excite") + 1])
        (OUT / f"sparams_{name}.e{e}.json").write_text(json.dumps(run(c, name, e)))
        return
    if "--merge" in sys.argv:
        runs = [json.loads((OUT / f"sparams_{name}.e{e}.json").read_text()) for e in (1, 2)]
    else:
        runs = [run(c, name, e) for e in (1, 2)]
    gold = {"source": "skyhoffert/CourantEM 20261017.0 solver core, built by oracle/Makefile",
            "config": name, "kw": {k: (list(v) if isinstance(v, tuple) else v)
                                    for k, v in scenes.CONFIGS[name]["kw"].items()},
            "runs": runs}
    if len(runs) == 2 and "z0" in runs[0]:
        # full 2x2 at each frequency, renormalised from the port impedances to 50 ohm by the reference
        ren = []
        for q in range(len(runs[0]["freqs"])):
            S = [complex(*runs[0]["S"][0][q]), complex(*runs[0]["S"][1][q]),
                 complex(*runs[1]["S"][0][q]), complex(*runs[1]["S"][1][q])]   # S11 S21 S12 S22
            ren.append(cpx(c.renormalize2(S, runs[0]["z0"][0][q], runs[0]["z0"][1][q], 50.0)))
        gold["S50"] = ren
    (OUT / f"sparams_{name}.json").write_text(json.dumps(gold))
    print("wrote", OUT / f"sparams_{name}.json")


if __name__ == "__main__":
    main()
