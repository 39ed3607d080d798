"""ctypes driver of the oracle restatement (fdtd_oracle.c) - TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the product never imports it.

`OracleSim.from_plan(sim, steps)` builds an f64 CPU stepper from the plan a
courant.h library exports for `sim` (courant_b200.api.Sim), so the oracle and
the GPU engine start from the same coefficients.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libfdtd_oracle.so"
REF_LIB = HERE / "_ref" / "libcourant_ref.so"

_dp = C.POINTER(C.c_double)
_dpp = C.POINTER(_dp)
_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} missing: run `make -C oracle restatement`")
        L = C.CDLL(str(LIB))
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double] + [_dpp] * 10 + [C.POINTER(C.c_int)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_frequencies.argtypes = [C.c_void_p, C.c_int, _dp]
        L.orc_add_port.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_double]
        L.orc_add_vprobe.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_add_iprobe.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_set_mode_source.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.orc_set_waveforms.argtypes = [C.c_void_p, C.c_long, _dp, _dp, C.c_int, C.c_int]
        L.orc_set_disp.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_set_sibc.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_step.argtypes = [C.c_void_p, C.c_long]
        L.orc_step_count.restype = C.c_long
        L.orc_step_count.argtypes = [C.c_void_p]
        L.orc_energy.restype = C.c_double
        L.orc_energy.argtypes = [C.c_void_p]
        for n in ("orc_field",):
            getattr(L, n).restype = _dp
            getattr(L, n).argtypes = [C.c_void_p, C.c_int]
        for n in ("orc_port_v", "orc_port_i", "orc_vprobe", "orc_iprobe"):
            getattr(L, n).restype = _dp
            getattr(L, n).argtypes = [C.c_void_p, C.c_int]
        L.orc_source_spectrum.restype = _dp
        L.orc_source_spectrum.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


class OracleSim:
    """f64 CPU stepper over an exported plan (keeps the plan arrays alive)."""

    def __init__(self, plan: dict, freqs, steps: int, waves: dict):
        L = load()
        self.L, self.plan = L, plan
        self.nf = len(freqs)
        self.N = plan["N"]
        keep = []

        def ptrs(arrs):
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
            keep.extend(arrs)
            return (_dp * 3)(*[_p(a) for a in arrs])

        npml = (C.c_int * 6)(*plan["npml"])
        self.h = L.orc_create(plan["nx"], plan["ny"], plan["nz"], plan["dt"], ptrs(plan["ca"]), ptrs(plan["cb"]),
                              ptrs(plan["ide"]), ptrs(plan["idh"]), ptrs(plan["be"]), ptrs(plan["ce"]),
                              ptrs(plan["bh"]), ptrs(plan["ch"]), ptrs(plan["d"]), ptrs(plan["dd"]), npml)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        keep.append(f)
        L.orc_set_frequencies(self.h, len(f), _p(f))
        for pt in plan["ports"]:
            L.orc_add_port(self.h, len(pt["idx"]), _p(pt["idx"]), _p(pt["vw"]), _p(pt["cs"]), pt["R"])
        for v in plan["vprobes"]:
            L.orc_add_vprobe(self.h, len(v["idx"]), _p(v["idx"]), _p(v["w"]))
        for v in plan["iprobes"]:
            L.orc_add_iprobe(self.h, len(v["idx"]), _p(v["idx"]), _p(v["w"]))
        ms = plan["modeSource"]
        has_mode = len(ms["idx"]) > 0
        if has_mode:
            L.orc_set_mode_source(self.h, len(ms["idx"]), _p(ms["idx"]), _p(ms["w"]))
        wl = np.ascontiguousarray(waves["lumped"], dtype=np.float64)
        wm = np.ascontiguousarray(waves["mode"], dtype=np.float64)
        keep += [wl, wm]
        L.orc_set_waveforms(self.h, steps, _p(wl), _p(wm), plan["excitedLumped"], int(has_mode))
        if plan.get("disp"):
            d = plan["disp"]
            L.orc_set_disp(self.h, len(d["idx"]), plan["npole"], _p(d["idx"]), _p(d["cb"]), _p(d["beta"]), _p(d["k"]))
        if plan.get("sibc"):
            s = plan["sibc"]
            L.orc_set_sibc(self.h, len(s["idx"]), len(s["c"]), _p(s["idx"]), _p(s["hidx"]), _p(s["hw"]), _p(s["c"]),
                           _p(s["e"]))
        self._keep = keep

    @classmethod
    def from_sim(cls, sim, freqs, steps: int) -> "OracleSim":
        """Oracle for a finalized courant_b200.api.Sim, covering `steps` steps of source waveform."""
        return cls(sim.plan(), freqs, steps, sim.waveforms(0, steps))

    def step(self, n: int):
        self.L.orc_step(self.h, n)

    @property
    def steps(self) -> int:
        return self.L.orc_step_count(self.h)

    def energy(self) -> float:
        return self.L.orc_energy(self.h)

    def field(self, comp: int) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_field(self.h, comp), shape=(self.N,)).copy()

    def field_view(self, comp: int) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_field(self.h, comp), shape=(self.N,))

    def _spec(self, ptr) -> np.ndarray:
        a = np.ctypeslib.as_array(ptr, shape=(2 * self.nf,)).copy()
        return a[0::2] + 1j * a[1::2]

    def portV(self, p):
        return self._spec(self.L.orc_port_v(self.h, p))

    def portI(self, p):
        return self._spec(self.L.orc_port_i(self.h, p))

    def vprobe(self, p):
        return self._spec(self.L.orc_vprobe(self.h, p))

    def iprobe(self, p):
        return self._spec(self.L.orc_iprobe(self.h, p))

    def sourceSpectrum(self):
        return self._spec(self.L.orc_source_spectrum(self.h))

    def __del__(self):
        try:
            self.L.orc_destroy(self.h)
        except Exception:
            pass
