"""Python host side of the courant.h C ABI.

`Courant` and `Sim` mirror the reference's TypeScript wrapper
(skyhoffert/CourantEM web/src/solver/courant.ts: class Courant :120-214,
class Sim :216-455): the same method names, argument meanings and error
behaviour (a negative return code raises CourantError with cem_last_error()).
They bind any library exporting that ABI: by default libcourant_b200.so, the
B200 engine of this package; test code can pass another library path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Sequence

import numpy as np

Axis = {"X": 0, "Y": 1, "Z": 2}
Face = {"XLo": 0, "XHi": 1, "YLo": 2, "YHi": 3, "ZLo": 4, "ZHi": 5}
Boundary = {"PEC": 0, "CPML": 1}
C0 = 299792458.0
MU0 = 1.25663706212e-6
EPS0 = 8.8541878128e-12

_d = C.c_double
_i = C.c_int
_l = C.c_long
_p = C.c_void_p
_dp = C.POINTER(C.c_double)
_sz = C.c_size_t

class ModePortDef(C.Structure):
    """cem_mode_port_def of courant.h"""
    _fields_ = [(n, C.c_int) for n in ("dir", "i_src", "i_mon", "j0", "j1", "k0", "k1", "vj", "vk0", "vk1", "vsign",
                                        "ja", "jb", "ka", "kb")] + [("x_ref", C.c_double), ("f0", C.c_double),
                                                                    ("neff0", C.c_double)]


# (name, restype, argtypes) for every function of include/courant.h
_PROTOS = [
    ("cem_create", _p, [_i, _i, _i, _dp, _dp, _dp]),
    ("cem_destroy", None, [_p]),
    ("cem_last_error", C.c_char_p, []),
    ("cem_set_boundary", _i, [_p, _i, _i, _i]),
    ("cem_material_box", _i, [_p, _d, _d, _d, _d, _d, _d, _d, _d]),
    ("cem_set_debye_poles", _i, [_p, _i, _dp]),
    ("cem_material_box_debye", _i, [_p, _d, _d, _d, _d, _d, _d, _d, _d, _dp]),
    ("cem_set_conductor_loss", _i, [_p, _d, _i, _d, _d, _d, _d]),
    ("cem_conductor_fit_error", _d, [_p]),
    ("cem_conductor_zs", None, [_p, _d, _dp, _dp]),
    ("cem_fit_djordjevic_sarkar", _d, [_d, _d, _d, _d, _d, _i, _dp, _dp, _dp]),
    ("cem_pec_box", _i, [_p, _d, _d, _d, _d, _d, _d]),
    ("cem_pec_sheet", _i, [_p, _i, _d, _d, _d, _d, _d]),
    ("cem_pec_edges_plane", _i, [_p, _i, _i, _p, _p]),
    ("cem_pec_cells", _i, [_p, _i, _i, _i, _i, _i, _i, _p]),
    ("cem_add_lumped_port", _i, [_p, _i, _i, _i, _i, _i, _i, _d]),
    ("cem_set_gaussian", _i, [_p, _i, _d, _d, _d]),
    ("cem_set_frequencies", _i, [_p, _i, _dp]),
    ("cem_add_vprobe", _i, [_p, _i, _i, _i, _i, _i, _i]),
    ("cem_add_iprobe", _i, [_p, _i, _i, _i, _i, _i, _i]),
    ("cem_finalize", _i, [_p, _d]),
    ("cem_dt", _d, [_p]),
    ("cem_step_count", _l, [_p]),
    ("cem_step", None, [_p, _l]),
    ("cem_run", _l, [_p, _l, _d, _i]),
    ("cem_energy", _d, [_p]),
    ("cem_nfreq", _i, [_p]),
    ("cem_port_v", _dp, [_p, _i]),
    ("cem_port_i", _dp, [_p, _i]),
    ("cem_source_spectrum", _dp, [_p]),
    ("cem_vprobe", _dp, [_p, _i]),
    ("cem_iprobe", _dp, [_p, _i]),
    ("cem_port_impedance", _d, [_p, _i]),
    ("cem_excited_port", _i, [_p]),
    ("cem_field", _dp, [_p, _i]),
    ("cem_index", _sz, [_p, _i, _i, _i]),
    ("cem_dims", None, [_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    ("cem_mode2d_create", _p, [_i, _i, _dp, _dp]),
    ("cem_mode2d_destroy", None, [_p]),
    ("cem_mode2d_set_media", None, [_p, _dp, _dp, _dp, _p, _p, _p]),
    ("cem_mode2d_solve", _i, [_p, _d, _d, _dp, _i, _d]),
    ("cem_mode2d_set_debye", None, [_p, _i, _dp, _dp, _dp, _dp]),
    ("cem_mode2d_set_loss", None, [_p, _dp, _dp, _dp]),
    ("cem_mode2d_set_pml", None, [_p, _i, _dp, _dp, _dp]),
    ("cem_mode2d_beta", _d, [_p]),
    ("cem_mode2d_alpha", _d, [_p]),
    ("cem_mode2d_eu", _dp, [_p]),
    ("cem_mode2d_ev", _dp, [_p]),
    ("cem_mode2d_hu", _dp, [_p]),
    ("cem_mode2d_hv", _dp, [_p]),
    ("cem_mode2d_power", _d, [_p]),
    ("cem_mode2d_conductor_alpha", _d, [_p, _d]),
    ("cem_mode2d_vi", None, [_p, _i, _i, _i, _i, _i, _i, _i, _dp, _dp]),
    ("cem_add_mode_port", _i, [_p, C.POINTER(ModePortDef)]),
    ("cem_add_mode_port_args", _i, [_p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _d, _d, _d]),
    ("cem_set_mode_excitation", _i, [_p, _i, _d, _d]),
    ("cem_mode_port_waves", _i, [_p, _i, _dp, _dp, _dp, _dp]),
    ("cem_mode_port_alpha", _i, [_p, _i, _dp]),
    ("cem_mode_port_alpha_c", _i, [_p, _i, _dp]),
    ("cem_s2_renormalize", None, [_dp, _d, _d, _d]),
    ("cem_plan_array", _dp, [_p, _i, _i]),
    ("cem_plan_npml", _i, [_p, _i]),
    ("cem_plan_has_pml", _i, [_p]),
    ("cem_plan_nport", _i, [_p]),
    ("cem_plan_nvprobe", _i, [_p]),
    ("cem_plan_niprobe", _i, [_p]),
    ("cem_plan_ndisp", _i, [_p]),
    ("cem_plan_nsibc", _i, [_p]),
    ("cem_plan_port", _i, [_p, _i, _dp, _dp, _dp]),
    ("cem_plan_vprobe", _i, [_p, _i, _dp, _dp]),
    ("cem_plan_iprobe", _i, [_p, _i, _dp, _dp]),
    ("cem_plan_mode_source", _i, [_p, _dp, _dp]),
    ("cem_plan_waveforms", None, [_p, _l, _i, _dp, _dp]),
    ("cem_plan_excited_lumped", _i, [_p]),
    ("cem_plan_npole", _i, [_p]),
    ("cem_plan_disp", _i, [_p, _dp, _dp, _dp, _dp]),
    ("cem_plan_sibc", _i, [_p, _dp, _dp, _dp, _dp, _dp, C.POINTER(_i)]),
    ("cem_push_samples", None, [_p, _i, _dp, _dp, _dp, _dp]),
    ("cem_checkpoint_size", _sz, [_p]),
    ("cem_checkpoint_save", _i, [_p, _dp]),
    ("cem_checkpoint_load", _i, [_p, _dp]),
    ("cem_state_array", _dp, [_p, _i, _i, _i]),
    ("cem_state_len", _sz, [_p, _i, _i, _i]),
    ("cem_mt_pre", None, [_p]),
    ("cem_version", C.c_char_p, []),
    ("cem_mt_H", None, [_p, _i, _i]),
    ("cem_mt_mid", None, [_p]),
    ("cem_mt_E", None, [_p, _i, _i]),
    ("cem_mt_post", None, [_p]),
    ("cem_set_step", None, [_p, _l]),
    ("cem_cross_section_x", _p, [_p, _i, _i, _i, _i, _i]),
]

API_NAMES = [n for n, _, _ in _PROTOS]

# include/courant_b200.h (extensions without a reference counterpart)
_EXT_PROTOS = [
    ("cemx_step_timed", _i, [_p, _l, _dp]),
    ("cemx_profile_steps", _i, [_p, _l, _dp, C.POINTER(_l)]),
    ("cemx_sizes", _i, [_p, C.POINTER(C.c_longlong), _i]),
    ("cemx_synchronize", _i, [_p]),
    ("cemx_select_device", _i, [_i]),
    ("cemx_release_device", _i, [_p]),
    ("cemx_use_fused", _i, [_p, _i]),
    ("cemx_tune", _i, [_p, _i]),
    ("cemx_tune_state", _i, [_p, _dp, _i]),
    ("cemx_energy_noalloc", _i, [_p, _dp]),
    ("cemx_prepare_device", _i, [_p, _i]),
    ("cemx_batch_create", _p, [_i]),
    ("cemx_batch_destroy", None, [_p]),
    ("cemx_batch_add", _i, [_p, _p, _l]),
    ("cemx_batch_remove", _i, [_p, _p]),
    ("cemx_batch_left", _l, [_p, _p]),
    ("cemx_batch_run", _i, [_p, _l]),
    ("cemx_batch_tune", _i, [_p, _i]),
    ("cemx_batch_stats", _i, [_p, _dp, _i]),
]


class CourantError(RuntimeError):
    pass


def default_library() -> Path:
    return Path(__file__).resolve().parent / "lib" / "libcourant_b200.so"


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _c64(pairs: np.ndarray) -> np.ndarray:
    return pairs[0::2] + 1j * pairs[1::2]


@dataclass
class DebyeModel:
    eps_inf: float
    fp: list
    deps: list
    tan_delta_error: float


class Courant:
    """A loaded courant.h library (mirrors class Courant of courant.ts)."""

    _cache: dict = {}

    def __init__(self, lib: str | Path | None = None):
        path = Path(lib) if lib else default_library()
        if not path.exists():
            raise CourantError(f"{path} is missing: build it with `python -m courant_b200.build`")
        key = str(path.resolve())
        if key not in Courant._cache:
            dll = C.CDLL(key, mode=C.RTLD_LOCAL)
            for name, res, args in _PROTOS + (_EXT_PROTOS if hasattr(dll, "cemx_sizes") else []):
                fn = getattr(dll, name)
                fn.restype = res
                fn.argtypes = args
            Courant._cache[key] = dll
        self.ex = Courant._cache[key]
        self.path = path

    def last_error(self) -> str:
        return (self.ex.cem_last_error() or b"").decode()

    lastError = last_error

    def version(self) -> str:
        return self.ex.cem_version().decode()

    def fitDjordjevicSarkar(self, dk, df, fref, fmin, fmax, npole=8) -> DebyeModel:
        ei = C.c_double(0)
        fp = np.zeros(npole)
        de = np.zeros(npole)
        err = self.ex.cem_fit_djordjevic_sarkar(dk, df, fref, fmin, fmax, npole, C.byref(ei), _ptr(fp), _ptr(de))
        return DebyeModel(ei.value, list(fp), list(de), err)

    def renormalize2(self, S: Sequence[complex], z1: float, z2: float, zref: float) -> list[complex]:
        v = _f64([x for c in S for x in (c.real, c.imag)])
        self.ex.cem_s2_renormalize(_ptr(v), z1, z2, zref)
        return [complex(v[2 * q], v[2 * q + 1]) for q in range(4)]

    def createBatch(self, device: int = -1) -> "Batch":
        """Simulations advanced together on one device (include/courant_b200.h)."""
        h = self.ex.cemx_batch_create(device)
        if not h:
            raise CourantError(f"cemx_batch_create: {self.last_error()}")
        return Batch(self, h)

    def selectDevice(self, device: int):
        if self.ex.cemx_select_device(device) != 0:
            raise CourantError(f"select_device: {self.last_error()}")

    def createSim(self, x, y, z) -> "Sim":
        x, y, z = _f64(x), _f64(y), _f64(z)
        h = self.ex.cem_create(len(x) - 1, len(y) - 1, len(z) - 1, _ptr(x), _ptr(y), _ptr(z))
        if not h:
            raise CourantError(f"cem_create: {self.last_error()}")
        return Sim(self, h, len(x) - 1, len(y) - 1, len(z) - 1)


class Sim:
    """One simulation (mirrors class Sim of courant.ts)."""

    def __init__(self, c: Courant, handle: int, nx: int, ny: int, nz: int):
        self.c, self.h, self.nx, self.ny, self.nz = c, handle, nx, ny, nz
        self.N = (nx + 1) * (ny + 1) * (nz + 1)
        self.nf = 0

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            raise CourantError(f"{what}: {self.c.last_error()}")
        return rc

    # ---- setup
    def setBoundary(self, face: int, type_: int, ncells: int = 0):
        self._check(self.c.ex.cem_set_boundary(self.h, face, type_, ncells), "set_boundary")

    def materialBox(self, x0, x1, y0, y1, z0, z1, epsR, sigma=0.0):
        self._check(self.c.ex.cem_material_box(self.h, x0, x1, y0, y1, z0, z1, epsR, sigma), "material_box")

    def pecBox(self, x0, x1, y0, y1, z0, z1):
        self._check(self.c.ex.cem_pec_box(self.h, x0, x1, y0, y1, z0, z1), "pec_box")

    def pecSheet(self, axis, pos, a0, a1, b0, b1):
        self._check(self.c.ex.cem_pec_sheet(self.h, axis, pos, a0, a1, b0, b1), "pec_sheet")

    def pecEdgesPlane(self, axis, m, mask_u=None, mask_v=None):
        mu = None if mask_u is None else np.ascontiguousarray(mask_u, dtype=np.uint8)
        mv = None if mask_v is None else np.ascontiguousarray(mask_v, dtype=np.uint8)
        self._check(self.c.ex.cem_pec_edges_plane(self.h, axis, m, None if mu is None else mu.ctypes.data,
                                                   None if mv is None else mv.ctypes.data), "pec_edges_plane")

    def pecCells(self, i0, j0, k0, mask):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        ni, nj, nk = m.shape
        self._check(self.c.ex.cem_pec_cells(self.h, i0, j0, k0, ni, nj, nk, m.ctypes.data), "pec_cells")

    def addLumpedPort(self, axis, n1, n2, m0, m1, dir_, R) -> int:
        return self._check(self.c.ex.cem_add_lumped_port(self.h, axis, n1, n2, m0, m1, dir_, R), "add_lumped_port")

    def setGaussian(self, port, amp, t0, tau):
        self._check(self.c.ex.cem_set_gaussian(self.h, port, amp, t0, tau), "set_gaussian")

    def setFrequencies(self, f):
        f = _f64(f)
        self._check(self.c.ex.cem_set_frequencies(self.h, len(f), _ptr(f)), "set_frequencies")
        self.nf = len(f)

    def addVProbe(self, axis, n1, n2, m0, m1, dir_) -> int:
        return self._check(self.c.ex.cem_add_vprobe(self.h, axis, n1, n2, m0, m1, dir_), "add_vprobe")

    def addIProbe(self, axis, m, a0, a1, b0, b1) -> int:
        return self._check(self.c.ex.cem_add_iprobe(self.h, axis, m, a0, a1, b0, b1), "add_iprobe")

    def setDebyePoles(self, fp):
        fp = _f64(fp)
        self._check(self.c.ex.cem_set_debye_poles(self.h, len(fp), _ptr(fp)), "set_debye_poles")

    def materialBoxDebye(self, x0, x1, y0, y1, z0, z1, m: DebyeModel, sigma=0.0):
        d = _f64(m.deps)
        self._check(self.c.ex.cem_material_box_debye(self.h, x0, x1, y0, y1, z0, z1, m.eps_inf, sigma, _ptr(d)),
                    "material_box_debye")

    def setConductorLoss(self, sigma, fmin, fmax, rough=0, p1=0.0, p2=0.0):
        self._check(self.c.ex.cem_set_conductor_loss(self.h, sigma, rough, p1, p2, fmin, fmax), "set_conductor_loss")

    def conductorFitError(self) -> float:
        return self.c.ex.cem_conductor_fit_error(self.h)

    def addModePort(self, d: dict) -> int:
        return self._check(self.c.ex.cem_add_mode_port_args(
            self.h, d["dir"], d["iSrc"], d["iMon"], d["j0"], d["j1"], d["k0"], d["k1"], d["vj"], d["vk0"], d["vk1"],
            d["vsign"], d["ja"], d["jb"], d["ka"], d["kb"], d["xRef"], d["f0"], d["neff0"]), "add_mode_port")

    def setModeExcitation(self, port, t0, tau):
        self._check(self.c.ex.cem_set_mode_excitation(self.h, port, t0, tau), "set_mode_excitation")

    def finalize(self, cfl=0.99):
        if self.c.ex.cem_finalize(self.h, cfl) != 0:
            raise CourantError(f"finalize: {self.c.last_error()}")
        self.nf = self.c.ex.cem_nfreq(self.h)

    # ---- running
    @property
    def dt(self) -> float:
        return self.c.ex.cem_dt(self.h)

    @property
    def steps(self) -> int:
        return int(self.c.ex.cem_step_count(self.h))

    def step(self, n: int):
        before = self.steps
        self.c.ex.cem_step(self.h, n)
        if n > 0 and self.steps != before + n:
            raise CourantError(f"step: {self.c.last_error()}")

    def run(self, max_steps: int, decay: float = 1e-5, check_every: int = 200) -> int:
        return int(self.c.ex.cem_run(self.h, max_steps, decay, check_every))

    def energy(self) -> float:
        return self.c.ex.cem_energy(self.h)

    # ---- results
    def _spectrum(self, ptr) -> np.ndarray:
        if not ptr:
            raise CourantError(f"spectrum: {self.c.last_error()}")
        return _c64(np.ctypeslib.as_array(ptr, shape=(2 * self.nf,)).copy())

    def portV(self, p: int) -> np.ndarray:
        return self._spectrum(self.c.ex.cem_port_v(self.h, p))

    def portI(self, p: int) -> np.ndarray:
        return self._spectrum(self.c.ex.cem_port_i(self.h, p))

    def vprobe(self, p: int) -> np.ndarray:
        return self._spectrum(self.c.ex.cem_vprobe(self.h, p))

    def iprobe(self, p: int) -> np.ndarray:
        return self._spectrum(self.c.ex.cem_iprobe(self.h, p))

    def sourceSpectrum(self) -> np.ndarray:
        return self._spectrum(self.c.ex.cem_source_spectrum(self.h))

    def modePortWaves(self, port: int) -> dict:
        nf = self.nf
        a, b, z0, beta = np.zeros(2 * nf), np.zeros(2 * nf), np.zeros(nf), np.zeros(nf)
        if self.c.ex.cem_mode_port_waves(self.h, port, _ptr(a), _ptr(b), _ptr(z0), _ptr(beta)) != 0:
            raise CourantError(f"mode_port_waves: {self.c.last_error()}")
        return {"a": _c64(a), "b": _c64(b), "z0": z0, "beta": beta}

    def modePortAlpha(self, port: int) -> np.ndarray:
        out = np.zeros(self.nf)
        self._check(self.c.ex.cem_mode_port_alpha(self.h, port, _ptr(out)), "mode_port_alpha")
        return out

    # ---- fields and state
    def field(self, comp: int) -> np.ndarray:
        p = self.c.ex.cem_field(self.h, comp)
        return np.ctypeslib.as_array(p, shape=(self.N,)).copy()

    def fieldView(self, comp: int) -> np.ndarray:
        """Writable view of the library's host copy of a field (cem_field)."""
        p = self.c.ex.cem_field(self.h, comp)
        return np.ctypeslib.as_array(p, shape=(self.N,))

    def setField(self, comp: int, data):
        self.fieldView(comp)[:] = np.asarray(data, dtype=np.float64).ravel()

    def index(self, i, j, k) -> int:
        return int(self.c.ex.cem_index(self.h, i, j, k))

    def checkpoint(self) -> np.ndarray:
        n = self.c.ex.cem_checkpoint_size(self.h)
        buf = np.zeros(n)
        self._check(self.c.ex.cem_checkpoint_save(self.h, _ptr(buf)), "checkpoint")
        return buf

    def restore(self, buf):
        b = _f64(buf)
        self._check(self.c.ex.cem_checkpoint_load(self.h, _ptr(b)), "restore")

    def stateLen(self, which, comp=0, w=0) -> int:
        return int(self.c.ex.cem_state_len(self.h, which, comp, w))

    # ---- plan (mirrors Sim.plan of courant.ts)
    def plan(self) -> dict:
        ex, h = self.c.ex, self.h
        n = [self.nx, self.ny, self.nz]
        N = self.N

        def arr(which, comp, length):
            p = ex.cem_plan_array(h, which, comp)
            return np.ctypeslib.as_array(p, shape=(length,)).copy()

        per = lambda which, extra: [arr(which, a, n[a] + extra) for a in range(3)]
        out = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "N": N, "dt": self.dt,
               "ca": [arr(0, c, N) for c in range(3)], "cb": [arr(1, c, N) for c in range(3)],
               "ide": per(2, 1), "idh": per(3, 0), "be": per(4, 1), "ce": per(5, 1), "bh": per(6, 0),
               "ch": per(7, 0), "d": per(8, 0), "dd": per(9, 1),
               "npml": [ex.cem_plan_npml(h, f) for f in range(6)], "hasPml": ex.cem_plan_has_pml(h) != 0,
               "excitedLumped": ex.cem_plan_excited_lumped(h)}
        ports = []
        for p in range(ex.cem_plan_nport(h)):
            ln = ex.cem_plan_port(h, p, None, None, None)
            a, b, c = np.zeros(ln), np.zeros(ln), np.zeros(ln)
            ex.cem_plan_port(h, p, _ptr(a), _ptr(b), _ptr(c))
            ports.append({"idx": a, "vw": b, "cs": c, "R": ex.cem_port_impedance(h, p)})
        out["ports"] = ports

        def lst(fn, count):
            res = []
            for p in range(count):
                ln = fn(p, None, None)
                a, b = np.zeros(max(ln, 1)), np.zeros(max(ln, 1))
                fn(p, _ptr(a), _ptr(b))
                res.append({"idx": a[:ln], "w": b[:ln]})
            return res

        out["vprobes"] = lst(lambda p, a, b: ex.cem_plan_vprobe(h, p, a, b), ex.cem_plan_nvprobe(h))
        out["iprobes"] = lst(lambda p, a, b: ex.cem_plan_iprobe(h, p, a, b), ex.cem_plan_niprobe(h))
        out["modeSource"] = lst(lambda p, a, b: ex.cem_plan_mode_source(h, a, b), 1)[0]
        nd, npole = ex.cem_plan_ndisp(h), ex.cem_plan_npole(h)
        out["ndisp"], out["nsibc"], out["npole"] = nd, ex.cem_plan_nsibc(h), npole
        if nd:
            a, b, c, k = np.zeros(nd), np.zeros(nd), np.zeros(nd * npole), np.zeros(npole)
            ex.cem_plan_disp(h, _ptr(a), _ptr(b), _ptr(c), _ptr(k))
            out["disp"] = {"idx": a, "cb": b, "beta": c, "k": k}
        ns = out["nsibc"]
        if ns:
            a, hi, hw, cc, ee = np.zeros(ns), np.zeros(4 * ns), np.zeros(4 * ns), np.zeros(16), np.zeros(16)
            nt = C.c_int(0)
            ex.cem_plan_sibc(h, _ptr(a), _ptr(hi), _ptr(hw), _ptr(cc), _ptr(ee), C.byref(nt))
            out["sibc"] = {"idx": a, "hidx": hi, "hw": hw, "c": cc[:nt.value], "e": ee[:nt.value]}
        return out

    def waveforms(self, n0: int, n: int) -> dict:
        a, b = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        self.c.ex.cem_plan_waveforms(self.h, n0, n, _ptr(a), _ptr(b))
        return {"lumped": a[:n], "mode": b[:n]}

    # ---- extensions (courant_b200.h)
    def stepTimed(self, n: int) -> float:
        """Advance n steps; device milliseconds measured on the engine stream."""
        ms = C.c_double(0)
        self._check(self.c.ex.cemx_step_timed(self.h, n, C.byref(ms)), "step_timed")
        return ms.value

    def profileSteps(self, n: int) -> dict:
        ms, cnt = np.zeros(5), (C.c_long * 5)()
        self._check(self.c.ex.cemx_profile_steps(self.h, n, _ptr(ms), cnt), "profile_steps")
        names = ["update_h", "update_e", "sibc", "post", "dft"]
        return {k: {"ms": float(ms[q]), "launches": int(cnt[q])} for q, k in enumerate(names)}

    def sizes(self) -> dict:
        out = (C.c_longlong * 19)()
        self._check(self.c.ex.cemx_sizes(self.h, out, 19), "sizes")
        keys = ["cells", "points", "psiE", "psiH", "ndisp", "npole", "nsibc", "sibc_terms", "tab_x", "tab_y", "tab_z",
                "device_bytes", "launches_per_step", "h_fast_pts", "h_general_pts", "e_fast_pts", "e_general_pts",
                "e_debye_pts", "jbox_points"]
        return dict(zip(keys, [int(v) for v in out]))

    def useFused(self, on: bool = True) -> bool:
        """Select the single-pass fused H+E kernel (True) or the separate kernels."""
        return bool(self.c.ex.cemx_use_fused(self.h, int(on)))

    def tune(self, on: bool = True) -> bool:
        """Choose this simulation's launch shape per grid shape (cemx_tune)."""
        return bool(self.c.ex.cemx_tune(self.h, int(on)))

    def tuneState(self) -> dict:
        v = np.zeros(7)
        self._check(self.c.ex.cemx_tune_state(self.h, _ptr(v), 7), "tune_state")
        return {"tuned": bool(v[0]), "from_cache": bool(v[1]), "thin": int(v[2]), "side_stream": bool(v[3]),
                "graph_steps": int(v[4]), "ms_per_step": float(v[5]), "z_tails": bool(v[6])}

    def prepareDevice(self, device: int = -1):
        """Create the device state now rather than at the first step."""
        self._check(self.c.ex.cemx_prepare_device(self.h, device), "prepare_device")

    def releaseDevice(self):
        self._check(self.c.ex.cemx_release_device(self.h), "release_device")

    def synchronize(self):
        self._check(self.c.ex.cemx_synchronize(self.h), "synchronize")

    def energyNoAlloc(self) -> float:
        """cem_energy without device allocation (static scratch; see courant_b200.h)."""
        w = C.c_double()
        self._check(self.c.ex.cemx_energy_noalloc(self.h, C.byref(w)), "energy_noalloc")
        return w.value

    def destroy(self):
        if getattr(self, "h", None):
            self.c.ex.cem_destroy(self.h)
            self.h = None


def s_params(v1, i1, v2, i2, R):
    """S11, S21 from lumped-port spectra with port 1 excited (courant.ts sParams :458-470)."""
    sq = np.sqrt(R)
    a1 = (v1 + R * i1) / (2 * sq)
    b1 = (v1 - R * i1) / (2 * sq)
    b2 = (v2 - R * i2) / (2 * sq)
    return b1 / a1, b2 / a1


class Batch:
    """Several finalized simulations advanced together on one device: batched
    launches over a work-list across the members, graph-captured chunks.
    Results stay readable through each Sim between runs."""

    def __init__(self, c: Courant, h):
        self.c, self.h = c, h
        self.members: list[Sim] = []

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            raise CourantError(f"{what}: {self.c.last_error()}")
        return rc

    def add(self, sim: "Sim", steps: int) -> int:
        rc = self._check(self.c.ex.cemx_batch_add(self.h, sim.h, int(steps)), "batch_add")
        self.members.append(sim)
        return rc

    def remove(self, sim: "Sim"):
        self._check(self.c.ex.cemx_batch_remove(self.h, sim.h), "batch_remove")
        self.members.remove(sim)

    def left(self, sim: "Sim") -> int:
        return int(self.c.ex.cemx_batch_left(self.h, sim.h))

    def run(self, max_steps: int) -> int:
        """Advance every member by up to max_steps; returns members still short of their budget."""
        return self._check(self.c.ex.cemx_batch_run(self.h, int(max_steps)), "batch_run")

    def tune(self, on: bool = True) -> bool:
        return bool(self.c.ex.cemx_batch_tune(self.h, int(on)))

    def stats(self) -> dict:
        v = (C.c_double * 6)()
        self._check(self.c.ex.cemx_batch_stats(self.h, v, 6), "batch_stats")
        return {"ms": v[0], "steps": int(v[1]), "launches": int(v[2]), "chunk": int(v[3]), "order": int(v[4]),
                "members": int(v[5])}

    def destroy(self):
        if getattr(self, "h", None):
            self.c.ex.cemx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
