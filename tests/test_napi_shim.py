"""The Node shim's call translation (courant_b200/napi), driven through its C
ABI exactly as the reference's TypeScript wrapper drives its wasm module
(web/src/solver/courant.ts:19-85, :166-176): numbers in and out, buffers
allocated with malloc in one memory buffer and addressed by offsets, the
solver's own arrays returned as offsets of copies, field and state arrays
kept live around every call. Node itself is not installed here: the module
source (napi/courant_napi.cc) is compiled against the documented N-API
declarations only, and loading it into node is for a host that has it."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from courant_b200 import build, scenes

NAPI = ROOT / "courant_b200" / "napi"


class Module:
    """Python stand-in for the `Exports` object the N-API module returns."""

    def __init__(self, library, arena_mb=64):
        if build.needs_build():
            build.build()
        L = C.CDLL(str(build.SHIM_LIB))
        L.cnapi_open.restype = C.c_void_p
        L.cnapi_open.argtypes = [C.c_char_p, C.c_double]
        L.cnapi_close.argtypes = [C.c_void_p]
        L.cnapi_error.restype = C.c_char_p
        L.cnapi_memory.restype = C.c_void_p
        L.cnapi_memory.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.cnapi_malloc.restype = C.c_double
        L.cnapi_malloc.argtypes = [C.c_void_p, C.c_double]
        L.cnapi_free.argtypes = [C.c_void_p, C.c_double]
        L.cnapi_find.argtypes = [C.c_char_p]
        L.cnapi_call.restype = C.c_double
        L.cnapi_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int)]
        self.L = L
        self.h = L.cnapi_open(str(library).encode(), arena_mb)
        assert self.h, L.cnapi_error().decode()
        size = C.c_double()
        base = L.cnapi_memory(self.h, C.byref(size))
        self.buffer = (C.c_uint8 * int(size.value)).from_address(base)   # memory.buffer

    def close(self):
        self.L.cnapi_close(self.h)

    def malloc(self, n):
        return self.L.cnapi_malloc(self.h, n)

    def free(self, p):
        assert self.L.cnapi_free(self.h, p) == 0, self.L.cnapi_error().decode()

    def __getattr__(self, name):
        idx = self.L.cnapi_find(name.encode())
        if idx < 0:
            raise AttributeError(name)

        def fn(*args):
            a = (C.c_double * max(len(args), 1))(*[float(x) for x in args])
            st = C.c_int()
            r = self.L.cnapi_call(self.h, idx, a, len(args), C.byref(st))
            if st.value < 0:
                raise RuntimeError(self.L.cnapi_error().decode())
            return None if st.value == 1 else r
        return fn

    # the typed-array views courant.ts makes of memory.buffer
    def f64(self, off, n):
        return np.frombuffer(self.buffer, dtype=np.float64, count=n, offset=int(off))

    def put(self, values):
        v = np.asarray(values, dtype=np.float64)
        p = self.malloc(8 * v.size)
        self.f64(p, v.size)[:] = v
        return p


def build_parity(m):
    """The reference's parity scene (solver/apps/parity.c) through the module, as courant.ts would build it."""
    from courant_b200.scenes import _parity_grid
    x, y, z = _parity_grid()
    px, py, pz = m.put(x), m.put(y), m.put(z)
    s = m.cem_create(len(x) - 1, len(y) - 1, len(z) - 1, px, py, pz)
    for p in (px, py, pz):
        m.free(p)
    NY = len(y) - 1
    for f in range(6):
        if f != 4:
            assert m.cem_set_boundary(s, f, 1, 4) == 0
    m.cem_material_box(s, -1, 1, -1, 1, 0, z[5], 3.4, 0.02)
    m.cem_pec_box(s, -1, 1, y[NY - 6], 1, 0, z[5])
    m.cem_pec_sheet(s, 2, z[5], x[5], x[19], y[8], y[10])
    p1 = m.cem_add_lumped_port(s, 2, 5, 9, 0, 5, -1, 50)
    m.cem_add_lumped_port(s, 2, 19, 9, 0, 5, -1, 50)
    m.cem_set_gaussian(s, p1, 1.0, 60e-12, 15e-12)
    pf = m.put([5e9, 20e9, 40e9])
    m.cem_set_frequencies(s, 3, pf)
    m.free(pf)
    m.cem_add_vprobe(s, 2, 12, 9, 0, 5, -1)
    m.cem_add_iprobe(s, 0, 12, 7, 11, 4, 5)
    assert m.cem_finalize(s, 0.95) == 0
    return s


@pytest.fixture
def ref_module(ref_lib):
    import oracle
    m = Module(oracle.REF_LIB)
    yield m
    m.close()


def test_module_steps_like_the_library(ref_module, ref_lib):
    """The parity scene stepped through the module (the reference core behind
    it, which steps on the CPU) gives the library's own results bit for bit;
    spectra come back as offsets of copies in the memory buffer."""
    m = ref_module
    s = build_parity(m)
    m.cem_step(s, 300)
    assert m.cem_step_count(s) == 300
    r, meta = scenes.parity_scene(ref_lib)
    r.step(300)
    nf = int(m.cem_nfreq(s))
    for q, p in enumerate(meta["ports"]):
        v = m.f64(m.cem_port_v(s, p), 2 * nf)
        assert np.array_equal(v[0::2] + 1j * v[1::2], r.portV(p))
    assert m.cem_energy(s) == r.energy()
    assert m.cem_dt(s) == r.dt
    m.cem_destroy(s)


def test_field_arrays_are_live(ref_module, ref_lib):
    """An initial condition written into the cem_field array before stepping
    is taken up, and the same array shows the fields after every step, as
    with the library's own pointer."""
    m = ref_module
    s = build_parity(m)
    r, _ = scenes.parity_scene(ref_lib)
    N = len(r.field(1))
    view = m.f64(m.cem_field(s, 1), N)
    rng = np.random.default_rng(5)
    init = np.zeros(N)
    idx = rng.integers(0, N, 50)
    init[idx] = rng.normal(size=50)
    view[:] = init
    r.fieldView(1)[:] = init
    for _ in range(3):
        m.cem_step(s, 40)
        r.step(40)
        assert np.array_equal(view, r.field(1))
    m.cem_destroy(s)


def test_plan_arrays_and_errors_through_the_module(lib):
    """libcourant_b200 behind the module (no GPU needed for set-up): plan
    arrays equal the library's own, pointer arguments of zero mean NULL,
    and cem_last_error comes back as a string in the buffer."""
    m = Module(build.LIB)
    try:
        s = build_parity(m)
        ref, _ = scenes.parity_scene(lib)
        plan = ref.plan()
        N = plan["N"]
        assert np.array_equal(m.f64(m.cem_plan_array(s, 0, 1), N), plan["ca"][1])
        assert np.array_equal(m.f64(m.cem_plan_array(s, 2, 0), plan["nx"] + 1), plan["ide"][0])
        n = int(m.cem_plan_port(s, 0, 0, 0, 0))
        a, b, c = m.malloc(8 * n), m.malloc(8 * n), m.malloc(8 * n)
        assert m.cem_plan_port(s, 0, a, b, c) == n
        assert np.array_equal(m.f64(a, n), plan["ports"][0]["idx"])
        assert m.cem_set_boundary(s, 0, 1, 4) == -1          # setters refuse after finalize
        p = int(m.cem_last_error())
        msg = bytes(m.buffer[p:p + 200]).split(b"\0")[0].decode()
        assert "finalized" in msg
        m.cem_destroy(s)
        with pytest.raises(RuntimeError, match="handle"):
            m.cem_dt(s)
        with pytest.raises(RuntimeError, match="outside"):
            m.cem_set_frequencies(build_parity(m), 1, 1e12)
    finally:
        m.close()


def test_arena_allocator_reuses_and_coalesces(lib):
    m = Module(build.LIB, arena_mb=1)
    try:
        a = m.malloc(1000)
        b = m.malloc(1000)
        assert a and b and a % 16 == 0 and b >= a + 1000
        m.free(a)
        m.free(b)
        c = m.malloc(1900)       # the two freed neighbours merged
        assert c == a
        assert m.malloc(10 * 1048576) == 0   # larger than the buffer: NULL
        with pytest.raises(AssertionError):
            m.free(c + 16)                   # not a block malloc returned
    finally:
        m.close()


def test_every_exports_entry_is_served():
    """Each function of courant.ts's Exports interface has a translation."""
    import re
    lib = C.CDLL(str(build.SHIM_LIB))
    lib.cnapi_find.argtypes = [C.c_char_p]
    src = (ROOT / "courant_b200" / "napi" / "shim_functions.inc").read_text()
    names = re.findall(r"CNAPI_FN\((cem_\w+)\)", src)
    for n in names:
        if n != "cem_dims":
            assert lib.cnapi_find(n.encode()) >= 0, n


def test_module_source_compiles_against_node_api():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                        "-DNODE_GYP_MODULE_NAME=courant_napi", f"-I{ROOT / 'tests' / 'napi_stub'}",
                        str(NAPI / "courant_napi.cc")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    gyp = (NAPI / "binding.gyp").read_text()
    for f in ("courant_napi.cc", "shim.cpp", "shim_exports.cpp", "arena.cpp"):
        assert f in gyp
