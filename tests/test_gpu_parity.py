"""GPU engine against the oracle (f64 CPU restatement of the reference step,
itself pinned to the reference bit for bit).

Tolerances: fields relative L2 <= 1e-5 per component at matching steps (the
FP32 engine against the f64 core); probe and port spectra relative to their
peak <= 1e-5; energy <= 1e-5; S-parameters within 1e-3 dB and 0.01 degree
where |S| > -40 dB, f >= 1 GHz. Checkpoint resume and slab-split phased
stepping must match straight stepping bit for bit."""
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from courant_b200 import scenes
from tests_util import db_deg, rel_l2

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
SPEC_TOL = 1e-5
# The FP32 engine's rounding error is ~1e-6 of the peak field; once a pulse
# has left the domain the remaining field is a few percent of that peak, so
# late-time errors are normalised by the peak (see test_scene_against_oracle).


def spectra(s, meta):
    out = {}
    for p in meta.get("ports", []):
        out[f"V{p}"], out[f"I{p}"] = s.portV(p), s.portI(p)
    for p in meta.get("vprobes", []):
        out[f"vp{p}"] = s.vprobe(p)
    for p in meta.get("iprobes", []):
        out[f"ip{p}"] = s.iprobe(p)
    out["src"] = s.sourceSpectrum()
    return out


def field_errors(gpu, orc, scale=None):
    """Relative L2 error per component; with `scale` (per-component norms),
    relative to those instead of the current norm."""
    out = {}
    for c in range(6):
        a, r = gpu.field(c), orc.field(c)
        n = scale[c] if scale is not None else np.linalg.norm(r)
        out[f"field{c}"] = float(np.linalg.norm(a - r) / n)
    return out


def spectrum_errors(gpu, orc, meta):
    sg, so = spectra(gpu, meta), spectra(orc, meta)
    return {k: float(np.max(np.abs(sg[k] - so[k])) / max(np.max(np.abs(so[k])), 1e-300)) for k in sg}


def board_scene(lib):
    """A seeded 4-layer board (three Debye cores at different heights, CPML
    on five faces, traces, vias, lumped ports): many update rectangles of
    every class, so a block classed fast by mistake would show here."""
    from courant_b200 import boards
    s, meta = boards.seeded_board(lib, 7, 1.2e5, ports="lumped", nf=16, steps=800, excite=1)
    return s, meta


@pytest.mark.parametrize("fused", [False, True], ids=["separate", "fused"])
@pytest.mark.parametrize("fn", [scenes.parity_scene, scenes.lossy_scene, scenes.modeport_scene, board_scene],
                         ids=["parity", "lossy", "modeport", "board"])
def test_scene_against_oracle(lib, oracle_lib, fn, fused):
    """At step 600 (fields near their peak, the step of the reference's own
    GPU-vs-CPU check) every component is within relative L2 1e-5 of the f64
    oracle, and max|diff|/max|field| per E/H family as the reference measures
    it. At the end of the run, where the fields have decayed to a few percent
    of their peak, errors are measured against the largest peak norm of the
    component's family (E or H) over the run: FP32 rounding scales with the
    whole field, so a small component such as the longitudinal E of a line
    carries errors of its family's size. Spectra and energy against their own
    magnitude."""
    s, meta = fn(lib)
    s.useFused(fused)
    n = meta["steps"]
    o = oracle_lib.OracleSim.from_sim(s, meta["freqs"], n)
    peak = np.zeros(6)
    done = 0
    for upto in (300, 600, n):
        s.step(upto - done)
        o.step(upto - done)
        done = upto
        peak = np.maximum(peak, [np.linalg.norm(o.field(c)) for c in range(6)])
        if upto == 600:
            e = field_errors(s, o)
            assert max(e.values()) < FIELD_TOL, e
            for fam in (range(3), range(3, 6)):
                worst = max(np.max(np.abs(s.field(c) - o.field(c))) for c in fam)
                scale = max(np.max(np.abs(o.field(c))) for c in fam)
                assert worst / scale < FIELD_TOL
    assert s.steps == o.steps == n
    fam = np.repeat([peak[:3].max(), peak[3:].max()], 3)
    e = field_errors(s, o, fam)
    assert max(e.values()) < FIELD_TOL, e
    sp = spectrum_errors(s, o, meta)
    assert max(sp.values()) < SPEC_TOL, sp
    assert abs(s.energy() - o.energy()) / o.energy() < SPEC_TOL


def test_parity_scene_against_reference_printout(lib):
    """The reference known-answer printout (tests/golden/parity_scene.txt)."""
    s, meta = scenes.parity_scene(lib)
    s.step(1500)
    ref = {}
    for line in (ROOT / "tests" / "golden" / "parity_scene.txt").read_text().splitlines():
        k, *v = line.split()
        ref[k] = [float(x) for x in v]
    assert s.dt == ref["dt"][0]
    assert abs(s.energy() - ref["energy"][0]) / ref["energy"][0] < 1e-5
    arrs = {"V1": s.portV(0), "V2": s.portV(1), "Vp": s.vprobe(0), "Ip": s.iprobe(0)}
    for name, a in arrs.items():
        r = np.array([complex(*ref[f"{name}[{q}]"]) for q in range(3)])
        assert np.max(np.abs(a - r)) / np.max(np.abs(r)) < SPEC_TOL, name


@pytest.mark.parametrize("fused", [False, True], ids=["separate", "fused"])
def test_checkpoint_resume_bit_exact(lib, fused):
    A, _ = scenes.lossy_scene(lib)
    B, _ = scenes.lossy_scene(lib)
    C, meta = scenes.lossy_scene(lib)
    for x in (A, B, C):
        x.useFused(fused)
    A.step(900)
    B.step(400)
    buf = B.checkpoint()
    C.restore(buf)
    C.step(500)
    for c in range(6):
        assert np.array_equal(A.field(c), C.field(c)), c
    for p in meta["ports"]:
        assert np.array_equal(A.portV(p), C.portV(p))
    assert np.array_equal(A.vprobe(0), C.vprobe(0))


def test_checkpoint_from_reference_resumes(lib, ref_lib):
    """A checkpoint written by the reference core at step 400 resumes on the
    GPU engine; 200 steps later fields and spectra match the reference run."""
    R, meta = scenes.lossy_scene(ref_lib)
    R.step(400)
    buf = R.checkpoint()
    G, _ = scenes.lossy_scene(lib)
    G.restore(buf)
    assert G.steps == 400
    G.step(200)
    R.step(200)
    for c in range(6):
        assert rel_l2(G.field(c), R.field(c)) < FIELD_TOL, c
    for p in meta["ports"]:
        assert np.max(np.abs(G.portV(p) - R.portV(p))) / np.max(np.abs(R.portV(p))) < SPEC_TOL


@pytest.mark.parametrize("fused", [False, True], ids=["separate", "fused"])
def test_phased_stepping_matches_cem_step(lib, fused):
    """The cem_mt_* phases (separate kernels, any slab split) give the same bits as cem_step."""
    A, _ = scenes.parity_scene(lib)
    B, _ = scenes.parity_scene(lib)
    A.useFused(fused)
    A.step(50)
    nx = B.nx
    for _ in range(50):
        B.c.ex.cem_mt_pre(B.h)
        B.c.ex.cem_mt_H(B.h, 0, nx // 3)
        B.c.ex.cem_mt_H(B.h, nx // 3, nx + 1)
        B.c.ex.cem_mt_mid(B.h)
        B.c.ex.cem_mt_E(B.h, 0, 7)
        B.c.ex.cem_mt_E(B.h, 7, nx)
        B.c.ex.cem_mt_post(B.h)
    assert B.steps == 50
    for c in range(6):
        assert np.array_equal(A.field(c), B.field(c)), c
    assert np.array_equal(A.portV(0), B.portV(0))


def test_graph_runs_match_single_steps(lib):
    """cem_step replays runs of 32 steps as one captured graph; stepping 7 at a
    time never does. Across a DFT ring flush (1024 steps) on the lossy scene
    (SIBC, Debye, CPML) both give the same bits."""
    A, meta = scenes.lossy_scene(lib)
    B, _ = scenes.lossy_scene(lib)
    A.step(1100)
    for _ in range(1100 // 7):
        B.step(7)
    B.step(1100 % 7)
    assert A.steps == B.steps == 1100
    for c in range(6):
        assert np.array_equal(A.field(c), B.field(c)), c
    for p in meta["ports"]:
        assert np.array_equal(A.portV(p), B.portV(p))
        assert np.array_equal(A.portI(p), B.portI(p))


def test_field_initial_condition_and_live_pointer(lib, oracle_lib):
    """Initial E written through cem_field is taken up; the pointer stays live."""
    s, meta = scenes.parity_scene(lib)
    o = oracle_lib.OracleSim.from_sim(s, meta["freqs"], 300)
    view = s.fieldView(1)
    rng = np.random.default_rng(3)
    init = np.zeros(s.N)
    idx = rng.integers(0, s.N, 400)
    init[idx] = rng.normal(size=400)
    view[:] = init
    o.field_view(1)[:] = np.float32(init)   # the engine holds FP32 fields
    for _ in range(3):
        s.step(100)
        o.step(100)
        assert rel_l2(view, o.field(1)) < FIELD_TOL


def test_run_stops_on_energy_decay(lib, oracle_lib):
    s, meta = scenes.parity_scene(lib)
    n = s.run(20000, 1e-3, 100)
    assert 0 < n < 20000 and n % 100 == 0
    o = oracle_lib.OracleSim.from_sim(s, meta["freqs"], n)
    o.step(n)
    assert abs(s.energy() - o.energy()) / o.energy() < 1e-4


@pytest.mark.parametrize("fused", [False, True], ids=["separate", "fused"])
def test_gcpw_lumped_sparams(lib, oracle_lib, fused):
    """S11/S21 of a short lumped-port GCPW within 1e-3 dB / 0.01 degree of the f64 oracle."""
    kw = dict(length=3e-3, hmin=50e-6, hmax=200e-6, dx=100e-6, yair=0.6e-3, zair=0.8e-3, npml=6, df=1e9, steps=3000)
    s, meta = scenes.gcpw_line(lib, **kw)
    s.useFused(fused)
    n = meta["steps"]
    o = oracle_lib.OracleSim.from_sim(s, meta["freqs"], n)
    s.step(n)
    o.step(n)
    from courant_b200.api import s_params
    p1, p2 = meta["ports"]
    g11, g21 = s_params(s.portV(p1), s.portI(p1), s.portV(p2), s.portI(p2), 50.0)
    r11, r21 = s_params(o.portV(p1), o.portI(p1), o.portV(p2), o.portI(p2), 50.0)
    f = np.asarray(meta["freqs"])
    for g, r in ((g11, r11), (g21, r21)):
        sel = (f >= 1e9) & (np.abs(r) > 0.01)
        ddb, ddeg = db_deg(g[sel], r[sel])
        assert ddb.max() < 1e-3 and ddeg.max() < 0.01, (ddb.max(), ddeg.max())
    # the same gate through Touchstone files, as a user would compare them
    from courant_b200 import touchstone
    a = touchstone.write_s2p(None, f, g11, g21, title="gcpw b200")
    b = touchstone.write_s2p(None, f, r11, r21, title="gcpw oracle")
    cmp = touchstone.compare(touchstone.read_s2p(a), touchstone.read_s2p(b), "b200")
    assert cmp["ok"], cmp


def test_reference_parity_program_through_the_drop_in():
    """The reference's known-answer program solver/apps/parity.c, compiled
    unchanged against libcourant_b200 (oracle/_ref/dropin_parity): its printout
    matches the reference's own (tests/golden/parity_scene.txt): dt to the
    bit, energy and every spectrum entry within 1e-5 of the largest entry of
    its array."""
    exe = ROOT / "oracle" / "_ref" / "dropin_parity"
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (make -C oracle dropin)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr

    def parse(txt):
        out = {}
        for line in txt.splitlines():
            k, *v = line.split()
            out[k] = np.array([float(x) for x in v])
        return out

    got, ref = parse(r.stdout), parse((ROOT / "tests" / "golden" / "parity_scene.txt").read_text())
    assert set(got) == set(ref)
    assert got["dt"][0] == ref["dt"][0]
    assert abs(got["energy"][0] - ref["energy"][0]) / ref["energy"][0] < 1e-5
    for name in ("V1", "V2", "Vp", "Ip"):
        keys = [k for k in ref if k.startswith(name + "[")]
        scale = max(np.hypot(*ref[k]) for k in keys)
        for k in keys:
            assert np.hypot(*(got[k] - ref[k])) / scale < SPEC_TOL, (k, got[k], ref[k])


@pytest.mark.parametrize("prog", ["test_checkpoint", "test_mode2d", "test_cavity", "test_cpml", "test_sibc"])
def test_reference_program_links_and_passes(prog):
    """The reference's own known-answer programs, linked unchanged against libcourant_b200."""
    exe = ROOT / "oracle" / "_ref" / f"dropin_{prog}"
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (make -C oracle dropin)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0 and f"{prog} passed" in r.stdout, r.stdout + r.stderr
