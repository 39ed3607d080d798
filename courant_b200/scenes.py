"""Scenario builders over the courant.h ABI (any library: B200 engine or oracle).

Each builder takes a `courant_b200.api.Courant` and returns `(sim, meta)`:
a finalized `Sim` and a dict with the frequencies, port/probe indices and the
step count the scenario is meant to run.

- parity_scene: the reference's every-feature known-answer scene
  (skyhoffert/CourantEM solver/apps/parity.c:11-31): non-uniform grid, CPML on
  five faces, lossy dielectric, PEC box and sheet, two lumped ports, V and I
  probes, 1500 steps.
- lossy_scene: the reference checkpoint scene (solver/tests/test_checkpoint.c:11-33):
  the same grid with 3 Debye poles and copper surface impedance.
- gcpw_line: grounded coplanar waveguide between two ports in the manner of
  solver/apps/gcpw_line.c (graded mesh :43-78, geometry :181-239, ports
  :243-268), parameterised for the benchmark workloads.
"""
from __future__ import annotations

import math

import numpy as np

from .api import Courant, DebyeModel

CPML = 1
X, Y, Z = 0, 1, 2


def _parity_grid(NX=24, NY=18, NZ=14, warp_y=True):
    x = np.array([1e-4 * i + 2e-6 * i * i for i in range(NX + 1)])
    if warp_y:
        y = np.array([1e-4 * (j - NY // 2) * (1 + 0.01 * abs(j - NY / 2.0)) for j in range(NY + 1)])
    else:
        y = np.array([1e-4 * (j - NY // 2) for j in range(NY + 1)])
    z = np.array([5e-5 * k + 1e-6 * k * k for k in range(NZ + 1)])
    return x, y, z


def parity_scene(c: Courant, cfl: float = 0.95):
    x, y, z = _parity_grid()
    NY = len(y) - 1
    s = c.createSim(x, y, z)
    for f in range(6):
        if f != 4:
            s.setBoundary(f, CPML, 4)
    s.materialBox(-1, 1, -1, 1, 0, z[5], 3.4, 0.02)
    s.pecBox(-1, 1, y[NY - 6], 1, 0, z[5])
    s.pecSheet(Z, z[5], x[5], x[19], y[8], y[10])
    p1 = s.addLumpedPort(Z, 5, 9, 0, 5, -1, 50)
    p2 = s.addLumpedPort(Z, 19, 9, 0, 5, -1, 50)
    s.setGaussian(p1, 1.0, 60e-12, 15e-12)
    freqs = [5e9, 20e9, 40e9]
    s.setFrequencies(freqs)
    v = s.addVProbe(Z, 12, 9, 0, 5, -1)
    ip = s.addIProbe(X, 12, 7, 11, 4, 5)
    s.finalize(cfl)
    return s, {"freqs": freqs, "ports": [p1, p2], "vprobes": [v], "iprobes": [ip], "steps": 1500}


def lossy_scene(c: Courant, cfl: float = 0.95, rough: int = 0, p1: float = 0.0, p2: float = 0.0):
    x, y, z = _parity_grid(warp_y=False)
    s = c.createSim(x, y, z)
    for f in range(6):
        if f != 4:
            s.setBoundary(f, CPML, 4)
    s.setDebyePoles([1e9, 10e9, 100e9])
    s.materialBoxDebye(-1, 1, -1, 1, 0, z[5], DebyeModel(3.4, [], [0.02, 0.03, 0.02], 0.0))
    s.setConductorLoss(5.8e7, 1e9, 40e9, rough, p1, p2)
    s.pecSheet(Z, z[5], x[5], x[19], y[8], y[10])
    a = s.addLumpedPort(Z, 5, 9, 0, 5, -1, 50)
    b = s.addLumpedPort(Z, 19, 9, 0, 5, -1, 50)
    s.setGaussian(a, 1.0, 60e-12, 15e-12)
    freqs = [5e9, 20e9, 40e9]
    s.setFrequencies(freqs)
    v = s.addVProbe(Z, 12, 9, 0, 5, -1)
    ip = s.addIProbe(X, 12, 7, 11, 4, 5)
    s.finalize(cfl)
    return s, {"freqs": freqs, "ports": [a, b], "vprobes": [v], "iprobes": [ip], "steps": 900}


# ---------------------------------------------------------------- GCPW line

def graded(fix, ref, hmin, hmax, ratio=1.3):
    """Graded 1D mesh: every fixed line kept; spacing hmin at refinement points,
    growing by `ratio` per cell up to hmax; each segment's remainder spread
    uniformly (the rule of gcpw_line.c:41-78, restated)."""
    pts = sorted(fix)
    out = [pts[0]]
    for a, b in zip(pts[:-1], pts[1:]):
        if b - a < 1e-15:
            continue
        seg = []
        x = a
        while True:
            d = min(abs(x - r) for r in ref) if ref else 1e300
            h = min(hmax, hmin + (ratio - 1) * d)
            d2 = min(abs(x + h - r) for r in ref) if ref else 1e300
            h = min(h, min(hmax, hmin + (ratio - 1) * d2))
            if x + h >= b - 0.5 * h:
                break
            x += h
            seg.append(x)
        if seg:
            last = seg[-1]
            prev = last - seg[-2] if len(seg) > 1 else last - a
            k = (b - a) / ((last - a) + prev)
            out += [a + (v - a) * k for v in seg]
        out.append(b)
    return np.array(out)


def _nearest(a, x):
    return int(np.argmin(np.abs(np.asarray(a) - x)))


def gcpw_line(c: Courant, *, w=0.45e-3, gap=0.2e-3, h=0.254e-3, er=4.3, length=10e-3, hmin=25e-6, hmax=200e-6,
              dx=None, fence=0.3e-3, yair=1.0e-3, zair=1.5e-3, npml=8, fmax=40e9, df=0.1e9, nf=None,
              tcu=0.0, mask=0.0, mask_er=3.5, debye_poles=0, sigma_cu=0.0, huray=None, modeports=False,
              feed=4.0e-3, mon=2.5e-3, excite=1, cfl=0.99, steps=20000, probes=False, fstart=None):
    """Grounded coplanar waveguide: trace (width w) and top grounds as PEC sheets
    (or copper boxes of thickness tcu), PEC floor, PEC fence walls beyond each
    gap, CPML on the open faces. Lumped 50-ohm ports at both ends of the line,
    or 2D eigenmode ports (modeports=True) fed from behind the reference planes.
    Optional: solder mask (thickness `mask`, eps `mask_er`), a Djordjevic-Sarkar
    substrate fitted by `debye_poles` poles (Df 0.02 at 1 GHz), copper surface
    impedance (sigma_cu) with Huray roughness huray=(radius, density)."""
    a = w / 2
    b = w / 2 + gap
    yf = b + fence
    yext = yf + yair
    top = h + tcu + mask
    ztop = top + zair
    t1, t2 = hmin / 3, 2 * hmin / 3
    snap = tcu > 0
    if snap:
        yfix = [-yext, -yf, -b, -a, 0, a, b, yf, yext]
    else:
        yfix = [-yext, -yf, -b - t1, -b + t2, -a - t2, -a + t1, 0, a - t1, a + t2, b - t2, b + t1, yf, yext]
    Ym = graded(yfix, [-b, -a, a, b], hmin, hmax)
    zfix = [0.0, h, ztop]
    zref = [h]
    if tcu > 0:
        zfix.append(h + tcu)
        zref.append(h + tcu)
    if mask > 0:
        zfix.append(top)
        zref.append(top)
    Zm = graded(zfix, zref, hmin, hmax)
    Y = np.concatenate([Ym[0] - hmax * np.arange(npml, 0, -1), Ym, Ym[-1] + hmax * np.arange(1, npml + 1)])
    Zv = np.concatenate([Zm, Zm[-1] + hmax * np.arange(1, npml + 1)])
    dxl = dx if dx else hmax / 2
    nlen = int(round(length / dxl))
    nfeed = int(round((feed if modeports else 0.5e-3) / dxl))
    Xv = dxl * np.arange(-nfeed - npml, nlen + nfeed + npml + 1)
    nx, ny, nz = len(Xv) - 1, len(Y) - 1, len(Zv) - 1
    ip1, ip2 = nfeed + npml, nfeed + npml + nlen
    j0 = _nearest(Y, 0.0)
    kh = _nearest(Zv, h)
    kt = _nearest(Zv, h + tcu) if tcu > 0 else kh
    s = c.createSim(Xv, Y, Zv)
    for f in (0, 1, 2, 3, 5):
        s.setBoundary(f, CPML, npml)
    xlo, xhi, ylo, yhi = Xv[0] - 1, Xv[-1] + 1, Y[0] - 1, Y[-1] + 1
    if debye_poles:
        m = c.fitDjordjevicSarkar(er, 0.02, 1e9, 1e8 if df >= 1e8 else df, fmax, debye_poles)
        s.setDebyePoles(m.fp)
        s.materialBoxDebye(xlo, xhi, ylo, yhi, 0, h, m)
    else:
        s.materialBox(xlo, xhi, ylo, yhi, 0, h, er, 0)
    if mask > 0:
        s.materialBox(xlo, xhi, ylo, yhi, h + tcu, top, mask_er, 0)
    s.pecBox(xlo, xhi, ylo, -yf, 0, h)
    s.pecBox(xlo, xhi, yf, yhi, 0, h)
    xs0, xs1 = (xlo, xhi) if modeports else (Xv[ip1], Xv[ip2])
    if tcu > 0:
        s.pecBox(xlo, xhi, ylo, -b, h, h + tcu)
        s.pecBox(xlo, xhi, b, yhi, h, h + tcu)
        s.pecBox(xs0, xs1, -a, a, h, h + tcu)
    else:
        s.pecSheet(Z, h, xlo, xhi, ylo, -b)
        s.pecSheet(Z, h, xlo, xhi, b, yhi)
        s.pecSheet(Z, h, xs0, xs1, -a, a)
    if sigma_cu > 0:
        rough, p1, p2 = (2, huray[0], huray[1]) if huray else (0, 0.0, 0.0)
        s.setConductorLoss(sigma_cu, df, fmax, rough, p1, p2)
    tau = math.sqrt(6.9) / (math.pi * 1.25 * fmax)
    jl, jr = _nearest(Y, -(a + b) / 2), _nearest(Y, (a + b) / 2)
    ja, jb = max(jl, 0), jr - 1
    meta = {"dims": (nx, ny, nz), "cells": nx * ny * nz, "ip1": ip1, "ip2": ip2, "tau": tau, "steps": steps,
            "excite": excite}
    if not modeports:
        p1 = s.addLumpedPort(Z, ip1, j0, 0, kh, -1, 50.0)
        p2 = s.addLumpedPort(Z, ip2, j0, 0, kh, -1, 50.0)
        s.setGaussian(p1 if excite == 1 else p2, 1.0, 4.5 * tau, tau)
        meta["ports"] = [p1, p2]
    else:
        monc = int(round(mon / dxl))
        d = dict(j0=0, j1=ny, k0=0, k1=nz, vj=j0, vk0=0, vk1=kh, vsign=-1, ja=ja, jb=jb, ka=kh - 1, kb=kt,
                 f0=0.5 * fmax, neff0=math.sqrt((er + 1) / 2))
        d1 = dict(d, dir=1, iSrc=npml + 2, iMon=npml + 2 + monc, xRef=Xv[ip1])
        d2 = dict(d, dir=-1, iSrc=nx - npml - 2, iMon=nx - npml - 2 - monc - 1, xRef=Xv[ip2])
        m1, m2 = s.addModePort(d1), s.addModePort(d2)
        s.setModeExcitation(m1 if excite == 1 else m2, 4.5 * tau, tau)
        meta["modeports"] = [m1, m2]
    if nf:
        freqs = np.linspace(fmax / nf, fmax, nf)
    elif fstart:      # fstart, fstart + df, ..., fmax
        freqs = df * np.arange(int(round(fstart / df)), int(round(fmax / df)) + 1)
    elif modeports:   # the mode solve needs f > 0 (gcpw_line.c:270-272)
        freqs = df * np.arange(1, int(round(fmax / df)) + 1)
    else:             # 0, df, ..., fmax
        freqs = np.linspace(0.0, fmax, int(round(fmax / df)) + 1)
    s.setFrequencies(freqs)
    meta["freqs"] = freqs
    if probes:
        meta["vprobes"] = [s.addVProbe(Z, (ip1 + ip2) // 2, j0, 0, kh, -1)]
        meta["iprobes"] = [s.addIProbe(X, (ip1 + ip2) // 2, ja, jb, kh - 1, kt)]
    s.finalize(cfl)
    return s, meta


# The two GCPW configurations of the benchmark, as gcpw_line keyword sets.
# c1: lossless GCPW, lumped 50-ohm ports, eps_r 4.3, h 254 um, w 450 um, gap 200 um, 10 mm, graded 25-200 um
#     (121 x 62 x 40 cells), 20 000 steps, 401 frequencies 0-40 GHz.
# c2: the same line with 35 um copper, a 20 um eps_r 3.5 mask, a Djordjevic-Sarkar substrate (6 Debye poles), copper
#     surface impedance with Huray roughness (sphere radius 0.5 um, 2e11 spheres per m^2 of flat area:
#     K(inf) = 1 + 4 pi a^2 N = 1.63, standing in for Rq = 1 um), 2D eigenmode ports (416 x 161 x 86 cells),
#     40 000 steps, 351 frequencies 5-40 GHz (below about 4.4 GHz the reference's 2D mode solver stops converging on
#     this cross-section as a second mode approaches the shift of its inverse iteration, so the reference core cannot
#     give S-parameters there).
CONFIGS = {
    "c1": dict(desc="lossless GCPW, lumped 50-ohm ports, er 4.3, h 254um, w 450um, gap 200um, 10 mm",
               kw=dict(hmin=25e-6, hmax=200e-6, dx=105e-6, zair=4.2e-3, yair=0.9e-3, steps=20000)),
    "c2": dict(desc="lossy GCPW 2-port: DS substrate (6 Debye poles), 35um Cu + Huray SIBC, 20um mask, mode ports",
               kw=dict(hmin=10e-6, hmax=30e-6, dx=45e-6, yair=1.2e-3, zair=1.8e-3, tcu=35e-6, mask=20e-6,
                       debye_poles=6, sigma_cu=5.8e7, huray=(0.5e-6, 2.0e11), modeports=True, steps=40000,
                       fstart=5e9)),
}


def config_line(c: Courant, name: str, excite: int = 1, **over):
    """One of the benchmark GCPW configurations (CONFIGS), driven at port `excite`."""
    return gcpw_line(c, **dict(CONFIGS[name]["kw"], excite=excite, **over))


def s_column(s, meta: dict) -> dict:
    """The excited column of the modal or lumped S-matrix: the waves at every
    port divided by the incident wave at the driven port. Mode ports use
    cem_mode_port_waves (a, b at the reference planes, normalised to each port's
    own Z0); lumped ports use V and I with the 50-ohm port resistance."""
    e = meta.get("excite", 1) - 1
    if "modeports" in meta:
        w = [s.modePortWaves(p) for p in meta["modeports"]]
        a = w[e]["a"]
        return {"b": [x["b"] / a for x in w], "z0": [x["z0"] for x in w], "beta": [x["beta"] for x in w]}
    v = [s.portV(p) for p in meta["ports"]]
    i = [s.portI(p) for p in meta["ports"]]
    sq = np.sqrt(50.0)
    a = (v[e] + 50.0 * i[e]) / (2 * sq)
    return {"b": [(v[q] - 50.0 * i[q]) / (2 * sq) / a for q in range(len(v))]}


two_port_s = s_column


def modeport_scene(c: Courant):
    """Small lossy GCPW between 2D eigenmode ports, exercising every step
    kernel at once: CPML on five faces, a 4-pole Djordjevic-Sarkar substrate,
    35 um copper with Huray-rough surface impedance, a solder mask, the modal
    source plane, and the port and probe line integrals. 1600 steps (the modal
    pulse peaks near step 1250)."""
    s, meta = gcpw_line(c, length=2e-3, hmin=50e-6, hmax=250e-6, dx=125e-6, yair=0.5e-3, zair=0.7e-3, npml=6,
                        feed=1e-3, mon=0.5e-3, nf=8, tcu=35e-6, mask=20e-6, debye_poles=4, sigma_cu=5.8e7,
                        huray=(0.5e-6, 2.0e11), modeports=True, probes=True, steps=1600)
    meta["vprobes"] = list(range(c.ex.cem_plan_nvprobe(s.h)))
    meta["iprobes"] = list(range(c.ex.cem_plan_niprobe(s.h)))
    return s, meta
