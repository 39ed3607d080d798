"""Seeded synthetic printed-circuit boards over the courant.h ABI.

The generator follows the layered board model of the reference's importer
(skyhoffert/CourantEM web/src/board/kicad.ts:51-76: a stackup of dielectric
cores with copper on their faces, traces, vias, planes) and its mesh rules
(web/src/mesh/mesher.ts:1-12: cells refined where copper is), restated in
Python since the reference builds boards in TypeScript. A board is four copper
layers on three cores:

- L1 (z = 0): the bottom ground, the PEC z-low face of the domain;
- L2 (top of core 1): a ground plane over the whole grid with random
  rectangular clearances;
- L3 (top of core 2): stripline traces;
- L4 (top of core 3): microstrip traces under air;

cores 0.2-1.0 mm thick with eps_r uniform in 3.0-4.5, each a 4-pole
Djordjevic-Sarkar (tan d 0.02 at 1 GHz) Debye fit sharing one set of poles;
traces of width 0.1-0.5 mm running along x with random 45-degree bends
(staircased on the grid); through-vias as PEC columns; CPML on the open faces.
Two ports sit at the ends of trace 0 (on L4, over the L2 plane): 2D
eigenmode ports, or 50-ohm lumped ports. All randomness comes from numpy's PCG64 seeded with `seed`; the
grid is uniform in x and y and graded in z, sized by `cells`.
"""
from __future__ import annotations

import math

import numpy as np

from .api import Courant

CPML = 1
X, Y, Z = 0, 1, 2


def _dims(cells: float) -> tuple[int, int, int]:
    """Cell counts with the aspect of the 1500 x 1000 x 64 reference board,
    z at least 24 cells (layers, air, CPML)."""
    nz = int(np.clip(round(64 * (cells / 96e6) ** (1 / 3)), 24, 64))
    nxy = cells / nz
    ny = max(int(round(math.sqrt(nxy / 1.5))), 24)
    nx = max(int(round(nxy / ny)), 32)
    return nx, ny, nz


def seeded_board(c: Courant, seed: int, cells: float = 2e6, *, ports: str = "mode", nf: int = 32,
                 fmax: float = 20e9, steps: int | None = None, traces: int = 20, vias: int = 30,
                 npml: int = 8, cfl: float = 0.99, excite: int = 1):
    """Finalized board simulation and its metadata (dims, cells, ports,
    frequencies, step count). `cells` sets the grid size; `traces` and `vias`
    scale down for small grids so features stay at least two cells wide;
    `excite` (1 or 2) picks the driven port, the two excitations of a full
    2-port measurement."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, ny, nz = _dims(cells)
    cores = rng.uniform(0.2e-3, 1.0e-3, 3)
    eps = rng.uniform(3.0, 4.5, 3)
    zl = np.concatenate([[0.0], np.cumsum(cores)])          # L1..L4 heights
    air = 1.5e-3
    # z: cores split evenly over most cells, air above, CPML cells at the top
    ncore = max(4, (nz - npml - 6) // 3)
    zs = [0.0]
    for q in range(3):
        zs += list(zl[q] + cores[q] * np.arange(1, ncore + 1) / ncore)
    nair = nz - 3 * ncore
    dz_air = air / max(nair - npml, 1)
    zs += list(zl[3] + dz_air * np.arange(1, nair + 1))
    z = np.array(zs)
    kl = [0] + [ncore * (q + 1) for q in range(3)]           # k index of L1..L4
    # x, y uniform 0.1 mm cells: the board grows with the grid
    dx = 0.1e-3
    x = dx * np.arange(nx + 1)
    y = dx * np.arange(ny + 1)
    s = c.createSim(x, y, z)
    for f in (0, 1, 2, 3, 5):
        s.setBoundary(f, CPML, npml)
    fmin = 1e8
    fits = [c.fitDjordjevicSarkar(float(e), 0.02, 1e9, fmin, fmax, 4) for e in eps]
    s.setDebyePoles(fits[0].fp)
    big = 1.0
    for q in range(3):
        s.materialBoxDebye(-big, big, -big, big, zl[q], zl[q + 1], fits[q])
    # keep copper away from the CPML, and the x ends (the port cross-sections) clear of all but trace 0
    i_lo, i_hi = npml + 12, max(nx - npml - 12, npml + 20)
    j_lo, j_hi = npml + 2, ny - npml - 2
    xs, ys = x, y
    # L2 ground plane with clearances
    nclr = max(1, min(6, (j_hi - j_lo) // 12))
    clear = []
    for _ in range(nclr):
        ci = int(rng.integers(i_lo + 4, max(i_lo + 5, i_hi - 8)))
        cj = int(rng.integers(j_lo + 2, max(j_lo + 3, j_hi - 6)))
        clear.append((ci, ci + int(rng.integers(2, 6)), cj, cj + int(rng.integers(2, 5))))
    # the plane spans the whole grid (uniform cross-sections at the ports), split in y bands at the
    # clearance edges, each band covered by the x intervals outside its clearances
    yb = sorted({0, ny} | {a for cl in clear for a in (cl[2], cl[3])})
    for b0, b1 in zip(yb[:-1], yb[1:]):
        if b1 <= b0:
            continue
        cuts = sorted((cl[0], cl[1]) for cl in clear if cl[2] <= b0 and cl[3] >= b1)
        a = 0
        for c0, c1 in cuts:
            if c0 > a:
                s.pecSheet(Z, zl[1], xs[a], xs[c0], ys[b0], ys[b1])
            a = max(a, c1)
        if a < nx:
            s.pecSheet(Z, zl[1], xs[a], xs[nx], ys[b0], ys[b1])
    # traces: x-directed runs with 45-degree staircased jogs; trace 0 on L4 is the port trace
    ntr = max(1, min(traces, (j_hi - j_lo) // 6))
    rows = np.linspace(j_lo + 2, j_hi - 4, ntr).astype(int)
    t0_j, t0_w = None, None
    for t in range(ntr):
        layer = 3 if t % 2 == 0 else 2
        zt = zl[layer]
        w = int(max(1, round(rng.uniform(0.1e-3, 0.5e-3) / dx)))
        j = int(rows[t])
        if t == 0:
            t0_j, t0_w = j, w
            s.pecSheet(Z, zt, xs[0] - 1.0, xs[nx] + 1.0, ys[j], ys[j + w])   # straight, through the ports
            continue
        i = i_lo
        while i < i_hi:
            run = int(rng.integers(6, 20))
            i1 = min(i + run, i_hi)
            s.pecSheet(Z, zt, xs[i], xs[i1], ys[j], ys[j + w])
            i = i1
            if i >= i_hi:
                break
            jog = int(rng.integers(-3, 4))
            step = 1 if jog > 0 else -1
            for _ in range(abs(jog)):                        # one cell right and one up per step
                j2 = j + step
                if j2 < j_lo or j2 + w > j_hi:
                    break
                i2 = min(i + 1, i_hi)
                s.pecSheet(Z, zt, xs[i], xs[i2], ys[min(j, j2)], ys[max(j, j2) + w])
                i, j = i2, j2
    # through-vias (PEC columns of one or two cells), L1 to L4, away from trace 0
    nv = max(1, min(vias, (i_hi - i_lo) * (j_hi - j_lo) // 200))
    for _ in range(nv):
        vi = int(rng.integers(i_lo, i_hi - 2))
        vj = int(rng.integers(j_lo, j_hi - 2))
        if t0_j - 2 <= vj <= t0_j + t0_w + 2:
            continue
        e = int(rng.integers(1, 3))
        s.pecBox(xs[vi], xs[vi + e], ys[vj], ys[vj + e], 0.0, zl[3])
    tau = math.sqrt(6.9) / (math.pi * 1.25 * fmax)
    freqs = np.linspace(fmax / nf, fmax, nf)
    meta = {"seed": seed, "dims": (nx, ny, nz), "cells": nx * ny * nz, "tau": tau, "freqs": freqs, "excite": excite}
    ktop = kl[3]
    if ports == "mode":
        d = dict(j0=0, j1=ny, k0=0, k1=nz, vj=t0_j, vk0=kl[1], vk1=ktop, vsign=-1, ja=max(t0_j - 1, 0),
                 jb=t0_j + t0_w, ka=ktop - 1, kb=ktop, f0=0.5 * fmax, neff0=math.sqrt((float(eps[2]) + 1) / 2))
        p1 = s.addModePort(dict(d, dir=1, iSrc=npml + 2, iMon=npml + 6, xRef=xs[npml + 8]))
        p2 = s.addModePort(dict(d, dir=-1, iSrc=nx - npml - 2, iMon=nx - npml - 7, xRef=xs[nx - npml - 8]))
        s.setModeExcitation(p1 if excite == 1 else p2, 4.5 * tau, tau)
        meta["modeports"] = [p1, p2]
    else:
        p1 = s.addLumpedPort(Z, npml + 4, t0_j, kl[1], ktop, -1, 50.0)     # L2 ground to the L4 trace
        p2 = s.addLumpedPort(Z, nx - npml - 4, t0_j, kl[1], ktop, -1, 50.0)
        s.setGaussian(p1 if excite == 1 else p2, 1.0, 4.5 * tau, tau)
        meta["ports"] = [p1, p2]
    s.setFrequencies(freqs)
    s.finalize(cfl)
    meta["steps"] = int(steps if steps is not None else min(40000, max(4000, int(12 * tau / s.dt) * 10)))
    return s, meta
