"""Rule-based non-uniform mesh lines of one axis.

A restatement in numpy of the reference's board mesher
(skyhoffert/CourantEM web/src/mesh/mesher.ts: meshAxis :52-132, withPml
:136-141, lambdaOver20 :48-50), which the TypeScript board runner uses and
which cannot run here (no node). The rules:

1. fixed lines: the domain ends; planes (thick copper faces, layer
   interfaces) exactly on the grid; zero-thickness metal edges by the thirds
   rule (a line h/3 inside the metal and 2h/3 outside); lines closer than
   hmin/4 are merged, the higher-priority one kept;
2. a minimum number of cells across spans (gaps, dielectric layers);
3. maximum cells per region (lambda/20 in the densest material);
4. neighbouring cells change by at most `ratio`: every constraint is a cap on
   the local cell size that relaxes away from where it applies with slope
   0.8 (ratio - 1), and each interval between fixed lines is filled with
   n = ceil(integral of dx / size(x)) cells at equal steps of that integral.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C0 = 299792458.0
_EPS = 1e-12


def lambda_over_20(fmax: float, er: float) -> float:
    """lambda/20 at fmax in a material of relative permittivity er (mesher.ts:48-50)."""
    return C0 / (fmax * math.sqrt(er)) / 20


@dataclass
class AxisFeatures:
    """mesher.ts AxisFeatures (:16-33): the domain [lo, hi] without CPML."""
    lo: float
    hi: float
    sheet_edges: list = field(default_factory=list)   # (x, 'lo' | 'hi'): metal below / above x
    planes: list = field(default_factory=list)
    spans: list = field(default_factory=list)         # (a, b, n)
    max_cell: list = field(default_factory=list)      # (a, b, h)
    refine: list | None = None
    extra: list = field(default_factory=list)


def _fixed_lines(feat: AxisFeatures, h0: float) -> tuple[list, list]:
    fixed = [(feat.lo, 3), (feat.hi, 3)]
    refine = list(feat.refine) if feat.refine is not None else []
    for p in feat.planes:
        fixed.append((p, 2))
        if feat.refine is None:
            refine.append(p)
    for x, metal in feat.sheet_edges:
        s = -1.0 if metal == "lo" else 1.0   # direction into the metal
        fixed += [(x + s * h0 / 3, 1), (x - s * 2 * h0 / 3, 1)]
        if feat.refine is None:
            refine.append(x)
    fixed += [(x, 2) for x in feat.extra]
    fixed.sort(key=lambda t: t[0])
    lines, pri = [], []
    for x, p in fixed:
        if x < feat.lo - _EPS or x > feat.hi + _EPS:
            continue
        if lines and x - lines[-1] < h0 / 4:
            if p > pri[-1]:
                lines[-1], pri[-1] = x, p
            continue
        lines.append(x)
        pri.append(p)
    return lines, refine


def _size(x: np.ndarray, caps: np.ndarray, refine: np.ndarray, h0: float, hmax: float, g: float) -> np.ndarray:
    """The local cell-size cap of mesher.ts :91-97 at the points x. caps: one
    row (a, b, h) per max_cell region and per span (h = (b - a) / n)."""
    s = np.full(x.shape, hmax)
    if caps.size:
        a, b, h = caps[:, 0:1], caps[:, 1:2], caps[:, 2:3]
        d = np.where(x < a, a - x, np.where(x > b, x - b, 0.0))
        s = np.minimum(s, (h + g * d).min(axis=0))
    if refine.size:
        # nearest refinement point per sample: sorted search instead of a loop over all points
        idx = np.clip(np.searchsorted(refine, x), 1, refine.size - 1) if refine.size > 1 else np.zeros(x.shape, int)
        d = np.abs(x - refine[idx])
        if refine.size > 1:
            d = np.minimum(d, np.abs(x - refine[idx - 1]))
        s = np.minimum(s, h0 + g * d)
    return np.maximum(s, h0 * 0.5)


def mesh_axis(feat: AxisFeatures, hmin: float, hmax: float, ratio: float = 1.3) -> np.ndarray:
    """Node lines of one axis (mesher.ts meshAxis :52-132)."""
    h0 = hmin
    lines, refine = _fixed_lines(feat, h0)
    refine = np.unique(np.asarray(refine, dtype=np.float64))
    caps = np.array([(a, b, h) for a, b, h in feat.max_cell] + [(a, b, (b - a) / n) for a, b, n in feat.spans],
                    dtype=np.float64).reshape(-1, 3)
    g = 0.8 * (ratio - 1)
    nodes = [lines[0]]
    for a, b in zip(lines[:-1], lines[1:]):
        M = max(64, math.ceil((b - a) / (h0 / 8)))
        xs = a + (b - a) * np.arange(M + 1) / M
        inv = 1.0 / _size(xs, caps, refine, h0, hmax, g)
        cum = np.concatenate([[0.0], np.cumsum((xs[1:] - xs[:-1]) * 0.5 * (inv[:-1] + inv[1:]))])
        I = cum[-1]
        n = max(1, math.ceil(I - 1e-6))
        if n > 1:
            target = I * np.arange(1, n) / n
            m = np.clip(np.searchsorted(cum, target, side="left") - 1, 0, M - 1)
            t = (target - cum[m]) / (cum[m + 1] - cum[m])
            nodes += list(a + (b - a) * (m + t) / M)
        nodes.append(b)
    return np.asarray(nodes)


def with_pml(nodes: np.ndarray, n: int, h: float, lo: bool = True, hi: bool = True) -> np.ndarray:
    """n CPML cells of size h appended at the chosen ends (mesher.ts withPml :136-141)."""
    parts = []
    if lo:
        parts.append(nodes[0] - h * np.arange(n, 0, -1))
    parts.append(nodes)
    if hi:
        parts.append(nodes[-1] + h * np.arange(1, n + 1))
    return np.concatenate(parts)


def report(nodes: np.ndarray) -> dict:
    c = np.diff(nodes)
    r = np.maximum(c[1:] / c[:-1], c[:-1] / c[1:]) if c.size > 1 else np.ones(1)
    return {"cells": int(c.size), "min_cell": float(c.min()), "max_cell": float(c.max()), "max_ratio": float(r.max())}
