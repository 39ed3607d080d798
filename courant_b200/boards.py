"""Seeded synthetic printed-circuit boards over the courant.h ABI.

The generator follows the layered board model of the reference's importer
(skyhoffert/CourantEM web/src/import/kicad.ts:51-76: a stackup of dielectric
cores with copper on their faces, traces, vias, planes) and the reference's
board runner (web/src/import/boardsim.ts planBoard :110-209 and buildBoardSim
:211-331): the geometry is drawn in physical coordinates, each axis is meshed
by the rule-based mesher (courant_b200.mesher, a restatement of
web/src/mesh/mesher.ts), CPML cells are added outside, copper is rasterised
edge by edge on its layer planes, vias become solid PEC cells inside their
drill radius, and the port trace runs through feed extensions to 2D
eigenmode (or lumped) ports. The reference builds boards in TypeScript, which
cannot run here, so this is a restatement in Python.

A board has four copper layers on three cores:

- L1 (z = 0): the bottom ground, the PEC z-low face of the domain;
- L2 (top of core 1): a ground plane over the whole board with random
  rectangular clearances;
- L3 (top of core 2): stripline traces;
- L4 (top of core 3): microstrip traces under air;

cores 0.2-1.0 mm thick with eps_r uniform in 3.0-4.5, each a 4-pole
Djordjevic-Sarkar (tan d 0.02 at 1 GHz) Debye fit sharing one set of poles
(the pole frequencies depend only on the band, boardsim.ts :231-233);
traces of width 0.1-0.5 mm running along x with random 45-degree bends
(centres, widths, jogs, clearances and vias on a 50 um routing grid),
through-vias (L1 to L4) placed clear of the traces. Trace 0 (on L4) is the
port trace of ports 1 and 2: it runs straight through both port planes, and
the board ends next to the port planes hold nothing but it and the L2 plane,
so the port cross-sections are uniform. A board of 3 or 4 ports also runs the
trace of the row farthest from trace 0 straight through, on L3, for ports 3
and 4. All randomness comes from numpy's PCG64 seeded with `seed`.

Size: the minimum cell and the board's extent are searched so that the mesh
has about the requested number of cells with the 1500 x 1000 x 64 aspect of
the large synthetic board (z at least 28 cells: four per core, the air above
and the CPML).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import mesher
from .api import Courant

CPML = 1
X, Y, Z = 0, 1, 2


@dataclass
class Layout:
    """Everything random about a board, drawn once per seed; positions as
    fractions of the board, widths and radii in metres."""
    cores: np.ndarray
    eps: np.ndarray
    widths: np.ndarray         # per trace
    rows: np.ndarray           # per trace, fraction of the board's y extent
    runs: list                 # per trace: [(run fraction of the span, jog fraction of the band), ...]
    via_uv: np.ndarray         # candidate via positions (fractions)
    via_r: np.ndarray
    clear: np.ndarray          # clearances: u0, v0, du, dv (fractions)


def draw_layout(seed: int, traces: int, vias: int) -> Layout:
    rng = np.random.Generator(np.random.PCG64(seed))
    cores = rng.uniform(0.2e-3, 1.0e-3, 3)
    eps = rng.uniform(3.0, 4.5, 3)
    widths = rng.uniform(0.1e-3, 0.5e-3, traces)
    rows = (np.arange(traces) + 0.5) / traces
    rows = np.roll(rows, -(traces // 2))         # trace 0 in the middle row
    runs = []
    for _ in range(traces):
        segs, u = [], 0.0
        while u < 1.0:
            r = float(rng.uniform(0.04, 0.15))
            j = float(rng.uniform(-0.8, 0.8))
            segs.append((r, j))
            u += r
        runs.append(segs)
    via_uv = rng.uniform(0.0, 1.0, (4 * vias, 2))
    via_r = rng.uniform(0.1e-3, 0.2e-3, 4 * vias)
    nclr = 6
    clear = np.column_stack([rng.uniform(0.1, 0.85, nclr), rng.uniform(0.05, 0.9, nclr),
                             rng.uniform(0.01, 0.05, nclr), rng.uniform(0.01, 0.05, nclr)])
    return Layout(cores, eps, widths, rows, runs, via_uv, via_r, clear)


@dataclass
class Geometry:
    """A board in physical coordinates (metres)."""
    Lx: float
    Ly: float
    zl: np.ndarray              # L1..L4 heights
    eps: np.ndarray
    traces: list                # (layer 2 or 3, width, [(x, y), ...] polyline)
    vias: list                  # (x, y, r)
    clear: list                 # (x0, x1, y0, y1) holes in the L2 plane
    end: float                  # length at each board end holding only trace 0 and the plane
    feed: float


GRID = 50e-6   # routing grid: trace centres, widths, jogs, clearances and vias snap to it


def _snap(v: float) -> float:
    return round(v / GRID) * GRID


def second_port_trace(lay: Layout) -> int:
    """The trace of ports 3 and 4: the one whose row lies farthest from trace 0's."""
    return int(np.argmax(np.abs(lay.rows - lay.rows[0])))


def realize(lay: Layout, Lx: float, Ly: float, feed: float, nports: int = 2) -> Geometry:
    """The layout on a board of Lx x Ly: trace 0 (and, for 3 or 4 ports, the
    second port trace, listed second) straight through both board ends, the
    others with their jogs."""
    ntr = len(lay.widths)
    t2 = second_port_trace(lay) if nports >= 3 else -1
    band = Ly / ntr
    end = max(0.06 * Lx, 3e-3)
    zl = np.concatenate([[0.0], np.cumsum(lay.cores)])
    traces = []
    for t in range(ntr):
        w = max(GRID * 2, _snap(float(lay.widths[t])))
        y0 = _snap(float(lay.rows[t]) * Ly)
        layer = 3 if t % 2 == 0 else 2
        if t == 0 or t == t2:
            layer = 3 if t == 0 else 2                      # the second port trace is a stripline on L3
            traces.insert(min(t, 1), (layer, w, [(-feed - 1.0, y0), (Lx + feed + 1.0, y0)]))
            continue
        xa, xb = end + 1e-3, Lx - end - 1e-3
        if xb <= xa:
            continue
        lo, hi = y0 - 0.35 * band + w / 2, y0 + 0.35 * band - w / 2
        pts = [(xa, y0)]
        x, y = xa, y0
        for r, jf in lay.runs[t]:
            x = min(_snap(x + r * (xb - xa)), xb)
            pts.append((x, y))
            if x >= xb:
                break
            dy = _snap(float(np.clip(y + jf * 0.35 * band, lo, hi)) - y)
            if abs(dy) > 1e-9 and x + abs(dy) < xb:
                x, y = x + abs(dy), y + dy                  # a 45-degree jog
                pts.append((x, y))
        if pts[-1][0] < xb:
            pts.append((xb, y))
        traces.append((layer, w, pts))
    clear = [(_snap(u0 * Lx), _snap((u0 + du) * Lx), _snap(v0 * Ly), _snap((v0 + dv) * Ly))
             for u0, v0, du, dv in lay.clear if u0 * Lx > end and (u0 + du) * Lx < Lx - end]
    geo = Geometry(Lx, Ly, zl, lay.eps, traces, [], clear, end, feed)
    return geo


def place_vias(geo: Geometry, lay: Layout, count: int) -> None:
    """The first `count` candidate positions that keep a via clear of every
    trace (0.2 mm) and of the board ends."""
    # every trace segment as (x0, y0, x1, y1, half width)
    seg = np.array([(x0, y0, x1, y1, w / 2) for _, w, pts in geo.traces
                    for (x0, y0), (x1, y1) in zip(pts[:-1], pts[1:])], dtype=np.float64).reshape(-1, 5)
    out = []
    for (u, v), r in zip(lay.via_uv, lay.via_r):
        if len(out) >= count:
            break
        x, y = _snap(geo.end + u * (geo.Lx - 2 * geo.end)), _snap(0.03 * geo.Ly + v * 0.94 * geo.Ly)
        if seg.size:
            dx, dy = seg[:, 2] - seg[:, 0], seg[:, 3] - seg[:, 1]
            L2 = dx * dx + dy * dy
            t = np.clip(np.where(L2 > 0, ((x - seg[:, 0]) * dx + (y - seg[:, 1]) * dy) / np.where(L2 > 0, L2, 1), 0),
                        0.0, 1.0)
            d = np.hypot(x - seg[:, 0] - t * dx, y - seg[:, 1] - t * dy)
            if np.any(d <= seg[:, 4] + r + 0.2e-3):
                continue
        if all(math.hypot(x - a, y - b) > r + q + 0.3e-3 for a, b, q in out):
            out.append((float(x), float(y), float(r)))
    geo.vias = out


def _dist_polyline(x, y, pts) -> float:
    best = math.inf
    for (x0, y0), (x1, y1) in zip(pts[:-1], pts[1:]):
        dx, dy = x1 - x0, y1 - y0
        L2 = dx * dx + dy * dy
        t = 0.0 if L2 == 0 else min(1.0, max(0.0, ((x - x0) * dx + (y - y0) * dy) / L2))
        best = min(best, math.hypot(x - x0 - t * dx, y - y0 - t * dy))
    return best


# ------------------------------------------------------------------ meshing

def axis_features(geo: Geometry, fmax: float, hmin: float):
    """The mesher inputs of the three axes (boardsim.ts planBoard :154-188)."""
    er_max = float(max(geo.eps))
    h_air = min(mesher.lambda_over_20(fmax, 1.0), 200e-6)
    h_diel = mesher.lambda_over_20(fmax, er_max)
    side = 1e-3
    # y: trace edges of the x-directed runs, clearance edges, vias
    yedges = set()
    xedges = set()
    for _, w, pts in geo.traces:
        for (x0, y0), (x1, y1) in zip(pts[:-1], pts[1:]):
            if abs(y1 - y0) < 1e-12:
                yedges.add((round(y0 - w / 2, 9), "hi"))
                yedges.add((round(y0 + w / 2, 9), "lo"))
        xs = pts[0][0], pts[-1][0]
        if 0 < xs[0] < geo.Lx:
            xedges.add((round(xs[0], 9), "hi"))
        if 0 < xs[1] < geo.Lx:
            xedges.add((round(xs[1], 9), "lo"))
    for x0, x1, y0, y1 in geo.clear:
        yedges |= {(round(y0, 9), "lo"), (round(y1, 9), "hi")}
        xedges |= {(round(x0, 9), "lo"), (round(x1, 9), "hi")}
    via_r = min((r for _, _, r in geo.vias), default=0.0)
    h_via = max(hmin, via_r / 2) if via_r else math.inf
    fy = mesher.AxisFeatures(lo=-side, hi=geo.Ly + side, sheet_edges=sorted(yedges), planes=[0.0, geo.Ly],
                             refine=[e for e, _ in yedges] + [y for _, y, _ in geo.vias],
                             max_cell=[(0.0, geo.Ly, h_diel)] + [(y - r, y + r, h_via) for _, y, r in geo.vias])
    X0, X1 = -geo.feed, geo.Lx + geo.feed
    fx = mesher.AxisFeatures(lo=X0, hi=X1, sheet_edges=sorted(xedges), planes=[0.0, geo.Lx],
                             refine=[e for e, _ in xedges] + [x for x, _, _ in geo.vias],
                             max_cell=[(X0, X1, min(h_diel, 4 * hmin))] + [(x - r, x + r, h_via) for x, _, r in geo.vias])
    ztop = float(geo.zl[-1])
    fz = mesher.AxisFeatures(lo=0.0, hi=ztop + 1.5e-3, planes=[float(v) for v in geo.zl],
                             spans=[(float(geo.zl[q]), float(geo.zl[q + 1]), 4) for q in range(3)],
                             max_cell=[(float(geo.zl[q]), float(geo.zl[q + 1]), h_diel) for q in range(3)],
                             refine=[float(v) for v in geo.zl])
    return fx, fy, fz, h_air


def _mesh_z(geo, fmax, hmin, npml):
    _, _, fz, h_air = axis_features(geo, fmax, hmin)
    return mesher.with_pml(mesher.mesh_axis(fz, hmin, h_air), npml, h_air / 2, lo=False, hi=True)


def _search(f, lo, hi, target, increasing, iters=10):
    """Argument in [lo, hi] for which the monotone integer-valued f comes
    closest to `target`: secant steps on log(arg) with the bracket kept, then
    the best of those tried."""
    import math as _m
    tried = {}

    def ev(v):
        if v not in tried:
            tried[v] = f(v)
        return tried[v]
    a, b = lo, hi
    fa, fb = ev(a), ev(b)
    x = _m.sqrt(a * b)
    for _ in range(iters):
        fx = ev(x)
        if fx == target:
            break
        if (fx < target) == increasing:
            a, fa = x, fx
        else:
            b, fb = x, fx
        # secant on log(argument) against the value, inside the bracket
        la, lb = _m.log(a), _m.log(b)
        if fb != fa:
            t = (target - fa) / (fb - fa)
            nx_ = _m.exp(la + min(max(t, 0.05), 0.95) * (lb - la))
        else:
            nx_ = _m.sqrt(a * b)
        if abs(_m.log(nx_ / x)) < 1e-9:
            break
        x = nx_
    return min(tried, key=lambda v: (abs(tried[v] - target), v))


def plan_mesh(lay: Layout, cells: float, fmax: float, npml: int, vias: int, feed: float,
              target: tuple | None = None, nports: int = 2):
    """Minimum cell, board extent and node lines for about `cells` cells:
    hmin sets nz, then Ly sets ny and Lx sets nx (aspect 1.5 : 1)."""
    if target is None:
        nz_t = int(np.clip(round(64 * (cells / 96e6) ** (1 / 3)), 28, 64))
        ny_t = math.sqrt(cells / nz_t / 1.5)
        target = (1.5 * ny_t, ny_t, nz_t)
    nx_t, ny_t, nz_t = target
    probe = realize(lay, 0.1, 0.07, feed, nports)
    h_air = min(mesher.lambda_over_20(fmax, 1.0), 200e-6)
    hmin = _search(lambda h: len(_mesh_z(probe, fmax, h, npml)) - 1, 5e-6, h_air, nz_t, increasing=False, iters=14)

    def ny_of(Ly):
        geo = realize(lay, 1.5 * Ly, Ly, feed, nports)
        place_vias(geo, lay, vias)
        _, fy, _, h_air = axis_features(geo, fmax, hmin)
        return len(mesher.mesh_axis(fy, hmin, h_air)) - 1 + 2 * npml

    Ly = _search(ny_of, 2e-3, 2.0, ny_t, increasing=True)

    def nx_of(Lx):
        geo = realize(lay, Lx, Ly, feed, nports)
        place_vias(geo, lay, vias)
        fx, _, _, h_air = axis_features(geo, fmax, hmin)
        return len(mesher.mesh_axis(fx, hmin, h_air)) - 1 + 2 * npml

    Lx = _search(nx_of, 3e-3, 3.0, nx_t, increasing=True)
    geo = realize(lay, Lx, Ly, feed, nports)
    place_vias(geo, lay, vias)
    fx, fy, fz, h_air = axis_features(geo, fmax, hmin)
    hp = h_air / 2
    x = mesher.with_pml(mesher.mesh_axis(fx, hmin, h_air), npml, hp)
    y = mesher.with_pml(mesher.mesh_axis(fy, hmin, h_air), npml, hp)
    z = mesher.with_pml(mesher.mesh_axis(fz, hmin, h_air), npml, hp, lo=False, hi=True)
    return geo, hmin, x, y, z


# ------------------------------------------------------------------ rasterising

def _capsule_marks(mask, xs, ys, x0, y0, x1, y1, r):
    """Mark the points of the grid xs (rows) x ys (columns) within r of segment (x0, y0)-(x1, y1)."""
    i0, i1 = np.searchsorted(xs, min(x0, x1) - r, "left"), np.searchsorted(xs, max(x0, x1) + r, "right")
    j0, j1 = np.searchsorted(ys, min(y0, y1) - r, "left"), np.searchsorted(ys, max(y0, y1) + r, "right")
    if i1 <= i0 or j1 <= j0:
        return
    X, Yv = np.meshgrid(xs[i0:i1], ys[j0:j1], indexing="ij")
    dx, dy = x1 - x0, y1 - y0
    L2 = dx * dx + dy * dy
    t = np.zeros_like(X) if L2 == 0 else np.clip(((X - x0) * dx + (Yv - y0) * dy) / L2, 0.0, 1.0)
    d2 = (X - x0 - t * dx) ** 2 + (Yv - y0 - t * dy) ** 2
    mask[i0:i1, j0:j1] |= d2 <= r * r * (1 + 1e-12)


def _trace_masks(x, y, traces):
    """Edge masks of a z-normal plane (cem_pec_edges_plane layout: u = x edges
    nx x (ny+1), v = y edges (nx+1) x ny): an edge is copper when both its
    nodes and its midpoint are (boardsim.ts :253-265)."""
    xm, ym = 0.5 * (x[1:] + x[:-1]), 0.5 * (y[1:] + y[:-1])
    node = np.zeros((len(x), len(y)), bool)
    midx = np.zeros((len(xm), len(y)), bool)
    midy = np.zeros((len(x), len(ym)), bool)
    for w, pts in traces:
        for (x0, y0), (x1, y1) in zip(pts[:-1], pts[1:]):
            for m, xs, ys in ((node, x, y), (midx, xm, y), (midy, x, ym)):
                _capsule_marks(m, xs, ys, x0, y0, x1, y1, w / 2)
    mu = node[:-1, :] & node[1:, :] & midx
    mv = node[:, :-1] & node[:, 1:] & midy
    return mu, mv


def _plane_masks(x, y, holes):
    """Edge masks of a full plane with rectangular holes (open rectangles)."""
    def inside(X, Yv):
        m = np.zeros(X.shape, bool)
        for x0, x1, y0, y1 in holes:
            m |= (X > x0) & (X < x1) & (Yv > y0) & (Yv < y1)
        return ~m
    xm, ym = 0.5 * (x[1:] + x[:-1]), 0.5 * (y[1:] + y[:-1])
    node = inside(*np.meshgrid(x, y, indexing="ij"))
    mu = node[:-1, :] & node[1:, :] & inside(*np.meshgrid(xm, y, indexing="ij"))
    mv = node[:, :-1] & node[:, 1:] & inside(*np.meshgrid(x, ym, indexing="ij"))
    return mu, mv


def _nearest(a, v):
    return int(np.argmin(np.abs(np.asarray(a) - v)))


def hammerstad_neff(w: float, h: float, er: float) -> float:
    """Quasi-static effective index of a microstrip (Hammerstad), the shift of the port mode solve."""
    u = w / h
    e = (er + 1) / 2 + (er - 1) / 2 * (1 + 12 / u) ** -0.5
    if u < 1:
        e += (er - 1) / 2 * 0.04 * (1 - u) ** 2
    return math.sqrt(e)


def covered_neff(w: float, h: float, er: float, d: float, er_cover: float) -> float:
    """Estimated effective index of a microstrip under a dielectric cover of
    thickness d (air above it), the shift of its mode solve: Hammerstad's
    filling factor q = (e_ms - 1) / (er - 1) splits the field between the
    substrate and the half-space above; under an infinite cover that half-space
    holds er_cover, and the air share of a finite cover decays as exp(-2 d / h)."""
    e_ms = hammerstad_neff(w, h, er) ** 2
    q = (e_ms - 1) / (er - 1)
    e_full = q * er + (1 - q) * er_cover
    return math.sqrt(e_full - (e_full - e_ms) * math.exp(-2 * d / h))


@dataclass
class BoardPlan:
    """Everything of a seeded board that needs no solver library: node lines,
    stackup, copper edge masks per layer, via cells, port placement. It is
    plain numpy data, so a process pool can make it (the server's planners)
    and any thread turn it into a simulation with board_sim()."""
    seed: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    zl: np.ndarray
    eps: np.ndarray
    kl: list
    layers: list          # (k plane, mask_u, mask_v)
    via_cells: list       # (i0, j0, mask over cells i, j; L1 to L4)
    ports: str
    port: list            # per port: mode-port definition without dir/iSrc/iMon/xRef, or lumped placement;
                          # "end" 0 (x-low) or 1 (x-high)
    Lx: float
    meta: dict
    npml: int
    nf: int
    fmax: float
    steps: int | None
    cfl: float
    excite: int


def plan_board(seed: int, cells: float = 2e6, *, ports: str = "mode", nf: int = 32, fmax: float = 20e9,
               steps: int | None = None, traces: int = 20, vias: int = 30, npml: int = 8, cfl: float = 0.99,
               excite: int = 1, target: tuple | None = None, nports: int = 2) -> BoardPlan:
    """The library-free part of seeded_board (its arguments, less the library)."""
    if not 1 <= nports <= 4 or not 1 <= excite <= nports:
        raise ValueError(f"a board has 1 to 4 ports and drives one of them (nports {nports}, excite {excite})")
    ntr = max(3, min(traces, int(round((cells / 2e4) ** 0.5))))
    nvia = max(2, min(vias, int(cells / 1e5)))
    lay = draw_layout(seed, ntr, 4 * nvia)
    feed = 4e-3 if ports == "mode" else 0.0
    geo, hmin, x, y, z = plan_mesh(lay, cells, fmax, npml, nvia, feed, target, nports)
    nx, ny, nz = len(x) - 1, len(y) - 1, len(z) - 1
    zl = geo.zl
    kl = [_nearest(z, v) for v in zl]
    # L2 plane with clearances, then the trace layers (the bottom copper is the PEC floor)
    layers = [(kl[1], *_plane_masks(x, y, geo.clear))]
    for layer in (2, 3):
        sel = [(w, pts) for ly, w, pts in geo.traces if ly == layer]
        if sel:
            layers.append((kl[layer], *_trace_masks(x, y, sel)))
    # via barrels: solid PEC cells inside the drill radius, L1 to L4 (boardsim.ts :281-297)
    via_cells = []
    for vx, vy, r in geo.vias:
        i0, i1 = max(0, _nearest(x, vx - r) - 1), min(nx - 1, _nearest(x, vx + r) + 1)
        j0, j1 = max(0, _nearest(y, vy - r) - 1), min(ny - 1, _nearest(y, vy + r) + 1)
        cx = 0.5 * (x[i0:i1 + 1] + x[i0 + 1:i1 + 2])
        cy = 0.5 * (y[j0:j1 + 1] + y[j0 + 1:j1 + 2])
        inside = (cx[:, None] - vx) ** 2 + (cy[None, :] - vy) ** 2 <= r * r
        if inside.any() and kl[3] > 0:
            via_cells.append((i0, j0, inside))
    # ports: 1 and 2 at the x-low and x-high ends of trace 0 (L4), 3 and 4 at those of the
    # second port trace (L3). The two traces are the only copper of the port planes but the
    # L2 plane. A section holding both has two quasi-TEM modes: trace 0's ports keep the
    # whole section (their shift lies near trace 0's mode, the lower index of the two), and
    # the second trace's cross-section stops at a wall between the traces, one trace-0
    # height beyond trace 0's strip edge (the midpoint at most), so that its solve sees
    # one line.
    ysplit = None
    if nports >= 3:
        (_, w0, p0), (_, _, p1) = geo.traces[0], geo.traces[1]
        y0, y1 = p0[0][1], p1[0][1]
        ysplit = y0 + math.copysign(min(w0 / 2 + float(zl[3] - zl[1]), abs(y1 - y0) / 2), y1 - y0)
    port = []
    for q in range(nports):
        layer, w, pts = geo.traces[q // 2]
        yc, kh = pts[0][1], kl[layer]
        if ports == "mode":
            jl, jr = _nearest(y, yc - w / 2), _nearest(y, yc + w / 2)
            ja = max(0, (jl if y[jl] <= yc - w / 2 else jl - 1) - 1)
            jb = min(ny - 1, jr if y[jr] >= yc + w / 2 else jr + 1)
            j0, j1 = 0, ny
            if q >= 2:
                js = _nearest(y, ysplit)
                j0, j1 = (js, ny) if yc > ysplit else (0, js)
            if layer == 3:      # microstrip over cores 1 and 2
                er = float(np.average(geo.eps[1:3], weights=np.diff(zl)[1:3]))
                neff0 = hammerstad_neff(w, float(zl[3] - zl[1]), er)
            else:               # core 1 below, core 2 over it, air above
                neff0 = covered_neff(w, float(zl[2] - zl[1]), float(geo.eps[1]), float(zl[3] - zl[2]),
                                     float(geo.eps[2]))
            port.append(dict(j0=j0, j1=j1, k0=0, k1=nz, vj=_nearest(y, yc), vk0=kl[1], vk1=kh, vsign=-1, ja=ja,
                             jb=jb, ka=kh - 1, kb=kh, f0=0.5 * fmax, neff0=neff0, end=q % 2))
        else:
            port.append(dict(j=_nearest(y, yc), k0=kl[1], k1=kh, end=q % 2))
    meta = {"seed": seed, "dims": (nx, ny, nz), "cells": nx * ny * nz, "excite": excite, "hmin": hmin,
            "nports": nports,
            "board_mm": (geo.Lx * 1e3, geo.Ly * 1e3), "traces": len(geo.traces), "vias": len(geo.vias),
            "mesh": {a: mesher.report(v) for a, v in (("x", x), ("y", y), ("z", z))}}
    return BoardPlan(seed, x, y, z, zl, np.asarray(geo.eps), kl, layers, via_cells, ports, port, geo.Lx, meta, npml,
                     nf, fmax, steps, cfl, excite)


def board_sim(c: Courant, b: BoardPlan):
    """The finalized simulation of a board plan on library `c`, and its metadata."""
    x, y, z = b.x, b.y, b.z
    nx = len(x) - 1
    s = c.createSim(x, y, z)
    for f in (0, 1, 2, 3, 5):
        s.setBoundary(f, CPML, b.npml)
    fits = [c.fitDjordjevicSarkar(float(e), 0.02, 1e9, 1e8, b.fmax, 4) for e in b.eps]
    s.setDebyePoles(fits[0].fp)
    big = 1.0
    for q in range(3):
        s.materialBoxDebye(-big, big, -big, big, float(b.zl[q]), float(b.zl[q + 1]), fits[q])
    for k, mu, mv in b.layers:
        s.pecEdgesPlane(Z, k, mu, mv)
    for i0, j0, inside in b.via_cells:
        s.pecCells(i0, j0, 0, np.repeat(inside[:, :, None], b.kl[3], axis=2).astype(np.uint8))
    tau = math.sqrt(6.9) / (math.pi * 1.25 * b.fmax)
    freqs = np.linspace(b.fmax / b.nf, b.fmax, b.nf)
    meta = dict(b.meta, tau=tau, freqs=freqs)
    ids = []
    if b.ports == "mode":
        mon = 2.5e-3
        i1, i2 = b.npml + 2, nx - b.npml - 2
        for pt in b.port:
            d = {k: v for k, v in pt.items() if k != "end"}
            if pt["end"] == 0:
                ids.append(s.addModePort(dict(d, dir=1, iSrc=i1, iMon=_nearest(x, x[i1] + mon), xRef=0.0)))
            else:
                ids.append(s.addModePort(dict(d, dir=-1, iSrc=i2, iMon=_nearest(x, x[i2] - mon) - 1, xRef=b.Lx)))
        s.setModeExcitation(ids[b.excite - 1], 4.5 * tau, tau)
        meta["modeports"] = ids
    else:
        for pt in b.port:      # the L2 ground to the trace
            i = b.npml + 4 if pt["end"] == 0 else nx - b.npml - 4
            ids.append(s.addLumpedPort(Z, i, pt["j"], pt["k0"], pt["k1"], -1, 50.0))
        s.setGaussian(ids[b.excite - 1], 1.0, 4.5 * tau, tau)
        meta["ports"] = ids
    s.setFrequencies(freqs)
    s.finalize(b.cfl)
    meta["steps"] = int(b.steps if b.steps is not None else min(40000, max(4000, int(12 * tau / s.dt) * 10)))
    return s, meta


def seeded_board(c: Courant, seed: int, cells: float = 2e6, *, ports: str = "mode", nf: int = 32,
                 fmax: float = 20e9, steps: int | None = None, traces: int = 20, vias: int = 30,
                 npml: int = 8, cfl: float = 0.99, excite: int = 1, target: tuple | None = None,
                 nports: int = 2):
    """Finalized board simulation and its metadata (dims, cells, ports,
    frequencies, step count, mesh report). `cells` sets the grid size (or
    `target` = (nx, ny, nz) directly); `traces` and `vias` scale down for
    small boards so features keep a few cells between them; `nports` (1 to
    4) ports, 1 and 2 at the x-low and x-high ends of trace 0 (L4), 3 and 4
    at those of trace 1 (L3); `excite` picks the driven port, one column of
    the S-matrix per excitation."""
    return board_sim(c, plan_board(seed, cells, ports=ports, nf=nf, fmax=fmax, steps=steps, traces=traces, vias=vias,
                                 npml=npml, cfl=cfl, excite=excite, target=target, nports=nports))


class SeededBoard:
    """A seeded board request in two parts: `plan()` (no library, picklable,
    for a process pool) and `realize(lib, plan)` (board_sim); calling it with
    a library does both."""

    def __init__(self, seed: int, cells: float = 2e6, **kw):
        self.seed, self.cells, self.kw = seed, cells, kw

    def plan(self) -> BoardPlan:
        return plan_board(self.seed, self.cells, **self.kw)

    @staticmethod
    def realize(c: Courant, plan: BoardPlan):
        return board_sim(c, plan)

    def __call__(self, c: Courant):
        return board_sim(c, self.plan())
