"""Helpers shared by the tests."""
import hashlib

import numpy as np


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


def cmp_plans(x, y, path="", skip=()):
    """Paths where two plans differ (bit for bit); keys in `skip` are left out."""
    bad = []
    if isinstance(x, dict):
        for k in x:
            if k not in skip:
                bad += cmp_plans(x[k], y[k], f"{path}.{k}")
    elif isinstance(x, list):
        if len(x) != len(y):
            return [path]
        for i, (u, v) in enumerate(zip(x, y)):
            bad += cmp_plans(u, v, f"{path}[{i}]")
    elif isinstance(x, np.ndarray):
        if x.shape != y.shape or not np.array_equal(x, y):
            bad.append(path)
    elif x != y:
        bad.append(path)
    return bad


def rel_l2(a, b) -> float:
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def db_deg(s_test, s_ref):
    """|20 log10 |S| difference| (dB) and phase difference (degrees)."""
    d_db = np.abs(20 * np.log10(np.abs(s_test)) - 20 * np.log10(np.abs(s_ref)))
    d_deg = np.abs(np.angle(s_test / s_ref, deg=True))
    return d_db, d_deg


def mode_source_diff(a: dict, b: dict) -> float:
    """Largest difference of two mode-source tables (global E index -> weight,
    missing entries zero), relative to the largest weight of `a`."""
    wa = dict(zip(a["idx"].tolist(), a["w"].tolist()))
    wb = dict(zip(b["idx"].tolist(), b["w"].tolist()))
    scale = max((abs(v) for v in wa.values()), default=0.0)
    if scale == 0:
        return 0.0 if not wb else float("inf")
    return max(abs(wa.get(k, 0.0) - wb.get(k, 0.0)) for k in set(wa) | set(wb)) / scale
