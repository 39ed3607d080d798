"""Touchstone 2-port files and their comparison.

`write_s2p` writes what the reference's app exports (skyhoffert/CourantEM
web/src/app/touchstone.ts:1-28): RI format, frequencies in Hz, a 50-ohm
reference line, the 2-port order S11 S21 S12 S22, and, when only port 1 was
excited, S22 = S11 and S12 = S21 with a header comment saying so.

`read_s2p` reads any Touchstone v1 2-port file (RI, MA or DB; Hz to GHz; any
reference resistance) and `compare` checks two results against a gate, in the
manner of the reference's tools/compare_s2p.py:1-120 (|S21| in dB and phase
in degrees on the first file's frequencies inside the overlap, the second
file interpolated in dB and unwrapped phase, both renormalised to 50 ohm).
"""
from __future__ import annotations

import io
import math
from pathlib import Path

import numpy as np

UNITS = {"hz": 1.0, "khz": 1e3, "mhz": 1e6, "ghz": 1e9}

# |S21| dB, S21 phase degrees, and the band they apply to
GATES = {
    "b200": {"s21_db": 1e-3, "s21_deg": 0.01, "fmin": 1e9},      # the FP32 engine against the f64 core
    "gpu": {"s21_db": 0.01, "s21_deg": 0.1, "fmin": 0.0},        # the reference's own GPU-vs-CPU rule
}


def write_s2p(dest, f, s11, s21, s12=None, s22=None, title: str = "", version: str = "20261017.0-b200") -> str:
    """Write a 2-port in RI format with a 50-ohm reference; returns the text.
    `dest`: a path, a writable text stream, or None."""
    full = s12 is not None and s22 is not None
    s12 = s21 if s12 is None else s12
    s22 = s11 if s22 is None else s22
    lines = [f"! courant-b200 {version} — {title}",
             "! reference 50; " + ("both ports excited" if full else "port 1 excited, S22 = S11 and S12 = S21 assumed"),
             "# HZ S RI R 50"]
    for q, fq in enumerate(np.asarray(f, dtype=float)):
        vals = [s11[q], s21[q], s12[q], s22[q]]
        lines.append(" ".join([f"{fq:.6e}"] + [f"{v:.9e}" for z in vals for v in (z.real, z.imag)]))
    text = "\n".join(lines) + "\n"
    if isinstance(dest, (str, Path)):
        Path(dest).write_text(text)
    elif dest is not None:
        dest.write(text)
    return text


def read_s2p(src):
    """f (Hz), S (n, 2, 2) complex and the reference resistance of a 2-port
    file; `src` a path or the file's text."""
    text = Path(src).read_text() if isinstance(src, Path) or (isinstance(src, str) and "\n" not in src) else src
    unit, fmt, R = 1e9, "ma", 50.0
    vals = []
    for line in io.StringIO(text):
        line = line.split("!", 1)[0].strip()
        if not line:
            continue
        if line.startswith("#"):
            tok = line[1:].lower().split()
            for q, t in enumerate(tok):
                if t in UNITS:
                    unit = UNITS[t]
                elif t in ("ri", "ma", "db"):
                    fmt = t
                elif t == "r" and q + 1 < len(tok):
                    R = float(tok[q + 1])
            continue
        vals.extend(float(v) for v in line.split())
    d = np.array(vals).reshape(-1, 9)
    f = d[:, 0] * unit
    p = d[:, 1:].reshape(-1, 4, 2)
    if fmt == "ri":
        z = p[..., 0] + 1j * p[..., 1]
    else:
        mag = 10 ** (p[..., 0] / 20) if fmt == "db" else p[..., 0]
        z = mag * np.exp(1j * np.radians(p[..., 1]))
    S = np.empty((len(f), 2, 2), complex)
    S[:, 0, 0], S[:, 1, 0], S[:, 0, 1], S[:, 1, 1] = z[:, 0], z[:, 1], z[:, 2], z[:, 3]
    return f, S, R


def renormalise(S, R: float, R0: float = 50.0):
    """S-parameters referred to R, re-referred to R0 (through Z)."""
    if abs(R - R0) < 1e-12:
        return S
    eye = np.eye(2)
    out = np.empty_like(S)
    for q in range(len(S)):
        Z = R * (eye + S[q]) @ np.linalg.inv(eye - S[q])
        out[q] = (Z - R0 * eye) @ np.linalg.inv(Z + R0 * eye)
    return out


def _db(x):
    return 20 * np.log10(np.maximum(np.abs(x), 1e-300))


def compare(a, b, gate: str = "b200") -> dict:
    """Largest |S21| (dB) and phase (degrees) differences of b against a on
    a's frequencies inside both bands (and above the gate's lowest frequency),
    b interpolated; `ok` when both are within the gate. a, b: (f, S, R) as
    read_s2p returns, or file paths / texts."""
    fa, Sa, Ra = read_s2p(a) if not isinstance(a, tuple) else a
    fb, Sb, Rb = read_s2p(b) if not isinstance(b, tuple) else b
    Sa, Sb = renormalise(Sa, Ra), renormalise(Sb, Rb)
    g = GATES[gate]
    sel = (fa >= max(fb.min(), g["fmin"])) & (fa <= fb.max())
    f = fa[sel]
    a21 = Sa[sel, 1, 0]
    b21 = Sb[:, 1, 0]
    bdb = np.interp(f, fb, _db(b21))
    bph = np.interp(f, fb, np.unwrap(np.angle(b21)))
    ddb = np.abs(_db(a21) - bdb)
    dph = np.abs(np.degrees(np.angle(np.exp(1j * (np.angle(a21) - bph)))))
    out = {"points": int(len(f)), "s21_db": float(ddb.max()) if len(f) else math.nan,
           "s21_deg": float(dph.max()) if len(f) else math.nan}
    out["ok"] = bool(len(f) and out["s21_db"] <= g["s21_db"] and out["s21_deg"] <= g["s21_deg"])
    return out
