"""Touchstone 2-port files (courant_b200/touchstone.py): the reference app's
RI export format, reading all v1 formats, renormalisation, and the S21 gate."""
import numpy as np
import pytest

from courant_b200 import touchstone


def line(n=41, loss_db=0.5, delay=80e-12):
    f = np.linspace(1e9, 40e9, n)
    s21 = 10 ** (-loss_db * f / 40e9 / 20) * np.exp(-2j * np.pi * f * delay)
    s11 = 0.05 * np.exp(-1j * np.pi * f / 20e9)
    return f, s11, s21


def test_write_read_round_trip():
    f, s11, s21 = line()
    text = touchstone.write_s2p(None, f, s11, s21, title="t")
    assert "# HZ S RI R 50" in text and "S22 = S11 and S12 = S21 assumed" in text
    g, S, R = touchstone.read_s2p(text)
    assert R == 50.0 and np.allclose(g, f, rtol=1e-6)
    assert np.allclose(S[:, 1, 0], s21, rtol=1e-8, atol=1e-12) and np.allclose(S[:, 0, 1], s21, rtol=1e-8, atol=1e-12)
    assert np.allclose(S[:, 0, 0], s11, rtol=1e-8, atol=1e-12) and np.allclose(S[:, 1, 1], s11, rtol=1e-8, atol=1e-12)


def test_reads_ma_and_db_in_ghz():
    f, s11, s21 = line(5)
    rows = []
    for q in range(5):
        vals = [s11[q], s21[q], s21[q], s11[q]]
        rows.append(" ".join([f"{f[q] / 1e9:.9f}"] + [f"{20 * np.log10(abs(v)):.12f} {np.degrees(np.angle(v)):.12f}" for v in vals]))
    g, S, R = touchstone.read_s2p("# GHz S DB R 50\n" + "\n".join(rows) + "\n")
    assert np.allclose(g, f) and np.allclose(S[:, 1, 0], s21, rtol=1e-9)


def test_renormalise_round_trip():
    f, s11, s21 = line(7)
    S = np.empty((7, 2, 2), complex)
    S[:, 0, 0], S[:, 1, 0], S[:, 0, 1], S[:, 1, 1] = s11, s21, s21, s11
    back = touchstone.renormalise(touchstone.renormalise(S, 50.0, 75.0), 75.0, 50.0)
    assert np.allclose(back, S, atol=1e-12)
    assert touchstone.renormalise(S, 50.0) is S


def test_gate_passes_identical_and_catches_offsets():
    f, s11, s21 = line()
    a = touchstone.read_s2p(touchstone.write_s2p(None, f, s11, s21))
    assert touchstone.compare(a, a)["ok"]
    off = touchstone.read_s2p(touchstone.write_s2p(None, f, s11, s21 * 10 ** (0.002 / 20)))   # +0.002 dB
    c = touchstone.compare(a, off, "b200")
    assert not c["ok"] and c["s21_db"] == pytest.approx(0.002, rel=1e-3)
    assert touchstone.compare(a, off, "gpu")["ok"]
    rot = touchstone.read_s2p(touchstone.write_s2p(None, f, s11, s21 * np.exp(1j * np.radians(0.05))))
    assert not touchstone.compare(a, rot, "b200")["ok"]
