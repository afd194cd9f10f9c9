"""Frequency-map pieces that need no GPU: the .fm table writer (the reference's '(12a14)' header
and '(12e14.5)' rows, '*' for particles out of the RF bucket, no row for lost ones), calc_tune's
interpolation on a pure tone, and the eigenvector ordering behind the normalisation."""
import importlib
import math

import numpy as np
import pytest

import fma_reference as F

lib = importlib.import_module("bmad-ecosystem_b200.lib")


def test_fm_table_format(tmp_path):
    off = np.array([[1.5e-3, 0, -2e-4, 0, 0, 0.01], [0.02, 0, 0, 0, 0, 0], [1e-3, 0, 1e-3, 0, 0, -0.003]])
    tunes = np.array([[0.2226313, 0.0966893, 0.95929, 0.2226320, 0.0966890, 0.959291], [0] * 6, [0] * 6])
    path = str(tmp_path / "t.fm")
    lib.fma_write(path, off, tunes, [0, 1, 2])
    lines = open(path).read().splitlines()
    assert lines[0] == "".join("%14s" % h for h in ("# x", "y", "pz", "Qx0", "Qy0", "Qz0", "Qx1", "Qy1", "Qz1",
                                                   "dQx", "dQy", "dQz"))
    assert len(lines) == 3
    row = lines[1]
    assert len(row) == 12 * 14
    cols = [row[14 * k:14 * (k + 1)] for k in range(12)]
    assert cols[0] == "   0.15000E-02"
    assert cols[1] == "  -0.20000E-03"
    assert cols[2] == "   0.10000E-01"
    assert cols[3] == "   0.22263E+00"
    assert cols[9] == "   0.70000E-06"
    assert lines[2][:42] == "   0.10000E-02   0.10000E-02  -0.30000E-02"
    assert lines[2][42:] == "%14s" % "*" * 9


def test_calc_tune_pure_tone():
    N = 256
    for q in (0.1234, 0.31, 0.777):
        j = np.arange(1, N + 1)
        sig = np.exp(2j * np.pi * q * np.arange(N)) * 2 * np.sin(np.pi * j / N) ** 2
        spec = np.abs(np.fft.ifft(sig) * N)
        # the backward transform puts exp(+2 pi i q j) at 1 - q, and the reference reads bin k as
        # (k + 1) / N: one bin above
        assert F.calc_tune(spec) == pytest.approx((1 - q) + 1.0 / N, abs=1e-6)


def test_mat_eigen_ordering():
    def rot(mu, beta, alpha):
        g = (1 + alpha ** 2) / beta
        return np.array([[math.cos(mu) + alpha * math.sin(mu), beta * math.sin(mu)],
                         [-g * math.sin(mu), math.cos(mu) - alpha * math.sin(mu)]])
    M = np.zeros((6, 6))
    mus = (2 * math.pi * 0.31, 2 * math.pi * 0.17, 2 * math.pi * 0.02)
    M[4:, 4:] = rot(mus[2], 2.0, 0.0)
    M[:2, :2] = rot(mus[0], 8.0, -0.4)
    M[2:4, 2:4] = rot(mus[1], 3.0, 0.6)
    vals, vecs = lib.mat_eigen(M)
    for plane in range(3):
        assert abs(np.angle(vals[2 * plane])) == pytest.approx(mus[plane], abs=1e-12)
        e = vecs[2 * plane]
        # the odd member of each pair has positive symplectic norm and lives in its plane
        assert sum(2 * np.imag(np.conj(e[k]) * e[k + 1]) for k in range(0, 6, 2)) > 0
        assert np.sum(np.abs(e[2 * plane:2 * plane + 2]) ** 2) > 0.99 * np.sum(np.abs(e) ** 2)
    norm = lib.fma_normalization(M)
    assert norm.shape == (6, 6)
