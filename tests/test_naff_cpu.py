"""The NAFF restatement (test infrastructure) against the reference's own known-answer test:
regression_tests/sim_utils_test (three tones, 32 samples), expected frequencies and amplitudes
from its output.correct with its REL tolerances (fixture tests/golden/naff_kat.json, made by
tests/golden/make_naff_kat.py)."""
import json
import os

import numpy as np

import naff_reference as NR

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "naff_kat.json")))


def kat_signal():
    d = np.array(KAT["cdata"])
    return d[:, 0] + 1j * d[:, 1]


def check_kat(freqs, amps):
    for e in KAT["expected"]:
        k = e["k"] - 1
        got = (freqs[k], amps[k].real, amps[k].imag)
        want = (e["freq"], e["amp"][0], e["amp"][1])
        for g, w in zip(got, want):
            assert abs(g - w) <= e["rel"] * abs(w), (e["k"], got, want)


def test_restatement_matches_reference_kat():
    f, a = NR.naff(kat_signal(), 3)
    check_kat(f, a)


def test_restatement_pure_tones():
    n = 512
    t = np.arange(n)
    tones = [(0.5 - 0.2j, 0.3141), (0.05 + 0.01j, 0.7182), (0.002j, 0.1234)]
    sig = sum(a * np.exp(-2j * np.pi * f * t) for a, f in tones)
    freqs, amps = NR.naff(sig, 3)
    for (a, f), gf, ga in zip(tones, freqs, amps):
        assert abs(gf - f) < 1e-8
        assert abs(ga - a) < 1e-4 * abs(a) + 1e-7  # the phase error 2 pi N df of the 1e-8 stop


def test_constant_signal():
    f, a = NR.naff(np.full(64, 1.0 + 2.0j), 2)
    assert np.all(f == 0) and np.all(a == 0)
