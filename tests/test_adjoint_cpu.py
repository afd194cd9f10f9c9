"""The hand-written adjoint (csrc/adjoint.cuh) compiled for the host (test-only build,
csrc/hostcheck_adjoint.cpp), on CPU:

  - every element form on the adjoint path: the vector-Jacobian product equals central finite
    differences of the same element's forward map, in all seven inputs (x, px, y, py, z, pz,
    beta) and in the element strength (k1 of a quadrupole, k2 of a sextupole, k3 of an octupole);
  - the whole per-particle sweep (checkpoints, turn and element recomputation) on a small ring
    equals central finite differences of the oracle's tracking, the reference restatement, at
    h = 1e-7 relative."""
import ctypes
import importlib
import os
import subprocess
import zlib

import numpy as np
import pytest

from conftest import ROOT, load_abi, load_oracle
from helpers import oracle_track

abi = load_abi()
rings = importlib.import_module("bmad-ecosystem_b200.rings")
HA = os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_hostadjoint.so")


@pytest.fixture(scope="module")
def ha():
    if not os.path.exists(HA):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    lib = ctypes.CDLL(HA)
    P, D = ctypes.POINTER, ctypes.POINTER(ctypes.c_double)
    lib.bmadgpu_hostadjoint_element_track.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), ctypes.c_int32, D, D]
    lib.bmadgpu_hostadjoint_element_vjp.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), ctypes.c_int32, D, D, D]
    lib.bmadgpu_hostadjoint_loss_grad.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), P(abi.Bunch),
                                                  ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                  P(ctypes.c_int32), D, D]
    return lib


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def beta_of(p, pz):
    pc = p.p0c * (1 + pz)
    return pc / np.sqrt(pc * pc + p.mass * p.mass)


STRENGTH = {abi.QUADRUPOLE: "k1", abi.SEXTUPOLE: "k2", abi.OCTUPOLE: "k3"}


def element_cases():
    p = abi.electron_param(3e9)
    ap = dict(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
    return [
        ("drift", abi.default_element(abi.DRIFT, l=1.0, **ap)),
        ("quad_f", abi.default_element(abi.QUADRUPOLE, l=0.4, k1=0.8, **ap)),
        ("quad_d", abi.default_element(abi.QUADRUPOLE, l=0.4, k1=-0.8, **ap)),
        ("quad_weak", abi.default_element(abi.QUADRUPOLE, l=0.4, k1=1e-3, **ap)),
        ("quad_misaligned", abi.default_element(abi.QUADRUPOLE, l=0.4, k1=0.8, x_offset=5e-5, y_offset=-3e-5,
                                                tilt=1e-3, **ap)),
        ("quad_multipoles", abi.default_element(abi.QUADRUPOLE, l=0.4, k1=-0.6, b_pole={3: 2e-3, 5: 1e-2},
                                                **ap)),
        ("sextupole", abi.default_element(abi.SEXTUPOLE, l=0.2, k2=12.0, **ap)),
        ("sextupole_misaligned", abi.default_element(abi.SEXTUPOLE, l=0.2, k2=-18.0, x_offset=4e-5, y_offset=2e-5,
                                                     tilt=2e-4, **ap)),
        ("sextupole_b3_b10", abi.default_element(abi.SEXTUPOLE, l=0.2, k2=12.0,
                                                 b_pole={n: 1e-4 * (n - 2) for n in range(3, 11)}, **ap)),
        ("octupole", abi.default_element(abi.OCTUPOLE, l=0.3, k3=50.0, **ap)),
        ("sbend", abi.default_element(abi.SBEND, l=1.5, g=2 * np.pi / 100 / 1.5, fringe_type=abi.FRINGE_NONE, **ap)),
        ("sbend_ref_tilt", abi.default_element(abi.SBEND, l=1.5, g=0.05, ref_tilt=0.2, fringe_type=abi.FRINGE_NONE,
                                               **ap)),
        ("rfcavity", abi.default_element(abi.RFCAVITY, l=0.0, voltage=2e6, rf_frequency=5e8, **ap)),
        ("rfcavity_long", abi.default_element(abi.RFCAVITY, l=0.6, voltage=3e6, rf_frequency=5e8, phi0=0.1, **ap)),
        ("marker", abi.default_element(abi.MARKER, **ap)),
    ], p


CASES, PARAM = element_cases()


@pytest.mark.parametrize("name,ele", CASES, ids=[c[0] for c in CASES])
def test_element_vjp_matches_finite_differences(ha, name, ele):
    p = PARAM
    arr = abi.element_array([ele])
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    scale = np.array([2e-3, 3e-4, 1.5e-3, 2e-4, 2e-3, 1e-3])
    for trial in range(5):
        s = np.empty(7)
        s[:6] = rng.normal(0, 1, 6) * scale
        s[6] = beta_of(p, s[5])
        lam = rng.normal(0, 1, 7)
        lam_in = lam.copy()
        gs = ctypes.c_double()
        r = ha.bmadgpu_hostadjoint_element_vjp(arr, 1, ctypes.byref(p), 0, dptr(s), dptr(lam_in), ctypes.byref(gs))
        assert r == 0

        def out_of(state, elements=arr):
            out = np.empty(7)
            st = ha.bmadgpu_hostadjoint_element_track(elements, 1, ctypes.byref(p), 0, dptr(state), dptr(out))
            assert st == abi.ALIVE
            return out

        def column(k, h):
            # fourth-order central difference of every output on its own (outputs near 1, such as
            # beta, or differences of near-equal terms, such as the bend's z, would otherwise
            # bury the derivative in rounding); h large enough that rounding stays below 1e-8
            def at(d):
                q = s.copy()
                q[k] += d
                return out_of(q)
            return (8 * (at(h) - at(-h)) - (at(2 * h) - at(-2 * h))) / (12 * h)

        fd = np.array([float(lam @ column(k, 1e-2 * scale[k] if k < 6 else 1e-5)) for k in range(7)])
        err = np.abs(lam_in - fd) / (np.abs(fd) + 1e-6 * np.max(np.abs(fd)) + 1e-300)
        assert np.all(err < 1e-6), (name, trial, lam_in, fd, err)
        # strength: gs = k dL/dk
        key = STRENGTH.get(ele.key)
        if key is None:
            assert gs.value == 0.0
            continue
        k0 = getattr(ele, key)
        h = 1e-3   # relative, fourth-order stencil

        def at_k(d):
            e2 = abi.element_array([ele])
            setattr(e2[0], key, k0 * (1 + d))
            return out_of(s, e2)
        fd_k = float(lam @ ((8 * (at_k(h) - at_k(-h)) - (at_k(2 * h) - at_k(-2 * h))) / (12 * h)))
        assert abs(gs.value - fd_k) <= 1e-6 * abs(fd_k) + 1e-12 * np.max(np.abs(fd)), (name, gs.value, fd_k)


def ring_params(eles):
    """Gradient slots: every quadrupole (k1) and sextupole (k2), in element order."""
    slots = np.full(len(eles), -1, dtype=np.int32)
    names = []
    for i, e in enumerate(eles):
        if e.key in (abi.QUADRUPOLE, abi.SEXTUPOLE):
            slots[i] = len(names)
            names.append((i, STRENGTH[e.key]))
    return slots, names


def host_loss_grad(ha, eles, p, vec, n_turns, every):
    arr = abi.element_array(eles)
    slots, names = ring_params(eles)
    v = np.ascontiguousarray(vec, dtype=np.float64).copy()
    n = v.shape[1]
    beta = beta_of(p, v[5]).copy()
    state = np.full(n, abi.ALIVE, dtype=np.int32)
    b = abi.Bunch(n, v.ctypes.data, beta.ctypes.data, None, state.ctypes.data, None, None, None)
    loss = ctypes.c_double()
    gs = np.zeros(len(names))
    r = ha.bmadgpu_hostadjoint_loss_grad(arr, len(arr), ctypes.byref(p), ctypes.byref(b), n_turns, every, len(names),
                                         slots.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                         ctypes.byref(loss), dptr(gs))
    assert r == 0
    k = np.array([getattr(eles[i], key) for i, key in names])
    return loss.value, gs / k, names, state


def oracle_loss(eles, p, vec, n_turns):
    o = oracle_track(eles, p, vec, n_turns)
    alive = o["state"] == abi.ALIVE
    return float(np.sum(o["vec"][0, alive] ** 2 + o["vec"][2, alive] ** 2) / vec.shape[1]), alive


def fd_grad(eles, p, vec, n_turns, names, slots_idx, h):
    out = np.empty(len(slots_idx))
    for q, s in enumerate(slots_idx):
        i, key = names[s]
        vals = []
        for sgn in (1, -1):
            e2 = abi.element_array(eles)
            setattr(e2[i], key, getattr(eles[i], key) * (1 + sgn * h))
            vals.append(oracle_loss(e2, p, vec, n_turns)[0])
        out[q] = (vals[0] - vals[1]) / (2 * h * getattr(eles[i], key))
    return out


def test_ring_adjoint_matches_oracle_central_differences(ha):
    """Config-0 ring (50 cells), a small bunch and few turns so the oracle's differences run in
    seconds. Central differences at h = 1e-5 relative (truncation ~h^2, rounding well below) agree
    with the adjoint to 1e-6 of the largest gradient component. At h = 1e-7 the differences carry
    the tracking's rounding noise (coordinates vary by ~1e-11 relative between neighbouring
    strengths after 12 turns), about 1e-5 of the gradient; they agree to that. The sextupole
    gradients are ~1e4 times smaller, so their differences need h = 5e-3 to rise above the same
    noise (the loss is close to linear in k2 there: truncation stays below 1e-7)."""
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 32, seed=2)
    n_turns, every = 12, 5
    loss, grad, names, state = host_loss_grad(ha, eles, p, vec, n_turns, every)
    lo, alive = oracle_loss(eles, p, vec, n_turns)
    assert np.all(alive) and np.all(state == abi.ALIVE)
    assert abs(loss - lo) <= 1e-12 * abs(lo)
    pick = [0, 1, 2, 3, 40, 41, 98, 99, 101, 150, 198, 199]
    g = grad[pick]
    quads = np.array([names[s][1] == "k1" for s in pick])
    sexts = ~quads
    for fam, h in ((quads, 1e-5), (sexts, 5e-3)):
        fd = fd_grad(eles, p, vec, n_turns, names, [s for s, q in zip(pick, fam) if q], h)
        rel = np.abs(g[fam] - fd) / np.abs(fd)
        assert rel.max() < 1e-6, (rel, g[fam], fd)
    fd7 = fd_grad(eles, p, vec, n_turns, names, pick, 1e-7)
    assert np.linalg.norm(g[quads] - fd7[quads]) / np.linalg.norm(fd7[quads]) < 1e-4
