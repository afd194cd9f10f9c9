"""Differentiation on the GPU (bmadgpu_loss_grad, autograd.TrackingLoss): d(loss)/d(quadrupole
k1, sextupole k2) by the hand-written adjoint kernel.

  - the device adjoint equals the host build of the same code up to the device libm's ulp
    differences, amplified by the tracking as in the forward parity tests (loss 1e-10, gradient
    1e-8 of the largest component);
  - it matches central finite differences of the oracle (the reference restatement) to 1e-6:
    quadrupoles at h = 1e-5 relative, sextupoles (gradients ~1e4 times smaller) at h = 5e-3; at
    the benchmark's h = 1e-7 the differences themselves carry ~1e-5 rounding noise;
  - the checkpoint interval changes no bit of the gradient;
  - the torch.autograd.Function gives the same gradient and an optimiser step lowers the loss;
  - unsupported element forms are refused."""
import ctypes
import importlib

import numpy as np
import pytest
import torch

from conftest import load_abi
from test_adjoint_cpu import HA, fd_grad, host_loss_grad, oracle_loss, ring_params

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
autograd = importlib.import_module("bmad-ecosystem_b200.autograd")
abi = load_abi()


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _load_ha():
    lib_ = ctypes.CDLL(HA)
    P, D = ctypes.POINTER, ctypes.POINTER(ctypes.c_double)
    lib_.bmadgpu_hostadjoint_loss_grad.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), P(abi.Bunch),
                                                   ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                   P(ctypes.c_int32), D, D]
    return lib_


def gpu_loss_grad(ctx, eles, p, vec, n_turns, every, param_ele):
    lat = lib.Lattice(ctx, eles, p)
    b = lib.HostBunch.from_vec(vec, p)
    return lib.loss_grad(ctx, lat, b, n_turns, param_ele, checkpoint_every=every)


def test_device_adjoint_equals_host_build(ctx):
    ha = _load_ha()
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 64, seed=2)
    slots, names = ring_params(eles)
    param_ele = [i for i, _ in names]
    loss_g, grad_g = gpu_loss_grad(ctx, eles, p, vec, 20, 7, param_ele)
    loss_h, grad_h, _, _ = host_loss_grad(ha, eles, p, vec, 20, 7)
    assert abs(loss_g - loss_h) <= 1e-10 * abs(loss_h)
    quads = np.array([k == "k1" for _, k in names])
    for fam in (quads, ~quads):
        rel = np.abs(grad_g[fam] - grad_h[fam]) / np.max(np.abs(grad_h[fam]))
        assert rel.max() < 1e-8, rel.max()


def test_gradient_matches_oracle_finite_differences(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 48, seed=2)
    n_turns = 32
    slots, names = ring_params(eles)
    param_ele = [i for i, _ in names]
    loss, grad = gpu_loss_grad(ctx, eles, p, vec, n_turns, 16, param_ele)
    lo, alive = oracle_loss(eles, p, vec, n_turns)
    assert np.all(alive)
    assert abs(loss - lo) <= 1e-11 * abs(lo)
    pick_q = [s for s in range(len(names)) if names[s][1] == "k1"][::23]
    pick_s = [s for s in range(len(names)) if names[s][1] == "k2"][::23]
    for pick, h in ((pick_q, 1e-5), (pick_s, 5e-3)):
        fd = fd_grad(eles, p, vec, n_turns, names, pick, h)
        rel = np.abs(grad[pick] - fd) / np.abs(fd)
        assert rel.max() < 1e-6, (rel, grad[pick], fd)


def test_checkpoint_interval_changes_no_bit(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 40, seed=5)
    _, names = ring_params(eles)
    param_ele = [i for i, _ in names]
    ref = gpu_loss_grad(ctx, eles, p, vec, 24, 1, param_ele)
    for every in (5, 16, 24, 100):
        got = gpu_loss_grad(ctx, eles, p, vec, 24, every, param_ele)
        assert got[0] == ref[0]
        assert np.array_equal(got[1], ref[1]), every


def test_autograd_function_and_descent(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 128, seed=2)
    _, names = ring_params(eles)
    param_ele = [i for i, _ in names]
    b = lib.HostBunch.from_vec(vec, p)
    prob = autograd.StrengthProblem(ctx, eles, p, param_ele, b, n_turns=16, checkpoint_every=8)
    k = torch.tensor(prob.strengths(), dtype=torch.float64, requires_grad=True)
    loss = autograd.TrackingLoss.apply(k, prob)
    loss.backward()
    l0, g0 = gpu_loss_grad(ctx, eles, p, vec, 16, 8, param_ele)
    assert float(loss.detach()) == l0
    assert np.array_equal(k.grad.numpy(), g0)
    # a small step against the gradient lowers the loss by what the gradient predicts
    with torch.no_grad():
        g = k.grad
        alpha = 1e-6 * float(k.abs().max()) / float(g.abs().max())
        k2 = k - alpha * g
    l1 = float(autograd.TrackingLoss.apply(k2, prob))
    predicted = -alpha * float((g * g).sum())
    assert l1 < l0
    assert abs((l1 - l0) - predicted) < 0.05 * abs(predicted), (l1 - l0, predicted)


def test_unsupported_forms_refused(ctx):
    eles, p = rings.ring(10, fringe=True)   # Hwang edge kicks are outside the adjoint path
    lat = lib.Lattice(ctx, eles, p)
    b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, 8, seed=1), p)
    with pytest.raises(lib.BmadGpuError) as ex:
        lib.loss_grad(ctx, lat, b, 4, [1])
    assert ex.value.code == abi.EUNSUPPORTED
    eles, p = rings.ring(10)
    lat = lib.Lattice(ctx, eles, p)
    with pytest.raises(lib.BmadGpuError) as ex:
        lib.loss_grad(ctx, lat, b, 4, [0])       # a drift has no strength
    assert ex.value.code == abi.EINVAL


def test_full_size_gradient_matches_oracle_differences(ctx):
    """The differentiation workload at full size (50-cell ring, 4096 particles, 256 turns,
    checkpoints every 16) against the oracle's fourth-order central differences committed in
    tests/golden/adjoint_config4_fd.json (tests/golden/make_adjoint_fd.py) for 12 quadrupoles and
    12 sextupoles: the quadrupoles <= 1e-6 relative (measured up to 8.7e-7), the sextupoles <= 1e-6
    of the largest sextupole component (measured up to 6.6e-7; relative to their own values up to
    6.8e-6 on the smallest, within the differences' rounding noise). The second-order differences
    at h = 1e-7 carry that noise in full (measured 4.5e-6 and 4.3e-5) and are compared at 5e-4."""
    import json
    import os
    from conftest import ROOT
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "adjoint_config4_fd.json")))
    eles, p = rings.ring(d["n_cells"])
    vec = rings.matched_gaussian(eles, d["n_particles"], seed=d["seed"])
    loss, grad = gpu_loss_grad(ctx, eles, p, vec, d["n_turns"], 16, d["param_ele"])
    assert abs(loss - d["loss"]) <= 1e-9 * d["loss"]
    quads = np.arange(len(grad)) % 2 == 0       # slots alternate quadrupole, sextupole
    for e in d["entries"]:
        g = grad[e["slot"]]
        if e["order"] == 2:
            assert abs(g - e["fd"]) <= 5e-4 * abs(e["fd"]), (e, g)
        elif e["attr"] == "k1":
            assert abs(g - e["fd"]) <= 1e-6 * abs(e["fd"]), (e, g)
        else:
            # a sextupole difference carries ~1e-16 of rounding noise (its spread over step sizes,
            # measured on the GPU): 1e-6 of the largest sextupole component bounds it
            assert abs(g - e["fd"]) <= 1e-6 * np.max(np.abs(grad[~quads])), (e, g)


def _gpu_fd6(ctx, eles, p, vec, names, hq, hs, n_turns):
    """Sixth-order central differences [45 (L1 - L-1) - 9 (L2 - L-2) + (L3 - L-3)] / (60 h k) of the
    loss of the GPU's forward tracking for every strength in names; the 6 x len(names) perturbed
    rings are tracked together as one batch."""
    n = vec.shape[1]
    steps = (1, -1, 2, -2, 3, -3)
    lats, hs_ = [], []
    for i, attr in names:
        h = hq if attr == "k1" else hs
        hs_.append(h)
        for m in steps:
            e2 = abi.element_array(eles)
            setattr(e2[i], attr, getattr(eles[i], attr) * (1 + m * h))
            lats.append(lib.Lattice(ctx, e2, p))
    whole = lib.concat_bunches([lib.HostBunch.from_vec(vec, p)] * len(lats))
    batch = lib.Batch(ctx, lats, [n] * len(lats))
    batch.upload(-1, whole)
    batch.track(n_turns)
    out = lib.HostBunch(np.zeros((6, whole.n)), np.zeros(whole.n))
    batch.download(-1, out)
    batch.close()
    for lat in lats:
        lat.close()
    L = []
    for part in lib.split_bunch(out, [n] * len(lats)):
        assert (part.state == abi.ALIVE).all()
        L.append(float(np.sum(part.vec[0] ** 2 + part.vec[2] ** 2) / n))
    L = np.array(L).reshape(len(names), 6)
    k = np.array([getattr(eles[i], attr) for i, attr in names])
    return (45 * (L[:, 0] - L[:, 1]) - 9 * (L[:, 2] - L[:, 3]) + (L[:, 4] - L[:, 5])) / (60 * np.array(hs_) * k)


def test_all_200_components_match_gpu_finite_differences(ctx):
    """Every one of the 200 gradient components of the full-size workload against central
    differences of the GPU's own forward tracking (whose parity with the oracle is checked
    elsewhere): sixth-order stencils at three step sizes (h = 2, 3, 4 x 1e-5 relative for
    quadrupoles, 4, 6, 8 x 1e-3 for sextupoles), whose median is the reference value and whose
    spread is the differences' own uncertainty -- the loss carries ~1e-11 relative rounding noise
    after 256 turns, which a difference divides by h k.
      - per family (100 quadrupoles, 100 sextupoles): |g - fd| / |fd| <= 1e-6 as vectors;
      - every component: |g - fd| <= 1e-6 of the family's largest component, and <= 1e-6 of its
        own difference plus that difference's spread (the smallest sextupole components, ~0.5 %
        of the largest, are resolved by the differences only to ~1e-5 of themselves)."""
    n_turns, every = 256, 16
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 4096, seed=2)
    slots, names = ring_params(eles)
    param_ele = [i for i, _ in names]
    loss, grad = gpu_loss_grad(ctx, eles, p, vec, n_turns, every, param_ele)
    F = np.stack([_gpu_fd6(ctx, eles, p, vec, names, m * 1e-5, m * 2e-3, n_turns) for m in (2, 3, 4)])
    fd, spread = np.median(F, axis=0), F.max(axis=0) - F.min(axis=0)
    quads = np.array([attr == "k1" for _, attr in names])
    for fam in (quads, ~quads):
        g, f = grad[fam], fd[fam]
        assert np.linalg.norm(g - f) / np.linalg.norm(f) <= 1e-6
        assert np.max(np.abs(g - f)) <= 1e-6 * np.max(np.abs(g))
        assert np.all(np.abs(g - f) <= 1e-6 * np.abs(f) + spread[fam])
    assert np.all(np.abs(grad[quads] - fd[quads]) <= 1e-6 * np.abs(fd[quads]))
