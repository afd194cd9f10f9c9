"""Long-term-tracking bunch data on CPU: the library's host reduction (bunchdata.cpp, through
bmadgpu_bunch_data_from_sums, which needs no GPU) against the numpy restatement of
ltt_calc_bunch_data / calc_bunch_params / mat_eigen (tests/ltt_reference.py) on synthetic
bunches: uncoupled and coupled (x-y and x-z), with and without an energy spread, with lost
particles, and below the 10- and 6-particle thresholds of the reference."""
import importlib

import numpy as np
import pytest

from ltt_reference import bunch_data, two_pass_sums

lib = importlib.import_module("bmad-ecosystem_b200.lib")
abi = importlib.import_module("bmad-ecosystem_b200.abi")

P0C, MASS = 3e9, 0.51099895069e6


def bunch(n, seed, couple=0.0, sig_pz=1e-3, lost_frac=0.0):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((6, n))
    sig = np.array([3e-4, 2e-5, 4e-5, 3e-6, 3e-3, sig_pz])
    v = r * sig[:, None]
    v[0] += 1.5 * v[5]                      # dispersion
    v[2] += couple * v[0]                   # x-y coupling
    v[1] -= 0.3 * v[0] / 10                 # alpha
    v[4] += couple * 5 * v[0]               # x-z correlation
    v += np.array([1e-5, -2e-7, 3e-6, 1e-8, 2e-4, 1e-5])[:, None]
    t = rng.normal(1e-6, 1e-11, n)
    state = np.ones(n, np.int32)
    state[rng.random(n) < lost_frac] = 4
    return v, t, state


@pytest.mark.parametrize("case", [dict(n=5000, seed=1), dict(n=5000, seed=2, couple=0.05),
                                  dict(n=20000, seed=3, couple=0.2, lost_frac=0.1),
                                  dict(n=3000, seed=4, sig_pz=0.0), dict(n=8, seed=5), dict(n=5, seed=6)])
def test_host_reduction_matches_reference(case):
    v, t, st = bunch(**case)
    got = lib.bunch_data_from_sums(two_pass_sums(v, t, st), P0C, MASS)
    want = bunch_data(v, t, st, P0C, MASS)
    assert got["n_live"] == want["n_live"]
    keys = ["centroid", "t", "sigma_t", "sigma", "proj_emit", "proj_beta", "proj_alpha", "eta", "etap",
            "sigma_vec", "sig1", "skew", "kurt", "emit", "norm_emit"]
    if case.get("sig_pz", 1e-3) == 0.0:
        # <pz.pz> is rounding noise: dispersion and projected Twiss divide by it in both codes
        keys = [k for k in keys if not k.startswith("proj_") and k not in ("eta", "etap")]
    for k in keys:
        if k not in want:
            assert np.all(np.asarray(got[k]) == 0), k      # not computed below the thresholds
            continue
        g, w = np.asarray(got[k], float).ravel(), np.asarray(want[k], float).ravel()
        if k == "sigma":
            g = g.reshape(6, 6).ravel()
        scale = np.max(np.abs(w)) if np.any(w) else 1.0
        assert np.allclose(g, w, rtol=1e-10, atol=1e-12 * scale), (k, g, w)
    if want["n_live"] >= 6:
        assert got["emit_valid"] == 1
        if case.get("sig_pz", 1e-3) == 0.0:
            assert got["emit"][2] == 0.0     # no energy spread: transverse modes only (dim = 4)


def test_combined_amplitude_is_the_sigma_quadratic_form():
    """The reference ranks particles by sum_k (j_2k^2 + j_2k+1^2) / emit_k with j = N^-1 (p - c)
    and Sigma = N diag(emit) N^T; that is (p - c)^T Sigma^-1 (p - c), the form the core-emittance
    code evaluates. Checked on a sigma matrix built from a random symplectic N."""
    rng = np.random.default_rng(3)
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    N = np.eye(6)
    for _ in range(3):  # products of symplectic maps exp(S H) with H symmetric
        H = rng.normal(size=(6, 6))
        H = 0.1 * (H + H.T)
        import scipy.linalg
        N = N @ scipy.linalg.expm(S @ H)
    assert np.max(np.abs(N.T @ S @ N - S)) < 1e-9
    emit = np.array([2e-9, 3e-10, 4e-9])
    D = np.diag(np.repeat(emit, 2))
    Sigma = N @ D @ N.T
    d = rng.normal(size=(6, 50)) * np.sqrt(np.diag(Sigma))[:, None]
    j = np.linalg.solve(N, d)
    amp_modes = sum((j[2 * k] ** 2 + j[2 * k + 1] ** 2) / emit[k] for k in range(3))
    amp_form = np.einsum("in,ij,jn->n", d, np.linalg.inv(Sigma), d)
    assert np.allclose(amp_modes, amp_form, rtol=1e-8)


def _coupled_sigma(seed):
    import scipy.linalg
    rng = np.random.default_rng(seed)
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    H = rng.normal(size=(6, 6))
    M = scipy.linalg.expm(S @ (0.2 * (H + H.T)))
    e = np.repeat([2e-9 * (1 + rng.random()), 3e-10 * (1 + rng.random()), 4e-6 * (1 + rng.random())], 2)
    return M @ np.diag(e) @ M.T


@pytest.mark.parametrize("seed", range(12))
def test_sigma_normal_form_matches_restatement(seed):
    """bmadgpu_sigma_normal_form (Jacobi eigenvectors, then mat_eigen's flip and phase, normalize_e
    and Wolski's Q) against the numpy restatement that follows the reference step by step from
    LAPACK's geev: coupled sigma matrices, and the sample sigma of a synthetic bunch."""
    from ltt_reference import normal_form_n
    if seed < 8:
        sig = _coupled_sigma(seed)
    else:
        v, t, st = bunch(4000, seed, couple=0.05 * (seed - 7))
        sig = np.cov(v, bias=True)
    emit, N = lib.sigma_normal_form(sig)
    e_ref, N_ref = normal_form_n(sig)
    assert np.allclose(emit, e_ref, rtol=1e-10, atol=0)
    assert np.max(np.abs(N - N_ref)) <= 1e-10 * np.max(np.abs(N_ref))


def test_sigma_normal_form_structure():
    """N diagonalises sigma (N^-1 sigma N^-T = diag(emit), up to the 7e-8 of Q's single-precision
    entries), is symplectic to the same level, and carries mat_eigen's phase: each mode's own-plane
    row has N(2p, 2p) = 0 and N(2p, 2p+1) > 0. A sigma that is not positive definite is refused."""
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    for seed in range(5):
        sig = _coupled_sigma(100 + seed)
        emit, N = lib.sigma_normal_form(sig)
        n_inv = np.linalg.inv(N)
        D = n_inv @ sig @ n_inv.T
        assert np.allclose(np.diag(D), np.repeat(emit, 2), rtol=2e-7, atol=0)
        off = D - np.diag(np.diag(D))
        assert np.max(np.abs(off)) < 1e-9 * np.max(emit)
        assert np.max(np.abs(N.T @ S @ N + S)) < 2e-7       # N^T S N = -S in this convention
        for pl in range(3):
            assert abs(N[2 * pl, 2 * pl]) < 1e-12 * np.max(np.abs(N))
            assert N[2 * pl, 2 * pl + 1] > 0
    bad = np.eye(6)
    bad[0, 0] = -1.0
    with pytest.raises(lib.BmadGpuError):
        lib.sigma_normal_form(bad)


@pytest.mark.parametrize("seed", range(4))
def test_make_n_normal_form_of_a_one_turn_matrix(seed):
    """lib.make_n (make_N of mode3_mod) on a stable coupled one-turn matrix t6 = A B R B^-1 A^-1
    with planted tunes: N^-1 t6 N is three rotation blocks with those tunes, N is symplectic, and
    its phase convention holds (N(1,2) = N(3,4) = N(5,6) = 0 with positive diagonal partners)."""
    import scipy.linalg
    rng = np.random.default_rng(seed)
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    H = rng.normal(size=(6, 6))
    A = scipy.linalg.expm(S @ (0.15 * (H + H.T)))
    tunes = np.array([0.22, 0.31, 0.013]) + 0.02 * rng.random(3)
    R = np.zeros((6, 6))
    for k in range(3):
        c, s = np.cos(2 * np.pi * tunes[k]), np.sin(2 * np.pi * tunes[k])
        R[2 * k:2 * k + 2, 2 * k:2 * k + 2] = [[c, s], [-s, c]]
    B = np.diag([3.0, 1 / 3.0, 2.0, 0.5, 10.0, 0.1])
    t6 = A @ B @ R @ np.linalg.inv(B) @ np.linalg.inv(A)
    N = lib.make_n(t6)
    U = np.linalg.inv(N) @ t6 @ N
    for k in range(3):
        blk = U[2 * k:2 * k + 2, 2 * k:2 * k + 2]
        assert np.allclose(blk, R[2 * k:2 * k + 2, 2 * k:2 * k + 2], atol=1e-10)
    off = U.copy()
    for k in range(3):
        off[2 * k:2 * k + 2, 2 * k:2 * k + 2] = 0
    assert np.max(np.abs(off)) < 1e-10
    assert np.allclose(N.T @ S @ N, S, atol=1e-10)
    for k in range(3):
        assert abs(N[2 * k, 2 * k + 1]) < 1e-12 * np.max(np.abs(N)) and N[2 * k, 2 * k] > 0


def test_sigma_normal_form_without_longitudinal_spread():
    """dim 4 (zero z and pz spread, as calc_emittances_and_twiss_from_sigma_matrix decides it): the
    transverse modes as in 6D, the c emittance zero, and N's longitudinal block the identity (the
    reference leaves it unset)."""
    from ltt_reference import normal_form_n
    sig6 = _coupled_sigma(3)
    sig = sig6.copy()
    sig[4:, :] = 0
    sig[:, 4:] = 0
    emit, N = lib.sigma_normal_form(sig)
    assert emit[2] == 0 and emit[0] > 0 and emit[1] > 0
    assert np.array_equal(N[4:, 4:], np.eye(2)) and not np.any(N[4:, :4]) and not np.any(N[:4, 4:])
    n_inv = np.linalg.inv(N[:4, :4])
    D = n_inv @ sig[:4, :4] @ n_inv.T
    assert np.allclose(np.diag(D), np.repeat(emit[:2], 2), rtol=2e-7, atol=0)
