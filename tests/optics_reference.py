"""numpy restatement of the optics set-up before tracking (test infrastructure, for checking the device path):

  closed_orbit_calc          bmad/code/closed_orbit_calc.f90:192-862: the fixed point of the
                             one-turn map, here Newton's method on the ORACLE's tracking
                             (helpers.oracle_track), apertures off, RF off for dims 4 and 5
  twiss_from_mat6            bmad/code/twiss_from_mat6.f90:24-126
  mat_symp_decouple          bmad/low_level/mat_symp_decouple.f90:22-157
  twiss_from_mat2            bmad/low_level/twiss_from_mat2.f90:19-60
  init_random_distribution   bmad/multiparticle/beam_utils.f90:551-721
  init_bunch_distribution    beam_utils.f90:491-509 (dispersion and make_v_mats coupling),
                             bunch_init_end_calc beam_utils.f90:1920-1923 (centre)
  Philox4x32-10              Salmon, Moraes, Dror, Shaw, SC11 (the published block function)
"""
import ctypes

import numpy as np

from conftest import load_abi
from helpers import oracle_track

abi = load_abi()

FD_STEP = 1e-5
OFFSETS = (1.0, -1.0, 2.0, -2.0)


def orbit_lattice(elements, param, rf_off):
    """Copies with apertures off and, for rf_off, the cavities switched off."""
    arr = abi.element_array(elements)
    if rf_off:
        for e in arr:
            if e.key == abi.RFCAVITY:
                e.is_on = 0
    p = type(param).from_buffer_copy(param)
    p.aperture_limit_on = 0
    return arr, p


def one_turn(arr, p, x):
    """(f(x), fourth-order central-difference one-turn matrix) with the oracle's tracking."""
    vec = np.repeat(np.asarray(x, float)[:, None], 25, axis=1)
    for k in range(6):
        for m, o in enumerate(OFFSETS):
            vec[k, 1 + 4 * k + m] += o * FD_STEP
    out = oracle_track(arr, p, vec, 1)
    assert np.all(out["state"] == abi.ALIVE)
    f = out["vec"]
    M = np.zeros((6, 6))
    for k in range(6):
        c = 1 + 4 * k
        M[:, k] = (8 * (f[:, c] - f[:, c + 1]) - (f[:, c + 2] - f[:, c + 3])) / (12 * FD_STEP)
    return f[:, 0].copy(), M


def closed_orbit(elements, param, dim, guess=None, rel_tol=1e-9, abs_tol=1e-12, max_iter=100):
    """Newton iteration to the reference's stopping rule (closed_orbit_calc.f90:519-534)."""
    arr, p = orbit_lattice(elements, param, rf_off=(dim != 6))
    x = np.zeros(6) if guess is None else np.array(guess, float)
    if dim != 6:
        x[4] = 0.0
    ix = [0, 1, 2, 3, 5] if dim == 5 else list(range(dim))
    for _ in range(max_iter):
        f, M = one_turn(arr, p, x)
        res = f[:dim] - x[:dim]
        if np.all(np.abs(res) < np.abs(x[:dim]) * rel_tol + abs_tol):
            return x, M
        J = M[:dim][:, ix] - np.eye(6)[:dim][:, ix]
        dx = np.linalg.solve(J, -res)
        x[ix] += dx
    raise AssertionError("closed orbit not converging")


def symp_conj(m):
    """Symplectic conjugate of an even-sized matrix: -S m^T S (mat_symp_conj)."""
    n = m.shape[0]
    S = np.zeros((n, n))
    for k in range(n // 2):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    return -S @ m.T @ S


def twiss_from_mat2(m):
    det = m[0, 0] * m[1, 1] - m[0, 1] * m[1, 0]
    m = m / det
    c = (m[0, 0] + m[1, 1]) / 2
    if abs(c) >= 1:
        return None
    s = np.copysign(1.0, m[0, 1]) * np.sqrt(1 - c * c)
    phi = np.arctan2(s, c)
    if phi < 0:
        phi += 2 * np.pi
    alpha = (m[0, 0] - m[1, 1]) / (2 * s)
    radical = -(1 + alpha ** 2) * m[0, 1] / m[1, 0]
    if radical <= 0:
        return None
    beta = np.sqrt(radical)
    return dict(beta=beta, alpha=alpha, gamma=(1 + alpha ** 2) / beta, phi=phi)


def twiss_from_mat6(mat6, orb0=None):
    """dict with the bmadgpu_twiss field names; status as matrix_status (1 = ok)."""
    orb0 = np.zeros(6) if orb0 is None else np.asarray(orb0, float)
    m4 = np.array(mat6[:4, :4], float)
    if np.max(np.abs(m4)) > 1e10:
        return dict(status=4)
    S = np.zeros((4, 4))
    S[0, 1] = S[2, 3] = 1.0
    S[1, 0] = S[3, 2] = -1.0
    if np.max(np.abs(m4.T @ S @ m4 - S)) > 1:
        return dict(status=3)
    M, m, n, N = m4[:2, :2], m4[:2, 2:], m4[2:, :2], m4[2:, 2:]
    if np.all(m == 0):
        gamma, C = 1.0, np.zeros((2, 2))
    else:
        H = m + symp_conj(n)
        t = np.trace(M) - np.trace(N)
        denom = t * t + 4 * np.linalg.det(H)
        if denom <= 0:
            return dict(status=2)
        gamma = np.sqrt(0.5 + 0.5 * np.sqrt(t * t / denom))
        C = -np.copysign(1.0, t) / (gamma * np.sqrt(denom)) * H
    V = np.zeros((4, 4))
    V[:2, :2] = V[2:, 2:] = gamma * np.eye(2)
    V[:2, 2:] = C
    V[2:, :2] = -symp_conj(C)
    U = symp_conj(V) @ m4 @ V
    ta, tb = U[0, 0] + U[1, 1], U[2, 2] + U[3, 3]
    if abs(ta) > 2 or abs(tb) > 2:
        return dict(status=4 if (abs(ta) > 2 and abs(tb) > 2) else (5 if abs(ta) > 2 else 6))
    a, b = twiss_from_mat2(U[:2, :2]), twiss_from_mat2(U[2:, 2:])
    if a is None:
        return dict(status=5)
    if b is None:
        return dict(status=6)
    out = dict(status=1, gamma_c=gamma, c_mat=C)
    for k, v in a.items():
        out[k + "_a"] = v
    for k, v in b.items():
        out[k + "_b"] = v
    eta = np.linalg.solve(np.eye(4) - m4, np.asarray(mat6)[:4, 5])
    out.update(eta_x=eta[0], etap_x=eta[1], eta_y=eta[2], etap_y=eta[3])
    en = symp_conj(V) @ eta
    out.update(eta_a=en[0], etap_a=en[1], eta_b=en[2], etap_b=en[3])
    return out


# ---- matched beam ----------------------------------------------------------------------------

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 on uint64 arrays holding 32-bit words."""
    c = [np.asarray(v, np.uint64) & 0xFFFFFFFF for v in (c0, c1, c2, c3)]
    k0, k1 = np.uint64(k0), np.uint64(k1)
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
        k0 = (k0 + np.uint64(W0)) & mask
        k1 = (k1 + np.uint64(W1)) & mask
    return c


def deviates(seed, n, sigma_cutoff=0.0):
    """[6 n + 8]: deviate k of particle i from counter (i, attempt, k), then the jitters."""
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32

    def draw(idx, k):
        idx = np.asarray(idx, np.uint64)
        out = np.zeros(idx.shape)
        todo = np.ones(idx.shape, bool)
        for a in range(64):
            c = philox4x32_10(idx & np.uint64(0xFFFFFFFF), idx >> np.uint64(32), np.full(idx.shape, a, np.uint64),
                              np.full(idx.shape, k, np.uint64), k0, k1)
            u1 = (((c[0] << np.uint64(21)) | (c[1] >> np.uint64(11))).astype(np.float64) + 0.5) * 2.0 ** -53
            u2 = (((c[2] << np.uint64(21)) | (c[3] >> np.uint64(11))).astype(np.float64) + 0.5) * 2.0 ** -53
            r = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
            ok = todo & ((sigma_cutoff <= 0) | (np.abs(r) <= sigma_cutoff))
            out[ok] = r[ok]
            todo &= ~ok
            if not todo.any():
                break
        return out

    i = np.arange(n, dtype=np.uint64)
    parts = [draw(i, k) for k in range(6)]
    extra = [draw(np.array([n]), k)[0] for k in range(2)] + [draw(np.array([n + 1]), k)[0] for k in range(6)]
    return np.concatenate(parts + [np.array(extra)])


def init_random_distribution(normals, n, tw, a_emit, b_emit, sig_z, sig_pz, dpz_dz=0.0, sig_z_jitter=0.0,
                             sig_pz_jitter=0.0, center=None, center_jitter=None, renorm_center=True,
                             renorm_sigma=True, orbit=None):
    """vec [6, n] as init_bunch_distribution builds it from the given deviates."""
    r = np.array(normals[:6 * n], float).reshape(6, n)
    extra = np.asarray(normals[6 * n:], float)
    if renorm_sigma:
        ave = r.sum(axis=1) / n
        sig = (r @ r.T) / n
        r = r - ave[:, None]
        sig = sig - np.outer(ave, ave)
        if n > 6:
            for i in range(4, -1, -1):
                for j in range(i + 1, 6):
                    b = -sig[i, j] / sig[j, j]
                    r[i] = r[i] + b * r[j]
                    sig[i, i] = sig[i, i] + 2 * b * sig[i, j] + b * b * sig[j, j]
                    for j2 in range(6):
                        if j2 == i:
                            continue
                        sig[i, j2] = sig[i, j2] + b * sig[j, j2]
                        sig[j2, i] = sig[i, j2]
        if n > 1:
            r = r * np.sqrt(1 / np.diag(sig))[:, None]
    s = [np.sqrt(a_emit * tw["beta_a"]), np.sqrt(a_emit / tw["beta_a"]), np.sqrt(b_emit * tw["beta_b"]),
         np.sqrt(b_emit / tw["beta_b"]), sig_z * (1 + sig_z_jitter * extra[0]),
         sig_pz * (1 + sig_pz_jitter * extra[1])]
    a = 0.0 if (s[5] == 0 or dpz_dz == 0) else dpz_dz * s[4] / s[5]
    b = np.sqrt(1 - a * a)
    v = np.empty_like(r)
    v[0] = s[0] * r[0]
    v[1] = -s[1] * (r[1] + r[0] * tw["alpha_a"])
    v[2] = s[2] * r[2]
    v[3] = -s[3] * (r[3] + r[2] * tw["alpha_b"])
    v[4] = s[4] * r[4]
    v[5] = s[5] * (r[5] * b + r[4] * a)
    if renorm_center:
        v = v - (v.sum(axis=1) / n)[:, None]
    eta = np.array([tw["eta_a"], tw["etap_a"], tw["eta_b"], tw["etap_b"]])
    C = np.asarray(tw["c_mat"], float).reshape(2, 2)
    g = tw["gamma_c"]
    V = np.zeros((4, 4))
    V[:2, :2] = V[2:, 2:] = g * np.eye(2)
    V[:2, 2:] = C
    V[2:, :2] = -symp_conj(C)
    pt = v[:4] + v[5][None, :] * eta[:, None]
    v[:4] = V @ pt
    cen = np.zeros(6) if center is None else np.asarray(center, float)
    cj = np.zeros(6) if center_jitter is None else np.asarray(center_jitter, float)
    v = v + (cen + cj * extra[2:8])[:, None]
    if orbit is not None:
        v = v + np.asarray(orbit, float)[:, None]
    return v
