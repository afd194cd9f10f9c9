"""Synthetic storage rings and beams of the benchmark workloads, built programmatically.

The reference reads lattices from .bmad files (bmad/parsing/); here the rings are assembled
directly as element records (abi.Element), with Bmad's element defaults applied
(abi.default_element). Beams are Gaussian, matched to the periodic linear optics of the ring
(uncoupled, with dispersion), the role of init_random_distribution
(bmad/multiparticle/beam_utils.f90:551-721) plus the closed-orbit/Twiss setup of
long_term_tracking (bsim/modules/lt_tracking_mod.f90:1556-1559).
"""
import math

import numpy as np

from . import abi

E_TOT = 3e9                 # 3 GeV electrons
RF_VOLTAGE = 2e6            # 2 MV
RF_FREQUENCY = 500e6        # 500 MHz
APERTURE_X = 0.020          # +-20 mm
APERTURE_Y = 0.010          # +-10 mm


def _aperture():
    return dict(x1_limit=APERTURE_X, x2_limit=APERTURE_X, y1_limit=APERTURE_Y, y2_limit=APERTURE_Y)


def fodo_cell(angle, k1f=0.8, k1d=-0.8, k2f=12.0, k2d=-18.0, fringe=False, sext_poles=None):
    """One cell: drift 1.0, quad 0.4 (k1f), drift 0.3, sbend 1.5 (angle), drift 0.3, sextupole 0.2 (k2f),
    quad 0.4 (k1d), sextupole 0.2 (k2d), sbend 1.5 (angle). sext_poles: optional pair of dicts
    {n: bN} of extra normal multipoles for the two sextupoles (scaled by k2 L, r0_mag = 0)."""
    ap = _aperture()
    fr = dict() if fringe else dict(fringe_type=abi.FRINGE_NONE)
    g = angle / 1.5
    sp = sext_poles or ({}, {})
    return [
        abi.default_element(abi.DRIFT, l=1.0, **ap),
        abi.default_element(abi.QUADRUPOLE, l=0.4, k1=k1f, **ap),
        abi.default_element(abi.DRIFT, l=0.3, **ap),
        abi.default_element(abi.SBEND, l=1.5, g=g, **fr, **ap),
        abi.default_element(abi.DRIFT, l=0.3, **ap),
        abi.default_element(abi.SEXTUPOLE, l=0.2, k2=k2f, b_pole=sp[0], **ap),
        abi.default_element(abi.QUADRUPOLE, l=0.4, k1=k1d, **ap),
        abi.default_element(abi.SEXTUPOLE, l=0.2, k2=k2d, b_pole=sp[1], **ap),
        abi.default_element(abi.SBEND, l=1.5, g=g, **fr, **ap),
    ]


def rf_cavity(voltage=RF_VOLTAGE, frequency=RF_FREQUENCY):
    return abi.default_element(abi.RFCAVITY, l=0.0, voltage=voltage, rf_frequency=frequency, phi0=0.0,
                               **_aperture())


def set_ref_time(elements, param):
    """delta_ref_time = L / (beta0 c) for every element (constant reference energy)."""
    beta0 = param.p0c / param.e_tot
    for e in elements:
        e.delta_ref_time = e.l / (beta0 * abi.C_LIGHT)
    return elements


def ring(n_cells, fringe=False, multipole_sigma=0.0, multipole_seed=1, rf=True, cell_kw=None):
    """A ring of n_cells FODO cells (2 n_cells bends closing 2 pi) and one RF cavity.
    multipole_sigma > 0 gives every sextupole random normal multipoles b3..b10 ~ N(0, sigma)
    relative to its k2 (seed multipole_seed)."""
    angle = 2 * math.pi / (2 * n_cells)
    rng = np.random.default_rng(multipole_seed)
    eles = []
    for _ in range(n_cells):
        sp = None
        if multipole_sigma > 0:
            sp = tuple({n: float(rng.normal(0.0, multipole_sigma)) for n in range(3, 11)} for _ in range(2))
        eles += fodo_cell(angle, fringe=fringe, sext_poles=sp, **(cell_kw or {}))
    if rf:
        eles.append(rf_cavity())
    param = abi.electron_param(E_TOT)
    set_ref_time(eles, param)
    return eles, param


def perturbed_ring(n_cells, seed, strength_sigma=1e-3, offset_sigma=50e-6, tilt_sigma=1e-4):
    """A ring variant: quad/sextupole strengths scaled by 1 + N(0, strength_sigma), x/y offsets
    N(0, offset_sigma) and tilts N(0, tilt_sigma) on quadrupoles and sextupoles (per-variant seed)."""
    eles, param = ring(n_cells)
    rng = np.random.default_rng(seed)
    for e in eles:
        if e.key in (abi.QUADRUPOLE, abi.SEXTUPOLE):
            f = 1 + rng.normal(0.0, strength_sigma)
            if e.key == abi.QUADRUPOLE:
                e.k1 = e.k1 * f
            else:
                e.k2 = e.k2 * f
            e.x_offset = rng.normal(0.0, offset_sigma)
            e.y_offset = rng.normal(0.0, offset_sigma)
            e.tilt = rng.normal(0.0, tilt_sigma)
    return eles, param


# ---------------------------------------------------------------------------------------------
# Linear optics (on-momentum transfer matrices of the thick elements)

def _plane_quad(k, L):
    if abs(k) < 1e-14:
        return np.array([[1.0, L], [0.0, 1.0]])
    if k > 0:  # focusing
        s = math.sqrt(k)
        return np.array([[math.cos(s * L), math.sin(s * L) / s], [-s * math.sin(s * L), math.cos(s * L)]])
    s = math.sqrt(-k)
    return np.array([[math.cosh(s * L), math.sinh(s * L) / s], [s * math.sinh(s * L), math.cosh(s * L)]])


def element_matrix5(e):
    """5x5 linear map of (x, px, y, py, pz) for one element (pz carried for dispersion)."""
    m = np.eye(5)
    L = e.l
    if e.key == abi.QUADRUPOLE:
        m[0:2, 0:2] = _plane_quad(e.k1, L)
        m[2:4, 2:4] = _plane_quad(-e.k1, L)
    elif e.key == abi.SBEND and e.g != 0:
        g, a = e.g, e.g * L
        m[0:2, 0:2] = [[math.cos(a), math.sin(a) / g], [-g * math.sin(a), math.cos(a)]]
        m[0, 4] = (1 - math.cos(a)) / g
        m[1, 4] = math.sin(a)
        m[2:4, 2:4] = [[1.0, L], [0.0, 1.0]]
    else:
        m[0:2, 0:2] = [[1.0, L], [0.0, 1.0]]
        m[2:4, 2:4] = [[1.0, L], [0.0, 1.0]]
    return m


def periodic_optics(elements):
    """Twiss (beta, alpha) of both planes and dispersion (eta, eta') at the ring start."""
    M = np.eye(5)
    for e in elements:
        M = element_matrix5(e) @ M
    out = {}
    for name, i in (("a", 0), ("b", 2)):
        m = M[i:i + 2, i:i + 2]
        cos_mu = 0.5 * (m[0, 0] + m[1, 1])
        if abs(cos_mu) >= 1:
            raise ValueError("linear optics unstable in plane " + name)
        sin_mu = math.copysign(math.sqrt(1 - cos_mu ** 2), m[0, 1])
        out["beta_" + name] = m[0, 1] / sin_mu
        out["alpha_" + name] = (m[0, 0] - m[1, 1]) / (2 * sin_mu)
        out["tune_" + name] = math.acos(cos_mu) / (2 * math.pi) if sin_mu > 0 else 1 - math.acos(cos_mu) / (2 * math.pi)
    A = np.eye(2) - M[0:2, 0:2]
    eta = np.linalg.solve(A, M[0:2, 4])
    out["eta_x"], out["etap_x"] = float(eta[0]), float(eta[1])
    return out


def matched_gaussian(elements, n, seed, emit_a=1e-9, emit_b=10e-12, sig_z=3e-3, sig_pz=1e-3, scale=1.0):
    """n particles, 6D Gaussian with the given emittances and sigmas (times `scale`), matched to
    the ring's periodic Twiss at its start (x/px include dispersion). Returns vec[6, n]."""
    tw = periodic_optics(elements)
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((6, n))
    vec = np.empty((6, n))
    sa, sb = math.sqrt(emit_a), math.sqrt(emit_b)
    ba, bb = tw["beta_a"], tw["beta_b"]
    vec[5] = scale * sig_pz * r[5]
    vec[4] = scale * sig_z * r[4]
    vec[0] = scale * sa * math.sqrt(ba) * r[0] + tw["eta_x"] * vec[5]
    vec[1] = -scale * sa / math.sqrt(ba) * (r[1] + r[0] * tw["alpha_a"]) + tw["etap_x"] * vec[5]
    vec[2] = scale * sb * math.sqrt(bb) * r[2]
    vec[3] = -scale * sb / math.sqrt(bb) * (r[3] + r[2] * tw["alpha_b"])
    return vec


def da_grid(n, delta_values=(-0.01, 0.0, 0.01), r_max=0.025, n_rays=None):
    """Dynamic-aperture grid: particles on polar rays of x-y amplitude 0..r_max for each delta
    (bmad/modules/dynamic_aperture_mod.f90 scans rays; here the rays are sampled on a grid).
    Returns vec[6, n]."""
    nd = len(delta_values)
    per_delta = max(1, n // nd)
    if n_rays is None:
        n_rays = max(1, int(round(math.sqrt(per_delta / 4))))
    n_amp = max(1, per_delta // n_rays)
    vec = np.zeros((6, n))
    k = 0
    for d in delta_values:
        for ir in range(n_rays):
            th = (ir + 0.5) * (math.pi / 2) / n_rays   # first quadrant (symmetric ring)
            for ia in range(n_amp):
                if k >= n:
                    break
                amp = r_max * (ia + 1) / n_amp
                vec[0, k] = amp * math.cos(th)
                vec[2, k] = amp * math.sin(th)
                vec[5, k] = d
                k += 1
    while k < n:  # fill the remainder on the delta = 0 axis
        vec[0, k] = r_max * (k % 97 + 1) / 97
        k += 1
    return vec


def fma_grid(n, x_max=0.02, y_max=0.01, delta=0.0):
    """Frequency-map grid: particles on an nx x ny grid of starting amplitudes
    (0, x_max] x (0, y_max] at momentum deviation delta, as frequency_map scans the x-y plane
    (bsim/frequency_map/frequency_map.f90:183-330). Returns vec[6, n]."""
    vec = np.zeros((6, n))
    if n == 0:
        return vec
    nx = max(1, int(round(math.sqrt(n * x_max / y_max))))
    ny = max(1, -(-n // nx))
    k = np.arange(n)
    vec[0] = x_max * (k % nx + 1) / nx
    vec[2] = y_max * (k // nx + 1) / ny
    vec[5] = delta
    return vec


def serving_stream(n_jobs, seed=0, mean_gap=5e-3, cells=(50, 100, 200, 400), n_range=(256, 262144),
                   turn_range=(64, 4096)):
    """A Poisson request stream of tracking jobs: arrival time, base ring (cells), perturbation
    seed, particle count and turn count (both log-uniform), and kind ('gauss' or 'fma')."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(mean_gap, n_jobs))
    out = []
    for i in range(n_jobs):
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        turns = int(round(math.exp(rng.uniform(math.log(turn_range[0]), math.log(turn_range[1])))))
        out.append(dict(arrival=float(t[i]), cells=int(cells[rng.integers(len(cells))]),
                        variant_seed=int(rng.integers(1 << 30)), n=n, turns=turns,
                        kind="gauss" if rng.random() < 0.5 else "fma"))
    return out
