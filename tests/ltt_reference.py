"""numpy restatement of the long-term-tracking bunch data (test infrastructure, for checking the device path):

  ltt_calc_bunch_data            bsim/modules/lt_tracking_mod.f90:2369-2421
  calc_bunch_params              bmad/multiparticle/beam_utils.f90:1326-1431
  calc_bunch_sigma_matrix_etc    beam_utils.f90:1757-1844 (two passes, centred sums)
  calc_emittances_and_twiss_from_sigma_matrix  beam_utils.f90:1454-1690 (projected Twiss)
  mat_eigen                      sim_utils/matrix/mat_eigen.f90:37-187 (LAPACK geev through
                                 numpy.linalg.eig, pairing and the greedy plane sort)

Also the per-particle sums the device computes, for the host-only reduction test, and readers of
the averages / phase-space files."""
import numpy as np


def two_pass_sums(vec, t, state):
    """The 63 sums of the device's two passes, summed sequentially in particle order."""
    alive = state == 1
    v = vec[:, alive]
    tt = t[alive] if t is not None else np.zeros(v.shape[1])
    n = v.shape[1]
    s1 = [float(n)] + [float(np.sum(v[i])) for i in range(6)] + [float(np.sum(tt)), float(np.sum(tt * tt))]
    for i in range(6):
        for j in range(i, 6):
            s1.append(float(np.sum(v[i] * v[j])))
    a = np.array(s1[1:7]) / n if n else np.zeros(6)
    d = v - a[:, None]
    s2 = []
    for i in range(6):
        for j in range(i, 6):
            s2.append(float(np.sum(d[i] * d[j])))
    s2 += [float(np.sum(d[i] ** 3)) for i in range(6)]
    s2 += [float(np.sum(d[i] ** 4)) for i in range(6)]
    return np.array(s1 + s2)


def mat_eigen_emittances(sigma_s):
    """Normal-mode emittances as mat_eigen + calc_emittances_and_twiss_from_sigma_matrix give them:
    aimag of the odd eigenvalue of each pair after the sort and the normalisation flip."""
    n = sigma_s.shape[0]
    nn = n // 2
    w, vr = np.linalg.eig(sigma_s)
    # LAPACK (geev) returns complex-conjugate pairs in adjacent slots, positive imaginary part first
    pairs = [(2 * k, 2 * k + 1) for k in range(nn)]
    amp = np.zeros((nn, nn))
    for ii, (p, q) in enumerate(pairs):
        v = vr[:, p]
        re, im = v.real, v.imag
        for kk in range(nn):
            amp[kk, ii] = np.sum(re[2 * kk:2 * kk + 2] ** 2) + np.sum(im[2 * kk:2 * kk + 2] ** 2)
        amp[:, ii] /= np.sum(amp[:, ii])
    sort = np.zeros(nn, int)
    for _ in range(nn):
        amp2 = amp.copy()
        dmax = np.zeros(nn)
        for jj in range(nn):
            m = int(np.argmax(amp2[jj]))
            amp2[jj, m] = -1
            m2 = int(np.argmax(amp2[jj]))
            dmax[jj] = amp[jj, m] - amp[jj, m2]
        k = int(np.argmax(dmax))
        m = int(np.argmax(amp[k]))
        sort[m] = k
        amp[k, :] = 0
        amp[:, m] = 0
    emit = np.zeros(3)
    for ii, (p, q) in enumerate(pairs):
        emit[sort[ii]] = abs(w[p].imag)
    return emit


def bunch_data(vec, t, state, p0c, mass):
    """Dict of the bunch data fields (same names as lib.BunchData)."""
    alive = state == 1
    n = int(np.sum(alive))
    out = dict(n_live=n, p0c=p0c)
    if n == 0:
        return out
    v = vec[:, alive]
    tt = t[alive] if t is not None else np.zeros(n)
    avg = v.sum(axis=1) / n
    out["centroid"] = avg
    out["t"] = tt.sum() / n
    out["sigma_t"] = np.sqrt(max(0.0, (tt * tt).sum() / n - out["t"] ** 2))
    d = v - avg[:, None]
    sig = (d @ d.T) / n
    out["sigma"] = sig
    f_emit = p0c * (1 + avg[5]) / mass
    pe, pb, pa = np.zeros(3), np.zeros(3), np.zeros(3)
    eta, etap = np.zeros(2), np.zeros(2)
    for p, (i, j, xd, pxd) in enumerate([(0, 1, sig[0, 5], sig[1, 5]), (2, 3, sig[2, 5], sig[3, 5]),
                                          (4, 5, 0.0, 0.0)]):
        x2, px2, xpx = sig[i, i], sig[j, j], sig[i, j]
        if sig[5, 5] != 0:
            if p < 2:
                eta[p], etap[p] = xd / sig[5, 5], pxd / sig[5, 5]
            x2, xpx, px2 = x2 - xd ** 2 / sig[5, 5], xpx - xd * pxd / sig[5, 5], px2 - pxd ** 2 / sig[5, 5]
        e = np.sqrt(max(0.0, x2 * px2 - xpx ** 2))
        pe[p] = e
        if e != 0:
            pa[p], pb[p] = -xpx / e, x2 / e
    out.update(proj_emit=pe, proj_beta=pb, proj_alpha=pa, eta=eta, etap=etap)
    if n >= 6:
        S = np.zeros((6, 6))
        for k in range(3):
            S[2 * k + 1, 2 * k] = -1
            S[2 * k, 2 * k + 1] = 1
        ss = sig @ S
        cut = 1e-20 * np.max(np.abs(sig))
        dim = 4 if (abs(sig[4, 4]) < cut or abs(sig[5, 5]) < cut) else 6
        out["emit"] = mat_eigen_emittances(ss[:dim, :dim])
        out["norm_emit"] = out["emit"] * f_emit
    if n < 10:
        return out
    s_sum = v.sum(axis=1)
    sv, sig1 = [], np.zeros(6)
    for i in range(6):
        for j in range(i, 6):
            x = np.sum(v[i] * v[j]) / n - s_sum[i] * s_sum[j] / n ** 2
            if abs(x) < 1e-15 * abs(s_sum[i] * s_sum[j]) / n:
                x = 0.0
            sv.append(x)
            if i == j:
                sig1[i] = np.sqrt(max(0.0, x))
    out["sigma_vec"] = np.array(sv)
    out["sig1"] = sig1
    skew, kurt = np.zeros(3), np.zeros(3)
    for p, i in enumerate((0, 2, 4)):
        if sig1[i] != 0:
            ave = s_sum[i] / n
            skew[p] = np.sum((v[i] - ave) ** 3) / (n * sig1[i] ** 3)
            kurt[p] = np.sum((v[i] - ave) ** 4) / (n * sig1[i] ** 4) - 3.0
    out.update(skew=skew, kurt=kurt)
    return out


def read_table(path):
    """Rows of numbers of an LTT output file (comment lines start with '#')."""
    rows = []
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        rows.append(line.split())
    return rows


def beam_fraction(x):
    """ltt_beam_fraction (lt_tracking_mod.f90:2566-2570)."""
    jc = -np.log(x)
    return 1.0 - x * (1 + jc + 0.5 * jc ** 2)


def core_emit(vec, t, state, p0c, mass, cutoff, combined=True):
    """Core emittances of ltt_calc_bunch_data (lt_tracking_mod.f90:2432-2560). Combined
    calculation: rank the live particles by sum_k (j_2k^2 + j_2k+1^2) / emit_k, j = N^-1 (p - c) --
    the quadratic form (p - c)^T Sigma^-1 (p - c) -- keep the int(cutoff n_live) smallest, rank again
    about the core, and scale the core's normal-mode emittances by f(cutoff). Per mode
    (combined=False): the same with each mode's action (j_2k^2 + j_2k+1^2) / 2 and N^-1 from
    normal_form_n, f = cutoff / (1 - (1 + s) e^-s), s = -ln(1 - cutoff)."""
    from scipy.optimize import brentq
    bd = bunch_data(vec, t, state, p0c, mass)
    if bd["n_live"] < 10 or "emit" not in bd or np.any(bd["emit"] == 0):
        return np.zeros(3)
    n_cut = int(cutoff * bd["n_live"])
    if n_cut == 0:
        return np.zeros(3)
    cut = min(1.0 - 1e-8, cutoff)
    alive = state == 1
    if not combined:
        s = -np.log(1 - cut)
        f = cut / (1 - (1 + s) * np.exp(-s))
        out = np.zeros(3)
        for m in range(3):
            def core_m(ref):
                n_inv = np.linalg.inv(normal_form_n(ref["sigma"])[1])
                j = n_inv @ (vec - np.asarray(ref["centroid"])[:, None])
                amp = 0.5 * (j[2 * m] ** 2 + j[2 * m + 1] ** 2)
                amp[~alive] = 1e100
                st = np.zeros_like(state)
                st[np.argsort(amp, kind="stable")[:n_cut]] = 1
                return bunch_data(vec, t, st, p0c, mass)
            out[m] = f * core_m(core_m(bd))["emit"][m]
        return out
    x = brentq(lambda u: beam_fraction(u) - cut, 1e-12, 1.0, xtol=1e-300, rtol=1e-15)
    s = -np.log(x)
    f = cut / (1 - (1 + s + s ** 2 / 2 + s ** 3 / 6) * np.exp(-s))

    def core(ref):
        d = vec - np.asarray(ref["centroid"])[:, None]
        amp = np.einsum("in,ij,jn->n", d, np.linalg.inv(ref["sigma"]), d)
        amp[~alive] = 1e100
        idx = np.argsort(amp, kind="stable")[:n_cut]
        st = np.zeros_like(state)
        st[idx] = 1
        return bunch_data(vec, t, st, p0c, mass)

    c1 = core(bd)
    c2 = core(c1)
    return f * np.asarray(c2["emit"])


def mat_eigen(mat):
    """mat_eigen (sim_utils/matrix/mat_eigen.f90:37-187) for a stable matrix: LAPACK geev (through
    numpy.linalg.eig), the greedy plane sort, the complex-conjugate pair layout, the flip that makes
    fnorm positive and the phase that makes each eigenvector's own-plane component real and
    positive. Returns (eigen_val[n], eigen_vec[n, n]) with eigenvectors as rows, 0-based."""
    n = mat.shape[0]
    nn = n // 2
    w, v = np.linalg.eig(mat)
    # geev's real layout: a pair (p, p+1) keeps Re and Im of the first (positive imaginary) vector
    vec = np.zeros((n, n))
    eval_r, eval_i = w.real.copy(), w.imag.copy()
    p = 0
    while p < n:
        if w[p].imag != 0:
            vec[:, p], vec[:, p + 1] = v[:, p].real, v[:, p].imag
            p += 2
        else:
            vec[:, p] = v[:, p].real
            p += 1
    amp = np.zeros((nn, nn))
    for ii in range(nn):
        for kk in range(nn):
            amp[kk, ii] = np.sum(vec[2 * kk:2 * kk + 2, 2 * ii:2 * ii + 2] ** 2)
        amp[:, ii] /= np.sum(amp[:, ii])
    sort = np.zeros(nn, int)
    for _ in range(nn):
        amp2 = amp.copy()
        dmax = np.zeros(nn)
        for j in range(nn):
            m = int(np.argmax(amp2[j]))
            amp2[j, m] = -1
            m2 = int(np.argmax(amp2[j]))
            dmax[j] = amp[j, m] - amp[j, m2]
        k = int(np.argmax(dmax))
        m = int(np.argmax(amp[k]))
        sort[m] = k
        amp[k, :] = 0
        amp[:, m] = 0
    eigen_val = np.zeros(n, complex)
    eigen_vec = np.zeros((n, n), complex)
    for ii in range(nn):
        i = 2 * ii + 1          # 0-based index of the Fortran i = 2 ii
        k = 2 * sort[ii]        # 0-based index of the Fortran j - 1
        if eval_i[i - 1] == 0:
            raise ValueError("unstable mode")
        eigen_val[k] = complex(eval_r[i], eval_i[i])
        eigen_val[k + 1] = complex(eval_r[i - 1], eval_i[i - 1])
        eigen_vec[k] = vec[:, i - 1] - 1j * vec[:, i]
        eigen_vec[k + 1] = vec[:, i - 1] + 1j * vec[:, i]
        fnorm = sum(2 * (np.conj(eigen_vec[k, jj]) * eigen_vec[k, jj + 1]).imag for jj in range(0, n, 2))
        if fnorm < 0:
            eigen_vec[[k, k + 1]] = eigen_vec[[k + 1, k]]
            eigen_val[[k, k + 1]] = eigen_val[[k + 1, k]]
            fnorm = -fnorm
        if abs(eigen_vec[k, k]) == 0:
            sgn = 1.0 / np.sqrt(fnorm)
        else:
            sgn = abs(eigen_vec[k, k]) / (np.sqrt(fnorm) * eigen_vec[k, k])
        eigen_vec[k] = sgn * eigen_vec[k]
        eigen_vec[k + 1] = np.conj(sgn) * eigen_vec[k + 1]
    return eigen_val, eigen_vec


# Wolski's Q of calc_emittances_and_twiss_from_sigma_matrix (beam_utils.f90:1533-1545): the real
# entries are the default-real (single precision) expression 1.0/sqrt(2.0), the imaginary ones
# i_imag / sqrt(2.0) with the single-precision square root widened.
Q_RE = float(np.float32(1.0) / np.sqrt(np.float32(2.0)))
Q_IM = 1.0 / float(np.sqrt(np.float32(2.0)))


def normal_form_n(sigma):
    """(emit[3], n_mat[6, 6]) of calc_emittances_and_twiss_from_sigma_matrix (beam_utils.f90:
    1495-1551): eigen-decomposition of sigma.S by mat_eigen, normalize_e (:1639-1688), N = E Q
    (Wolski Eq. 44). Only the 6-dimensional case (non-zero longitudinal spread)."""
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1, -1
    ev, e = mat_eigen(sigma @ S)
    for i2 in range(3):
        i = 2 * i2
        e[i] = np.conj(e[i + 1])
        temp = S @ e[i + 1]
        wronsk = np.sum(e[i] * temp)
        factor = np.sqrt(1j) / np.sqrt(wronsk)
        e[i + 1] = e[i + 1] * factor
        e[i] = np.conj(e[i + 1])
    emit = np.array([ev[0].imag, ev[2].imag, ev[4].imag])
    E = e.T
    q = np.zeros((6, 6), complex)
    for k in range(3):
        q[2 * k, 2 * k] = q[2 * k + 1, 2 * k] = Q_RE
        q[2 * k, 2 * k + 1] = 1j * Q_IM
        q[2 * k + 1, 2 * k + 1] = -1j * Q_IM
    return emit, (E @ q).real


def action_angle(vec, t, state, p0c, mass):
    """[6, n] = J_a, angle_a, J_b, angle_b, J_c, angle_c of write_this_data's action-angle file
    (lt_tracking_mod.f90:2024-2045): j = N^-1 (p - centroid) with N of the bunch (zero where
    calc_bunch_params fails), J = (j_2k^2 + j_2k+1^2) / 2, angle = atan2(j_2k+1, j_2k)."""
    bd = bunch_data(vec, t, state, p0c, mass)
    n_inv = np.zeros((6, 6))
    if bd["n_live"] >= 6 and "emit" in bd:
        n_inv = np.linalg.inv(normal_form_n(bd["sigma"])[1])
    c = np.asarray(bd.get("centroid", np.zeros(6)))
    j = n_inv @ (vec - c[:, None])
    out = np.zeros((6, vec.shape[1]))
    for m in range(3):
        out[2 * m] = 0.5 * (j[2 * m] ** 2 + j[2 * m + 1] ** 2)
        out[2 * m + 1] = np.arctan2(j[2 * m + 1], j[2 * m])
    return out
