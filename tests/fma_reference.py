"""numpy restatement of frequency_map's per-particle tune calculation (test infrastructure, the
checker): bsim/frequency_map/frequency_map.f90:280-375 -- turn-by-turn tracking on the ORACLE,
normalisation psv_norm = norm (vec - co), Hanning window 2 sin^2(pi j / N), FFTW_BACKWARD spectra
(numpy's ifft times N), calc_tune's interpolated peak and the 1 - Q flip."""
import ctypes

import numpy as np

from conftest import load_abi, load_oracle

abi = load_abi()


def calc_tune(rft):
    """frequency_map.f90:364-375 (iQ is 1-based; the neighbour past the last bin counts as 0)."""
    N = len(rft)
    iq = 1
    for k in range(2, N + 1):
        if rft[iq - 1] < rft[k - 1]:
            iq = k
    d = rft[iq - 1]
    b = rft[iq] if iq < N else 0.0
    c = np.cos(2 * np.pi / N)
    A = (-(d + b * c) * (d - b) + b * np.sqrt(c * c * (d + b) * (d + b) - 2 * d * b * (2 * c * c - c - 1))) / \
        (d * d + b * b + 2 * d * b * c)
    return iq / N + (1.0 / (2 * np.pi)) * np.arcsin(A * np.sin(2 * np.pi / N))


def record(elements, param, start, n_turn, norm, co, z_limit):
    """Normalised coordinates per turn [n_turn, 6, n] and the per-particle status (0 ok, 1 lost,
    2 outside the bucket), tracking with the oracle one turn at a time."""
    lib = load_oracle()
    arr = abi.element_array(elements)
    vec = np.ascontiguousarray(start, dtype=np.float64).copy()
    n = vec.shape[1]
    pc = param.p0c * (1 + vec[5])
    beta = np.ascontiguousarray(np.where(vec[5] == 0, param.p0c / param.e_tot,
                                         pc / np.sqrt(pc * pc + param.mass * param.mass)))
    state = np.full(n, abi.ALIVE, np.int32)
    ix_ele = np.full(n, -1, np.int32)
    ix_turn = np.full(n, -1, np.int32)
    loc = np.zeros(n, np.int32)
    t = np.zeros(n)
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, t.ctypes.data, state.ctypes.data, ix_ele.ctypes.data,
                  ix_turn.ctypes.data, loc.ctypes.data)
    hist = np.zeros((n_turn, 6, n))
    status = np.zeros(n, np.int32)
    for j in range(n_turn):
        assert lib.oracle_track_ring(arr, len(arr), ctypes.byref(param), ctypes.byref(b), j, 1, 0, None) == 0
        psv = vec - np.asarray(co, float)[:, None]
        for i in range(n):
            if status[i]:
                continue
            if state[i] != abi.ALIVE:
                status[i] = 1
            elif z_limit > 0 and abs(psv[4, i]) > z_limit:
                status[i] = 2
            elif z_limit > 0 and j == n_turn - 1 and not abs(vec[4, i]) < z_limit:
                status[i] = 2
        hist[j] = np.asarray(norm, float) @ psv
    return hist, status


def tunes(hist, N, flip_a, flip_b):
    """[n, 6] tunes (x, y, z of the first N turns, then of the last N turns)."""
    n_turn, _, n = hist.shape
    j = np.arange(1, N + 1)
    hann = 2 * np.sin(np.pi * j / N) ** 2
    out = np.zeros((n, 6))
    for p in range(n):
        for half, j0 in ((0, 0), (1, n_turn - N)):
            h = hist[j0:j0 + N, :, p]
            for plane, sig in enumerate((h[:, 0] + 1j * h[:, 1], h[:, 2] + 1j * h[:, 3], h[:, 4] - 1j * h[:, 5])):
                spec = np.abs(np.fft.ifft(sig * hann) * N)
                q = calc_tune(spec)
                if (plane == 0 and flip_a) or (plane == 1 and flip_b):
                    q = 1.0 - q
                out[p, 3 * half + plane] = q
    return out
