"""numpy restatement of NAFF (test infrastructure, for checking the device path): sim_utils/math/naff.f90:72-131
(naff), :140-150 (projdd, ed), :160-205 (maximize_projection with a Hanning window), :230-290
(interpolated_fft_gsl: Gaussian window r = 8, FFT backward, log-parabola peak interpolation).

The maximiser is Brent's method (R. P. Brent, Algorithms for Minimization without Derivatives,
1973, ch. 5) from a golden-ratio bracket around the interpolated-FFT estimate, to the reference's
tolerances (rel 1e-8, abs 1e-15); `polish` refines further to the maximiser itself."""
import math

import numpy as np

GOLD = (1 + math.sqrt(5)) / 2
CGOLD = (3 - math.sqrt(5)) / 2


def ed(f, n):
    return np.exp(-2j * np.pi * f * np.arange(n))


def projdd(a, b):
    return np.sum(np.conj(a) * b) / len(a)


def interpolated_fft(cdata):
    n = len(cdata)
    h = (n - 1) / 2.0
    i = np.arange(1, n + 1)
    w = np.exp(-0.5 * (8.0 * (i - h - 1.0) / (n - 1.0)) ** 2)
    amp = np.abs(np.fft.ifft(cdata * w) * n)
    k = int(np.argmax(amp[1:n - 1])) + 1          # 0-based; the reference's maxloc over 2..n-1
    if amp[k] == 0:
        return None
    lk, lkm, lkp = np.log(amp[k]), np.log(amp[k - 1]), np.log(amp[k + 1])
    den = 2.0 * lk - lkp - lkm
    if den == 0:
        return None
    return (k + (lkp - lkm) / 2.0 / den) / n


def bracket(g, a, b, it_max=200):
    fa, fb = g(a), g(b)
    if fb > fa:
        a, b, fa, fb = b, a, fb, fa
    c = b + GOLD * (b - a)
    fc = g(c)
    for _ in range(it_max):
        if fc >= fb:
            break
        a, b, fa, fb = b, c, fb, fc
        c = b + GOLD * (b - a)
        fc = g(c)
    return a, b, c


def brent(g, a, b, c, rel_tol, abs_tol, it_max=100):
    lo, hi = min(a, c), max(a, c)
    x = w = v = b
    fx = fw = fv = g(x)
    d = e = 0.0
    for _ in range(it_max):
        mid = 0.5 * (lo + hi)
        tol1 = rel_tol * abs(x) + abs_tol
        tol2 = 2.0 * tol1
        if abs(x - mid) <= tol2 - 0.5 * (hi - lo):
            break
        golden = True
        if abs(e) > tol1:
            r = (x - w) * (fx - fv)
            q = (x - v) * (fx - fw)
            p = (x - v) * q - (x - w) * r
            q = 2.0 * (q - r)
            if q > 0:
                p = -p
            q = abs(q)
            e_old, e = e, d
            if abs(p) < abs(0.5 * q * e_old) and q * (lo - x) < p < q * (hi - x):
                d = p / q
                u = x + d
                if u - lo < tol2 or hi - u < tol2:
                    d = math.copysign(tol1, mid - x)
                golden = False
        if golden:
            e = (lo - x) if x >= mid else (hi - x)
            d = CGOLD * e
        u = x + d if abs(d) >= tol1 else x + math.copysign(tol1, d)
        fu = g(u)
        if fu <= fx:
            if u >= x:
                lo = x
            else:
                hi = x
            v, w, x = w, x, u
            fv, fw, fx = fw, fx, fu
        else:
            if u < x:
                lo = u
            else:
                hi = u
            if fu <= fw or w == x:
                v, w, fv, fw = w, u, fw, fu
            elif fu <= fv or v == x or v == w:
                v, fv = u, fu
    return x


def maximize_projection(seed, cdata, polish=False):
    n = len(cdata)
    h = (n - 1) / 2.0
    i = np.arange(1, n + 1)
    wc = cdata * (0.5 * (1.0 + np.cos(2 * np.pi * (i - h - 1) / (n - 1))))

    def g(f):
        return -abs(projdd(wc, ed(f, n)))

    a, b, c = bracket(g, seed, seed + 0.1 / n)
    x = brent(g, a, b, c, 1e-8, 1e-15)
    if polish:
        x = brent(g, x - 1e-6 / n, x, x + 1e-6 / n, 1e-15, 1e-18)
    return x


def naff(cdata, n_comp, zero_first=False, polish=False, freqs_in=None):
    """(freqs, amps) as naff() returns them. freqs_in: use these frequencies instead of searching
    (to compare the Gram-Schmidt amplitudes at another implementation's frequencies)."""
    cdata = np.array(cdata, complex)
    n = len(cdata)
    freqs = -np.ones(n_comp)
    amps = np.zeros(n_comp, complex)
    if np.all(cdata == cdata[0]):
        return np.zeros(n_comp), amps
    u = np.zeros((n_comp, n), complex)
    for i in range(n_comp):
        if freqs_in is not None:
            freqs[i] = freqs_in[i]
        elif i == 0 and zero_first:
            freqs[i] = 0.0
        else:
            f = interpolated_fft(cdata)
            if f is None:
                return freqs, amps
            freqs[i] = maximize_projection(f, cdata, polish)
        u[i] = ed(freqs[i], n)
        for j in range(1, i + 1):
            u[i] = u[i] - projdd(u[j - 1], u[i]) * u[j - 1]
        amps[i] = projdd(u[i], cdata)
        cdata = cdata - amps[i] * u[i]
    return freqs, amps
