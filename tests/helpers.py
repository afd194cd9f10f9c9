"""Test helpers: run the same bunch through the CPU oracle (checker) and compare results."""
import ctypes

import numpy as np

from conftest import load_abi, load_oracle


def oracle_track(elements, param, vec, n_turns, n_threads=0, moments=False, t=None):
    """Track vec[6, n] through the element list with the oracle. Returns a dict of arrays."""
    abi, lib = load_abi(), load_oracle()
    arr = abi.element_array(elements) if not isinstance(elements, ctypes.Array) else elements
    vec = np.ascontiguousarray(vec, dtype=np.float64).copy()
    n = vec.shape[1]
    pc = param.p0c * (1 + vec[5])
    beta = np.where(vec[5] == 0, param.p0c / param.e_tot, pc / np.sqrt(pc * pc + param.mass * param.mass))
    beta = np.ascontiguousarray(beta)
    state = np.full(n, abi.ALIVE, dtype=np.int32)
    ix_ele = np.full(n, -1, dtype=np.int32)
    ix_turn = np.full(n, -1, dtype=np.int32)
    loc = np.zeros(n, dtype=np.int32)
    tt = np.zeros(n) if t is None else np.ascontiguousarray(t, dtype=np.float64).copy()
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, tt.ctypes.data, state.ctypes.data, ix_ele.ctypes.data,
                  ix_turn.ctypes.data, loc.ctypes.data)
    mom = np.zeros((max(n_turns, 1), abi.N_MOMENTS)) if moments else None
    err = lib.oracle_track_ring(arr, len(arr), ctypes.byref(param), ctypes.byref(b), 0, n_turns, n_threads,
                                mom.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if moments else None)
    assert err == 0, err
    return dict(vec=vec, beta=beta, state=state, ix_ele=ix_ele, ix_turn=ix_turn, location=loc, t=tt, moments=mom)


def rel_err(got, want, floor):
    """Per-coordinate error relative to max(|want|, floor)."""
    return np.abs(got - want) / np.maximum(np.abs(want), floor)


def coord_floor(vec, frac=1.0):
    """Per-coordinate scale for relative errors: frac * RMS of the coordinate over the bunch.
    A coordinate passing near zero has no meaningful relative error of its own; its error is
    measured against the coordinate's spread in the bunch."""
    rms = np.sqrt(np.mean(vec * vec, axis=1))
    return np.maximum(frac * rms, 1e-30)[:, None]


_NOISE = None


def noise_track(elements, param, vec, n_turns):
    """Track with the host build of the device code whose transcendental results are moved by one
    ulp for about half of the calls (csrc/hostcheck_noise.cpp): the spread that 1-ulp libm
    differences alone produce, against which the GPU (CUDA libm vs glibc) is judged."""
    global _NOISE
    import os
    import subprocess
    from conftest import ROOT
    abi = load_abi()
    if _NOISE is None:
        path = os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_hostnoise.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"),
                                   "hostcheck-lib"])
        _NOISE = ctypes.CDLL(path)
    arr = abi.element_array(elements) if not isinstance(elements, ctypes.Array) else elements
    vec = np.array(vec, dtype=np.float64, copy=True)
    n = vec.shape[1]
    pc = param.p0c * (1 + vec[5])
    beta = np.ascontiguousarray(np.where(vec[5] == 0, param.p0c / param.e_tot,
                                         pc / np.sqrt(pc * pc + param.mass * param.mass)))
    state = np.full(n, abi.ALIVE, dtype=np.int32)
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, None, state.ctypes.data, None, None, None)
    assert _NOISE.bmadgpu_hostcheck_noise_track(arr, len(arr), ctypes.byref(param), ctypes.byref(b), n_turns) == 0
    return dict(vec=vec, beta=beta, state=state)


def per_particle_err(got, want):
    """Max over coordinates of the RMS-relative error, per particle."""
    return rel_err(got, want, coord_floor(want)).max(axis=0)


_CRLIB = None


def cr_libm(kind="cr"):
    """Addresses of the eight libm functions for oracle_set_libm: "cr", the correctly rounded functions
    the device maps use (host build of csrc/crmath.cuh); "quad", libquadmath's rounded once, an
    independent correctly rounded set."""
    global _CRLIB
    import os
    import subprocess
    from conftest import ROOT
    if _CRLIB is None:
        path = os.path.join(ROOT, "bmad-ecosystem_b200", "_build", "libbmadgpu_crmath.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"),
                                   "hostcheck-lib"])
        _CRLIB = ctypes.CDLL(path)
    pre = "bmadgpu_cr_" if kind == "cr" else "bmadgpu_q_"
    return [ctypes.cast(getattr(_CRLIB, pre + f), ctypes.c_void_p) for f in ("sin", "cos", "asin", "atan2", "sinh",
                                                                            "cosh", "exp", "tan")]


class oracle_libm:
    """Context manager: the oracle tracks with the given libm ("cr" or "quad"), then the host's."""

    def __init__(self, kind="cr"):
        self.kind = kind

    def __enter__(self):
        lib = load_oracle()
        lib.oracle_set_libm.argtypes = [ctypes.c_void_p] * 8
        lib.oracle_set_libm(*cr_libm(self.kind))
        return self

    def __exit__(self, *exc):
        lib = load_oracle()
        lib.oracle_set_libm(*([None] * 8))
        return False
