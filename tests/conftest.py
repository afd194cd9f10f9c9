"""Shared fixtures: the package under test, the CPU oracle (checker only) and the GPU marker."""
import ctypes
import importlib
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    return importlib.import_module("bmad-ecosystem_b200")


def load_abi():
    return importlib.import_module("bmad-ecosystem_b200.abi")


_ORACLE = None


def load_oracle():
    """The CPU oracle shared library (built from oracle/ by its Makefile; BMADGPU_ORACLE_LIB names
    another build of the same source, as the sanitizer test does)."""
    global _ORACLE
    if _ORACLE is None:
        path = os.environ.get("BMADGPU_ORACLE_LIB") or os.path.join(ROOT, "oracle", "_build", "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        lib = ctypes.CDLL(path)
        abi = load_abi()
        P = ctypes.POINTER
        lib.oracle_track1.argtypes = [ctypes.c_void_p, P(abi.Element), ctypes.c_int32, P(abi.Param)]
        lib.oracle_init_coord.argtypes = [ctypes.c_void_p, P(ctypes.c_double), P(abi.Param)]
        lib.oracle_hwang_bend_edge_kick.argtypes = [P(abi.Element), P(abi.Param), ctypes.c_int32,
                                                    ctypes.c_void_p, P(ctypes.c_double)]
        lib.oracle_element_num_steps.argtypes = [P(abi.Element), P(abi.Param)]
        lib.oracle_element_num_steps.restype = ctypes.c_int32
        lib.oracle_track_ring.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), P(abi.Bunch),
                                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          P(ctypes.c_double)]
        lib.oracle_max_threads.restype = ctypes.c_int32
        _ORACLE = lib
    return _ORACLE


class OracleCoord(ctypes.Structure):
    """Mirror of oracle_coord (oracle/bmad_oracle.h)."""
    _fields_ = [("vec", ctypes.c_double * 6), ("beta", ctypes.c_double), ("p0c", ctypes.c_double),
                ("s", ctypes.c_double), ("t", ctypes.c_double), ("phase1", ctypes.c_double),
                ("state", ctypes.c_int32), ("location", ctypes.c_int32), ("ix_ele", ctypes.c_int32),
                ("direction", ctypes.c_int32), ("time_dir", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("t_qp", ctypes.c_ubyte * 16)]


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def abi():
    return load_abi()


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()
