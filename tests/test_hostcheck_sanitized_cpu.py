"""The device element code compiled for the host with AddressSanitizer and UBSan (the default and the
correctly rounded builds), run through every host-build check (tests/test_hostcheck_cpu.py: single
elements, rings with every element form, losses, NaN and infinite coordinates): no access outside
the element table, the multipole and function tables or the particle arrays, and no undefined
integer arithmetic, on the inputs those checks use. The oracle, built the same way, runs under them
as the checker, and through the reference's golden vectors (tests/test_oracle_golden.py)."""
import os
import shutil
import subprocess
import sys

import pytest

from conftest import ROOT


def test_host_build_under_sanitizers(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    csrc = os.path.join(ROOT, "bmad-ecosystem_b200", "csrc")
    san = ["-O1", "-g", "-std=c++17", "-fPIC", "-shared", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined"]
    lib = str(tmp_path / "libbmadgpu_hostcheck_san.so")
    lib_cr = str(tmp_path / "libbmadgpu_hostcheck_cr_san.so")
    for out, extra, src in ((lib, [], "hostcheck.cpp"),
                            (lib_cr, ["-mfma", "-ffp-contract=off", "-DBG_CR_MATH"], "hostcheck_cr.cpp")):
        build = subprocess.run([gxx] + san + extra + ["-o", out, os.path.join(csrc, src), os.path.join(csrc, "lattice.cpp")],
                               capture_output=True, text=True)
        assert build.returncode == 0, build.stderr[-2000:]
    oracle = str(tmp_path / "liboracle_san.so")
    build = subprocess.run([gxx, "-O1", "-g", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-fopenmp", "-std=c++17",
                            "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
                            "-I" + os.path.join(ROOT, "include"), "-shared", "-o", oracle,
                            os.path.join(ROOT, "oracle", "bmad_oracle.cpp"), "-lquadmath"], capture_output=True, text=True)
    assert build.returncode == 0, build.stderr[-2000:]
    runtimes = [subprocess.run([gxx, "-print-file-name=lib%s.so" % r], capture_output=True, text=True).stdout.strip()
                for r in ("asan", "ubsan")]
    if not all(os.path.isabs(r) and os.path.exists(r) for r in runtimes):
        pytest.skip("no sanitizer runtime")
    env = dict(os.environ, BMADGPU_HOSTCHECK_LIB=lib, BMADGPU_HOSTCHECK_CR_LIB=lib_cr, BMADGPU_ORACLE_LIB=oracle,
               LD_PRELOAD=" ".join(runtimes),
               ASAN_OPTIONS="detect_leaks=0", UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider", "-m", "not gpu",
                          os.path.join(ROOT, "tests", "test_hostcheck_cpu.py"),
                          os.path.join(ROOT, "tests", "test_oracle_golden.py")],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert run.returncode == 0, (run.stdout[-3000:], run.stderr[-3000:])
    assert " passed" in run.stdout
