"""The Fortran shim's marshalling (fortran/bmadgpu_mod.f90, track_on_gpu), restated in C
(tests/c/shim_marshal.c) and run through the C-ABI: coord records gathered into the shim's
column-major vec(n,6) buffer, tracked, scattered back with the shim's bookkeeping. The result
must equal the same tracking through the Python binding's SoA buffers bit for bit, with lost
particles' ix_ele (1-based), ix_turn and location, and survivors' ix_ele = ix_end and location
downstream_end, as track1 leaves them (bmad/code/track1.f90:92, 296-304)."""
import ctypes
import importlib
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_abi

lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()

REC = np.dtype([("vec", "<f8", 6), ("beta", "<f8"), ("t", "<f8"), ("state", "<i4"), ("ix_ele", "<i4"),
                ("ix_turn", "<i4"), ("location", "<i4")])
SRC = os.path.join(ROOT, "tests", "c", "shim_marshal.c")


def build(tmp_path, libname="bmadgpu"):
    exe = str(tmp_path / ("shim_marshal_" + libname))
    libdir = os.path.join(ROOT, "bmad-ecosystem_b200", "lib")
    subprocess.check_call(["gcc", "-O2", "-std=c11", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", exe, SRC,
                           "-L", libdir, "-l" + libname, "-Wl,-rpath," + libdir])
    return exe


def test_marshalling_program_builds_against_both_libraries(tmp_path):
    for name in ("bmadgpu", "bmadgpu_cr"):
        assert os.path.exists(build(tmp_path, name))


@pytest.mark.gpu
@pytest.mark.parametrize("span", ["ring", "one_element"])
def test_shim_marshalling_round_trip(tmp_path, span):
    exe = build(tmp_path)
    eles, p = rings.ring(50)
    # wide enough that particles are lost in the call: 12 sigma over 20 turns, 180 sigma in one bend
    vec = rings.matched_gaussian(eles, 5000, seed=8, scale=12.0 if span == "ring" else 180.0)
    n = vec.shape[1]
    if span == "ring":
        ix_start, ix_end, turn0, n_turns = 0, len(eles), 7, 20
    else:
        ix_start, ix_end, turn0, n_turns = 3, 4, 2, 1      # the per-element hook: sbend of cell 0
    hb = lib.HostBunch.from_vec(vec, p)
    rec = np.zeros(n, REC)
    rec["vec"] = vec.T
    rec["beta"] = hb.beta
    rec["state"] = abi.ALIVE
    rec["ix_ele"] = -7
    rec["ix_turn"] = -7
    arr = abi.element_array(eles)
    (tmp_path / "e.bin").write_bytes(bytes(arr))
    (tmp_path / "p.bin").write_bytes(bytes(p))
    rec.tofile(str(tmp_path / "r.bin"))
    subprocess.check_call([exe, str(tmp_path / "e.bin"), str(tmp_path / "p.bin"), str(tmp_path / "r.bin"), str(n),
                           str(ix_start), str(ix_end), str(turn0), str(n_turns), str(tmp_path / "o.bin")])
    out = np.fromfile(str(tmp_path / "o.bin"), REC)
    ctx = lib.Context(0)
    lat = lib.Lattice(ctx, eles, p)
    ref = lib.HostBunch.from_vec(vec, p)
    lib.track_bunch(ctx, lat, ref, n_turns=n_turns, ix_start=ix_start, ix_end=ix_end, turn0=turn0)
    assert np.array_equal(out["vec"].T, ref.vec)
    assert np.array_equal(out["beta"], ref.beta)
    assert np.array_equal(out["state"], ref.state)
    lost = ref.state != abi.ALIVE
    assert lost.sum() > 10
    assert np.array_equal(out["ix_ele"][lost], ref.ix_ele[lost] + 1)
    assert np.array_equal(out["ix_turn"][lost], ref.ix_turn[lost])
    assert np.all((out["ix_turn"][lost] >= turn0) & (out["ix_turn"][lost] < turn0 + n_turns))
    assert np.array_equal(out["location"][lost], ref.location[lost])
    assert np.all(out["ix_ele"][~lost] == ix_end)
    assert np.all(out["location"][~lost] == abi.DOWNSTREAM_END)
    lat.close()
    ctx.close()
