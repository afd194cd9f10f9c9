"""The allocation-free tracking entry point, bmadgpu_track_bunch_device_noalloc.

Callers that cannot call cudaMalloc while tracking -- programs whose own pool allocator holds
the GPU's memory, or loops that may not stall on an allocation -- use this entry point; its scratch (the
live-particle lists of loss compaction) is a fixed array inside the library. This file checks,
through the C-ABI, that it gives the same result as bmadgpu_track_bunch_device with the same
compaction schedule, on two calls in a row (the second call finds the first call's leftovers in
the shared array). It is collected last so a failure here comes after every other test ran.
"""
import ctypes
import importlib

import numpy as np
import pytest

from conftest import load_abi

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


def _device_bunch(torch, hb):
    keys = ("vec", "beta", "state", "ix_ele", "ix_turn", "location")
    d = {k: torch.from_numpy(getattr(hb, k)).cuda() for k in keys}
    torch.cuda.synchronize()
    view = abi.Bunch(hb.n, d["vec"].data_ptr(), d["beta"].data_ptr(), None, d["state"].data_ptr(),
                     d["ix_ele"].data_ptr(), d["ix_turn"].data_ptr(), d["location"].data_ptr())
    return d, view


def test_noalloc_matches_allocating_entry_point_twice_in_a_row():
    torch = pytest.importorskip("torch")
    so = lib.load()
    so.bmadgpu_track_bunch_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(abi.Bunch),
                                                     ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    so.bmadgpu_track_bunch_device_noalloc.restype = ctypes.c_int
    ctx = lib.Context(0)
    eles, p = rings.ring(50)
    lat = lib.Lattice(ctx, eles, p)
    hb = lib.HostBunch.from_vec(rings.matched_gaussian(eles, 30000, seed=21, scale=10.0), p)
    ref, ref_v = _device_bunch(torch, hb)
    new, new_v = _device_bunch(torch, hb)
    ctx.set_tuning(turns_per_launch=4, compact=1)
    for call in range(2):
        turn0 = 10 * call
        lib.check(so.bmadgpu_track_bunch_device(ctx.handle, lat.handle, ctypes.byref(ref_v), 0, lat.n_ele, turn0, 10,
                                                None))
        lib.check(so.bmadgpu_track_bunch_device_noalloc(ctx.handle, lat.handle, ctypes.byref(new_v), turn0, 10, 4))
        ctx.synchronize()
        st_ref, st_new = ref["state"].cpu().numpy(), new["state"].cpu().numpy()
        assert (st_ref != abi.ALIVE).sum() > 0        # losses happen, so compaction is exercised
        assert np.array_equal(st_new, st_ref)
        for k in ("ix_ele", "ix_turn", "location"):
            assert np.array_equal(new[k].cpu().numpy(), ref[k].cpu().numpy()), k
        # the same kernels on the same inputs: the same bits
        assert np.array_equal(new["vec"].cpu().numpy(), ref["vec"].cpu().numpy())
        assert np.array_equal(new["beta"].cpu().numpy(), ref["beta"].cpu().numpy())
    lib.check(so.bmadgpu_ctx_synchronize(ctx.handle))      # no staging time-out was left pending
    ctx.set_tuning(turns_per_launch=0, compact=0)


def test_noalloc_rejects_bunches_above_the_limit():
    so = lib.load()
    so.bmadgpu_track_bunch_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(abi.Bunch),
                                                     ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    ctx = lib.Context(0)
    eles, p = rings.ring(50)
    lat = lib.Lattice(ctx, eles, p)
    big = abi.Bunch(262144 + 1, None, None, None, None, None, None, None)   # rejected before any use
    r = so.bmadgpu_track_bunch_device_noalloc(ctx.handle, lat.handle, ctypes.byref(big), 0, 1, 0)
    assert r == abi.EINVAL
    assert b"BMADGPU_NOALLOC_MAX_PARTICLES" in so.bmadgpu_last_error()
