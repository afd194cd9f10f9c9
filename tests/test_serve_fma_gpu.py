"""Frequency-map jobs in the server (bmadgpu_server_submit_fma): the per-turn record happens
inside the served rounds, the tunes when the job completes. A served job's tunes and statuses
equal the standalone frequency map (bmadgpu_fma) bit for bit, alone and mixed with bunch jobs and
other frequency-map jobs of other lattices and turn counts submitted while they run; the bunch
jobs in the mix equal their results alone."""
import importlib

import numpy as np
import pytest

from conftest import load_abi

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def grid(n_x, n_y, x_max, y_max, pz=(0.0, 0.002)):
    return np.array([[x_max * (ix + 1) / n_x, 0, y_max * (iy + 1) / n_y, 0, 0, d]
                     for d in pz for iy in range(n_y) for ix in range(n_x)])


def fma_job(ctx, n_cells, seed, n_turns, fft_turns, n_x=6, n_y=5):
    eles, p = rings.perturbed_ring(n_cells, seed=seed)
    lat = lib.Lattice(ctx, eles, p)
    orbit, norm, tunes = lib.fma_setup(ctx, lat)
    off = grid(n_x, n_y, 0.011, 0.005)
    alone = lib.fma(ctx, lat, off, n_turns, fft_turns=fft_turns, orbit=orbit, norm=norm, tunes=tunes)
    vec = (orbit[None, :] + off).T
    return dict(lat=lat, p=p, vec=vec, n_turns=n_turns, fft_turns=fft_turns, orbit=orbit, norm=norm, tunes=tunes,
                alone=alone)


def submit(srv, j):
    b = lib.PinnedBunch(j["vec"], np.zeros(j["vec"].shape[1]))
    pc = j["p"].p0c * (1 + b.vec[5])
    b.beta[:] = np.where(b.vec[5] == 0, j["p"].p0c / j["p"].e_tot, pc / np.sqrt(pc * pc + j["p"].mass ** 2))
    return srv.submit_fma(j["lat"], b, j["n_turns"], j["norm"], j["orbit"], j["tunes"], fft_turns=j["fft_turns"])


def same(got, want):
    q, st, tl, ie = got
    qa, sta, tla, iea = want
    assert np.array_equal(st, sta)
    ok = st == 0
    assert np.array_equal(q[ok], qa[ok])
    assert np.array_equal(tl[~ok], tla[~ok])
    assert np.array_equal(ie[st == 1], iea[st == 1])


def test_served_fma_alone(ctx):
    j = fma_job(ctx, 20, 5, 200, 0)
    srv = lib.Server(ctx, record_mib=256, element_steps=4096)
    jid = submit(srv, j)
    srv.wait(jid, 600)
    same(srv.fma_result(jid), j["alone"])
    assert np.sum(srv.fma_result(jid)[1] == 0) > 0
    srv.close()


def test_served_fma_in_the_mix(ctx):
    jobs = [fma_job(ctx, 20, 5, 200, 0), fma_job(ctx, 12, 9, 131, 64, n_x=4, n_y=3),
            fma_job(ctx, 30, 2, 96, 48, n_x=3, n_y=7)]
    # bunch jobs of other rings, run alone through the plain path for reference
    bunch_specs = [(10, 3, 3000, 37), (25, 4, 500, 80)]
    ref = []
    for n_cells, seed, n, turns in bunch_specs:
        eles, p = rings.perturbed_ring(n_cells, seed=seed)
        lat = lib.Lattice(ctx, eles, p)
        vec = rings.matched_gaussian(eles, n, seed=seed, scale=2.0)
        srv1 = lib.Server(ctx, record_mib=16)
        b1 = lib.PinnedBunch(vec, np.zeros(n))
        b1.beta[:] = lib.HostBunch.from_vec(vec, p).beta
        srv1.wait(srv1.submit(lat, b1, turns), 600)
        srv1.close()
        ref.append((lat, p, vec, turns, np.array(b1.vec), np.array(b1.state)))
    srv = lib.Server(ctx, record_mib=512, element_steps=2048, max_particles=4000)
    ids, bunches = [], []
    for k in range(3):
        ids.append(("fma", k, submit(srv, jobs[k])))
        lat, p, vec, turns, _, _ = ref[k % 2]
        b = lib.PinnedBunch(vec, np.zeros(vec.shape[1]))
        b.beta[:] = lib.HostBunch.from_vec(vec, p).beta
        bunches.append(b)
        ids.append(("bunch", k % 2, srv.submit(lat, b, turns)))
    srv.wait(-1, 900)
    nb = 0
    for kind, k, jid in ids:
        if kind == "fma":
            same(srv.fma_result(jid), jobs[k]["alone"])
        else:
            b = bunches[nb]
            nb += 1
            assert np.array_equal(np.array(b.vec), ref[k][4])
            assert np.array_equal(np.array(b.state), ref[k][5])
    assert srv.stats()["jobs_done"] == 6
    srv.close()


def test_fma_record_too_large_refused(ctx):
    j = fma_job(ctx, 10, 1, 64, 0, n_x=2, n_y=2)
    srv = lib.Server(ctx, record_mib=1)
    vec = np.repeat(j["vec"], 1000, axis=1)  # 8000 particles x 64 turns x 48 B > 1 MiB
    b = lib.PinnedBunch(vec, np.ones(vec.shape[1]))
    with pytest.raises(lib.BmadGpuError):
        srv.submit_fma(j["lat"], b, 64, j["norm"], j["orbit"], j["tunes"])
    srv.close()
