"""Long-term tracking outputs on the GPU (bmadgpu_bunch_stats, bmadgpu_ltt_run):

  - the device two-pass sums give the same bunch data as the numpy restatement of
    ltt_calc_bunch_data on the same particles;
  - ltt_run's averages files (.ave, .sigma, .emit) and phase-space files hold, at every output
    turn, what the oracle's tracking to that turn gives through the restated statistics, to the
    printed precision (es14.6 / es16.8), and the reference's column layout;
  - the stop conditions: with dead_cutoff, tracking ends at the first turn where the lost count
    reaches nint(dead_cutoff * n), as the reference's turn loop does, and no output is written for
    that turn;
  - core emittances (combined and per mode), the action-angle files and the per-particle files
    against the restatement on the oracle's tracking."""
import glob
import importlib
import os

import numpy as np
import pytest
import torch

from conftest import load_abi
from helpers import oracle_track
from ltt_reference import action_angle, bunch_data, core_emit, read_table

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def close(got, want, rel, what):
    got, want = np.asarray(got, float), np.asarray(want, float)
    scale = np.maximum(np.abs(want), 1e-300)
    assert np.all(np.abs(got - want) <= rel * scale + 1e-300), (what, got, want)


def test_device_stats_match_reference(ctx):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 50000, seed=11, scale=2.0)
    hb = lib.HostBunch.from_vec(vec, p, t=np.random.default_rng(1).normal(0, 1e-11, 50000))
    lat = lib.Lattice(ctx, eles, p)
    lib.track_bunch(ctx, lat, hb, n_turns=7)
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.array(getattr(hb, k))).to(dev) for k in ("vec", "beta", "t", "state")}
    view = abi.Bunch(hb.n, t["vec"].data_ptr(), t["beta"].data_ptr(), t["t"].data_ptr(), t["state"].data_ptr(),
                     None, None, None)
    got = lib.bunch_stats(ctx, lat, view)
    want = bunch_data(hb.vec, hb.t, hb.state, p.p0c, p.mass)
    assert got["n_live"] == want["n_live"]
    for k in ("centroid", "t", "sigma_t", "sigma_vec", "sig1", "skew", "kurt", "proj_emit", "emit"):
        w = np.asarray(want[k], float).ravel()
        g = np.asarray(got[k], float).ravel()
        assert np.allclose(g, w, rtol=1e-9, atol=1e-13 * np.max(np.abs(w))), (k, g, w)


def test_ltt_run_outputs_match_oracle(ctx, tmp_path):
    eles, p = rings.ring(50)
    n, n_turns = 3000, 20
    vec = rings.matched_gaussian(eles, n, seed=4, scale=4.0)
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(n))
    lat = lib.Lattice(ctx, eles, p)
    base = str(tmp_path / "run")
    done = lib.ltt_run(ctx, lat, hb, n_turns, averages_file=base, phase_space_file=str(tmp_path / "ps#.dat"),
                       averages_every_n_turns=5, particle_every_n_turns=10)
    assert done == n_turns
    ave, sig, emi = (read_table(base + ext) for ext in (".ave", ".sigma", ".emit"))
    turns = [int(r[0]) for r in ave]
    assert turns == [0, 5, 10, 15, 20]
    for line in open(base + ".sigma"):
        if line.startswith("##") and "Turn" in line:
            assert "<x.x>" in line and "<pz.pz>" in line
    heads = [line for line in open(base + ".emit") if line.startswith("##")]
    assert "50% Core" in heads[-2] and heads[-1].rstrip().endswith("Emit_c   |")
    for row_a, row_s, row_e in zip(ave, sig, emi):
        T = int(row_a[0])
        o = oracle_track(eles, p, vec, T, t=np.zeros(n)) if T > 0 else dict(
            vec=vec, t=np.zeros(n), state=np.ones(n, np.int32))
        w = bunch_data(o["vec"], o["t"], o["state"], p.p0c, p.mass)
        assert int(row_a[1]) == w["n_live"] == int(row_s[1]) == int(row_e[1])
        close([float(x) for x in row_a[7:13]], w["centroid"], 2e-6, "centroid T=%d" % T)
        close([float(x) for x in row_a[15:21]], w["sig1"], 2e-6, "sig1 T=%d" % T)
        close([float(x) for x in row_s[3:24]], w["sigma_vec"], 2e-6, "sigma T=%d" % T)
        close([float(x) for x in row_e[3:6]], w["emit"], 2e-6, "emit T=%d" % T)
        close([float(x) for x in row_e[6:9]], w["kurt"], 2e-5, "kurt T=%d" % T)
        assert len(row_e) == 15                       # the reference's default: one 50 % core group
        close([float(x) for x in row_e[12:15]], core_emit(o["vec"], o["t"], o["state"], p.p0c, p.mass, 0.5), 2e-6,
              "core emit T=%d" % T)
    files = sorted(glob.glob(str(tmp_path / "ps*.dat")))
    assert [os.path.basename(f) for f in files] == ["ps00.dat", "ps10.dat", "ps20.dat"]
    rows = read_table(str(tmp_path / "ps10.dat"))
    o = oracle_track(eles, p, vec, 10, t=np.zeros(n))
    alive = np.nonzero(o["state"] == abi.ALIVE)[0]
    assert [int(r[0]) - 1 for r in rows] == list(alive)          # only live particles, 1-based index
    assert all(int(r[1]) == 10 and r[-1] == "Alive" for r in rows)
    coords = np.array([[float(x) for x in r[2:8]] for r in rows]).T
    scale = np.sqrt(np.mean(o["vec"][:, alive] ** 2, axis=1))[:, None]
    assert np.max(np.abs(coords - o["vec"][:, alive]) / scale) < 1e-7


def test_dead_cutoff_stops_at_the_reference_turn(ctx, tmp_path):
    eles, p = rings.ring(50)
    n, n_turns = 4000, 40
    vec = rings.da_grid(n, r_max=0.02)
    o = oracle_track(eles, p, vec, n_turns)
    lost_turn = np.where(o["state"] != abi.ALIVE, o["ix_turn"], n_turns + 1)
    cutoff = 0.3
    limit = int(np.rint(cutoff * n))
    # after turn i the lost count is #(lost_turn <= i); the loop exits after the first such turn
    stop = next(i + 1 for i in range(n_turns) if np.sum(lost_turn <= i) >= limit)
    assert stop < n_turns
    hb = lib.HostBunch.from_vec(vec, p)
    lat = lib.Lattice(ctx, eles, p)
    base = str(tmp_path / "cut")
    done = lib.ltt_run(ctx, lat, hb, n_turns, averages_file=base, averages_every_n_turns=1, dead_cutoff=cutoff)
    assert done == stop
    turns = [int(r[0]) for r in read_table(base + ".ave")]
    assert turns == list(range(0, stop))            # nothing written for the stopping turn
    o2 = oracle_track(eles, p, vec, stop)
    assert np.array_equal(hb.state, o2["state"])
    assert np.array_equal(hb.ix_turn[hb.state != abi.ALIVE], o2["ix_turn"][o2["state"] != abi.ALIVE])
    # the same with outputs only at the end: the stop falls inside one long chunk, which is re-run
    # from its start for exactly the turns up to the stop
    hb2 = lib.HostBunch.from_vec(vec, p)
    done2 = lib.ltt_run(ctx, lat, hb2, n_turns, averages_file=str(tmp_path / "cut2"), dead_cutoff=cutoff)
    assert done2 == stop
    assert np.array_equal(hb2.vec, hb.vec) and np.array_equal(hb2.state, hb.state)
    assert read_table(str(tmp_path / "cut2.ave")) == []          # the last turn was never reached


def test_checkpoint_and_resume_continue_bit_for_bit(ctx, tmp_path):
    """Beam files every 8 turns (exact layout); resuming from the turn-16 file reaches the same
    final bunch as the uninterrupted run, bit for bit (the reference resumes LTT from a beam file
    with ix_turn_start the same way)."""
    eles, p = rings.ring(50)
    n, n_turns = 2000, 24
    vec = rings.matched_gaussian(eles, n, seed=8, scale=4.0)
    lat = lib.Lattice(ctx, eles, p)
    full = lib.HostBunch.from_vec(vec, p, t=np.zeros(n))
    assert lib.ltt_run(ctx, lat, full, n_turns, beam_file=str(tmp_path / "beam.dat"), beam_every_n_turns=8,
                       beam_exact=True) == n_turns
    names = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "beam-*.dat")))
    assert names == ["beam-08.dat", "beam-16.dat", "beam-24.dat"]
    b = lib.beam_read(str(tmp_path / "beam-16.dat"), p)
    assert lib.ltt_run(ctx, lat, b, n_turns, ix_turn_start=16) == n_turns
    for f in ("vec", "beta", "t", "state", "ix_ele", "location"):
        assert np.array_equal(getattr(b, f), getattr(full, f)), f
    late = (full.state != abi.ALIVE) & (full.ix_turn >= 16)
    assert np.array_equal(b.ix_turn[late], full.ix_turn[late])
    final = lib.beam_read(str(tmp_path / "beam-24.dat"), p)
    assert np.array_equal(final.vec, full.vec) and np.array_equal(final.state, full.state)


@pytest.mark.parametrize("cutoff", [0.5, 0.9, 0.13])
def test_core_emittance_matches_reference(ctx, cutoff):
    """bmadgpu_bunch_core_emit against the numpy restatement of the combined core calculation, on a
    bunch with losses (dead particles excluded from the ranking)."""
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 20000, seed=21, scale=3.0)
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(20000))
    lat = lib.Lattice(ctx, eles, p)
    lib.track_bunch(ctx, lat, hb, n_turns=6)
    hb.state[::97] = abi.LOST_POS_X  # dead particles stay out of the ranking and the sums
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.array(getattr(hb, k))).to(dev) for k in ("vec", "beta", "t", "state")}
    view = abi.Bunch(hb.n, t["vec"].data_ptr(), t["beta"].data_ptr(), t["t"].data_ptr(), t["state"].data_ptr(),
                     None, None, None)
    got = lib.bunch_core_emit(ctx, lat, view, cutoff)
    want = core_emit(hb.vec, hb.t, hb.state, p.p0c, p.mass, cutoff)
    assert np.all(want > 0)
    assert np.allclose(got, want, rtol=1e-9, atol=0), (got, want)
    # the core is smaller than the bunch for cutoffs below 1 (before the f scaling)
    bd = bunch_data(hb.vec, hb.t, hb.state, p.p0c, p.mass)
    assert np.all(got < bd["emit"] * 1.5)


def test_ltt_core_columns_follow_the_cutoff_list(ctx, tmp_path):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 3000, seed=2, scale=2.0)
    lat = lib.Lattice(ctx, eles, p)
    for cuts, groups in (([], 0), ([0.5, 0.9], 2)):
        hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(3000))
        base = str(tmp_path / ("c%d" % groups))
        lib.ltt_run(ctx, lat, hb, 4, averages_file=base, averages_every_n_turns=2, core_emit_cutoff=cuts)
        rows = read_table(base + ".emit")
        assert all(len(r) == 12 + 3 * groups for r in rows)
        heads = [line for line in open(base + ".emit") if line.startswith("##")]
        assert heads[-2].count("% Core") == groups
        if groups:
            o = oracle_track(eles, p, vec, 4, t=np.zeros(3000))
            close([float(x) for x in rows[-1][15:18]], core_emit(o["vec"], o["t"], o["state"], p.p0c, p.mass, 0.9),
                  2e-6, "90 % core")


@pytest.mark.parametrize("cutoff", [0.5, 0.9])
def test_core_emittance_per_mode_matches_reference(ctx, cutoff):
    """The per-mode core calculation (core_emit_combined_calc = F): each mode's core ranked by that
    mode's action with N^-1 of the bunch and then of the core, against the numpy restatement."""
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 20000, seed=23, scale=3.0)
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(20000))
    lat = lib.Lattice(ctx, eles, p)
    lib.track_bunch(ctx, lat, hb, n_turns=5)
    hb.state[::89] = abi.LOST_NEG_Y
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.array(getattr(hb, k))).to(dev) for k in ("vec", "beta", "t", "state")}
    view = abi.Bunch(hb.n, t["vec"].data_ptr(), t["beta"].data_ptr(), t["t"].data_ptr(), t["state"].data_ptr(),
                     None, None, None)
    got = lib.bunch_core_emit(ctx, lat, view, cutoff, combined_calc=False)
    want = core_emit(hb.vec, hb.t, hb.state, p.p0c, p.mass, cutoff, combined=False)
    assert np.all(want > 0)
    assert np.allclose(got, want, rtol=1e-9, atol=0), (got, want)
    combined = lib.bunch_core_emit(ctx, lat, view, cutoff, combined_calc=True)
    assert not np.allclose(got, combined, rtol=1e-6, atol=0)       # a different calculation


def test_ltt_action_angle_and_per_particle_files(ctx, tmp_path):
    eles, p = rings.ring(50)
    n, n_turns = 600, 10
    vec = rings.matched_gaussian(eles, n, seed=8, scale=5.0)
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(n))
    lat = lib.Lattice(ctx, eles, p)
    base = str(tmp_path / "run")
    done = lib.ltt_run(ctx, lat, hb, n_turns, averages_file=base, averages_every_n_turns=5,
                       particle_every_n_turns=5, only_live_particles_out=False,
                       action_angle_file=str(tmp_path / "aa#.dat"), per_particle_file=str(tmp_path / "pp"),
                       core_emit_combined_calc=False)
    assert done == n_turns
    files = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "aa*.dat")))
    assert files == ["aa00.dat", "aa05.dat", "aa10.dat"]
    head = [line for line in open(str(tmp_path / "aa05.dat")) if line.startswith("##")][-1]
    assert head.split()[4:10] == ["Ja", "Angle_a", "Jb", "Angle_b", "Jc", "Angle_c"]
    states = {}
    for T in (0, 5, 10):
        o = oracle_track(eles, p, vec, T, t=np.zeros(n)) if T > 0 else dict(
            vec=vec, t=np.zeros(n), state=np.ones(n, np.int32))
        states[T] = o
        rows = read_table(str(tmp_path / ("aa%02d.dat" % T)))
        assert [int(r[0]) for r in rows] == list(range(1, n + 1))   # dead particles too
        got = np.array([[float(x) for x in r[2:8]] for r in rows]).T
        want = action_angle(o["vec"], o["t"], o["state"], p.p0c, p.mass)
        for m in range(3):
            # printed to 9 digits; a particle with a tiny action in one mode sees the rounding of
            # N^-1 leak in from the larger modes, hence the absolute floor and the scaled angle bound
            J, Jw = got[2 * m], want[2 * m]
            assert np.all(np.abs(J - Jw) <= 1e-7 * np.abs(Jw) + 1e-9 * np.max(Jw)), ("J", m, T)
            dphi = np.abs(got[2 * m + 1] - want[2 * m + 1])
            tol = 1e-7 * np.maximum(1.0, np.sqrt(np.median(Jw) / np.maximum(Jw, 1e-300)))
            assert np.all(np.minimum(dphi, 2 * np.pi - dphi) <= tol), ("angle", m, T)
        names = [r[-1] for r in rows]
        assert names.count("Alive") == int(np.sum(o["state"] == abi.ALIVE))
    # the per-mode core emittances reached the .emit file
    emi = read_table(base + ".emit")
    o = states[10]
    close([float(x) for x in emi[-1][12:15]],
          core_emit(o["vec"], o["t"], o["state"], p.p0c, p.mass, 0.5, combined=False), 2e-6, "per-mode core")
    # per-particle files: pp.001 .. pp.600, a header and one line per output turn
    pp = sorted(glob.glob(str(tmp_path / "pp.*")))
    assert len(pp) == n and os.path.basename(pp[0]) == "pp.001" and os.path.basename(pp[-1]) == "pp.600"
    for ip in (1, 77, 600):
        lines = open(str(tmp_path / ("pp.%03d" % ip))).read().splitlines()
        assert "# ix_particle     = %d" % ip in lines
        rows = [ln.split() for ln in lines if not ln.startswith("#")]
        assert [int(r[0]) for r in rows] == [0, 5, 10]
        for r, T in zip(rows, (0, 5, 10)):
            want = states[T]["vec"][:, ip - 1]
            got = np.array([float(x) for x in r[1:7]])
            assert np.all(np.abs(got - want) <= 1e-8 * np.abs(want) + 1e-300), (ip, T, got, want)
            assert float(r[8]) == pytest.approx(p.p0c, rel=1e-8)


def test_per_particle_output_refuses_large_bunches(ctx, tmp_path):
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 1001, seed=1)
    hb = lib.HostBunch.from_vec(vec, p)
    lat = lib.Lattice(ctx, eles, p)
    with pytest.raises(lib.BmadGpuError):
        lib.ltt_run(ctx, lat, hb, 2, per_particle_file=str(tmp_path / "pp"))


def test_ltt_action_angle_from_the_one_turn_matrix(ctx, tmp_path):
    """action_angle_calc_uses_1turn_matrix: actions about zero with N^-1 of make_N on the one-turn
    matrix at the closed orbit. The file holds N^-1 p of the oracle's particles, and for small
    amplitudes the actions are turn-by-turn invariants (the normal form is right)."""
    eles, p = rings.ring(50)
    n, n_turns = 400, 10
    lat = lib.Lattice(ctx, eles, p)
    orbit = lib.closed_orbit(ctx, lat)[0]
    vec = rings.matched_gaussian(eles, n, seed=12, scale=0.5) + orbit[:, None]
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(n))
    done = lib.ltt_run(ctx, lat, hb, n_turns, particle_every_n_turns=10, action_angle_file=str(tmp_path / "aa#"),
                       action_angle_calc_uses_1turn_matrix=True)
    assert done == n_turns
    n_inv = np.linalg.inv(lib.make_n(lib.one_turn_matrix(ctx, lat, orbit, rf_on=True)[0]))
    J = {}
    for T in (0, 10):
        o = oracle_track(eles, p, vec, T, t=np.zeros(n)) if T > 0 else dict(vec=vec, state=np.ones(n, np.int32))
        rows = read_table(str(tmp_path / ("aa%02d" % T)))
        got = np.array([[float(x) for x in r[2:8]] for r in rows]).T
        j = n_inv @ o["vec"]
        for m in range(3):
            want = 0.5 * (j[2 * m] ** 2 + j[2 * m + 1] ** 2)
            assert np.all(np.abs(got[2 * m] - want) <= 1e-7 * want + 1e-9 * np.max(want)), ("J", m, T)
        J[T] = got[0::2]
    # about zero, the closed orbit itself shows as a constant offset: compare the changes of J of
    # the transverse modes over 10 turns with their spread; they are a small fraction of it
    for m in range(2):
        dJ = np.abs(J[10][m] - J[0][m])
        assert np.median(dJ) < 0.05 * np.median(J[0][m]), m


@pytest.mark.parametrize("combined", [True, False])
def test_core_emittance_with_tied_amplitudes(ctx, combined):
    """Every particle three times: the amplitudes tie in threes and the cut splits a tie, which the
    device selection must resolve to the lower particle indices as a stable sort does."""
    eles, p = rings.ring(50)
    base = rings.matched_gaussian(eles, 6001, seed=31, scale=2.0)
    vec = np.ascontiguousarray(np.repeat(base, 3, axis=1))
    n = vec.shape[1]
    hb = lib.HostBunch.from_vec(vec, p, t=np.zeros(n))
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(np.array(getattr(hb, k))).to(dev) for k in ("vec", "beta", "t", "state")}
    view = abi.Bunch(hb.n, t["vec"].data_ptr(), t["beta"].data_ptr(), t["t"].data_ptr(), t["state"].data_ptr(),
                     None, None, None)
    lat = lib.Lattice(ctx, eles, p)
    for cutoff in (0.5, 0.37):
        assert int(cutoff * n) % 3 != 0          # the cut falls inside a group of three
        got = lib.bunch_core_emit(ctx, lat, view, cutoff, combined_calc=combined)
        want = core_emit(hb.vec, hb.t, hb.state, p.p0c, p.mass, cutoff, combined=combined)
        assert np.allclose(got, want, rtol=1e-9, atol=0), (cutoff, got, want)


def test_core_selection_mask_ties_to_lower_index(ctx):
    """The selection itself: ties at scattered indices, split by the cut, go to the lower indices
    (a stable sort's order); dead (1e100), infinite and NaN amplitudes are never taken, and a cut
    that would need one of them reports no core."""
    rng = np.random.default_rng(5)
    n = 50000
    keys = rng.choice(rng.uniform(0.0, 3.0, 700), n)        # about 70 copies of each value
    keys[rng.choice(n, 900, replace=False)] = 1e100
    keys[rng.choice(n, 30, replace=False)] = np.inf
    keys[rng.choice(n, 30, replace=False)] = np.nan
    keys[17] = 0.0
    dev = torch.from_numpy(keys).to("cuda:0")
    finite = np.count_nonzero(keys < 1e99)
    order = np.argsort(np.where(np.isnan(keys), np.inf, keys), kind="stable")
    for n_cut in (1, 2, 12345, n // 2, finite - 1, finite):
        got = lib.select_smallest(ctx, dev, n_cut)
        want = np.zeros(n, np.int32)
        want[order[:n_cut]] = abi.ALIVE
        assert got is not None, n_cut
        assert np.array_equal(got, want), n_cut
        t = keys[order[n_cut - 1]]
        assert n_cut < 3 or np.count_nonzero(keys == t) > 1      # the cut falls inside a tie
    for n_cut in (finite + 1, n):
        assert lib.select_smallest(ctx, dev, n_cut) is None
