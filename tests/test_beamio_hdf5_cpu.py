"""HDF5 (openPMD) beam files (bmadgpu_beam_read_hdf5 / bmadgpu_beam_write_hdf5), host-only, on CPU.

Pinned to the reference's hdf5_test (regression_tests/hdf5_test): its old-layout beam file
bunch_old.h5 (committed as tests/golden/hdf5_test_bunch_old.h5) holds the ten particles of
beam_1.dat (tests/golden/hdf5_test_beam_1.dat) as bunch 1 and a photon bunch as bunch 2; the test
checks that reading the file gives back the particles of the ASCII beam ("Old-Bunch1" TTTTTTTTTT,
output.correct:11) and prints particle 7 of that beam (output.correct:2-5)."""
import importlib
import os

import numpy as np
import pytest

lib = importlib.import_module("bmad-ecosystem_b200.lib")
abi = importlib.import_module("bmad-ecosystem_b200.abi")
rings = importlib.import_module("bmad-ecosystem_b200.rings")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OLD_H5 = os.path.join(GOLDEN, "hdf5_test_bunch_old.h5")
BEAM_1 = os.path.join(GOLDEN, "hdf5_test_beam_1.dat")

# regression_tests/hdf5_test/output.correct:2-5 (particle 7 of bunch 1, REL 1e-10)
P7_VEC = [1.6387488057E-03, -2.9985054496E-06, 1.8144481648E-03, -7.8926417700E-05, -1.5942344121E-04,
          5.2241291487E-04]
P7_T, P7_P0C, P7_BETA = 5.3177942856E-13, 9.9999986944E+08, 9.9999986958E-01


def positron_1gev():
    """lat.bmad of hdf5_test: positron (Bmad's default species), beginning e_tot = 1e9."""
    p = abi.Param()
    p.mass, p.charge, p.e_tot = 0.51099895069e6, 1.0, 1e9
    p.p0c = (p.e_tot ** 2 - p.mass ** 2) ** 0.5
    return p


def rel(a, b):
    return abs(a - b) / abs(b)


def test_old_layout_particle_7_matches_reference_output():
    p = positron_1gev()
    assert rel(p.p0c, P7_P0C) < 1e-10
    b, n_bunch = lib.beam_read_hdf5(OLD_H5, p, 0)
    assert n_bunch == 2 and b.vec.shape == (6, 10)
    for i in range(6):
        assert rel(b.vec[i, 6], P7_VEC[i]) < 1e-10, i
    assert rel(b.t[6], P7_T) < 1e-10
    assert rel(b.beta[6], P7_BETA) < 1e-10
    # output.correct:5: state alive, location downstream_end
    assert b.state[6] == abi.ALIVE and b.location[6] == abi.DOWNSTREAM_END


def test_old_layout_bunch_equals_ascii_beam():
    """The reference's Old-Bunch1 check: the HDF5 bunch equals the ASCII beam particle for particle."""
    p = positron_1gev()
    b, _ = lib.beam_read_hdf5(OLD_H5, p, 0)
    a = lib.beam_read(BEAM_1, p)
    assert np.allclose(b.vec, a.vec, rtol=1e-12, atol=1e-18)
    assert np.array_equal(b.state, a.state)


def test_photon_bunch_and_bad_index_are_refused():
    p = positron_1gev()
    with pytest.raises(lib.BmadGpuError) as e:
        lib.beam_read_hdf5(OLD_H5, p, 1)          # bunch 2 of the file is a photon bunch
    assert e.value.code == abi.EUNSUPPORTED
    with pytest.raises(lib.BmadGpuError) as e:
        lib.beam_read_hdf5(OLD_H5, p, 2)
    assert e.value.code == abi.EINVAL


def sample(n=300, seed=3):
    eles, p = rings.ring(10)
    rng = np.random.default_rng(seed)
    b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, n, seed=seed), p, t=rng.normal(0, 1e-9, n))
    b.state[[3, 10, 11]] = [abi.LOST_POS_X, abi.LOST_NEG_Y, abi.LOST_PZ]
    b.ix_ele[[3, 10, 11]] = [17, 0, 35]
    b.location[:] = abi.DOWNSTREAM_END
    b.location[[3, 10, 11]] = [abi.DOWNSTREAM_END, abi.UPSTREAM_END, abi.INSIDE]
    return b, p


def test_round_trip(tmp_path):
    b, p = sample()
    path = str(tmp_path / "beam.h5")
    lib.beam_write_hdf5(path, b, p, s_position=12.5)
    r, n_bunch = lib.beam_read_hdf5(path, p)
    assert n_bunch == 1
    # px, py and z pass through px * p0c, py * p0c and t - t_ref as in the reference's file
    assert np.allclose(r.vec, b.vec, rtol=4e-16, atol=1e-300)
    assert np.array_equal(r.beta, b.beta)
    assert np.allclose(r.t, b.t, rtol=4e-16, atol=1e-300)
    lost = b.state != abi.ALIVE
    assert np.array_equal(r.state, b.state)
    assert np.array_equal(r.ix_ele[lost], b.ix_ele[lost])
    assert np.array_equal(r.location, b.location)


def test_alive_only_and_constant_records(tmp_path):
    b, p = sample()
    path = str(tmp_path / "alive.h5")
    lib.beam_write_hdf5(path, b, p, flags=lib.BEAM_ALIVE_ONLY)
    r, _ = lib.beam_read_hdf5(path, p)
    alive = b.state == abi.ALIVE
    assert r.vec.shape[1] == alive.sum()
    assert np.all(r.state == abi.ALIVE)            # particleStatus all equal: a constant record
    assert np.allclose(r.vec, b.vec[:, alive], rtol=4e-16, atol=1e-300)
    # a bunch with one particle: every record is a constant record component
    one = lib.HostBunch.from_vec(b.vec[:, :1].copy(), p, t=b.t[:1].copy())
    lib.beam_write_hdf5(path, one, p)
    r1, _ = lib.beam_read_hdf5(path, p)
    assert np.allclose(r1.vec, one.vec, rtol=4e-16, atol=1e-300)


def test_append(tmp_path):
    """hdf5_write_beam with append: the file's bunches stay, the new one takes the next number."""
    b, p = sample(20)
    c, _ = sample(30, seed=4)
    path = str(tmp_path / "x.h5")
    lib.beam_write_hdf5(path, b, p, flags=lib.BEAM_APPEND)          # no file yet: a new one
    lib.beam_write_hdf5(path, c, p, flags=lib.BEAM_APPEND)
    for k, ref in enumerate((b, c)):
        r, n_bunch = lib.beam_read_hdf5(path, p, k)
        assert n_bunch == 2
        assert np.allclose(r.vec, ref.vec, rtol=4e-16, atol=1e-300) and np.array_equal(r.state, ref.state)
    # onto a copy of the reference's own file (bunch 1 positrons, bunch 2 photons): both kept
    old = str(tmp_path / "old.h5")
    open(old, "wb").write(open(OLD_H5, "rb").read())
    q = positron_1gev()
    c = lib.HostBunch.from_vec(c.vec, q, t=c.t)                      # beta of this species and energy
    lib.beam_write_hdf5(old, c, q, flags=lib.BEAM_APPEND)
    first, n_bunch = lib.beam_read_hdf5(old, q, 0)
    assert n_bunch == 3
    assert np.array_equal(first.vec, lib.beam_read_hdf5(OLD_H5, q, 0)[0].vec)
    with pytest.raises(lib.BmadGpuError):
        lib.beam_read_hdf5(old, q, 1)                                  # still the photon bunch
    third, _ = lib.beam_read_hdf5(old, q, 2)
    assert np.allclose(third.vec, c.vec, rtol=4e-16, atol=1e-300)
    assert np.array_equal(third.beta, c.beta)


def test_unknown_species_is_refused(tmp_path):
    b, p = sample(20)
    path = str(tmp_path / "x.h5")
    q = abi.Param()
    q.p0c, q.e_tot, q.mass, q.charge = p.p0c, p.e_tot, 105.6583755e6, -1.0     # a muon
    with pytest.raises(lib.BmadGpuError) as e:
        lib.beam_write_hdf5(path, b, q)
    assert e.value.code == abi.EUNSUPPORTED


def test_truncated_file_is_an_error(tmp_path):
    data = open(OLD_H5, "rb").read()
    path = str(tmp_path / "cut.h5")
    for cut in (50, 4000, len(data) // 2):
        open(path, "wb").write(data[:cut])
        with pytest.raises(lib.BmadGpuError):
            lib.beam_read_hdf5(path, positron_1gev(), 0)


def test_file_name_picks_the_format(tmp_path):
    """write_beam_file / read_beam_file: HDF5 for .h5 and .hdf5 names, ASCII otherwise."""
    b, p = sample(50)
    for name, hdf5 in (("a.h5", True), ("a.hdf5", True), ("a.dat", False), ("a_h5", False)):
        path = str(tmp_path / name)
        lib.write_beam_file(path, b, p, flags=lib.BEAM_EXACT)
        head = open(path, "rb").read(8)
        assert (head == b"\x89HDF\r\n\x1a\n") == hdf5, name
        r = lib.read_beam_file(path, p)
        assert np.allclose(r.vec, b.vec, rtol=4e-16, atol=1e-300), name
        assert np.array_equal(r.state, b.state), name


def test_writer_uses_the_encodings_of_the_reference_file(tmp_path):
    """The writer's superblock fields, datatypes, dataspaces and fill-value message are byte for byte
    those libhdf5 wrote into the reference's bunch_old.h5 (independent of this library's reader)."""
    ref = open(OLD_H5, "rb").read()
    eles, p = rings.ring(10)
    b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, 10, seed=1), p, t=np.zeros(10))
    path = str(tmp_path / "enc.h5")
    lib.beam_write_hdf5(path, b, p)
    ours = open(path, "rb").read()
    assert ours[:24] == ref[:24]                                    # signature, versions, sizes, K values
    pieces = [
        "11203f000800000000004000340b0034ff030000",                # IEEE f64 little-endian
        "100800000400000000002000",                                # signed i32 little-endian
        "0202020100000000",                                        # fill value message
        "0100000000000000",                                        # scalar dataspace (string attributes)
        "01010100000000000a000000000000000a00000000000000",        # 1-D dataspace of 10 with max 10
        "13000000",                                                # fixed-length null-terminated string
    ]
    for h in pieces:
        assert bytes.fromhex(h) in ref and bytes.fromhex(h) in ours, h
    for sig in (b"TREE", b"HEAP", b"SNOD"):
        assert sig in ours


def test_files_of_other_openpmd_writers():
    """Two more of the reference's particle files, written by another openPMD writer (null-padded
    strings, 64-bit integer attributes, basePath "/" without %T, particlesPath "." or "particles/",
    no totalMomentumOffset): regression_tests/pytao/sr_wakes/particles3.h5 (3 positrons, read by
    tao.startup with the lattice's e_tot = 10e6) and regression_tests/space_charge_test/
    initial_particles.h5 (10 electrons before cathode emission)."""
    p = abi.Param()
    p.mass, p.charge, p.e_tot = 0.51099895069e6, 1.0, 10e6
    p.p0c = (p.e_tot ** 2 - p.mass ** 2) ** 0.5
    b, n_bunch = lib.beam_read_hdf5(os.path.join(GOLDEN, "sr_wakes_particles3.h5"), p)
    assert n_bunch == 1 and b.vec.shape == (6, 3)
    assert np.all(b.state == abi.ALIVE)
    # no reference momentum in the file: pz relative to the lattice's p0c (sig_pz ~ 6e-3 in tao.startup)
    assert np.all(np.abs(b.vec[5]) < 0.05)
    pc = p.p0c * (1 + b.vec[5])
    assert np.allclose(b.beta, pc / np.sqrt(pc * pc + p.mass ** 2), rtol=1e-15)
    # no timeOffset record: t = time and z = -beta c time
    assert np.array_equal(b.vec[4], -b.beta * 2.99792458e8 * b.t)
    p.charge = -1.0
    g, _ = lib.beam_read_hdf5(os.path.join(GOLDEN, "space_charge_initial_particles.h5"), p)
    assert g.vec.shape == (6, 10)
    assert np.all(g.state == 0)                     # pre_born$ (openPMD status 0) is kept


def test_several_bunches_in_one_file(tmp_path):
    """hdf5_write_beam's bunches(:): one group per bunch, /data/00001/ ... ; each read back by index."""
    eles, p = rings.ring(10)
    bunches = []
    for k, n in enumerate((7, 1, 40)):
        b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, n, seed=10 + k), p, t=np.full(n, 1e-9 * k))
        bunches.append(b)
    bunches[2].state[5] = abi.LOST_NEG_X
    bunches[2].ix_ele[5] = 12
    bunches[2].location[:] = abi.DOWNSTREAM_END
    path = str(tmp_path / "three.h5")
    lib.beam_write_hdf5(path, bunches, p)
    for k, b in enumerate(bunches):
        r, n_bunch = lib.beam_read_hdf5(path, p, k)
        assert n_bunch == 3 and r.vec.shape == b.vec.shape
        assert np.allclose(r.vec, b.vec, rtol=4e-16, atol=1e-300)
        assert np.array_equal(r.state, b.state)
    r, _ = lib.beam_read_hdf5(path, p, 2)
    assert r.ix_ele[5] == 12
    # many bunches: the data group's names span several symbol-table nodes
    many = [bunches[1]] * 20
    lib.beam_write_hdf5(path, many, p)
    r, n_bunch = lib.beam_read_hdf5(path, p, 19)
    assert n_bunch == 20 and np.allclose(r.vec, bunches[1].vec, rtol=4e-16, atol=1e-300)
    with pytest.raises(lib.BmadGpuError):
        lib.beam_write_hdf5(path, [bunches[1]] * 257, p)


def test_corrupted_files_never_read_out_of_bounds(tmp_path):
    """The HDF5 and ASCII readers, and appending to an HDF5 file, under AddressSanitizer and UBSan on
    1,500 corrupted copies of each reference beam file and of an ASCII file written here."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "beamfile_fuzz")
    build = subprocess.run([gxx, "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                            "-o", exe, os.path.join(root, "tests", "c", "beamfile_fuzz.cpp"),
                            os.path.join(root, "bmad-ecosystem_b200", "csrc", "h5beam.cpp"),
                            os.path.join(root, "bmad-ecosystem_b200", "csrc", "beamio.cpp")],
                           capture_output=True, text=True)
    if build.returncode != 0 and "asan" in build.stderr.lower():
        pytest.skip("no sanitizer runtime")
    assert build.returncode == 0, build.stderr[-2000:]
    b, p = sample(40)
    v4 = str(tmp_path / "v4.dat")
    lib.beam_write(v4, b, p)
    cases = [("hdf5", os.path.join(GOLDEN, n)) for n in
             ("hdf5_test_bunch_old.h5", "sr_wakes_particles3.h5", "space_charge_initial_particles.h5")]
    cases += [("ascii", BEAM_1), ("ascii", v4), ("append", OLD_H5)]
    for i, (kind, path) in enumerate(cases):
        run = subprocess.run([exe, kind, path, str(11 + i), "1500", str(tmp_path / "m.bin")],
                             capture_output=True, text=True, timeout=600)
        assert run.returncode == 0, (path, run.stderr[-3000:])
        assert run.stdout.startswith("read "), run.stdout


def test_reading_at_the_beginning_element(tmp_path):
    """hdf5_read_beam given the lattice's beginning element (conserve_momentum at its default), for a
    file whose reference momentum differs from the lattice's: px and py over the lattice's p0c, pz
    over the file's, beta from (1 + pz) times the lattice's p0c, every particle at the element's exit."""
    b, p = sample(25)
    path = str(tmp_path / "p.h5")
    lib.beam_write_hdf5(path, b, p)                                 # file p0c = p.p0c
    q = abi.Param()
    q.mass, q.charge, q.p0c = p.mass, p.charge, p.p0c * 1.01
    q.e_tot = (q.p0c ** 2 + q.mass ** 2) ** 0.5
    plain, _ = lib.beam_read_hdf5(path, q)
    at, _ = lib.beam_read_hdf5(path, q, flags=lib.BEAM_AT_ELEMENT)
    assert np.allclose(plain.vec, b.vec, rtol=4e-16, atol=1e-300)   # without an element: the file's p0c
    assert np.allclose(at.vec[[1, 3]], b.vec[[1, 3]] * p.p0c / q.p0c, rtol=1e-15, atol=1e-300)
    assert np.allclose(at.vec[5], b.vec[5], rtol=4e-16, atol=1e-300)
    pc = (1 + at.vec[5]) * q.p0c
    assert np.allclose(at.beta, pc / np.sqrt(pc * pc + q.mass ** 2), rtol=1e-15)
    # the file stores t - t_ref = -z / (beta c): z follows the new beta
    assert np.allclose(at.vec[4], b.vec[4] * at.beta / b.beta, rtol=1e-15, atol=1e-300)
    assert np.all(at.ix_ele == -1) and np.all(at.location == abi.DOWNSTREAM_END)
    assert np.array_equal(at.state, b.state)
