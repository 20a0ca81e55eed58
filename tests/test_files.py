"""Host-side input files: the library's LAMMPS data reader / writer and params.in
reader against the reference's own (MC/src/io.cpp, compiled from its sources into
oracle/_ref/libref_host.so by `make -C oracle ref-host`).  Values must be
bit-identical: the same atoms, bonds, box, parameters, derived Ewald alpha and LJ
shift table; files the library writes read back identically in both readers."""
import ctypes as C
import os

import numpy as np
import pytest

from ph_brush_b200 import _abi, files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INPUTS = os.path.join(ROOT, "tests", "golden", "inputs")
REF_HOST = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
CASES = ["cfg1_pme", "cfg1_coul_cut", "cfg1_pme_odd_mesh", "small_pme", "dropin_small"]
_ip, _dp = C.POINTER(C.c_int), C.POINTER(C.c_double)

needs_ref = pytest.mark.skipif(not os.path.exists(REF_HOST), reason="reference host code not built (make -C oracle ref-host)")


def ref_read_data(path, cap=100000):
    lib = C.CDLL(REF_HOST)
    counts, box = np.zeros(3, np.int32), np.zeros(3)
    idv, mol, typ = (np.zeros(cap, np.int32) for _ in range(3))
    q, x, y, z = (np.zeros(cap) for _ in range(4))
    head, lst = np.zeros(cap + 1, np.int32), np.zeros(4 * cap, np.int32)
    err = C.create_string_buffer(256)
    rc = lib.refh_read_data(str(path).encode(), counts.ctypes.data_as(_ip), box.ctypes.data_as(_dp), idv.ctypes.data_as(_ip),
                            mol.ctypes.data_as(_ip), typ.ctypes.data_as(_ip), q.ctypes.data_as(_dp), x.ctypes.data_as(_dp),
                            y.ctypes.data_as(_dp), z.ctypes.data_as(_dp), head.ctypes.data_as(_ip), lst.ctypes.data_as(_ip),
                            cap, err, 256)
    if rc:
        raise RuntimeError(err.value.decode())
    n = int(counts[0])
    return {"natoms": n, "nbonds": int(counts[1]), "ntypes": int(counts[2]), "box": box, "id": idv[:n], "mol": mol[:n],
            "type": typ[:n], "q": q[:n], "x": x[:n], "y": y[:n], "z": z[:n], "head": head[:n + 1], "list": lst[:head[n]]}


def ref_read_params(path, ntypes):
    lib = C.CDLL(REF_HOST)
    d, i = np.zeros(11), np.zeros(16, np.int32)
    eps, sig, sh = (np.zeros(ntypes * ntypes) for _ in range(3))
    err = C.create_string_buffer(256)
    rc = lib.refh_read_params(str(path).encode(), ntypes, d.ctypes.data_as(_dp), i.ctypes.data_as(_ip), eps.ctypes.data_as(_dp),
                              sig.ctypes.data_as(_dp), sh.ctypes.data_as(_dp), err, 256)
    if rc:
        raise RuntimeError(err.value.decode())
    return d, i, eps.reshape(ntypes, ntypes), sig.reshape(ntypes, ntypes), sh.reshape(ntypes, ntypes)


def adjacency(n, bi, bj):
    """The reference's symmetric sorted 1-2 CSR (MC/src/io.cpp:148-169) from a bond list."""
    nb = [set() for _ in range(n)]
    for a, b in zip(bi, bj):
        nb[a].add(b)
        nb[b].add(a)
    head = np.zeros(n + 1, np.int32)
    for k in range(n):
        head[k + 1] = head[k] + len(nb[k])
    return head, np.array([j for k in range(n) for j in sorted(nb[k])], np.int32)


def assert_same_atoms(ours, ref):
    # the wrapper reports the bonds it kept (bonds naming unknown atom ids are dropped by both)
    assert ours["natoms"] == ref["natoms"] and len(ours["bond_i"]) == ref["nbonds"] and ours["ntypes"] == ref["ntypes"]
    assert np.array_equal(ours["box"], ref["box"])
    for k in ("id", "mol", "type"):
        assert np.array_equal(ours[k], ref[k]), k
    for k in ("q", "x", "y", "z"):  # the reference's FP32 values, promoted
        assert np.array_equal(ours[k].astype(np.float64), ref[k]), k
    head, lst = adjacency(ours["natoms"], ours["bond_i"], ours["bond_j"])
    assert np.array_equal(head, ref["head"]) and np.array_equal(lst, ref["list"])


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_data_file_matches_the_reference_reader(case):
    path = os.path.join(INPUTS, case + ".data")
    assert_same_atoms(files.read_lammps(path, wrap=True), ref_read_data(path))


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_params_match_the_reference_reader(case):
    path = os.path.join(INPUTS, case + ".params")
    ntypes = files.read_lammps(os.path.join(INPUTS, case + ".data"))["ntypes"]
    v, eps, sig, sh, unknown = files.read_params(path, ntypes)
    d, i, reps, rsig, rsh = ref_read_params(path, ntypes)
    ours_d = [v[k] for k in ("rc", "ewald_alpha", "epsilon_r", "pme_spacing", "pme_3dc_zfac", "beta", "ewald_rtol",
                             "target_pct", "w_z_extra_nm", "mu_eta", "nacc_frac_round")]
    assert ours_d == list(d)
    coul = {0: _abi.COUL_CUT, 1: _abi.COUL_EWALD, 2: -1}[int(i[1])]
    ours_i = [v["lj_shift"], v["coulomb"], v["pme_order"], v["pme_3dc"], v["nh_n_type"], v["nh_p_type"], v["w_type"],
              v["cl_type"], v["rng_seed"], v["energy_interval"], v["patience"], v["max_attempts"],
              v["direct_pct_threshold"], v["gc_block_fixed"], v["epoch_attempt_max"], v["phase2_wc"]]
    assert ours_i == [int(i[0]), coul] + [int(t) for t in i[2:]]
    assert np.array_equal(eps, reps) and np.array_equal(sig, rsig) and np.array_equal(sh, rsh)
    assert unknown == []


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_written_file_reads_back_the_same_in_both_readers(case, tmp_path):
    d = files.read_lammps(os.path.join(INPUTS, case + ".data"), wrap=True)
    out = tmp_path / "w.data"
    files.write_lammps(out, d)
    again = files.read_lammps(out, wrap=True)
    for k in ("id", "mol", "type", "q", "x", "y", "z", "bond_type", "bond_i", "bond_j", "box"):
        assert np.array_equal(again[k], d[k]), k
    assert_same_atoms(again, ref_read_data(out))


@needs_ref
def test_unusual_data_files_are_read_like_the_reference(tmp_path):
    """Comments after values, image flags, Masses and Velocities sections, CRLF line ends,
    bonds to unknown atom ids (dropped) and positions outside the box (wrapped)."""
    text = ("title line\r\n\r\n4 atoms\r\n3 bonds\r\n2 atom types\r\n1 bond types\r\n"
            "-1.5 6.5 xlo xhi\r\n0 8 ylo yhi\r\n0.0 10.0 zlo zhi\r\n\r\nMasses\r\n\r\n1 1.0\r\n2 1.0\r\n\r\n"
            "Atoms # full\r\n\r\n1 1 1 0.5 -2.25 1.0 3.0 0 0 0\r\n2 1 2 -0.5 9.0 8.0 -1e-3 # tail\r\n"
            "7 2 1 1e0 0.1 0.2 0.3\r\n3 2 2 -1 4 5 6\r\n\r\nVelocities\r\n\r\n1 0 0 0\r\n\r\n"
            "Bonds\r\n\r\n1 1 1 2\r\n2 1 2 99\r\n3 1 7 3\r\n")
    path = tmp_path / "odd.data"
    path.write_bytes(text.encode())
    ours, ref = files.read_lammps(path, wrap=True), ref_read_data(path)
    assert_same_atoms(ours, ref)
    assert ours["nbonds"] == 3 and len(ours["bond_i"]) == 2


@needs_ref
def test_superset_and_unknown_keys(tmp_path):
    base = open(os.path.join(INPUTS, "small_pme.params")).read()
    path = tmp_path / "p.in"
    path.write_text(base + "\npH = 6.5\npKa = 7.3\nsalt_conc = 0.01\nwall_lo = 0\nwall_hi = 60\npme_mesh = 32 32 96\n"
                           "frobnicate = 3\n")
    ntypes = files.read_lammps(os.path.join(INPUTS, "small_pme.data"))["ntypes"]
    v, eps, sig, sh, unknown = files.read_params(path, ntypes)
    assert (v["pH"], v["pKa"], v["salt_conc"], v["wall_hi"], v["mesh"]) == (6.5, 7.3, 0.01, 60.0, (32, 32, 96))
    assert np.isnan(v["fene_k"]) and unknown == ["frobnicate"]
    d, i, *_ = ref_read_params(path, ntypes)  # the reference ignores what it does not know
    assert [v["rc"], v["ewald_alpha"]] == [d[0], d[1]]
    with pytest.raises(_abi.PhmcError, match="frobnicate"):
        files.read_params(path, ntypes, strict=True)


def test_readers_report_errors(tmp_path):
    missing = tmp_path / "none.data"
    with pytest.raises(_abi.PhmcError):
        files.read_lammps(missing)
    bad = tmp_path / "bad.data"
    bad.write_text("3 atoms\n1 atom types\n0 1 xlo xhi\n0 1 ylo yhi\n0 1 zlo zhi\n\nAtoms\n\n1 1 1 0 0 0 0\n")
    with pytest.raises(_abi.PhmcError, match="mismatch"):
        files.read_lammps(bad)
    p = tmp_path / "p.in"
    p.write_text("epsilon_r = 2\n")
    with pytest.raises(_abi.PhmcError, match="cutoff_nm"):
        files.read_params(p, 8)
