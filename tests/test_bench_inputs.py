"""The reference arm's inputs are the engine's workloads.

bench.py's reference arm loads no library of this repository: it writes the
config-5 replicas and config 2 in the reference's input format with
oracle/_build/ref_inputs (the engine's generator source compiled into a small
program) from spec lines it computes itself.  Here those files, read back with
the library's reader, must hold exactly the particles of
ph_brush_b200.configs' systems (positions, charges, bonds; types mapped to the
reference's), plus one W bead per titratable site inside the slab, and the
reference-model set-up must give the reference's mesh rule and alpha.
"""
import os
import subprocess

import numpy as np
import pytest

import bench
from ph_brush_b200 import configs, files

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ref_inputs_built():
    if not os.path.exists(bench.REF_INPUTS):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "..", "oracle"), "inputs"], check=True)
    return bench.REF_INPUTS


def check_same(sys_native, data_path):
    d = files.read_lammps(data_path, wrap=True)
    n = sys_native.n
    for k in ("x", "y", "z", "q"):
        assert np.array_equal(d[k][:n], getattr(sys_native, k)), k
    assert np.array_equal(d["type"][:n], configs.NATIVE_TO_REF[sys_native.type])
    assert np.array_equal(d["bond_i"], sys_native.bond_i) and np.array_equal(d["bond_j"], sys_native.bond_j)
    n_sites = int(np.count_nonzero(sys_native.flags & 2))
    assert d["natoms"] == n + n_sites
    w = d["type"][n:]
    assert np.all(w == configs.REF_W_TYPE)
    H = sys_native.meta["height"]
    assert np.all((d["z"][n:] >= 0) & (d["z"][n:] < H))
    assert np.all(d["q"][n:] == 0)


def test_config5_spec_lines_reproduce_the_package_systems(tmp_path, ref_inputs_built):
    reps = configs.config5(n_rep=256)
    lines = bench.config5_spec_lines(2029, 256)
    pick = [0, 1, 2, int(np.argmin([s.n for s, _ in reps])), 255]
    info = bench.write_ref_inputs([lines[k] for k in pick], str(tmp_path))
    for k in pick:
        s, p = reps[k]
        name = f"c5_{k:04d}"
        assert info[name][1] == s.n
        check_same(s, str(tmp_path / (name + ".data")))
        ex = open(tmp_path / (name + ".extra")).read().split()
        assert float(ex[ex.index("pH") + 1]) == p.pH
        nmob = int(ex[ex.index("mobile") + 1])
        assert nmob == int(np.count_nonzero(s.flags & 1))


def test_config2_spec_line_reproduces_the_package_system(tmp_path, ref_inputs_built):
    s2, _ = configs.config2()
    info = bench.write_ref_inputs([bench.config2_spec_line()], str(tmp_path))
    assert info["c2"][1] == s2.n
    check_same(s2, str(tmp_path / "c2.data"))
    s, p = files.reference_model(str(tmp_path / "c2.data"), str(tmp_path / "c2.params"))
    assert tuple(p.mesh) == configs.ref_mesh(s.box, 0.7, 4)
    assert abs(s.box[2] - 300.0) < 1e-9 and p.slab == 1 and p.order == 4 and p.ref_moduli == 1
    assert abs(p.ewald_alpha - configs.ewald_alpha(3.0, 1e-5)) < 1e-6
