"""Generates tests/golden/ref_energies.json on a GPU machine.

Writes small brush systems in the reference's own input format
(tests/golden/inputs/*.data, *.params), runs the reference's unmodified
energy routines on them (oracle/_ref/ref_harness, built by `make -C oracle
ref` from the reference sources: read_lammps_full, build_half_neighbors_gpu,
compute_lj_sr_energy_gpu, compute_coul_sr_energy_gpu, pmeCreate, pmeEnergy)
and records the printed energies.  Usage: python tests/golden/make_ref_fixtures.py
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ph_brush_b200 import configs  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def cases():
    small, _ = configs.small_system(seed=3)
    c1, _ = configs.config1()
    yield "small_pme", configs.to_reference_semantics(small, n_w=16, spacing=0.5, seed=1), 0.5, "pme"
    yield "cfg1_pme", configs.to_reference_semantics(c1, n_w=64, spacing=0.5, seed=2), 0.5, "pme"
    yield "cfg1_pme_odd_mesh", configs.to_reference_semantics(c1, n_w=0, spacing=0.6, seed=3), 0.6, "pme"
    yield "cfg1_coul_cut", configs.to_reference_semantics(c1, n_w=0, spacing=0.5, seed=4), 0.5, "coul_cut"


def main(inputs_only=False):
    os.makedirs(os.path.join(HERE, "inputs"), exist_ok=True)
    out = {}
    for name, (s, p), spacing, coul in cases():
        dpath = os.path.join(HERE, "inputs", name + ".data")
        ppath = os.path.join(HERE, "inputs", name + ".params")
        configs.write_lammps_data(dpath, s)
        configs.write_params_in(ppath, p, spacing, coulombtype=coul)
        if inputs_only:
            continue
        r = subprocess.run([HARNESS, "energy", dpath, ppath], capture_output=True, text=True, check=True)
        out[name] = json.loads(r.stdout.strip().splitlines()[-1])
        out[name]["spacing"] = spacing
        out[name]["coulombtype"] = coul
        print(name, out[name])
    if inputs_only:
        return
    with open(os.path.join(HERE, "ref_energies.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(inputs_only="--inputs-only" in sys.argv)
