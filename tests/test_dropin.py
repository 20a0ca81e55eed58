"""Drop-in: the reference's own driver (MC/src/main.cu with its protonation phase
and phase-2 swaps, MC/src/mc.cu, io.cpp, report.cpp) linked against the engine
through ph_brush_b200/csrc/ref_api_shim.cu, against the same driver built with
the reference's own energy sources.  Same input, same seed: the same pair
count, energies within FP32 rounding of the reference, and the same trajectory
(every phase's accept counts and pools)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "MC_ref")
DROPIN_BIN = os.path.join(ROOT, "oracle", "_ref", "MC_phmc")
INPUTS = os.path.join(ROOT, "tests", "golden", "inputs")
RTOL = 2e-5  # the reference accumulates in FP32


def run(binary, workdir):
    os.makedirs(workdir)
    shutil.copy(os.path.join(INPUTS, "dropin_small.data"), os.path.join(workdir, "in.data"))
    shutil.copy(os.path.join(INPUTS, "dropin_small.params"), os.path.join(workdir, "params.in"))
    r = subprocess.run([binary, "in.data", "params.in"], cwd=workdir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (binary, r.returncode, r.stderr[-500:])
    return open(os.path.join(workdir, "report.txt")).read()


NUM = r"-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?"


def numbers(line):
    return re.findall(NUM, line)


@pytest.mark.gpu
def test_reference_driver_over_the_engine_matches_the_reference_build(tmp_path):
    if not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)):
        pytest.skip("reference driver binaries not built (make -C oracle mc-ref dropin, needs the reference sources)")
    ref = run(REF_BIN, str(tmp_path / "ref")).splitlines()
    got = run(DROPIN_BIN, str(tmp_path / "dropin")).splitlines()
    assert len(ref) == len(got), (len(ref), len(got))
    energy_keys = ("E_LJ", "E_Coulomb", "E_total", "[summary]", "[sgmc]", "step=")
    checked = 0
    for a, b in zip(ref, got):
        na, nb = numbers(a), numbers(b)
        if any(k in a for k in energy_keys):
            # integers (counts, steps) equal, energies within FP32 rounding of the reference
            assert len(na) == len(nb), (a, b)
            for x, y in zip(na, nb):
                if not any(c in x + y for c in ".eE"):
                    assert x == y, (a, b)  # counts and steps
                else:
                    assert abs(float(x) - float(y)) <= RTOL * abs(float(x)) + 1e-3, (a, b)
            checked += 1
        else:
            assert a == b, (a, b)
    assert checked >= 6
    assert any("[phase2]" in line and "accepted=" in line for line in got)
