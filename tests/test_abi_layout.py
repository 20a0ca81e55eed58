"""The ctypes mirrors of include/phmc.h (ph_brush_b200/_abi.py) against the C
compiler's layout: every mirrored struct's size and every field's offset, from
a program compiled against the header (no device needed)."""
import ctypes as C
import os
import subprocess

from ph_brush_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = {
    "phmc_system": _abi.System, "phmc_params": _abi.Params, "phmc_energy_components": _abi.EnergyComponents,
    "phmc_change": _abi.Change, "phmc_trial": _abi.Trial, "phmc_run_stats": _abi.RunStats,
    "phmc_tuning": _abi.Tuning, "phmc_lammps_info": _abi.LammpsInfo, "phmc_file_params": _abi.FileParams,
    "phmc_profile": _abi.Profile, "phmc_da_stats": _abi.DAStats, "phmc_brush_spec": _abi.BrushSpec,
    "phmc_gc_event": _abi.GcEvent, "phmc_gc_job": _abi.GcJob, "phmc_gc_result": _abi.GcResult,
    "phmc_phase2_event": _abi.Phase2Event, "phmc_phase2_job": _abi.Phase2Job, "phmc_phase2_result": _abi.Phase2Result,
}


def test_ctypes_mirrors_match_the_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "phmc.h"', "int main(void) {"]
    for cname, py in PAIRS.items():
        lines.append(f'    printf("{cname} . %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, v = ln.split()
        got[(s, f)] = int(v)
    bad = []
    for cname, py in PAIRS.items():
        if got[(cname, ".")] != C.sizeof(py):
            bad.append((cname, "sizeof", got[(cname, ".")], C.sizeof(py)))
        for f in py._fields_:
            off = getattr(py, f[0]).offset
            if got[(cname, f[0])] != off:
                bad.append((cname, f[0], got[(cname, f[0])], off))
    assert not bad, bad
