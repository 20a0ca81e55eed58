"""Writes the drop-in workflow fixture (tests/golden/inputs/dropin_small.data,
.params): a small brush in the reference's model and input format with a W-bead
pool, and phase settings short enough for a test, so that the reference's own
driver (MC/src/main.cu: protonation phase and phase-2 swaps) can run it both in
its own build and linked against the engine's reference-API shim.
dropin_gc.params runs the same system through a longer protonation phase;
dropin_already.params sets the target to the current protonation (29 of 108
sites), so the protonation phase reports "already at target" in the stream
state the plan summary left behind.
With --large DIR it writes instead the timing input of the drop-in builds: the
config-2 system (10x10 chains of 50, ~17k atoms with the W pool) in the
reference's model, target 95 % (the direct protonation phase) and 3000
phase-2 attempts.
Usage: python tests/golden/make_dropin_inputs.py [--large DIR]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ph_brush_b200 import configs  # noqa: E402

PHASES = {"target_pct": "30", "rng_seed": "2025", "max_attempts": "1500", "patience": "400",
          "energy_interval": "100", "gc_block_fixed": "300", "sgmc_epoch_attempt_max": "1500", "phase2_wc": "yes"}
# the same system with a protonation phase of many blocks and mu updates (dropin_gc.params)
PHASES_GC = dict(PHASES, target_pct="35", gc_block_fixed="10", sgmc_epoch_attempt_max="40")
# target = the current protonation: floor(27.32 / 100 * 108) = 29 (dropin_already.params)
PHASES_ALREADY = dict(PHASES, target_pct="27.32")


LARGE = {"target_pct": "95", "rng_seed": "2025", "max_attempts": "3000", "patience": "100000",
         "energy_interval": "500", "gc_block_fixed": "1000", "sgmc_epoch_attempt_max": "3000", "phase2_wc": "yes"}


def large(out):
    s2, _ = configs.config2()
    s, p = configs.to_reference_semantics(s2, n_w=s2.meta["n_sites"], spacing=0.5, seed=6)
    os.makedirs(out, exist_ok=True)
    configs.write_lammps_data(os.path.join(out, "in.data"), s)
    configs.write_params_in(os.path.join(out, "params.in"), p, 0.5, extra=LARGE)


def main():
    if len(sys.argv) == 3 and sys.argv[1] == "--large":
        large(sys.argv[2])
        return
    small, _ = configs.small_system(seed=9, chains=3, length=12, box_xy=12.0, height=14.0, salt_pairs=6, ion_frac=0.2)
    s, p = configs.to_reference_semantics(small, n_w=small.meta["n_sites"], spacing=0.5, seed=6)
    os.makedirs(os.path.join(HERE, "inputs"), exist_ok=True)
    configs.write_lammps_data(os.path.join(HERE, "inputs", "dropin_small.data"), s)
    configs.write_params_in(os.path.join(HERE, "inputs", "dropin_small.params"), p, 0.5, extra=PHASES)
    configs.write_params_in(os.path.join(HERE, "inputs", "dropin_gc.params"), p, 0.5, extra=PHASES_GC)
    configs.write_params_in(os.path.join(HERE, "inputs", "dropin_already.params"), p, 0.5, extra=PHASES_ALREADY)


if __name__ == "__main__":
    main()
