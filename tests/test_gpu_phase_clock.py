"""Phase clocks of the MC kernel (phmc_set_phase_clock / phmc_get_phase_cycles).

Measuring must not change the chain: a run with the clocks on leaves the same
state, bit for bit, as the same run with them off; the counters cover every
trial run and every phase a trial of the move mix reaches.
"""
import numpy as np
import pytest

from ph_brush_b200 import Engine, _abi, configs


@pytest.mark.gpu
def test_phase_clocks_leave_the_chain_unchanged_and_count_every_trial():
    reps = [configs.small_system(seed=40 + k, p_swap=0.1, salt_conc=0.02) for k in range(3)]
    states = []
    for on in (False, True):
        with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
            e.set_phase_clock(on)
            e.run(1500)
            pc = e.phase_cycles(reset=True)
            states.append([e.state(r) for r in range(len(reps))])
            if on:
                assert pc["trials"] == 3 * 1500
                e.run(100)
                assert e.phase_cycles()["trials"] == 3 * 100
                for k in ("proposal", "cells_stencils_direct", "offsets_pair_tables", "candidate_pairs",
                          "phi_pending_reduce", "decision_commit"):
                    assert pc[k] > 0, k
                assert pc["first_stage"] >= 0 and pc["ended_early"] >= 0
                again = e.phase_cycles(reset=True)
                assert all(again[k] > 0 for k in ("proposal", "decision_commit"))
            else:
                assert all(pc[k] == 0 for k in _abi.PHASES)
    for a, b in zip(*states):
        for k in ("x", "y", "z", "q", "type", "flags"):
            assert np.array_equal(a[k], b[k]), k


def test_phase_clock_refuses_a_null_engine():
    lib = _abi.lib()
    assert lib.phmc_set_phase_clock(None, 1) == 1
