"""Failure paths of the device code, forced without faulting anything.

* A cell list too small for the generated system: the cell-assignment kernel
  counts every member but stores only cell_cap of them and raises
  PHMC_ERR_CAPACITY in the replica's state; engine creation reports it.
* A cell that fills up during a displacement run: the MC kernel refuses the
  move's cell insertion, raises PHMC_ERR_CAPACITY, and the replica's block stops
  at its next proposal; phmc_run reports it.  The system and seed are ones on
  which the oracle's Monte Carlo (the same proposal stream) pushes a cell past
  its initial maximum occupancy within the first ~120 trials.
* A launch budget of one: phmc_run returns PHMC_ERR_BUDGET between launches,
  and the engine continues consistently once the budget is lifted.
"""
import numpy as np
import pytest

from ph_brush_b200 import Engine, _abi, configs


@pytest.mark.gpu
def test_cell_capacity_exceeded_at_creation_is_reported():
    s, p = configs.config1()
    p.cell_cap = 2
    with pytest.raises(_abi.PhmcError) as ei:
        Engine(s, p)
    assert ei.value.code == 3 and "capacity" in str(ei.value)


@pytest.mark.gpu
def test_cell_filled_by_a_displacement_is_reported():
    s, p = configs.small_system(seed=5)
    p.p_disp, p.p_titr, p.p_swap = 1.0, 0.0, 0.0
    with Engine(s, p) as e:
        cells, _ = e.cells()
    occ = np.bincount(cells[cells >= 0]).max()
    p.cell_cap = int(occ)
    with Engine(s, p) as e:
        with pytest.raises(_abi.PhmcError) as ei:
            e.run(5000)
        assert ei.value.code == 3 and "capacity" in str(ei.value)


@pytest.mark.gpu
def test_launch_budget_stops_a_run_between_launches():
    s, p = configs.small_system(seed=6)
    p.pending_max = 6  # many launches for the run below
    with Engine(s, p) as e:
        e.set_launch_budget(1)
        with pytest.raises(_abi.PhmcError) as ei:
            e.run(4000)
        assert ei.value.code == 4
        e.set_launch_budget(0)
        st = e.run(2000)[0]
        fresh = e.energy()[0]["total"]
    assert abs(st["energy"] - fresh) <= 1e-6 * abs(fresh) + 1e-3, (st["energy"], fresh)


def test_launch_budget_refuses_a_null_engine():
    """Host-side argument check (no device needed: a null engine is refused first)."""
    lib = _abi.lib()
    assert lib.phmc_set_launch_budget(None, 1) == 1
