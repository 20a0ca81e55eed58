"""Batched replicas: every replica is an independent Markov chain, so a batched
run (ragged particle counts, meshes and boxes in one launch per phase) must
reproduce each replica's solo run bit for bit, and each replica's tracked
energy must match a full recompute."""
import numpy as np
import pytest

from ph_brush_b200 import Engine, configs


def ragged_set():
    out = []
    for k, (chains, length, box, mesh) in enumerate([(2, 6, 12.0, (16, 16, 48)), (3, 8, 12.0, (24, 24, 48)),
                                                      (2, 10, 16.0, (32, 32, 54)), (3, 5, 15.0, (20, 20, 60))]):
        s, p = configs.small_system(seed=40 + k, chains=chains, length=length, box_xy=box, height=box, mesh=mesh)
        p.pending_max = 12
        out.append((s, p))
    return out


@pytest.mark.gpu
def test_batched_equals_solo_runs():
    reps = ragged_set()
    with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
        e.run(1500)
        batched = [e.state(r) for r in range(len(reps))]
        eb = [c["total"] for c in e.energy()]
    for r, (s, p) in enumerate(reps):
        with Engine(s, p) as e1:
            e1.run(1500)
            solo = e1.state()
            es = e1.energy()[0]["total"]
        for k in solo:
            assert np.array_equal(batched[r][k], solo[k]), (r, k)
        assert abs(eb[r] - es) <= 1e-9 * abs(es) + 1e-9


@pytest.mark.gpu
def test_batched_tracked_energy():
    reps = ragged_set()
    with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
        st = e.run(2000)
        fresh = e.energy()
    for r in range(len(reps)):
        assert abs(st[r]["energy"] - fresh[r]["total"]) <= 1e-6 * abs(fresh[r]["total"]) + 1e-3


@pytest.mark.gpu
def test_config3_replicas_build_and_run():
    reps = configs.config3(n_rep=6)
    with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
        st = e.run(300)
    assert all(s_["attempted"][0] > 0 for s_ in st)
