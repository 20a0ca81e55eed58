"""z-density profiles accumulated by the MC kernel (phmc_set_zhist / phmc_get_zhist).

A sample taken at the end of a run must equal the histogram of the state the
engine hands back (computed here on the host), bin for bin; samples are taken
exactly when a replica's trial count reaches a multiple of `every`, in every
replica of a batched engine; the profile gives the degree of ionisation.
"""
import numpy as np
import pytest

from ph_brush_b200 import Engine, _abi, configs


def host_hist(st, p, nb):
    pres = (st["flags"] & _abi.F_GHOST) == 0
    cls = np.full(len(pres), -1)
    tit = (st["flags"] & _abi.F_TITRATABLE) != 0
    cls[tit & (st["q"] != 0)] = 0
    cls[~tit & ((st["flags"] & _abi.F_ANION) != 0)] = 1
    cls[~tit & ((st["flags"] & _abi.F_ANION) == 0) & ((st["flags"] & _abi.F_CATION) != 0)] = 2
    keep = pres & (cls >= 0)
    z = st["z"][keep].astype(np.float32)
    inv = np.float32(nb) / np.float32(p.wall_hi - p.wall_lo)
    b = np.clip(((z - np.float32(p.wall_lo)) * inv).astype(np.int64), 0, nb - 1)
    h = np.zeros((3, nb))
    np.add.at(h, (cls[keep], b), 1)
    return h


@pytest.mark.gpu
def test_end_of_run_sample_equals_the_host_histogram_of_the_state():
    s, p = configs.small_system(seed=12, p_swap=0.1, salt_conc=0.02)
    s.capacity += 20
    nb = 12
    with Engine(s, p) as e:
        e.run(500)
        e.set_zhist(nb, every=1500)
        e.run(1000)  # trial 1500 is the first multiple: one sample, the state after it
        h, n = e.zhist()
        st = e.state()
    assert n == 1
    assert np.array_equal(h, host_hist(st, p, nb))


@pytest.mark.gpu
def test_samples_every_k_trials_in_every_replica():
    reps = [configs.small_system(seed=70 + k) for k in range(3)]
    with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
        e.set_zhist(8, every=100)
        st = e.run(1000)
        for r, (s, _) in enumerate(reps):
            h, n = e.zhist(r)
            assert n == 10
            alpha = h[0].sum() / (n * s.meta["n_sites"])
            assert 0.0 <= alpha <= 1.0
            assert h[0].sum() <= n * s.meta["n_sites"]
        e.set_zhist(0)
        with pytest.raises(_abi.PhmcError):
            e.zhist(0)
    assert all(x["attempted"][0] > 0 for x in st)
