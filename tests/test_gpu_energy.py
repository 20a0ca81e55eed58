"""Energy parity of the CUDA engine against the FP64 oracle (through the C ABI).

Tolerance (the engine computes pair terms and the mesh in FP32 and sums in
FP64): |E_gpu - E_oracle| <= 1e-6 |E_oracle| + 1e-4 kT per component and per
trial dE.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from ph_brush_b200 import Engine, _abi, configs

RTOL, ATOL = 1e-6, 1e-4
COMPS = ("lj", "fene", "coul_real", "coul_recip", "self", "qcorr", "slab", "total")


def close(a, b, rtol=RTOL, atol=ATOL):
    return abs(a - b) <= rtol * abs(b) + atol


def assert_components(got, ref, rtol=RTOL, atol=ATOL):
    bad = {k: (got[k], ref[k]) for k in COMPS if not close(got[k], ref[k], rtol, atol)}
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 5, 6])
def test_small_system_energy(order):
    s, p = configs.small_system(seed=3, order=order)
    with Engine(s, p) as e:
        got = e.energy()[0]
    assert_components(got, O.energy(s, p))


@pytest.mark.gpu
def test_config1_energy():
    s, p = configs.config1()
    with Engine(s, p) as e:
        got = e.energy()[0]
    assert_components(got, O.energy(s, p))


@pytest.mark.gpu
def test_reference_semantics_energy():
    """Engine with the reference's model (shared LJ cutoff, 1-2 exclusions, cubic
    SPME with the reference's moduli and spacing rule) against the restatement of
    compute_lj_sr_energy_gpu + pmeEnergy (MC/src/energy_gpu.cu:14-75, MC/src/pme.cu:344-457)."""
    sn, _ = configs.config1()
    s, p = configs.to_reference_semantics(sn, n_w=64, spacing=0.5)
    ref = O.ref_energies(s, p)
    with Engine(s, p) as e:
        got = e.energy()[0]
    assert close(got["lj"], ref["lj"]), (got["lj"], ref["lj"])
    assert close(got["coul_real"], ref["real"]), (got["coul_real"], ref["real"])
    assert close(got["coul_recip"], ref["recip"]), (got["coul_recip"], ref["recip"])
    assert close(got["self"], ref["self"])
    assert close(got["qcorr"] + got["slab"], ref["qcorr_slab"])
    assert close(got["total"], ref["lj"] + ref["coul_total"])


def random_trials(s, p, rng, n):
    """Displacements, protonation/deprotonation with counterion insert/delete, pair insert/delete."""
    pres = np.flatnonzero((s.flags & _abi.F_GHOST) == 0)
    mobile = [i for i in pres if s.flags[i] & _abi.F_MOBILE]
    sites = [i for i in pres if s.flags[i] & _abi.F_TITRATABLE]
    anions = [i for i in pres if s.flags[i] & _abi.F_ANION]
    free = [int(i) for i in np.flatnonzero(s.flags & _abi.F_GHOST)] + list(range(s.n, s.capacity))
    H = p.wall_hi
    out = []
    for k in range(n):
        kind = k % 4
        if kind == 0:
            i = int(rng.choice(mobile))
            x = (s.x[i] + rng.uniform(-0.3, 0.3)) % s.box[0]
            y = (s.y[i] + rng.uniform(-0.3, 0.3)) % s.box[1]
            z = min(max(s.z[i] + rng.uniform(-0.3, 0.3), 0.0), H - 1e-3)
            out.append([dict(index=i, x=x, y=y, z=z, q=s.q[i], type=s.type[i])])
        elif kind == 1:
            i = int(rng.choice(sites))
            g = free[k % len(free)]
            newq = 0.0 if s.q[i] != 0 else 1.0
            ch = [dict(index=i, x=s.x[i], y=s.y[i], z=s.z[i], q=newq, type=1 if newq else 0)]
            if newq:
                ch.append(dict(index=g, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]), z=rng.uniform(0, H),
                               q=-1.0, type=2))
            else:
                a = int(rng.choice(anions))
                ch.append(dict(index=a, present=0, x=s.x[a], y=s.y[a], z=s.z[a], q=s.q[a], type=s.type[a]))
            out.append(ch)
        elif kind == 2:
            g1, g2 = free[0], free[1]
            out.append([dict(index=g1, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]), z=rng.uniform(0, H), q=1.0, type=3),
                        dict(index=g2, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]), z=rng.uniform(0, H), q=-1.0, type=2)])
        else:
            a = int(rng.choice(anions))
            out.append([dict(index=a, present=0, x=s.x[a], y=s.y[a], z=s.z[a], q=s.q[a], type=s.type[a])])
    return out


def apply_host(s, changes):
    t = s.copy()
    for c in changes:
        i = c["index"]
        t.x[i], t.y[i], t.z[i], t.q[i], t.type[i] = c["x"], c["y"], c["z"], c["q"], c["type"]
        if c.get("present", 1):
            if t.flags[i] & _abi.F_GHOST or i >= s.n:
                t.flags[i] = _abi.F_MOBILE | (_abi.F_ANION if c["q"] < 0 else _abi.F_CATION if c["q"] > 0 else 0)
        else:
            t.flags[i] = _abi.F_GHOST
    return t


def padded(s):
    """Slots up to capacity as explicit ghosts (so host copies can hold insertions)."""
    n, cap = s.n, s.capacity
    t = s.copy()
    for f in ("x", "y", "z", "q"):
        setattr(t, f, np.concatenate([getattr(s, f), np.zeros(cap - n, np.float32)]))
    t.type = np.concatenate([s.type, np.zeros(cap - n, np.int32)])
    t.flags = np.concatenate([s.flags, np.full(cap - n, _abi.F_GHOST, np.int32)])
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", ["small", "config1"])
def test_delta_energy_matches_oracle(cfg):
    s, p = configs.small_system(seed=4) if cfg == "small" else configs.config1()
    rng = np.random.default_rng(1)
    trials = random_trials(s, p, rng, 24)
    sp = padded(s)
    e0 = O.energy(sp, p)["total"]
    with Engine(sp, p) as e:
        dE = e.delta_energy(trials)
    for k, tr in enumerate(trials):
        ref = O.energy(apply_host(sp, tr), p)["total"] - e0
        if not np.isfinite(ref):
            assert not np.isfinite(dE[k]) or dE[k] > 1e6
            continue
        assert close(dE[k], ref), (k, tr, dE[k], ref)


@pytest.mark.gpu
def test_commit_sequence_matches_oracle():
    s, p = configs.small_system(seed=9)
    sp = padded(s)
    rng = np.random.default_rng(2)
    cur = sp.copy()
    with Engine(sp, p) as e:
        for k in range(6):
            tr = random_trials(cur, p, rng, 4)[k % 4]
            before = O.energy(cur, p)["total"]
            after_sys = apply_host(cur, tr)
            after = O.energy(after_sys, p)["total"]
            if not np.isfinite(after):
                continue
            d = e.delta_energy([tr])[0]
            assert close(d, after - before), (d, after - before)
            e.commit(tr)
            cur = after_sys
            assert_components(e.energy()[0], O.energy(cur, p))


@pytest.mark.gpu
def test_register_plane_passes_match_the_oracle_at_every_lateral_size():
    """The rebuild's first and last passes run in registers for square lateral meshes
    16, 32, 36, 48, 54 and 64 (one kernel, the replica's size picked at run time):
    each size alone, and all four of the larger ones batched in one engine, give the
    oracle's reciprocal energy (and every other component) within the tolerance."""
    sizes = (36, 48, 54, 64)
    reps = [configs.small_system(seed=20 + k, mesh=(n, n, 48)) for k, n in enumerate(sizes)]
    refs = [O.energy(s, p) for s, p in reps]
    for (s, p), ref in zip(reps, refs):
        with Engine(s, p) as e:
            assert_components(e.energy()[0], ref)
    with Engine([s for s, _ in reps], [p for _, p in reps]) as e:
        for got, ref in zip(e.energy(), refs):
            assert_components(got, ref)
