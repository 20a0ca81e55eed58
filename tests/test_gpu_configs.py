"""Parity at the benchmark's own configurations, against the FP64 oracle.

The timed workloads run kernels that the small systems of the other parity
tests do not reach: the register z pass of the potential-mesh rebuild is one
template instance per mesh depth (nz = N1 x N2, two register stages), the
first and last plane passes one per lateral mesh, and a batched engine whose
replicas differ in nz takes the shared-memory Stockham z pass instead.  Here
every one of those variants, the three lateral meshes of the config-5 replica
set (48, 54, 64 x 243), config 2 (64 x 64 x 384) and config-3 replicas of each
depth are held to the oracle:

* energy components of the generated and of a relaxed state;
* trial dE of displacement, protonation (counterion insertion / deletion) and
  salt-pair moves against two oracle energies;
* the energy the engine tracks through a 2000-trial run against the oracle's
  energy of the final state;
* a batched 8-replica config-5 engine, replica for replica.

Tolerances (FP32 pair terms and mesh, FP64 sums): 1e-6 relative or 1e-4 kT per
component and per dE; 2e-5 relative for dE beyond 20 kT (hard-core overlaps,
acceptance < e^-20, where (sigma/r)^12 amplifies the FP32 rounding of r^2);
tracked energies 1e-6 relative + 1e-3 kT after thousands of accepted moves.
"""
import copy

import numpy as np
import pytest

from oracle import pyoracle as O
from ph_brush_b200 import Engine, _abi, configs

RTOL, ATOL = 1e-6, 1e-4
DE_DECISIVE, RTOL_OVERLAP = 20.0, 2e-5
COMPS = ("lj", "fene", "coul_real", "coul_recip", "self", "qcorr", "slab", "total")
# nz of the register z-pass variants (k_rebuild.cu) and two Stockham-only depths
ZREG_NZ = (48, 128, 162, 192, 216, 243, 256, 288, 384)
STOCKHAM_NZ = (200, 320)


def close(a, b, rtol=RTOL, atol=ATOL):
    return abs(a - b) <= rtol * abs(b) + atol


def assert_components(got, ref, rtol=RTOL, atol=ATOL, what="", overlaps=False):
    """Every component within rtol / atol; with overlaps=True (a generated state, whose
    randomly placed ions overlap beads: pair energies of 1e6-1e7 kT) the pair term and
    the total within RTOL_OVERLAP, the rule for hard-core dE."""
    def rt(k):
        return RTOL_OVERLAP if overlaps and k in ("lj", "total") else rtol
    bad = {k: (got[k], ref[k]) for k in COMPS if not close(got[k], ref[k], rt(k), atol)}
    assert not bad, (what, bad)


def with_state(s, st):
    """A copy of SystemArrays s holding every slot of engine state st (empty slots flagged)."""
    out = copy.deepcopy(s)
    for k in ("x", "y", "z", "q"):
        setattr(out, k, np.ascontiguousarray(st[k], np.float32))
    out.type = np.ascontiguousarray(st["type"], np.int32)
    out.flags = np.ascontiguousarray(st["flags"], np.int32)
    out.capacity = len(st["x"])
    return out


def trials_for(s, p, rng, n):
    """n trials cycling displacement, protonation with counterion insertion,
    deprotonation with anion deletion, salt-pair insertion and anion deletion."""
    pres = np.flatnonzero((s.flags & _abi.F_GHOST) == 0)
    mobile = pres[(s.flags[pres] & _abi.F_MOBILE) != 0]
    sites = pres[(s.flags[pres] & _abi.F_TITRATABLE) != 0]
    anions = pres[(s.flags[pres] & _abi.F_ANION) != 0]
    free = np.flatnonzero(s.flags & _abi.F_GHOST)
    H = p.wall_hi
    out = []
    for k in range(n):
        kind = k % 4
        if kind == 0:
            i = int(rng.choice(mobile))
            x = float((s.x[i] + rng.uniform(-0.3, 0.3)) % s.box[0])
            y = float((s.y[i] + rng.uniform(-0.3, 0.3)) % s.box[1])
            z = float(min(max(s.z[i] + rng.uniform(-0.3, 0.3), p.wall_lo), H - 1e-3))
            out.append([dict(index=i, x=x, y=y, z=z, q=s.q[i], type=s.type[i])])
        elif kind == 1:
            i = int(rng.choice(sites))
            if s.q[i] == 0:
                g = int(free[k % len(free)])
                out.append([dict(index=i, x=s.x[i], y=s.y[i], z=s.z[i], q=1.0, type=1),
                            dict(index=g, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]),
                                 z=rng.uniform(p.wall_lo, H), q=-1.0, type=2)])
            else:
                a = int(rng.choice(anions))
                out.append([dict(index=i, x=s.x[i], y=s.y[i], z=s.z[i], q=0.0, type=0),
                            dict(index=a, present=0, x=s.x[a], y=s.y[a], z=s.z[a], q=s.q[a], type=s.type[a])])
        elif kind == 2:
            g1, g2 = int(free[0]), int(free[1])
            out.append([dict(index=g1, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]),
                             z=rng.uniform(p.wall_lo, H), q=1.0, type=3),
                        dict(index=g2, x=rng.uniform(0, s.box[0]), y=rng.uniform(0, s.box[1]),
                             z=rng.uniform(p.wall_lo, H), q=-1.0, type=2)])
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
            if t.flags[i] & _abi.F_GHOST:
                t.flags[i] = _abi.F_MOBILE | (_abi.F_ANION if c["q"] < 0 else _abi.F_CATION if c["q"] > 0 else 0)
        else:
            t.flags[i] = _abi.F_GHOST
    return t


def relaxed(e, s, trials):
    """Run the engine to clear the generator's overlaps, then reload its own state so
    that the tracked energies start from a full recompute."""
    e.run(trials)
    st = e.state()
    e.set_state(st)
    return with_state(s, st)


def check_config(s, p, n_dE=52, relax=None, run=2000, seed=0):
    """Generated-state energy, relaxed-state energy, trial dE and tracked energy of one
    replica against the oracle."""
    with Engine(s, p) as e:
        assert_components(e.energy()[0], O.energy(s, p), what="generated state", overlaps=True)
        cur = relaxed(e, s, relax if relax is not None else 20 * s.n)
        e0 = O.energy(cur, p)
        assert_components(e.energy()[0], e0, what="relaxed state")
        trials = trials_for(cur, p, np.random.default_rng(seed), n_dE)
        dE = e.delta_energy(trials)
        bad = []
        for k, tr in enumerate(trials):
            ref = O.energy(apply_host(cur, tr), p)["total"] - e0["total"]
            rt = RTOL if abs(ref) <= DE_DECISIVE else RTOL_OVERLAP
            if not abs(dE[k] - ref) <= rt * abs(ref) + ATOL:
                bad.append((k, len(tr), dE[k], ref))
        assert not bad, bad[:8]
        st = e.run(run)[0]
        assert sum(st["accepted"]) > 0
        fin = with_state(s, e.state())
    ref = O.energy(fin, p)["total"]
    assert abs(st["energy"] - ref) <= 1e-6 * abs(ref) + 1e-3, (st["energy"], ref)


@pytest.mark.gpu
@pytest.mark.parametrize("nz", ZREG_NZ + STOCKHAM_NZ)
def test_every_z_pass_depth_matches_the_oracle(nz):
    """Each register z-pass variant (and the Stockham pass for depths without one) on a
    small brush: energy components, and after a run the tracked energy."""
    s, p = configs.small_system(seed=60 + nz % 17, mesh=(16, 16, nz))
    with Engine(s, p) as e:
        assert_components(e.energy()[0], O.energy(s, p), what=f"nz={nz}")
        st = e.run(1500)[0]
        fin = with_state(s, e.state())
        assert_components(e.energy()[0], O.energy(fin, p), what=f"nz={nz} after run")
    ref = O.energy(fin, p)["total"]
    assert abs(st["energy"] - ref) <= 1e-6 * abs(ref) + 1e-3, (st["energy"], ref)


def config5_by_lateral_mesh():
    reps = configs.config5(n_rep=256)
    out = {}
    for k, (s, p) in enumerate(reps):
        out.setdefault(p.mesh[0], (k, s, p))
    return [out[m] for m in sorted(out)]


@pytest.mark.gpu
@pytest.mark.parametrize("lateral", [48, 54, 64])
def test_config5_replica_matches_the_oracle(lateral):
    """One config-5 replica per lateral mesh (nz 243: the headline's register z pass
    k_rb_zreg<27, 9>), at full size."""
    k, s, p = {pp.mesh[0]: (kk, ss, pp) for kk, ss, pp in config5_by_lateral_mesh()}[lateral]
    assert tuple(p.mesh) == (lateral, lateral, 243)
    check_config(s, p, seed=k)


@pytest.mark.gpu
def test_config2_matches_the_oracle():
    """Config 2 at full size: 64 x 64 x 384 (register z pass k_rb_zreg<32, 12>)."""
    s, p = configs.config2()
    assert tuple(p.mesh) == (64, 64, 384)
    check_config(s, p, seed=2)


@pytest.mark.gpu
def test_config3_replica_of_every_depth_matches_the_oracle():
    """A config-3 replica of every mesh depth (162 ... 288), each alone (register z
    pass), then all of them in one batched engine (the depths differ: Stockham z pass)."""
    reps = configs.config3()
    by_nz = {}
    for s, p in reps:
        by_nz.setdefault(p.mesh[2], (s, p))
    assert sorted(by_nz) == [162, 192, 216, 243, 256, 288]
    picked = [by_nz[n] for n in sorted(by_nz)]
    refs = [O.energy(s, p) for s, p in picked]
    for (s, p), ref in zip(picked, refs):
        with Engine(s, p) as e:
            assert_components(e.energy()[0], ref, what=f"config 3 mesh {p.mesh}", overlaps=True)
    with Engine([s for s, _ in picked], [p for _, p in picked]) as e:
        for (s, p), got, ref in zip(picked, e.energy(), refs):
            assert_components(got, ref, what=f"config 3 batched, mesh {p.mesh}", overlaps=True)
        sts = e.run(3000)
        fin = [with_state(s, e.state(r)) for r, (s, _) in enumerate(picked)]
    for st, f, (s, p) in zip(sts, fin, picked):
        ref = O.energy(f, p)["total"]
        assert abs(st["energy"] - ref) <= 1e-6 * abs(ref) + 1e-3, (p.mesh, st["energy"], ref)


@pytest.mark.gpu
def test_batched_config5_replicas_match_the_oracle_replica_for_replica():
    """Eight config-5 replicas (all three lateral meshes) in one engine: each replica's
    energy equals the oracle's energy of that replica alone, at the generated state and
    after 2000 trials per replica (tracked energies against the final states)."""
    reps = configs.config5(n_rep=256)
    meshes = {}
    for k, (s, p) in enumerate(reps):
        meshes.setdefault(p.mesh[0], []).append(k)
    pick = sorted(meshes[48][:3] + meshes[54][:3] + meshes[64][:2])
    S, P = [reps[k][0] for k in pick], [reps[k][1] for k in pick]
    with Engine(S, P) as e:
        for r, got in enumerate(e.energy()):
            assert_components(got, O.energy(S[r], P[r]), what=f"replica {pick[r]}", overlaps=True)
        e.run(20 * max(s.n for s in S))
        e.set_state(e.state(-1), -1)
        sts = e.run(2000)
        fin = [with_state(S[r], e.state(r)) for r in range(len(S))]
        fresh = e.energy()
    for r in range(len(S)):
        ref = O.energy(fin[r], P[r])
        assert_components(fresh[r], ref, what=f"replica {pick[r]} after the run")
        assert abs(sts[r]["energy"] - ref["total"]) <= 1e-6 * abs(ref["total"]) + 1e-3, (pick[r], sts[r]["energy"])


@pytest.mark.gpu
def test_cell_ordered_full_recompute_matches_the_oracle():
    """The full recompute in cell order (energy_block 0: one warp per cell) on config 2 and
    a config-5 replica: every component against the oracle, as the particle-ordered pass."""
    k, s5, p5 = config5_by_lateral_mesh()[-1]
    for s, p in (configs.config2(), (s5, p5)):
        ref = O.energy(s, p)
        with Engine(s, p) as e:
            e.set_tile_shapes(energy_block=0)
            assert e.tuning()["energy_block"] == 0
            assert_components(e.energy()[0], ref, what="cell order", overlaps=True)
