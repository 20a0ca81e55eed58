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


def _with_state(s, st):
    """A copy of SystemArrays s holding every slot of state st (empty slots flagged)."""
    import copy
    out = copy.deepcopy(s)
    for k in ("x", "y", "z", "q"):
        setattr(out, k, np.ascontiguousarray(st[k], np.float32))
    out.type = np.ascontiguousarray(st["type"], np.int32)
    out.flags = np.ascontiguousarray(st["flags"], np.int32)
    out.capacity = len(st["x"])
    return out


@pytest.mark.gpu
def test_state_upload_one_and_all_replicas():
    """phmc_set_state for one replica and for all replicas at once (concatenated
    arrays): lists, cells and the potential mesh are rebuilt, the energies are those
    of the uploaded states (FP64 oracle), and the chains continue from them."""
    from oracle import pyoracle as O
    reps = ragged_set()
    S, P = [s for s, _ in reps], [p for _, p in reps]
    with Engine(S, P) as e:
        e.run(800)
        st_all = e.state(-1)
        # perturb: flip the charge state of one titratable site of replica 1 (slot arrays of all replicas)
        off = sum(e.caps[:1])
        f1 = st_all["flags"][off:off + e.caps[1]]
        site = int(np.nonzero((f1 & 2) != 0)[0][0])
        st_all["q"][off + site] = 1.0 - st_all["q"][off + site]
        st_all["type"][off + site] = 1 - st_all["type"][off + site]
        e.set_state(st_all, -1)
        got = [c["total"] for c in e.energy()]
        for r in range(len(reps)):
            o = sum(e.caps[:r])
            sub = {k: v[o:o + e.caps[r]] for k, v in st_all.items()}
            ref = O.energy(_with_state(S[r], sub), P[r])["total"]
            assert abs(got[r] - ref) <= 1e-6 * abs(ref) + 1e-4, (r, got[r], ref)
        # one replica: put replica 2 back to its generated state
        g = S[2]
        cap = e.caps[2]
        one = {"x": np.zeros(cap, np.float32), "y": np.zeros(cap, np.float32), "z": np.zeros(cap, np.float32),
               "q": np.zeros(cap, np.float32), "type": np.zeros(cap, np.int32), "flags": np.full(cap, 4, np.int32)}
        for k in ("x", "y", "z", "q", "type", "flags"):
            one[k][:g.n] = getattr(g, k)
        e.set_state(one, 2)
        assert abs(e.energy()[2]["total"] - O.energy(g, P[2])["total"]) <= 1e-6 * abs(O.energy(g, P[2])["total"]) + 1e-4
        st = e.run(600)
        fresh = e.energy()
        for a, b in zip(st, fresh):
            assert abs(a["energy"] - b["total"]) <= 1e-6 * abs(b["total"]) + 1e-3
        assert all(0 <= x["n_charged_sites"] <= x["n_titratable"] for x in st)
