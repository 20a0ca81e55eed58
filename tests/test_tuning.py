"""Tuning: the pending-stencil capacity, the block size and the tile shapes (z pass
of the rebuild, the pair pass's round width, the full recompute's block size)
change between runs without changing the physics, and the autotuner keeps the
fastest candidate of each of its stages."""
import numpy as np
import pytest

from ph_brush_b200 import Engine, _abi, configs


@pytest.mark.gpu
def test_retuning_keeps_tracked_energy_consistent():
    s, p = configs.config1(seed=51)
    with Engine(s, p) as e:
        for pend, th in ((8, 128), (64, 256), (16, 256), (48, 128)):
            e.set_tuning(pend, th)
            assert e.tuning()["pending_max"] == pend and e.tuning()["threads"] == th
            st = e.run(3000)[0]
            fresh = e.energy()[0]["total"]
            assert abs(st["energy"] - fresh) <= 1e-6 * abs(fresh) + 1e-3, (pend, th, st["energy"], fresh)


@pytest.mark.gpu
@pytest.mark.parametrize("tiles", [(-1, -1, -1, -1), (0, 2, 64, -1), (-1, 8, 256, -1), (-1, 2, -1, 4),
                                   (0, 2, 0, 3), (-1, 2, -1, 21), (-1, 4, -1, 21)])
def test_tuning_leaves_the_trial_stream_unchanged_on_a_short_run(tiles):
    """Same seed, different tuning and tile shapes (config 1's nz = 128: the Stockham
    z pass against the register split; pair-pass rounds of 2 and 8 candidates; 3 and 4 G
    rows in flight, and one pair per warp with lanes over its plane; full recompute blocks of 64 and 256 and the cell-ordered pass): the same proposals;
    decisions agree unless a dE
    sits within FP32 rounding of its acceptance threshold (none on a short run)."""
    s, p = configs.config1(seed=52)
    logs = []
    for k, (pend, th) in enumerate(((8, 128), (48, 256))):
        with Engine(s, p) as e:
            e.set_tuning(pend, th)
            if k == 1:
                e.set_tile_shapes(zpass=tiles[0], cand_round=tiles[1], energy_block=tiles[2], g_rows=tiles[3])
                t = e.tuning()
                assert tiles[1] < 0 or t["cand_round"] == tiles[1]
                assert tiles[0] < 0 or t["zpass"] == tiles[0]
                assert tiles[3] < 0 or t["g_rows"] == tiles[3]
            log = e.set_trial_log(4000)
            e.run(4000)
            logs.append((log[0].copy(), log[1].copy(), log[2].copy()))
    (m0, d0, a0), (m1, d1, a1) = logs
    assert np.array_equal(m0, m1)
    assert np.array_equal(a0, a1)
    fin = np.isfinite(d0) & np.isfinite(d1)
    assert np.allclose(d0[fin], d1[fin], rtol=1e-5, atol=1e-4)


@pytest.mark.gpu
def test_autotune_keeps_the_fastest_candidate():
    S, P = [], []
    for k in range(4):
        s, p = configs.config1(seed=60 + k)
        S.append(s)
        P.append(p)
    with Engine(S, P) as e:
        res = e.autotune(1500)
        zp = [r for r in res if r["rebuild_us"] > 0]
        eb = [r for r in res if r["recompute_us"] > 0]
        runs = [r for r in res if r["us_per_trial"] > 0]
        grid = [r for r in runs if r["cand_round"] == 4]
        assert len(zp) >= 2 and {r["zpass"] for r in zp} >= {0, 2}  # Stockham and nz = 128's default split
        assert {r["energy_block"] for r in eb} == {0, 64, 128, 256}
        assert len(grid) >= 10 and {r["cand_round"] for r in runs} == {2, 4, 8}
        assert {(r["cand_round"], r["g_rows"]) for r in runs} >= {(2, 2), (8, 2), (2, 3), (2, 4), (2, 21), (4, 21)}
        t = e.tuning()
        best = min(grid, key=lambda r: r["us_per_trial"])
        assert (t["pending_max"], t["threads"]) == (best["pending_max"], best["threads"])
        shapes = [best] + [r for r in runs if (r["cand_round"], r["g_rows"]) != (4, 2)]
        fastest = min(shapes, key=lambda r: r["us_per_trial"])
        assert (t["cand_round"], t["g_rows"]) == (fastest["cand_round"], fastest["g_rows"])
        assert t["zpass"] == min(zp, key=lambda r: r["rebuild_us"])["zpass"]
        assert t["energy_block"] == min(eb, key=lambda r: r["recompute_us"])["energy_block"]
        st = e.run(2000)
        fresh = e.energy()
        for a, b in zip(st, fresh):
            assert abs(a["energy"] - b["total"]) <= 1e-6 * abs(b["total"]) + 1e-3


@pytest.mark.gpu
def test_launch_quorum_keeps_the_chains_and_energies():
    """A launch quorum ends MC launches early for the replicas that have not filled
    their pending buffers: more rebuilds, the same proposals and decisions (up to
    FP32 rounding of the reciprocal dE), tracked energies equal to a recompute."""
    S, P = [], []
    for k in range(4):
        s, p = configs.config1(seed=70 + k)
        S.append(s)
        P.append(p)
    logs, flushes = [], []
    for q in (1.0, 0.25):
        with Engine(S, P) as e:
            e.set_tuning(16, 256)
            e.set_quorum(q)
            log = e.set_trial_log(3000)
            st = e.run(3000)
            logs.append((log[0].copy(), log[1].copy(), log[2].copy()))
            flushes.append(sum(d["flushes"] for d in st))
            for a, b in zip(st, e.energy()):
                assert abs(a["energy"] - b["total"]) <= 1e-6 * abs(b["total"]) + 1e-3, (q, a["energy"], b["total"])
    (m0, d0, a0), (m1, d1, a1) = logs
    assert np.array_equal(m0, m1)
    assert np.array_equal(a0, a1)
    fin = np.isfinite(d0) & np.isfinite(d1)
    assert np.allclose(d0[fin], d1[fin], rtol=1e-5, atol=1e-4)
    assert flushes[1] >= flushes[0], flushes


def test_tuning_arguments_are_checked_without_a_gpu():
    lib = _abi.lib()
    assert lib.phmc_set_tile_shapes(None, 0, 4, 2, 128, 0) != 0
    assert lib.phmc_set_tuning(None, 16, 256) != 0
    assert lib.phmc_autotune(None, 100, None, 0, None) != 0
    assert lib.phmc_set_quorum(None, 0.5) != 0


@pytest.mark.gpu
def test_pipelined_first_pass_gives_the_same_chains_bit_for_bit():
    """The rebuild's first pass with bulk-copied planes (persistent blocks) computes the
    same arithmetic on the same fixed-point charges as one block per plane: a batched
    run under either gives identical states and energies (launch quorum 1)."""
    reps = [configs.small_system(seed=90 + k, mesh=(n, n, 48)) for k, n in enumerate((32, 36, 48, 64))]
    S, P = [s for s, _ in reps], [p for _, p in reps]
    out = []
    for pipe in (0, 1):
        with Engine(S, P) as e:
            e.set_quorum(1.0)
            e.set_tuning(16, 256)
            e.set_tile_shapes(plane_pipe=pipe)
            assert e.tuning()["plane_pipe"] == pipe
            st = e.run(3000)
            out.append(([e.state(r) for r in range(len(S))], [x["energy"] for x in st], e.energy()))
    (s0, e0, f0), (s1, e1, f1) = out
    for a, b in zip(s0, s1):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    assert e0 == e1
    assert [x["total"] for x in f0] == [x["total"] for x in f1]


@pytest.mark.gpu
def test_pair_shapes_agree_on_a_config5_replica():
    """Every compiled pair-pass shape on the smallest config-5 replica (its 48 x 48 x 243 mesh,
    48 pending stencils): the same proposals and decisions from the same state, and trial dE
    within 1e-6 relative (1e-4 kT) of the default shape's."""
    reps = configs.config5(seed=2029, n_rep=256)
    s, p = min(reps, key=lambda r: r[0].n)
    logs = []
    for shape in ((4, 2), (2, 2), (8, 2), (2, 3), (2, 4), (2, 21), (4, 21)):
        with Engine(s, p) as e:
            e.set_tuning(48, 256)
            e.set_tile_shapes(cand_round=shape[0], g_rows=shape[1])
            e.run(500)
            log = e.set_trial_log(1500)
            e.run(1500)
            logs.append((shape, log[0].copy(), log[1].copy(), log[2].copy()))
    _, m0, d0, a0 = logs[0]
    for shape, m, dd, a in logs[1:]:
        assert np.array_equal(m0, m), shape
        assert np.array_equal(a0, a), shape
        fin = np.isfinite(d0) & np.isfinite(dd)
        assert np.allclose(dd[fin], d0[fin], rtol=1e-6, atol=1e-4), shape
