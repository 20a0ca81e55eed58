"""Degree of ionisation alpha(pH) and z-density profiles against the reference's own build.

The reference cannot sample at a fixed pH: its grand-canonical phase steers mu
to a target fraction and stops there (MC/src/mc.cu:468-499,519-530).  Its
reference alpha therefore comes from the reference harness (oracle/_ref/
ref_harness, mode `alpha`): the reference's energy routines and its pair-flip
acceptance (MC/src/mc.cu:379-440) with mu held at kT ln10 (pKa - pH), no
feedback and no target stop.  The device runs the same flips in the
engine's grand-canonical phase with fixed_mu set, on the same input files,
from the same std::mt19937 seed (the phase draws the reference's own stream),
in blocks whose ends are the sampling points (pools then rebuilt in index
order on both sides).  Per pH, alpha and the z-profiles of the protonated
sites and of the Cl ions come from block-end snapshots, each side's standard
error from its block-end series by the blocking method (consecutive snapshots
are correlated).  The two chains part ways trajectory by trajectory (their
float energies differ in the last bits, so near-threshold decisions go either
way), so the comparison is statistical: a single comparison at two standard
errors fails by chance about one time in twenty, and the twelve below would
fail a correct build about half the time.  So every difference must lie
within three standard errors, alpha's over the four pH values must pass a
chi-square test at the 1 % level, and at most one of them may lie beyond two.
"""
import os
import subprocess

import numpy as np
import pytest

import bench
from ph_brush_b200 import Engine, files

PKA = 7.5
PHS = (6.5, 7.25, 7.75, 8.5)
BLOCKS, BLOCK_LEN, NBINS = 24, 250, 8
NHN, NHP, W, CL = 3, 4, 6, 7  # the reference's types 4, 5, 7, 8, 0-based


def mt19937_state(seed):
    mt = np.zeros(625, np.uint32)
    v = seed
    mt[0] = v
    for i in range(1, 624):
        v = (1812433253 * (v ^ (v >> 30)) + i) & 0xFFFFFFFF
        mt[i] = v
    mt[624] = 624
    return mt


def pools(t, z, z_cut):
    return dict(nh_n=np.flatnonzero(t == NHN), nh_p=np.flatnonzero(t == NHP),
                w=np.flatnonzero((t == W) & (z < z_cut)), cl=np.flatnonzero((t == CL) & (z < z_cut)))


def hist(z, idx, height):
    b = np.clip((z[idx] / height * NBINS).astype(np.int64), 0, NBINS - 1)
    return np.bincount(b, minlength=NBINS)


def device_blocks(s, p, mu_kT, seed, height):
    t0 = s.type
    sites = np.flatnonzero((t0 == NHN) | (t0 == NHP))
    z_cut = float(np.max(s.z[sites])) + 1.0
    mt = mt19937_state(seed)
    out = []
    with Engine(s, p) as e:
        st = e.state()
        for _ in range(BLOCKS):
            job = dict(replica=0, nh_n_type=NHN, nh_p_type=NHP, w_type=W, cl_type=CL, beta=1.0, target_pct=50.0,
                       max_trials=BLOCK_LEN, fixed_mu=1, mu_kT=mu_kT, mt_state=mt, **pools(st["type"], st["z"], z_cut))
            (res, _), = e.gc_phase([job])
            assert res["attempted"] == BLOCK_LEN and res["reached_target"] == 0
            st = e.state()
            t = st["type"]
            out.append({"alpha": np.count_nonzero(t == NHP) / len(sites),
                        "sites": hist(st["z"], np.flatnonzero(t == NHP), height),
                        "cl": hist(st["z"], np.flatnonzero((t == CL) & (st["z"] < z_cut)), height)})
    return out


def stats(blocks, key):
    """Mean over the block-end samples and its standard error.  Consecutive samples of one
    chain are correlated, so the error is the blocking method's (the largest naive error of
    the series averaged over 1, 2, 4, ... samples while five or more remain), not the
    naive one, which would understate it."""
    a = np.array([b[key] for b in blocks], np.float64)
    return a.mean(0), bench.blocking_se(a)


def mean_height(blocks, key, height):
    centres = (np.arange(NBINS) + 0.5) * height / NBINS
    m = np.array([np.dot(b[key], centres) / max(np.sum(b[key]), 1) for b in blocks])
    return m.mean(), float(bench.blocking_se(m[:, None])[0])


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    harness = bench.REF_HARNESS
    if not os.path.exists(harness) or not os.path.exists(bench.REF_INPUTS):
        pytest.skip("reference build not present (make -C oracle ref inputs)")
    d = tmp_path_factory.mktemp("alpha")
    line = (f"a1 4 4 4.0 20 20 0 1 40.0 120.0 0.5 {20.0 / (16 * 16 * 40)!r} 0.97 0.9 2025 -1 7 0.5 7.5 {PKA}")
    bench.write_ref_inputs([line], str(d))
    base = str(d / "a1")
    s, p = files.reference_model(base + ".data", base + ".params")
    height = 40.0
    out = {}
    for pH in PHS:
        mu = float(np.log(10.0) * (PKA - pH))
        r = subprocess.run([harness, "alpha", base, repr(mu), str(BLOCKS), str(BLOCK_LEN), str(NBINS), "2025"],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-500:]
        import json
        ref = json.loads(r.stdout.strip().splitlines()[-1])["blocks"]
        dev = device_blocks(s, p, mu, 2025, height)
        out[pH] = (ref, dev, height)
    return out


CHI2_4_1PCT = 13.277  # chi-square with 4 degrees of freedom, upper 1 % point


@pytest.mark.gpu
def test_alpha_agrees_with_the_reference(runs):
    z = []
    for pH in PHS:
        ref, dev, _ = runs[pH]
        ma, sa = stats(ref, "alpha")
        mb, sb = stats(dev, "alpha")
        z.append(float((ma - mb) / np.hypot(sa, sb)))
    z = np.array(z)
    assert np.all(np.abs(z) <= 3.0), dict(zip(PHS, z))
    assert float(np.sum(z ** 2)) <= CHI2_4_1PCT, dict(zip(PHS, z))
    assert int(np.sum(np.abs(z) > 2.0)) <= 1, dict(zip(PHS, z))


@pytest.mark.gpu
@pytest.mark.parametrize("pH", PHS)
def test_z_profiles_agree_with_the_reference(runs, pH):
    ref, dev, height = runs[pH]
    for key in ("sites", "cl"):
        ha, ea = mean_height(ref, key, height)
        hb, eb = mean_height(dev, key, height)
        assert abs(ha - hb) <= 3 * np.hypot(ea, eb) + 1e-9, (pH, key, ha, hb, ea, eb)
        ma, sa = stats(ref, key)
        mb, sb = stats(dev, key)
        se = np.hypot(sa, sb)
        occupied = (ma + mb) > 0
        assert np.all(np.abs(ma - mb)[occupied] <= 3 * se[occupied] + 1e-9), (pH, key, ma, mb, se)


@pytest.mark.gpu
def test_alpha_follows_the_titration_curve(runs):
    """Sanity of the sampling itself: alpha falls with pH on both sides."""
    a_ref = [stats(runs[pH][0], "alpha")[0] for pH in PHS]
    a_dev = [stats(runs[pH][1], "alpha")[0] for pH in PHS]
    assert all(x > y for x, y in zip(a_ref, a_ref[1:])) and all(x > y for x, y in zip(a_dev, a_dev[1:]))
