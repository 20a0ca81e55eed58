"""The reference's move phases on the device: grand-canonical mu control
(MC/src/mc.cu:320-548, phmc_gc_phase) and swaps with patience (MC/src/mc.cu:159-318,
phmc_phase2), with their report lines written from device event records.

* CPU: the device's restatement of the reference's random stream (std::mt19937,
  uniform_int_distribution<int>, uniform_real_distribution<float>; GCC 13
  libstdc++) against libstdc++ itself, draw for draw, plus the generator's
  stream format; the report formatter against the reference's statements.
* GPU: the reference's own driver with its phase_gc_mu_control and
  phase2_swap_jitter calls renamed to the device phases (oracle/_ref/MC_phmc_dev)
  against the reference's complete build (oracle/_ref/MC_ref) on the same input
  and seed: every report line, [sgmc] and [phase2] (phase 2 only agrees if the
  first phase left the same atoms and generator state); and through the Python
  handle: pools, energies, the restored half of rejected four-point moves, and
  determinism.
"""
import os
import subprocess

import numpy as np
import pytest

from ph_brush_b200 import Engine, _abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MT_HEADER = os.path.join(ROOT, "ph_brush_b200", "csrc", "mt_std.cuh")

MT_CHECK = r"""
#include <cstdio>
#include <random>
#include <sstream>
#include "mt_std.cuh"
int main() {
    long long bad = 0, n = 0;
    for (unsigned seed : {2025u, 1u, 0u, 4294967295u, 12345u}) {
        std::mt19937 g(seed);
        MtState s;
        mt_seed(s, seed);
        for (int k = 0; k < 200000; ++k) {
            if (k % 3 == 0) {
                uint32_t m = 1 + (k * 2654435761u) % 5000;
                if (k % 7 == 0) m = 1;
                if (k % 11 == 0) m = 2000000000u;
                std::uniform_int_distribution<int> d(0, (int)m - 1);
                if (d(g) != mt_index(s, m)) ++bad;
            } else {
                std::uniform_real_distribution<float> u(0.0f, 1.0f);
                if (u(g) != mt_unit_float(s)) ++bad;
            }
            ++n;
        }
        // the stream format: 624 words, then the position
        std::stringstream ss;
        ss << g;
        MtState t;
        for (int i = 0; i < 624; ++i) ss >> t.x[i];
        ss >> t.p;
        for (int i = 0; i < 624; ++i) bad += t.x[i] != s.x[i];
        bad += t.p != s.p;
    }
    printf("%lld %lld\n", n, bad);
    return 0;
}
"""


def test_generator_restatement_matches_libstdcxx(tmp_path):
    src = tmp_path / "mt_check.cpp"
    src.write_text(MT_CHECK)
    exe = tmp_path / "mt_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.dirname(MT_HEADER), "-o", str(exe), str(src)], check=True)
    n, bad = map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split())
    assert n == 1000000 and bad == 0


def fmt(ev, res):
    buf = __import__("ctypes").create_string_buffer(512)
    n = _abi.lib().phmc_gc_event_format(ev, res, buf, 512)
    assert n == len(buf.value)
    return buf.value.decode()


def f6(x):
    return f"{float(np.float32(x)):.6f}"


def test_report_lines_follow_the_reference_statements():
    res = _abi.GcResult(Nh=40, target_count=12, R0=9, Nacc_target=1, epoch_attempt_max=1500, gc_block=300)
    ev = _abi.GcEvent(kind=_abi.GC_EV_CHUNK, acc_since_mu=3, att_since_mu=300, acc_rate=np.float32(3 / 300),
                      fwd_total=3, bwd_total=0, remaining=6)
    assert fmt(ev, res) == (f"[sgmc] chunk acc=3/1 attempts=300 acc_rate={f6(3 / 300)} fwd_total=3 bwd_total=0 "
                            "gc_block=300 remaining=6")
    mu = np.float32(-0.8472979)
    ev = _abi.GcEvent(kind=_abi.GC_EV_MU, epoch=0, cause_amax=0, mu_kT=mu, f=np.float32(0.175), acc_since_mu=3,
                      att_since_mu=300, fwd_total=3, bwd_total=0, remaining=6, w_info=1.0)
    assert fmt(ev, res) == (f"[sgmc] mu-update#1 cause=Nacc mu/kT={f6(mu)} f={f6(0.175)} acc=3/1 attempts=300/1500 "
                            "fwd_total=3 bwd_total=0 remaining=6 R0=9 w_info=1.000000")
    ev.cause_amax = 1
    assert " cause=Amax " in fmt(ev, res)
    E = np.float32(-1234.5678)
    ev = _abi.GcEvent(kind=_abi.GC_EV_REACHED, epoch=2, step_in_block=17, nprot=12, mu_kT=mu, E=E, fwd_total=10,
                      bwd_total=1)
    assert fmt(ev, res) == (f"[sgmc] reached target in epoch=2 step_in_block=17 Nprot=12/40 mu/kT={f6(mu)} E={f6(E)} "
                            "fwd_acc=10 bwd_acc=1 remaining=0")
    ev = _abi.GcEvent(kind=_abi.GC_EV_NO_PAIRS)
    assert fmt(ev, res) == "[sgmc] no valid pairs to flip; stop."
    ev = _abi.GcEvent(kind=_abi.GC_EV_ALREADY, nprot=12, mu_kT=mu, E=E)
    assert fmt(ev, res) == f"[sgmc] already at target: Nprot=12/40 target=12 mu/kT={f6(mu)} E={f6(E)} remaining=0"


def test_phase2_report_lines_follow_the_reference_statements():
    def f2(ev):
        buf = __import__("ctypes").create_string_buffer(512)
        n = _abi.lib().phmc_phase2_event_format(ev, buf, 512)
        assert n == len(buf.value)
        return buf.value.decode()
    E, acc = np.float32(-98.765432), np.float32(283 / 500)
    ev = _abi.Phase2Event(kind=_abi.P2_EV_STEP, attempted=500, accepted=283, since_best=0, patience=400, mode_wc=0,
                          E=E, acc=acc)
    assert f2(ev) == f"[phase2] step=500 E={f6(E)} accepted=283 acc={float(acc):.3f} since_best=0/400 mode=4-pt"
    ev.mode_wc = 1
    assert f2(ev).endswith(" mode=wc-only")
    z = np.float32(5.3329029)
    ev = _abi.Phase2Event(kind=_abi.P2_EV_POOLS, n_nh_p=32, n_nh_n=76, n_cl=12, n_w=39, z_cut=z)
    assert f2(ev) == f"[phase2] pools: NH_P=32 NH_N=76 Cl=12 W=39 (z_cut={f6(z)})"
    assert f2(_abi.Phase2Event(kind=_abi.P2_EV_PATIENCE, since_best=400, patience=400)) == \
        "[phase2] patience reached: 400/400. Stop."
    assert f2(_abi.Phase2Event(kind=_abi.P2_EV_NONE_AT_START)) == \
        "[phase2] no valid proposals (no 4-pt and no wc-only). Stop."
    assert f2(_abi.Phase2Event(kind=_abi.P2_EV_WC_EMPTY)) == "[phase2] wc-only requested but pools empty; Stop."
    assert f2(_abi.Phase2Event(kind=_abi.P2_EV_NONE)) == "[phase2] no valid proposals; Stop."


# The oracle's restatement of the phases (oracle/pyoracle.py: libstdc++'s own
# std::mt19937 and distributions, FP64 reference-model energies rounded as the
# reference's float build rounds them).  Pinned to the reference's output: on
# the drop-in fixture the reference build's report line of its GC phase (MC_ref
# on a B200; the device phase printed the same line, counts equal and energies
# within 2e-5, in test_device_gc_phase_reproduces_the_reference_driver) is
#   [sgmc] reached target in epoch=0 step_in_block=41 Nprot=32/108
#          mu/kT=-0.847298 E=110.129379 fwd_acc=6 bwd_acc=3 remaining=0
REF_GC_LINE = {"epoch": 0, "step_in_block": 41, "nprot": 32, "Nh": 108, "mu_kT": -0.847298, "E": 110.129379,
               "fwd_total": 6, "bwd_total": 3}


def oracle_inputs(params):
    from oracle import pyoracle as O
    if not os.path.exists(O.REF_HOST):
        pytest.skip("reference host library not built (make -C oracle ref-host)")
    inputs = os.path.join(ROOT, "tests", "golden", "inputs")
    return O, O.ref_host_read(os.path.join(inputs, "dropin_small.data"), os.path.join(inputs, params))


def test_oracle_gc_phase_reproduces_the_reference_line():
    O, (s, p, raw) = oracle_inputs("dropin_small.params")
    plan = O.ref_plan(s, raw)
    res, evs = O.ref_gc_phase(s, p, raw, plan, O.RefGenerator(raw["rng_seed"]))
    assert len(evs) == 1 and evs[0]["kind"] == _abi.GC_EV_REACHED
    ev = evs[0]
    for k in ("epoch", "step_in_block", "nprot", "fwd_total", "bwd_total"):
        assert ev[k] == REF_GC_LINE[k], (k, ev[k])
    assert res["Nh"] == REF_GC_LINE["Nh"] and res["attempted"] == 41
    assert abs(ev["mu_kT"] - REF_GC_LINE["mu_kT"]) < 5e-7
    assert abs(ev["E"] - REF_GC_LINE["E"]) <= 2e-5 * abs(REF_GC_LINE["E"]) + 1e-3


def test_oracle_workflow_bookkeeping():
    """plan -> grand-canonical phase -> phase 2 on the longer-phase input: the restatement's
    own bookkeeping (events, blocks, epochs, patience, identities exchanged, not created)."""
    O, (s, p, raw) = oracle_inputs("dropin_gc.params")
    plan = O.ref_plan(s, raw)
    gen = O.RefGenerator(raw["rng_seed"])
    t0 = s.type.copy()
    res, evs = O.ref_gc_phase(s, p, raw, plan, gen)
    assert res["stop"] == 1 and res["Nprot"] == res["target_count"]
    kinds = [e["kind"] for e in evs]
    assert kinds[-1] == _abi.GC_EV_REACHED
    assert kinds.count(_abi.GC_EV_CHUNK) == (res["attempted"] - 1) // raw["gc_block_fixed"]
    assert kinds.count(_abi.GC_EV_MU) == res["blocks_done"] >= 2
    assert res["accepted_forward"] - res["accepted_backward"] == plan["to_flip"]
    NHN, NHP, W, CL = (raw[k] - 1 for k in ("NH_N_type", "NH_P_type", "W_type", "Cl_type"))
    t = s.type
    assert int(np.sum(t == NHP)) - int(np.sum(t0 == NHP)) == plan["to_flip"]
    assert int(np.sum(t == CL)) - int(np.sum(t0 == CL)) == plan["to_flip"]
    z = np.asarray(s.z, np.float32)
    pools = {"nh_p": list(np.where(t == NHP)[0]), "nh_n": list(np.where(t == NHN)[0]),
             "w": list(np.where((t == W) & (z < plan["z_cut"]))[0]), "cl": list(np.where((t == CL) & (z < plan["z_cut"]))[0])}
    t1 = t.copy()
    r2, e2 = O.ref_phase2(s, p, raw, pools, plan["z_cut"], gen)
    assert e2[0]["kind"] == _abi.P2_EV_POOLS and e2[0]["n_nh_p"] == len(pools["nh_p"])
    steps = [e for e in e2 if e["kind"] == _abi.P2_EV_STEP]
    assert len(steps) == r2["attempted"] // raw["energy_interval"]
    assert r2["stop"] in (1, 2)
    if r2["stop"] == 1:
        assert e2[-1]["kind"] == _abi.P2_EV_PATIENCE and r2["since_best"] >= raw["patience"]
    for ty in (NHN, NHP, W, CL):
        assert int(np.sum(s.type == ty)) == int(np.sum(t1 == ty))
    assert r2["best_E"] <= r2["E"]


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "MC_ref")
DEV_BIN = os.path.join(ROOT, "oracle", "_ref", "MC_phmc_dev")


def run_driver(binary, workdir, params):
    import shutil
    inputs = os.path.join(ROOT, "tests", "golden", "inputs")
    os.makedirs(workdir)
    shutil.copy(os.path.join(inputs, "dropin_small.data"), os.path.join(workdir, "in.data"))
    shutil.copy(os.path.join(inputs, params), os.path.join(workdir, "params.in"))
    r = subprocess.run([binary, "in.data", "params.in"], cwd=workdir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (binary, r.returncode, r.stderr[-500:])
    return open(os.path.join(workdir, "report.txt")).read().splitlines()


@pytest.mark.gpu
@pytest.mark.parametrize("params,long_phase", [("dropin_small.params", False), ("dropin_gc.params", True),
                                               ("dropin_already.params", None)])
def test_device_gc_phase_reproduces_the_reference_driver(tmp_path, params, long_phase):
    """long_phase None: the target is the current protonation, so the phase writes its
    "already at target" line in whatever stream state the plan summary left (fixed,
    precision 2), and phase 2 gets empty pools."""
    if not (os.path.exists(REF_BIN) and os.path.exists(DEV_BIN)):
        pytest.skip("reference driver binaries not built (make -C oracle mc-ref dropin-dev, needs the reference sources)")
    from test_dropin import RTOL, numbers
    ref = run_driver(REF_BIN, str(tmp_path / "ref"), params)
    got = run_driver(DEV_BIN, str(tmp_path / "dev"), params)
    assert len(ref) == len(got), (len(ref), len(got), ref[-5:], got[-5:])
    sgmc = [line for line in got if line.startswith("[sgmc]")]
    if long_phase is None:
        assert any("already at target" in line for line in sgmc), sgmc
        la = [line for line in ref if "already at target" in line]
        lb = [line for line in got if "already at target" in line]
        decimals = lambda line: [len(x.split(".")[1]) if "." in x else 0 for x in numbers(line)]
        assert len(la) == len(lb) == 1 and decimals(la[0]) == decimals(lb[0]), (la, lb)  # the same stream precision
    else:
        assert any("reached target" in line for line in sgmc), sgmc
    if long_phase:  # chunk lines and mu updates of several epochs
        assert sum("mu-update#" in line for line in sgmc) >= 2 and sum("chunk" in line for line in sgmc) >= 3, sgmc
    for a, b in zip(ref, got):
        if a == b:
            continue
        na, nb = numbers(a), numbers(b)
        assert len(na) == len(nb) and re_words(a) == re_words(b), (a, b)
        for x, y in zip(na, nb):
            if not any(c in x + y for c in ".eE"):
                assert x == y, (a, b)  # counts, steps, pools
            else:
                assert abs(float(x) - float(y)) <= RTOL * abs(float(x)) + 1e-3, (a, b)
    if long_phase is not None:
        assert sum(line.startswith("[phase2] step=") for line in got) >= 3, got


def re_words(line):
    import re
    return re.sub(r"-?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?", "#", line)


def mt_seeded(seed):
    """std::mt19937(seed)'s state words and position (Knuth's initialisation)."""
    x = np.zeros(625, np.uint32)
    v = seed & 0xFFFFFFFF
    x[0] = v
    for i in range(1, 624):
        v = (1812433253 * (v ^ (v >> 30)) + i) & 0xFFFFFFFF
        x[i] = v
    x[624] = 624
    return x


NHN, NHP, W, CL = 3, 4, 6, 7  # the reference's types 4, 5, 7, 8, 0-based


def gc_setup(seed=11, n_w=60, target_pct=60.0):
    s0, _ = configs.small_system(seed=seed, chains=3, length=8, box_xy=12.0, height=12.0, salt_pairs=6)
    s, p = configs.to_reference_semantics(s0, n_w=n_w, seed=seed)
    t = s.type
    sites = np.where((t == NHN) | (t == NHP))[0]
    z_cut = float(np.max(s.z[sites])) + 1.0
    pools = {"nh_n": np.where(t == NHN)[0], "nh_p": np.where(t == NHP)[0],
             "w": np.where((t == W) & (s.z < z_cut))[0], "cl": np.where((t == CL) & (s.z < z_cut))[0]}
    job = dict(replica=0, nh_n_type=NHN, nh_p_type=NHP, w_type=W, cl_type=CL, q_nh_p=1.0, q_cl=-1.0, beta=1.0,
               target_pct=target_pct, gc_block=50, epoch_attempt_max=200, **pools)
    return s, p, job


@pytest.mark.gpu
def test_gc_phase_through_the_python_handle():
    s, p, job = gc_setup()
    runs = []
    for _ in range(2):
        mt = mt_seeded(2025)
        with Engine(s, p) as e:
            (res, evs), = e.gc_phase([dict(job, mt_state=mt)])
            st = e.state()
            comp = e.energy()[0]
        runs.append((res, evs, mt.copy(), st))
        assert res["stop"] in (_abi.GC_STOP_REACHED, _abi.GC_STOP_ALREADY), res
        assert res["reached_target"] == 1 and res["Nprot"] == res["target_count"]
        Nh = len(job["nh_n"]) + len(job["nh_p"])
        assert res["Nh"] == Nh and res["target_count"] == int(np.floor(np.float32(job["target_pct"]) / 100.0 * Nh))
        # the engine's identities follow the accepted flips: protonated sites, and as many
        # new Cl as net forward flips
        t, q = st["type"], st["q"]
        sites = np.concatenate([job["nh_n"], job["nh_p"]])
        assert int(np.sum(t[sites] == NHP)) == res["Nprot"]
        assert np.all(q[sites][t[sites] == NHP] == 1.0) and np.all(q[sites][t[sites] == NHN] == 0.0)
        ions = np.concatenate([job["w"], job["cl"]])
        assert int(np.sum(t[ions] == CL)) - len(job["cl"]) == res["accepted_forward"] - res["accepted_backward"]
        assert res["accepted_forward"] - res["accepted_backward"] == res["Nprot"] - len(job["nh_p"])
        # the phase's tracked energy (the reference's real) against a fresh recompute
        e_ref = np.float32(comp["lj"]) + np.float32(comp["coul_real"] + comp["coul_recip"] + comp["self"] +
                                                     comp["qcorr"] + comp["slab"])
        assert abs(float(res["E"]) - float(e_ref)) <= 2e-5 * abs(float(e_ref)) + 1e-3, (res["E"], e_ref)
        # events: one chunk line per completed block, the last one the target
        kinds = [ev["kind"] for ev in evs]
        assert kinds[-1] in (_abi.GC_EV_REACHED, _abi.GC_EV_ALREADY)
        if kinds[-1] == _abi.GC_EV_REACHED:  # the block the target was reached in reports no chunk line
            assert kinds.count(_abi.GC_EV_CHUNK) == (res["attempted"] - 1) // 50
        assert res["attempted"] > 0 and not np.array_equal(mt, mt_seeded(2025))
    # one block per job, no launch quorum: the phase is deterministic
    (r0, e0, m0, s0), (r1, e1, m1, s1) = runs
    assert r0 == r1 and e0 == e1 and np.array_equal(m0, m1)
    assert np.array_equal(s0["type"], s1["type"]) and np.array_equal(s0["q"], s1["q"])


@pytest.mark.gpu
def test_gc_phase_rejects_bad_jobs():
    s, p, job = gc_setup()
    with Engine(s, p) as e:
        bad = dict(job, mt_state=mt_seeded(1))
        bad["w"] = np.concatenate([job["w"], job["nh_n"][:1]])  # a slot in two pools
        with pytest.raises(_abi.PhmcError):
            e.gc_phase([bad])
        with pytest.raises(_abi.PhmcError):
            e.gc_phase([dict(job, mt_state=mt_seeded(1), cl_type=99)])


@pytest.mark.gpu
@pytest.mark.parametrize("wc_only", [False, True])
def test_phase2_through_the_python_handle(wc_only):
    s, p, job = gc_setup()
    pools = {k: job[k] for k in ("nh_p", "nh_n", "w", "cl")}
    if wc_only:
        pools["nh_n"] = pools["nh_n"][:0]  # no NH_N left: Cl/W moves only
    p2 = dict(replica=0, nh_n_type=NHN, nh_p_type=NHP, w_type=W, cl_type=CL, q_nh_p=1.0, q_cl=-1.0, beta=1.0,
              max_attempts=300, patience=120, energy_interval=50, z_cut=5.0, **pools)
    t0 = s.type.copy()
    runs = []
    for _ in range(2):
        mt = mt_seeded(77)
        with Engine(s, p) as e:
            (res, evs), = e.phase2([dict(p2, mt_state=mt)])
            st = e.state()
            comp = e.energy()[0]
        runs.append((res, evs, mt.copy(), st))
        assert 0 < res["attempted"] <= 300
        assert res["stop"] in (_abi.P2_STOP_PATIENCE, _abi.P2_STOP_MAX_ATTEMPTS)
        if res["stop"] == _abi.P2_STOP_PATIENCE:
            assert res["since_best"] >= 120
        # identities are exchanged, never created: every type keeps its count, and the
        # changed atoms are pool members
        t = st["type"]
        for ty in (NHN, NHP, W, CL):
            assert int(np.sum(t == ty)) == int(np.sum(t0 == ty))
        changed = np.where(t != t0)[0]
        assert set(changed) <= set(np.concatenate([pools[k] for k in pools]).tolist())
        if wc_only:
            assert not np.any(np.isin(changed, np.concatenate([job["nh_p"], job["nh_n"]])))
        # tracked energy (accepted moves only) against a fresh recompute: the NH half of
        # every rejected four-point move was restored
        e_ref = np.float32(comp["lj"]) + np.float32(comp["coul_real"] + comp["coul_recip"] + comp["self"] +
                                                     comp["qcorr"] + comp["slab"])
        assert abs(float(res["E"]) - float(e_ref)) <= 2e-5 * abs(float(e_ref)) + 1e-3, (res["E"], e_ref)
        assert res["best_E"] <= res["E"] + 1e-6
        kinds = [ev["kind"] for ev in evs]
        assert kinds[0] == _abi.P2_EV_POOLS and kinds.count(_abi.P2_EV_STEP) == res["attempted"] // 50
        steps = [ev for ev in evs if ev["kind"] == _abi.P2_EV_STEP]
        assert all(ev["mode_wc"] == (1 if wc_only else 0) for ev in steps)
    (r0, e0, m0, s0), (r1, e1, m1, s1) = runs
    assert r0 == r1 and e0 == e1 and np.array_equal(m0, m1) and np.array_equal(s0["type"], s1["type"])


@pytest.mark.gpu
def test_phases_batched_over_replicas_equal_single_runs():
    """Two jobs on a two-replica engine run in the same launches (one block each) and
    give exactly what each job gives alone."""
    s, p, job = gc_setup()
    seeds = (2025, 99)
    single = []
    for sd in seeds:
        mt = mt_seeded(sd)
        with Engine(s, p) as e:
            (res, evs), = e.gc_phase([dict(job, mt_state=mt)])
            single.append((res, evs, mt.copy(), e.state()["type"].copy()))
    mts = [mt_seeded(sd) for sd in seeds]
    with Engine([s, s], [p, p]) as e:
        out = e.gc_phase([dict(job, replica=k, mt_state=mts[k]) for k in range(2)])
        types = [e.state(k)["type"].copy() for k in range(2)]
    for k in range(2):
        res, evs, mt, t = single[k]
        assert out[k][0] == res and out[k][1] == evs
        assert np.array_equal(mts[k], mt) and np.array_equal(types[k], t)


def test_report_formatters_truncate_and_refuse_nulls():
    import ctypes
    lib = _abi.lib()
    res = _abi.GcResult(Nh=40, target_count=12)
    ev = _abi.GcEvent(kind=_abi.GC_EV_NO_PAIRS)
    full = "[sgmc] no valid pairs to flip; stop."
    assert lib.phmc_gc_event_format(ev, res, None, 0) == len(full)  # length only
    buf = ctypes.create_string_buffer(8)
    assert lib.phmc_gc_event_format(ev, res, buf, 8) == len(full) and buf.value.decode() == full[:7]
    assert lib.phmc_gc_event_format(None, res, buf, 8) == -1
    ev2 = _abi.Phase2Event(kind=_abi.P2_EV_NONE)
    assert lib.phmc_phase2_event_format(ev2, buf, 8) == len("[phase2] no valid proposals; Stop.")
    assert lib.phmc_phase2_event_format(None, buf, 8) == -1


def test_phase_entry_points_refuse_bad_arguments_before_any_device_call():
    lib = _abi.lib()
    job, res, ev = _abi.GcJob(), _abi.GcResult(), _abi.GcEvent()
    assert lib.phmc_gc_phase(None, 1, job, res, ev, 1) == 1  # PHMC_ERR_ARG
    j2, r2, e2 = _abi.Phase2Job(), _abi.Phase2Result(), _abi.Phase2Event()
    assert lib.phmc_phase2(None, 1, j2, r2, e2, 1) == 1


@pytest.mark.gpu
def test_event_records_stream_while_the_phase_runs():
    """With a stream callback every record reaches the caller during the call, in order,
    launch by launch (a fixed-mu phase of many launches never reaches a target and would
    otherwise report nothing until max_trials), also beyond the stored records' capacity;
    the stored records are the stream's first ones."""
    s, p, job = gc_setup()
    streamed = []
    with Engine(s, p) as e:
        e.set_tuning(8, 128)  # short launches: many of them
        e.set_event_callback(lambda j, ph, rec: streamed.append(
            (j, ph, _abi.GcEvent.from_address(rec).asdict())))
        (res, evs), = e.gc_phase([dict(job, mt_state=mt_seeded(7), fixed_mu=1, mu_kT=0.5, max_trials=1200)],
                                 event_cap=3)
        e.set_event_callback(None)
        (res2, _), = e.gc_phase([dict(job, mt_state=mt_seeded(8), fixed_mu=1, mu_kT=0.5, max_trials=100)])
    assert res["attempted"] == 1200 and res["stop"] == _abi.GC_STOP_MAX_TRIALS and res["reached_target"] == 0
    assert len(streamed) == res["n_events"] + res["events_dropped"] == 1200 // 50
    assert all(j == 0 and ph == 1 for j, ph, _ in streamed)
    assert [r for _, _, r in streamed][:3] == evs
    assert [r["kind"] for _, _, r in streamed] == [_abi.GC_EV_CHUNK] * 24
    assert len(streamed) == 24 and res2["attempted"] == 100  # no callback after it was switched off
