#!/usr/bin/env python3
"""Benchmark: Monte Carlo sweeps/s of the plain engine on the config-2 brush.

Workload: 10x10 grafted chains x 50 titratable beads (pKa 7.5, pH 6.5), box
40x40x100 sigma padded to 300 for the slab correction, 0.1 M salt (about 12k
particles), SPME mesh 64x64x384 order 5, WCA + FENE + erfc Coulomb, moves 90 %
displacement (0.3 sigma) / 10 % protonation with counterion insert/delete.
One step = one sweep = N_particles trial moves of the replica.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank runs its own replica
(replicas only, weak scaling); the timed region is bracketed by barriers and
the max device time over ranks is reported.  `--impl reference` runs the
reference's own CUDA build (compiled from its sources into oracle/_ref) on the
same system in the reference's model and prints the same metric.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC sweeps/s on 1 B200: batched+surrogate vs plain, α(pH) within 0.005"
UNIT = "sweeps/s"
FALLBACK_HBM_GBS = 6650.0
WORKLOAD = ("config 2: plain constant-pH MC, 10x10 chains x 50 titratable beads, 40x40x100 box padded to 300, "
            "0.1 M salt, ~12k particles, SPME 64x64x384 order 5, rc 3, 90% displacement / 10% protonation")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--harvest", type=int, default=262144, help="surrogate training samples harvested (config 5)")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--da-threshold", type=float, default=0.3)
    ap.add_argument("--no-alpha", action="store_true")
    ap.add_argument("--batched-replicas", type=int, default=256)
    ap.add_argument("--tuning", default=None, help="pending_max,threads instead of the autotuner (for profiling)")
    ap.add_argument("--batched-only", action="store_true",
                    help="only the config-5 batched section (its own JSON object; for profiling)")
    ap.add_argument("--alpha-eq", type=int, default=300, help="sweeps of equilibration in the alpha(pH) check")
    ap.add_argument("--alpha-sample", type=int, default=200, help="sweeps sampled in the alpha(pH) check")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.path = tempfile.mktemp(suffix=".csv")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(dev)], stdout=open(self.path, "w"),
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(kernel, {}).get("dram_bytes_per_launch")
    except Exception:
        return None


def reduce_max(val, world, dev):
    if world == 1:
        return val
    import torch
    import torch.distributed as dist
    t = torch.tensor([val], dtype=torch.float64, device=f"cuda:{dev}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(s, p, seconds):
    """The FP64 oracle's Monte Carlo (same move set, energy from scratch per trial) on the host cores."""
    from oracle import pyoracle as O
    mc = O.MC(s, p)
    n = 0
    t0 = time.perf_counter()
    while True:
        mc.step()
        n += 1
        el = time.perf_counter() - t0
        if el > seconds and n >= 2:
            break
    mc.close()
    tps = n / el
    cores = os.cpu_count()
    return {"value": tps / s.n, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} trials of the config-2 system in {el:.1f} s (FP64, O(N^2) pairs + FP64 FFT per trial, "
                      f"{cores} OpenMP threads); sweeps/s = trials/s / {s.n}",
            "trials_per_s": tps}


def tune_engine(eng, args, trials):
    """Autotune (pending capacity x block size), or apply --tuning."""
    if args.tuning:
        pm, th = (int(v) for v in args.tuning.split(","))
        eng.set_tuning(pm, th)
        return None
    return eng.autotune(trials)


def _alpha(stats, n_sites):
    return [st["n_charged_sites"] / n for st, n in zip(stats, n_sites)]


def alpha_check(local, sweeps_eq, sweeps_sample, snaps=20):
    """alpha(pH) of delayed acceptance against the plain engine on config-5 chemistry (small
    diblock replicas that equilibrate within the run).  The plain engine equilibrates, its
    exact dE of the last part of the equilibration train the surrogate, a second engine takes
    over the equilibrated states with delayed acceptance, and both engines then sample."""
    import numpy as np
    from ph_brush_b200 import Engine, Surrogate, configs
    reps = configs.diblock_small()
    S, P = [a for a, _ in reps], [b for _, b in reps]
    for p in P:
        p.p_disp, p.p_titr = 0.5, 0.5  # titration-heavy: alpha relaxes within the run
    ns = [a.meta["n_sites"] for a in S]
    nmax = max(a.n for a in S)
    A = Engine(S, P, device=local)
    A.autotune(2000)
    A.run(sweeps_eq * nmax)
    A.harvest(131072)
    A.run(max(nmax * 10, 2 * 131072 // len(S)))
    sur = Surrogate(seed=31)
    loss = A.surrogate_fit(sur, epochs=12, batch=2048, lr=1e-3, clip=25.0, seed=3)
    A.harvest(0)
    B = Engine(S, P, device=local)
    tn = A.tuning()
    B.set_tuning(tn["pending_max"], tn["threads"])
    for r in range(len(S)):
        B.set_state(A.state(r), r)
    B.attach_surrogate(sur, threshold=0.0, window=0)
    per = max(1, sweeps_sample * nmax // snaps)
    a_p, a_d = [], []
    for _ in range(snaps):
        a_p.append(_alpha(A.run(per), ns))
        a_d.append(_alpha(B.run(per), ns))
    da = B.da_stats()
    A.close()
    B.close()
    a_p, a_d = np.array(a_p), np.array(a_d)
    mp, md = a_p.mean(0), a_d.mean(0)
    half = snaps // 2
    drift = float(np.abs(a_p[half:].mean(0) - a_p[:half].mean(0)).mean())
    se = np.sqrt(a_p.var(0, ddof=1) / snaps + a_d.var(0, ddof=1) / snaps)
    pH = np.array([p.pH for p in P])
    curve = []
    for lo in (5.0, 6.0, 7.0, 8.0):
        m = (pH >= lo) & (pH < lo + 1.0 + (1e-9 if lo == 8.0 else 0.0))
        curve.append({"pH": [lo, lo + 1.0], "replicas": int(m.sum()), "alpha_plain": float(mp[m].mean()),
                      "alpha_da": float(md[m].mean()), "diff": float(md[m].mean() - mp[m].mean()),
                      "stderr": float(np.sqrt((se[m] ** 2).sum()) / m.sum())})
    ev = sum(d["evaluated"] for d in da)
    ps = sum(d["passed"] for d in da)
    ac = sum(d["accepted"] for d in da)
    return {"workload": "config-5 chemistry, 24 replicas of 4x4 diblock chains (20 permanent +1 + 30 titratable, "
                        "pKa 7.3), pH 5-9, salt 0.01-0.1 M, 50% displacement / 50% protonation",
            "sweeps_equilibrate": sweeps_eq, "sweeps_sample": sweeps_sample, "snapshots": snaps,
            "fit_loss": loss, "exact_dE_skipped": 1.0 - ps / max(ev, 1), "second_stage_agreement": ac / max(ps, 1),
            "pH_curve": curve, "max_curve_diff": float(max(abs(c["diff"]) for c in curve)),
            "mean_abs_diff_per_replica": float(np.abs(md - mp).mean()), "median_stderr_per_replica": float(np.median(se)),
            "plain_drift_between_halves": drift}


def run_batched(args, local, n_rep=256, trials=400, plain_samples=3):
    """Config 5: 256 diblock replicas in one engine (one block per replica per MC
    phase, captured in CUDA graphs) against the plain engine, which runs the same
    replicas one at a time.  Aggregate sweeps/s = sum over replicas of sweeps / time.
    Then the learned surrogate: exact dE harvested from the replicas, one network
    (pH and salt among its inputs) trained on the GPU, delayed acceptance on the
    config's move mix and on a titration-only phase."""
    import numpy as np
    from ph_brush_b200 import Engine, Surrogate, configs
    reps = configs.config5(n_rep=n_rep)
    ns = [s.n for s, _ in reps]
    n_sites = [int(s.meta["n_sites"]) for s, _ in reps]
    eng = Engine([s for s, _ in reps], [p for _, p in reps], device=local)
    tune = tune_engine(eng, args, trials)
    tuned = eng.tuning()
    eng.run(trials // 4)
    eng.set_profiling(True)
    eng.profile(reset=True)
    eng.flush_l2(256 << 20)
    ms = eng.run_timed(trials)
    prof = eng.profile(reset=True)
    eng.set_profiling(False)
    agg = sum(trials / n for n in ns) / (ms / 1e3)
    # plain engine: the same replicas one at a time (each autotuned); its aggregate rate
    # over the set is R sweeps / sum_r (N_r * t_r), t_r the per-trial time of replica r alone
    idx = sorted(range(n_rep), key=lambda r: ns[r])
    pick = [idx[0], idx[len(idx) // 2], idx[-1]][:plain_samples]
    per_sweep_s = []
    for r in pick:
        s, p = reps[r]
        e1 = Engine(s, p, device=local)
        tune_engine(e1, args, trials)
        e1.run(trials // 4)
        e1.flush_l2(256 << 20)
        t = e1.run_timed(trials) / 1e3 / trials
        e1.close()
        per_sweep_s.append(ns[r] * t)
    plain = 1.0 / (sum(per_sweep_s) / len(per_sweep_s))
    peak, kind = measured_peak()
    rl = {}
    if prof["mc_launches"] and prof["mc_ms"] > 0:
        rl["k_mc"] = {"achieved": prof["mc_alg_bytes"] / (prof["mc_ms"] / 1e3) / 1e9, "share": prof["mc_ms"] / ms}
    if prof["flush_launches"] and prof["flush_ms"] > 0:
        rl["mesh_rebuild"] = {"achieved": prof["flush_alg_bytes"] / (prof["flush_ms"] / 1e3) / 1e9,
                              "share": prof["flush_ms"] / ms}
    for v in rl.values():
        v.update({"bound": "hbm", "peak": peak, "unit": "GB/s", "frac": v["achieved"] / peak, "peak_source": kind})

    # ---- surrogate: harvest (titration-heavy mix), GPU training ----
    p0 = reps[0][1]
    sur = Surrogate(seed=2029)
    eng.set_move_mix(0.5, 0.5, 0.0)
    eng.harvest(args.harvest)
    eng.run(2 * args.harvest // n_rep + 1)
    n_samples = eng.harvest_count()
    t0 = time.perf_counter()
    loss = eng.surrogate_fit(sur, epochs=args.epochs, batch=4096, lr=1e-3, clip=25.0, seed=7)
    t_fit = time.perf_counter() - t0
    eng.harvest(0)
    steps = args.epochs * (n_samples // 4096)
    # 4 rows per sample; forward 2*(80*128 + 2*128*128 + 128) flops per row, backward twice that
    fl_row = 2.0 * (80 * 128 + 2 * 128 * 128 + 128)
    train = {"samples": n_samples, "epochs": args.epochs, "batch": 4096, "lr": 1e-3, "final_loss": loss,
             "seconds": t_fit, "samples_per_s": steps * 4096 / t_fit,
             "tflops": steps * 4096 * 4 * 3 * fl_row / t_fit / 1e12}

    # ---- batched + surrogate on the config's move mix ----
    eng.set_move_mix(p0.p_disp, p0.p_titr, p0.p_swap)
    eng.attach_surrogate(sur, threshold=args.da_threshold, window=256)
    eng.run(trials // 4)
    eng.flush_l2(256 << 20)
    ms_da = eng.run_timed(trials)
    agg_da = sum(trials / n for n in ns) / (ms_da / 1e3)
    da_mix = eng.da_stats()

    # ---- titration-only phase (the reference's protonation phase): plain vs delayed acceptance ----
    eng.set_move_mix(0.0, 1.0, 0.0)
    eng.attach_surrogate(None)
    tt = int(max(n_sites))
    eng.run(tt)
    eng.flush_l2(256 << 20)
    ms_tp = eng.run_timed(tt)
    eng.attach_surrogate(sur, threshold=0.0, window=0)
    eng.run(tt // 4)
    eng.flush_l2(256 << 20)
    ms_td = eng.run_timed(tt)
    da_t = eng.da_stats()
    eng.close()
    ev, ps, ac = (sum(d[k] for d in da_t) for k in ("evaluated", "passed", "accepted"))
    evm, psm, acm = (sum(d[k] for d in da_mix) for k in ("evaluated", "passed", "accepted"))
    tp_plain = n_rep * tt / (ms_tp / 1e3)
    tp_da = n_rep * tt / (ms_td / 1e3)
    surrogate = {
        "training": train,
        "aggregate_sweeps_per_s": agg_da, "speedup_vs_plain": agg_da / plain,
        "speedup_vs_batched_exact": agg_da / agg,
        "config_mix": {"exact_dE_skipped": 1.0 - psm / max(evm, 1), "second_stage_agreement": acm / max(psm, 1),
                       "fallbacks": int(sum(d["fallback"] for d in da_mix)), "threshold": args.da_threshold},
        "titration_phase": {"trials_per_replica": tt, "plain_trials_per_s": tp_plain, "da_trials_per_s": tp_da,
                            "gain": tp_da / tp_plain, "exact_dE_skipped": 1.0 - ps / max(ev, 1),
                            "second_stage_agreement": ac / max(ps, 1)},
    }
    if not args.no_alpha:
        surrogate["alpha_check"] = alpha_check(local, args.alpha_eq, args.alpha_sample)
    return {"workload": "config 5: 256 diblock replicas (20 permanent +1 + 30 titratable beads, pKa 7.3), 64-144 chains, "
                        "pH 5-9, salt 0.001-0.3 M, slab 60 padded to 180, SPME order 5, lateral mesh 48-64",
            "replicas": n_rep, "particles_min_max": [min(ns), max(ns)], "trials_per_replica": trials,
            "tuning": tuned, "autotune": tune,
            "aggregate_sweeps_per_s": agg, "trials_per_s": n_rep * trials / (ms / 1e3),
            "plain_aggregate_sweeps_per_s": plain, "plain_sampled_replicas": pick, "speedup_vs_plain": agg / plain,
            "roofline": rl, "device_ms": ms, "gpu_launches": int(prof["kernel_launches"]),
            "surrogate": surrogate}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from ph_brush_b200 import configs
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build missing: run `make -C oracle ref`"}))
        return
    sn, _ = configs.config2()
    n_sites = int(((sn.flags & 2) != 0).sum())
    n_charged = int(((sn.flags & 2) != 0).__and__(sn.q != 0).sum())
    spacing = 0.7  # reference mesh rule: 60x60x432 (1.56 M points) for the 40x40x300 box
    s, p = configs.to_reference_semantics(sn, n_w=n_sites, spacing=spacing, seed=5)
    d = tempfile.mkdtemp()
    configs.write_lammps_data(os.path.join(d, "in.data"), s)
    pct = 100.0 * (n_charged + 0.5) / n_sites  # floor(pct/100 * sites) == current count (build_plan needs target >= current)
    configs.write_params_in(os.path.join(d, "params.in"), p, spacing, extra={"target_pct": f"{pct:.8f}"})
    per_step = 20
    r = subprocess.run([harness, "time", os.path.join(d, "in.data"), os.path.join(d, "params.in"),
                        str(per_step * args.steps), str(per_step * args.warmup)], capture_output=True, text=True)
    if r.returncode != 0:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness failed: " + r.stderr.strip()[-200:]}))
        return
    out = json.loads(r.stdout.strip().splitlines()[-1])
    sweeps = out["trials_per_s"] / sn.n
    line = {"impl": "reference", "metric": METRIC, "value": sweeps, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * out["seconds"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded brush generator)",
            "config": {"workload": WORKLOAD + " (reference model: LJ cut at 3 sigma, 1-2 exclusions, cubic SPME, "
                                  "mesh from pme_spacing 0.7 -> %s; moves: the reference's phase-2 identity swaps)"
                                  % out["mesh"], "particles": sn.n, "reference_atoms": out["natoms"],
                       "trials_per_step": per_step},
            "cpu_baseline": {"value": sweeps, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{out['trials']} trials of phase2_swap_jitter (MC/src/mc.cu:159-318) in the "
                                       f"reference's CUDA build on this B200 (one host thread), CUDA-event timed"},
            "e2e": {"value": sweeps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "trials_per_s": out["trials_per_s"], "reference_seconds": out["seconds"]}
    print(json.dumps(line))


def run_ours(args):
    rank, world, local = dist_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import numpy as np
    from ph_brush_b200 import Engine, configs

    s, p = configs.config2(seed=2026 + rank)
    N = s.n
    eng = Engine(s, p, device=local)
    tune = tune_engine(eng, args, max(2000, N // 4))
    tuned = eng.tuning()
    for _ in range(args.warmup):
        eng.run(N)
    # ---- device-timed region: inputs resident, L2 flushed between steps ----
    eng.set_profiling(True)
    eng.profile(reset=True)
    clocks = Clocks(local)
    barrier(world)
    dev_ms = 0.0
    for _ in range(args.steps):
        eng.flush_l2(256 << 20)
        dev_ms += eng.run_timed(N)
    barrier(world)
    clk = clocks.stop()
    prof = eng.profile(reset=True)
    eng.set_profiling(False)
    max_ms = reduce_max(dev_ms, world, local)
    value = world * args.steps / (max_ms / 1e3)

    # ---- end to end through the public API: pinned host state in, state + energy out ----
    st = eng.state()
    try:
        import torch
        pinned = {k: torch.from_numpy(v.copy()).pin_memory().numpy() for k, v in st.items()}
    except Exception:
        pinned = {k: v.copy() for k, v in st.items()}
    cap = len(st["x"])
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.set_state(pinned)
        res = eng.run(N)
        out = eng.state()
        energy = res[0]["energy"]
    e2e_s = time.perf_counter() - t0
    barrier(world)
    e2e_s = reduce_max(e2e_s, world, local)
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": cap * (16 + 4 + 4), "d2h_bytes_per_step": cap * (16 + 4 + 4) + 8,
           "timing": "host wall clock around phmc_set_state + phmc_run + phmc_get_state (synchronous calls)"}

    # ---- roofline of the dominant kernel ----
    peak, peak_kind = measured_peak()
    kern = []
    if prof["mc_launches"]:
        ms = prof["mc_ms"] / prof["mc_launches"]
        by = prof["mc_alg_bytes"] / prof["mc_launches"]
        kern.append(("k_mc", prof["mc_ms"], ms, by))
    if prof["flush_launches"]:
        ms = prof["flush_ms"] / prof["flush_launches"]
        by = prof["flush_alg_bytes"] / prof["flush_launches"]
        kern.append(("mesh_rebuild", prof["flush_ms"], ms, by))
    kern.sort(key=lambda k: -k[1])
    rl = {}
    for name, tot, ms, by in kern:
        ach = by / (ms / 1e3) / 1e9
        rl[name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "peak_source": peak_kind, "traffic": ncu_traffic(name), "alg_bytes_per_launch": by,
                    "avg_launch_ms": ms, "launches": prof[("mc" if name == "k_mc" else "flush") + "_launches"],
                    "share_of_timed": tot / dev_ms if dev_ms else None}
    dominant = kern[0][0] if kern else None

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 accumulation and Metropolis)",
            "data": "synthetic (seeded brush generator, seed 2026 + rank)",
            "config": {"workload": WORKLOAD, "particles": N, "trials_per_step": N, "mesh": list(p.mesh),
                       "order": p.order, "tuning": tuned, "autotune": tune,
                       "l2": "flushed between steps (256 MiB write on the engine stream)",
                       "parallelism": f"replicas only x{world}"},
            "roofline": dict(rl[dominant], kernel=dominant) if dominant else None,
            "roofline_other": {k: v for k, v in rl.items() if k != dominant},
            "e2e": e2e, "gpu_launches": int(prof["kernel_launches"]),
            "trials_per_s": world * prof["trials"] / (max_ms / 1e3) if prof["trials"] else None,
            "clocks": clk}
    eng.close()
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched"] = run_batched(args, local, n_rep=args.batched_replicas)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(s, p, args.cpu_seconds)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def main():
    args = parse()
    if args.batched_only:
        print(json.dumps({"batched": run_batched(args, dist_env()[2], n_rep=args.batched_replicas)}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
