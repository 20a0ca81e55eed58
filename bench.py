#!/usr/bin/env python3
"""Benchmark: aggregate MC sweeps/s of batched delayed-acceptance MC on config 5.

Headline workload (config 5): 256 diblock brush replicas (64-144 chains of 20
permanent +1 and 30 titratable beads, pKa 7.3; pH 5-9 and salt 0.001-0.3 M
drawn from the seed; 4.6k-20k particles; slab 60 sigma padded to 180; SPME
order 5), all in one engine: one MC block per replica per launch and one fused
potential-mesh rebuild per chunk, captured in CUDA graphs, with the learned
surrogate (trained on the GPU on exact dE harvested from the replicas, pH and
salt among its inputs) as the first stage of delayed acceptance.  Moves: 90 %
displacement (0.3 sigma), 10 % protonation with counterion insert/delete.
One step = `--trials` trials of every replica; value = sum over replicas of
sweeps (trials / N_replica) per second, all ranks together.

Beside it: the plain engine on the same replicas one at a time (the
`speedup_vs_plain` of the metric), the titration-only phase, the alpha(pH) check
of delayed acceptance against the plain engine, and the plain engine on config 2
(10x10 chains x 50 titratable beads, ~12k particles) against the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) the replica set holds 256 N
replicas, split over the ranks by estimated cost (ph_brush_b200.replicas;
replicas only, weak scaling); the timed region is bracketed by barriers and
the max device time over ranks is reported.

`--impl reference` runs the reference's own CUDA build (compiled from its
sources into oracle/_ref; this process loads no library of this repository) on
the same replica set: the systems are written in the reference's input format
by oracle/_build/ref_inputs (the same generator, so the same particles), and
the reference's per-trial loop -- its full energy per trial, one replica after
the other -- runs a bounded sample of every replica's trials in the same move
mix; value in the same unit.  Its line also carries the reference on config 2.
"""
import argparse
import json
import math
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
WORKLOAD = ("config 5: 256 diblock brush replicas (20 permanent +1 + 30 titratable beads per chain, pKa 7.3), "
            "64-144 chains, pH 5-9, salt 0.001-0.3 M, slab 60 padded to 180, SPME order 5, batched in one engine, "
            "delayed acceptance with the GPU-trained surrogate; 90% displacement / 10% protonation")
CFG2 = ("config 2: plain constant-pH MC, 10x10 chains x 50 titratable beads, 40x40x100 box padded to 300, "
        "0.1 M salt, ~12k particles, SPME 64x64x384 order 5, rc 3, 90% displacement / 10% protonation")
MOVE_MIX = "90% displacement (max 0.3 sigma) / 10% protonation"
REF_INPUTS = os.path.join(ROOT, "oracle", "_build", "ref_inputs")
REF_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def workload_config(n_rep, ns):
    """The `config` both arms print (the same dict for the same workload)."""
    return {"workload": WORKLOAD, "replicas": int(n_rep), "particles_min_max": [int(min(ns)), int(max(ns))],
            "move_mix": MOVE_MIX, "parallelism": "replicas only"}


# ---------------------------------------------------------------------------
# the workloads as brush specs for oracle/_build/ref_inputs: the values
# ph_brush_b200.configs draws (config5, config2), restated here so that the
# reference arm imports nothing of the package (tests/test_bench_inputs.py
# checks the files against the package's systems)
# ---------------------------------------------------------------------------
def _molar(c):
    return c * 0.6022 * 0.5 ** 3


def _ideal(pH, pKa):
    return 1.0 / (1.0 + 10.0 ** (pH - pKa))


def config5_spec_lines(seed=2029, n_rep=256, pme_spacing=0.75):
    import numpy as np
    rng = np.random.default_rng(seed)
    H = 60.0
    out = []
    for k in range(n_rep):
        side = int(rng.integers(8, 13))
        pH = float(rng.uniform(5.0, 9.0))
        salt = float(math.exp(rng.uniform(math.log(0.001), math.log(0.3))))
        out.append(f"c5_{k:04d} {side} {side} 4.0 50 50 20 0 {H!r} {3 * H!r} {_ideal(pH, 7.3)!r} {_molar(salt)!r} "
                   f"0.97 0.9 {seed + 1000 + k} -1 {seed + 5000 + k} {pme_spacing!r} {pH!r} 7.3")
    return out


def config2_spec_line(pme_spacing=0.7):
    return (f"c2 10 10 4.0 50 50 0 1 100.0 300.0 {_ideal(6.5, 7.5)!r} {_molar(0.1)!r} 0.97 0.9 2026 -1 5 "
            f"{pme_spacing!r} 6.5 7.5")


def write_ref_inputs(lines, out_dir):
    """Run oracle/_build/ref_inputs on spec lines; returns {name: (natoms, n_native, n_sites)}."""
    spec = os.path.join(out_dir, "spec.txt")
    with open(spec, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    r = subprocess.run([REF_INPUTS, spec, out_dir], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("ref_inputs failed: " + r.stderr.strip()[-300:])
    out = {}
    for ln in r.stdout.split("\n"):
        f = ln.split()
        if len(f) == 4:
            out[f[0]] = tuple(int(v) for v in f[1:])
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--replicas", type=int, default=256)
    ap.add_argument("--trials", type=int, default=1000, help="trials per replica per step")
    ap.add_argument("--harvest", type=int, default=262144, help="surrogate training samples harvested")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--da-threshold", type=float, default=0.3)
    ap.add_argument("--tuning", default=None, help="pending_max,threads[,cand_round,g_rows,zpass,plane_pipe,first_stage] "
                                                    "instead of the autotuner (for profiling)")
    ap.add_argument("--quorum", type=float, default=None,
                    help="launch quorum of blocked replicas (default: the engine's, 0.2; for sweeps)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="headline only (plain comparison, phases, alpha skipped)")
    ap.add_argument("--no-alpha", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="no surrogate (profiling the exact path)")
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--no-config3", action="store_true")
    ap.add_argument("--no-config4", action="store_true")
    ap.add_argument("--plain-config2-only", action="store_true",
                    help="only the plain engine on config 2 (one JSON line of its figures; for profiling)")
    ap.add_argument("--alpha-eq", type=int, default=400, help="sweeps of equilibration in the alpha(pH) check")
    ap.add_argument("--alpha-sample", type=int, default=300, help="sweeps sampled in the alpha(pH) check")
    ap.add_argument("--ref-trials", type=int, default=4,
                    help="reference arm: trials per replica per step (its bounded sample of the step)")
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


def ncu_traffic_ratio(kernel):
    """DRAM bytes per algorithmic byte of `kernel` from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        return json.load(open(path)).get(kernel, {}).get("dram_bytes_per_alg_byte")
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


def reduce_sum(val, world, dev):
    if world == 1:
        return val
    import torch
    import torch.distributed as dist
    t = torch.tensor([val], dtype=torch.float64, device=f"cuda:{dev}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def tune_engine(eng, args, trials):
    """Autotune, or apply --tuning pending_max,threads[,cand_round,g_rows,zpass,plane_pipe,first_stage]
    (fixed shapes for profiling commands; -1 keeps a field)."""
    if getattr(args, "quorum", None) is not None:
        eng.set_quorum(args.quorum)
    if args.tuning:
        v = [int(x) for x in args.tuning.split(",")]
        eng.set_tuning(v[0], v[1])
        if len(v) > 2:
            v += [-1] * (7 - len(v))
            eng.set_tile_shapes(zpass=v[4], cand_round=v[2], g_rows=v[3], plane_pipe=v[5])
            if v[6] >= 0:
                eng.set_first_stage(v[6])
        return None
    return eng.autotune(trials)


def sums(stats, keys=("evaluated", "passed", "accepted")):
    return [sum(d[k] for d in stats) for k in keys]


# ---------------------------------------------------------------------------
# headline: batched + delayed acceptance on config 5
# ---------------------------------------------------------------------------
def headline_replicas(args, rank, world):
    """This rank's share of the config-5 replica set (256 per GPU), split by estimated
    cost with the library's partitioner."""
    from ph_brush_b200 import configs
    from ph_brush_b200.replicas import partition, replica_cost
    allr = configs.config5(seed=2029, n_rep=args.replicas * world)
    a, b = partition([replica_cost(s.n, p.mesh) for s, p in allr], world)[rank]
    return allr[a:b], [s.n for s, _ in allr]


def build_headline(args, local, rank, world):
    """Config-5 engine, autotuned, with a surrogate trained on the GPU on exact dE
    harvested from its own replicas (all of this is set-up, outside the timed region)."""
    from ph_brush_b200 import Engine, Surrogate
    reps, n_all = headline_replicas(args, rank, world)
    eng = Engine([s for s, _ in reps], [p for _, p in reps], device=local)
    if args.no_surrogate:  # profiling the exact path: no harvest, training or first stage
        return reps, n_all, eng, None, tune_engine(eng, args, args.trials), {}
    p0 = reps[0][1]
    sur = Surrogate(seed=2029)
    eng.set_move_mix(0.5, 0.5, 0.0)  # titration-heavy harvest
    eng.harvest(args.harvest)
    eng.run(2 * args.harvest // len(reps) + 1)
    n_samples = eng.harvest_count()
    t0 = time.perf_counter()
    loss = eng.surrogate_fit(sur, epochs=args.epochs, batch=4096, lr=1e-3, clip=25.0, seed=7)
    t_fit = time.perf_counter() - t0
    eng.harvest(0)
    eng.set_move_mix(p0.p_disp, p0.p_titr, p0.p_swap)
    eng.attach_surrogate(sur, threshold=args.da_threshold, window=256)
    # tuned as the timed steps run: surrogate attached, the step's trials per candidate
    tune = tune_engine(eng, args, args.trials)
    steps = args.epochs * (n_samples // 4096)
    fl_row = 2.0 * (80 * 128 + 2 * 128 * 128 + 128)  # forward flops per row; backward twice that
    train = {"samples": n_samples, "epochs": args.epochs, "batch": 4096, "lr": 1e-3, "final_loss": loss,
             "seconds": t_fit, "samples_per_s": steps * 4096 / t_fit,
             "tflops": steps * 4096 * 4 * 3 * fl_row / t_fit / 1e12}
    return reps, n_all, eng, sur, tune, train


def plain_aggregate(args, reps, local, trials, samples=3):
    """The plain engine (exact dE, no batching) on sampled replicas one at a time;
    aggregate rate over the set = R sweeps / sum_r (N_r t_r) estimated from the samples."""
    from ph_brush_b200 import Engine
    ns = [s.n for s, _ in reps]
    idx = sorted(range(len(reps)), key=lambda r: ns[r])
    pick = sorted({idx[0], idx[len(idx) // 2], idx[-1]})[:samples]
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
    return 1.0 / (sum(per_sweep_s) / len(per_sweep_s)), pick


def titration_phase(eng, sur, n_sites, threshold):
    """The reference's protonation phase as a move mix: titration only, plain against
    delayed acceptance, on the same engine."""
    eng.set_move_mix(0.0, 1.0, 0.0)
    eng.attach_surrogate(None)
    tt = int(max(n_sites))
    eng.run(tt)
    eng.flush_l2(256 << 20)
    ms_p = eng.run_timed(tt)
    eng.attach_surrogate(sur, threshold=0.0, window=0)
    eng.run(tt // 4)
    eng.flush_l2(256 << 20)
    ms_d = eng.run_timed(tt)
    ev, ps, ac = sums(eng.da_stats())
    R = len(n_sites)
    return {"trials_per_replica": tt, "plain_trials_per_s": R * tt / (ms_p / 1e3), "da_trials_per_s": R * tt / (ms_d / 1e3),
            "gain": ms_p / ms_d, "exact_dE_skipped": 1.0 - ps / max(ev, 1), "second_stage_agreement": ac / max(ps, 1)}


def engine_rate(eng, ns, trials, steps=3):
    """Aggregate sweeps/s and trials/s of `steps` timed runs of `trials` trials per replica
    (L2 flushed before each), with each kernel family's share and algorithmic bandwidth."""
    eng.set_profiling(True)
    eng.profile(reset=True)
    ms = 0.0
    for _ in range(steps):
        eng.flush_l2(256 << 20)
        ms += eng.run_timed(trials)
    prof = eng.profile(reset=True)
    eng.set_profiling(False)
    sweeps = steps * sum(trials / n for n in ns)
    out = {"sweeps_per_s": sweeps / (ms / 1e3), "trials_per_s": steps * trials * len(ns) / (ms / 1e3),
           "ms_per_run": ms / steps, "tuning": eng.tuning()}
    peak, kind = measured_peak()
    for name, t_ms, by, nl in (("k_mc", prof["mc_ms"], prof["mc_alg_bytes"], prof["mc_launches"]),
                               ("mesh_rebuild", prof["flush_ms"], prof["flush_alg_bytes"], prof["flush_launches"])):
        if nl:
            gbs = by / (t_ms / 1e3) / 1e9
            out[name] = {"share": t_ms / ms, "alg_gbs": gbs, "frac": gbs / peak, "peak_source": kind,
                         "launches": nl, "avg_launch_ms": t_ms / nl}
    return out


def config1_run(local, trials=20000):
    """Config 1: one small brush (16 chains x 20 beads, 4x4 lattice, 16x16x40 padded to 120,
    mesh 32x32x128, order 5), the plain engine (exact dE), autotuned."""
    from ph_brush_b200 import Engine, configs
    s, p = configs.config1()
    with Engine(s, p, device=local) as eng:
        tune = eng.autotune(4000)
        eng.run(trials)
        out = engine_rate(eng, [s.n], trials)
    out.update(workload="config 1: 16 chains x 20 titratable beads (pKa 7.5, pH 7.5), 16x16x40 padded to 120, "
                        "mesh 32x32x128, order 5, 90% displacement / 10% protonation, plain engine",
               particles=s.n, autotune_candidates=len(tune))
    return out


def config3_run(local, trials=1000):
    """Config 3: 96 replicas, pH 4.0-9.75 x salt 0.001-0.5 M, grafting density 0.05/0.1/0.2,
    chain length 30-60: uneven particle counts and meshes in one engine (one MC launch per
    chunk for all replicas, the Stockham z pass for the differing nz), exact dE, autotuned."""
    from ph_brush_b200 import Engine, configs
    reps = configs.config3()
    ns = [s.n for s, _ in reps]
    with Engine([s for s, _ in reps], [p for _, p in reps], device=local) as eng:
        tune = eng.autotune(trials)
        eng.run(trials)
        out = engine_rate(eng, ns, trials)
    out.update(workload="config 3: 96 replicas, pH 4.0-9.75 x salt {0.001, 0.01, 0.1, 0.5} M, grafting density "
                        "0.05/0.1/0.2, chains of 30-60 beads, meshes 32-36 x 162-288, batched exact",
               replicas=len(reps), particles_min_max=[min(ns), max(ns)], autotune_candidates=len(tune))
    return out


def config4_run(local, samples=2_000_000, epochs=4, trials=4000):
    """Config 4: the config-2 system (10x10 chains x 50 titratable beads, 0.1 M salt) with
    reservoir Na+/Cl- pair swaps (85 % displacement / 10 % protonation / 5 % swaps), at 8 pH
    values batched in one engine; 2e6 (descriptor, exact dE) samples harvested on the device
    from exact sweeps, the surrogate trained on them on the GPU (Adam lr 1e-3, batch 4096),
    then delayed acceptance against the exact engine on the same replicas."""
    import numpy as np
    from ph_brush_b200 import Engine, Surrogate, configs
    pHs = [5.5, 6.0, 6.5, 7.0, 7.5, 8.0, 8.5, 9.0]
    reps = []
    for k, pH in enumerate(pHs):
        s, p = configs.config4(seed=2026 + k)
        p.pH = pH
        reps.append((s, p))
    ns = [s.n for s, _ in reps]
    eng = Engine([s for s, _ in reps], [p for _, p in reps], device=local)
    eng.set_tuning(32, 256)
    eng.run(20 * max(ns))  # clear the generator's overlaps
    eng.harvest(samples)
    t0 = time.perf_counter()
    sweeps_h = 0.0
    while eng.harvest_count() < samples:
        eng.run(200000)
        sweeps_h += 200000 / float(np.mean(ns))
    t_h = time.perf_counter() - t0
    n = eng.harvest_count()
    sur = Surrogate(seed=41)
    t0 = time.perf_counter()
    loss = eng.surrogate_fit(sur, epochs=epochs, batch=4096, lr=1e-3, clip=25.0, seed=9)
    t_fit = time.perf_counter() - t0
    eng.harvest(0)
    fl_row = 2.0 * (80 * 128 + 2 * 128 * 128 + 128)
    steps = epochs * (n // 4096)
    train = {"samples": n, "epochs": epochs, "batch": 4096, "lr": 1e-3, "final_loss": loss, "seconds": t_fit,
             "samples_per_s": steps * 4096 / t_fit, "tflops": steps * 4096 * 4 * 3 * fl_row / t_fit / 1e12,
             "harvest_seconds": t_h, "harvest_sweeps_per_replica": sweeps_h}
    sweeps = float(sum(trials / x for x in ns))
    eng.run(trials // 4)
    eng.flush_l2(256 << 20)
    ms_ex = eng.run_timed(trials)
    eng.attach_surrogate(sur, threshold=0.3, window=256)
    eng.run(trials // 4)
    d0 = sums(eng.da_stats())
    eng.flush_l2(256 << 20)
    ms_da = eng.run_timed(trials)
    d1 = sums(eng.da_stats())
    # the titration and swap moves alone, where the first stage judges every trial
    eng.set_move_mix(0.0, 0.67, 0.33)
    eng.attach_surrogate(None)
    eng.run(trials // 4)
    ms_ex2 = eng.run_timed(trials)
    eng.attach_surrogate(sur, threshold=0.0, window=0)
    eng.run(trials // 4)
    e0 = sums(eng.da_stats())
    ms_da2 = eng.run_timed(trials)
    e1 = sums(eng.da_stats())
    eng.close()
    ev, ps, ac = (b - a for a, b in zip(d0, d1))
    ev2, ps2, ac2 = (b - a for a, b in zip(e0, e1))
    return {"workload": "config 4: config-2 system with reservoir Na+/Cl- swaps, 8 replicas at pH 5.5-9.0 "
                        "(85% displacement / 10% protonation / 5% swaps)",
            "particles": ns, "training": train,
            "exact_sweeps_per_s": sweeps / (ms_ex / 1e3), "da_sweeps_per_s": sweeps / (ms_da / 1e3),
            "gain": ms_ex / ms_da, "exact_dE_skipped": 1.0 - ps / max(ev, 1),
            "second_stage_agreement": ac / max(ps, 1),
            "titration_swap_only": {"exact_trials_per_s": len(ns) * trials / (ms_ex2 / 1e3),
                                    "da_trials_per_s": len(ns) * trials / (ms_da2 / 1e3), "gain": ms_ex2 / ms_da2,
                                    "exact_dE_skipped": 1.0 - ps2 / max(ev2, 1),
                                    "second_stage_agreement": ac2 / max(ps2, 1)}}


def _alpha(stats, n_sites):
    return [st["n_charged_sites"] / n for st, n in zip(stats, n_sites)]


def blocking_se(x):
    """Standard error of the mean of a correlated series (axis 0: consecutive samples): the
    largest naive error of the series averaged in blocks of 1, 2, 4, ... samples while at least
    five blocks remain (the blocking method, Flyvbjerg & Petersen 1989)."""
    import numpy as np
    x = np.asarray(x, np.float64)
    best = np.zeros(x.shape[1:])
    while x.shape[0] >= 5:
        best = np.maximum(best, np.sqrt(x.var(0, ddof=1) / x.shape[0]))
        m = x.shape[0] // 2
        x = 0.5 * (x[0:2 * m:2] + x[1:2 * m:2])
    return best


def alpha_check(local, sweeps_eq, sweeps_sample, per_bin=6, blocks=20, nbins=16, max_rounds=3):
    """alpha(pH) and z-profiles of delayed acceptance against the plain engine on real config-5
    replicas (in each pH bin 5-6, 6-7, 7-8, 8-9 the `per_bin` smallest of the headline set; its
    move mix; batched exact is the plain engine): the plain engine equilibrates until the drift
    of its degree of ionisation between the two halves of a sample is below 0.002 (at most
    max_rounds rounds); a second engine, with a surrogate trained on exact dE harvested from
    the equilibrated replicas as first stage, starts from the state the plain engine's last
    sample started from, so both sample the same `sweeps_sample` sweeps after the same state.
    Every 250 trials each replica's MC kernel adds its z-histogram (phmc_set_zhist), read
    back per block; the error of each replica's alpha difference is the blocking-method error
    of its per-block difference series."""
    import numpy as np
    from ph_brush_b200 import Engine, Surrogate, configs
    t0 = time.perf_counter()
    allr = configs.config5(seed=2029, n_rep=256)
    pH_all = np.array([p.pH for _, p in allr])
    idx = []
    for lo in (5.0, 6.0, 7.0, 8.0):
        m = [k for k in range(len(allr)) if lo <= pH_all[k] < lo + 1.0 + (1e-9 if lo == 8.0 else 0.0)]
        idx += sorted(m, key=lambda k: allr[k][0].n)[:per_bin]
    S, P = [allr[k][0] for k in idx], [allr[k][1] for k in idx]
    ns_site = np.array([s.meta["n_sites"] for s in S], np.float64)
    nmax = max(s.n for s in S)
    per_block = max(1, sweeps_sample * nmax // blocks)

    def sample(eng):
        """per-block alpha [blocks, R] and mean profiles [R, 3, nbins] over the sample"""
        eng.set_zhist(nbins, every=250)
        prev = [(np.zeros((3, nbins)), 0)] * len(S)
        a = []
        for _ in range(blocks):
            eng.run(per_block)
            cur = [eng.zhist(r) for r in range(len(S))]
            a.append([(c[0][0].sum() - p_[0][0].sum()) / max(c[1] - p_[1], 1) / ns_site[r]
                      for r, (c, p_) in enumerate(zip(cur, prev))])
            prev = cur
        prof = np.array([c[0] / max(c[1], 1) for c in prev])
        eng.set_zhist(0)
        return np.array(a), prof

    A = Engine(S, P, device=local)
    A.autotune(2000)
    A.run(sweeps_eq * nmax)
    # the first stage's network, trained on exact dE harvested from these equilibrated replicas
    # (the headline's network saw the generated, unrelaxed brushes only)
    A.harvest(131072)
    while A.harvest_count() < 131072:
        A.run(20000)
    sur = Surrogate(seed=31)
    fit_loss = A.surrogate_fit(sur, epochs=12, batch=2048, lr=1e-3, clip=25.0, seed=3)
    A.harvest(0)
    rounds, drift = 0, 1.0
    while True:
        rounds += 1
        start = A.state(-1)
        a_p, prof_p = sample(A)
        half = blocks // 2
        drift = float(np.abs(a_p[half:].mean(0) - a_p[:half].mean(0)).mean())
        if drift < 0.002 or rounds >= max_rounds:
            break
    B = Engine(S, P, device=local)
    tn = A.tuning()
    B.set_tuning(tn["pending_max"], tn["threads"])
    B.set_state(start, -1)
    B.attach_surrogate(sur, threshold=0.0, window=0)
    a_d, prof_d = sample(B)
    ev, ps, ac = sums(B.da_stats())
    A.close()
    B.close()
    mp, md = a_p.mean(0), a_d.mean(0)
    se = blocking_se(a_d - a_p)  # per replica: both chains' blocks cover the same trials after one state
    se_unpaired = np.sqrt(blocking_se(a_p) ** 2 + blocking_se(a_d) ** 2)
    pH = np.array([p.pH for p in P])
    curve = []
    for lo in (5.0, 6.0, 7.0, 8.0):
        m = (pH >= lo) & (pH < lo + 1.0 + (1e-9 if lo == 8.0 else 0.0))
        if not m.any():
            continue
        se_b = float(np.sqrt((se[m] ** 2).sum()) / m.sum())
        diff = float(md[m].mean() - mp[m].mean())
        curve.append({"pH": [lo, lo + 1.0], "replicas": int(m.sum()), "alpha_plain": float(mp[m].mean()),
                      "alpha_da": float(md[m].mean()), "diff": diff, "stderr": se_b,
                      "stderr_unpaired": float(np.sqrt((se_unpaired[m] ** 2).sum()) / m.sum()),
                      "within_2se": abs(diff) <= 2 * se_b})
    # z-profiles: per bin, the replica-mean profile difference against its spread over replicas
    dprof = prof_d - prof_p
    zscore = np.abs(dprof.mean(0)) / (dprof.std(0, ddof=1) / np.sqrt(len(S)) + 1e-12)
    max_diff = float(max(abs(c["diff"]) for c in curve))
    return {"workload": f"config-5 replicas, the {per_bin} smallest in each pH bin 5-6, 6-7, 7-8, 8-9 "
                        f"({min(s.n for s in S)}-{nmax} particles), 90% displacement / 10% protonation, "
                        "batched exact as the plain engine",
            "sweeps_equilibrate": sweeps_eq + (rounds - 1) * sweeps_sample, "sweeps_sample": sweeps_sample,
            "blocks": blocks, "rounds": rounds, "fit_loss": fit_loss, "exact_dE_skipped": 1.0 - ps / max(ev, 1),
            "second_stage_agreement": ac / max(ps, 1), "pH_curve": curve,
            "stderr_method": "blocking method on each replica's per-block difference series; both chains "
                             "start from the same state and sample the same number of trials",
            "max_curve_diff": max_diff, "within_0_005": max_diff <= 0.005,
            "all_within_2se": bool(all(c["within_2se"] for c in curve)),
            "mean_abs_diff_per_replica": float(np.abs(md - mp).mean()),
            "median_stderr_per_replica": float(np.median(se)), "plain_drift_between_halves": drift,
            "z_profile_bins": nbins,
            "z_profile_max_zscore": {"sites": float(zscore[0].max()), "anions": float(zscore[1].max()),
                                     "cations": float(zscore[2].max())},
            "seconds": time.perf_counter() - t0}


def plain_config2(args, local):
    """The plain engine (one replica, exact dE) on config 2: the comparison with the
    reference's CUDA build on the same system."""
    from ph_brush_b200 import Engine, configs
    s, p = configs.config2()
    eng = Engine(s, p, device=local)
    tuned = tune_engine(eng, args, max(2000, s.n // 4))
    eng.run(s.n)
    eng.set_profiling(True)
    eng.profile(reset=True)
    ms = 0.0
    for _ in range(3):
        eng.flush_l2(256 << 20)
        ms += eng.run_timed(s.n)
    prof = eng.profile(reset=True)
    out = {"workload": CFG2, "particles": s.n, "sweeps_per_s": 3 / (ms / 1e3), "trials_per_s": 3 * s.n / (ms / 1e3),
           "tuning": eng.tuning(), "autotune": tuned,
           "k_mc_share": prof["mc_ms"] / ms if ms else None,
           "k_mc_alg_gbs": prof["mc_alg_bytes"] / (prof["mc_ms"] / 1e3) / 1e9 if prof["mc_ms"] else None}
    eng.close()
    return out, (s, p)


def reference_phase2_on_device(local, ref_dir, attempts=2000):
    """The reference's phase 2 (MC/src/mc.cu:159-318) run on the device (phmc_phase2) on
    the files the reference arm's harness times it on (config 2 in the reference's model,
    written by oracle/_build/ref_inputs, read through the library's readers), with the
    same settings and generator seed (std::mt19937(2025)): attempts/s of the same loop,
    the same draws and acceptance rule, device loop against the reference's host loop."""
    import numpy as np
    from ph_brush_b200 import Engine, files
    s, p = files.reference_model(os.path.join(ref_dir, "c2.data"), os.path.join(ref_dir, "c2.params"))
    t = s.type
    nhn, nhp, w, cl = 3, 4, 6, 7  # the reference's types 4, 5, 7, 8, 0-based
    sites = np.where((t == nhn) | (t == nhp))[0]
    z_cut = float(np.max(s.z[sites])) + 1.0  # w_z_extra_nm's default (MC/include/types.hpp)
    job = dict(replica=0, nh_n_type=nhn, nh_p_type=nhp, w_type=w, cl_type=cl, beta=1.0, patience=1 << 30,
               energy_interval=1 << 30, z_cut=z_cut, nh_p=np.where(t == nhp)[0], nh_n=np.where(t == nhn)[0],
               w=np.where((t == w) & (s.z < z_cut))[0], cl=np.where((t == cl) & (s.z < z_cut))[0])
    mt = np.zeros(625, np.uint32)  # std::mt19937(2025)
    v = 2025
    mt[0] = v
    for i in range(1, 624):
        v = (1812433253 * (v ^ (v >> 30)) + i) & 0xFFFFFFFF
        mt[i] = v
    mt[624] = 624
    with Engine(s, p, device=local) as eng:
        eng.phase2([dict(job, mt_state=mt, max_attempts=50)])  # warm-up
        t0 = time.perf_counter()
        (res, _), = eng.phase2([dict(job, mt_state=mt, max_attempts=attempts)])
        sec = time.perf_counter() - t0
    return {"workload": "config 2 in the reference's model (" + str(s.n) + " atoms), its phase 2 on the device "
                        "(four-point identity swaps, float Metropolis on the reference's energies)",
            "attempts": res["attempted"], "accepted": res["accepted"], "seconds": sec,
            "attempts_per_s": res["attempted"] / sec, "mesh": list(p.mesh),
            "timing": "host wall clock around the synchronous call (launches, rebuilds, event copies)"}


def cpu_baseline(ref_dir, name, seconds):
    """The reference's per-trial loop restated in FP64 on the host cores (oracle.pyoracle.
    RefTrialLoop: half list built once, LJ + cubic SPME recomputed every trial, OpenMP)
    on one config-5 replica in the reference's model, in the benchmark's move mix."""
    import numpy as np
    from oracle import pyoracle as O
    from ph_brush_b200 import files
    base = os.path.join(ref_dir, name)
    s, p = files.reference_model(base + ".data", base + ".params")
    ex = open(base + ".extra").read().split()
    kv = {ex[k]: ex[k + 1] for k in range(0, ex.index("mobile"), 2)}
    nmob = int(ex[ex.index("mobile") + 1])
    mobile = np.array([int(v) for v in ex[ex.index("mobile") + 2:ex.index("mobile") + 2 + nmob]])
    loop = O.RefTrialLoop(s, p, mobile, float(kv["height"]), float(kv["pH"]), float(kv["pKa"]), seed=5)
    n = 0
    t0 = time.perf_counter()
    while True:
        loop.trial(0.9)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds and n >= 2:
            break
    tps = n / el
    n_native = int(kv["n_native"])
    cores = os.cpu_count()
    return {"value": tps / n_native, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} trials of config-5 replica {name} ({n_native} particles, {s.n} atoms in the reference's "
                      f"model, mesh {list(p.mesh)}) in {el:.1f} s: the reference's per-trial loop restated in FP64 "
                      f"(half list built once, LJ + cubic SPME per trial) on {cores} OpenMP threads; sweeps/s = "
                      f"trials/s / {n_native}: one replica's rate, the host's aggregate over a replica set run one "
                      f"at a time",
            "trials_per_s": tps}


def run_ours(args):
    rank, world, local = dist_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import numpy as np

    reps, n_all, eng, sur, tune, train = build_headline(args, local, rank, world)
    ns = np.array([s.n for s, _ in reps], np.float64)
    T = args.trials
    sweeps_per_step = float((T / ns).sum())  # this rank's replicas
    total_sweeps_per_step = reduce_sum(sweeps_per_step, world, local)  # all ranks
    for _ in range(args.warmup):
        eng.run(T)
    # ---- device-timed region: inputs resident, L2 flushed between steps ----
    eng.set_profiling(True)
    eng.profile(reset=True)
    da0 = sums(eng.da_stats())
    clocks = Clocks(local)
    barrier(world)
    dev_ms = 0.0
    for _ in range(args.steps):
        eng.flush_l2(256 << 20)
        dev_ms += eng.run_timed(T)
    barrier(world)
    clk = clocks.stop()
    prof = eng.profile(reset=True)
    eng.set_profiling(False)
    da1 = sums(eng.da_stats())
    max_ms = reduce_max(dev_ms, world, local)
    value = args.steps * total_sweeps_per_step / (max_ms / 1e3)

    # ---- end to end through the public API: pinned host state of every replica in,
    #      state and energies out, every step ----
    st = eng.state(-1)
    try:
        import torch
        pinned = {k: torch.from_numpy(v.copy()).pin_memory().numpy() for k, v in st.items()}
        readback = {k: torch.from_numpy(v.copy()).pin_memory().numpy() for k, v in st.items()}
    except Exception:
        pinned = {k: v.copy() for k, v in st.items()}
        readback = {k: v.copy() for k, v in st.items()}
    slots = len(st["x"])
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.set_state(pinned, -1)
        res = eng.run(T)
        out = eng.state(-1, out=readback)
        energies = [r["energy"] for r in res]
    e2e_s = time.perf_counter() - t0
    barrier(world)
    e2e_s = reduce_max(e2e_s, world, local)
    e2e = {"value": args.steps * total_sweeps_per_step / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": slots * (16 + 4 + 4), "d2h_bytes_per_step": slots * (16 + 4 + 4) + 8 * len(reps),
           "timing": "host wall clock around phmc_set_state(all replicas, from pinned host arrays) + phmc_run + "
                     "phmc_get_state(all replicas, into pinned host arrays), synchronous calls"}
    del out, energies

    # ---- roofline of the dominant kernel (MC kernel or the fused rebuild) ----
    peak, peak_kind = measured_peak()
    kern = []
    if prof["mc_launches"]:
        kern.append(("k_mc", prof["mc_ms"], prof["mc_launches"], prof["mc_alg_bytes"]))
    if prof["flush_launches"]:
        kern.append(("mesh_rebuild", prof["flush_ms"], prof["flush_launches"], prof["flush_alg_bytes"]))
    kern.sort(key=lambda k: -k[1])
    rl = {}
    for name, tot, n_l, by in kern:
        ms = tot / n_l
        per = by / n_l
        ach = per / (ms / 1e3) / 1e9
        ratio = ncu_traffic_ratio(name)
        rl[name] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "peak_source": peak_kind, "traffic": ratio * per if ratio else None,
                    "alg_bytes_per_launch": per, "avg_launch_ms": ms, "launches": n_l,
                    "share_of_timed": tot / dev_ms if dev_ms else None}
        if name == "k_mc":  # share of the launches' replica slots (one block per replica) that did work
            rl[name]["replica_busy_fraction"] = prof["mc_busy_ms"] / (len(reps) * tot) if tot else None
    dominant = kern[0][0] if kern else None

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 pair/mesh/FFT, f64 accumulation and Metropolis, bf16 surrogate",
            "data": "synthetic (seeded brush generator, config-5 seed 2029; 256 replicas per GPU split by cost)",
            "config": workload_config(len(n_all), n_all),
            "step": {"trials_per_replica": T, "sweeps": total_sweeps_per_step, "replicas_this_rank": len(reps),
                     "l2": "flushed between steps (256 MiB write on the engine stream)"},
            "tuning": {"chosen": eng.tuning(), "autotune": tune, "da_threshold": args.da_threshold},
            "roofline": dict(rl[dominant], kernel=dominant) if dominant else None,
            "roofline_other": {k: v for k, v in rl.items() if k != dominant},
            "e2e": e2e, "gpu_launches": int(prof["kernel_launches"]),
            "trials_per_s": world * prof["trials"] / (max_ms / 1e3) if prof["trials"] else None,
            "surrogate": {"training": train,
                          "first_stage": bool(eng.tuning()["first_stage"]),
                          "judged_trials": int(da1[0] - da0[0]),
                          "exact_dE_skipped": (1.0 - (da1[1] - da0[1]) / (da1[0] - da0[0])) if da1[0] > da0[0] else None,
                          "second_stage_agreement": ((da1[2] - da0[2]) / (da1[1] - da0[1])) if da1[1] > da0[1] else None,
                          "fallbacks": int(sum(d["fallback"] for d in eng.da_stats()))},
            "clocks": clk}
    if rank == 0 and world == 1:
        # where a trial's time goes (after the timed region): SM cycles per trial of each MC-kernel
        # phase, summed over the replicas' blocks (one extra barrier per trial while measured)
        eng.set_phase_clock(True)
        eng.phase_cycles(reset=True)
        eng.run(max(T // 4, 1))
        pc = eng.phase_cycles(reset=True)
        eng.set_phase_clock(False)
        if pc["trials"]:
            line["k_mc_phase_cycles_per_trial"] = {k: v / pc["trials"] for k, v in pc.items() if k != "trials"}
    if rank == 0 and world == 1 and not args.no_extras:
        plain, pick = plain_aggregate(args, reps, local, 400)
        line["plain_aggregate_sweeps_per_s"] = plain
        line["plain_sampled_replicas"] = pick
        line["speedup_vs_plain"] = value / plain
        # batched exact (no surrogate) on the same engine, for the split of the gain
        eng.attach_surrogate(None)
        eng.run(T // 4)
        eng.flush_l2(256 << 20)
        ms_ex = eng.run_timed(T)
        line["batched_exact_sweeps_per_s"] = sweeps_per_step / (ms_ex / 1e3)
        if sur is not None:
            line["titration_phase"] = titration_phase(eng, sur, [int(s.meta["n_sites"]) for s, _ in reps],
                                                      args.da_threshold)
    eng.close()
    ref_dir = tempfile.mkdtemp(prefix="phmc_ref_")
    if rank == 0 and world == 1 and (not args.no_extras or not args.no_cpu_baseline):
        k_small = int(np.argmin(n_all))
        write_ref_inputs([config2_spec_line(), config5_spec_lines(2029, len(n_all))[k_small]], ref_dir)
    if rank == 0 and world == 1 and not args.no_extras:
        line["plain_config2"], c2 = plain_config2(args, local)
        try:
            line["reference_phase2_on_device"] = reference_phase2_on_device(local, ref_dir)
        except Exception as e:  # an extra: the headline line is printed regardless
            line["reference_phase2_on_device"] = {"error": str(e)[:300]}
        if not args.no_alpha:
            line["alpha_check"] = alpha_check(local, args.alpha_eq, args.alpha_sample)
        for key, fn, off in (("config1", config1_run, args.no_config1), ("config3", config3_run, args.no_config3),
                             ("config4", config4_run, args.no_config4)):
            if off:
                continue
            try:
                line[key] = fn(local)
            except Exception as e:  # an extra: the headline line is printed regardless
                line[key] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ref_dir, f"c5_{k_small:04d}", args.cpu_seconds)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# reference arm: the reference's CUDA build, one replica at a time
# ---------------------------------------------------------------------------
def run_harness(args_):
    r = subprocess.run([REF_HARNESS] + [str(a) for a in args_], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference harness failed: " + (r.stderr.strip() or r.stdout.strip())[-300:])
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    n_gpus = max(world, args.gpus)
    if not (os.path.exists(REF_HARNESS) and os.path.exists(REF_INPUTS)):
        print(json.dumps({"impl": "reference", "unavailable": "reference CUDA build or input writer missing: run "
                                                              "`make -C oracle ref inputs`"}))
        return
    if local:
        os.environ.setdefault("CUDA_VISIBLE_DEVICES", str(local))
    d = tempfile.mkdtemp(prefix="phmc_ref_")
    n_rep = args.replicas * n_gpus
    try:
        t0 = time.perf_counter()
        info = write_ref_inputs(config5_spec_lines(2029, n_rep) + [config2_spec_line()], d)
        t_inputs = time.perf_counter() - t0
        names = [f"c5_{k:04d}" for k in range(n_rep)]
        with open(os.path.join(d, "list.txt"), "w") as fh:
            fh.write("\n".join(os.path.join(d, nm) for nm in names) + "\n")
        mix = run_harness(["mix", os.path.join(d, "list.txt"), args.steps, args.warmup, args.ref_trials, 0.9, 0.3, 2025])
        with open(os.path.join(d, "list2.txt"), "w") as fh:
            fh.write(os.path.join(d, "c2") + "\n")
        mix2 = run_harness(["mix", os.path.join(d, "list2.txt"), 3, 1, 400, 0.9, 0.3, 2025])
        p2 = run_harness(["time", os.path.join(d, "c2.data"), os.path.join(d, "c2.params"), 2000, 50])
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)[:300]}))
        return
    n_native = mix["n_native"]
    assert n_native == [info[nm][1] for nm in names]
    sweeps_per_step = sum(args.ref_trials / n for n in n_native)
    secs = mix["seconds"]
    value = args.steps * sweeps_per_step / secs
    n2 = info["c2"][1]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n_gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (the same seeded brush generator: oracle/_build/ref_inputs)",
            "config": workload_config(n_rep, n_native),
            "step": {"trials_per_replica": args.ref_trials, "sweeps": sweeps_per_step,
                     "note": "a bounded sample of the step: every replica, a few trials each"},
            "reference_path": "the reference's CUDA build (oracle/_ref/ref_harness linked with MC/src/*.o, sm_100a): "
                              "per trial its device writes (set_atom_identity), its total energy (LJ over the half "
                              "list + pmeEnergy: memset, cubic spread, cuFFT R2C, influence, Thrust reductions; "
                              "MC/src/mc.cu:43-60), its acceptance (GC pair flips, MC/src/mc.cu:379-440, mu = kT "
                              "ln10 (pKa - pH); displacements: Metropolis on its float energies), writes back on "
                              "rejection; replicas one after the other",
            "model_differences": "in its own model: LJ cut and shifted at 3 sigma (no WCA / FENE), cubic SPME (the "
                                 "reference has no other order), mesh from pme_spacing 0.75 (" +
                                 str(sorted({tuple(m) for m in mix["meshes"]})) + "), a W-bead identity pool per "
                                 "titratable site, the half list built once (not rebuilt after displacements); each "
                                 "of these makes its trial cheaper, not dearer",
            "attempted": mix["attempted"], "accepted": mix["accepted"], "setup_seconds": mix["setup_seconds"],
            "inputs_seconds": t_inputs,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{args.ref_trials * args.steps} timed trials per replica of all {n_rep} "
                                       "replicas in the reference's CUDA build on this B200 (one host thread drives "
                                       "it), CUDA-event timed per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "config2": {"workload": CFG2 + " -- in the reference's model (" + str(info["c2"][0]) + " atoms, mesh " +
                                    str(mix2["meshes"][0]) + ")",
                        "mix_sweeps_per_s": 3 * 400 / n2 / mix2["seconds"], "mix_trials_per_s": 3 * 400 / mix2["seconds"],
                        "phase2_attempts_per_s": p2["trials_per_s"], "phase2_wall_attempts_per_s":
                            p2["trials"] / p2["wall_seconds"], "phase2_attempts": p2["trials"]}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.plain_config2_only:
        rank, world, local = dist_env()
        out, _ = plain_config2(args, local)
        if rank == 0:
            print(json.dumps(out))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
