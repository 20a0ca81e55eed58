"""Learned surrogate and delayed acceptance.

CPU: the oracle's network gradient against finite differences, the BF16
emulation against the exact gradient, and the antisymmetry of the descriptor
rows under move reversal (the property delayed acceptance relies on).
GPU: the engine's descriptor rows against the oracle bit for bit; the BF16
tensor-core forward, backward and Adam step against the oracle; in-kernel
inference against the standalone GEMM path; exactness of delayed acceptance
with an untrained network; the fallback threshold; and what a trained network
gains over the plain method on an interacting brush.
"""
import numpy as np
import pytest

from oracle import surrogate_oracle as SO
from ph_brush_b200 import Engine, Surrogate, _abi, configs

K, R = _abi.SUR_INPUTS, _abi.SUR_ROWS


def random_samples(rng, n, nin=K):
    x = rng.normal(0.0, 1.0, (n, R, nin)).astype(np.float32)
    m = min(64, nin)
    x[:, :, :m] = rng.poisson(3.0, (n, R, m)).astype(np.float32)
    sign = np.zeros((n, R), np.float32)
    sign[:, 0], sign[:, 1] = -1.0, 1.0
    sign[rng.random(n) < 0.5, 2] = 1.0
    t = rng.normal(0.0, 3.0, n).astype(np.float32)
    return x, sign, t


def small_params(rng, nin, H):
    sizes = [nin * H, H, H * H, H, H * H, H, H, 1]
    parts = []
    for k, n in enumerate(sizes):
        fan = nin if k == 0 else H
        parts.append(rng.normal(0.0, np.sqrt(2.0 / fan) if k % 2 == 0 or k == 6 else 0.1, n))
    return np.concatenate(parts).astype(np.float32)


# ---------------------------------------------------------------------------
# CPU: oracle pins
# ---------------------------------------------------------------------------
def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    nin, H, n = 6, 16, 5
    p = small_params(rng, nin, H).astype(np.float64)
    x, sign, t = random_samples(rng, n, nin)
    mu, sd = np.zeros(nin), np.ones(nin)
    loss, g = SO.loss_grad(p, nin, H, mu, sd, 2.0, x, sign, t, 25.0, bf=False)
    idx = rng.choice(len(p), 40, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = SO.loss_grad(pp, nin, H, mu, sd, 2.0, x, sign, t, 25.0, bf=False)
        lm, _ = SO.loss_grad(pm, nin, H, mu, sd, 2.0, x, sign, t, 25.0, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_gradient_tracks_exact_gradient():
    rng = np.random.default_rng(2)
    nin, H, n = K, 128, 64
    p = small_params(rng, nin, H)
    x, sign, t = random_samples(rng, n)
    mu, sd = x.reshape(-1, nin).mean(0), x.reshape(-1, nin).std(0) + 1.0
    _, g_bf = SO.loss_grad(p, nin, H, mu, sd, 3.0, x, sign, t, 25.0, bf=True)
    _, g_ex = SO.loss_grad(p, nin, H, mu, sd, 3.0, x, sign, t, 25.0, bf=False)
    cos = g_bf @ g_ex / (np.linalg.norm(g_bf) * np.linalg.norm(g_ex))
    assert cos > 0.995, cos


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], np.float32)
    r = SO.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -6) and r[3] == -2.5
    assert abs(r[4] - 1e-3) < 1e-3 * 2 ** -8


def _brush_state(seed=5):
    s, p = configs.config1(seed=seed)
    st = {"x": s.x.copy(), "y": s.y.copy(), "z": s.z.copy(), "q": s.q.copy(), "flags": s.flags.copy()}
    return s, p, st


def _grid(s, p):
    rmax = max(float(np.max(p.lj_rc)) if p.lj_rc is not None else p.rc_lj, p.rc_coul)
    dims = [int(np.floor(s.box[k] / rmax)) for k in range(3)]
    return SO.Geometry(s.box, dims, p)


def test_descriptor_rows_flip_sign_under_reversal():
    """The rows of a move and of its reverse (taken in the moved state) are the same
    rows with opposite signs: the environment excludes the changed particles."""
    s, p, st = _brush_state()
    geo = _grid(s, p)
    rng = np.random.default_rng(3)
    n = len(st["x"])
    sites = np.nonzero(((st["flags"] & _abi.F_TITRATABLE) != 0) & (st["q"] == 0))[0]
    i = int(sites[0])
    g = n  # append one empty slot for the inserted counterion
    for k in ("x", "y", "z", "q"):
        st[k] = np.append(st[k], np.float32(0.0))
    st["flags"] = np.append(st["flags"], np.int32(_abi.F_GHOST))
    pos = (np.float32(rng.uniform(0, s.box[0])), np.float32(rng.uniform(0, s.box[1])), np.float32(rng.uniform(0, 40.0)))
    fwd = [(i, True, (st["x"][i], st["y"][i], st["z"][i], np.float32(1.0))), (g, True, pos + (np.float32(-1.0),))]
    rows_f, sg_f, nr_f = SO.descriptor(st, geo, fwd)
    # apply the move
    st2 = {k: v.copy() for k, v in st.items()}
    st2["q"][i] = 1.0
    st2["x"][g], st2["y"][g], st2["z"][g], st2["q"][g] = pos + (np.float32(-1.0),)
    st2["flags"][g] = _abi.F_MOBILE | _abi.F_ANION
    rev = [(i, True, (st2["x"][i], st2["y"][i], st2["z"][i], np.float32(0.0))), (g, False, None)]
    rows_r, sg_r, nr_r = SO.descriptor(st2, geo, rev)
    assert nr_f == nr_r == 3
    key = lambda rows, sg, nr: sorted((tuple(rows[k]), float(sg[k])) for k in range(nr))
    assert key(rows_f, sg_f, nr_f) == key(rows_r, -sg_r, nr_r)
    assert rows_f[:nr_f, :64].sum() > 0


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.fixture(params=[1, 0], ids=["tcgen05", "mma_sync"])
def gemm_path(request):
    """The training products on the fifth-generation tensor cores (tcgen05.mma, TMEM
    accumulator) and on the mma.sync path; the process-wide switch is restored after."""
    lib = _abi.lib()
    assert lib.phmc_surrogate_set_gemm(request.param) == 0
    yield request.param
    lib.phmc_surrogate_set_gemm(1)


@pytest.mark.gpu
def test_forward_matches_oracle(gemm_path):
    rng = np.random.default_rng(10)
    sur = Surrogate(seed=3)
    x = rng.normal(0, 1, (300, K)).astype(np.float32)
    mu, sd = rng.normal(0, 0.2, K).astype(np.float32), rng.uniform(0.5, 2.0, K).astype(np.float32)
    sur.set_scaling(mu, sd, 2.5)
    y = sur.predict(x)
    yo, _, _ = SO.forward(sur.params(), K, 128, mu, sd, x, bf=True)
    yo = 2.5 * yo
    err = np.abs(y - yo) / (np.abs(yo) + 1.0)
    assert np.median(err) < 2e-3 and err.max() < 3e-2, (np.median(err), err.max())


@pytest.mark.gpu
def test_gradient_matches_oracle(gemm_path):
    rng = np.random.default_rng(11)
    sur = Surrogate(seed=4)
    x, sign, t = random_samples(rng, 256)
    mu = x.reshape(-1, K).mean(0)
    sd = x.reshape(-1, K).std(0) + 0.5
    sur.set_scaling(mu, sd, 3.0)
    loss, g = sur.gradient(x, sign, t, clip=25.0)
    lo, go = SO.loss_grad(sur.params(), K, 128, mu, sd, 3.0, x, sign, t, 25.0, bf=True)
    _, gx = SO.loss_grad(sur.params(), K, 128, mu, sd, 3.0, x, sign, t, 25.0, bf=False)
    assert abs(loss - lo) <= 1e-3 * abs(lo) + 1e-6, (loss, lo)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel < 1e-2, rel
    cos = g @ gx / (np.linalg.norm(g) * np.linalg.norm(gx))
    assert cos > 0.99, cos


@pytest.mark.gpu
def test_tcgen05_and_mma_sync_gradients_agree_at_batch_4096():
    """A training batch's products (M = 16384 rows, weight gradients split over K) on both
    tensor-core paths: the same FP32 sums in other orders, so the same gradient to FP32
    rounding of the BF16 products' sums."""
    rng = np.random.default_rng(14)
    x, sign, t = random_samples(rng, 4096)
    mu, sd = x.reshape(-1, K).mean(0), x.reshape(-1, K).std(0) + 0.5
    out = []
    lib = _abi.lib()
    try:
        for path in (1, 0):
            lib.phmc_surrogate_set_gemm(path)
            sur = Surrogate(seed=15)
            sur.set_scaling(mu, sd, 3.0)
            out.append(sur.gradient(x, sign, t, clip=25.0))
    finally:
        lib.phmc_surrogate_set_gemm(1)
    (l1, g1), (l0, g0) = out
    assert abs(l1 - l0) <= 1e-4 * abs(l0), (l1, l0)
    assert np.linalg.norm(g1 - g0) <= 2e-3 * np.linalg.norm(g0), np.linalg.norm(g1 - g0) / np.linalg.norm(g0)


@pytest.mark.gpu
def test_adam_first_step_matches_oracle():
    rng = np.random.default_rng(12)
    sur = Surrogate(seed=5)
    x, sign, t = random_samples(rng, 128)
    mu, sd = x.reshape(-1, K).mean(0), x.reshape(-1, K).std(0) + 0.5
    sur.set_scaling(mu, sd, 3.0)
    p0 = sur.params()
    _, g = sur.gradient(x, sign, t)
    sur.train(x, sign, t, epochs=1, batch=128, lr=1e-3, rescale=False)
    p1 = sur.params()
    pe, _, _ = SO.adam_step(p0.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, 1e-3)
    big = np.abs(g) > 1e-4 * np.abs(g).max()
    assert np.max(np.abs((p1 - pe)[big])) < 1e-5, np.max(np.abs((p1 - pe)[big]))


@pytest.mark.gpu
def test_training_fits_a_smooth_target():
    rng = np.random.default_rng(13)
    n = 8192
    x, sign, _ = random_samples(rng, n)
    w = rng.normal(0, 0.1, K).astype(np.float32)
    per_row = x @ w + 0.05 * np.sin(x[..., 3])
    t = (sign * per_row).sum(1).astype(np.float32)
    sur = Surrogate(seed=6)
    l0 = sur.train(x, sign, t, epochs=1, batch=512, lr=1e-3)
    l1 = sur.train(x, sign, t, epochs=30, batch=512, lr=1e-3, rescale=False)
    assert l1 < 0.05 * l0, (l0, l1)


@pytest.mark.gpu
def test_save_load_roundtrip(tmp_path):
    sur = Surrogate(seed=7)
    rng = np.random.default_rng(14)
    sur.set_scaling(rng.normal(0, 1, K), rng.uniform(0.5, 1.5, K), 1.7)
    x = rng.normal(0, 1, (16, K)).astype(np.float32)
    sur.save(tmp_path / "s.bin")
    s2 = Surrogate.load(tmp_path / "s.bin")
    assert np.array_equal(sur.params(), s2.params())
    assert np.array_equal(sur.predict(x), s2.predict(x))


def _move_trials(st, box, height, rng):
    """A protonation (+ counterion insert), a deprotonation (+ anion delete), a
    salt-pair insert and a salt-pair delete, as external trials."""
    fl, q, n = st["flags"], st["q"], len(st["flags"])
    ghosts = np.nonzero(fl & _abi.F_GHOST)[0]
    neutral = np.nonzero(((fl & _abi.F_TITRATABLE) != 0) & (q == 0))[0]
    charged = np.nonzero(((fl & _abi.F_TITRATABLE) != 0) & (q != 0))[0]
    anions = np.nonzero(fl & _abi.F_ANION)[0]
    cations = np.nonzero(fl & _abi.F_CATION)[0]
    rp = lambda: (float(np.float32(rng.uniform(0, box[0]))), float(np.float32(rng.uniform(0, box[1]))),
                  float(np.float32(rng.uniform(0, height))))
    site = lambda i, qn, tn: {"index": int(i), "present": 1, "x": st["x"][i], "y": st["y"][i], "z": st["z"][i], "q": qn, "type": tn}
    ion = lambda i, pos, qn, tn: {"index": int(i), "present": 1, "x": pos[0], "y": pos[1], "z": pos[2], "q": qn, "type": tn}
    gone = lambda i: {"index": int(i), "present": 0, "x": 0.0, "y": 0.0, "z": 0.0, "q": 0.0, "type": int(st["type"][i])}
    trials = []
    for k in range(6):
        trials.append([site(neutral[k], 1.0, 1), ion(ghosts[-1 - k], rp(), -1.0, 2)])
        trials.append([site(charged[k], 0.0, 0), gone(anions[k])])
        trials.append([ion(ghosts[-1 - k], rp(), 1.0, 3), ion(ghosts[-7 - k], rp(), -1.0, 2)])
        if len(cations) > k:
            trials.append([gone(cations[k]), gone(anions[-1 - k])])
    return trials


def _oracle_rows(st, geo, trial):
    ch = [(c["index"], bool(c["present"]), tuple(np.float32(v) for v in (c["x"], c["y"], c["z"], c["q"])))
          for c in trial]
    return SO.descriptor(st, geo, ch)


def _small_four_cells():
    # 12 x 12 sigma lateral box: 4 cells per axis, fewer than the 8-sigma window's 7
    s, p = configs.small_system(seed=71, chains=3, length=12, box_xy=12.0, height=14.0, salt_pairs=8)
    return s, p


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["config1", "four_cells"])
def test_descriptor_rows_match_oracle_bit_for_bit(case):
    s, p = configs.config1(seed=31) if case == "config1" else _small_four_cells()
    height = float(s.meta["height"])
    rng = np.random.default_rng(15)
    with Engine(s, p) as e:
        e.run(20000)  # move away from the generated state
        st = e.state()
        _, dims = e.cells()
        geo = SO.Geometry(s.box, dims, p)
        trials = _move_trials(st, s.box, height, rng)
        out = e.describe(trials)
    for t, o in zip(trials, out):
        rows, sg, nr = _oracle_rows(st, geo, t)
        assert o["nrows"] == nr
        assert np.array_equal(o["sign"][:nr], sg[:nr])
        assert np.array_equal(o["rows"][:nr], rows[:nr]), np.argwhere(o["rows"][:nr] != rows[:nr])[:5]
        assert o["rows"][:nr, :64].sum() > 0


@pytest.mark.gpu
def test_in_kernel_inference_matches_gemm_path():
    s, p = configs.config1(seed=32)
    rng = np.random.default_rng(16)
    sur = Surrogate(seed=8)
    sur.set_scaling(np.full(K, 2.0), np.full(K, 3.0), 4.0)
    with Engine(s, p) as e:
        st = e.state()
        e.attach_surrogate(sur)
        out = e.describe(_move_trials(st, s.box, 40.0, rng))
    for o in out:
        nr = o["nrows"]
        F = sur.predict(o["rows"][:nr])
        assert np.allclose(o["F"][:nr], F, rtol=1e-5, atol=1e-5), (o["F"][:nr], F)
        # estimate = per changed particle F(new) - F(old), plus the exact terms
        assert np.isfinite(o["dEs"])


def _ideal(seed):
    s, p = configs.small_system(seed=seed, chains=3, length=12, box_xy=12.0, height=14.0, salt_pairs=0, lb=0.0)
    p.lj_eps = p.lj_eps * 0
    p.fene_k = 0.0
    p.p_disp, p.p_titr = 0.5, 0.5
    return s, p


@pytest.mark.gpu
def test_delayed_acceptance_is_exact_with_an_untrained_network():
    """Ideal titration: any first stage must leave alpha(pH) = 1/(1+10^(pH-pKa))."""
    sur = Surrogate(seed=9)
    sur.set_scaling(np.zeros(K), np.full(K, 4.0), 2.0)
    for pH in (6.6, 7.5):
        systems = []
        for k in range(8):
            s, p = _ideal(40 + k)
            p.pH, p.pKa, p.seed = pH, 7.0, 900 + k
            systems.append((s, p))
        ns = systems[0][0].meta["n_sites"]
        with Engine([a for a, _ in systems], [b for _, b in systems]) as e:
            e.attach_surrogate(sur, threshold=0.0, window=0)
            e.run(4000)
            samples = []
            for _ in range(60):
                samples += [r["n_charged_sites"] / ns for r in e.run(400)]
            da = e.da_stats()
        expect = 1.0 / (1.0 + 10 ** (pH - 7.0))
        assert sum(d["evaluated"] for d in da) > 0
        assert all(d["fallback"] == 0 for d in da)
        # the random network rejects part of the moves in stage one
        assert sum(d["passed"] for d in da) < sum(d["evaluated"] for d in da)
        assert abs(np.mean(samples) - expect) < 0.015, (pH, np.mean(samples), expect)


@pytest.mark.gpu
def test_fallback_when_agreement_is_poor():
    sur = Surrogate(seed=10)
    sur.set_scaling(np.zeros(K), np.full(K, 1.0), 30.0)  # wild estimates
    s, p = configs.config1(seed=33)
    p.p_disp, p.p_titr = 0.5, 0.5
    with Engine(s, p) as e:
        e.attach_surrogate(sur, threshold=0.9, window=50)
        e.run(40000)
        d = e.da_stats()[0]
    assert d["fallback"] == 1, d


def _titration_engines(seeds, pH=7.5):
    sys_, prm = [], []
    for k in seeds:
        s, p = configs.config1(seed=2025 + k)
        p.p_disp, p.p_titr, p.pH, p.seed = 0.5, 0.5, pH, 5000 + k
        sys_.append(s)
        prm.append(p)
    return sys_, prm


@pytest.mark.gpu
def test_trained_surrogate_gain_over_plain_method():
    """Harvest exact dE on config-1 brushes, train on the GPU, then run delayed
    acceptance: the trained first stage skips the exact dE for a large part of the
    titration trials, keeps the second-stage agreement high (an untrained network
    does not), and leaves the degree of ionisation unchanged."""
    S, P = _titration_engines(range(4))
    sur = Surrogate(seed=11)
    with Engine(S, P) as e:
        e.harvest(200000)
        e.run(120000)
        n = e.harvest_count()
        assert n > 50000
        loss = e.surrogate_fit(sur, epochs=15, batch=1024, lr=1e-3, clip=25.0)
        assert np.isfinite(loss)
        e.harvest(0)
    runs = {}
    for name, net in (("plain", None), ("trained", sur), ("untrained", Surrogate(seed=12))):
        S, P = _titration_engines(range(10, 14))
        with Engine(S, P) as e:
            if net is not None:
                e.attach_surrogate(net, threshold=0.0, window=0)
            e.run(20000)
            ns = S[0].meta["n_sites"]
            alpha = []
            for _ in range(40):
                alpha += [r["n_charged_sites"] / ns for r in e.run(2000)]
            runs[name] = (np.mean(alpha), e.da_stats())
    a_plain, a_tr = runs["plain"][0], runs["trained"][0]
    d_tr = runs["trained"][1]
    d_un = runs["untrained"][1]
    ev, ps, ac = (sum(d[k] for d in d_tr) for k in ("evaluated", "passed", "accepted"))
    evu, psu, acu = (sum(d[k] for d in d_un) for k in ("evaluated", "passed", "accepted"))
    skipped = 1.0 - ps / ev
    agree, agree_un = ac / max(ps, 1), acu / max(psu, 1)
    print(f"alpha plain {a_plain:.4f} trained-DA {a_tr:.4f}; exact dE skipped {skipped:.3f}; "
          f"agreement trained {agree:.3f} untrained {agree_un:.3f}")
    assert abs(a_plain - a_tr) < 0.03, (a_plain, a_tr)
    assert skipped > 0.2, skipped
    assert agree > agree_un, (agree, agree_un)
    assert agree > 0.5, agree
