"""Python handle on the C-ABI engine (include/phmc.h).

Thin: every call goes through libphmc.so; arrays are converted to the ABI's
plain pointers.  Errors raise PhmcError with the library's message.
"""
import ctypes as C

import numpy as np

from . import _abi


class Engine:
    def __init__(self, systems, params, device=0):
        if not isinstance(systems, (list, tuple)):
            systems, params = [systems], [params]
        assert len(systems) == len(params) and len(systems) >= 1
        self.R = len(systems)
        self._keep = []
        S = (_abi.System * self.R)()
        P = (_abi.Params * self.R)()
        for r, (s, p) in enumerate(zip(systems, params)):
            S[r], k1 = s.to_struct()
            P[r], k2 = p.to_struct()
            self._keep += [k1, k2]
        self.caps = [int(s.capacity) for s in systems]
        self._h = C.c_void_p()
        self._lib = _abi.lib()
        _abi.check(self._lib.phmc_create(self.R, S, P, device, C.byref(self._h)))
        self._keep = None  # the engine copied everything it needs

    def close(self):
        if self._h:
            self._lib.phmc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- energies ----
    def energy(self):
        out = (_abi.EnergyComponents * self.R)()
        _abi.check(self._lib.phmc_energy(self._h, out))
        return [o.asdict() for o in out]

    @staticmethod
    def make_trial(changes):
        t = _abi.Trial()
        t.n_changes = len(changes)
        for k, ch in enumerate(changes):
            c = t.c[k]
            c.index, c.present = int(ch["index"]), int(ch.get("present", 1))
            c.x, c.y, c.z, c.q = float(ch["x"]), float(ch["y"]), float(ch["z"]), float(ch["q"])
            c.type = int(ch["type"])
        return t

    def delta_energy(self, trials, replica=0):
        n = len(trials)
        arr = (_abi.Trial * n)(*[self.make_trial(t) for t in trials])
        dE = np.zeros(n, np.float64)
        _abi.check(self._lib.phmc_delta_energy(self._h, replica, arr, n, _abi.dptr(dE)))
        return dE

    def delta_energy_components(self, trials, replica=0):
        n = len(trials)
        arr = (_abi.Trial * n)(*[self.make_trial(t) for t in trials])
        out = (_abi.EnergyComponents * n)()
        _abi.check(self._lib.phmc_delta_energy_components(self._h, replica, arr, n, out))
        return [o.asdict() for o in out]

    def commit(self, changes, replica=0):
        t = self.make_trial(changes)
        _abi.check(self._lib.phmc_commit(self._h, replica, C.byref(t)))

    def set_identity(self, i, type_, q, replica=0):
        _abi.check(self._lib.phmc_set_identity(self._h, replica, i, type_, q))

    # ---- Monte Carlo ----
    def run(self, n_trials):
        st = (_abi.RunStats * self.R)()
        _abi.check(self._lib.phmc_run(self._h, int(n_trials), st))
        return [{"attempted": list(s.attempted), "accepted": list(s.accepted), "flushes": s.flushes,
                 "n_titratable": s.n_titratable, "n_charged_sites": s.n_charged_sites,
                 "n_cations": s.n_cations, "n_anions": s.n_anions, "energy": s.energy,
                 "energy_drift": s.energy_drift} for s in st]

    def set_trial_log(self, capacity):
        self._log = (np.full(capacity, -1, np.int32), np.zeros(capacity, np.float64), np.zeros(capacity, np.int32))
        _abi.check(self._lib.phmc_set_trial_log(self._h, capacity, _abi.iptr(self._log[0]),
                                                _abi.dptr(self._log[1]), _abi.iptr(self._log[2])))
        return self._log

    def set_replay(self, decisions):
        if decisions is None:
            _abi.check(self._lib.phmc_set_replay(self._h, 0, C.cast(None, C.POINTER(C.c_int))))
            return
        self._replay = np.ascontiguousarray(decisions, np.int32)
        _abi.check(self._lib.phmc_set_replay(self._h, len(self._replay), _abi.iptr(self._replay)))

    def set_tuning(self, pending_max, threads):
        _abi.check(self._lib.phmc_set_tuning(self._h, int(pending_max), int(threads)))

    def checkpoint_save(self, path):
        """Everything the chains' continuation depends on, for an exact resume (not the surrogate)."""
        _abi.check(self._lib.phmc_checkpoint_save(self._h, str(path).encode()))

    def checkpoint_load(self, path):
        """Restore a checkpoint written by an engine of the same systems and parameters."""
        _abi.check(self._lib.phmc_checkpoint_load(self._h, str(path).encode()))

    def set_quorum(self, quorum):
        """MC launch quorum (0, 1]: a launch ends once that fraction of its running replicas is blocked."""
        _abi.check(self._lib.phmc_set_quorum(self._h, float(quorum)))

    def set_tile_shapes(self, zpass=-1, cand_round=-1, energy_block=-1, g_rows=-1, plane_pipe=-1):
        """z pass of the rebuild (0 Stockham, k > 0 a register split), pair-pass round width,
        full-recompute block size, G rows in flight per thread, pipelined first pass; -1 keeps
        a field."""
        _abi.check(self._lib.phmc_set_tile_shapes(self._h, int(zpass), int(cand_round), int(g_rows),
                                                  int(energy_block), int(plane_pipe)))

    def set_first_stage(self, on):
        """Delayed acceptance's first stage on (1) or bypassed (0) with the surrogate still attached."""
        _abi.check(self._lib.phmc_set_first_stage(self._h, int(on)))

    def set_launch_budget(self, max_launches):
        """Bound on the MC launches of one run / device-phase call (0: unbounded);
        a call that reaches it raises PhmcError(PHMC_ERR_BUDGET) with the state consistent."""
        _abi.check(self._lib.phmc_set_launch_budget(self._h, int(max_launches)))

    def set_zhist(self, nbins, every=1000):
        """z-density profiles: every `every` trials each replica's MC kernel adds its histogram
        (nbins bins between the walls) of charged sites, anions and cations; 0 bins: off."""
        _abi.check(self._lib.phmc_set_zhist(self._h, int(nbins), int(every)))
        self._zh_bins = int(nbins)

    def zhist(self, replica=0):
        """(counts[3, nbins] summed over samples: sites, anions, cations; number of samples)."""
        nb = self._zh_bins
        c = np.zeros(3 * nb, np.float64)
        n = C.c_int64()
        _abi.check(self._lib.phmc_get_zhist(self._h, int(replica), _abi.dptr(c), C.byref(n)))
        return c.reshape(3, nb), n.value

    def tuning(self):
        t = _abi.Tuning()
        _abi.check(self._lib.phmc_get_tuning(self._h, C.byref(t)))
        return t.asdict()

    def autotune(self, trials):
        """Every candidate timed (z pass: rebuild_us; full-recompute block: recompute_us; pending
        capacity x threads and pair-pass round width: us_per_trial); the engine keeps the best."""
        res = (_abi.Tuning * 64)()
        n = C.c_int()
        _abi.check(self._lib.phmc_autotune(self._h, int(trials), res, 64, C.byref(n)))
        return [res[k].asdict() for k in range(min(n.value, 64))]

    def set_move_mix(self, p_disp, p_titr, p_swap=0.0, replica=-1):
        _abi.check(self._lib.phmc_set_move_mix(self._h, int(replica), float(p_disp), float(p_titr), float(p_swap)))

    # ---- state ----
    def state(self, replica=0, out=None):
        """Slot arrays of one replica, or of all replicas concatenated (replica=-1).  `out`: a dict
        of preallocated arrays (x, y, z, q float32; type, flags int32; e.g. in pinned memory) to
        fill instead of new ones."""
        n = sum(self.caps) if replica < 0 else self.caps[replica]
        if out is not None:
            x, y, z, q, t, f = (out[k] for k in ("x", "y", "z", "q", "type", "flags"))
            for a, dt in ((x, np.float32), (y, np.float32), (z, np.float32), (q, np.float32), (t, np.int32), (f, np.int32)):
                if a.dtype != dt or a.shape != (n,) or not a.flags.c_contiguous:
                    raise ValueError(f"state(out=...): arrays must be contiguous {n}-element float32 / int32")
        else:
            x, y, z, q = (np.zeros(n, np.float32) for _ in range(4))
            t, f = np.zeros(n, np.int32), np.zeros(n, np.int32)
        _abi.check(self._lib.phmc_get_state(self._h, replica, _abi.fptr(x), _abi.fptr(y), _abi.fptr(z),
                                            _abi.fptr(q), _abi.iptr(t), _abi.iptr(f)))
        return {"x": x, "y": y, "z": z, "q": q, "type": t, "flags": f}

    def set_event_callback(self, fn):
        """fn(job, phase, record_address) after each launch of a device phase for every new
        event record (phase 1: phmc_gc_event, 2: phmc_phase2_event); None switches it off."""
        if fn is None:
            self._ev_cb = None
            _abi.check(self._lib.phmc_set_event_callback(self._h, _abi.EventFn(), None))
            return
        self._ev_cb = _abi.EventFn(lambda user, job, phase, rec: fn(job, phase, rec))
        _abi.check(self._lib.phmc_set_event_callback(self._h, self._ev_cb, None))

    def gc_phase(self, jobs, event_cap=1 << 14):
        """The reference's grand-canonical mu-control phase (MC/src/mc.cu:320-548) on the
        device, one job per replica.  Each job is a dict with the keys of phmc_gc_job:
        replica, nh_n_type, nh_p_type, w_type, cl_type (engine types), q_nh_p, q_cl, beta,
        target_pct, optional mu_eta, nacc_frac, gc_block, epoch_attempt_max, max_trials,
        fixed_mu and mu_kT (mu held at mu_kT / beta: no feedback, no target stop),
        the pools nh_n, nh_p, w, cl (slot indices in the reference's order) and mt_state
        (uint32[625], updated in place).  Returns [(result dict, [event dicts])]."""
        n = len(jobs)
        J = (_abi.GcJob * n)()
        keep = []
        for k, j in enumerate(jobs):
            st = j["mt_state"]
            assert isinstance(st, np.ndarray) and st.dtype == np.uint32 and st.shape == (625,) and st.flags.c_contiguous
            J[k].replica = j.get("replica", k)
            for key in ("nh_n_type", "nh_p_type", "w_type", "cl_type"):
                setattr(J[k], key, int(j[key]))
            J[k].q_nh_p = j.get("q_nh_p", 1.0)
            J[k].q_cl = j.get("q_cl", -1.0)
            J[k].beta = j["beta"]
            J[k].target_pct = j["target_pct"]
            J[k].mu_eta = j.get("mu_eta", 0.0)
            J[k].nacc_frac = j.get("nacc_frac", 0.0)
            J[k].gc_block = j.get("gc_block", 0)
            J[k].epoch_attempt_max = j.get("epoch_attempt_max", 0)
            J[k].max_trials = j.get("max_trials", 0)
            J[k].fixed_mu = 1 if j.get("fixed_mu") else 0
            J[k].mu_kT = j.get("mu_kT", 0.0)
            for key in ("nh_n", "nh_p", "w", "cl"):
                a = _abi.as_i32(j[key])
                keep.append(a)
                setattr(J[k], key, _abi.iptr(a))
                setattr(J[k], "n_" + key, len(a))
            J[k].mt_state = st.ctypes.data_as(C.POINTER(C.c_uint32))
        R = (_abi.GcResult * n)()
        E = (_abi.GcEvent * (n * event_cap))()
        _abi.check(self._lib.phmc_gc_phase(self._h, n, J, R, E, event_cap))
        return [(R[k].asdict(), [E[k * event_cap + i].asdict() for i in range(R[k].n_events)]) for k in range(n)]

    def phase2(self, jobs, event_cap=1 << 14):
        """The reference's phase 2, swaps with patience (MC/src/mc.cu:159-318), on the device,
        one job per replica.  Each job is a dict with the keys of phmc_phase2_job: replica,
        nh_n_type, nh_p_type, w_type, cl_type, q_nh_p, q_cl, beta, max_attempts, patience,
        energy_interval, z_cut, the pools nh_p, nh_n, w, cl (W and Cl below z_cut, the
        reference's order) and mt_state (uint32[625], updated in place).
        Returns [(result dict, [event dicts])]."""
        n = len(jobs)
        J = (_abi.Phase2Job * n)()
        keep = []
        for k, j in enumerate(jobs):
            st = j["mt_state"]
            assert isinstance(st, np.ndarray) and st.dtype == np.uint32 and st.shape == (625,) and st.flags.c_contiguous
            J[k].replica = j.get("replica", k)
            for key in ("nh_n_type", "nh_p_type", "w_type", "cl_type", "max_attempts", "patience", "energy_interval"):
                setattr(J[k], key, int(j[key]))
            J[k].q_nh_p = j.get("q_nh_p", 1.0)
            J[k].q_cl = j.get("q_cl", -1.0)
            J[k].beta = j["beta"]
            J[k].z_cut = j.get("z_cut", 0.0)
            for key in ("nh_p", "nh_n", "w", "cl"):
                a = _abi.as_i32(j[key])
                keep.append(a)
                setattr(J[k], key, _abi.iptr(a))
                setattr(J[k], "n_" + key, len(a))
            J[k].mt_state = st.ctypes.data_as(C.POINTER(C.c_uint32))
        R = (_abi.Phase2Result * n)()
        E = (_abi.Phase2Event * (n * event_cap))()
        _abi.check(self._lib.phmc_phase2(self._h, n, J, R, E, event_cap))
        return [(R[k].asdict(), [E[k * event_cap + i].asdict() for i in range(R[k].n_events)]) for k in range(n)]

    def set_state(self, st, replica=0):
        a = [_abi.as_f32(st[k]) for k in ("x", "y", "z", "q")] + [_abi.as_i32(st["type"]), _abi.as_i32(st["flags"])]
        _abi.check(self._lib.phmc_set_state(self._h, replica, *(_abi.fptr(v) for v in a[:4]), _abi.iptr(a[4]),
                                            _abi.iptr(a[5])))

    # ---- measurement ----
    def set_profiling(self, on=True):
        _abi.check(self._lib.phmc_set_profiling(self._h, int(on)))

    def profile(self, reset=False):
        p = _abi.Profile()
        _abi.check(self._lib.phmc_get_profile(self._h, C.byref(p), int(reset)))
        return p.asdict()

    def set_phase_clock(self, on=True):
        """Per-phase SM cycle counters of the MC kernel (phmc_set_phase_clock)."""
        _abi.check(self._lib.phmc_set_phase_clock(self._h, int(on)))

    def phase_cycles(self, reset=False):
        """{phase name: SM cycles summed over replicas, "trials": trials run}."""
        c = (C.c_int64 * 8)()
        t = C.c_int64()
        _abi.check(self._lib.phmc_get_phase_cycles(self._h, c, C.byref(t), int(reset)))
        out = {k: int(v) for k, v in zip(_abi.PHASES, c)}
        out["trials"] = int(t.value)
        return out

    def run_timed(self, n_trials):
        ms = C.c_double()
        _abi.check(self._lib.phmc_run_timed(self._h, int(n_trials), C.byref(ms)))
        return ms.value

    def flush_l2(self, nbytes=256 << 20):
        _abi.check(self._lib.phmc_flush_l2(self._h, int(nbytes)))

    def cells(self, replica=0):
        n = self.caps[replica]
        c = np.zeros(n, np.int32)
        dims = np.zeros(3, np.int32)
        _abi.check(self._lib.phmc_get_cells(self._h, replica, _abi.iptr(c), _abi.iptr(dims)))
        return c, tuple(int(v) for v in dims)

    # ---- learned surrogate / delayed acceptance ----
    def harvest(self, capacity):
        _abi.check(self._lib.phmc_harvest(self._h, int(capacity)))

    def harvest_count(self):
        n = C.c_int()
        _abi.check(self._lib.phmc_harvest_count(self._h, C.byref(n)))
        return n.value

    def harvest_get(self, n=None):
        n = self.harvest_count() if n is None else int(n)
        x = np.zeros((n, _abi.SUR_ROWS, _abi.SUR_INPUTS), np.float32)
        sg = np.zeros((n, _abi.SUR_ROWS), np.float32)
        t = np.zeros(n, np.float32)
        _abi.check(self._lib.phmc_harvest_get(self._h, n, _abi.fptr(x), _abi.fptr(sg), _abi.fptr(t)))
        return x, sg, t

    def surrogate_fit(self, sur, epochs=10, batch=4096, lr=1e-3, clip=25.0, seed=1):
        loss = C.c_double()
        _abi.check(self._lib.phmc_surrogate_fit(self._h, sur._h, int(epochs), int(batch), float(lr), float(clip),
                                                int(seed), C.byref(loss)))
        return loss.value

    def attach_surrogate(self, sur, threshold=0.0, window=0):
        _abi.check(self._lib.phmc_surrogate_attach(self._h, sur._h if sur is not None else None,
                                                   float(threshold), int(window)))
        self._sur = sur  # keep the network alive while attached

    def da_stats(self):
        out = (_abi.DAStats * self.R)()
        _abi.check(self._lib.phmc_get_da_stats(self._h, out))
        return [o.asdict() for o in out]

    def describe(self, trials, replica=0):
        n = len(trials)
        arr = (_abi.Trial * n)(*[self.make_trial(t) for t in trials])
        out = np.zeros((n, _abi.SUR_DESC_STRIDE), np.float32)
        dEs = np.zeros(n, np.float64)
        _abi.check(self._lib.phmc_surrogate_describe(self._h, replica, arr, n, _abi.fptr(out), _abi.dptr(dEs)))
        R, K = _abi.SUR_ROWS, _abi.SUR_INPUTS
        res = []
        for k in range(n):
            o = out[k]
            res.append({"rows": o[:R * K].reshape(R, K).copy(), "sign": o[R * K:R * K + R].copy(),
                        "F": o[R * K + R:R * K + 2 * R].copy(), "cross": float(o[R * K + 2 * R]),
                        "mom": float(o[R * K + 2 * R + 1]), "nrows": int(o[R * K + 2 * R + 2]),
                        "inner": int(o[R * K + 2 * R + 3]), "dEs": float(dEs[k])})
        return res

    def set_da_log(self):
        cap = len(self._log[0])
        self._da_log = (np.full(cap, -1, np.int32), np.zeros(cap, np.float64))
        _abi.check(self._lib.phmc_set_da_log(self._h, _abi.iptr(self._da_log[0]), _abi.dptr(self._da_log[1])))
        return self._da_log


class Surrogate:
    """The MLP surrogate (include/phmc.h, phmc_surrogate_*): GPU training and inference."""

    def __init__(self, n_in=_abi.SUR_INPUTS, hidden=128, seed=0, _handle=None):
        self._lib = _abi.lib()
        self._h = C.c_void_p()
        if _handle is not None:
            self._h = _handle
        else:
            _abi.check(self._lib.phmc_surrogate_create(int(n_in), int(hidden), int(seed), C.byref(self._h)))
        self.n_params = self._lib.phmc_surrogate_num_params(self._h)

    @classmethod
    def load(cls, path):
        lib = _abi.lib()
        h = C.c_void_p()
        _abi.check(lib.phmc_surrogate_load(str(path).encode(), C.byref(h)))
        return cls(_handle=h)

    def save(self, path):
        _abi.check(self._lib.phmc_surrogate_save(self._h, str(path).encode()))

    def close(self):
        if self._h:
            self._lib.phmc_surrogate_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.n_params, np.float32)
        _abi.check(self._lib.phmc_surrogate_get_params(self._h, _abi.fptr(p), self.n_params))
        return p

    def set_params(self, p):
        p = _abi.as_f32(p)
        _abi.check(self._lib.phmc_surrogate_set_params(self._h, _abi.fptr(p), len(p)))

    def set_scaling(self, mu, sd, scale):
        mu, sd = _abi.as_f32(mu), _abi.as_f32(sd)
        _abi.check(self._lib.phmc_surrogate_set_scaling(self._h, _abi.fptr(mu), _abi.fptr(sd), float(scale)))

    def scaling(self, n_in=_abi.SUR_INPUTS):
        mu, sd = np.zeros(n_in, np.float32), np.zeros(n_in, np.float32)
        sc = C.c_float()
        _abi.check(self._lib.phmc_surrogate_get_scaling(self._h, _abi.fptr(mu), _abi.fptr(sd), C.byref(sc)))
        return mu, sd, sc.value

    def predict(self, x):
        x = _abi.as_f32(x)
        n = x.shape[0]
        y = np.zeros(n, np.float32)
        _abi.check(self._lib.phmc_surrogate_predict(self._h, _abi.fptr(x), n, _abi.fptr(y)))
        return y

    def gradient(self, x, sign, t, clip=25.0):
        x, sign, t = _abi.as_f32(x), _abi.as_f32(sign), _abi.as_f32(t)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double()
        _abi.check(self._lib.phmc_surrogate_gradient(self._h, _abi.fptr(x), _abi.fptr(sign), _abi.fptr(t), len(t),
                                                     float(clip), C.byref(loss), _abi.fptr(g)))
        return loss.value, g

    def train(self, x, sign, t, epochs=1, batch=256, lr=1e-3, clip=25.0, seed=1, rescale=True):
        x, sign, t = _abi.as_f32(x), _abi.as_f32(sign), _abi.as_f32(t)
        loss = C.c_double()
        _abi.check(self._lib.phmc_surrogate_train(self._h, _abi.fptr(x), _abi.fptr(sign), _abi.fptr(t), len(t),
                                                  int(epochs), int(batch), float(lr), float(clip), int(seed),
                                                  int(bool(rescale)), C.byref(loss)))
        return loss.value
