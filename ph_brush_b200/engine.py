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

    # ---- state ----
    def state(self, replica=0):
        n = self.caps[replica]
        x, y, z, q = (np.zeros(n, np.float32) for _ in range(4))
        t, f = np.zeros(n, np.int32), np.zeros(n, np.int32)
        _abi.check(self._lib.phmc_get_state(self._h, replica, _abi.fptr(x), _abi.fptr(y), _abi.fptr(z),
                                            _abi.fptr(q), _abi.iptr(t), _abi.iptr(f)))
        return {"x": x, "y": y, "z": z, "q": q, "type": t, "flags": f}

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
