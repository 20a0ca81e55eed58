"""ORACLE — test infrastructure only (ctypes wrapper over oracle/_build/libphoracle.so).

Imported by tests/, the smoke check and bench.py's CPU-baseline leg only.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

from ph_brush_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libphoracle.so")
REF_HOST = os.path.join(HERE, "_ref", "libref_host.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)


def build():
    subprocess.run(["make", "-s", "-C", HERE, "lib"], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    sigs = {
        "orc_ref_good_fft_dim": ([C.c_int], C.c_int),
        "orc_ref_ewald_alpha": ([C.c_double, C.c_double], C.c_double),
        "orc_ref_alpha_bisect": ([C.c_double, C.c_double], C.c_double),
        "orc_moduli": ([C.c_int, C.c_int, C.c_int, _dp], None),
        "orc_bspline_weights": ([C.c_int, C.c_double, _dp], None),
        "orc_ref_bond_csr": ([C.c_int, C.c_int, _ip, _ip, _ip, _ip], None),
        "orc_ref_half_list": ([C.c_int, _dp, _dp, _dp, _dp, C.c_double, _ip, _ip, _ip, _ip, C.c_int], C.c_int),
        "orc_ref_lj_shift": ([C.c_int, _dp, _dp, C.c_double, _dp], None),
        "orc_ref_lj": ([C.c_int, _dp, _dp, _dp, _ip, _ip, _ip, C.c_int, _dp, _dp, _dp, _dp, C.c_int], C.c_double),
        "orc_ref_coul_cut": ([C.c_int, _dp, _dp, _dp, _dp, _ip, _ip, _dp, C.c_double], C.c_double),
        "orc_ref_pme": ([C.c_int, _dp, _dp, _dp, _dp, _ip, _ip, _dp, C.c_double, C.c_double, C.c_int, C.c_int,
                         C.c_int, C.c_int, C.c_int, _dp], C.c_double),
        "orc_direct_ewald": ([C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, _dp], None),
        "orc_energy": ([C.POINTER(_abi.System), C.POINTER(_abi.Params), C.POINTER(_abi.EnergyComponents)], C.c_int),
        "orc_philox": ([_u32p, _u32p, _u32p], None),
        "orc_mc_create": ([C.POINTER(_abi.System), C.POINTER(_abi.Params)], C.c_void_p),
        "orc_mc_destroy": ([C.c_void_p], None),
        "orc_mc_step": ([C.c_void_p, C.c_int, _ip, _dp, _ip], C.c_int),
        "orc_mc_energy": ([C.c_void_p], C.c_double),
        "orc_mc_get_state": ([C.c_void_p, _fp, _fp, _fp, _fp, _ip, _ip], None),
        "orc_mc_counts": ([C.c_void_p, _ip, _ip, _ip], None),
        "orc_cells": ([C.c_void_p, C.c_int, C.c_int, C.c_int, _ip], None),
        "orc_fft3d": ([_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int], None),
        "orc_mt_create": ([C.c_uint32], C.c_void_p),
        "orc_mt_destroy": ([C.c_void_p], None),
        "orc_mt_index": ([C.c_void_p, C.c_int], C.c_int),
        "orc_mt_unit_float": ([C.c_void_p], C.c_float),
        "orc_mt_state": ([C.c_void_p, _u32p], None),
    }
    for k, (a, r) in sigs.items():
        f = getattr(lib, k)
        f.argtypes = a
        f.restype = r
    return lib


L = _load()


def d(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(_dp)


def i32(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(_ip)


def energy(sysa, prm):
    s, k1 = sysa.to_struct()
    p, k2 = prm.to_struct()
    out = _abi.EnergyComponents()
    L.orc_energy(C.byref(s), C.byref(p), C.byref(out))
    return out.asdict()


def moduli(n, order, ref_style):
    out = np.zeros(n)
    L.orc_moduli(n, order, ref_style, out.ctypes.data_as(_dp))
    return out


def bspline_weights(p, t):
    out = np.zeros(p)
    L.orc_bspline_weights(p, t, out.ctypes.data_as(_dp))
    return out


def bond_csr(n, bi, bj):
    head = np.zeros(n + 1, np.int32)
    lst = np.zeros(2 * len(bi) + 1, np.int32)
    a, pa = i32(bi)
    b, pb = i32(bj)
    L.orc_ref_bond_csr(n, len(bi), pa, pb, head.ctypes.data_as(_ip), lst.ctypes.data_as(_ip))
    return head, lst[:head[-1]]


def half_list(x, y, z, box, rc, bhead=None, blist=None):
    n = len(x)
    xs, px = d(x); ys, py = d(y); zs, pz = d(z); bs, pb = d(box)
    head = np.zeros(n + 1, np.int32)
    if bhead is not None:
        bh, pbh = i32(bhead); bl, pbl = i32(blist if len(blist) else np.zeros(1, np.int32))
    else:
        pbh = pbl = C.cast(None, _ip)
    nnz = L.orc_ref_half_list(n, px, py, pz, pb, rc, pbh, pbl, head.ctypes.data_as(_ip), C.cast(None, _ip), 0)
    lst = np.zeros(max(nnz, 1), np.int32)
    L.orc_ref_half_list(n, px, py, pz, pb, rc, pbh, pbl, head.ctypes.data_as(_ip), lst.ctypes.data_as(_ip), nnz)
    return head, lst[:nnz]


def ref_energies(sysa, prm, spacing=None):
    """Reference-semantics energies (MC/src/energy_gpu.cu + MC/src/pme.cu) for a
    system in reference types: returns dict(lj, real, recip, self, qcorr_slab, coul_total, nnz)."""
    x, y, z, q = (np.asarray(getattr(sysa, k), np.float64) for k in "xyzq")
    box = np.asarray(sysa.box, np.float64)
    bh, bl = bond_csr(sysa.n, sysa.bond_i, sysa.bond_j)
    head, lst = half_list(x, y, z, box, prm.rc_coul, bh, bl)
    T = prm.n_types
    eps = np.ascontiguousarray(prm.lj_eps, np.float64).ravel()
    sig = np.ascontiguousarray(prm.lj_sig, np.float64).ravel()
    sh = np.zeros(T * T)
    L.orc_ref_lj_shift(T, eps.ctypes.data_as(_dp), sig.ctypes.data_as(_dp), prm.rc_lj, sh.ctypes.data_as(_dp))
    xs, px = d(x); ys, py = d(y); zs, pz = d(z); qs, pq = d(q); bs, pb = d(box)
    ts, pt = i32(sysa.type)
    hs, ph = i32(head); ls, pl = i32(lst if len(lst) else np.zeros(1, np.int32))
    elj = L.orc_ref_lj(sysa.n, px, py, pz, pt, ph, pl, T, pb, eps.ctypes.data_as(_dp), sig.ctypes.data_as(_dp),
                       sh.ctypes.data_as(_dp), prm.lj_shift)
    out = np.zeros(4)
    ec = L.orc_ref_pme(sysa.n, px, py, pz, pq, ph, pl, pb, prm.ewald_alpha, prm.epsilon_r, prm.mesh[0], prm.mesh[1],
                       prm.mesh[2], prm.order, prm.slab, out.ctypes.data_as(_dp))
    return {"lj": elj, "real": out[0], "recip": out[1], "self": out[2], "qcorr_slab": out[3], "coul_total": ec,
            "nnz": len(lst)}


def direct_ewald(x, y, z, q, box, alpha, epsilon_r, slab, tol=1e-12):
    xs, px = d(x); ys, py = d(y); zs, pz = d(z); qs, pq = d(q); bs, pb = d(box)
    out = np.zeros(6)
    L.orc_direct_ewald(len(x), px, py, pz, pq, pb, alpha, epsilon_r, slab, tol, out.ctypes.data_as(_dp))
    return dict(zip(["real", "recip", "self", "qcorr", "slab", "total"], out))


class RefTrialLoop:
    """The reference's per-trial loop restated in FP64 on the host cores (the CPU
    baseline): its total energy recomputed for every trial (MC/src/mc.cu:43-60) -- LJ
    over the half list built once at set-up (MC/src/main.cu:127,
    MC/src/energy_gpu.cu:14-75) plus SPME with its cubic spreading, moduli and
    influence function (MC/src/pme.cu:132-457), OpenMP-parallel in the oracle library
    -- in the benchmark's move mix: displacements of mobile atoms within the slab
    (the reference has none; the half list is not rebuilt, as in the reference
    harness) and the reference's grand-canonical pair flips (MC/src/mc.cu:379-440)
    with mu held at kT ln10 (pKa - pH).  Works on a system in the reference's model
    (reference types, as ph_brush_b200.files.reference_model returns it)."""

    def __init__(self, sysa, prm, mobile, height, pH, pKa, seed=1, disp_max=0.3, nh=(3, 4), w_cl=(6, 7)):
        self.s, self.p = sysa, prm
        self.x, self.y, self.z, self.q = (np.array(getattr(sysa, k), np.float64) for k in "xyzq")
        self.t = np.ascontiguousarray(sysa.type, np.int32)
        self.box = np.asarray(sysa.box, np.float64)
        bh, bl = bond_csr(sysa.n, sysa.bond_i, sysa.bond_j)
        self.head, self.lst = half_list(self.x, self.y, self.z, self.box, prm.rc_coul, bh, bl)
        if not len(self.lst):
            self.lst = np.zeros(1, np.int32)
        T = prm.n_types
        self.eps = np.ascontiguousarray(prm.lj_eps, np.float64).ravel()
        self.sig = np.ascontiguousarray(prm.lj_sig, np.float64).ravel()
        self.sh = np.zeros(T * T)
        L.orc_ref_lj_shift(T, self.eps.ctypes.data_as(_dp), self.sig.ctypes.data_as(_dp), prm.rc_lj,
                           self.sh.ctypes.data_as(_dp))
        self.mobile = np.asarray(mobile, np.int64)
        self.height, self.dmax = float(height), float(disp_max)
        self.mu = math.log(10.0) * (pKa - pH)  # kT units, beta = 1
        self.nhn, self.nhp = nh
        self.wt, self.clt = w_cl
        self.rng = np.random.default_rng(seed)
        self.E = self.energy()

    def energy(self):
        s, p = self.s, self.p
        pl = lambda a: a.ctypes.data_as(_dp)
        elj = L.orc_ref_lj(s.n, pl(self.x), pl(self.y), pl(self.z), self.t.ctypes.data_as(_ip),
                           self.head.ctypes.data_as(_ip), self.lst.ctypes.data_as(_ip), p.n_types, pl(self.box),
                           pl(self.eps), pl(self.sig), pl(self.sh), p.lj_shift)
        out = np.zeros(4)
        ec = L.orc_ref_pme(s.n, pl(self.x), pl(self.y), pl(self.z), pl(self.q), self.head.ctypes.data_as(_ip),
                           self.lst.ctypes.data_as(_ip), pl(self.box), p.ewald_alpha, p.epsilon_r, p.mesh[0], p.mesh[1],
                           p.mesh[2], p.order, p.slab, pl(out))
        return elj + ec

    def trial(self, p_disp=0.9):
        r = self.rng
        if r.random() < p_disp:
            i = int(self.mobile[r.integers(len(self.mobile))])
            old = (self.x[i], self.y[i], self.z[i])
            nz = old[2] + self.dmax * (2 * r.random() - 1)
            nx = (old[0] + self.dmax * (2 * r.random() - 1)) % self.box[0]
            ny = (old[1] + self.dmax * (2 * r.random() - 1)) % self.box[1]
            if not 0.0 <= nz < self.height:
                return
            self.x[i], self.y[i], self.z[i] = nx, ny, nz
            Et = self.energy()
            if Et - self.E <= 0 or math.exp(max(-40.0, -(Et - self.E))) > r.random():
                self.E = Et
            else:
                self.x[i], self.y[i], self.z[i] = old
            return
        pools = [np.flatnonzero(self.t == k) for k in (self.nhn, self.nhp, self.wt, self.clt)]
        a, b, c, d = (len(v) for v in pools)
        wf, wb = a * c, b * d
        if wf + wb == 0:
            return
        fwd = r.random() < wf / (wf + wb)
        i = int(pools[0 if fwd else 1][r.integers(a if fwd else b)])
        j = int(pools[2 if fwd else 3][r.integers(c if fwd else d)])
        old = (self.t[i], self.q[i], self.t[j], self.q[j])
        self.t[i], self.q[i] = (self.nhp, 1.0) if fwd else (self.nhn, 0.0)
        self.t[j], self.q[j] = (self.clt, -1.0) if fwd else (self.wt, 0.0)
        Et = self.energy()
        s_after = (a - 1) * (c - 1) + (b + 1) * (d + 1) if fwd else (a + 1) * (c + 1) + (b - 1) * (d - 1)
        logH = math.log(wf + wb) - math.log(s_after) if s_after > 0 else 0.0
        expo = min(40.0, max(-40.0, -(Et - self.E - (1 if fwd else -1) * self.mu) + logH))
        if expo >= 0 or math.exp(expo) > r.random():
            self.E = Et
        else:
            self.t[i], self.q[i], self.t[j], self.q[j] = old


def philox(key, ctr):
    k = np.ascontiguousarray(key, np.uint32)
    c = np.ascontiguousarray(ctr, np.uint32)
    o = np.zeros(4, np.uint32)
    L.orc_philox(k.ctypes.data_as(_u32p), c.ctypes.data_as(_u32p), o.ctypes.data_as(_u32p))
    return o


class MC:
    """CPU Monte Carlo with the engine's move set (energies from scratch)."""

    def __init__(self, sysa, prm):
        s, self._k1 = sysa.to_struct()
        p, self._k2 = prm.to_struct()
        self.cap = sysa.capacity
        self.h = L.orc_mc_create(C.byref(s), C.byref(p))

    def step(self, forced=-1):
        mv, dE, acc = C.c_int(), C.c_double(), C.c_int()
        L.orc_mc_step(self.h, forced, C.byref(mv), C.byref(dE), C.byref(acc))
        return mv.value, dE.value, acc.value

    @property
    def energy(self):
        return L.orc_mc_energy(self.h)

    def state(self):
        n = self.cap
        x, y, z, q = (np.zeros(n, np.float32) for _ in range(4))
        t, f = np.zeros(n, np.int32), np.zeros(n, np.int32)
        L.orc_mc_get_state(self.h, *(a.ctypes.data_as(_fp) for a in (x, y, z, q)), t.ctypes.data_as(_ip),
                           f.ctypes.data_as(_ip))
        return {"x": x, "y": y, "z": z, "q": q, "type": t, "flags": f}

    def counts(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        L.orc_mc_counts(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def cells(self, dims):
        out = np.zeros(self.cap, np.int32)
        L.orc_cells(self.h, dims[0], dims[1], dims[2], out.ctypes.data_as(_ip))
        return out

    def close(self):
        if self.h:
            L.orc_mc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def ref_host_read(data_path, params_path, cap=200000):
    """Read a data file and params.in with the reference's own host code
    (MC/src/io.cpp via oracle/_ref/libref_host.so).  Returns (SystemArrays in
    0-based reference types with the slab-padded box, ModelParams in reference
    semantics, raw dict of the reference's Params)."""
    from ph_brush_b200 import _abi as A
    from ph_brush_b200.model import ModelParams, SystemArrays
    lib = C.CDLL(REF_HOST)
    counts = np.zeros(3, np.int32)
    box = np.zeros(3)
    idv, mol, typ = (np.zeros(cap, np.int32) for _ in range(3))
    q, x, y, z = (np.zeros(cap) for _ in range(4))
    head, lst = np.zeros(cap + 1, np.int32), np.zeros(4 * cap, np.int32)
    err = C.create_string_buffer(256)
    rc = lib.refh_read_data(data_path.encode(), counts.ctypes.data_as(_ip), box.ctypes.data_as(_dp),
                            idv.ctypes.data_as(_ip), mol.ctypes.data_as(_ip), typ.ctypes.data_as(_ip),
                            q.ctypes.data_as(_dp), x.ctypes.data_as(_dp), y.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                            head.ctypes.data_as(_ip), lst.ctypes.data_as(_ip), cap, err, 256)
    if rc:
        raise RuntimeError(err.value.decode())
    n, nb, T = (int(v) for v in counts)
    dd = np.zeros(11)
    ii = np.zeros(16, np.int32)
    eps, sig, sh = np.zeros(T * T), np.zeros(T * T), np.zeros(T * T)
    rc = lib.refh_read_params(params_path.encode(), T, dd.ctypes.data_as(_dp), ii.ctypes.data_as(_ip),
                              eps.ctypes.data_as(_dp), sig.ctypes.data_as(_dp), sh.ctypes.data_as(_dp), err, 256)
    if rc:
        raise RuntimeError(err.value.decode())
    raw = {"rc": dd[0], "ewald_alpha": dd[1], "epsilon_r": dd[2], "pme_spacing": dd[3], "pme_3dc_zfac": dd[4],
           "beta": dd[5], "lj_shift": int(ii[0]), "coulombtype": int(ii[1]), "pme_order": int(ii[2]),
           "pme_3dc": int(ii[3]), "lj_eps": eps.reshape(T, T), "lj_sig": sig.reshape(T, T), "lj_shift_tbl": sh.reshape(T, T),
           "target_pct": dd[7], "w_z_extra_nm": dd[8], "mu_eta": dd[9], "sgmc_nacc_frac_round": dd[10],
           "NH_N_type": int(ii[4]), "NH_P_type": int(ii[5]), "W_type": int(ii[6]), "Cl_type": int(ii[7]),
           "rng_seed": int(ii[8]), "energy_interval": int(ii[9]), "patience": int(ii[10]), "max_attempts": int(ii[11]),
           "direct_pct_threshold": int(ii[12]), "gc_block_fixed": int(ii[13]), "sgmc_epoch_attempt_max": int(ii[14]),
           "phase2_wc": int(ii[15])}
    bx = box.copy()
    if raw["pme_3dc"]:
        bx[2] *= max(2.0, raw["pme_3dc_zfac"])
    bi = [i for i in range(n) for j in lst[head[i]:head[i + 1]] if j > i]
    bj = [j for i in range(n) for j in lst[head[i]:head[i + 1]] if j > i]
    s = SystemArrays(x[:n].astype(np.float32), y[:n].astype(np.float32), z[:n].astype(np.float32),
                     q[:n].astype(np.float32), (typ[:n] - 1).astype(np.int32), np.zeros(n, np.int32),
                     np.array(bi, np.int32), np.array(bj, np.int32), bx, capacity=n)
    mesh = tuple(max(L.orc_ref_good_fft_dim(int(np.ceil(bx[k] / raw["pme_spacing"]))), raw["pme_order"]) for k in range(3))
    p = ModelParams(n_types=T, lj_eps=raw["lj_eps"], lj_sig=raw["lj_sig"], lj_rc=None, rc_lj=raw["rc"],
                    lj_shift=raw["lj_shift"], coulomb=A.COUL_EWALD if raw["coulombtype"] == 1 else A.COUL_CUT,
                    rc_coul=raw["rc"], epsilon_r=raw["epsilon_r"], ewald_alpha=raw["ewald_alpha"] or 1.0, mesh=mesh,
                    order=raw["pme_order"], ref_moduli=1, slab=raw["pme_3dc"], excl_bonded_lj=1, excl_bonded_coul=1,
                    beta=raw["beta"], p_disp=0.0, p_titr=0.0)
    return s, p, raw


# ---------------------------------------------------------------------------
# The reference's move phases (MC/src/mc.cu:67-122 build_plan, :159-318 phase 2,
# :320-548 grand-canonical mu control), restated on the oracle's FP64
# reference-model energies rounded as the reference's float build rounds them,
# drawing from libstdc++'s std::mt19937 itself (orc_mt_*).  Events are dicts with
# the fields of phmc_gc_event / phmc_phase2_event, filled as the device fills them.
# ---------------------------------------------------------------------------
_f32 = np.float32
_LIBM = C.CDLL("libm.so.6")
_LIBM.logf.restype = C.c_float
_LIBM.logf.argtypes = [C.c_float]
_LIBM.expf.restype = C.c_float
_LIBM.expf.argtypes = [C.c_float]


def _clampf(x, lo, hi):
    return lo if x < lo else (hi if x > hi else x)


class RefGenerator:
    """std::mt19937(seed) with the reference's two draws (libstdc++ via the oracle library)."""

    def __init__(self, seed):
        self.h = L.orc_mt_create(seed & 0xFFFFFFFF)

    def index(self, n):
        return L.orc_mt_index(self.h, n)

    def unit(self):
        return _f32(L.orc_mt_unit_float(self.h))

    def state(self):
        out = np.zeros(625, np.uint32)
        L.orc_mt_state(self.h, out.ctypes.data_as(_u32p))
        return out

    def __del__(self):
        try:
            L.orc_mt_destroy(self.h)
        except Exception:
            pass


def ref_total_real(s, p):
    """total_energy as the reference's float build returns it: the LJ part and the
    Coulomb part each rounded to float, then added (MC/src/mc.cu:43-60)."""
    e = ref_energies(s, p)
    return _f32(_f32(e["lj"]) + _f32(e["coul_total"]))


def ref_plan(s, raw):
    """build_plan (MC/src/mc.cu:67-122): pools by type, z_cut, to_flip, and the reference's checks."""
    t = s.type + 1
    z = np.asarray(s.z, np.float32)
    nh_n = [i for i in range(s.n) if t[i] == raw["NH_N_type"]]
    nh_p = [i for i in range(s.n) if t[i] == raw["NH_P_type"]]
    w_all = [i for i in range(s.n) if t[i] == raw["W_type"]]
    nh_total = len(nh_n) + len(nh_p)
    if nh_total == 0:
        raise RuntimeError("[plan] No NH sites found.")
    target = int(np.floor(float(_f32(raw["target_pct"])) / 100.0 * nh_total))
    to_flip = target - len(nh_p)
    if to_flip < 0:
        raise RuntimeError("[plan] Target < current; de-protonation not supported.")
    if len(nh_n) < to_flip:
        raise RuntimeError("[plan] Not enough NH_N to flip.")
    z_max = _f32(0.0)
    for i in nh_n + nh_p:
        z_max = max(z_max, z[i])
    z_cut = _f32(z_max + _f32(raw["w_z_extra_nm"]))
    w = [j for j in w_all if z[j] < z_cut]
    if len(w) < to_flip:
        raise RuntimeError("[plan] Not enough W below z_cut")
    return {"nh_n": nh_n, "nh_p": nh_p, "w": w, "to_flip": to_flip, "z_cut": z_cut}


def _gc_event(kind, st, **kw):
    ev = {"kind": kind, "epoch": st["epoch"], "step_in_block": 0, "acc_since_mu": st["acc_mu"],
          "att_since_mu": st["att_mu"], "block_accepted": st["block_acc"], "block_attempted": st["block_att"],
          "nprot": st["Nprot"], "remaining": max(0, st["target"] - st["Nprot"]), "cause_amax": 0,
          "fwd_total": st["fwd"], "bwd_total": st["bwd"], "mu_kT": float(_f32(st["beta"] * st["mu"])), "f": 0.0,
          "w_info": 0.0, "E": float(st["E"]), "acc_rate": 0.0}
    ev.update(kw)
    return ev


def ref_gc_phase(s, p, raw, plan, gen, max_trials=10 ** 6):
    """phase_gc_mu_control (MC/src/mc.cu:320-548).  s.q / s.type change in place.
    Returns (result dict, events)."""
    NHN, NHP, W, CL = (raw[k] - 1 for k in ("NH_N_type", "NH_P_type", "W_type", "Cl_type"))
    z = np.asarray(s.z, np.float32)
    nh_n, nh_p, w = list(plan["nh_n"]), list(plan["nh_p"]), list(plan["w"])
    cl = [j for j in range(s.n) if s.type[j] == CL and z[j] < plan["z_cut"]]
    beta = _f32(raw["beta"])
    lo, hi = _f32(1e-6), _f32(1.0 - 1e-6)
    fstar = _clampf(_f32(float(_f32(raw["target_pct"])) / 100.0), lo, hi)
    mu = _f32(_f32(_f32(1.0) / beta) * _LIBM.logf(_f32(fstar / _f32(_f32(1.0) - fstar))))
    bound = _f32(_f32(10.0) / beta)
    mu = _clampf(mu, -bound, bound)
    Nh = len(nh_n) + len(nh_p)
    st = {"epoch": 0, "acc_mu": 0, "att_mu": 0, "block_acc": 0, "block_att": 0, "Nprot": len(nh_p),
          "target": int(np.floor(float(_f32(raw["target_pct"])) / 100.0 * Nh)), "fwd": 0, "bwd": 0, "beta": beta,
          "mu": mu, "E": ref_total_real(s, p)}
    res = {"attempted": 0, "accepted": 0, "blocks_done": 0, "Nh": Nh, "target_count": st["target"]}
    events = []

    def done(stop):
        res.update(Nprot=st["Nprot"], accepted_forward=st["fwd"], accepted_backward=st["bwd"], E=float(st["E"]),
                   mu_eff=float(st["mu"]), stop=stop, reached_target=int(stop in (1, 4)))
        return res, events

    if st["Nprot"] == st["target"]:
        ev = {k: 0 for k in _gc_event(0, st)}
        ev.update(kind=5, nprot=st["Nprot"], mu_kT=float(_f32(beta * mu)), E=float(st["E"]))
        events.append(ev)
        return done(4)
    gc_block = raw["gc_block_fixed"] if raw["gc_block_fixed"] > 0 else 2000
    amax = raw["sgmc_epoch_attempt_max"] if raw["sgmc_epoch_attempt_max"] > 0 else 100000
    R0 = max(0, st["target"] - st["Nprot"])
    frac = _f32(raw["sgmc_nacc_frac_round"]) if raw["sgmc_nacc_frac_round"] > 0 else _f32(0.10)
    nacc = max(1, int(math.ceil(float(frac) * float(R0))))
    eta = _f32(raw["mu_eta"]) if raw["mu_eta"] > 0 else _f32(0.3)
    res.update(R0=R0, Nacc_target=nacc, epoch_attempt_max=amax, gc_block=gc_block)
    while True:
        st["acc_mu"] = st["att_mu"] = 0
        while st["acc_mu"] < nacc and st["att_mu"] < amax:
            st["block_acc"] = st["block_att"] = 0
            for t in range(gc_block):
                if res["attempted"] >= max_trials:
                    return done(3)
                a, b, c, d = len(nh_n), len(nh_p), len(w), len(cl)
                wf, wb = a * c, b * d
                if wf > 0 and wb > 0:
                    fwd = gen.unit() < _f32(_f32(wf) / _f32(wf + wb))
                elif wf > 0:
                    fwd = True
                elif wb > 0:
                    fwd = False
                else:
                    events.append(_gc_event(4, st))
                    return done(2)
                if fwd:
                    i = nh_n[gen.index(a)]
                    j = w[gen.index(c)]
                else:
                    i = nh_p[gen.index(b)]
                    j = cl[gen.index(d)]
                old = (s.type[i], s.q[i], s.type[j], s.q[j])
                if fwd:
                    s.type[i], s.q[i], s.type[j], s.q[j] = NHP, 1.0, CL, -1.0
                else:
                    s.type[i], s.q[i], s.type[j], s.q[j] = NHN, 0.0, W, 0.0
                Et = ref_total_real(s, p)
                dE = _f32(Et - st["E"])
                sgn = 1 if fwd else -1
                s_before = wf + wb
                s_after = (a - 1) * (c - 1) + (b + 1) * (d + 1) if fwd else (a + 1) * (c + 1) + (b - 1) * (d - 1)
                logH = math.log(s_before) - math.log(s_after) if s_before > 0 and s_after > 0 else 0.0
                expo = float(_f32(-beta * _f32(dE - _f32(_f32(sgn) * st["mu"])))) + logH
                expo = min(max(expo, -40.0), 40.0)
                accept = expo >= 0.0 or math.exp(expo) > float(gen.unit())
                res["attempted"] += 1
                st["block_att"] += 1
                st["att_mu"] += 1
                if accept:
                    res["accepted"] += 1
                    st["block_acc"] += 1
                    st["acc_mu"] += 1
                    st["fwd" if fwd else "bwd"] += 1
                    st["E"] = Et
                    if fwd:
                        nh_n.remove(i); nh_p.append(i); w.remove(j); cl.append(j)
                    else:
                        nh_p.remove(i); nh_n.append(i); cl.remove(j); w.append(j)
                    st["Nprot"] += sgn
                    if st["Nprot"] == st["target"]:
                        events.append(_gc_event(3, st, step_in_block=t + 1))
                        return done(1)
                else:
                    s.type[i], s.q[i], s.type[j], s.q[j] = old
            rate = _f32(_f32(st["block_acc"]) / _f32(st["block_att"]))
            events.append(_gc_event(1, st, acc_rate=float(rate)))
        st["block_acc"] = st["block_att"] = 0
        f = _f32(_f32(st["Nprot"]) / _f32(Nh)) if Nh > 0 else _f32(0.0)
        f0, f1 = _clampf(fstar, lo, hi), _clampf(f, lo, hi)
        logit = _f32(_LIBM.logf(_f32(f1 / _f32(_f32(1.0) - f1))) - _LIBM.logf(_f32(f0 / _f32(_f32(1.0) - f0))))
        early = st["att_mu"] >= amax and st["acc_mu"] < nacc
        w_info = _clampf(_f32(_f32(st["acc_mu"]) / _f32(max(1, nacc))), _f32(0.0), _f32(1.0)) if nacc > 0 else _f32(1.0)
        step = _f32(_f32(_f32(_f32(_f32(1.0) / beta) * eta) * logit) * w_info)
        st["mu"] = _f32(st["mu"] - step)
        res["blocks_done"] = st["epoch"] + 1
        events.append(_gc_event(2, st, cause_amax=int(early), f=float(f), w_info=float(w_info)))
        st["epoch"] += 1


def _p2_event(kind, **kw):
    ev = {"kind": kind, "attempted": 0, "accepted": 0, "since_best": 0, "patience": 0, "mode_wc": 0, "n_nh_p": 0,
          "n_nh_n": 0, "n_cl": 0, "n_w": 0, "E": 0.0, "acc": 0.0, "z_cut": 0.0}
    ev.update(kw)
    return ev


def ref_phase2(s, p, raw, pools, z_cut, gen):
    """phase2_swap_jitter (MC/src/mc.cu:159-318) on pools (nh_p, nh_n, w, cl; the
    phase-1 result's); s.q / s.type change in place.  Returns (result dict, events)."""
    NHN, NHP, W, CL = (raw[k] - 1 for k in ("NH_N_type", "NH_P_type", "W_type", "Cl_type"))
    z = np.asarray(s.z, np.float32)
    nh_p, nh_n = list(pools["nh_p"]), list(pools["nh_n"])
    w = [j for j in pools["w"] if 0 <= j < s.n and z[j] < z_cut]
    cl = [j for j in pools["cl"] if 0 <= j < s.n and z[j] < z_cut]
    beta = _f32(raw["beta"])
    E = ref_total_real(s, p)
    best = E
    res = {"attempted": 0, "accepted": 0, "since_best": 0}
    events = [_p2_event(11, n_nh_p=len(nh_p), n_nh_n=len(nh_n), n_cl=len(cl), n_w=len(w), z_cut=float(z_cut))]

    def done(stop):
        res.update(E=float(E), best_E=float(best), stop=stop)
        return res, events

    can_wc = lambda: len(w) > 0 and len(cl) > 0
    can_four = lambda: len(nh_p) > 0 and len(nh_n) > 0 and can_wc()
    prefer_wc = len(nh_n) == 0
    if not prefer_wc and not can_four() and can_wc():
        prefer_wc = True
    if not prefer_wc and not can_four() and not can_wc():
        events.append(_p2_event(12))
        return done(0)
    if prefer_wc and not can_wc():
        events.append(_p2_event(13))
        return done(0)
    eps = _f32(1e-9)
    since = 0
    interval = max(1, raw["energy_interval"])
    for _ in range(raw["max_attempts"]):
        four = (not prefer_wc) and can_four()
        wc = prefer_wc or (not four and can_wc())
        if not four and not wc:
            events.append(_p2_event(14))
            return done(3)
        res["attempted"] += 1
        if four:
            iP = nh_p[gen.index(len(nh_p))]
            iN = nh_n[gen.index(len(nh_n))]
            jC = cl[gen.index(len(cl))]
            jW = w[gen.index(len(w))]
            idx = (iP, iN, jC, jW)
            new = ((NHN, 0.0), (NHP, 1.0), (W, 0.0), (CL, -1.0))
        else:
            jC = cl[gen.index(len(cl))]
            jW = w[gen.index(len(w))]
            idx = (jC, jW)
            new = ((W, 0.0), (CL, -1.0))
        old = [(s.type[k], s.q[k]) for k in idx]
        for k, (ty, q) in zip(idx, new):
            s.type[k], s.q[k] = ty, q
        Et = ref_total_real(s, p)
        dE = _f32(Et - E)
        expo = _clampf(_f32(-beta * dE), _f32(-40.0), _f32(40.0))
        accept = dE <= 0 or _f32(_LIBM.expf(expo)) > gen.unit()
        if accept:
            res["accepted"] += 1
            E = Et
            if E < _f32(best - eps):
                best, since = E, 0
            else:
                since += 1
            if four:
                nh_p.remove(iP); nh_n.append(iP); nh_n.remove(iN); nh_p.append(iN)
            cl.remove(jC); w.append(jC); w.remove(jW); cl.append(jW)
        else:
            for k, (ty, q) in zip(idx, old):
                s.type[k], s.q[k] = ty, q
            since += 1
        res["since_best"] = since
        if res["attempted"] % interval == 0:
            acc = _f32(_f32(res["accepted"]) / _f32(res["attempted"]))
            events.append(_p2_event(15, attempted=res["attempted"], accepted=res["accepted"], since_best=since,
                                    patience=raw["patience"], mode_wc=int(not four and wc), E=float(E), acc=float(acc)))
        if since >= raw["patience"]:
            events.append(_p2_event(16, since_best=since, patience=raw["patience"]))
            return done(1)
    return done(2)
