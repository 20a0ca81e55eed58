"""ORACLE — test infrastructure only (ctypes wrapper over oracle/_build/libphoracle.so).

Imported by tests/, the smoke check and bench.py's CPU-baseline leg only.
"""
import ctypes as C
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
           "pme_3dc": int(ii[3]), "lj_eps": eps.reshape(T, T), "lj_sig": sig.reshape(T, T), "lj_shift_tbl": sh.reshape(T, T)}
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
