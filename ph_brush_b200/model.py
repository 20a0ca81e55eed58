"""Host-side containers for one replica: particle system and interaction/move model.

`SystemArrays` mirrors the reference's System (MC/include/types.hpp:25-32,
positions wrapped into [0, L) as MC/src/io.cpp:303-316 does) with SoA arrays,
per-particle move flags and capacity-padded slots for inserted ions.
`ModelParams` mirrors the reference's Params (MC/include/types.hpp:34-69) plus
the native model's keys (WCA cutoff, FENE, walls, pH/pKa, salt reservoir).
"""
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

KE = 138.935458  # MC/src/pme.cu:305


def ewald_alpha(rc, rtol):
    """alpha = erfcinv(clamp(rtol, 1e-12, 0.5)) / rc (MC/src/io.cpp:72-77)."""
    from scipy.special import erfcinv
    if rtol <= 0:
        rtol = 1e-5
    r = min(max(rtol, 1e-12), 0.5)
    return float(erfcinv(r)) / rc


@dataclass
class SystemArrays:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    q: np.ndarray
    type: np.ndarray
    flags: np.ndarray
    bond_i: np.ndarray
    bond_j: np.ndarray
    box: np.ndarray
    capacity: int
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.x)

    def to_struct(self):
        arrs = [_abi.as_f32(self.x), _abi.as_f32(self.y), _abi.as_f32(self.z), _abi.as_f32(self.q),
                _abi.as_i32(self.type), _abi.as_i32(self.flags), _abi.as_i32(self.bond_i), _abi.as_i32(self.bond_j)]
        s = _abi.System()
        s.n_particles = self.n
        s.capacity = int(self.capacity)
        s.x, s.y, s.z, s.q = (_abi.fptr(a) for a in arrs[:4])
        s.type, s.flags = _abi.iptr(arrs[4]), _abi.iptr(arrs[5])
        s.n_bonds = len(arrs[6])
        s.bond_i, s.bond_j = _abi.iptr(arrs[6]), _abi.iptr(arrs[7])
        for k in range(3):
            s.box[k] = float(self.box[k])
        return s, arrs

    def copy(self):
        return SystemArrays(*(np.array(getattr(self, f)) for f in
                              ("x", "y", "z", "q", "type", "flags", "bond_i", "bond_j", "box")),
                            capacity=self.capacity, meta=dict(self.meta))


@dataclass
class ModelParams:
    n_types: int
    lj_eps: np.ndarray
    lj_sig: np.ndarray
    lj_rc: np.ndarray = None
    rc_lj: float = 3.0
    lj_shift: int = 1
    coulomb: int = _abi.COUL_EWALD
    rc_coul: float = 3.0
    epsilon_r: float = 1.0
    ewald_alpha: float = 0.0
    mesh: tuple = (32, 32, 32)
    order: int = 4
    ref_moduli: int = 0
    slab: int = 0
    excl_bonded_lj: int = 0
    excl_bonded_coul: int = 0
    fene_k: float = 0.0
    fene_r0: float = 1.5
    wall_lo: float = 0.0
    wall_hi: float = 0.0
    beta: float = 1.0
    pH: float = 7.0
    pKa: float = 7.0
    type_site_neutral: int = 0
    type_site_charged: int = 1
    q_site_charged: float = 1.0
    type_counterion: int = 2
    q_counterion: float = -1.0
    salt_conc: float = 0.0
    type_cation: int = 3
    q_cation: float = 1.0
    p_disp: float = 0.9
    p_titr: float = 0.1
    p_swap: float = 0.0
    disp_max: float = 0.3
    seed: int = 2025
    cell_cap: int = 0
    pending_max: int = 0
    threads: int = 0

    def to_struct(self):
        eps = _abi.as_f64(self.lj_eps).ravel()
        sig = _abi.as_f64(self.lj_sig).ravel()
        keep = [eps, sig]
        p = _abi.Params()
        p.n_types = self.n_types
        p.lj_eps, p.lj_sig = _abi.dptr(eps), _abi.dptr(sig)
        if self.lj_rc is not None:
            rc = _abi.as_f64(self.lj_rc).ravel()
            keep.append(rc)
            p.lj_rc = _abi.dptr(rc)
        else:
            p.lj_rc = C.cast(None, C.POINTER(C.c_double))
        for name, _ in _abi.Params._fields_:
            if name in ("lj_eps", "lj_sig", "lj_rc", "n_types"):
                continue
            if name == "mesh":
                for k in range(3):
                    p.mesh[k] = int(self.mesh[k])
                continue
            setattr(p, name, getattr(self, name))
        return p, keep

    @property
    def elf(self):
        return KE / self.epsilon_r


def wca_tables(n_types, eps=1.0, sig=1.0):
    e = np.full((n_types, n_types), eps)
    s = np.full((n_types, n_types), sig)
    rc = np.full((n_types, n_types), 2.0 ** (1.0 / 6.0) * sig)
    return e, s, rc


def ideal_alpha(pH, pKa):
    """Degree of ionisation of an ideal weak base: 1 / (1 + 10^(pH - pKa))."""
    return 1.0 / (1.0 + 10.0 ** (pH - pKa))


def build_brush(chains_x, chains_y, spacing, len_min, len_max, height, lz, ion_frac, salt_conc,
                n_permanent=0, graft_titratable=1, seed=2025, extra=None, bond_len=0.97, min_dist=0.9):
    """Synthetic brush via the library's generator (phmc_build_brush)."""
    spec = _abi.BrushSpec(chains_x, chains_y, spacing, len_min, len_max, n_permanent, graft_titratable,
                          height, lz, ion_frac, salt_conc, bond_len, min_dist, seed)
    nch = chains_x * chains_y
    est_salt = int(salt_conc * chains_x * chains_y * spacing * spacing * height * 1.1) + 16
    cap = nch * len_max * 2 + 2 * est_salt + 64
    x = np.zeros(cap, np.float32); y = np.zeros(cap, np.float32); z = np.zeros(cap, np.float32)
    q = np.zeros(cap, np.float32); t = np.zeros(cap, np.int32); f = np.zeros(cap, np.int32)
    bi = np.zeros(nch * len_max, np.int32); bj = np.zeros(nch * len_max, np.int32)
    counts = np.zeros(2, np.int32); box = np.zeros(3, np.float64)
    _abi.check(_abi.lib().phmc_build_brush(C.byref(spec), cap, _abi.fptr(x), _abi.fptr(y), _abi.fptr(z),
                                           _abi.fptr(q), _abi.iptr(t), _abi.iptr(f), len(bi), _abi.iptr(bi),
                                           _abi.iptr(bj), _abi.iptr(counts), _abi.dptr(box)))
    n, nb = int(counts[0]), int(counts[1])
    n_sites = int(np.count_nonzero(f[:n] & _abi.F_TITRATABLE))
    if extra is None:
        extra = n_sites + 64
    return SystemArrays(x[:n].copy(), y[:n].copy(), z[:n].copy(), q[:n].copy(), t[:n].copy(), f[:n].copy(),
                        bi[:nb].copy(), bj[:nb].copy(), box, capacity=n + extra,
                        meta={"chains": nch, "n_sites": n_sites, "height": height})
