"""Workloads: the five brush configurations (seeded synthetic systems) and the
reference-semantics variant used for parity with the reference's own energy
routines.

Reduced units: sigma = 1, kT = 1 (beta = 1), Bjerrum length 1.4 sigma, i.e.
epsilon_r = 138.935458 / 1.4 with the reference's Coulomb constant.  Salt
molarities are converted with sigma = 0.5 nm (1 M = 0.6022 nm^-3).
Native particle types: 0 neutral site, 1 charged site, 2 anion, 3 cation,
4 permanently charged bead.
"""
import math

import numpy as np

from . import _abi
from .model import ModelParams, SystemArrays, build_brush, ewald_alpha, ideal_alpha, wca_tables

SIGMA_NM = 0.5
L_BJERRUM = 1.4
EPS_R = 138.935458 / L_BJERRUM
N_TYPES = 5


def molar_to_sigma3(c):
    return c * 0.6022 * SIGMA_NM ** 3


def smooth_mesh(n, lo=8, hi=512):
    """Smallest 2^a 3^b >= n (clamped to [lo, hi])."""
    n = max(lo, min(hi, int(math.ceil(n))))
    m = n
    while True:
        k = m
        for p in (2, 3):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def native_params(pH, pKa, mesh, height, seed, salt_conc=0.0, order=5, rc=3.0, rtol=1e-5,
                  p_disp=0.9, p_titr=0.1, p_swap=0.0, disp_max=0.3, lb=L_BJERRUM):
    eps, sig, rc_lj = wca_tables(N_TYPES)
    coul = _abi.COUL_EWALD if lb > 0 else _abi.COUL_NONE
    return ModelParams(n_types=N_TYPES, lj_eps=eps, lj_sig=sig, lj_rc=rc_lj, rc_lj=float(rc_lj[0, 0]), lj_shift=1,
                       coulomb=coul, rc_coul=rc, epsilon_r=(138.935458 / lb if lb > 0 else 1.0),
                       ewald_alpha=ewald_alpha(rc, rtol), mesh=tuple(mesh), order=order, ref_moduli=0, slab=1,
                       excl_bonded_lj=0, excl_bonded_coul=0, fene_k=30.0, fene_r0=1.5,
                       wall_lo=0.0, wall_hi=float(height), beta=1.0, pH=pH, pKa=pKa,
                       type_site_neutral=0, type_site_charged=1, q_site_charged=1.0,
                       type_counterion=2, q_counterion=-1.0, salt_conc=salt_conc, type_cation=3, q_cation=1.0,
                       p_disp=p_disp, p_titr=p_titr, p_swap=p_swap, disp_max=disp_max, seed=seed)


def config1(seed=2025, order=5, lb=L_BJERRUM):
    """16 chains x 20 beads on a 4x4 lattice (spacing 4) in 16x16x40 padded to 120; pH = pKa = 7.5;
    50% ionised; 20 salt pairs; mesh 32x32x128."""
    H = 40.0
    sysa = build_brush(4, 4, 4.0, 20, 20, H, 3 * H, 0.5, 20.0 / (16 * 16 * H), seed=seed)
    prm = native_params(7.5, 7.5, (32, 32, 128), H, seed, order=order, lb=lb)
    return sysa, prm


def config2(seed=2026, order=5):
    """10x10 chains x 50 titratable beads, spacing 4, 40x40x100 padded to 300, pH 6.5 / pKa 7.5,
    0.1 M salt (~12k particles), mesh 64x64x384."""
    H = 100.0
    pH, pKa = 6.5, 7.5
    sysa = build_brush(10, 10, 4.0, 50, 50, H, 3 * H, ideal_alpha(pH, pKa), molar_to_sigma3(0.1), seed=seed)
    prm = native_params(pH, pKa, (64, 64, 384), H, seed, order=order)
    return sysa, prm


def config4(seed=2026, order=5):
    """config 2 plus reservoir Na+/Cl- pair swaps at 0.1 M."""
    sysa, prm = config2(seed, order)
    sysa.capacity += 2048
    prm.p_disp, prm.p_titr, prm.p_swap = 0.85, 0.10, 0.05
    prm.salt_conc = molar_to_sigma3(0.1)
    return sysa, prm


def config3(seed=2027, order=5, n_rep=96):
    """96 replicas: pH 4.0..9.75 (step 0.25) x salt {0.001, 0.01, 0.1, 0.5} M; grafting density
    cycling 0.05/0.1/0.2 sigma^-2, chain length 30-60 per replica, lateral box ~24 sigma."""
    rng = np.random.default_rng(seed)
    out = []
    salts = [0.001, 0.01, 0.1, 0.5]
    for k in range(n_rep):
        pH = 4.0 + 0.25 * (k % 24)
        salt = salts[(k // 24) % 4]
        dens = [0.05, 0.1, 0.2][k % 3]
        a = 1.0 / math.sqrt(dens)
        nc = max(3, int(round(24.0 / a)))
        ln = int(rng.integers(30, 61))
        H = float(ln + 10)
        L = nc * a
        hx = L / 0.75
        mesh = (smooth_mesh(min(64, max(32, hx))), smooth_mesh(min(64, max(32, hx))), smooth_mesh(3 * H / 0.75))
        s = build_brush(nc, nc, a, ln, ln, H, 3 * H, ideal_alpha(pH, 7.5), molar_to_sigma3(salt), seed=seed + 1000 + k)
        p = native_params(pH, 7.5, mesh, H, seed + 1000 + k, salt_conc=0.0, order=order)
        out.append((s, p))
    return out


def config5(seed=2029, order=5, n_rep=256):
    """256 diblock replicas: 20 permanent +1 beads + 30 titratable beads (pKa 7.3) per chain,
    64-144 chains, pH 5-9, salt 0.001-0.3 M, slab height 60 padded to 180."""
    rng = np.random.default_rng(seed)
    out = []
    H = 60.0
    for k in range(n_rep):
        side = int(rng.integers(8, 13))
        pH = float(rng.uniform(5.0, 9.0))
        salt = float(math.exp(rng.uniform(math.log(0.001), math.log(0.3))))
        L = 4.0 * side
        nxy = smooth_mesh(min(64, max(32, L / 0.75)))
        mesh = (nxy, nxy, smooth_mesh(3 * H / 0.75))
        s = build_brush(side, side, 4.0, 50, 50, H, 3 * H, ideal_alpha(pH, 7.3), molar_to_sigma3(salt),
                        n_permanent=20, graft_titratable=0, seed=seed + 1000 + k)
        p = native_params(pH, 7.3, mesh, H, seed + 1000 + k, order=order)
        out.append((s, p))
    return out


def diblock_small(seed=2031, order=5, n_rep=24, side=4):
    """Config-5 chemistry on small replicas (side x side diblock chains: 20 permanent +1 and 30
    titratable beads, pKa 7.3), pH 5..9 evenly spaced, salt 0.01 / 0.03 / 0.1 M cycling; small enough
    for the degree of ionisation to equilibrate within a benchmark run."""
    out = []
    H = 60.0
    salts = [0.01, 0.03, 0.1]
    for k in range(n_rep):
        pH = 5.0 + 4.0 * k / max(n_rep - 1, 1)
        salt = salts[k % 3]
        L = 4.0 * side
        nxy = smooth_mesh(max(32, L / 0.75))
        mesh = (nxy, nxy, smooth_mesh(3 * H / 0.75))
        s = build_brush(side, side, 4.0, 50, 50, H, 3 * H, ideal_alpha(pH, 7.3), molar_to_sigma3(salt),
                        n_permanent=20, graft_titratable=0, seed=seed + k)
        p = native_params(pH, 7.3, mesh, H, seed + k, order=order)
        out.append((s, p))
    return out


def small_system(seed=7, chains=2, length=6, box_xy=12.0, height=12.0, salt_pairs=4, order=5, mesh=(16, 16, 48),
                 lb=L_BJERRUM, ion_frac=0.5, p_swap=0.0, salt_conc=0.0):
    """A few dozen particles for oracle-sized parity tests."""
    a = box_xy / chains
    s = build_brush(chains, chains, a, length, length, height, 3 * height, ion_frac,
                    salt_pairs / (box_xy * box_xy * height), seed=seed)
    p = native_params(7.0, 7.0, mesh, height, seed, order=order, lb=lb, p_swap=p_swap, salt_conc=salt_conc,
                      p_disp=0.9 - p_swap, p_titr=0.1)
    return s, p


# ---------------------------------------------------------------------------
# Reference semantics: LJ cut and shifted at the shared cutoff, 1-2 pairs
# excluded from LJ and real-space Coulomb (MC/src/neighbor.cu:17-19,97),
# cubic spreading with the reference's moduli and corner rule, mesh from
# pme_spacing (MC/src/pme.cu:46-51,312-317), slab padding pme_3dc yes zfac.
# Reference 1-based types: 3 permanent, 4 NH_N, 5 NH_P, 6 Na, 7 W, 8 Cl.
# ---------------------------------------------------------------------------
NATIVE_TO_REF = np.array([4, 5, 8, 6, 3], np.int32)
REF_W_TYPE = 7
REF_NTYPES = 8


def good_fft_dim(n):
    """MC/src/pme.cu:46-51."""
    nmax = max(16, n * 2 + 32)
    for m in range(max(8, n), nmax + 1):
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
    return n


def ref_mesh(box, spacing, order=4):
    return tuple(max(good_fft_dim(int(math.ceil(box[k] / spacing))), order) for k in range(3))


def to_reference_semantics(sysa, n_w=0, seed=1, spacing=0.5, rc=3.0, rtol=1e-5, order=4, zfac=3.0):
    """Map a native brush to the reference's model: reference types, W beads
    (non-interacting q=0 identity pool) appended, LJ eps=sigma=1 for all types
    except W (eps 0).  Returns (SystemArrays with 0-based reference types, ModelParams)."""
    rng = np.random.default_rng(seed)
    H = float(sysa.meta.get("height", sysa.box[2] / zfac))
    wx = rng.uniform(0, sysa.box[0], n_w).astype(np.float32)
    wy = rng.uniform(0, sysa.box[1], n_w).astype(np.float32)
    wz = rng.uniform(0, H, n_w).astype(np.float32)
    t = np.concatenate([NATIVE_TO_REF[sysa.type] - 1, np.full(n_w, REF_W_TYPE - 1, np.int32)])
    f = np.concatenate([sysa.flags, np.zeros(n_w, np.int32)])
    s = SystemArrays(np.concatenate([sysa.x, wx]), np.concatenate([sysa.y, wy]), np.concatenate([sysa.z, wz]),
                     np.concatenate([sysa.q, np.zeros(n_w, np.float32)]), t.astype(np.int32), f.astype(np.int32),
                     sysa.bond_i.copy(), sysa.bond_j.copy(), sysa.box.copy(), capacity=sysa.n + n_w,
                     meta=dict(sysa.meta, n_w=n_w))
    T = REF_NTYPES
    eps = np.ones((T, T))
    eps[REF_W_TYPE - 1, :] = 0.0
    eps[:, REF_W_TYPE - 1] = 0.0
    sig = np.ones((T, T))
    mesh = ref_mesh(s.box, spacing, order)
    p = ModelParams(n_types=T, lj_eps=eps, lj_sig=sig, lj_rc=None, rc_lj=rc, lj_shift=1, coulomb=_abi.COUL_EWALD,
                    rc_coul=rc, epsilon_r=EPS_R, ewald_alpha=ewald_alpha(rc, rtol), mesh=mesh, order=order,
                    ref_moduli=1, slab=1, excl_bonded_lj=1, excl_bonded_coul=1, fene_k=0.0, wall_lo=0.0, wall_hi=0.0,
                    beta=1.0, p_disp=0.0, p_titr=0.0, p_swap=0.0)
    return s, p


def write_lammps_data(path, s, ref_types_1based=True):
    """LAMMPS 'full' data file in the reference's input format (MC/src/io.cpp:79-146)."""
    n = s.n
    with open(path, "w") as fh:
        fh.write("# synthetic brush\n\n")
        fh.write(f"{n} atoms\n{len(s.bond_i)} bonds\n\n{REF_NTYPES} atom types\n1 bond types\n\n")
        fh.write(f"0.0 {s.box[0]:.10f} xlo xhi\n0.0 {s.box[1]:.10f} ylo yhi\n")
        zfac = s.meta.get("zfac", 3.0)
        fh.write(f"0.0 {s.box[2] / zfac:.10f} zlo zhi\n\nAtoms # full\n\n")
        for i in range(n):
            t = int(s.type[i]) + 1 if ref_types_1based else int(s.type[i])
            fh.write(f"{i + 1} {1 + i // 1000} {t} {float(s.q[i]):.1f} {float(s.x[i]):.9g} {float(s.y[i]):.9g} {float(s.z[i]):.9g}\n")
        if len(s.bond_i):
            fh.write("\nBonds\n\n")
            for k in range(len(s.bond_i)):
                fh.write(f"{k + 1} 1 {int(s.bond_i[k]) + 1} {int(s.bond_j[k]) + 1}\n")


def write_params_in(path, p, spacing, zfac=3.0, extra=None, coulombtype="pme"):
    """params.in in the reference's key = value format (MC/src/io.cpp:171-301).
    ewald_alpha is left to the reference's own rule (erfcinv(ewald_rtol)/cutoff)."""
    lines = [f"cutoff_nm = {p.rc_coul}", "lj_shift = yes", f"epsilon_r = {p.epsilon_r:.10g}",
             f"coulombtype = {coulombtype}", "ewald_rtol = 1e-5", f"pme_spacing = {spacing}", f"pme_order = {p.order}",
             f"pme_3dc = yes {zfac}", "beta = 1.0", "nh_n_type = 4", "nh_p_type = 5", "w_type = 7", "cl_type = 8"]
    if extra:
        lines += [f"{k} = {v}" for k, v in extra.items()]
    T = p.n_types
    for i in range(T):
        for j in range(i, T):
            lines.append(f"lj {i + 1} {j + 1} {p.lj_eps[i, j]:.6g} {p.lj_sig[i, j]:.6g}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
