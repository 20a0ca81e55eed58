"""Pins the FP64 oracle: known answers from first principles and the published
Philox vectors (the reference ships no tests or golden files)."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O
from ph_brush_b200 import _abi, configs
from ph_brush_b200.model import ModelParams, SystemArrays


def test_cubic_bspline_matches_reference_closed_form():
    # MC/src/pme.cu:132-138
    for t in (0.0, 0.13, 0.5, 0.77, 0.999):
        w = O.bspline_weights(4, t)
        ref = [(1 - 3 * t + 3 * t * t - t ** 3) / 6, (4 - 6 * t * t + 3 * t ** 3) / 6,
               (1 + 3 * t + 3 * t * t - 3 * t ** 3) / 6, t ** 3 / 6]
        assert np.allclose(w, ref, atol=1e-15)


@pytest.mark.parametrize("p", [4, 5, 6])
def test_bspline_partition_of_unity(p):
    for t in np.linspace(0, 0.999, 17):
        assert abs(O.bspline_weights(p, t).sum() - 1.0) < 1e-14


@pytest.mark.parametrize("p,n", [(4, 16), (4, 27), (5, 32), (6, 48)])
def test_moduli_equal_direct_dft(p, n):
    m = O.moduli(n, p, 1)
    w0 = O.bspline_weights(p, 0.0)
    vals = [w0[p - 1 - j] for j in range(1, p)]  # M_p(1..p-1)
    dft = np.abs([sum(vals[j - 1] * np.exp(2j * np.pi * k * j / n) for j in range(1, p)) for k in range(n)]) ** 2
    nz = dft > 1e-12
    assert np.allclose(m[nz], dft[nz], rtol=1e-12, atol=1e-15)


def test_native_moduli_interpolate_odd_order_nyquist():
    m = O.moduli(32, 5, 0)
    assert m[16] > 1e-4 and abs(m[16] - 0.5 * (m[15] + m[17])) < 1e-15


def test_fft3d_matches_numpy():
    rng = np.random.default_rng(0)
    g = rng.standard_normal((12, 10, 6)) + 1j * rng.standard_normal((12, 10, 6))
    re, im = np.ascontiguousarray(g.real).ravel(), np.ascontiguousarray(g.imag).ravel()
    O.L.orc_fft3d(re.ctypes.data_as(O._dp), im.ctypes.data_as(O._dp), 6, 10, 12, -1)
    assert np.abs((re + 1j * im).reshape(12, 10, 6) - np.fft.fftn(g)).max() < 1e-12


def test_madelung_constant_nacl():
    pts = [(i, j, k) for i in range(4) for j in range(4) for k in range(4)]
    x, y, z = (np.array([p[a] for p in pts], float) for a in range(3))
    q = np.array([(-1.0) ** sum(p) for p in pts])
    r = O.direct_ewald(x, y, z, q, np.array([4.0, 4.0, 4.0]), 1.2, 138.935458, 0, 1e-14)
    assert abs(-r["total"] / 32.0 - 1.747564594633182) < 1e-9


def test_direct_ewald_alpha_independent():
    rng = np.random.default_rng(3)
    n = 24
    x, y, z = rng.uniform(0, 6, n), rng.uniform(0, 7, n), rng.uniform(0, 5, n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    q[0] = 2.0  # net charge: exercises the neutralising-background term
    a = O.direct_ewald(x, y, z, q, np.array([6.0, 7.0, 15.0]), 0.9, 80.0, 1, 1e-13)
    b = O.direct_ewald(x, y, z, q, np.array([6.0, 7.0, 15.0]), 1.6, 80.0, 1, 1e-13)
    assert abs(a["total"] - b["total"]) < 1e-8 * abs(a["total"])


def _two_particle(r, types=(0, 0), q=(0.0, 0.0), coul=_abi.COUL_NONE, bonded=False, fene=0.0):
    s = SystemArrays(np.array([1.0, 1.0 + r], np.float32), np.array([1.0, 1.0], np.float32),
                     np.array([1.0, 1.0], np.float32), np.array(q, np.float32), np.array(types, np.int32),
                     np.array([1, 1], np.int32), np.array([0] if bonded else [], np.int32),
                     np.array([1] if bonded else [], np.int32), np.array([10.0, 10.0, 10.0]), capacity=2)
    eps, sig = np.ones((2, 2)), np.ones((2, 2))
    p = ModelParams(n_types=2, lj_eps=eps, lj_sig=sig, rc_lj=2.5, lj_shift=0, coulomb=coul, rc_coul=4.0,
                    epsilon_r=138.935458, ewald_alpha=0.8, mesh=(16, 16, 16), order=4, fene_k=fene, fene_r0=1.5)
    return s, p


def test_lj_minimum_and_wca_shift():
    rmin = 2.0 ** (1.0 / 6.0)
    s, p = _two_particle(rmin)
    assert abs(O.energy(s, p)["lj"] + 1.0) < 1e-6
    p.lj_rc = np.full((2, 2), rmin)
    p.lj_shift = 1
    assert abs(O.energy(s, p)["lj"]) < 1e-6  # WCA is zero at its cutoff
    s2, _ = _two_particle(1.0)
    assert abs(O.energy(s2, p)["lj"] - 1.0) < 1e-6  # 4(1-1)+1


def test_fene_closed_form():
    r = 1.1
    s, p = _two_particle(r, bonded=True, fene=30.0)
    p.lj_eps = np.zeros((2, 2))
    expect = -0.5 * 30.0 * 1.5 ** 2 * math.log(1 - (r / 1.5) ** 2)
    assert abs(O.energy(s, p)["fene"] - expect) < 1e-5


def test_spme_converges_to_direct_ewald():
    s, p = configs.small_system(seed=11, chains=2, length=5, box_xy=10.0, height=10.0, salt_pairs=3)
    p.lj_eps = p.lj_eps * 0
    pres = (s.flags & _abi.F_GHOST) == 0
    r = O.direct_ewald(s.x[pres], s.y[pres], s.z[pres], s.q[pres], s.box, 0.8, p.epsilon_r, 1, 1e-12)
    errs = []
    for mesh in [(16, 16, 48), (32, 32, 96), (64, 64, 192)]:
        p.mesh, p.order = mesh, 6
        e = O.energy(s, p)
        coul = e["coul_real"] + e["coul_recip"] + e["self"] + e["qcorr"] + e["slab"]
        errs.append(abs(coul - r["total"]))
    assert errs[2] < errs[0] and errs[2] < 1e-4 * abs(r["total"]) + 1e-3


def test_philox_known_answers():
    # Random123 published known-answer vectors for philox4x32-10
    assert [hex(v) for v in O.philox([0, 0], [0, 0, 0, 0])] == ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(v) for v in O.philox([0xffffffff] * 2, [0xffffffff] * 4)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(v) for v in O.philox([0xa4093822, 0x299f31d0], [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_oracle_mc_ideal_titration():
    """l_B = 0 and WCA off: the sampled degree of ionisation is 1/(1+10^(pH-pKa))."""
    s, p = configs.small_system(seed=5, chains=2, length=10, box_xy=10.0, height=10.0, salt_pairs=0, lb=0.0)
    p.lj_eps = p.lj_eps * 0
    p.fene_k = 0.0
    p.p_disp, p.p_titr = 0.0, 1.0
    p.pH, p.pKa = 7.3, 7.0
    mc = O.MC(s, p)
    ns = s.meta["n_sites"]
    samples = []
    for k in range(6000):
        mc.step()
        if k > 500 and k % 5 == 0:
            samples.append(mc.counts()[0] / ns)
    a = np.mean(samples)
    expect = 1.0 / (1.0 + 10 ** (p.pH - p.pKa))
    assert abs(a - expect) < 0.03
