"""CPU checks of the C-ABI library: it loads, exports every entry point the
header declares, validates arguments without touching a GPU, and the host-only
brush generator is deterministic and physically sane."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ph_brush_b200 import _abi, configs
from ph_brush_b200.model import build_brush

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*|int64_t|void)\s+\**(phmc_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_struct_sizes():
    assert _abi.lib().phmc_abi_version() == 1
    # layout sanity: the trial struct is 4 + 2*28 bytes
    assert C.sizeof(_abi.Change) == 28 and C.sizeof(_abi.Trial) == 60


def test_create_rejects_bad_arguments_before_any_device_call():
    s, p = configs.small_system(seed=1)
    s.capacity = s.n - 1  # capacity below the particle count
    S, k1 = s.to_struct()
    P, k2 = p.to_struct()
    h = C.c_void_p()
    rc = _abi.lib().phmc_create(1, C.byref(S), C.byref(P), 0, C.byref(h))
    assert rc == 1 and b"capacity" in _abi.lib().phmc_last_error()
    s, p = configs.small_system(seed=1)
    p.mesh = (14, 16, 48)  # 14 = 2*7 is not 2^a 3^b 5^c
    S, k1 = s.to_struct()
    P, k2 = p.to_struct()
    rc = _abi.lib().phmc_create(1, C.byref(S), C.byref(P), 0, C.byref(h))
    assert rc == 6
    s, p = configs.small_system(seed=1)
    s.x[3] = 1e3  # outside the box
    S, k1 = s.to_struct()
    P, k2 = p.to_struct()
    assert _abi.lib().phmc_create(1, C.byref(S), C.byref(P), 0, C.byref(h)) == 1


def test_brush_generator_deterministic_and_sane():
    a = build_brush(3, 3, 4.0, 12, 12, 30.0, 90.0, 0.5, 0.002, seed=9)
    b = build_brush(3, 3, 4.0, 12, 12, 30.0, 90.0, 0.5, 0.002, seed=9)
    for f in ("x", "y", "z", "q", "type", "flags", "bond_i", "bond_j"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    assert abs(a.q.sum()) < 1e-6  # neutral
    assert a.z.min() >= 0 and a.z.max() < 30.0
    d = np.stack([a.x[a.bond_i] - a.x[a.bond_j], a.y[a.bond_i] - a.y[a.bond_j], a.z[a.bond_i] - a.z[a.bond_j]], 1)
    d[:, 0] -= a.box[0] * np.round(d[:, 0] / a.box[0])
    d[:, 1] -= a.box[1] * np.round(d[:, 1] / a.box[1])
    assert np.allclose(np.linalg.norm(d, axis=1), 0.97, atol=1e-4)
    grafted = a.flags[:9 * 12:12] & _abi.F_MOBILE
    assert not grafted.any()


def test_config_sizes():
    s, p = configs.config1()
    assert 500 <= s.n <= 540 and tuple(p.mesh) == (32, 32, 128) and p.order == 5
    assert abs(p.ewald_alpha - 1.0402) < 1e-3


def test_reference_mesh_rule():
    # MC/src/pme.cu:46-51,312-317
    assert configs.good_fft_dim(7) == 8 and configs.good_fft_dim(31) == 32 and configs.good_fft_dim(61) == 64
    assert configs.ref_mesh((16.0, 16.0, 120.0), 0.5) == (32, 32, 240)
