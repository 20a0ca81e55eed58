"""The allocation-free reciprocal-energy entry point (phmc_recip_energy_static).

It serves callers that cannot call cudaMalloc (a process whose device memory
is all handed out by its own allocator, a plugin called back from one, a
per-trial loop that must not stall on an allocation) and keeps its scratch in
one file-scope device array.  Checked through the C ABI against the engine's
own reciprocal energy (phmc_create + phmc_energy, which allocates) and against
the FP64 oracle's, with the tolerance of the other energy tests, on two calls
in a row so that a leftover from the first call (the array keeps its contents)
would show up.  The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as O
from ph_brush_b200 import Engine, _abi, configs

RTOL, ATOL = 1e-6, 1e-4


def call_static(s, p):
    pres = (s.flags & _abi.F_GHOST) == 0
    x, y, z, q = (np.ascontiguousarray(getattr(s, k)[pres], np.float32) for k in "xyzq")
    box = np.ascontiguousarray(s.box, np.float64)
    mesh = np.ascontiguousarray(p.mesh, np.int32)
    out = C.c_double(0.0)
    rc = _abi.lib().phmc_recip_energy_static(_abi.fptr(x), _abi.fptr(y), _abi.fptr(z), _abi.fptr(q), len(x),
                                             _abi.dptr(box), _abi.iptr(mesh), p.order, p.ewald_alpha, p.epsilon_r,
                                             p.ref_moduli, C.byref(out))
    return rc, out.value


def test_static_entry_point_rejects_oversized_inputs():
    s, p = configs.small_system(seed=2)
    p.mesh = (64, 64, 64)  # 262144 points > PHMC_STATIC_MAX_MESH
    rc, _ = call_static(s, p)
    assert rc == 3 and b"PHMC_STATIC_MAX_MESH" in _abi.lib().phmc_last_error()
    n = 32769
    z = np.zeros(n, np.float32)
    out = C.c_double()
    rc = _abi.lib().phmc_recip_energy_static(_abi.fptr(z), _abi.fptr(z), _abi.fptr(z), _abi.fptr(z), n,
                                             _abi.dptr(np.ones(3)), _abi.iptr(np.array([16, 16, 16], np.int32)), 5,
                                             1.0, 1.0, 0, C.byref(out))
    assert rc == 3 and b"PHMC_STATIC_MAX_PARTICLES" in _abi.lib().phmc_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small", "config1", "reference_semantics"])
def test_static_recip_energy_matches_engine(case):
    if case == "small":
        s, p = configs.small_system(seed=31)
    elif case == "config1":
        s, p = configs.config1()
    else:
        sn, _ = configs.small_system(seed=32)
        s, p = configs.to_reference_semantics(sn, n_w=8, spacing=0.45)  # odd mesh 27x27x80, reference moduli
        assert p.mesh[0] % 2 == 1
    with Engine(s, p) as e:
        ref = e.energy()[0]["coul_recip"]
    orc = O.energy(s, p)["coul_recip"]
    for _ in range(2):
        rc, got = call_static(s, p)
        assert rc == 0, _abi.lib().phmc_last_error()
        assert abs(got - ref) <= RTOL * abs(ref) + ATOL, (got, ref)
        assert abs(got - orc) <= RTOL * abs(orc) + ATOL, (got, orc)
