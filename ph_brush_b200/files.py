"""Input files of the reference's driver through the library's host-side readers:
LAMMPS "full" data files and params.in (include/phmc.h, csrc/lammps_io.cpp)."""
import ctypes as C

import numpy as np

from . import _abi


def read_lammps(path, wrap=True):
    """Atoms (file order) and bonds (0-based atom indices) of a LAMMPS "full" data file."""
    lib = _abi.lib()
    info = _abi.LammpsInfo()
    _abi.check(lib.phmc_lammps_header(str(path).encode(), C.byref(info)))
    n, nb = info.natoms, max(info.nbonds, 0)
    i32 = lambda k: np.zeros(k, np.int32)
    f32 = lambda k: np.zeros(k, np.float32)
    out = {"id": i32(n), "mol": i32(n), "type": i32(n), "q": f32(n), "x": f32(n), "y": f32(n), "z": f32(n),
           "bond_type": i32(nb + 1), "bond_i": i32(nb + 1), "bond_j": i32(nb + 1)}
    _abi.check(lib.phmc_lammps_read(str(path).encode(), int(wrap), n, nb, *(_abi.iptr(out[k]) for k in ("id", "mol", "type")),
                                    *(_abi.fptr(out[k]) for k in ("q", "x", "y", "z")),
                                    *(_abi.iptr(out[k]) for k in ("bond_type", "bond_i", "bond_j")), C.byref(info)))
    for k in ("bond_type", "bond_i", "bond_j"):
        out[k] = out[k][:info.nbonds_read].copy()
    out.update(natoms=info.natoms, nbonds=info.nbonds, ntypes=info.ntypes, box=np.array(info.box[:]))
    return out


def write_lammps(path, d):
    """Write a LAMMPS "full" data file from read_lammps-style arrays (box from 0)."""
    lib = _abi.lib()
    a = {k: np.ascontiguousarray(d[k], np.int32) for k in ("id", "mol", "type", "bond_type", "bond_i", "bond_j")}
    a.update({k: np.ascontiguousarray(d[k], np.float32) for k in ("q", "x", "y", "z")})
    box = np.ascontiguousarray(d["box"], np.float64)
    _abi.check(lib.phmc_lammps_write(str(path).encode(), len(a["id"]), *(_abi.iptr(a[k]) for k in ("id", "mol", "type")),
                                     *(_abi.fptr(a[k]) for k in ("q", "x", "y", "z")), len(a["bond_type"]),
                                     *(_abi.iptr(a[k]) for k in ("bond_type", "bond_i", "bond_j")), int(d["ntypes"]),
                                     _abi.dptr(box)))


def read_params(path, ntypes, strict=False):
    """params.in: the reference's keys, defaults and derived values, plus the native model's keys.
    Returns (dict of values, lj_eps, lj_sig, lj_shift as ntypes x ntypes arrays, list of unknown entries)."""
    lib = _abi.lib()
    fp = _abi.FileParams()
    eps, sig, sh = (np.zeros(ntypes * ntypes) for _ in range(3))
    unk = C.create_string_buffer(4096)
    _abi.check(lib.phmc_params_read(str(path).encode(), ntypes, int(strict), C.byref(fp), _abi.dptr(eps), _abi.dptr(sig),
                                    _abi.dptr(sh), unk, 4096))
    vals = {k: getattr(fp, k) for k in _abi.FILE_PARAMS_D1 + _abi.FILE_PARAMS_I + _abi.FILE_PARAMS_D2}
    vals["mesh"] = tuple(fp.mesh)
    unknown = [u for u in unk.value.decode().split(",") if u]
    return vals, eps.reshape(ntypes, ntypes), sig.reshape(ntypes, ntypes), sh.reshape(ntypes, ntypes), unknown
