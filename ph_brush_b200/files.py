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


def reference_model(data_path, params_path):
    """A system in the reference's model from its input files, as its driver sets it up
    (MC/src/main.cu:102-139: positions wrapped, Lz padded by pme_3dc's factor, 0-based
    types, 1-2 pairs excluded from LJ and real-space Coulomb, cubic SPME with the
    reference's moduli, mesh from pme_spacing, slab correction with pme_3dc):
    returns (SystemArrays, ModelParams) for an Engine."""
    from .configs import ref_mesh
    from .model import ModelParams, SystemArrays
    d = read_lammps(data_path, wrap=True)
    T = int(d["ntypes"])
    v, eps, sig, sh, _ = read_params(params_path, T)
    box = np.array(d["box"], np.float64)
    slab = bool(v["pme_3dc"])
    if slab:
        box[2] *= max(2.0, v["pme_3dc_zfac"])
    n = int(d["natoms"])
    s = SystemArrays(d["x"].copy(), d["y"].copy(), d["z"].copy(), d["q"].copy(), (d["type"] - 1).astype(np.int32),
                     np.zeros(n, np.int32), d["bond_i"].astype(np.int32), d["bond_j"].astype(np.int32), box, capacity=n,
                     meta={"height": float(d["box"][2]), "zfac": float(box[2] / d["box"][2])})
    order = int(v["pme_order"]) if v["pme_order"] > 0 else 4
    coul = _abi.COUL_EWALD if v["coulomb"] == _abi.COUL_EWALD else v["coulomb"]
    p = ModelParams(n_types=T, lj_eps=eps, lj_sig=sig, lj_rc=None, rc_lj=v["rc"], lj_shift=int(v["lj_shift"]),
                    coulomb=coul, rc_coul=v["rc"], epsilon_r=v["epsilon_r"], ewald_alpha=v["ewald_alpha"],
                    mesh=ref_mesh(box, v["pme_spacing"], order), order=order, ref_moduli=1, slab=1 if slab else 0,
                    excl_bonded_lj=1, excl_bonded_coul=1, fene_k=0.0, wall_lo=0.0, wall_hi=0.0, beta=v["beta"],
                    p_disp=0.0, p_titr=0.0, p_swap=0.0)
    return s, p
