"""ctypes mirror of include/phmc.h and the loader of the in-tree libphmc.so.

The library is the only compute path: importing this module on a machine
without the built library raises immediately (there is no CPU fallback).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libphmc.so")

PHMC_OK = 0
ERRORS = {1: "ARG", 2: "CUDA", 3: "CAPACITY", 4: "BUDGET", 5: "STATE", 6: "UNSUPPORTED", 7: "IO"}
COUL_NONE, COUL_CUT, COUL_EWALD = 0, 1, 2
F_MOBILE, F_TITRATABLE, F_GHOST, F_CATION, F_ANION = 0x01, 0x02, 0x04, 0x08, 0x10
MOVE_DISP, MOVE_TITR, MOVE_SWAP, MOVE_NONE = 0, 1, 2, 3
SUR_INPUTS, SUR_ROWS = 80, 4
SUR_DESC_STRIDE = SUR_ROWS * SUR_INPUTS + 2 * SUR_ROWS + 4

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


class System(C.Structure):
    _fields_ = [("n_particles", C.c_int), ("capacity", C.c_int),
                ("x", _fp), ("y", _fp), ("z", _fp), ("q", _fp),
                ("type", _ip), ("flags", _ip),
                ("n_bonds", C.c_int), ("bond_i", _ip), ("bond_j", _ip),
                ("box", C.c_double * 3)]


class Params(C.Structure):
    _fields_ = [("n_types", C.c_int), ("lj_eps", _dp), ("lj_sig", _dp), ("lj_rc", _dp),
                ("rc_lj", C.c_double), ("lj_shift", C.c_int), ("coulomb", C.c_int),
                ("rc_coul", C.c_double), ("epsilon_r", C.c_double), ("ewald_alpha", C.c_double),
                ("mesh", C.c_int * 3), ("order", C.c_int), ("ref_moduli", C.c_int), ("slab", C.c_int),
                ("excl_bonded_lj", C.c_int), ("excl_bonded_coul", C.c_int),
                ("fene_k", C.c_double), ("fene_r0", C.c_double),
                ("wall_lo", C.c_double), ("wall_hi", C.c_double), ("beta", C.c_double),
                ("pH", C.c_double), ("pKa", C.c_double),
                ("type_site_neutral", C.c_int), ("type_site_charged", C.c_int), ("q_site_charged", C.c_float),
                ("type_counterion", C.c_int), ("q_counterion", C.c_float),
                ("salt_conc", C.c_double), ("type_cation", C.c_int), ("q_cation", C.c_float),
                ("p_disp", C.c_double), ("p_titr", C.c_double), ("p_swap", C.c_double), ("disp_max", C.c_double),
                ("seed", C.c_uint64),
                ("cell_cap", C.c_int), ("pending_max", C.c_int), ("threads", C.c_int)]


class LammpsInfo(C.Structure):
    _fields_ = [("natoms", C.c_int), ("nbonds", C.c_int), ("nbonds_read", C.c_int), ("ntypes", C.c_int),
                ("box", C.c_double * 3)]


FILE_PARAMS_D1 = ("rc", "epsilon_r", "ewald_rtol", "ewald_alpha", "pme_spacing", "pme_3dc_zfac", "beta", "target_pct",
                  "w_z_extra_nm", "mu_eta", "nacc_frac_round")
FILE_PARAMS_I = ("lj_shift", "coulomb", "pme_order", "pme_3dc", "nh_n_type", "nh_p_type", "w_type", "cl_type", "rng_seed",
                 "energy_interval", "patience", "max_attempts", "direct_pct_threshold", "gc_block_fixed",
                 "epoch_attempt_max", "phase2_wc")
FILE_PARAMS_D2 = ("pH", "pKa", "salt_conc", "wall_lo", "wall_hi", "fene_k", "fene_r0", "p_disp", "p_titr", "p_swap",
                  "disp_max")


# phmc_event_fn: (user, job, phase, record)
EventFn = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.c_void_p)


class FileParams(C.Structure):
    _fields_ = ([(k, C.c_double) for k in FILE_PARAMS_D1] + [(k, C.c_int) for k in FILE_PARAMS_I] +
                [(k, C.c_double) for k in FILE_PARAMS_D2] + [("mesh", C.c_int * 3)])


class EnergyComponents(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("lj", "fene", "coul_real", "coul_recip", "self", "qcorr", "slab", "total")]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Change(C.Structure):
    _fields_ = [("index", C.c_int), ("present", C.c_int), ("x", C.c_float), ("y", C.c_float),
                ("z", C.c_float), ("q", C.c_float), ("type", C.c_int)]


class Trial(C.Structure):
    _fields_ = [("n_changes", C.c_int), ("c", Change * 2)]


class RunStats(C.Structure):
    _fields_ = [("attempted", C.c_int64 * 3), ("accepted", C.c_int64 * 3), ("flushes", C.c_int64),
                ("n_titratable", C.c_int), ("n_charged_sites", C.c_int), ("n_cations", C.c_int),
                ("n_anions", C.c_int), ("energy", C.c_double), ("energy_drift", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("mc_ms", C.c_double), ("flush_ms", C.c_double), ("mc_launches", C.c_int64),
                ("flush_launches", C.c_int64), ("kernel_launches", C.c_int64), ("mc_alg_bytes", C.c_double),
                ("flush_alg_bytes", C.c_double), ("trials", C.c_int64), ("mc_busy_ms", C.c_double)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DAStats(C.Structure):
    _fields_ = [("evaluated", C.c_int64), ("passed", C.c_int64), ("accepted", C.c_int64),
                ("fallback", C.c_int), ("pad", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class Tuning(C.Structure):
    _fields_ = [("pending_max", C.c_int), ("threads", C.c_int), ("us_per_trial", C.c_double),
                ("zpass", C.c_int), ("zpass_n1", C.c_int), ("zpass_n2", C.c_int), ("cand_round", C.c_int),
                ("g_rows", C.c_int), ("plane_pipe", C.c_int),
                ("energy_block", C.c_int), ("rebuild_us", C.c_double), ("recompute_us", C.c_double),
                ("first_stage", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BrushSpec(C.Structure):
    _fields_ = [("chains_x", C.c_int), ("chains_y", C.c_int), ("graft_spacing", C.c_double),
                ("len_min", C.c_int), ("len_max", C.c_int), ("n_permanent", C.c_int),
                ("graft_titratable", C.c_int), ("height", C.c_double), ("lz", C.c_double),
                ("ion_frac", C.c_double), ("salt_conc", C.c_double), ("bond_len", C.c_double),
                ("min_dist", C.c_double), ("seed", C.c_uint64)]


GC_EV_CHUNK, GC_EV_MU, GC_EV_REACHED, GC_EV_NO_PAIRS, GC_EV_ALREADY = 1, 2, 3, 4, 5
GC_STOP_REACHED, GC_STOP_NO_PAIRS, GC_STOP_MAX_TRIALS, GC_STOP_ALREADY = 1, 2, 3, 4


class GcEvent(C.Structure):
    _fields_ = [("kind", C.c_int), ("epoch", C.c_int), ("step_in_block", C.c_int),
                ("acc_since_mu", C.c_int), ("att_since_mu", C.c_int),
                ("block_accepted", C.c_int), ("block_attempted", C.c_int),
                ("nprot", C.c_int), ("remaining", C.c_int), ("cause_amax", C.c_int),
                ("fwd_total", C.c_int64), ("bwd_total", C.c_int64),
                ("mu_kT", C.c_float), ("f", C.c_float), ("w_info", C.c_float), ("E", C.c_float),
                ("acc_rate", C.c_float)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GcJob(C.Structure):
    _fields_ = [("replica", C.c_int), ("nh_n_type", C.c_int), ("nh_p_type", C.c_int), ("w_type", C.c_int),
                ("cl_type", C.c_int), ("q_nh_p", C.c_float), ("q_cl", C.c_float), ("beta", C.c_double),
                ("target_pct", C.c_double), ("mu_eta", C.c_double), ("nacc_frac", C.c_double),
                ("gc_block", C.c_int), ("epoch_attempt_max", C.c_int), ("max_trials", C.c_int64),
                ("nh_n", _ip), ("n_nh_n", C.c_int), ("nh_p", _ip), ("n_nh_p", C.c_int),
                ("w", _ip), ("n_w", C.c_int), ("cl", _ip), ("n_cl", C.c_int),
                ("mt_state", C.POINTER(C.c_uint32)), ("fixed_mu", C.c_int), ("mu_kT", C.c_double)]


class GcResult(C.Structure):
    _fields_ = [("attempted", C.c_int), ("accepted", C.c_int), ("accepted_forward", C.c_int),
                ("accepted_backward", C.c_int), ("blocks_done", C.c_int), ("Nh", C.c_int), ("Nprot", C.c_int),
                ("target_count", C.c_int), ("reached_target", C.c_int), ("stop", C.c_int),
                ("E", C.c_float), ("mu_eff", C.c_float), ("R0", C.c_int), ("Nacc_target", C.c_int),
                ("epoch_attempt_max", C.c_int), ("gc_block", C.c_int), ("n_events", C.c_int),
                ("events_dropped", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


P2_EV_POOLS, P2_EV_NONE_AT_START, P2_EV_WC_EMPTY, P2_EV_NONE, P2_EV_STEP, P2_EV_PATIENCE = 11, 12, 13, 14, 15, 16
P2_STOP_PATIENCE, P2_STOP_MAX_ATTEMPTS, P2_STOP_NO_PROPOSALS = 1, 2, 3


class Phase2Event(C.Structure):
    _fields_ = [("kind", C.c_int), ("attempted", C.c_int), ("accepted", C.c_int), ("since_best", C.c_int),
                ("patience", C.c_int), ("mode_wc", C.c_int), ("n_nh_p", C.c_int), ("n_nh_n", C.c_int),
                ("n_cl", C.c_int), ("n_w", C.c_int), ("E", C.c_float), ("acc", C.c_float), ("z_cut", C.c_float),
                ("pad", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class Phase2Job(C.Structure):
    _fields_ = [("replica", C.c_int), ("nh_n_type", C.c_int), ("nh_p_type", C.c_int), ("w_type", C.c_int),
                ("cl_type", C.c_int), ("q_nh_p", C.c_float), ("q_cl", C.c_float), ("beta", C.c_double),
                ("max_attempts", C.c_int), ("patience", C.c_int), ("energy_interval", C.c_int), ("z_cut", C.c_float),
                ("nh_p", _ip), ("n_nh_p", C.c_int), ("nh_n", _ip), ("n_nh_n", C.c_int),
                ("w", _ip), ("n_w", C.c_int), ("cl", _ip), ("n_cl", C.c_int),
                ("mt_state", C.POINTER(C.c_uint32))]


class Phase2Result(C.Structure):
    _fields_ = [("attempted", C.c_int), ("accepted", C.c_int), ("E", C.c_float), ("best_E", C.c_float),
                ("stop", C.c_int), ("since_best", C.c_int), ("n_events", C.c_int), ("events_dropped", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PHASES = ("proposal", "first_stage", "cells_stencils_direct", "offsets_pair_tables", "candidate_pairs",
          "phi_pending_reduce", "decision_commit", "ended_early")

EXPORTS = ["phmc_abi_version", "phmc_last_error", "phmc_create", "phmc_destroy", "phmc_energy",
           "phmc_delta_energy", "phmc_commit", "phmc_set_identity", "phmc_run", "phmc_set_trial_log",
           "phmc_set_replay", "phmc_get_state", "phmc_get_cells", "phmc_capacity", "phmc_build_brush",
           "phmc_set_state", "phmc_set_quorum", "phmc_set_launch_budget", "phmc_set_tile_shapes", "phmc_set_event_callback", "phmc_set_first_stage", "phmc_set_zhist", "phmc_get_zhist", "phmc_checkpoint_save", "phmc_checkpoint_load", "phmc_lammps_header", "phmc_lammps_read", "phmc_lammps_write", "phmc_params_read", "phmc_set_profiling", "phmc_get_profile", "phmc_set_phase_clock", "phmc_get_phase_cycles", "phmc_run_timed", "phmc_flush_l2",
           "phmc_recip_energy_static",
           "phmc_surrogate_create", "phmc_surrogate_set_gemm", "phmc_surrogate_destroy", "phmc_surrogate_num_params",
           "phmc_surrogate_get_params", "phmc_surrogate_set_params", "phmc_surrogate_set_scaling",
           "phmc_surrogate_get_scaling", "phmc_surrogate_predict", "phmc_surrogate_gradient",
           "phmc_surrogate_train", "phmc_surrogate_save", "phmc_surrogate_load", "phmc_harvest",
           "phmc_harvest_count", "phmc_harvest_get", "phmc_surrogate_fit", "phmc_surrogate_attach",
           "phmc_get_da_stats", "phmc_surrogate_describe", "phmc_set_da_log", "phmc_set_move_mix",
           "phmc_set_tuning", "phmc_get_tuning", "phmc_autotune", "phmc_delta_energy_components",
           "phmc_gc_phase", "phmc_gc_event_format", "phmc_phase2", "phmc_phase2_event_format"]


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libphmc.so not built at {path}: run `make -C ph_brush_b200` "
                          "(the engine has no CPU fallback)")
    lib = C.CDLL(path)
    lib.phmc_last_error.restype = C.c_char_p
    eng = C.c_void_p
    sig = {
        "phmc_abi_version": ([], C.c_int),
        "phmc_create": ([C.c_int, C.POINTER(System), C.POINTER(Params), C.c_int, C.POINTER(eng)], C.c_int),
        "phmc_destroy": ([eng], C.c_int),
        "phmc_energy": ([eng, C.POINTER(EnergyComponents)], C.c_int),
        "phmc_delta_energy": ([eng, C.c_int, C.POINTER(Trial), C.c_int, _dp], C.c_int),
        "phmc_commit": ([eng, C.c_int, C.POINTER(Trial)], C.c_int),
        "phmc_set_identity": ([eng, C.c_int, C.c_int, C.c_int, C.c_float], C.c_int),
        "phmc_run": ([eng, C.c_int64, C.POINTER(RunStats)], C.c_int),
        "phmc_set_trial_log": ([eng, C.c_int64, _ip, _dp, _ip], C.c_int),
        "phmc_set_replay": ([eng, C.c_int64, _ip], C.c_int),
        "phmc_get_state": ([eng, C.c_int, _fp, _fp, _fp, _fp, _ip, _ip], C.c_int),
        "phmc_get_cells": ([eng, C.c_int, _ip, _ip], C.c_int),
        "phmc_capacity": ([eng, C.c_int], C.c_int),
        "phmc_build_brush": ([C.POINTER(BrushSpec), C.c_int, _fp, _fp, _fp, _fp, _ip, _ip, C.c_int, _ip, _ip, _ip, _dp], C.c_int),
        "phmc_set_state": ([eng, C.c_int, _fp, _fp, _fp, _fp, _ip, _ip], C.c_int),
        "phmc_set_profiling": ([eng, C.c_int], C.c_int),
        "phmc_lammps_header": ([C.c_char_p, C.POINTER(LammpsInfo)], C.c_int),
        "phmc_lammps_read": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(LammpsInfo)], C.c_int),
        "phmc_lammps_write": ([C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double)], C.c_int),
        "phmc_params_read": ([C.c_char_p, C.c_int, C.c_int, C.POINTER(FileParams), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_char_p, C.c_int], C.c_int),
        "phmc_checkpoint_save": ([eng, C.c_char_p], C.c_int),
        "phmc_checkpoint_load": ([eng, C.c_char_p], C.c_int),
        "phmc_set_quorum": ([eng, C.c_double], C.c_int),
        "phmc_set_launch_budget": ([eng, C.c_int64], C.c_int),
        "phmc_set_tile_shapes": ([eng, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "phmc_set_first_stage": ([eng, C.c_int], C.c_int),
        "phmc_set_event_callback": ([eng, EventFn, C.c_void_p], C.c_int),
        "phmc_set_zhist": ([eng, C.c_int, C.c_int64], C.c_int),
        "phmc_get_zhist": ([eng, C.c_int, _dp, C.POINTER(C.c_int64)], C.c_int),
        "phmc_get_profile": ([eng, C.POINTER(Profile), C.c_int], C.c_int),
        "phmc_set_phase_clock": ([eng, C.c_int], C.c_int),
        "phmc_get_phase_cycles": ([eng, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int], C.c_int),
        "phmc_run_timed": ([eng, C.c_int64, _dp], C.c_int),
        "phmc_flush_l2": ([eng, C.c_int64], C.c_int),
        "phmc_recip_energy_static": ([_fp, _fp, _fp, _fp, C.c_int, _dp, _ip, C.c_int, C.c_double, C.c_double,
                                      C.c_int, _dp], C.c_int),
        "phmc_surrogate_create": ([C.c_int, C.c_int, C.c_uint64, C.POINTER(eng)], C.c_int),
        "phmc_surrogate_set_gemm": ([C.c_int], C.c_int),
        "phmc_surrogate_destroy": ([eng], C.c_int),
        "phmc_surrogate_num_params": ([eng], C.c_int),
        "phmc_surrogate_get_params": ([eng, _fp, C.c_int], C.c_int),
        "phmc_surrogate_set_params": ([eng, _fp, C.c_int], C.c_int),
        "phmc_surrogate_set_scaling": ([eng, _fp, _fp, C.c_float], C.c_int),
        "phmc_surrogate_get_scaling": ([eng, _fp, _fp, _fp], C.c_int),
        "phmc_surrogate_predict": ([eng, _fp, C.c_int, _fp], C.c_int),
        "phmc_surrogate_gradient": ([eng, _fp, _fp, _fp, C.c_int, C.c_float, _dp, _fp], C.c_int),
        "phmc_surrogate_train": ([eng, _fp, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint64,
                                  C.c_int, _dp], C.c_int),
        "phmc_surrogate_save": ([eng, C.c_char_p], C.c_int),
        "phmc_surrogate_load": ([C.c_char_p, C.POINTER(eng)], C.c_int),
        "phmc_harvest": ([eng, C.c_int], C.c_int),
        "phmc_harvest_count": ([eng, _ip], C.c_int),
        "phmc_harvest_get": ([eng, C.c_int, _fp, _fp, _fp], C.c_int),
        "phmc_surrogate_fit": ([eng, eng, C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint64, _dp], C.c_int),
        "phmc_surrogate_attach": ([eng, eng, C.c_double, C.c_int], C.c_int),
        "phmc_get_da_stats": ([eng, C.POINTER(DAStats)], C.c_int),
        "phmc_surrogate_describe": ([eng, C.c_int, C.POINTER(Trial), C.c_int, _fp, _dp], C.c_int),
        "phmc_set_da_log": ([eng, _ip, _dp], C.c_int),
        "phmc_set_move_mix": ([eng, C.c_int, C.c_double, C.c_double, C.c_double], C.c_int),
        "phmc_set_tuning": ([eng, C.c_int, C.c_int], C.c_int),
        "phmc_delta_energy_components": ([eng, C.c_int, C.POINTER(Trial), C.c_int, C.POINTER(EnergyComponents)], C.c_int),
        "phmc_get_tuning": ([eng, C.POINTER(Tuning)], C.c_int),
        "phmc_autotune": ([eng, C.c_int64, C.POINTER(Tuning), C.c_int, _ip], C.c_int),
        "phmc_gc_phase": ([eng, C.c_int, C.POINTER(GcJob), C.POINTER(GcResult), C.POINTER(GcEvent), C.c_int], C.c_int),
        "phmc_gc_event_format": ([C.POINTER(GcEvent), C.POINTER(GcResult), C.c_char_p, C.c_int], C.c_int),
        "phmc_phase2": ([eng, C.c_int, C.POINTER(Phase2Job), C.POINTER(Phase2Result), C.POINTER(Phase2Event), C.c_int],
                        C.c_int),
        "phmc_phase2_event_format": ([C.POINTER(Phase2Event), C.c_char_p, C.c_int], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


class PhmcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"phmc error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def check(status):
    if status != PHMC_OK:
        raise PhmcError(status, lib().phmc_last_error().decode())
    return status


def fptr(a):
    return a.ctypes.data_as(_fp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def dptr(a):
    return a.ctypes.data_as(_dp)


def as_f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
