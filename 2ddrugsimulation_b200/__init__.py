"""cep_b200: B200-native cardiac drug-screening hot path.

Python access to the C ABI of libcep_b200.so (include/cep_b200.h). The
package directory name starts with a digit, so import it with
``importlib.import_module("2ddrugsimulation_b200")``.

The product path is the CUDA library only: every call goes through the
shared library, and constructing a Batch without a visible GPU or without
the built library raises instead of falling back to any CPU code.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libcep_b200.so"

# status codes (cep_b200.h)
OK, ERR_ARG, ERR_OOM, ERR_CUDA, ERR_NOT_CONVERGED, ERR_TIMEOUT, ERR_NONFINITE, ERR_UNSUPPORTED, ERR_STATE, \
    ERR_NO_DEVICE = range(10)
INST_RUNNING, INST_DONE, INST_NONFINITE, INST_IDLE = 0, 1, 2, 3
MODELS = {"ord2011": 0, "cipa2017": 1, "tt2006": 2, "tt2004": 3, "tomek2019": 4}
N_STATES = {"ord2011": 41, "cipa2017": 49, "tt2006": 19, "tt2004": 17, "tomek2019": 43}
PREC = {"fp64": 0, "mixed": 1}
FLAG_DUTTA, FLAG_QUIRKS, FLAG_TT04_MCELL, FLAG_NEO_ORD = 1, 2, 4, 8
CURRENTS = ("INa", "INaL", "Ito", "ICaL", "IKr", "IKs", "IK1")
APDR_FIELDS = ("pace", "recal", "bcl", "apd90", "di", "t")
LAYOUT_SOA, LAYOUT_AOS = 0, 1
# conductances cep_batch_scale multiplies (CEP_SCALE_*), by the reference
# deck's key stem (gna_scale -> "gna")
SCALE = {"gna": 0, "gnal": 1, "gto": 2, "gcal": 3, "gkr": 4, "gks": 5, "gk1": 6, "gbna": 7, "gbca": 8, "gpca": 9,
         "gpk": 10, "gkb": 11, "gncx": 12, "pnak": 13}
HILL_WIDTH = 20

BM_FIELDS = ("qnet", "inal_auc", "ical_auc", "dvmdt_repol", "dvmdt_max", "vm_peak", "vm_valley", "vm_dia",
             "apd90", "apd50", "apd_tri", "ca_peak", "ca_valley", "ca_dia", "cad90", "cad50", "cad_tri")


class Biomarkers(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in BM_FIELDS] + [
        ("steepest_pace", ctypes.c_int32), ("n_eligible", ctypes.c_int32), ("status", ctypes.c_int32),
        ("reserved", ctypes.c_int32)]


class HrvRecord(ctypes.Structure):
    _fields_ = [("beat", Biomarkers), ("bcl", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class CepJob(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("celltype", ctypes.POINTER(ctypes.c_double)),
                ("conc", ctypes.POINTER(ctypes.c_double)), ("hill", ctypes.POINTER(ctypes.c_double)),
                ("hill_stride", ctypes.c_int), ("bcl", ctypes.c_double), ("n_pace", ctypes.c_int),
                ("first_pace", ctypes.c_int), ("flags", ctypes.c_uint)]


class PopulationJob(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("n", ctypes.c_int), ("celltype", ctypes.POINTER(ctypes.c_double)),
                ("conc", ctypes.POINTER(ctypes.c_double)), ("hill", ctypes.POINTER(ctypes.c_double)),
                ("hill_stride", ctypes.c_int), ("flags", ctypes.c_uint), ("bcl", ctypes.c_double),
                ("amp_scale", ctypes.c_double), ("scale", ctypes.POINTER(ctypes.c_double)),
                ("states_init", ctypes.POINTER(ctypes.c_double)), ("dt", ctypes.c_double),
                ("dt_write", ctypes.c_double), ("n_pace", ctypes.c_int), ("first_pace", ctypes.c_int),
                ("precision", ctypes.c_int), ("refine_above_vm", ctypes.c_double), ("screen_paces", ctypes.c_int),
                ("steps_per_launch", ctypes.c_long)]


class TissueJob(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("h", ctypes.c_double), ("D", ctypes.c_double),
                ("dt", ctypes.c_double), ("duration", ctypes.c_double), ("conc", ctypes.c_double),
                ("hill", ctypes.POINTER(ctypes.c_double)), ("bcl", ctypes.c_double), ("stim_nx", ctypes.c_int),
                ("stim_ny", ctypes.c_int), ("rtol", ctypes.c_double)]


class ApdrRecord(ctypes.Structure):
    _fields_ = [("pace", ctypes.c_int32), ("recal", ctypes.c_int32), ("bcl", ctypes.c_double),
                ("apd90", ctypes.c_double), ("di", ctypes.c_double), ("t", ctypes.c_double)]


class JobTimes(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("cell_steps", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int), ("queued", ctypes.c_int), ("running", ctypes.c_int),
                ("slots_used", ctypes.c_int), ("completed", ctypes.c_longlong), ("launches", ctypes.c_longlong),
                ("cell_steps", ctypes.c_double), ("busy_ms", ctypes.c_double), ("wall_ms", ctypes.c_double)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4


class CepError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cep error {code}: {msg}")
        self.code = code


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None

# Every symbol include/cep_b200.h declares, with its ctypes signature.
_SIGS = {
    "cep_version": (ctypes.c_char_p, []),
    "cep_last_error": (ctypes.c_char_p, []),
    "cep_device_count": (ctypes.c_int, []),
    "cep_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "cep_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_batch_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "cep_batch_set_block": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cep_batch_set_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cep_batch_init": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int, ctypes.c_uint]),
    "cep_batch_set_pacing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double]),
    "cep_batch_set_protocol": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double]),
    "cep_batch_scale": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "cep_batch_get_conductance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "cep_batch_set_conductance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "cep_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    "cep_fem_set_wait_test": (ctypes.c_int, [ctypes.c_long, ctypes.c_uint]),
    "cep_population_run": (ctypes.c_int, [ctypes.POINTER(PopulationJob), ctypes.c_void_p, _ip]),
    "cep_population_late_mask": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_int, _ip]),
    "cep_batch_run_to_end": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    "cep_batch_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "cep_batch_set_states": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int]),
    "cep_batch_get_states": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int]),
    "cep_batch_device_states": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                               ctypes.POINTER(ctypes.c_long)]),
    "cep_batch_get_biomarkers": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Biomarkers)]),
    "cep_batch_get_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "cep_batch_get_clock": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                                           _dp]),
    "cep_batch_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_batch_rates": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp, _dp]),
    "cep_batch_rates_all": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp]),
    "cep_batch_checkpoint_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t)]),
    "cep_batch_checkpoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "cep_batch_restore": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "cep_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    "cep_batch_restitution": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_long, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int)]),
    "cep_batch_clamp": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, _dp]),
    "cep_batch_hrv": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_long, ctypes.c_void_p]),
    "cep_batch_reserve_biomarkers": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_double]),
    "cep_batch_init_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int,
                                            ctypes.c_uint]),
    "cep_batch_set_pacing_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "cep_batch_start_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "cep_batch_release_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "cep_batch_get_biomarkers_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                      ctypes.POINTER(Biomarkers)]),
    "cep_serve_start": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_long, ctypes.c_double, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "cep_serve_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CepJob), ctypes.POINTER(ctypes.c_uint64)]),
    "cep_serve_submit_tissue": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(TissueJob),
                                               ctypes.POINTER(ctypes.c_uint64)]),
    "cep_serve_tissue_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(JobTimes)]),
    "cep_serve_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, _ip]),
    "cep_serve_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double]),
    "cep_serve_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Biomarkers),
                                        ctypes.POINTER(JobTimes)]),
    "cep_serve_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "cep_serve_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "cep_serve_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServeStats)]),
    "cep_serve_stop": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_qinward": (ctypes.c_double, [ctypes.POINTER(Biomarkers), ctypes.POINTER(Biomarkers)]),
    "cep_fem_create_grid": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "cep_fem_create_csr": (ctypes.c_int, [ctypes.c_int, _ip, _ip, _dp, _dp, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "cep_fem_create_tet": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _ip, _dp, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "cep_fem_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_fem_info": (ctypes.c_int, [ctypes.c_void_p, _ip, ctypes.POINTER(ctypes.c_long), _ip, _ip]),
    "cep_fem_set_format": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cep_fem_get_csr": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, _dp, _dp]),
    "cep_fem_set_solver": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "cep_fem_spmv": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp]),
    "cep_fem_solve": (ctypes.c_int, [ctypes.c_void_p, _dp, _ip, _dp]),
    "cep_fem_solve_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cep_fem_stats": (ctypes.c_int, [ctypes.c_void_p, _ip, ctypes.POINTER(ctypes.c_long),
                                     ctypes.POINTER(ctypes.c_long), _ip, _dp]),
    "cep_fem_solve_csr_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                 ctypes.c_void_p, ctypes.c_void_p, _ip]),
    "cep_tissue_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "cep_tissue_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_tissue_set_stimulus": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "cep_tissue_set_activation_threshold": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cep_tissue_set_clock": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cep_tissue_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    "cep_tissue_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_tissue_get_v": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "cep_tissue_get_activation": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "cep_tissue_group_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_void_p)]),
    "cep_tissue_group_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    "cep_tissue_group_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_tissue_set_electrodes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.c_long, ctypes.c_long]),
    "cep_tissue_get_ecg": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_long)]),
    "cep_tissue_set_s2": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_uint8), ctypes.c_double]),
    "cep_tissue_group_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "cep_tissue_group_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long)]),
    "cep_tissue_stats": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_long),
                                        ctypes.POINTER(ctypes.c_long), _ip]),
    # slab parts (slab.py)
    "cep_part_split": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]),
    "cep_part_create_grid": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "cep_part_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cep_part_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long),
                                     ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]),
    "cep_part_get_csr": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "cep_part_set_solver": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "cep_part_pack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cep_part_cg_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "cep_part_cg_direction": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p]),
    "cep_part_cg_product": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "cep_part_cg_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p]),
    "cep_part_cg_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "cep_part_cg_end": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]),
    "cep_part_bind_cells": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]),
    "cep_part_ionic_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cep_part_get_activation": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
}


def lib() -> ctypes.CDLL:
    """Load libcep_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() or "
                              f"python 2ddrugsimulation_b200/build.py")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


def _check(rc: int) -> None:
    if rc != OK:
        raise CepError(rc, lib().cep_last_error().decode())


def _dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def device_count() -> int:
    return int(lib().cep_device_count())


class Batch:
    """A population of cells of one model resident on the GPU.

    Mirrors the reference's per-object cell-model API (initConsts, the
    pacing overrides, computeRates + solveAnalytical stepping) for n
    instances at once.
    """

    def __init__(self, model: str, n: int, precision: str = "fp64", stream: int | None = None):
        self.model = model
        self.n = int(n)
        self.ns = N_STATES[model]
        h = ctypes.c_void_p()
        _check(lib().cep_batch_create(MODELS[model], self.n, PREC[precision], stream, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cep_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def init(self, celltype=None, conc=None, hill=None, dutta: bool = False, quirks: bool = True,
             mcell: bool = False, neo: bool = False) -> "Batch":
        """neo (ORd 2011) selects the CEPCell_NEO build the HRV bench drives,
        in place of the quirks / intended choice."""
        ct = None if celltype is None else np.ascontiguousarray(np.broadcast_to(celltype, (self.n,)), np.float64)
        cc = None if conc is None else np.ascontiguousarray(np.broadcast_to(conc, (self.n,)), np.float64)
        hh = None
        stride = 0
        if hill is not None:
            hh = np.asarray(hill, np.float64)
            if hh.ndim == 1:
                hh = np.broadcast_to(hh, (self.n, hh.shape[0]))
            hh = np.ascontiguousarray(hh)
            stride = hh.shape[1]
        flags = (FLAG_DUTTA if dutta else 0) | (FLAG_QUIRKS if quirks and not neo else 0) | \
            (FLAG_TT04_MCELL if mcell else 0) | (FLAG_NEO_ORD if neo else 0)
        _check(lib().cep_batch_init(self._h, _dptr(ct), _dptr(cc), _dptr(hh), stride, flags))
        return self

    def set_pacing(self, bcl: float, stim_start: float = -1.0, stim_dur: float = -1.0, amp_scale: float = 1.0):
        _check(lib().cep_batch_set_pacing(self._h, bcl, stim_start, stim_dur, amp_scale))
        return self

    def scale(self, conductance: str, factor):
        """CONSTANTS[g] *= factor[i] for every instance i after init (the
        reference's G*_Scale keys and population-of-models sweeps);
        conductance is a SCALE key, factor a scalar or one value per
        instance."""
        f = np.ascontiguousarray(np.broadcast_to(np.asarray(factor, np.float64), (self.n,)))
        _check(lib().cep_batch_scale(self._h, SCALE[conductance], _dptr(f)))
        return self

    def conductance(self, conductance: str) -> np.ndarray:
        """The named conductance of every instance (its CONSTANTS value)."""
        v = np.zeros(self.n)
        _check(lib().cep_batch_get_conductance(self._h, SCALE[conductance], _dptr(v)))
        return v

    def set_conductance(self, conductance: str, values):
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), (self.n,)))
        _check(lib().cep_batch_set_conductance(self._h, SCALE[conductance], _dptr(v)))
        return self

    def set_protocol(self, dt: float, n_pace: int, first_pace: int = -1, dt_write: float = 1.0,
                     qnet_vm_threshold: float = -1e300):
        _check(lib().cep_batch_set_protocol(self._h, dt, n_pace, first_pace, dt_write, qnet_vm_threshold))
        return self

    def set_block(self, threads: int):
        _check(lib().cep_batch_set_block(self._h, threads))
        return self

    def set_kernel(self, variant: str):
        """'cell' (one thread per cell), 'roles' (4 warps per 32 cells) or
        'pairs' (2 warps per 32 cells)."""
        _check(lib().cep_batch_set_kernel(self._h, {"cell": 0, "roles": 1, "pairs": 2}[variant]))
        return self

    def run(self, n_steps: int):
        _check(lib().cep_batch_run(self._h, int(n_steps)))
        return self

    def checkpoint(self) -> bytes:
        """The whole batch mid-protocol as a self-describing blob."""
        n = ctypes.c_size_t()
        _check(lib().cep_batch_checkpoint_size(self._h, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(lib().cep_batch_checkpoint(self._h, buf, n.value))
        return buf.raw

    def restore(self, blob: bytes) -> "Batch":
        """Resume from a checkpoint() of a batch of the same model, size and precision."""
        _check(lib().cep_batch_restore(self._h, blob, len(blob)))
        return self

    def autotune(self, n_steps: int = 400) -> tuple[str, int]:
        """Time each kernel form and block size on this batch's instances
        (state restored after every trial) and keep the fastest."""
        v, blk = ctypes.c_int(), ctypes.c_int()
        _check(lib().cep_batch_autotune(self._h, int(n_steps), ctypes.byref(v), ctypes.byref(blk)))
        return {0: "cell", 1: "roles", 2: "pairs"}[v.value], blk.value

    def step(self, t: float, dt: float, stim_mode: int = -1):
        """One step of every instance from time t (computeRates + solveAnalytical)."""
        _check(lib().cep_batch_step(self._h, t, dt, int(stim_mode)))
        return self

    def run_to_end(self, steps_per_launch: int = 20000):
        _check(lib().cep_batch_run_to_end(self._h, int(steps_per_launch)))
        return self

    def sync(self):
        _check(lib().cep_batch_sync(self._h))
        return self

    def get_states(self, layout: int = LAYOUT_AOS) -> np.ndarray:
        out = np.zeros((self.n, self.ns) if layout == LAYOUT_AOS else (self.ns, self.n))
        _check(lib().cep_batch_get_states(self._h, _dptr(out), layout))
        return out

    def set_states(self, states: np.ndarray, layout: int = LAYOUT_AOS):
        s = np.ascontiguousarray(states, np.float64)
        _check(lib().cep_batch_set_states(self._h, _dptr(s), layout))
        return self

    def device_states(self) -> tuple[int, int]:
        p = ctypes.c_void_p()
        ld = ctypes.c_long()
        _check(lib().cep_batch_device_states(self._h, ctypes.byref(p), ctypes.byref(ld)))
        return p.value, ld.value

    def biomarkers(self) -> dict[str, np.ndarray]:
        arr = (Biomarkers * self.n)()
        _check(lib().cep_batch_get_biomarkers(self._h, arr))
        raw = np.ctypeslib.as_array(arr)
        out = {f: np.array(raw[f]) for f in BM_FIELDS}
        for f in ("steepest_pace", "n_eligible", "status"):
            out[f] = np.array(raw[f])
        return out

    def biomarker_structs(self):
        arr = (Biomarkers * self.n)()
        _check(lib().cep_batch_get_biomarkers(self._h, arr))
        return arr

    def status(self) -> np.ndarray:
        out = np.zeros(self.n, np.int32)
        _check(lib().cep_batch_get_status(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def clock(self, i: int = 0) -> tuple[int, float]:
        s = ctypes.c_long()
        t = ctypes.c_double()
        _check(lib().cep_batch_get_clock(self._h, i, ctypes.byref(s), ctypes.byref(t)))
        return s.value, t.value

    def rates(self, t: float) -> tuple[np.ndarray, np.ndarray]:
        dv = np.zeros(self.n)
        cur = np.zeros((7, self.n))
        _check(lib().cep_batch_rates(self._h, t, _dptr(dv), _dptr(cur)))
        return dv, cur

    def rates_all(self, t: float) -> np.ndarray:
        """The model's full RATES vector of every instance at its current
        state, [n, n_states]."""
        r = np.zeros((self.n, self.ns))
        _check(lib().cep_batch_rates_all(self._h, t, _dptr(r)))
        return r

    def restitution(self, bcls, n_pace: int, dt: float, steps_per_launch: int = 20000) -> dict[str, np.ndarray]:
        """Dynamic restitution (apdr_bench.cpp:103-232) of every instance: the
        recorded paces as arrays [n, records] keyed by APDR_FIELDS."""
        b = np.ascontiguousarray(bcls, np.float64)
        m = restitution_records(b, n_pace, dt)
        arr = (ApdrRecord * max(1, self.n * m))()
        cnt = ctypes.c_int()
        _check(lib().cep_batch_restitution(self._h, _dptr(b), len(b), int(n_pace), float(dt), int(steps_per_launch),
                                           arr, m, ctypes.byref(cnt)))
        if cnt.value != m:
            raise CepError(ERR_STATE, f"restitution produced {cnt.value} records per instance, expected {m}")
        raw = np.ctypeslib.as_array(arr)[: self.n * m].reshape(self.n, m)
        return {f: np.array(raw[f]) for f in APDR_FIELDS}

    def hrv(self, bcls, dt: float, dt_write: float = 1.0, num_pace1: int | None = None,
            steps_per_launch: int = 0) -> dict[str, np.ndarray]:
        """Heart-rate-variability pacing (CEPCell_NEO/modules/hrv_bench.cpp:
        146-343): one pace per entry of bcls (the bench appends 1000 ms to its
        interval file), the last 250 paces evaluated. Returns the printed
        beat of every instance keyed like biomarkers(), plus "bcl", the BCL
        printed with it. num_pace1 defaults to len(bcls)."""
        b = np.ascontiguousarray(bcls, np.float64)
        arr = (HrvRecord * self.n)()
        np1 = len(b) if num_pace1 is None else int(num_pace1)
        _check(lib().cep_batch_hrv(self._h, _dptr(b), len(b), float(dt), float(dt_write), np1,
                                   int(steps_per_launch), arr))
        raw = np.ctypeslib.as_array(arr)
        beat = raw["beat"]
        out = {f: np.array(beat[f]) for f in BM_FIELDS}
        for f in ("steepest_pace", "n_eligible", "status"):
            out[f] = np.array(beat[f])
        out["bcl"] = np.array(raw["bcl"])
        return out

    def clamp(self, v, t0: float, dt: float, current: str | int) -> np.ndarray:
        """Voltage-clamp replay (CEPPatch/benchpatch.cpp:83-100): V of every
        instance forced to v[k] before step k; returns the chosen channel
        current, [len(v), n]."""
        idx = CURRENTS.index(current) if isinstance(current, str) else int(current)
        vv = np.ascontiguousarray(v, np.float64)
        out = np.zeros((len(vv), self.n))
        _check(lib().cep_batch_clamp(self._h, _dptr(vv), len(vv), float(t0), float(dt), idx, _dptr(out)))
        return out


def restitution_records(bcls, n_pace: int, dt: float) -> int:
    """Recorded paces per instance of a restitution run: per BCL, the pace
    boundaries among iout = 1 .. (int)(n_pace*bcl/dt) + 1 minus the first two."""
    m = 0
    for bcl in np.asarray(bcls, np.float64):
        steps, imax = int(float(bcl) / dt), int((n_pace * float(bcl)) / dt)
        m += max(0, (imax + 1) // max(1, steps) - 2)
    return m


def apdr_bcls(bcl_init: float, bcl_end: float, bcl_decrement: float) -> list[float]:
    """The BCL list of apdr_bench.cpp:103,229-230: from bcl_init while
    bcl >= bcl_end, the decrement becoming 10 once bcl <= 300."""
    out, bcl, dec = [], float(bcl_init), float(bcl_decrement)
    while bcl >= bcl_end:
        out.append(bcl)
        if bcl <= 300.0:
            dec = 10.0
        bcl -= dec
    return out


def run_population(model: str, conc, hill, bcl: float, dt: float, n_pace: int, first_pace: int,
                   precision: str = "mixed", celltype=None, dutta: bool = False, quirks: bool = True,
                   dt_write: float = 1.0, refine_above_vm: float | None = -80.0,
                   steps_per_launch: int = 50000, amp_scale: float = 1.0,
                   states_init=None, scales=None, screen_paces: int = 1) -> dict[str, np.ndarray]:
    """A population run to the end of its protocol (the reference's bench loop
    for every instance, cep_population_run), returning the biomarker records.

    With precision "mixed" and refine_above_vm set, the instances whose
    diastolic Vm after screen_paces mixed paces is above refine_above_vm
    (drug-depolarised cells that do not repolarise: their 90 % level is
    crossed at ~0.1 mV/ms, so their APD90 moves by tenths of a ms under
    perturbations of 1e-5 and FP32 gates cannot hold it to 0.1 ms) run in
    FP64 from their initial state concurrently with the mixed population,
    and any instance whose record still shows such a diastolic Vm, an
    APD90 above 0.9 BCL or an intermittent rhythm (some evaluated beats
    without an action potential at the peak sample: the edge of 2:1 block)
    runs again in FP64
    afterwards; out["refined"] marks both (out["refined_how"]: 1
    concurrent, 2 afterwards). amp_scale multiplies the stimulus amplitude
    (CONSTANTS[amp] *= Stim_Amplitude, cipa_drug_bench.cpp:147);
    states_init, one state vector, replaces every instance's initial states
    after initConsts (Is_Using_Output, :149); scales maps SCALE keys to a
    factor (scalar or one per instance) applied after initConsts
    (CONSTANTS[GNa] *= gna_scale, :148)."""
    conc = np.ascontiguousarray(conc, np.float64)
    n = len(conc)
    hill = np.asarray(hill, np.float64)
    h = np.ascontiguousarray(np.broadcast_to(hill, (n, hill.shape[-1])) if hill.ndim == 1 else hill)
    ct = None if celltype is None else np.ascontiguousarray(np.broadcast_to(celltype, (n,)), np.float64)
    sc = None
    if scales:
        sc = np.ones((n, len(SCALE)))
        for g, f in scales.items():
            sc[:, SCALE[g]] = np.broadcast_to(np.asarray(f, np.float64), (n,))
    y0 = None if states_init is None else np.ascontiguousarray(np.asarray(states_init, np.float64).reshape(-1))
    flags = (FLAG_DUTTA if dutta else 0) | (FLAG_QUIRKS if quirks else 0)
    job = PopulationJob(MODELS[model], n, _dptr(ct), _dptr(conc), _dptr(h), h.shape[1], flags, bcl, amp_scale,
                        _dptr(sc), _dptr(y0), dt, dt_write, n_pace, first_pace, PREC[precision],
                        float("nan") if refine_above_vm is None else refine_above_vm, max(1, screen_paces),
                        steps_per_launch)
    arr = (Biomarkers * n)()
    how = np.zeros(n, np.int32)
    _check(lib().cep_population_run(ctypes.byref(job), arr, how.ctypes.data_as(_ip)))
    raw = np.ctypeslib.as_array(arr)
    out = {f: np.array(raw[f]) for f in BM_FIELDS}
    for f in ("steepest_pace", "n_eligible", "status"):
        out[f] = np.array(raw[f])
    out["refined"] = how > 0
    out["refined_how"] = how
    return out


def population_late_mask(records: dict, refine_above_vm: float, bcl: float, evaluated: int) -> np.ndarray:
    """Which mixed records run_population re-runs in FP64 after the run
    (cep_population_late_mask): a diastolic Vm not below refine_above_vm, an
    APD90 above 0.9 bcl, or an intermittent rhythm (0 < n_eligible <
    evaluated). records: a dict of arrays keyed like run_population's result
    (the fields a missing key stands for are 0)."""
    n = len(records["vm_valley"])
    if n == 0:
        return np.zeros(0, bool)
    arr = (Biomarkers * n)()
    raw = np.ctypeslib.as_array(arr)
    for f in BM_FIELDS + ("steepest_pace", "n_eligible", "status"):
        if f in records:
            raw[f] = np.asarray(records[f])
    mask = np.zeros(n, np.int32)
    _check(lib().cep_population_late_mask(ctypes.cast(arr, ctypes.c_void_p), n, refine_above_vm, bcl, evaluated,
                                          mask.ctypes.data_as(_ip)))
    return mask.astype(bool)


def qinward(control: Biomarkers, drug: Biomarkers) -> float:
    return float(lib().cep_qinward(ctypes.byref(control), ctypes.byref(drug)))


FEM_AUTO, FEM_CSR, FEM_ELL, FEM_STENCIL, FEM_CLASSED = -1, 0, 1, 2, 3
S2_NONE, S2_RESET, S2_ECTOPIC = 0, 1, 2


def _iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class Fem:
    """Monodomain diffusion operator A = M/dt + D K, B = M on the GPU with its
    Jacobi-PCG solver (Cfem, fem.cpp)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        n = ctypes.c_int()
        nnz = ctypes.c_long()
        fmt = ctypes.c_int()
        w = ctypes.c_int()
        _check(lib().cep_fem_info(self._h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(fmt), ctypes.byref(w)))
        self.n, self.nnz, self.ell_width = n.value, nnz.value, w.value

    @classmethod
    def grid(cls, dim: int, nx: int, ny: int, nz: int, h: float, dt: float, D, fmt: int = FEM_ELL,
             stream: int | None = None) -> "Fem":
        """D: scalar, per-element array [n_elem] or [n_elem, 3|6] tensors."""
        n_elem = (nx - 1) * (ny - 1) * ((nz - 1) if dim == 3 else 1)
        d = np.asarray(D, np.float64)
        if d.ndim == 0:
            d = np.full((n_elem, 1), float(d))
        elif d.ndim == 1:
            d = d.reshape(n_elem, 1)
        d = np.ascontiguousarray(d)
        hnd = ctypes.c_void_p()
        _check(lib().cep_fem_create_grid(dim, nx, ny, nz, h, dt, _dptr(d), d.shape[1], fmt, stream,
                                         ctypes.byref(hnd)))
        return cls(hnd)

    @classmethod
    def csr(cls, row_ptr, col_idx, a_val, b_val, dt: float, fmt: int = FEM_ELL, stream: int | None = None) -> "Fem":
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        av = np.ascontiguousarray(a_val, np.float64)
        bv = np.ascontiguousarray(b_val, np.float64)
        hnd = ctypes.c_void_p()
        _check(lib().cep_fem_create_csr(len(rp) - 1, _iptr(rp), _iptr(ci), _dptr(av), _dptr(bv), dt, fmt, stream,
                                        ctypes.byref(hnd)))
        return cls(hnd)

    @classmethod
    def tet(cls, xyz, conn, D, dt: float, fmt: int = FEM_ELL, stream: int | None = None) -> "Fem":
        """Operator of a P1 tetrahedral mesh: xyz [n, 3] cm, conn [e, 4] 0-based,
        D scalar, [e] or [e, 6] tensors; assembled on the device."""
        x = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
        c = np.ascontiguousarray(np.asarray(conn, np.int32).reshape(-1, 4))
        d = np.asarray(D, np.float64)
        d = np.ascontiguousarray(np.full((len(c), 1), float(d)) if d.ndim == 0 else d.reshape(len(c), -1))
        hnd = ctypes.c_void_p()
        _check(lib().cep_fem_create_tet(len(x), _dptr(x), len(c), _iptr(c), _dptr(d), d.shape[1], dt, fmt, stream,
                                        ctypes.byref(hnd)))
        return cls(hnd)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cep_fem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def format(self) -> int:
        fmt = ctypes.c_int()
        _check(lib().cep_fem_info(self._h, None, None, ctypes.byref(fmt), None))
        return fmt.value

    def set_format(self, fmt: int) -> "Fem":
        _check(lib().cep_fem_set_format(self._h, fmt))
        return self

    def get_csr(self):
        rp = np.zeros(self.n + 1, np.int32)
        ci = np.zeros(self.nnz, np.int32)
        av = np.zeros(self.nnz)
        bv = np.zeros(self.nnz)
        _check(lib().cep_fem_get_csr(self._h, _iptr(rp), _iptr(ci), _dptr(av), _dptr(bv)))
        return rp, ci, av, bv

    def set_solver(self, rtol: float = 1e-5, max_iter: int = 10000, precond_norm: bool = True) -> "Fem":
        _check(lib().cep_fem_set_solver(self._h, rtol, max_iter, int(precond_norm)))
        return self

    def spmv(self, x, which: str = "A") -> np.ndarray:
        xx = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.n)
        _check(lib().cep_fem_spmv(self._h, {"A": 0, "B": 1}[which], _dptr(xx), _dptr(y)))
        return y

    def solve(self, v) -> tuple[np.ndarray, int, float]:
        """One implicit step: returns (V, iterations, relative residual)."""
        vv = np.array(v, np.float64)
        it = ctypes.c_int()
        res = ctypes.c_double()
        _check(lib().cep_fem_solve(self._h, _dptr(vv), ctypes.byref(it), ctypes.byref(res)))
        return vv, it.value, res.value

    def stats(self) -> dict:
        li, nc = ctypes.c_int(), ctypes.c_int()
        tot, ns = ctypes.c_long(), ctypes.c_long()
        res = ctypes.c_double()
        _check(lib().cep_fem_stats(self._h, ctypes.byref(li), ctypes.byref(tot), ctypes.byref(ns), ctypes.byref(nc),
                                   ctypes.byref(res)))
        return {"last_iters": li.value, "total_iters": tot.value, "solves": ns.value, "not_converged": nc.value,
                "last_res": res.value}


class Tissue:
    """Godunov-split monodomain tissue: a Batch (one instance per node) and a
    Fem operator sharing one stream (Cheart, heart.cpp)."""

    def __init__(self, cells: Batch, fem: Fem, dt: float):
        self.cells, self.fem = cells, fem
        self.n = fem.n
        h = ctypes.c_void_p()
        _check(lib().cep_tissue_create(cells._h, fem._h, dt, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cep_tissue_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stimulus(self, mask, bcl: float, t_crt: float, dur: float, n_pace: int) -> "Tissue":
        m = np.ascontiguousarray(mask, np.uint8)
        _check(lib().cep_tissue_set_stimulus(self._h, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), bcl, t_crt,
                                             dur, n_pace))
        return self

    def set_electrodes(self, xyz, every: int = 1, max_records: int = 10000) -> "Tissue":
        """Record the pseudo-ECG at electrodes xyz [n_el, 3] (cm) every
        `every` steps (at most max_records records)."""
        e = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
        self._n_el = e.shape[0]
        _check(lib().cep_tissue_set_electrodes(self._h, self._n_el, _dptr(e), int(every), int(max_records)))
        return self

    def set_s2(self, kind: int, target: int, vm_threshold: float, region=None, ectopic_dur: float = 0.0) -> "Tissue":
        """Arm the S1-S2 reset (S2_RESET) or ectopic (S2_ECTOPIC) protocol on
        region [n] monitored at node `target`; S2_NONE disarms."""
        m = None
        if region is not None:
            m = np.ascontiguousarray(np.asarray(region, np.uint8).ravel())
        _check(lib().cep_tissue_set_s2(self._h, int(kind), int(target), float(vm_threshold),
                                       None if m is None else m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                       float(ectopic_dur)))
        self._s2_region = m
        return self

    def ecg(self) -> np.ndarray:
        """Pseudo-ECG records so far, [n_records, n_el]."""
        n = ctypes.c_long()
        _check(lib().cep_tissue_get_ecg(self._h, None, ctypes.byref(n)))
        out = np.empty((n.value, getattr(self, "_n_el", 0)))
        if n.value:
            _check(lib().cep_tissue_get_ecg(self._h, _dptr(out), ctypes.byref(n)))
        return out

    def set_activation_threshold(self, vm: float) -> "Tissue":
        _check(lib().cep_tissue_set_activation_threshold(self._h, vm))
        return self

    def set_clock(self, time: float) -> "Tissue":
        """Resume at `time` ms (node states loaded through the cells' batch)."""
        _check(lib().cep_tissue_set_clock(self._h, float(time)))
        return self

    def run(self, n_steps: int) -> "Tissue":
        _check(lib().cep_tissue_run(self._h, int(n_steps)))
        return self

    def sync(self) -> "Tissue":
        _check(lib().cep_tissue_sync(self._h))
        return self

    def v(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().cep_tissue_get_v(self._h, _dptr(out)))
        return out

    def activation(self) -> np.ndarray:
        out = np.zeros(self.n)
        _check(lib().cep_tissue_get_activation(self._h, _dptr(out)))
        return out

    def stats(self) -> dict:
        t = ctypes.c_double()
        st, it = ctypes.c_long(), ctypes.c_long()
        nc = ctypes.c_int()
        _check(lib().cep_tissue_stats(self._h, ctypes.byref(t), ctypes.byref(st), ctypes.byref(it), ctypes.byref(nc)))
        return {"time": t.value, "steps": st.value, "cg_iters": it.value, "not_converged": nc.value}


class Server:
    """Screening-job server with continuous batching (one resident pool)."""

    def __init__(self, model: str, precision: str = "mixed", capacity: int = 0, dt: float = 0.005,
                 dt_write: float = 1.0, max_bcl: float = 2000.0, steps_per_launch: int = 10000,
                 hbm_fraction: float = 0.8, stream: int | None = None):
        h = ctypes.c_void_p()
        _check(lib().cep_serve_start(MODELS[model], PREC[precision], capacity, dt, dt_write, max_bcl,
                                     steps_per_launch, hbm_fraction, stream, ctypes.byref(h)))
        self._h = h
        self.model = model
        self._n = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cep_serve_stop(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, conc, hill=None, bcl: float = 1000.0, n_pace: int = 1, first_pace: int = 0,
               celltype=None, quirks: bool = True, dutta: bool = False) -> int:
        cc = np.ascontiguousarray(conc, np.float64)
        n = len(cc)
        hh = None
        if hill is not None:
            hh = np.asarray(hill, np.float64)
            hh = np.ascontiguousarray(np.broadcast_to(hh, (n, hh.shape[-1])))
        ct = None if celltype is None else np.ascontiguousarray(np.broadcast_to(celltype, (n,)), np.float64)
        job = CepJob(n, _dptr(ct), _dptr(cc), _dptr(hh), 0 if hh is None else hh.shape[1], bcl, n_pace, first_pace,
                     (FLAG_QUIRKS if quirks else 0) | (FLAG_DUTTA if dutta else 0))
        jid = ctypes.c_uint64()
        _check(lib().cep_serve_submit(self._h, ctypes.byref(job), ctypes.byref(jid)))
        self._n[jid.value] = n
        return jid.value

    def submit_tissue(self, nx: int, ny: int, duration: float, conc: float = 0.0, hill=None, h: float = 0.025,
                      D: float = 0.0013, dt: float = 0.01, bcl: float = 1000.0, stim=(2, 2),
                      rtol: float = 1e-8) -> int:
        """A 2D TT2006 patch job (corner S1 block of stim = (nx, ny) nodes)."""
        hh = None if hill is None else np.ascontiguousarray(np.asarray(hill, np.float64)[:14])
        job = TissueJob(nx, ny, h, D, dt, duration, conc, _dptr(hh), bcl, stim[0], stim[1], rtol)
        jid = ctypes.c_uint64()
        _check(lib().cep_serve_submit_tissue(self._h, ctypes.byref(job), ctypes.byref(jid)))
        self._n[jid.value] = nx * ny
        return jid.value

    def tissue_result(self, jid: int) -> tuple[np.ndarray, np.ndarray, dict]:
        """Final V, activation times (-1: never) and timings of a patch job."""
        n = self._n[jid]
        v = np.empty(n)
        ta = np.empty(n)
        t = JobTimes()
        _check(lib().cep_serve_tissue_result(self._h, jid, _dptr(v), _dptr(ta), ctypes.byref(t)))
        return v, ta, {k: getattr(t, k) for k, _ in JobTimes._fields_}

    def poll(self, jid: int) -> int:
        st = ctypes.c_int()
        _check(lib().cep_serve_poll(self._h, jid, ctypes.byref(st)))
        return st.value

    def wait(self, jid: int, timeout_s: float = 0.0) -> None:
        _check(lib().cep_serve_wait(self._h, jid, timeout_s))

    def result(self, jid: int) -> tuple[dict, dict]:
        n = self._n[jid]
        arr = (Biomarkers * n)()
        t = JobTimes()
        _check(lib().cep_serve_result(self._h, jid, arr, ctypes.byref(t)))
        raw = np.ctypeslib.as_array(arr)
        out = {f: np.array(raw[f]) for f in BM_FIELDS}
        for f in ("steepest_pace", "n_eligible", "status"):
            out[f] = np.array(raw[f])
        return out, {k: getattr(t, k) for k, _ in JobTimes._fields_}

    def release(self, jid: int) -> None:
        _check(lib().cep_serve_release(self._h, jid))
        self._n.pop(jid, None)

    def cancel(self, jid: int) -> None:
        """Queued: leaves at once; running: leaves between two launches."""
        _check(lib().cep_serve_cancel(self._h, jid))

    def stats(self) -> dict:
        st = ServeStats()
        _check(lib().cep_serve_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}


class TissueGroup:
    """Tissues stepped together with one batched diffusion solve per step."""

    def __init__(self, tissues):
        self.tissues = list(tissues)
        arr = (ctypes.c_void_p * len(self.tissues))(*[t._h.value for t in self.tissues])
        h = ctypes.c_void_p()
        _check(lib().cep_tissue_group_create(arr, len(self.tissues), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cep_tissue_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n_steps: int) -> "TissueGroup":
        _check(lib().cep_tissue_group_run(self._h, int(n_steps)))
        return self

    def set_timing(self, on: bool = True) -> "TissueGroup":
        """Bracket each step's ionic and diffusion launches with CUDA events
        (resets the totals)."""
        _check(lib().cep_tissue_group_set_timing(self._h, int(bool(on))))
        return self

    def timing(self) -> dict:
        """Device milliseconds spent in the ionic and diffusion phases since
        set_timing, and the steps they cover (waits for them)."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_long()
        _check(lib().cep_tissue_group_timing(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)))
        return {"ionic_ms": a.value, "diffusion_ms": b.value, "steps": n.value}
