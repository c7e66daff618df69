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
INST_RUNNING, INST_DONE, INST_NONFINITE = 0, 1, 2
MODELS = {"ord2011": 0, "cipa2017": 1, "tt2006": 2, "tt2004": 3, "tomek2019": 4}
N_STATES = {"ord2011": 41, "cipa2017": 49, "tt2006": 19, "tt2004": 17, "tomek2019": 43}
PREC = {"fp64": 0, "mixed": 1}
FLAG_DUTTA, FLAG_QUIRKS = 1, 2
LAYOUT_SOA, LAYOUT_AOS = 0, 1
HILL_WIDTH = 20

BM_FIELDS = ("qnet", "inal_auc", "ical_auc", "dvmdt_repol", "dvmdt_max", "vm_peak", "vm_valley", "vm_dia",
             "apd90", "apd50", "apd_tri", "ca_peak", "ca_valley", "ca_dia", "cad90", "cad50", "cad_tri")


class Biomarkers(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in BM_FIELDS] + [
        ("steepest_pace", ctypes.c_int32), ("n_eligible", ctypes.c_int32), ("status", ctypes.c_int32),
        ("reserved", ctypes.c_int32)]


class CepError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cep error {code}: {msg}")
        self.code = code


_dp = ctypes.POINTER(ctypes.c_double)
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
    "cep_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
    "cep_batch_run_to_end": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_long]),
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
    "cep_qinward": (ctypes.c_double, [ctypes.POINTER(Biomarkers), ctypes.POINTER(Biomarkers)]),
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

    def init(self, celltype=None, conc=None, hill=None, dutta: bool = False, quirks: bool = True) -> "Batch":
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
        flags = (FLAG_DUTTA if dutta else 0) | (FLAG_QUIRKS if quirks else 0)
        _check(lib().cep_batch_init(self._h, _dptr(ct), _dptr(cc), _dptr(hh), stride, flags))
        return self

    def set_pacing(self, bcl: float, stim_start: float = -1.0, stim_dur: float = -1.0, amp_scale: float = 1.0):
        _check(lib().cep_batch_set_pacing(self._h, bcl, stim_start, stim_dur, amp_scale))
        return self

    def set_protocol(self, dt: float, n_pace: int, first_pace: int = -1, dt_write: float = 1.0,
                     qnet_vm_threshold: float = -1e300):
        _check(lib().cep_batch_set_protocol(self._h, dt, n_pace, first_pace, dt_write, qnet_vm_threshold))
        return self

    def set_block(self, threads: int):
        _check(lib().cep_batch_set_block(self._h, threads))
        return self

    def set_kernel(self, variant: str):
        """'cell' (one thread per cell) or 'roles' (4 warps per 32 cells)."""
        _check(lib().cep_batch_set_kernel(self._h, {"cell": 0, "roles": 1}[variant]))
        return self

    def run(self, n_steps: int):
        _check(lib().cep_batch_run(self._h, int(n_steps)))
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


def qinward(control: Biomarkers, drug: Biomarkers) -> float:
    return float(lib().cep_qinward(ctypes.byref(control), ctypes.byref(drug)))
