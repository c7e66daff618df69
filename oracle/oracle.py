"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle and to the
reference cell models compiled from their own sources.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only as the checker. The product library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libcep_oracle.so"
REF_DIR = HERE / "_ref"

MODELS = {"ord2011": 0, "cipa2017": 1, "tt2006": 2, "tt2004": 3, "tomek2019": 4}
N_STATES = {"ord2011": 41, "cipa2017": 49, "tt2006": 19, "tt2004": 17, "tomek2019": 43}
REF_LIBS = {
    "ord2011": "libref_ord2011.so",
    "ord2011_tissue": "libref_ord2011_tissue.so",
    "cipa2017": "libref_cipa2017.so",
    "tt2006": "libref_tt2006_epi.so",
    "tt2006_tissue": "libref_tt2006_epi_tissue.so",
    "tt2004": "libref_tt2004b.so",
    "tomek2019": "libref_tomek2019.so",
    "fem": "libref_fem.so",
    "ord2011_neo": "libref_ord2011_neo.so",
    "bench": "libref_bench.so",
}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(quiet: bool = True) -> None:
    """Compile the oracle (and, where the reference tree exists, the
    reference models) with the committed Makefile."""
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


class CepoCell(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("quirks", ctypes.c_int), ("tissue_stim", ctypes.c_int),
                ("is_s1", ctypes.c_int), ("p", ctypes.c_double * 256)]


class CepoCurrents(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("INa", "INaL", "Ito", "ICaL", "IKr", "IKs", "IK1", "dVdt")]


BEAT_FIELDS = ("qnet", "inal_auc", "ical_auc", "dvmdt_repol", "dvmdt_max", "vm_peak", "vm_valley",
               "vm_dia", "apd90", "apd50", "ca_peak", "ca_valley", "ca_dia", "cad90", "cad50")


class CepoBeat(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in BEAT_FIELDS]


class CepoHrvRecord(ctypes.Structure):
    _fields_ = [("beat", CepoBeat), ("bcl", ctypes.c_int), ("steepest_pace", ctypes.c_int)]


class CepoBiomarkers(ctypes.Structure):
    _fields_ = [("result", CepoBeat), ("steepest_pace", ctypes.c_int), ("n_eligible", ctypes.c_int),
                ("qnet_last", ctypes.c_double), ("status", ctypes.c_int)]


class CepoApdrRecord(ctypes.Structure):
    _fields_ = [("pace", ctypes.c_int), ("recal", ctypes.c_int), ("bcl", ctypes.c_double),
                ("apd90", ctypes.c_double), ("di", ctypes.c_double), ("t", ctypes.c_double)]


APDR_FIELDS = ("pace", "recal", "bcl", "apd90", "di", "t")

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        L = ctypes.CDLL(str(ORACLE_SO))
        L.cepo_init.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.cepo_init_states.argtypes = [ctypes.POINTER(CepoCell), _dp]
        L.cepo_set_pacing.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double]
        L.cepo_step.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_double, ctypes.c_double, _dp,
                                ctypes.POINTER(CepoCurrents)]
        L.cepo_rates.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_double, _dp, _dp,
                                 ctypes.POINTER(CepoCurrents)]
        L.cepo_run.argtypes = [ctypes.POINTER(CepoCell), _dp, ctypes.c_double, ctypes.c_long, _dp, _dp,
                               ctypes.c_long]
        L.cepo_run_biomarkers.argtypes = [ctypes.POINTER(CepoCell), _dp, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(CepoBiomarkers), _dp, ctypes.c_long, ctypes.c_long]
        L.cepo_run_batch.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_long, _dp,
                                     ctypes.c_int]
        L.cepo_run_batch.restype = ctypes.c_int
        L.cepo_restitution.argtypes = [ctypes.POINTER(CepoCell), _dp, _dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.POINTER(CepoApdrRecord), ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int)]
        L.cepo_restitution.restype = ctypes.c_int
        L.cepo_clamp.argtypes = [ctypes.POINTER(CepoCell), _dp, _dp, ctypes.c_long, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, _dp]
        L.cepo_tt04_mcell.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_double, _dp]
        _ip = ctypes.POINTER(ctypes.c_int)
        L.cepo_fem_nnz.argtypes = [ctypes.c_int] * 4
        L.cepo_fem_nnz.restype = ctypes.c_long
        L.cepo_fem_assemble.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, _dp, ctypes.c_int, _ip, _ip, _dp, _dp]
        L.cepo_scale.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_int, ctypes.c_double]
        L.cepo_ord_set_cumm.argtypes = [ctypes.POINTER(CepoCell), ctypes.c_double]
        L.cepo_hrv_run.argtypes = [ctypes.POINTER(CepoCell), _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, ctypes.POINTER(CepoHrvRecord)]
        L.cepo_fem_element.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int, _dp, _dp]
        L.cepo_element.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.cepo_pseudo_ecg.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp,
                                      ctypes.c_int, _dp, ctypes.c_int, _dp, _dp]
        L.cepo_spmv.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, _dp]
        L.cepo_pcg2.argtypes = [ctypes.c_int, _ip, _ip, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                _dp]
        L.cepo_pcg2.restype = ctypes.c_int
        L.cepo_tissue_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_long,
                                      ctypes.POINTER(ctypes.c_uint8), ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_int, _dp, _dp, _ip, ctypes.c_double, _dp]
        L.cepo_tissue_run.restype = ctypes.c_long
        L.cepo_tissue_run_s2.argtypes = L.cepo_tissue_run.argtypes + [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                                      ctypes.POINTER(ctypes.c_uint8), ctypes.c_double]
        L.cepo_tissue_run_s2.restype = ctypes.c_long
        L.cepo_tissue_run_csr.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _dp, ctypes.c_double,
                                          ctypes.c_long, ctypes.POINTER(ctypes.c_uint8), ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp, _ip,
                                          ctypes.c_double, _dp]
        L.cepo_tissue_run_csr.restype = ctypes.c_long
        L.cepo_fem_assemble_tet.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _dp, ctypes.c_int, ctypes.c_double,
                                            _ip, _ip, _dp, _dp]
        L.cepo_fem_assemble_tet.restype = ctypes.c_long
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Cell:
    """One oracle cell instance."""

    def __init__(self, model: str, celltype: float = 0.0, conc: float = 0.0, hill=None,
                 is_dutta: bool = False, quirks: bool = True, tissue_stim: bool = False, mcell: bool = False):
        self.model = model
        self.c = CepoCell()
        h = None if hill is None else np.ascontiguousarray(hill, dtype=np.float64)
        rc = lib().cepo_init(ctypes.byref(self.c), MODELS[model], float(celltype), float(conc),
                             _ptr(h), 0 if h is None else len(h), int(is_dutta), int(quirks))
        if rc != 0:
            raise RuntimeError(f"oracle init failed for {model}: {rc}")
        if mcell:
            if model != "tt2004":
                raise ValueError("mcell is the TT2004 2004_a variant")
            lib().cepo_tt04_mcell(ctypes.byref(self.c), float(conc), _ptr(h))
        self.c.tissue_stim = int(tissue_stim)
        self.y = np.zeros(64)
        lib().cepo_init_states(ctypes.byref(self.c), _ptr(self.y))

    @property
    def n(self) -> int:
        return N_STATES[self.model]

    @property
    def states(self) -> np.ndarray:
        return self.y[: self.n]

    def set_pacing(self, bcl: float, stim_start: float = -1.0, stim_dur: float = -1.0, amp_scale: float = 1.0):
        lib().cepo_set_pacing(ctypes.byref(self.c), bcl, stim_start, stim_dur, amp_scale)

    def scale(self, conductance: int, factor: float):
        """CONSTANTS[x] *= factor (conductance numbered as CEP_SCALE_*)."""
        if lib().cepo_scale(ctypes.byref(self.c), int(conductance), float(factor)) != 0:
            raise ValueError(f"{self.model} has no scalable conductance {conductance}")

    def step(self, t: float, dt: float) -> CepoCurrents:
        cur = CepoCurrents()
        lib().cepo_step(ctypes.byref(self.c), t, dt, _ptr(self.y), ctypes.byref(cur))
        return cur

    def rates(self, t: float) -> tuple[np.ndarray, CepoCurrents]:
        r = np.zeros(64)
        cur = CepoCurrents()
        lib().cepo_rates(ctypes.byref(self.c), t, _ptr(self.y), _ptr(r), ctypes.byref(cur))
        return r[: self.n], cur

    def run(self, t0: float, dt: float, n_steps: int, v_stride: int = 0):
        t = ctypes.c_double(t0)
        vt = np.zeros(max(1, n_steps // v_stride) if v_stride else 1)
        lib().cepo_run(ctypes.byref(self.c), ctypes.byref(t), dt, n_steps, _ptr(self.y),
                       _ptr(vt) if v_stride else None, v_stride)
        return t.value, (vt if v_stride else None)

    def run_biomarkers(self, dt: float, n_pace: int, first_pace: int, dt_write: float = 1.0,
                       qnet_vm_threshold: float = -1e300, v_stride: int = 0, v_cap: int = 0):
        bm = CepoBiomarkers()
        vt = np.zeros(max(1, v_cap))
        lib().cepo_run_biomarkers(ctypes.byref(self.c), _ptr(self.y), dt, n_pace, first_pace, dt_write,
                                  qnet_vm_threshold, ctypes.byref(bm), _ptr(vt) if v_stride else None,
                                  v_stride, v_cap)
        out = {f: getattr(bm.result, f) for f in BEAT_FIELDS}
        out.update(steepest_pace=bm.steepest_pace, n_eligible=bm.n_eligible, status=bm.status)
        return out, (vt if v_stride else None)


    def hrv(self, bcls, dt: float, dt_write: float = 1.0, num_pace1: int | None = None) -> dict:
        """hrv_bench.cpp:146-343 on the fixed-step scheme (ORd 2011, the
        CEPCell_NEO build: quirks=2): one pace per BCL. Returns the printed
        record's fields (the chosen beat, its BCL and pace)."""
        b = np.ascontiguousarray(bcls, dtype=np.float64)
        rec = CepoHrvRecord()
        st = lib().cepo_hrv_run(ctypes.byref(self.c), _ptr(self.y), _ptr(b), len(b), float(dt), float(dt_write),
                                int(len(b) if num_pace1 is None else num_pace1), ctypes.byref(rec))
        out = {f: getattr(rec.beat, f) for f in BEAT_FIELDS}
        out.update(bcl=rec.bcl, steepest_pace=rec.steepest_pace, status=st)
        return out

    def restitution(self, bcls, n_pace: int, dt: float, max_records: int = 100000):
        """apdr_bench.cpp:103-232 on the fixed-step scheme; returns (records as a
        dict of arrays, status)."""
        b = np.ascontiguousarray(bcls, dtype=np.float64)
        recs = (CepoApdrRecord * max_records)()
        n = ctypes.c_int(0)
        st = lib().cepo_restitution(ctypes.byref(self.c), _ptr(self.y), _ptr(b), len(b), int(n_pace), float(dt),
                                    recs, max_records, ctypes.byref(n))
        k = min(n.value, max_records)
        out = {f: np.array([getattr(recs[j], f) for j in range(k)]) for f in APDR_FIELDS}
        return out, st

    def clamp(self, v, t0: float, dt: float, current: int) -> np.ndarray:
        """CEPPatch/benchpatch.cpp:83-100: V forced to v[k] before step k."""
        vv = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros(len(vv))
        lib().cepo_clamp(ctypes.byref(self.c), _ptr(self.y), _ptr(vv), len(vv), float(t0), float(dt), int(current),
                         _ptr(out))
        return out


def apdr_bcls(bcl_init: float, bcl_end: float, bcl_decrement: float) -> list[float]:
    """BCL list of apdr_bench.cpp:103,229-230: from bcl_init while bcl >= bcl_end,
    the decrement becoming 10 once bcl <= 300."""
    out, bcl, dec = [], float(bcl_init), float(bcl_decrement)
    while bcl >= bcl_end:
        out.append(bcl)
        if bcl <= 300.0:
            dec = 10.0
        bcl -= dec
    return out


def run_batch(model: str, celltype, conc, hill, bcl: float, dt: float, n_steps: int,
              is_dutta: bool = False, quirks: bool = True, n_threads: int = 1):
    """Threaded fixed-step run over a batch (the CPU baseline)."""
    n = len(conc)
    ct = np.ascontiguousarray(celltype, dtype=np.float64)
    cc = np.ascontiguousarray(conc, dtype=np.float64)
    hh = np.ascontiguousarray(hill, dtype=np.float64)
    out = np.zeros((n, N_STATES[model]))
    used = lib().cepo_run_batch(MODELS[model], n, _ptr(ct), _ptr(cc), _ptr(hh), hh.shape[1], int(is_dutta),
                                int(quirks), bcl, dt, n_steps, _ptr(out), n_threads)
    return out, used


class RefCell:
    """The reference model object compiled from its own sources."""

    def __init__(self, key: str, celltype: float = 0.0, conc: float = 0.0, hill=None, is_dutta: bool = False):
        path = REF_DIR / REF_LIBS[key]
        if not path.exists():
            raise FileNotFoundError(path)
        L = ctypes.CDLL(str(path))
        L.ref_new.restype = ctypes.c_void_p
        for f in ("ref_states", "ref_consts", "ref_rates", "ref_alg"):
            getattr(L, f).restype = _dp
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.ref_init.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int]
        L.ref_run.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_long, _dp, ctypes.c_long]
        L.ref_compute_rates.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_solve.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ref_set_s1.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_set_ectopic.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_sizes.argtypes = [ctypes.c_void_p, _ip, _ip, _ip]
        L.ref_free.argtypes = [ctypes.c_void_p]
        self.L = L
        self.h = L.ref_new()
        self._hill = np.zeros(32) if hill is None else np.concatenate([np.asarray(hill, float), np.zeros(32)])
        L.ref_init(self.h, float(celltype), float(conc), _ptr(self._hill), int(is_dutta))
        ns, nc, na = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.ref_sizes(self.h, ctypes.byref(ns), ctypes.byref(nc), ctypes.byref(na))
        self.n, self.nc, self.na = ns.value, nc.value, na.value
        L.ref_set_s1(self.h, 0)
        L.ref_set_ectopic(self.h, 0)

    def __del__(self):
        try:
            self.L.ref_free(self.h)
        except Exception:
            pass

    def arr(self, which: str, n: int) -> np.ndarray:
        p = getattr(self.L, "ref_" + which)(self.h)
        return np.ctypeslib.as_array(p, shape=(n,))

    @property
    def states(self) -> np.ndarray:
        return self.arr("states", self.n)

    @property
    def consts(self) -> np.ndarray:
        return self.arr("consts", self.nc)

    def run(self, t0: float, dt: float, n_steps: int, v_stride: int = 0):
        t = ctypes.c_double(t0)
        vt = np.zeros(max(1, n_steps // v_stride) if v_stride else 1)
        self.L.ref_run(self.h, ctypes.byref(t), dt, n_steps, _ptr(vt) if v_stride else None, v_stride)
        return t.value, (vt if v_stride else None)


def ref_available(key: str) -> bool:
    return (REF_DIR / REF_LIBS[key]).exists()


def ref_cipa_bench(workdir: str, hill_rows, concs, celltype: float, bcl: float, dt: float, dt_write: float,
                   num_pace: int, drug: str = "pin") -> dict:
    """The reference's CiPA drug bench (cipa_drug_bench.cpp, compiled from
    its sources over the oracle's ORd; ref_shim/bench_shim.cpp) for every
    Hill row and concentration. Returns {conc_text: {"ap": [...], "ca":
    [...], "qni": [...]}}, each a list of rows of the printed text fields."""
    import tempfile
    import zipfile
    L = ctypes.CDLL(str(REF_DIR / REF_LIBS["bench"]))
    L.ref_cipa_bench.argtypes = [ctypes.c_char_p] * 4 + [ctypes.c_double] * 4 + [ctypes.c_int]
    wd = Path(workdir)
    (wd / "result").mkdir(parents=True, exist_ok=True)
    hill_path = wd / "hill.csv"
    rows = np.atleast_2d(np.asarray(hill_rows, np.float64))
    hill_path.write_text("header\n" + "".join(",".join(repr(float(x)) for x in r) + "\n" for r in rows))
    conc_text = "0," + ",".join(repr(float(c)) for c in concs)
    if L.ref_cipa_bench(str(wd).encode(), str(hill_path).encode(), conc_text.encode(), drug.encode(), celltype, bcl,
                        dt, dt_write, num_pace) != 0:
        raise RuntimeError("reference bench failed")
    z = zipfile.ZipFile(sorted((wd / "result").glob("*.zip"))[-1])
    out: dict = {}
    for name in z.namelist():
        parts = name.split("/")
        kind = "ap" if "ap_profile" in name else "ca" if "ca_profile" in name else "qni" if "qni" in name else None
        if kind is None:
            continue
        lines = z.read(name).decode().strip().splitlines()[1:]
        out.setdefault(parts[1], {})[kind] = [ln.split() for ln in lines]
    return out


def ref_fem_element(kind: str, xy, de: float, dt: float) -> tuple[np.ndarray, np.ndarray]:
    """The reference's own element matrices (Cfem::set_amat_bmat, fem.cpp:
    628-661, compiled from fem.cpp) of one square, hex or tet element with
    node coordinates xy[nn][dim] and scalar conductivity de."""
    L = ctypes.CDLL(str(REF_DIR / REF_LIBS["fem"]))
    L.ref_fem_element.argtypes = [ctypes.c_char_p, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
    x = np.ascontiguousarray(xy, np.float64)
    nn = len(x)
    ae = np.zeros(nn * nn)
    be = np.zeros(nn * nn)
    if L.ref_fem_element(kind.encode(), _ptr(x), de, dt, _ptr(ae), _ptr(be)) != 0:
        raise ValueError(kind)
    return ae.reshape(nn, nn), be.reshape(nn, nn)


# ------------------------------------------------------------------ FEM
_ip = ctypes.POINTER(ctypes.c_int)


def _iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def element_D(dim: int, nx: int, ny: int, nz: int, D) -> np.ndarray:
    n_elem = (nx - 1) * (ny - 1) * ((nz - 1) if dim == 3 else 1)
    d = np.asarray(D, np.float64)
    if d.ndim == 0:
        d = np.full((n_elem, 1), float(d))
    elif d.ndim == 1:
        d = d.reshape(n_elem, 1)
    return np.ascontiguousarray(d)


def fem_assemble(dim: int, nx: int, ny: int, nz: int, h: float, dt: float, D):
    """CSR (row_ptr, col, A, B) of the structured-grid operator."""
    if dim == 2:
        nz = 1
    d = element_D(dim, nx, ny, nz, D)
    n = nx * ny * nz
    nnz = lib().cepo_fem_nnz(dim, nx, ny, nz)
    rp = np.zeros(n + 1, np.int32)
    ci = np.zeros(nnz, np.int32)
    av = np.zeros(nnz)
    bv = np.zeros(nnz)
    lib().cepo_fem_assemble(dim, nx, ny, nz, h, dt, _ptr(d), d.shape[1], _iptr(rp), _iptr(ci), _ptr(av), _ptr(bv))
    return rp, ci, av, bv


def fem_assemble_tet(xyz, conn, D, dt: float):
    """CSR (row_ptr, col, A, B) of a P1 tetrahedral mesh (D: scalar, [n_elem] or [n_elem, 6])."""
    x = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    c = np.ascontiguousarray(np.asarray(conn, np.int32).reshape(-1, 4))
    d = np.asarray(D, np.float64)
    d = np.ascontiguousarray(np.full((len(c), 1), float(d)) if d.ndim == 0 else d.reshape(len(c), -1))
    n = len(x)
    rp = np.zeros(n + 1, np.int32)
    nnz = lib().cepo_fem_assemble_tet(n, _ptr(x), len(c), _iptr(c), _ptr(d), d.shape[1], dt, _iptr(rp), None, None,
                                      None)
    ci = np.zeros(nnz, np.int32)
    av = np.zeros(nnz)
    bv = np.zeros(nnz)
    lib().cepo_fem_assemble_tet(n, _ptr(x), len(c), _iptr(c), _ptr(d), d.shape[1], dt, _iptr(rp), _iptr(ci), _ptr(av),
                                _ptr(bv))
    return rp, ci, av, bv


def tissue_run_csr(model: str, rp, ci, a_val, b_val, dt: float, n_steps: int, s1_mask, bcl: float, t_crt: float,
                   dur: float, n_pace: int, conc: float = 0.0, hill=None, rtol: float = 1e-5,
                   precond_norm: bool = True, celltype=None, act_thr: float = -30.0):
    """Godunov tissue run on a CSR operator: (final V, CG iterations per step, activation times)."""
    n = len(rp) - 1
    m = np.ascontiguousarray(s1_mask, np.uint8)
    hh = None if hill is None else np.ascontiguousarray(hill, np.float64)
    ct = None if celltype is None else np.ascontiguousarray(celltype, np.float64)
    v = np.zeros(n)
    its = np.zeros(n_steps, np.int32)
    tact = np.zeros(n)
    lib().cepo_tissue_run_csr(MODELS[model], n, _iptr(np.ascontiguousarray(rp, np.int32)),
                              _iptr(np.ascontiguousarray(ci, np.int32)), _ptr(np.ascontiguousarray(a_val)),
                              _ptr(np.ascontiguousarray(b_val)), dt, n_steps,
                              m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), bcl, t_crt, dur, n_pace, conc,
                              _ptr(hh) if hh is not None else None, 0 if hh is None else len(hh), rtol,
                              int(precond_norm), _ptr(ct) if ct is not None else None, _ptr(v), _iptr(its), act_thr,
                              _ptr(tact))
    return v, its, tact


def pseudo_ecg(dim: int, nx: int, ny: int, nz: int, h: float, D, V, xyz) -> np.ndarray:
    """Pseudo-ECG of a grid tissue's V at electrodes xyz [n_el, 3] (cm)."""
    if dim == 2:
        nz = 1
    d = element_D(dim, nx, ny, nz, D)
    e = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    vv = np.ascontiguousarray(V, np.float64)
    out = np.zeros(e.shape[0])
    lib().cepo_pseudo_ecg(dim, nx, ny, nz, h, _ptr(d), d.shape[1], _ptr(vv), e.shape[0], _ptr(e), _ptr(out))
    return out


def fem_element(dim: int, h: float, dt: float, D) -> tuple[np.ndarray, np.ndarray]:
    d = np.ascontiguousarray(np.atleast_1d(np.asarray(D, np.float64)))
    nn = 4 if dim == 2 else 8
    ae = np.zeros(nn * nn)
    be = np.zeros(nn * nn)
    lib().cepo_fem_element(dim, h, dt, _ptr(d), len(d), _ptr(ae), _ptr(be))
    return ae.reshape(nn, nn), be.reshape(nn, nn)


def element(kind: str, xy, D, dt: float) -> tuple[np.ndarray, np.ndarray]:
    """Element matrices (A = M/dt + D K, B = M) of one square, hex or tet
    element with node coordinates xy[nn][dim]."""
    x = np.ascontiguousarray(xy, np.float64)
    d = np.ascontiguousarray(np.atleast_1d(np.asarray(D, np.float64)))
    nn = len(x)
    ae = np.zeros(nn * nn)
    be = np.zeros(nn * nn)
    lib().cepo_element({"square": 0, "hex": 1, "tet": 2}[kind], _ptr(x), _ptr(d), len(d), dt, _ptr(ae), _ptr(be))
    return ae.reshape(nn, nn), be.reshape(nn, nn)


def spmv(rp, ci, val, x) -> np.ndarray:
    xx = np.ascontiguousarray(x, np.float64)
    y = np.zeros(len(rp) - 1)
    lib().cepo_spmv(len(rp) - 1, _iptr(rp), _iptr(ci), _ptr(np.ascontiguousarray(val)), _ptr(xx), _ptr(y))
    return y


def pcg(rp, ci, a_val, b, rtol: float, max_iter: int = 10000, precond_norm: bool = True):
    """Jacobi-PCG from x = 0: (x, iterations (negative if not converged), rel. residual)."""
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(len(rp) - 1)
    res = ctypes.c_double()
    it = lib().cepo_pcg2(len(rp) - 1, _iptr(rp), _iptr(ci), _ptr(np.ascontiguousarray(a_val)), _ptr(bb), _ptr(x),
                         rtol, max_iter, int(precond_norm), ctypes.byref(res))
    return x, it, res.value


def tissue_run(model: str, dim: int, nx: int, ny: int, nz: int, h: float, D, dt: float, n_steps: int, s1_mask,
               bcl: float, t_crt: float, dur: float, n_pace: int, conc: float = 0.0, hill=None,
               rtol: float = 1e-5, precond_norm: bool = True, celltype=None, act_thr: float = -30.0,
               s2_kind: int = 0, s2_target: int = 0, s2_thr: float = -45.0, s2_region=None, ecto_dur: float = 0.0):
    """Godunov-split tissue run: (final V, CG iterations per step, activation times); s2_kind 1/2 adds the
    S1-S2 reset / ectopic protocol on s2_region monitored at node s2_target."""
    if dim == 2:
        nz = 1
    d = element_D(dim, nx, ny, nz, D)
    n = nx * ny * nz
    m = np.ascontiguousarray(s1_mask, np.uint8)
    hh = None if hill is None else np.ascontiguousarray(hill, np.float64)
    ct = None if celltype is None else np.ascontiguousarray(celltype, np.float64)
    v = np.zeros(n)
    its = np.zeros(n_steps, np.int32)
    tact = np.zeros(n)
    reg = np.ascontiguousarray(np.zeros(n, np.uint8) if s2_region is None else np.asarray(s2_region, np.uint8).ravel())
    lib().cepo_tissue_run_s2(MODELS[model], dim, nx, ny, nz, h, _ptr(d), d.shape[1], dt, n_steps,
                             m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), bcl, t_crt, dur, n_pace, conc,
                             _ptr(hh) if hh is not None else None, 0 if hh is None else len(hh), rtol,
                             int(precond_norm), _ptr(ct) if ct is not None else None, _ptr(v), _iptr(its), act_thr,
                             _ptr(tact), int(s2_kind), int(s2_target), float(s2_thr),
                             reg.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), float(ecto_dur))
    return v, its, tact


class SlabPart:
    """CPU restatement of one slab part (the cep_part_* operations of the
    product: csrc/slab.cu) over the oracle's grid operator: the rows of part
    `part` of n_parts (contiguous planes of the last axis, PETSC_DECIDE's
    split, fem.cpp:667-670), columns in the part's extended numbering
    [lower halo plane | owned rows | upper halo plane], and the split
    Jacobi-PCG whose dot products are per-part partials added in part
    order. Vectors are numpy arrays or CPU torch tensors (so that gloo can
    carry the exchange)."""

    def __init__(self, dim: int, nx: int, ny: int, nz: int, h: float, dt: float, D, part: int, n_parts: int):
        if dim == 2:
            nz = 1
        rp, ci, av, bv = fem_assemble(dim, nx, ny, nz, h, dt, D)
        n_planes = ny if dim == 2 else nz
        self.plane = nx if dim == 2 else nx * ny
        if not (1 <= n_parts <= n_planes and 0 <= part < n_parts):
            raise ValueError("bad split")
        base, rem = divmod(n_planes, n_parts)
        first, planes = part * base + min(part, rem), base + (1 if part < rem else 0)
        self.index, self.n_parts, self.dim, self.dt = part, n_parts, dim, dt
        self.row0, self.n_own = first * self.plane, planes * self.plane
        self.has_lo, self.has_hi = part > 0, part < n_parts - 1
        lo = self.plane if self.has_lo else 0
        r0, r1 = rp[self.row0], rp[self.row0 + self.n_own]
        self.rp = (rp[self.row0: self.row0 + self.n_own + 1] - r0).astype(np.int64)
        self.ci = (ci[r0:r1] - (self.row0 - lo)).astype(np.int64)
        self.av, self.bv = av[r0:r1].copy(), bv[r0:r1].copy()
        rows = np.repeat(np.arange(self.n_own), np.diff(self.rp))
        diag = self.av[self.ci == rows + lo]
        self.dinv = 1.0 / diag
        self._rows = rows
        self.rtol, self.max_iter, self.precond_norm = 1e-5, 10000, True
        n = self.n_own
        self.x, self.r, self.z, self.q, self.p = (np.zeros(n) for _ in range(5))
        self.st = [dict(rz=0.0, n0=0.0, res=0.0, used=0, done=0, conv=0) for _ in range(2)]

    @staticmethod
    def _np(x):
        return None if x is None else (x.numpy() if hasattr(x, "numpy") else x)

    def buffer(self, n: int):
        import torch
        return torch.zeros(n, dtype=torch.float64)

    def set_solver(self, rtol: float, max_iter: int = 10000, precond_norm: bool = True):
        self.rtol, self.max_iter, self.precond_norm = float(rtol), int(max_iter), bool(precond_norm)

    def _apply(self, val, lo, own, hi):
        parts = ([self._np(lo)] if self.has_lo else []) + [self._np(own)[: self.n_own]] + \
            ([self._np(hi)] if self.has_hi else [])
        ext = np.concatenate(parts)
        return np.bincount(self._rows, weights=val * ext[self.ci], minlength=self.n_own)

    @staticmethod
    def _dot(a, b) -> float:
        return float(np.sum(a * b))

    @staticmethod
    def _total(all_partials, n_parts):
        a = SlabPart._np(all_partials)
        s0 = s1 = 0.0
        for k in range(n_parts):
            s0 += float(a[2 * k])
            s1 += float(a[2 * k + 1])
        return s0, s1

    def pack(self, v, lo, hi):
        vv = self._np(v)
        if lo is not None:
            self._np(lo)[:] = vv[: self.plane]
        if hi is not None:
            self._np(hi)[:] = vv[self.n_own - self.plane: self.n_own]

    def cg_begin(self, v, v_lo, v_hi, partial):
        b = self._apply(self.bv, v_lo, v, v_hi) / self.dt
        self.r[:] = b
        self.z[:] = self.dinv * b
        self.x[:] = 0.0
        self.p[:] = 0.0
        self.st[0] = dict(rz=0.0, n0=0.0, res=0.0, used=0, done=0, conv=0)
        out = self._np(partial)
        out[0] = self._dot(b, self.z)
        out[1] = self._dot(self.z, self.z) if self.precond_norm else self._dot(b, b)

    def cg_direction(self, it: int, all_partials, send_lo, send_hi):
        s = self.st[it & 1]
        t = dict(s)
        beta = 0.0
        if not s["done"]:
            a0, a1 = self._total(all_partials, self.n_parts)
            if it == 0:
                t["rz"], t["n0"] = a0, float(np.sqrt(a1))
                t["res"] = 1.0 if t["n0"] > 0.0 else 0.0
                if t["n0"] == 0.0:
                    t["done"] = t["conv"] = 1
            else:
                nr = float(np.sqrt(a1))
                t["res"], t["used"] = nr / s["n0"], it
                if nr <= self.rtol * s["n0"]:
                    t["done"] = t["conv"] = 1
                elif it >= self.max_iter:
                    t["done"] = 1
                beta = a0 / s["rz"]
                t["rz"] = a0
        self.st[(it + 1) & 1] = t
        if t["done"]:
            return
        self.p[:] = beta * self.p + self.z
        if self.has_lo and send_lo is not None:
            self._np(send_lo)[:] = self.p[: self.plane]
        if self.has_hi and send_hi is not None:
            self._np(send_hi)[:] = self.p[self.n_own - self.plane:]

    def cg_product(self, it: int, p_lo, p_hi, partial):
        if self.st[(it + 1) & 1]["done"]:
            return
        self.q[:] = self._apply(self.av, p_lo, self.p, p_hi)
        out = self._np(partial)
        out[0] = self._dot(self.p, self.q)
        out[1] = 0.0

    def cg_update(self, it: int, all_partials, partial):
        s = self.st[(it + 1) & 1]
        if s["done"]:
            return
        pq, _ = self._total(all_partials, self.n_parts)
        alpha = s["rz"] / pq
        self.x += alpha * self.p
        self.r -= alpha * self.q
        self.z[:] = self.dinv * self.r
        out = self._np(partial)
        out[0] = self._dot(self.r, self.z)
        out[1] = self._dot(self.z, self.z) if self.precond_norm else self._dot(self.r, self.r)

    def cg_status(self, it: int):
        s = self.st[(it + 1) & 1]
        return bool(s["done"]), (s["used"] if s["conv"] else -self.max_iter), s["res"]

    def cg_end(self, v, t_new: float = 0.0):
        self._np(v)[: self.n_own] = self.x
