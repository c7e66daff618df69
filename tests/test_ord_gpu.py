"""ORd 2011 on the GPU against the oracle / the reference's golden traces.

Tolerances (stated by the specification of this path):
  FP64 path : Vm trace max |err| <= 1e-6 mV against the same fixed-step
              integrator; APD90 within 0.01 ms.
  mixed path: APD90 <= 0.1 ms, qNet <= 1 %, CaTD90 <= 0.1 ms against the
              FP64 oracle.
"""
from __future__ import annotations

import threading
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
ORD_CASES = sorted(GOLD.glob("ord_*.npz"))

VM_TOL_FP64 = 1e-6      # mV
APD_TOL_FP64 = 0.01     # ms
APD_TOL_MIXED = 0.1     # ms
CAD_TOL_MIXED = 0.1     # ms
QNET_RTOL_MIXED = 0.01  # relative


@pytest.mark.gpu
@pytest.mark.parametrize("path", ORD_CASES, ids=lambda p: p.stem)
def test_ord_fp64_trace_matches_reference(cep, gpu, path):
    g = np.load(path)
    b = cep.Batch("ord2011", 1, "fp64")
    b.init(celltype=float(g["celltype"]), conc=float(g["conc"]), hill=g["hill"], dutta=bool(g["dutta"]),
           quirks=True)
    b.set_pacing(float(g["bcl"]))
    y0 = b.get_states()[0]
    assert np.array_equal(y0, g["y0"])
    dv, _ = b.rates(0.0)
    assert abs(dv[0] - g["rates0"][0]) <= 1e-12 * max(1.0, abs(g["rates0"][0]))
    stride = int(g["stride"])
    v = np.zeros(len(g["v_trace"]))
    for k in range(len(v)):
        b.run(stride)
        v[k] = b.get_states()[0, 0]
    err = np.abs(v - g["v_trace"]).max()
    assert err <= VM_TOL_FP64, f"max |dVm| = {err:.3e} mV"
    fin = b.get_states()[0]
    rel = np.abs(fin - g["final_states"]) / np.maximum(np.abs(g["final_states"]), 1e-6)
    assert rel.max() < 1e-6
    step, t = b.clock(0)
    assert step == int(g["n_steps"]) and t == float(g["t_final"])


def _oracle_biomarkers(oracle, cases, n_pace, first_pace, dt, bcl, model="ord2011", quirks=True):
    out = [None] * len(cases)

    def work(k, c):
        cell = oracle.Cell(model, c["celltype"], c["conc"], c["hill"], is_dutta=c["dutta"], quirks=quirks)
        cell.set_pacing(bcl)
        bm, _ = cell.run_biomarkers(dt, n_pace, first_pace, dt_write=1.0)
        bm["final"] = cell.states.copy()
        out[k] = bm

    th = [threading.Thread(target=work, args=(k, c)) for k, c in enumerate(cases)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return out


def _config1_cases(seed=7, n_conc=5):
    """Single-cell drug configuration: one drug, IC50 log-uniform in
    [0.1, 100] uM, h uniform in [0.6, 1.8], Cmax log-uniform in [0.01, 10] uM,
    concentrations 0..4 x Cmax."""
    rng = np.random.default_rng(seed)
    hill = np.zeros(14)
    hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1::2] = rng.uniform(0.6, 1.8, 7)
    cmax = 10 ** rng.uniform(-2, 1)
    return [dict(celltype=0.0, conc=k * cmax, hill=hill, dutta=False) for k in range(n_conc)]


def _gpu_biomarkers(cep, cases, precision, n_pace, first_pace, dt, bcl, model="ord2011", quirks=True):
    n = len(cases)
    b = cep.Batch(model, n, precision)
    b.init(celltype=np.array([c["celltype"] for c in cases]), conc=np.array([c["conc"] for c in cases]),
           hill=np.stack([c["hill"] for c in cases]), dutta=cases[0]["dutta"], quirks=quirks)
    b.set_pacing(bcl)
    b.set_protocol(dt, n_pace, first_pace, dt_write=1.0)
    b.run_to_end(50000)
    bm = b.biomarkers()
    st = b.get_states()
    return bm, st


BM_KEYS = ("apd90", "apd50", "dvmdt_max", "dvmdt_repol", "vm_peak", "vm_dia", "cad90", "cad50", "ca_peak",
           "ca_dia")


@pytest.mark.gpu
def test_ord_fp64_biomarkers_match_oracle_short(cep, gpu, oracle):
    cases = _config1_cases(seed=11)
    ref = _oracle_biomarkers(oracle, cases, 4, 3, 0.005, 1000.0)
    bm, st = _gpu_biomarkers(cep, cases, "fp64", 4, 3, 0.005, 1000.0)
    for k, r in enumerate(ref):
        assert bm["status"][k] == cep.INST_DONE
        assert abs(bm["apd90"][k] - r["apd90"]) <= APD_TOL_FP64
        assert abs(bm["apd50"][k] - r["apd50"]) <= APD_TOL_FP64
        assert abs(bm["cad90"][k] - r["cad90"]) <= APD_TOL_FP64
        assert abs(bm["qnet"][k] - r["qnet"] / 1000.0) <= 1e-9 * max(1.0, abs(r["qnet"]))
        assert abs(bm["dvmdt_max"][k] - r["dvmdt_max"]) <= 1e-6 * abs(r["dvmdt_max"])
        assert abs(st[k, 0] - r["final"][0]) <= VM_TOL_FP64
        assert bm["steepest_pace"][k] == r["steepest_pace"]


@pytest.mark.gpu
def test_ord_config1_fp64_100_paces(cep, gpu, oracle):
    """The single-cell configuration end to end on the FP64 path: 5
    concentrations, 100 paces at BCL 1000 ms, dt 0.005 ms, last-beat
    biomarkers, against the oracle."""
    cases = _config1_cases(seed=7)
    ref = _oracle_biomarkers(oracle, cases, 100, 99, 0.005, 1000.0)
    b64, s64 = _gpu_biomarkers(cep, cases, "fp64", 100, 99, 0.005, 1000.0)
    for k, r in enumerate(ref):
        assert abs(s64[k, 0] - r["final"][0]) <= VM_TOL_FP64
        for key in ("apd90", "apd50", "cad90", "cad50"):
            assert abs(b64[key][k] - r[key]) <= APD_TOL_FP64, (key, k, b64[key][k], r[key])


@pytest.mark.gpu
def test_ord_config1_100_paces_mixed(cep, gpu, oracle):
    """The single-cell configuration end to end: 5 concentrations, 100 paces
    at BCL 1000 ms, dt 0.005 ms, last-beat biomarkers; mixed precision
    against the FP64 oracle."""
    cases = _config1_cases(seed=7)
    ref = _oracle_biomarkers(oracle, cases, 100, 99, 0.005, 1000.0)
    bmx, smx = _gpu_biomarkers(cep, cases, "mixed", 100, 99, 0.005, 1000.0)
    for k, r in enumerate(ref):
        assert abs(bmx["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED, (k, bmx["apd90"][k], r["apd90"])
        assert abs(bmx["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED, (k, bmx["cad90"][k], r["cad90"])
        q = r["qnet"] / 1000.0
        assert abs(bmx["qnet"][k] - q) <= QNET_RTOL_MIXED * abs(q), (k, bmx["qnet"][k], q)


@pytest.mark.gpu
@pytest.mark.parametrize("quirks", [True, False])
def test_ord_mixed_biomarkers_within_tolerance(cep, gpu, oracle, quirks):
    rng = np.random.default_rng(3)
    cases = []
    for k in range(6):
        hill = np.zeros(14)
        hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
        hill[1::2] = rng.uniform(0.6, 1.8, 7)
        cases.append(dict(celltype=float(k % 3), conc=float(10 ** rng.uniform(-2, 1)), hill=hill, dutta=True))
    ref = _oracle_biomarkers(oracle, cases, 6, 5, 0.005, 1000.0, quirks=quirks)
    bm, _ = _gpu_biomarkers(cep, cases, "mixed", 6, 5, 0.005, 1000.0, quirks=quirks)
    for k, r in enumerate(ref):
        assert abs(bm["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED
        assert abs(bm["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED
        q = r["qnet"] / 1000.0
        assert abs(bm["qnet"][k] - q) <= QNET_RTOL_MIXED * abs(q)


@pytest.mark.gpu
def test_ord_split_launches_equal_single_launch(cep, gpu):
    """K steps in one launch equal the same K steps in many launches
    (state, clock and biomarker state persist exactly across launches)."""
    cases = _config1_cases(seed=5, n_conc=3)
    one = cep.Batch("ord2011", 3, "fp64")
    one.init(conc=np.array([c["conc"] for c in cases]), hill=np.stack([c["hill"] for c in cases]))
    one.set_pacing(1000.0)
    one.set_protocol(0.005, 3, 2, dt_write=1.0)
    one.run_to_end(700000)  # the whole protocol in one launch
    a, sa = one.biomarkers(), one.get_states()
    assert one.clock(0)[0] == 600000
    b = cep.Batch("ord2011", 3, "fp64")
    b.init(conc=np.array([c["conc"] for c in cases]), hill=np.stack([c["hill"] for c in cases]))
    b.set_pacing(1000.0)
    b.set_protocol(0.005, 3, 2, dt_write=1.0)
    b.run_to_end(777)
    bb = b.biomarkers()
    assert np.array_equal(sa, b.get_states())
    for key in BM_KEYS:
        assert np.array_equal(a[key], bb[key]), key


@pytest.mark.gpu
def test_ord_bad_inputs_rejected(cep, gpu):
    b = cep.Batch("ord2011", 2, "fp64")
    hill = np.zeros((2, 14))
    hill[1, 0] = np.nan
    with pytest.raises(cep.CepError) as e:
        b.init(conc=np.array([1.0, 1.0]), hill=hill)
    assert e.value.code == cep.ERR_ARG
    with pytest.raises(cep.CepError):
        b.init(conc=np.array([-1.0, 1.0]))
    with pytest.raises(cep.CepError) as e:
        cep.Batch("ord2011", 0)
    assert e.value.code == cep.ERR_ARG
    b.init()
    with pytest.raises(cep.CepError):
        b.set_protocol(0.005, 10, 10)


@pytest.mark.gpu
@pytest.mark.parametrize("cajsr", [0.5, 1e-4, -0.005, -0.05])
def test_ord_rates_hold_the_jrel_floor_at_any_cajsr(cep, gpu, oracle, cajsr):
    """Forward Euler lets cajsr dip below zero in long protocols (the
    oracle's own trajectory of the HRV epicardial case does from pace 139
    on). For -0.0123 < cajsr < 0 the written time constant bt / (1 +
    0.0123 / cajsr) is negative and the reference floors it at 0.001 ms
    (Ohara_Rudy_2011.cpp:1063-1066); the device's rate form must take the
    same floor there, or the release gates grow without bound. Every RATES
    entry at such states against the oracle's computeRates, within 1e-9 of
    the largest rate."""
    ct, conc = np.array([0.0, 1.0]), np.array([0.0, 0.5])
    hill = np.tile(np.array([5.0, 1.0, 20.0, 1.1, 30.0, 0.9, 8.0, 1.2, 4.0, 0.8, 15.0, 1.0, 0.6, 1.1]), (2, 1))
    b = cep.Batch("ord2011", 2, "fp64")
    b.init(celltype=ct, conc=conc, hill=hill, dutta=True, quirks=False)
    y = b.get_states()
    y[:, 0] = -10.0  # an open L-type channel: a nonzero release target
    y[:, 8] = cajsr
    y[:, 39:41] = [0.02, 0.03]  # Jrelnp, Jrelp away from their targets
    b.set_states(y)
    r = b.rates_all(0.0)
    b.close()
    for k in range(2):
        c = oracle.Cell("ord2011", ct[k], conc[k], hill[k], is_dutta=True, quirks=False)
        c.y[:41] = y[k]
        ro, _ = c.rates(0.0)
        scale = np.abs(ro[:41]).max()
        assert np.isfinite(r[k]).all()
        assert np.abs(r[k] - ro[:41]).max() <= 1e-9 * scale, (k, np.abs(r[k] - ro[:41]).argmax())
