"""ten Tusscher 2006 (epicardial, IK1 Ko units) on the GPU against the oracle.

The oracle is pinned bit for bit to the reference's own compiled model
(test_oracle_pin.py); the reference integrates it with its fixed-step
solveAnalytical in the tissue drivers. Tolerances as in test_ord_gpu.py.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

VM_TOL_FP64 = 1e-6
APD_TOL_FP64 = 0.01
APD_TOL_MIXED = 0.1
CAD_TOL_MIXED = 0.1
QNET_RTOL_MIXED = 0.01


def tt06_population(n: int, seed: int):
    """Seeded Hill table for the channels the TT2006 hook blocks (ICaL, IK1,
    IKs, INa, Ito, IKr), concentrations 0..3 x a seeded Cmax."""
    rng = np.random.default_rng(seed)
    hill = np.zeros((n, 14))
    for c in (0, 2, 4, 6, 10, 12):
        hill[:, c] = 10 ** rng.uniform(-0.5, 1.5, n)
        hill[:, c + 1] = rng.uniform(0.7, 1.5, n)
    conc = rng.uniform(0.0, 3.0, n) * 10 ** rng.uniform(-1, 0.5)
    conc[0] = 0.0
    return conc, hill


@pytest.mark.gpu
def test_tt2006_fp64_trace_matches_oracle(cep, gpu, oracle):
    conc, hill = tt06_population(4, seed=11)
    n = len(conc)
    dt = 0.01
    b = cep.Batch("tt2006", n, "fp64")
    b.init(conc=conc, hill=hill)
    b.set_pacing(1000.0)
    cells = []
    for k in range(n):
        c = oracle.Cell("tt2006", 0.0, conc[k], hill[k])
        c.set_pacing(1000.0)
        cells.append(c)
    y0 = b.get_states()
    for k in range(n):
        assert np.array_equal(y0[k], cells[k].states)
    b.set_protocol(dt, 2, -1, dt_write=1.0)
    stride, n_chunks = 200, 500  # 1000 ms
    vg = np.zeros((n_chunks, n))
    traces = [None] * n

    def work(k):
        _, traces[k] = cells[k].run(0.0, dt, stride * n_chunks, stride)

    th = [threading.Thread(target=work, args=(k,)) for k in range(n)]
    [x.start() for x in th]
    for i in range(n_chunks):
        b.run(stride)
        vg[i] = b.get_states()[:, 0]
    [x.join() for x in th]
    for k in range(n):
        err = np.abs(vg[:, k] - traces[k]).max()
        assert err <= VM_TOL_FP64, f"instance {k}: max |dVm| = {err:.3e} mV"
    fin = b.get_states()
    for k in range(n):
        rel = np.abs(fin[k] - cells[k].states) / np.maximum(np.abs(cells[k].states), 1e-9)
        assert rel.max() < 1e-5


@pytest.mark.gpu
def test_tt2006_biomarkers_fp64_and_mixed(cep, gpu, oracle):
    conc, hill = tt06_population(6, seed=5)
    n_pace, first, dt, bcl = 4, 1, 0.01, 1000.0
    ref = [None] * len(conc)

    def work(k):
        c = oracle.Cell("tt2006", 0.0, conc[k], hill[k])
        c.set_pacing(bcl)
        bm, _ = c.run_biomarkers(dt, n_pace, first, dt_write=1.0)
        bm["final"] = c.states.copy()
        ref[k] = bm

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(conc))]
    [x.start() for x in th]
    [x.join() for x in th]
    out = {}
    for prec in ("fp64", "mixed"):
        b = cep.Batch("tt2006", len(conc), prec)
        b.init(conc=conc, hill=hill)
        b.set_pacing(bcl)
        b.set_protocol(dt, n_pace, first, dt_write=1.0)
        b.run_to_end(20000)
        out[prec] = (b.biomarkers(), b.get_states())
    b64, s64 = out["fp64"]
    bmx, _ = out["mixed"]
    for k, r in enumerate(ref):
        assert b64["status"][k] == cep.INST_DONE
        assert abs(s64[k, 0] - r["final"][0]) <= VM_TOL_FP64
        assert b64["steepest_pace"][k] == r["steepest_pace"]
        for key in ("apd90", "apd50", "cad90", "cad50"):
            assert abs(b64[key][k] - r[key]) <= APD_TOL_FP64, (key, k, b64[key][k], r[key])
        assert abs(bmx["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED, (k, bmx["apd90"][k], r["apd90"])
        assert abs(bmx["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED, (k, bmx["cad90"][k], r["cad90"])


@pytest.mark.gpu
def test_tt2006_fp64_matches_reference_golden(cep, gpu):
    """Single-cell build of the reference, two beats: the GPU FP64 trace
    against the reference's own trace."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "tt2006_single.npz")
    b = cep.Batch("tt2006", 1, "fp64")
    b.init()
    assert np.array_equal(b.get_states()[0], g["y0"])
    b.set_protocol(float(g["dt"]), 3, -1)
    stride = int(g["stride"])
    v = np.zeros(len(g["v_trace"]))
    for k in range(len(v)):
        b.run(stride)
        v[k] = b.get_states()[0, 0]
    assert np.abs(v - g["v_trace"]).max() <= VM_TOL_FP64
