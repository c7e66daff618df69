"""ten Tusscher 2004 (the reference's 2004_b build) on the GPU against the
reference's own traces and the oracle. Tolerances as in test_ord_gpu.py."""
from __future__ import annotations

import threading
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
VM_TOL_FP64 = 1e-6
APD_TOL_FP64 = 0.01
APD_TOL_MIXED = 0.1
CAD_TOL_MIXED = 0.1


@pytest.mark.gpu
@pytest.mark.parametrize("path", sorted(GOLD.glob("tt2004_*.npz")), ids=lambda p: p.stem)
def test_tt2004_fp64_matches_reference_golden(cep, gpu, path):
    g = np.load(path)
    b = cep.Batch("tt2004", 1, "fp64")
    b.init(conc=np.array([float(g["conc"])]), hill=g["hill"][None, :])
    assert np.array_equal(b.get_states()[0], g["y0"])
    b.set_protocol(float(g["dt"]), 3, -1)
    stride = int(g["stride"])
    v = np.zeros(len(g["v_trace"]))
    for k in range(len(v)):
        b.run(stride)
        v[k] = b.get_states()[0, 0]
    assert np.abs(v - g["v_trace"]).max() <= VM_TOL_FP64
    fin = b.get_states()[0]
    rel = np.abs(fin - g["final_states"]) / np.maximum(np.abs(g["final_states"]), 1e-9)
    assert rel.max() < 1e-5


@pytest.mark.gpu
def test_tt2004_biomarkers_fp64_and_mixed(cep, gpu, oracle):
    rng = np.random.default_rng(9)
    n = 6
    hill = np.zeros((n, 14))
    hill[:, 0::2] = 10 ** rng.uniform(-0.5, 1.5, (n, 7))
    hill[:, 1::2] = rng.uniform(0.7, 1.5, (n, 7))
    conc = rng.uniform(0.0, 2.0, n)
    conc[0] = 0.0
    n_pace, first, dt, bcl = 4, 1, 0.01, 1000.0
    ref = [None] * n

    def work(k):
        c = oracle.Cell("tt2004", 0.0, conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        bm, _ = c.run_biomarkers(dt, n_pace, first, dt_write=1.0)
        bm["final"] = c.states.copy()
        ref[k] = bm

    th = [threading.Thread(target=work, args=(k,)) for k in range(n)]
    [x.start() for x in th]
    [x.join() for x in th]
    out = {}
    for prec in ("fp64", "mixed"):
        b = cep.Batch("tt2004", n, prec)
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
def test_tt2004_published_gmma_without_quirks(cep, gpu, oracle):
    """Without the quirk flag the NaCa partition is the published 0.35: the
    GPU follows the oracle's non-quirk model."""
    b = cep.Batch("tt2004", 1, "fp64")
    b.init(quirks=False)
    b.set_protocol(0.01, 2, -1)
    c = oracle.Cell("tt2004", quirks=False)
    stride, n = 200, 500
    _, vo = c.run(0.0, 0.01, stride * n, stride)
    v = np.zeros(n)
    for k in range(n):
        b.run(stride)
        v[k] = b.get_states()[0, 0]
    assert np.abs(v - vo).max() <= VM_TOL_FP64
