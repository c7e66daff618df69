"""ToR-ORd (Tomek 2019) on the GPU against the oracle (whose RATES are the
reference computeRates bit for bit; the reference integrates this model
only with CVODE, so the fixed-step trajectory is the oracle's). Tolerances
as in test_ord_gpu.py."""
from __future__ import annotations

import threading

import numpy as np
import pytest

VM_TOL_FP64 = 1e-6
APD_TOL_FP64 = 0.01
APD_TOL_MIXED = 0.1
CAD_TOL_MIXED = 0.1
QNET_RTOL_MIXED = 0.01


def _cases(seed: int, n: int):
    rng = np.random.default_rng(seed)
    hill = np.zeros((n, 14))
    hill[:, 0::2] = 10 ** rng.uniform(-1, 2, (n, 7))
    hill[:, 1::2] = rng.uniform(0.6, 1.8, (n, 7))
    conc = rng.uniform(0.0, 3.0, n)
    conc[0] = 0.0
    celltype = np.arange(n) % 3 * 1.0
    return celltype, conc, hill


@pytest.mark.gpu
def test_tomek_fp64_trace_matches_oracle(cep, gpu, oracle):
    ct, conc, hill = _cases(21, 3)
    n = len(conc)
    b = cep.Batch("tomek2019", n, "fp64")
    b.init(celltype=ct, conc=conc, hill=hill)
    cells = [oracle.Cell("tomek2019", ct[k], conc[k], hill[k], quirks=True) for k in range(n)]
    y0 = b.get_states()
    for k in range(n):
        assert np.array_equal(y0[k], cells[k].states), k
    b.set_protocol(0.005, 2, -1)
    stride, n_chunks = 400, 500  # 1000 ms
    vg = np.zeros((n_chunks, n))
    traces = [None] * n

    def work(k):
        _, traces[k] = cells[k].run(0.0, 0.005, stride * n_chunks, stride)

    th = [threading.Thread(target=work, args=(k,)) for k in range(n)]
    [x.start() for x in th]
    for i in range(n_chunks):
        b.run(stride)
        vg[i] = b.get_states()[:, 0]
    [x.join() for x in th]
    for k in range(n):
        err = np.abs(vg[:, k] - traces[k]).max()
        assert err <= VM_TOL_FP64, f"instance {k}: max |dVm| = {err:.3e} mV"


@pytest.mark.gpu
def test_tomek_biomarkers_fp64_and_mixed(cep, gpu, oracle):
    ct, conc, hill = _cases(22, 6)
    n = len(conc)
    n_pace, first, dt, bcl = 3, 1, 0.005, 1000.0
    ref = [None] * n

    def work(k):
        c = oracle.Cell("tomek2019", ct[k], conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        bm, _ = c.run_biomarkers(dt, n_pace, first, dt_write=1.0)
        ref[k] = bm

    th = [threading.Thread(target=work, args=(k,)) for k in range(n)]
    [x.start() for x in th]
    [x.join() for x in th]
    out = {}
    for prec in ("fp64", "mixed"):
        b = cep.Batch("tomek2019", n, prec)
        b.init(celltype=ct, conc=conc, hill=hill)
        b.set_pacing(bcl)
        b.set_protocol(dt, n_pace, first, dt_write=1.0)
        b.run_to_end(30000)
        out[prec] = b.biomarkers()
    b64, bmx = out["fp64"], out["mixed"]
    for k, r in enumerate(ref):
        assert b64["status"][k] == cep.INST_DONE and bmx["status"][k] == cep.INST_DONE
        assert b64["steepest_pace"][k] == r["steepest_pace"]
        for key in ("apd90", "apd50", "cad90", "cad50"):
            assert abs(b64[key][k] - r[key]) <= APD_TOL_FP64, (key, k, b64[key][k], r[key])
        assert abs(bmx["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED, (k, bmx["apd90"][k], r["apd90"])
        assert abs(bmx["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED, (k, bmx["cad90"][k], r["cad90"])
        q = r["qnet"] / 1000
        assert abs(bmx["qnet"][k] - q) <= QNET_RTOL_MIXED * abs(q) + 1e-6, (k, bmx["qnet"][k], q)


@pytest.mark.gpu
def test_tomek_mixed_at_its_largest_dt(cep, gpu, oracle):
    """The mixed path at dt = 0.01 ms, the largest its slow-gate series form
    accepts (j and jp reach tau ~0.1 ms near +50 mV), against the FP64
    oracle at the same dt; a larger dt is refused in mixed precision and
    accepted in FP64."""
    ct, conc, hill = _cases(23, 4)
    n = len(conc)
    n_pace, first, dt, bcl = 3, 1, 0.01, 1000.0
    ref = [None] * n

    def work(k):
        c = oracle.Cell("tomek2019", ct[k], conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        ref[k], _ = c.run_biomarkers(dt, n_pace, first, dt_write=1.0)

    th = [threading.Thread(target=work, args=(k,)) for k in range(n)]
    [x.start() for x in th]
    [x.join() for x in th]
    b = cep.Batch("tomek2019", n, "mixed")
    b.init(celltype=ct, conc=conc, hill=hill)
    b.set_pacing(bcl)
    with pytest.raises(cep.CepError) as e:
        b.set_protocol(0.02, n_pace, first, dt_write=1.0)
    assert e.value.code == cep.ERR_UNSUPPORTED
    b.set_protocol(dt, n_pace, first, dt_write=1.0)
    b.run_to_end(30000)
    bmx = b.biomarkers()
    for k, r in enumerate(ref):
        assert bmx["status"][k] == cep.INST_DONE
        assert abs(bmx["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED, (k, bmx["apd90"][k], r["apd90"])
        assert abs(bmx["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED, (k, bmx["cad90"][k], r["cad90"])
        q = r["qnet"] / 1000
        assert abs(bmx["qnet"][k] - q) <= QNET_RTOL_MIXED * abs(q) + 1e-6, (k, bmx["qnet"][k], q)
    f = cep.Batch("tomek2019", n, "fp64")
    f.init(celltype=ct, conc=conc, hill=hill)
    f.set_protocol(0.02, n_pace, first, dt_write=1.0)
