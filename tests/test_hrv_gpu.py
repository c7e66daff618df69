"""Heart-rate-variability pacing on the GPU (cep_batch_hrv; CEPCell_NEO/
modules/hrv_bench.cpp:146-343 on the fixed-step scheme) against the
oracle's restatement (oracle/src/protocols.c cepo_hrv_run, itself pinned to
the reference bench compiled here: test_oracle_pin.py) and against what
that reference bench printed (tests/golden/hrv_bench_records.json).

Tolerances as in test_biomarkers_gpu.py. FP64: times within 0.01 ms, the
beat integrals within 1e-9 relative, potentials within 1e-6 mV, slopes
within 1e-6 relative, Ca values within 1e-9 relative, the chosen pace and
its BCL equal. Mixed: APD90/50 and CaD90/50 within 0.1 ms, qNet and the
AUCs within 1 %, potentials within 0.5 mV, slopes within 2 %, Ca values
within 1 %."""
from __future__ import annotations

import json
import threading
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
HILL = np.array([5.0, 1.0, 20.0, 1.1, 30.0, 0.9, 8.0, 1.2, 4.0, 0.8, 15.0, 1.0, 0.6, 1.1])
TIME_KEYS = ("apd90", "apd50", "cad90", "cad50")


def _oracle_hrv(oracle, celltype, conc, hill, bcls, dt, num_pace1=None):
    out = [None] * len(conc)

    def work(k):
        c = oracle.Cell("ord2011", celltype[k], conc[k], hill[k], is_dutta=True, quirks=2)
        out[k] = c.hrv(bcls, dt, 1.0, num_pace1)
        out[k]["y"] = c.y[:41].copy()  # the oracle keeps room for any model's states

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(conc))]
    [t.start() for t in th]
    [t.join() for t in th]
    return out


def _gpu_hrv(cep, celltype, conc, hill, bcls, dt, prec, kernel=None, num_pace1=None):
    b = cep.Batch("ord2011", len(conc), prec)
    b.init(celltype=celltype, conc=conc, hill=hill, dutta=True, neo=True)
    if kernel:
        b.set_kernel(kernel)
    r = b.hrv(bcls, dt, 1.0, num_pace1)
    y = b.get_states()
    b.close()
    return r, y


def _check(got, ref, prec):
    fp = prec == "fp64"
    for k, r in enumerate(ref):
        assert got["status"][k] == 1, k
        if fp:
            assert got["steepest_pace"][k] == r["steepest_pace"], (k, got["steepest_pace"][k], r["steepest_pace"])
            assert got["bcl"][k] == r["bcl"], k
        for key in TIME_KEYS:
            assert abs(got[key][k] - r[key]) <= (0.01 if fp else 0.1), (key, k, got[key][k], r[key])
        q = r["qnet"] / 1000.0
        for key, want in (("qnet", q), ("inal_auc", r["inal_auc"]), ("ical_auc", r["ical_auc"])):
            tol = 1e-9 * max(abs(want), 1e-12) if fp else 0.01 * abs(want)
            assert abs(got[key][k] - want) <= tol, (key, k, got[key][k], want)
        for key in ("vm_peak", "vm_valley", "vm_dia"):
            assert abs(got[key][k] - r[key]) <= (1e-6 if fp else 0.5), (key, k, got[key][k], r[key])
        for key in ("dvmdt_max", "dvmdt_repol"):
            assert abs(got[key][k] - r[key]) <= (1e-6 if fp else 0.02) * abs(r[key]), (key, k, got[key][k], r[key])
        for key in ("ca_peak", "ca_valley", "ca_dia"):
            assert abs(got[key][k] - r[key]) <= (1e-9 if fp else 0.01) * abs(r[key]), (key, k, got[key][k], r[key])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_hrv_matches_the_reference_bench(cep, gpu, prec):
    """The device's HRV records against what the reference's hrv_bench.cpp
    printed (compiled over the oracle's CEPCell_NEO ORd): 259 intervals plus
    the appended 1000 ms, dt 0.02 ms, a control and a drug, every printed
    field within the tolerances above plus the printed rounding (5e-7)."""
    g = json.loads((GOLD / "hrv_bench_records.json").read_text())
    c, bcls, rec = g["case"], g["bcls"] + [1000.0], g["records"]
    concs = [0.0] + list(c["concs"])
    hill = np.tile(np.array(c["hill"]), (len(concs), 1))
    got, _ = _gpu_hrv(cep, [c["celltype"]] * len(concs), concs, hill, bcls, c["dt"], prec)
    fp = prec == "fp64"
    t_tol, rel = (0.01, 1e-6) if fp else (0.1, 0.02)
    for k, conc in enumerate(concs):
        key = f"{conc:.2f}"
        ap = [float(x) for x in rec[key]["ap"][0]]
        ca = [float(x) for x in rec[key]["ca"][0]]
        qn = [float(x) for x in rec[key]["qni"][0]]
        assert got["status"][k] == 1
        for v, want in ((got["apd90"][k], ap[5]), (got["apd50"][k], ap[6]), (got["cad90"][k], ca[3]),
                        (got["cad50"][k], ca[4])):
            assert abs(v - want) <= t_tol + 5e-7, (key, v, want)
        for v, want in ((got["dvmdt_max"][k], ap[2]), (got["dvmdt_repol"][k], ap[1])):
            assert abs(v - want) <= rel * abs(want) + 5e-7, (key, v, want)
        for v, want in ((got["vm_peak"][k], ap[3]), (got["vm_dia"][k], ap[4])):
            assert abs(v - want) <= (1e-6 if fp else 0.5) + 5e-7, (key, v, want)
        for v, want in ((got["ca_peak"][k], ca[1]), (got["ca_dia"][k], ca[2])):
            assert abs(v - want) <= (1e-9 if fp else 0.01) * abs(want) + 5e-7, (key, v, want)
        assert abs(got["qnet"][k] - qn[1]) <= (1e-9 if fp else 0.01) * abs(qn[1]) + 5e-7, (key, got["qnet"][k])
        if fp:
            assert got["steepest_pace"][k] == int(ap[8]) and got["bcl"][k] == int(ap[9]), key
    if len(concs) > 1:  # qInward of the drug against the control, as printed
        qi = 0.5 * (got["inal_auc"][1] / got["inal_auc"][0] + got["ical_auc"][1] / got["ical_auc"][0])
        want = float(rec[f"{concs[1]:.2f}"]["qni"][0][2])
        assert abs(qi - want) <= (1e-9 if fp else 0.01) * abs(want) + 5e-7, (qi, want)


@pytest.mark.gpu
def test_hrv_every_field_fp64_against_the_oracle(cep, gpu, oracle):
    """Four instances (the three celltypes, which the CEPCell_NEO build
    honours, and a drugged one) over 251 random intervals of 280-360 ms plus
    1000 ms at dt 0.02 ms: every record field and the final states."""
    rng = np.random.default_rng(11)
    bcls = list(np.round(rng.uniform(280.0, 360.0, 251), 1)) + [1000.0]
    ct = np.array([0.0, 1.0, 2.0, 0.0])
    conc = np.array([0.0, 0.0, 0.0, 2.0])
    hill = np.tile(HILL, (4, 1))
    ref = _oracle_hrv(oracle, ct, conc, hill, bcls, 0.02)
    got, y = _gpu_hrv(cep, ct, conc, hill, bcls, 0.02, "fp64")
    _check(got, ref, "fp64")
    assert (got["n_eligible"] == 250).all()
    for k, r in enumerate(ref):
        assert abs(y[k, 0] - r["y"][0]) <= 1e-6, (k, y[k, 0], r["y"][0])


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["cell", "roles", "pairs"])
def test_hrv_short_protocols_and_the_one_off_replacement(cep, gpu, oracle, kernel):
    """Fewer than 250 paces evaluate no beat (the bench's size_t
    subtraction wraps): the record is the initial beat, equal to the
    oracle's bit for bit, and the final states follow the oracle's
    trajectory through every rewound pace start. With num_pace1 = 250 the
    one-off replacement (:336-338) fires at the end of pace 0 and copies the
    unevaluated beat, as the bench does. The three kernel forms agree to
    1e-9 (relative to max(1, |state|))."""
    bcls = [812.5, 640.0, 700.3, 1000.0]
    ct = np.array([0.0, 1.0])
    conc = np.array([0.0, 1.0])
    hill = np.tile(HILL, (2, 1))
    for np1 in (None, 250):
        ref = _oracle_hrv(oracle, ct, conc, hill, bcls, 0.02, np1)
        got, y = _gpu_hrv(cep, ct, conc, hill, bcls, 0.02, "fp64", kernel=kernel, num_pace1=np1)
        for k, r in enumerate(ref):
            for f in cep.BM_FIELDS:
                if f in ("apd_tri", "cad_tri"):
                    continue
                want = r[f] / 1000.0 if f == "qnet" else r[f]
                assert got[f][k] == want, (np1, k, f, got[f][k], want)
            assert got["steepest_pace"][k] == r["steepest_pace"] and got["bcl"][k] == r["bcl"]
            assert got["n_eligible"][k] == 0 and got["status"][k] == 1
            assert abs(y[k, 0] - r["y"][0]) <= 1e-6, (k, y[k, 0], r["y"][0])
            assert np.all(np.abs(y[k] - r["y"]) <= 1e-6 * np.maximum(1.0, np.abs(r["y"]))), k
        if kernel != "cell":  # the forms add the same terms, the FMA contractions differ (as in the run kernels)
            yc = _gpu_hrv(cep, ct, conc, hill, bcls, 0.02, "fp64", kernel="cell", num_pace1=np1)[1]
            assert np.all(np.abs(y - yc) <= 1e-9 * np.maximum(1.0, np.abs(yc))), kernel


@pytest.mark.gpu
def test_hrv_argument_checks(cep, gpu):
    b = cep.Batch("cipa2017", 2, "fp64")
    b.init()
    with pytest.raises(cep.CepError) as e:
        b.hrv([500.0], 0.02)
    assert e.value.code == cep.ERR_UNSUPPORTED
    with pytest.raises(cep.CepError) as e:
        b.init(neo=True)
    assert e.value.code == cep.ERR_UNSUPPORTED
    b.close()
    o = cep.Batch("ord2011", 2, "mixed")
    o.init(neo=True)
    with pytest.raises(cep.CepError) as e:
        o.hrv([500.0], 0.1)  # above the mixed path's validated step
    assert e.value.code == cep.ERR_UNSUPPORTED
    for bad in ([], [500.0, -1.0], [float("nan")]):
        with pytest.raises(cep.CepError) as e:
            o.hrv(bad, 0.02)
        assert e.value.code == cep.ERR_ARG
    with pytest.raises(cep.CepError) as e:
        o.hrv([500.0], 0.02, dt_write=0.001)
    assert e.value.code == cep.ERR_ARG
    o.close()
