"""Every field of the device biomarker records against the oracle's
restatement of the CiPA bench's state machine (CEPCell_NEO/modules/
cipa_drug_bench.cpp:225-330, records cipa_t, commons.hpp:18-36), and the
qInward ratio (cipa_drug_bench.cpp:376) on control/drug pairs.

Tolerances. FP64: times (APD90/50, CaD90/50) within 0.01 ms; the beat
integrals (qNet, INaL and ICaL AUCs) within 1e-9 relative; sampled
potentials (Vm peak, valley, diastolic) within 1e-6 mV (the trace bound);
dVm/dt max and repolarisation slope within 1e-6 relative; Ca peak,
valley and diastolic within 1e-9 relative; the steepest pace and the number
of eligible beats equal. Mixed: APD90, CaD90 within 0.1 ms and qNet within
1 % (the mixed path's stated bars), APD50 and CaD50 within 0.1 ms, the AUCs
and qInward within 1 %, potentials within 0.5 mV, slopes within 2 %, Ca
values within 1 %.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

TIME_KEYS = ("apd90", "apd50", "cad90", "cad50")


def _cases(model, seed, n_samples):
    rng = np.random.default_rng(seed)
    hw = 20 if model == "cipa2017" else 14
    rows, conc = [], []
    for _ in range(n_samples):
        h = np.zeros(hw)
        h[0:14:2] = 10 ** rng.uniform(-0.5, 1.5, 7)
        h[1:14:2] = rng.uniform(0.7, 1.5, 7)
        if model == "cipa2017":
            h[12] = h[13] = 0.0
            h[14:20] = [5e3, 2e-3, 0.9, 1e4, -40.0, 3.5e-5]
        cmax = 10 ** rng.uniform(-1, 0.5)
        for k in range(3):  # control, 1x, 3x
            rows.append(h)
            conc.append((0.0, 1.0, 3.0)[k] * cmax)
    return np.array(conc), np.array(rows)


def _oracle(oracle, model, conc, hill, n_pace, first_pace, dt, bcl):
    out = [None] * len(conc)

    def work(k):
        c = oracle.Cell(model, 0.0, conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        out[k], _ = c.run_biomarkers(dt, n_pace, first_pace, dt_write=1.0)

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(conc))]
    [t.start() for t in th]
    [t.join() for t in th]
    return out


def _gpu(cep, model, conc, hill, prec, n_pace, first_pace, dt, bcl):
    b = cep.Batch(model, len(conc), prec)
    b.init(conc=conc, hill=hill, quirks=True)
    b.set_pacing(bcl)
    b.set_protocol(dt, n_pace, first_pace, dt_write=1.0)
    b.run_to_end(50000)
    bm = b.biomarkers()
    structs = b.biomarker_structs()
    b.close()
    return bm, structs


def _check(bm, ref, prec):
    fp = prec == "fp64"
    for k, r in enumerate(ref):
        assert bm["status"][k] == 1, k
        assert bm["steepest_pace"][k] == r["steepest_pace"] or not fp, k
        assert bm["n_eligible"][k] == r["n_eligible"], k
        for key in TIME_KEYS:
            assert abs(bm[key][k] - r[key]) <= (0.01 if fp else 0.1), (key, k, bm[key][k], r[key])
        assert abs(bm["apd_tri"][k] - (r["apd90"] - r["apd50"])) <= (0.02 if fp else 0.2)
        assert abs(bm["cad_tri"][k] - (r["cad90"] - r["cad50"])) <= (0.02 if fp else 0.2)
        q = r["qnet"] / 1000.0
        for key, ref_v in (("qnet", q), ("inal_auc", r["inal_auc"]), ("ical_auc", r["ical_auc"])):
            tol = 1e-9 * max(abs(ref_v), 1e-12) if fp else 0.01 * abs(ref_v)
            assert abs(bm[key][k] - ref_v) <= tol, (key, k, bm[key][k], ref_v)
        for key in ("vm_peak", "vm_valley", "vm_dia"):
            assert abs(bm[key][k] - r[key]) <= (1e-6 if fp else 0.5), (key, k, bm[key][k], r[key])
        for key in ("dvmdt_max", "dvmdt_repol"):
            assert abs(bm[key][k] - r[key]) <= (1e-6 if fp else 0.02) * abs(r[key]), (key, k, bm[key][k], r[key])
        for key in ("ca_peak", "ca_valley", "ca_dia"):
            assert abs(bm[key][k] - r[key]) <= (1e-9 if fp else 0.01) * abs(r[key]), (key, k, bm[key][k], r[key])


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["ord2011", "cipa2017"])
def test_every_biomarker_field_fp64(cep, gpu, oracle, model):
    conc, hill = _cases(model, seed=41, n_samples=2)
    ref = _oracle(oracle, model, conc, hill, 4, 1, 0.005, 1000.0)
    bm, _ = _gpu(cep, model, conc, hill, "fp64", 4, 1, 0.005, 1000.0)
    _check(bm, ref, "fp64")


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["ord2011", "cipa2017"])
def test_every_biomarker_field_mixed(cep, gpu, oracle, model):
    conc, hill = _cases(model, seed=42, n_samples=2)
    ref = _oracle(oracle, model, conc, hill, 4, 1, 0.005, 1000.0)
    bm, _ = _gpu(cep, model, conc, hill, "mixed", 4, 1, 0.005, 1000.0)
    _check(bm, ref, "mixed")


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_qinward_of_control_drug_pairs(cep, gpu, oracle, prec):
    """cep_qinward on each sample's control (conc 0) and drug records equals
    ((INaL_auc_drug / INaL_auc_control) + (ICaL_auc_drug / ICaL_auc_control))
    / 2 from the oracle's AUCs (cipa_drug_bench.cpp:370-380)."""
    conc, hill = _cases("ord2011", seed=43, n_samples=2)
    ref = _oracle(oracle, "ord2011", conc, hill, 3, 1, 0.005, 1000.0)
    _, structs = _gpu(cep, "ord2011", conc, hill, prec, 3, 1, 0.005, 1000.0)
    for s in range(2):
        c = 3 * s
        for d in (c + 1, c + 2):
            qi = cep.qinward(structs[c], structs[d])
            qo = 0.5 * (ref[d]["inal_auc"] / ref[c]["inal_auc"] + ref[d]["ical_auc"] / ref[c]["ical_auc"])
            assert abs(qi - qo) <= (1e-9 if prec == "fp64" else 0.01) * abs(qo), (s, d, qi, qo)
            assert qi < 1.0  # the drug blocks INaL and ICaL


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_records_match_the_reference_bench(cep, gpu, prec):
    """The device's records against what the reference's own CiPA bench
    prints (tests/golden/cipa_bench_records.json: cipa_drug_bench.cpp over
    the oracle's ORd, 251 paces at BCL 500 ms, dt 0.02 ms, Dutta scaling,
    two Hill rows at a control and two drug concentrations), within this
    file's tolerances plus the printed rounding (5e-7)."""
    import json
    from pathlib import Path
    g = json.loads((Path(__file__).resolve().parent / "golden" / "cipa_bench_records.json").read_text())
    c, rec = g["case"], g["records"]
    concs = [0.0] + list(c["concs"])
    hill = np.repeat(np.array(c["hill"]), len(concs), axis=0)
    conc = np.tile(concs, len(c["hill"]))
    out = cep.run_population("ord2011", conc, hill, bcl=c["bcl"], dt=c["dt"], n_pace=c["num_pace"],
                             first_pace=c["num_pace"] - 250, precision=prec, celltype=c["celltype"], dutta=True,
                             quirks=False, dt_write=c["dt_write"], refine_above_vm=None)
    fp = prec == "fp64"
    t_tol, rel = (0.01, 1e-6) if fp else (0.1, 0.02)
    for k in range(len(conc)):
        i, key = k // len(concs), f"{conc[k]:.2f}"
        ap = [float(x) for x in rec[key]["ap"][i]]
        ca = [float(x) for x in rec[key]["ca"][i]]
        qn = [float(x) for x in rec[key]["qni"][i]]
        for got, want in ((out["apd90"][k], ap[5]), (out["apd50"][k], ap[6]), (out["cad90"][k], ca[3]),
                          (out["cad50"][k], ca[4])):
            assert abs(got - want) <= t_tol + 5e-7, (key, i, got, want)
        for got, want in ((out["dvmdt_max"][k], ap[2]), (out["dvmdt_repol"][k], ap[1])):
            assert abs(got - want) <= rel * abs(want) + 5e-7, (key, i, got, want)
        for got, want in ((out["vm_peak"][k], ap[3]), (out["vm_dia"][k], ap[4])):
            assert abs(got - want) <= (1e-6 if fp else 0.5) + 5e-7, (key, i, got, want)
        assert abs(out["qnet"][k] - qn[1]) <= (1e-9 if fp else 0.01) * abs(qn[1]) + 5e-7, (key, i)
        if fp:
            assert out["steepest_pace"][k] == int(ap[8])
