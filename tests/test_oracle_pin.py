"""Pin the CPU oracle: bitwise against the reference compiled from its own
sources (where oracle/_ref exists) and against the committed golden
fixtures generated from that reference (everywhere)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
ORD_CASES = sorted(GOLD.glob("ord_*.npz"))


@pytest.mark.parametrize("path", ORD_CASES, ids=lambda p: p.stem)
def test_ord_oracle_matches_reference_golden(oracle, path):
    g = np.load(path)
    c = oracle.Cell("ord2011", float(g["celltype"]), float(g["conc"]), g["hill"], is_dutta=bool(g["dutta"]),
                    quirks=True)
    c.set_pacing(float(g["bcl"]))
    assert np.array_equal(c.states, g["y0"])
    r, _ = c.rates(0.0)
    assert np.array_equal(r, g["rates0"]), "RATES at t=0 differ from the reference"
    t, v = c.run(0.0, float(g["dt"]), int(g["n_steps"]), int(g["stride"]))
    # the restatement follows the reference's evaluation order: bit-exact
    assert np.array_equal(v, g["v_trace"])
    assert np.array_equal(c.states, g["final_states"])
    assert t == float(g["t_final"])


@pytest.mark.parametrize("dutta", [0, 1])
@pytest.mark.parametrize("celltype", [0.0, 1.0, 2.0])
def test_ord_oracle_bitwise_vs_compiled_reference(oracle, dutta, celltype):
    if not oracle.ref_available("ord2011"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    rng = np.random.default_rng(int(celltype * 10 + dutta))
    hill = np.zeros(14)
    hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1::2] = rng.uniform(0.6, 1.8, 7)
    hill[6] = 0.0  # INa NA -> no block
    conc = 4.2
    r = oracle.RefCell("ord2011", celltype, conc, hill, is_dutta=bool(dutta))
    c = oracle.Cell("ord2011", celltype, conc, hill, is_dutta=bool(dutta), quirks=True)
    n = 60000
    t1, v1 = r.run(0.0, 0.005, n, 50)
    t2, v2 = c.run(0.0, 0.005, n, 50)
    assert np.array_equal(v1, v2)
    assert np.array_equal(r.states, c.states)


def test_ord_quirks_documented(oracle):
    """The quirk switch changes exactly what the oracle header documents:
    with no drug, no Dutta and celltype endo only the fcafp step differs."""
    a = oracle.Cell("ord2011", 0.0, 0.0, None, quirks=True)
    b = oracle.Cell("ord2011", 0.0, 0.0, None, quirks=False)
    a.set_pacing(1000.0)
    b.set_pacing(1000.0)
    a.run(0.0, 0.005, 4000)
    b.run(0.0, 0.005, 4000)
    d = np.abs(a.states - b.states)
    assert d[32] > 0  # fcafp (STATES index 32) uses 25 vs dt
    # celltype is honoured only without quirks
    e = oracle.Cell("ord2011", 1.0, 0.0, None, quirks=True)
    f = oracle.Cell("ord2011", 0.0, 0.0, None, quirks=True)
    e.run(0.0, 0.005, 2000)
    f.run(0.0, 0.005, 2000)
    assert np.array_equal(e.states, f.states)


def test_biomarker_state_machine_last_beat(oracle):
    """Last-beat biomarkers of the control ORd cell are physiological and
    self-consistent (APD90 > APD50 > 0, CaD90 > CaD50 > 0, qNet finite)."""
    c = oracle.Cell("ord2011", 0.0, 0.0, None, quirks=True)
    c.set_pacing(1000.0)
    bm, _ = c.run_biomarkers(0.005, 3, 2, dt_write=1.0)
    assert bm["status"] == 0 and bm["n_eligible"] == 1
    assert 150 < bm["apd90"] < 400 and 0 < bm["apd50"] < bm["apd90"]
    assert 0 < bm["cad50"] < bm["cad90"]
    assert bm["vm_peak"] > 0 and bm["dvmdt_max"] > 50
    assert np.isfinite(bm["qnet"])


CIPA_CASES = sorted(GOLD.glob("cipa_*.npz"))


@pytest.mark.parametrize("path", CIPA_CASES, ids=lambda p: p.stem)
def test_cipa_oracle_rates_match_reference_golden(oracle, path):
    """CiPA-ORd RATES of the oracle equal the reference computeRates bit for
    bit at every fixture state, and the oracle's fixed-step trajectory
    reproduces the fixture states exactly."""
    g = np.load(path)
    c = oracle.Cell("cipa2017", 0.0, float(g["conc"]), g["hill"], quirks=True)
    c.set_pacing(float(g["bcl"]))
    assert np.array_equal(c.states, g["states"][0])
    for t, st, rr in zip(g["times"], g["states"], g["ref_rates"]):
        c.y[: c.n] = st
        r, _ = c.rates(float(t))
        assert np.array_equal(r, rr), f"RATES differ at t={t}"
    c2 = oracle.Cell("cipa2017", 0.0, float(g["conc"]), g["hill"], quirks=True)
    c2.set_pacing(float(g["bcl"]))
    every = int(round((g["times"][1] - g["times"][0]) / float(g["dt"])))
    t = 0.0
    for k in range(1, len(g["times"])):
        for _ in range(every):
            c2.step(t, float(g["dt"]))
            t += float(g["dt"])
        assert np.array_equal(c2.states, g["states"][k])


def test_cipa_oracle_rates_bitwise_vs_compiled_reference(oracle):
    if not oracle.ref_available("cipa2017"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    rng = np.random.default_rng(17)
    hill = np.zeros(20)
    hill[0:14:2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1:14:2] = rng.uniform(0.6, 1.8, 7)
    hill[14:19] = [50.0, 0.002, 0.95, 300.0, -60.0]
    r = oracle.RefCell("cipa2017", 0.0, 1.5, hill)
    c = oracle.Cell("cipa2017", 0.0, 1.5, hill, quirks=True)
    assert np.array_equal(r.states, c.states)
    t = 0.0
    for k in range(60000):
        if k % 3000 == 0:
            r.states[:] = c.states
            r.L.ref_compute_rates(r.h, t)
            mr, _ = c.rates(t)
            assert np.array_equal(r.arr("rates", r.n), mr)
        c.step(t, 0.005)
        t += 0.005


def test_tt2006_oracle_matches_reference_golden(oracle):
    """ten Tusscher 2006 epi, single-cell build: V trace, final STATES and
    RATES at t = 0 equal the reference's bit for bit."""
    g = np.load(GOLD / "tt2006_single.npz")
    c = oracle.Cell("tt2006")
    assert np.array_equal(c.states, g["y0"])
    r, _ = c.rates(0.0)
    assert np.array_equal(r, g["rates0"])
    t, v = c.run(0.0, float(g["dt"]), int(g["n_steps"]), int(g["stride"]))
    assert np.array_equal(v, g["v_trace"])
    assert np.array_equal(c.states, g["final_states"])
    assert t == float(g["t_final"])


def test_tt2006_oracle_tissue_flag_matches_reference_golden(oracle):
    """The tissue build's stimulus: isS1 held for 1 ms, then released."""
    g = np.load(GOLD / "tt2006_tissue.npz")
    c = oracle.Cell("tt2006", tissue_stim=True)
    c.c.is_s1 = 1
    t, v1 = c.run(0.0, float(g["dt"]), int(g["n_on"]), int(g["stride"]))
    c.c.is_s1 = 0
    t, v2 = c.run(t, float(g["dt"]), int(g["n_off"]), int(g["stride"]))
    assert np.array_equal(np.concatenate([v1, v2]), g["v_trace"])
    assert np.array_equal(c.states, g["final_states"])


def test_tt2006_oracle_bitwise_vs_compiled_reference(oracle):
    if not oracle.ref_available("tt2006"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    r = oracle.RefCell("tt2006")
    c = oracle.Cell("tt2006")
    t1, v1 = r.run(0.0, 0.01, 150000, 50)
    t2, v2 = c.run(0.0, 0.01, 150000, 50)
    assert np.array_equal(v1, v2)
    assert np.array_equal(r.states, c.states)


TT04_CASES = sorted(GOLD.glob("tt2004_*.npz"))


@pytest.mark.parametrize("path", TT04_CASES, ids=lambda p: p.stem)
def test_tt2004_oracle_matches_reference_golden(oracle, path):
    """ten Tusscher 2004 (2004_b build): V trace, final STATES and RATES at
    t = 0 equal the reference's bit for bit (with the unassigned gmma at 0,
    the oracle's quirk setting)."""
    g = np.load(path)
    c = oracle.Cell("tt2004", 0.0, float(g["conc"]), g["hill"], quirks=True)
    assert np.array_equal(c.states, g["y0"])
    r, _ = c.rates(0.0)
    assert np.array_equal(r, g["rates0"])
    t, v = c.run(0.0, float(g["dt"]), int(g["n_steps"]), int(g["stride"]))
    assert np.array_equal(v, g["v_trace"])
    assert np.array_equal(c.states, g["final_states"])


def test_tt2004_oracle_bitwise_vs_compiled_reference(oracle):
    if not oracle.ref_available("tt2004"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    rng = np.random.default_rng(41)
    hill = np.zeros(14)
    hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1::2] = rng.uniform(0.6, 1.8, 7)
    r = oracle.RefCell("tt2004", 0.0, 0.8, hill)
    r.consts[27] = 0.0  # CONSTANTS[gmma], unassigned by the reference
    c = oracle.Cell("tt2004", 0.0, 0.8, hill, quirks=True)
    t1, v1 = r.run(0.0, 0.01, 120000, 50)
    t2, v2 = c.run(0.0, 0.01, 120000, 50)
    assert np.array_equal(v1, v2)
    assert np.array_equal(r.states, c.states)


TOMEK_CASES = sorted(GOLD.glob("tomek_*.npz"))


@pytest.mark.parametrize("path", TOMEK_CASES, ids=lambda p: p.stem)
def test_tomek_oracle_rates_match_reference_golden(oracle, path):
    """ToR-ORd RATES of the oracle equal the reference computeRates bit for
    bit at every fixture state (endo/epi/mid, with and without drug), and
    the oracle's fixed-step trajectory reproduces the fixture states."""
    g = np.load(path)
    c = oracle.Cell("tomek2019", float(g["celltype"]), float(g["conc"]), g["hill"], quirks=True)
    assert np.array_equal(c.states, g["states"][0])
    for t, st, rr in zip(g["times"], g["states"], g["ref_rates"]):
        c.y[: c.n] = st
        r, _ = c.rates(float(t))
        assert np.array_equal(r, rr), f"RATES differ at t={t}"
    c2 = oracle.Cell("tomek2019", float(g["celltype"]), float(g["conc"]), g["hill"], quirks=True)
    every = int(round((g["times"][1] - g["times"][0]) / float(g["dt"])))
    t = 0.0
    for k in range(1, len(g["times"])):
        for _ in range(every):
            c2.step(t, float(g["dt"]))
            t += float(g["dt"])
        assert np.array_equal(c2.states, g["states"][k])


@pytest.mark.parametrize("celltype", [0.0, 1.0, 2.0])
def test_tomek_oracle_rates_bitwise_vs_compiled_reference(oracle, celltype):
    if not oracle.ref_available("tomek2019"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    rng = np.random.default_rng(int(celltype) + 5)
    hill = np.zeros(14)
    hill[0::2] = 10 ** rng.uniform(-1, 2, 7)
    hill[1::2] = rng.uniform(0.6, 1.8, 7)
    r = oracle.RefCell("tomek2019", celltype, 1.1, hill)
    c = oracle.Cell("tomek2019", celltype, 1.1, hill, quirks=True)
    assert np.array_equal(r.states, c.states)
    t = 0.0
    for k in range(16000):  # 80 ms: stimulus, upstroke, early plateau
        if k % 1000 == 0:
            r.states[:] = c.states
            r.L.ref_compute_rates(r.h, t)
            assert np.array_equal(r.arr("rates", r.n), c.rates(t)[0])
        c.step(t, 0.005)
        t += 0.005


# ---------------------------------------------------------------- FEM
def _fem_cases():
    g = np.load(GOLD / "fem_elements.npz")
    dims = {"square": (4, 2), "hex": (8, 3), "tet": (4, 3)}
    out = []
    for k, kind in enumerate(g["kind"]):
        nn, dim = dims[str(kind)]
        out.append((str(kind), g["x"][k][:nn, :dim], g["A"][k][:nn, :nn], g["B"][k][:nn, :nn]))
    return out, float(g["dt"]), float(g["de"])


def test_fem_element_oracle_matches_reference_golden(oracle):
    """The oracle's element matrices (cepo_element) equal, bit for bit, the
    reference's Cfem::set_amat_bmat (fem.cpp:628-661) compiled from its own
    sources, for square, hex and tet elements at the origin, translated far
    from it, and distorted."""
    cases, dt, de = _fem_cases()
    assert len(cases) == 15
    for kind, x, A, B in cases:
        a, b = oracle.element(kind, x, de, dt)
        assert np.array_equal(a, A), kind
        assert np.array_equal(b, B), kind


def test_fem_grid_element_is_the_reference_origin_element(oracle):
    """The structured-grid assembly uses the reference's matrices of the
    element at the origin for every element; the reference's own matrices
    of a translated element differ from them only by the rounding of its
    node coordinates (eps |x| / h relative: the reference's operator is not
    translation invariant in the last bits)."""
    cases, dt, de = _fem_cases()
    for dim, kind in ((2, "square"), (3, "hex")):
        a, b = oracle.fem_element(dim, 0.025, dt, de)
        (x0, A0, B0), (xt, At, Bt) = [(x, A, B) for k, x, A, B in cases if k == kind][:2]
        assert np.array_equal(a, A0) and np.array_equal(b, B0)
        # the Jacobian sums coordinates of size |x| to get differences of
        # size h: its rounding is ~eps |x| / h relative
        scale = 4 * np.finfo(float).eps * np.abs(xt).max() / 0.025
        assert 0 < np.abs(At - A0).max() <= scale * np.abs(A0).max()
        assert np.abs(Bt - B0).max() <= scale * np.abs(B0).max()


@pytest.mark.parametrize("kind", ["square", "hex", "tet"])
def test_fem_element_bitwise_vs_compiled_reference(oracle, kind):
    if not oracle.ref_available("fem"):
        pytest.skip("reference not compiled here (oracle/_ref); golden fixtures cover this")
    rng = np.random.default_rng({"square": 1, "hex": 2, "tet": 3}[kind])
    h = 0.02
    base = {"square": [[0, 0], [h, 0], [h, h], [0, h]],
            "hex": [[0, 0, 0], [h, 0, 0], [h, h, 0], [0, h, 0], [0, 0, h], [h, 0, h], [h, h, h], [0, h, h]],
            "tet": [[0, 0, 0], [h, 0, 0], [0, h, 0], [0, 0, h]]}[kind]
    x0 = np.array(base, float)
    for trial in range(20):
        x = x0 + rng.uniform(-0.3, 0.3, x0.shape) * h + rng.uniform(-5, 5)
        de, dt = rng.uniform(5e-4, 3e-3), rng.choice([0.005, 0.01, 0.02])
        A, B = oracle.ref_fem_element(kind, x, de, dt)
        a, b = oracle.element(kind, x, de, dt)
        assert np.array_equal(a, A) and np.array_equal(b, B), (kind, trial)


# ------------------------------------------------------- biomarker machine
def _c_float(x: float) -> str:
    """A double as C's printf("%lf") writes it."""
    if x != x:
        return "-nan" if np.signbit(x) else "nan"
    return f"{x:.6f}"


def test_biomarker_machine_matches_reference_bench(oracle):
    """The oracle's restatement of the CiPA bench's biomarker state machine
    prints exactly what the reference's own bench prints. The goldens come
    from cipa_drug_bench.cpp compiled from its sources and run over the
    oracle's ORd 2011 (oracle/ref_shim/bench_shim.cpp: the CVODE call
    replaced by one fixed step of the oracle's scheme), 251 paces so that
    its last-250-paces evaluation runs: every field of ap_profile,
    ca_profile and qni (APD90/50/triangulation, dVm/dt max and repolarising,
    Vm peak and diastolic, Ca peak / diastolic, CaD90/50/triangulation,
    qNet, qInward) and the steepest pace, for two Hill rows at a control and
    two drug concentrations."""
    import json
    import threading
    g = json.loads((GOLD / "cipa_bench_records.json").read_text())
    c, rec = g["case"], g["records"]
    concs = [0.0] + list(c["concs"])
    res = {}

    def work(i, conc):
        cell = oracle.Cell("ord2011", c["celltype"], conc, np.array(c["hill"][i]), is_dutta=True, quirks=False)
        cell.set_pacing(c["bcl"])
        res[(i, conc)], _ = cell.run_biomarkers(c["dt"], c["num_pace"], c["num_pace"] - 250, dt_write=c["dt_write"])

    th = [threading.Thread(target=work, args=(i, conc)) for i in range(len(c["hill"])) for conc in concs]
    [t.start() for t in th]
    [t.join() for t in th]
    for i in range(len(c["hill"])):
        ctrl = res[(i, 0.0)]
        for conc in concs:
            r = res[(i, conc)]
            key = f"{conc:.2f}"
            ap, ca, qni = rec[key]["ap"][i], rec[key]["ca"][i], rec[key]["qni"][i]
            assert ap == [str(i), _c_float(r["dvmdt_repol"]), _c_float(r["dvmdt_max"]), _c_float(r["vm_peak"]),
                          _c_float(r["vm_dia"]), _c_float(r["apd90"]), _c_float(r["apd50"]),
                          _c_float(r["apd90"] - r["apd50"]), str(r["steepest_pace"])], (key, i, ap)
            assert ca == [str(i), _c_float(r["ca_peak"]), _c_float(r["ca_dia"]), _c_float(r["cad90"]),
                          _c_float(r["cad50"]), _c_float(r["cad90"] - r["cad50"]), str(r["steepest_pace"])], (key, i)
            qin = 0.0 if conc == 0.0 else 0.5 * (r["inal_auc"] / ctrl["inal_auc"] + r["ical_auc"] / ctrl["ical_auc"])
            assert qni == [str(i), _c_float(r["qnet"] / 1000.0), _c_float(qin)], (key, i, qni)


# ------------------------------------------------ CEPCell_NEO ORd, HRV bench
NEO_CASES = sorted(GOLD.glob("neo_ord_*.npz"))


@pytest.mark.parametrize("path", NEO_CASES, ids=lambda p: p.stem)
def test_ord_neo_rates_match_reference_golden(oracle, path):
    """The oracle's CEPCell_NEO ORd 2011 variant (quirks 2: celltype kept,
    Dutta on the intended constants, PCa-derived permeabilities not rescaled,
    the HRV stimulus window at cumm_BCL) gives, bit for bit, the RATES of the
    reference's CEPCell_NEO build compiled from its sources."""
    import ctypes
    g = np.load(path)
    c = oracle.Cell("ord2011", float(g["celltype"]), float(g["conc"]), g["hill"], is_dutta=bool(g["dutta"]),
                    quirks=2)
    c.c.tissue_stim = 2
    for t, cumm, y, r in zip(g["times"], g["cumm"], g["states"], g["ref_rates"]):
        c.y[:41] = y
        oracle.lib().cepo_ord_set_cumm(ctypes.byref(c.c), float(cumm))
        ro, _ = c.rates(float(t))
        assert np.array_equal(ro, r), (float(t), np.flatnonzero(ro != r))


def test_hrv_bench_matches_reference(oracle):
    """The oracle's restatement of the HRV bench prints exactly what the
    reference's hrv_bench.cpp (compiled from its sources over the oracle's
    CEPCell_NEO ORd) prints: every field of ap_profile (BCL of the chosen
    beat included), ca_profile and qni, for a control and a drug, over 259
    intervals plus the appended 1000 ms, with the zero-length first call of
    every pace."""
    import json
    import threading
    g = json.loads((GOLD / "hrv_bench_records.json").read_text())
    c, bcls, rec = g["case"], g["bcls"] + [1000.0], g["records"]
    concs = [0.0] + list(c["concs"])
    res = {}

    def work(conc):
        cell = oracle.Cell("ord2011", c["celltype"], conc, np.array(c["hill"]), is_dutta=True, quirks=2)
        res[conc] = cell.hrv(bcls, c["dt"], c["dt_write"])

    th = [threading.Thread(target=work, args=(x,)) for x in concs]
    [t.start() for t in th]
    [t.join() for t in th]
    ctrl = res[0.0]
    for conc in concs:
        r = res[conc]
        key = f"{conc:.2f}"
        assert rec[key]["ap"][0] == ["0", _c_float(r["dvmdt_repol"]), _c_float(r["dvmdt_max"]), _c_float(r["vm_peak"]),
                                     _c_float(r["vm_dia"]), _c_float(r["apd90"]), _c_float(r["apd50"]),
                                     _c_float(r["apd90"] - r["apd50"]), str(r["steepest_pace"]), str(r["bcl"])], key
        assert rec[key]["ca"][0] == ["0", _c_float(r["ca_peak"]), _c_float(r["ca_dia"]), _c_float(r["cad90"]),
                                     _c_float(r["cad50"]), _c_float(r["cad90"] - r["cad50"]),
                                     str(r["steepest_pace"])], key
        qin = 0.0 if conc == 0.0 else 0.5 * (r["inal_auc"] / ctrl["inal_auc"] + r["ical_auc"] / ctrl["ical_auc"])
        assert rec[key]["qni"][0] == ["0", _c_float(r["qnet"] / 1000.0), _c_float(qin)], key
