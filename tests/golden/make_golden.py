"""Generate the golden fixtures in tests/golden/ from the reference cell
models compiled from their own sources (oracle/_ref, built by
`make -C oracle ref` where the reference tree is present).

    python tests/golden/make_golden.py [ord cipa tt2006 tt2004 tomek fem bench neo hrv]

Each fixture holds the inputs (celltype, concentration, Hill row, flags),
the reference's V trace sampled every `stride` steps of its explicit loop
(computeRates(t); solveAnalytical(dt); t += dt), its final STATES, and its
RATES at t = 0. fem_elements.npz holds the reference's FEM element
matrices (fem.cpp set_amat_bmat) of square, hex and tet elements;
cipa_bench_records.json the records the reference's CiPA drug bench prints
(cipa_drug_bench.cpp) for the oracle's ORd trajectory; neo_ord_*.npz the
RATES of the CEPCell_NEO ORd build; hrv_bench_records.json the records of
the reference's HRV bench (hrv_bench.cpp). The
oracle and the GPU path are checked against these files on machines where
the reference itself is not available.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def hill_row(rng: np.random.Generator, skip: tuple[int, ...] = ()) -> np.ndarray:
    """Seeded Hill row: IC50 log-uniform in [0.1, 100] uM, h uniform in
    [0.6, 1.8] (the single-cell configuration's ranges)."""
    h = np.zeros(14)
    h[0::2] = 10 ** rng.uniform(-1, 2, 7)
    h[1::2] = rng.uniform(0.6, 1.8, 7)
    for ch in skip:
        h[2 * ch] = 0.0  # NA in the reference CSV -> 0 -> no block
    return h


def ord_cases():
    rng = np.random.default_rng(20240611)
    return [
        dict(name="ord_control", celltype=0.0, conc=0.0, hill=np.zeros(14), dutta=0),
        dict(name="ord_drug_dutta", celltype=0.0, conc=3.0, hill=hill_row(rng), dutta=1),
        dict(name="ord_drug_epi_skip", celltype=1.0, conc=10.0, hill=hill_row(rng, skip=(2,)), dutta=0),
        dict(name="ord_drug_mcell_dutta", celltype=2.0, conc=0.7, hill=hill_row(rng), dutta=1),
    ]


def make_ord(n_beats: int = 2, dt: float = 0.005, stride: int = 200, bcl: float = 1000.0):
    for c in ord_cases():
        r = O.RefCell("ord2011", c["celltype"], c["conc"], c["hill"], is_dutta=bool(c["dutta"]))
        r.consts[140] = bcl  # CONSTANTS[BCL]
        y0 = r.states.copy()
        r.L.ref_compute_rates(r.h, 0.0)
        rates0 = r.arr("rates", r.n).copy()
        n = int(round(n_beats * bcl / dt))
        t, v = r.run(0.0, dt, n, stride)
        np.savez_compressed(OUT / f"{c['name']}.npz", celltype=c["celltype"], conc=c["conc"], hill=c["hill"],
                            dutta=c["dutta"], dt=dt, stride=stride, bcl=bcl, n_steps=n, y0=y0, rates0=rates0,
                            v_trace=v, final_states=r.states.copy(), t_final=t)
        print("wrote", c["name"], "vmax", v.max())


def cipa_hill(rng: np.random.Generator) -> np.ndarray:
    """Seeded CiPA row: seven IC50/h pairs (hERG static block off: the
    dynamic model carries it), then Kmax, Ku, n, halfmax, Vhalf, Kt."""
    h = hill_row(rng)
    h[12] = h[13] = 0.0
    halfmax = 10 ** rng.uniform(3, 6)
    dyn = [halfmax * 10 ** rng.uniform(-1, 1), 10 ** rng.uniform(-4, -2), rng.uniform(0.8, 1.0), halfmax,
           rng.uniform(-100, -10), 3.5e-5]
    return np.concatenate([h, dyn])


def make_cipa(dt: float = 0.005, bcl: float = 1000.0, n_steps: int = 200000, every: int = 10000):
    """CiPA-ORd: the reference has no fixed-step integrator, so the fixture
    holds states along the oracle's fixed-step trajectory and the
    reference's RATES at each of them."""
    rng = np.random.default_rng(99)
    cases = [dict(name="cipa_control", conc=0.0, hill=np.zeros(20)),
             dict(name="cipa_drug", conc=2.5, hill=cipa_hill(rng))]
    for c in cases:
        r = O.RefCell("cipa2017", 0.0, c["conc"], c["hill"])
        cell = O.Cell("cipa2017", 0.0, c["conc"], c["hill"], quirks=True)
        cell.set_pacing(bcl)
        r.consts[15] = bcl  # CONSTANTS[stim_period]
        if c["hill"][19] > 1e-13:
            r.consts[100] = c["hill"][19]  # CONSTANTS[Kt]: the reference has no hill slot for it
        states, rates, times = [], [], []
        t = 0.0
        for k in range(n_steps):
            if k % every == 0:
                r.states[:] = cell.states
                r.L.ref_compute_rates(r.h, t)
                states.append(cell.states.copy())
                rates.append(r.arr("rates", r.n).copy())
                times.append(t)
            cell.step(t, dt)
            t += dt
        np.savez_compressed(OUT / f"{c['name']}.npz", conc=c["conc"], hill=c["hill"], dt=dt, bcl=bcl,
                            times=np.array(times), states=np.array(states), ref_rates=np.array(rates),
                            y0=r.states.copy() * 0 + np.array(states)[0])
        print("wrote", c["name"])


def make_tt2006(dt: float = 0.01, stride: int = 100):
    """ten Tusscher 2006 epi: the single-cell build (periodic stimulus, two
    1000-ms beats) and the tissue build (isS1 held for the first 1 ms, then
    released; 300 ms). The reference model has no drug hook."""
    r = O.RefCell("tt2006")
    y0 = r.states.copy()
    r.L.ref_compute_rates(r.h, 0.0)
    rates0 = r.arr("rates", r.n).copy()
    n = int(round(2000.0 / dt))
    t, v = r.run(0.0, dt, n, stride)
    np.savez_compressed(OUT / "tt2006_single.npz", dt=dt, stride=stride, n_steps=n, y0=y0, rates0=rates0,
                        v_trace=v, final_states=r.states.copy(), t_final=t)
    print("wrote tt2006_single vmax", v.max())
    r = O.RefCell("tt2006_tissue")
    r.L.ref_set_s1(r.h, 1)
    n_on = int(round(1.0 / dt))
    t, v1 = r.run(0.0, dt, n_on, stride)
    r.L.ref_set_s1(r.h, 0)
    n_off = int(round(299.0 / dt))
    t, v2 = r.run(t, dt, n_off, stride)
    np.savez_compressed(OUT / "tt2006_tissue.npz", dt=dt, stride=stride, n_on=n_on, n_off=n_off,
                        v_trace=np.concatenate([v1, v2]), final_states=r.states.copy(), t_final=t)
    print("wrote tt2006_tissue vmax", max(v1.max(), v2.max()))


def make_tt2004(dt: float = 0.01, stride: int = 100):
    """ten Tusscher 2004 (the reference's 2004_b build, every channel on):
    control and a seeded drug row, two 1000-ms beats each. The reference
    leaves CONSTANTS[gmma] unassigned; the fixture sets it to 0, the value
    the reference's heap held when it was built here (a denormal that acts
    as 0)."""
    rng = np.random.default_rng(2004)
    cases = [dict(name="tt2004_control", conc=0.0, hill=np.zeros(14)),
             dict(name="tt2004_drug", conc=2.0, hill=hill_row(rng))]
    for c in cases:
        r = O.RefCell("tt2004", 0.0, c["conc"], c["hill"])
        r.consts[27] = 0.0  # CONSTANTS[gmma]
        y0 = r.states.copy()
        r.L.ref_compute_rates(r.h, 0.0)
        rates0 = r.arr("rates", r.n).copy()
        n = int(round(2000.0 / dt))
        t, v = r.run(0.0, dt, n, stride)
        np.savez_compressed(OUT / f"{c['name']}.npz", conc=c["conc"], hill=c["hill"], dt=dt, stride=stride,
                            n_steps=n, y0=y0, rates0=rates0, v_trace=v, final_states=r.states.copy(), t_final=t)
        print("wrote", c["name"], "vmax", v.max())


def make_tomek(dt: float = 0.005, n_steps: int = 200000, every: int = 10000):
    """ToR-ORd: the reference has no fixed-step integrator (its
    solveAnalytical is empty), so like CiPA the fixture holds states along
    the oracle's fixed-step trajectory and the reference's RATES at each of
    them; endo control, epi with a drug row, mid with a drug row."""
    rng = np.random.default_rng(2019)
    cases = [dict(name="tomek_endo_control", celltype=0.0, conc=0.0, hill=np.zeros(14)),
             dict(name="tomek_epi_drug", celltype=1.0, conc=1.5, hill=hill_row(rng)),
             dict(name="tomek_mid_drug", celltype=2.0, conc=0.6, hill=hill_row(rng))]
    for c in cases:
        r = O.RefCell("tomek2019", c["celltype"], c["conc"], c["hill"])
        cell = O.Cell("tomek2019", c["celltype"], c["conc"], c["hill"], quirks=True)
        states, rates, times = [], [], []
        t = 0.0
        for k in range(n_steps):
            if k % every == 0:
                r.states[:] = cell.states
                r.L.ref_compute_rates(r.h, t)
                states.append(cell.states.copy())
                rates.append(r.arr("rates", r.n).copy())
                times.append(t)
            cell.step(t, dt)
            t += dt
        np.savez_compressed(OUT / f"{c['name']}.npz", celltype=c["celltype"], conc=c["conc"], hill=c["hill"], dt=dt,
                            times=np.array(times), states=np.array(states), ref_rates=np.array(rates))
        print("wrote", c["name"])


def fem_element_cases(seed: int = 20):
    """Element node coordinates of each kind: the grid element at the
    origin (edge 0.025 cm), one translated far from it, and distorted ones."""
    rng = np.random.default_rng(seed)
    h = 0.025
    base = {"square": np.array([[0, 0], [h, 0], [h, h], [0, h]], float),
            "hex": np.array([[0, 0, 0], [h, 0, 0], [h, h, 0], [0, h, 0], [0, 0, h], [h, 0, h], [h, h, h], [0, h, h]],
                            float),
            "tet": np.array([[0, 0, 0], [h, 0, 0], [0, h, 0], [0, 0, h]], float)}
    cases = []
    for kind, x in base.items():
        cases.append((kind, x.copy()))
        cases.append((kind, x + 7.3))
        for _ in range(3):
            cases.append((kind, x + rng.uniform(-0.25, 0.25, x.shape) * h + rng.uniform(-3, 3)))
    return cases


def make_fem(dt: float = 0.01, de: float = 0.0013):
    """The reference's element matrices (fem.cpp set_amat_bmat, compiled from
    fem.cpp) for every case of fem_element_cases()."""
    kinds, xs, As, Bs = [], [], [], []
    for kind, x in fem_element_cases():
        a, b = O.ref_fem_element(kind, x, de, dt)
        kinds.append(kind)
        xs.append(np.pad(x, ((0, 8 - len(x)), (0, 3 - x.shape[1]))))
        As.append(np.pad(a, ((0, 8 - len(a)), (0, 8 - len(a)))))
        Bs.append(np.pad(b, ((0, 8 - len(b)), (0, 8 - len(b)))))
    np.savez_compressed(OUT / "fem_elements.npz", kind=np.array(kinds), x=np.array(xs), A=np.array(As),
                        B=np.array(Bs), dt=dt, de=de)
    print("wrote fem_elements")


BENCH_CASE = dict(celltype=0.0, bcl=500.0, dt=0.02, dt_write=1.0, num_pace=251, concs=[1.5, 0.3],
                  hill=[[5.0, 1.0, 20.0, 1.1, 30.0, 0.9, 8.0, 1.2, 4.0, 0.8, 15.0, 1.0, 0.6, 1.1],
                        [2.5, 0.9, 60.0, 1.0, 10.0, 1.3, 40.0, 0.7, 1.2, 1.1, 80.0, 0.6, 3.0, 0.8]])


def make_bench():
    """The reference's CiPA drug bench (cipa_drug_bench.cpp compiled from its
    sources, run over the oracle's ORd with a fixed-step CVode stand-in) on
    BENCH_CASE: its printed records (ap_profile, ca_profile, qni) as text."""
    import json
    import tempfile
    c = BENCH_CASE
    with tempfile.TemporaryDirectory() as wd:
        rec = O.ref_cipa_bench(wd, c["hill"], c["concs"], c["celltype"], c["bcl"], c["dt"], c["dt_write"],
                               c["num_pace"])
    (OUT / "cipa_bench_records.json").write_text(json.dumps(dict(case=c, records=rec), indent=1))
    print("wrote cipa_bench_records")


NEO_CASES = [dict(celltype=0.0, dutta=True, conc=1.5), dict(celltype=1.0, dutta=True, conc=0.7),
             dict(celltype=2.0, dutta=False, conc=3.0)]
NEO_HILL = [5.0, 1.0, 20.0, 1.1, 30.0, 0.9, 8.0, 1.2, 4.0, 0.8, 15.0, 1.0, 0.6, 1.1]


def make_ord_neo(dt: float = 0.005, n_steps: int = 60000, every: int = 1000):
    """RATES of the CEPCell_NEO build of ORd 2011 (compiled from its own
    sources, HRV stimulus on) at states along the oracle's trajectory, the
    stimulus window moved to cumm_BCL = 150 ms halfway."""
    import ctypes
    for k, c in enumerate(NEO_CASES):
        r = O.RefCell("ord2011_neo", c["celltype"], c["conc"], np.array(NEO_HILL), is_dutta=c["dutta"])
        r.L.ref_set_hrv.argtypes = [ctypes.c_int]
        r.L.ref_set_hrv(1)
        cell = O.Cell("ord2011", c["celltype"], c["conc"], np.array(NEO_HILL), is_dutta=c["dutta"], quirks=2)
        cell.c.tissue_stim = 2
        t, cumm = 0.0, 0.0
        times, cumms, states, rates = [], [], [], []
        for i in range(n_steps):
            if i == n_steps // 2:
                cumm = 150.0
            if i % every == 0:
                r.states[:] = cell.states
                r.consts[141] = cumm
                r.L.ref_compute_rates(r.h, t)
                times.append(t); cumms.append(cumm); states.append(cell.states.copy())
                rates.append(r.arr("rates", r.n).copy())
            O.lib().cepo_ord_set_cumm(ctypes.byref(cell.c), cumm)
            cell.step(t, dt)
            t += dt
        np.savez_compressed(OUT / f"neo_ord_{k}.npz", hill=np.array(NEO_HILL), dt=dt, times=np.array(times),
                            cumm=np.array(cumms), states=np.array(states), ref_rates=np.array(rates), **c)
        print("wrote", f"neo_ord_{k}")


HRV_CASE = dict(celltype=0.0, dt=0.02, dt_write=1.0, concs=[1.5], hill=NEO_HILL, n_bcl=259, seed=3)


def hrv_bcls(case=HRV_CASE) -> list[float]:
    """The HRV file's intervals: a seeded slow oscillation with noise (ms,
    one decimal), n_bcl of them."""
    rng = np.random.default_rng(case["seed"])
    n = case["n_bcl"]
    return [float(x) for x in np.round(600 + 80 * np.sin(np.arange(n) / 7.0) + rng.normal(0, 20, n), 1)]


def make_hrv():
    """The reference's HRV bench (hrv_bench.cpp compiled from its sources
    over the oracle's ORd, CEPCell_NEO build) on HRV_CASE: its printed
    records as text."""
    import ctypes
    import json
    import tempfile
    c = HRV_CASE
    L = ctypes.CDLL(str(O.REF_DIR / O.REF_LIBS["bench"]))
    L.ref_hrv_bench.argtypes = [ctypes.c_char_p] * 5 + [ctypes.c_double] * 3 + [ctypes.c_int]
    bcls = hrv_bcls()
    with tempfile.TemporaryDirectory() as wd:
        w = Path(wd)
        (w / "result").mkdir()
        (w / "hrv.txt").write_text("".join(f"{b}\n" for b in bcls))
        (w / "hill.csv").write_text("header\n" + ",".join(repr(x) for x in c["hill"]) + "\n")
        concs = "0," + ",".join(repr(x) for x in c["concs"])
        rc = L.ref_hrv_bench(str(w).encode(), str(w / "hill.csv").encode(), str(w / "hrv.txt").encode(),
                             concs.encode(), b"hrv", c["celltype"], c["dt"], c["dt_write"], len(bcls) + 1)
        assert rc == 0
        rec = {}
        for f in sorted((w / "result").glob("*/*.plt")):
            kind = "ap" if "ap_profile" in f.name else "ca" if "ca_profile" in f.name else "qni"
            rec.setdefault(f.parent.name, {})[kind] = [ln.split() for ln in f.read_text().strip().splitlines()[1:]]
    (OUT / "hrv_bench_records.json").write_text(json.dumps(dict(case=c, bcls=bcls, records=rec), indent=1))
    print("wrote hrv_bench_records")


if __name__ == "__main__":
    if not O.ref_available("ord2011"):
        sys.exit("reference models not built: run `make -C oracle ref` where the reference tree exists")
    which = set(sys.argv[1:]) or {"ord", "cipa", "tt2006", "tt2004", "tomek", "fem", "bench", "neo", "hrv"}
    if "ord" in which:
        make_ord()
    if "cipa" in which:
        make_cipa()
    if "tt2006" in which:
        make_tt2006()
    if "tt2004" in which:
        make_tt2004()
    if "tomek" in which:
        make_tomek()
    if "fem" in which:
        make_fem()
    if "bench" in which:
        make_bench()
    if "neo" in which:
        make_ord_neo()
    if "hrv" in which:
        make_hrv()
