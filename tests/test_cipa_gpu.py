"""CiPA-ORd v1 2017 (dynamic hERG) on the GPU against the oracle.

The reference integrates this model only with CVODE; parity here is against
the oracle's fixed-step scheme (the reference's ORd update scheme applied to
this model, with the reference's computeRates pinned bit for bit).
Tolerances as in test_ord_gpu.py.
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


def cipa_population(n_samples: int, n_conc: int, seed: int):
    """Seeded CiPA population: a nominal drug (IC50 log-U[0.1,100] uM,
    h U[0.6,1.8], static hERG block off, dynamic hERG Kmax/Ku/n/halfmax/
    Vhalf seeded, Kt = 3.5e-5), samples lognormal around it (sigma 0.5 in
    ln-space), concentrations 0..n_conc-1 x Cmax."""
    rng = np.random.default_rng(seed)
    nom = np.zeros(20)
    nom[0:14:2] = 10 ** rng.uniform(-1, 2, 7)
    nom[1:14:2] = rng.uniform(0.6, 1.8, 7)
    halfmax = 10 ** rng.uniform(3, 6)
    nom[14:20] = [halfmax * 10 ** rng.uniform(-1, 1), 10 ** rng.uniform(-4, -2), rng.uniform(0.8, 1.0), halfmax,
                  rng.uniform(-100, -10), 3.5e-5]
    nom[12] = nom[13] = 0.0
    cmax = 10 ** rng.uniform(-2, 1)
    hill = np.repeat(nom[None, :], n_samples, axis=0)
    pert = np.exp(0.5 * rng.standard_normal((n_samples, 20)))
    pert[:, 12:14] = 1.0
    pert[:, 18:20] = 1.0  # Vhalf and Kt stay nominal
    hill = hill * pert
    hill = np.repeat(hill, n_conc, axis=0)
    conc = np.tile(np.arange(n_conc) * cmax, n_samples)
    return conc, hill


def _oracle(oracle, conc, hill, n_pace, first_pace, dt, bcl):
    out = [None] * len(conc)

    def work(k):
        c = oracle.Cell("cipa2017", 0.0, conc[k], hill[k], quirks=True)
        c.set_pacing(bcl)
        bm, _ = c.run_biomarkers(dt, n_pace, first_pace, dt_write=1.0)
        bm["final"] = c.states.copy()
        out[k] = bm

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(conc))]
    [t.start() for t in th]
    [t.join() for t in th]
    return out


def _gpu(cep, conc, hill, precision, n_pace, first_pace, dt, bcl):
    b = cep.Batch("cipa2017", len(conc), precision)
    b.init(conc=conc, hill=hill, quirks=True)
    b.set_pacing(bcl)
    b.set_protocol(dt, n_pace, first_pace, dt_write=1.0)
    b.run_to_end(50000)
    return b.biomarkers(), b.get_states()


@pytest.mark.gpu
def test_cipa_fp64_trace_matches_oracle(cep, gpu, oracle):
    conc, hill = cipa_population(2, 2, seed=3)
    n = len(conc)
    b = cep.Batch("cipa2017", n, "fp64")
    b.init(conc=conc, hill=hill, quirks=True)
    b.set_pacing(1000.0)
    cells = []
    for k in range(n):
        c = oracle.Cell("cipa2017", 0.0, conc[k], hill[k], quirks=True)
        c.set_pacing(1000.0)
        cells.append(c)
    y0 = b.get_states()
    for k in range(n):
        assert np.array_equal(y0[k], cells[k].states)
    stride, n_chunks = 400, 500  # 1000 ms
    vg = np.zeros((n_chunks, n))
    vo = np.zeros((n_chunks, n))
    t = 0.0
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
    fin = b.get_states()
    for k in range(n):
        rel = np.abs(fin[k] - cells[k].states) / np.maximum(np.abs(cells[k].states), 1e-9)
        assert rel.max() < 1e-5


@pytest.mark.gpu
def test_cipa_biomarkers_fp64_and_mixed(cep, gpu, oracle):
    """Steepest-repolarisation selection over the evaluated paces (the
    reference's last-250-paces rule, here the last 3 of 4 paces)."""
    conc, hill = cipa_population(3, 3, seed=8)
    ref = _oracle(oracle, conc, hill, 4, 1, 0.005, 1000.0)
    b64, s64 = _gpu(cep, conc, hill, "fp64", 4, 1, 0.005, 1000.0)
    bmx, _ = _gpu(cep, conc, hill, "mixed", 4, 1, 0.005, 1000.0)
    for k, r in enumerate(ref):
        assert b64["status"][k] == cep.INST_DONE
        assert abs(s64[k, 0] - r["final"][0]) <= VM_TOL_FP64
        assert b64["steepest_pace"][k] == r["steepest_pace"]
        for key in ("apd90", "apd50", "cad90", "cad50"):
            assert abs(b64[key][k] - r[key]) <= APD_TOL_FP64, (key, k, b64[key][k], r[key])
        assert abs(b64["qnet"][k] - r["qnet"] / 1000) <= 1e-9 * max(1.0, abs(r["qnet"]))
        assert abs(bmx["apd90"][k] - r["apd90"]) <= APD_TOL_MIXED, (k, bmx["apd90"][k], r["apd90"])
        assert abs(bmx["cad90"][k] - r["cad90"]) <= CAD_TOL_MIXED, (k, bmx["cad90"][k], r["cad90"])
        q = r["qnet"] / 1000
        assert abs(bmx["qnet"][k] - q) <= QNET_RTOL_MIXED * abs(q), (k, bmx["qnet"][k], q)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cipa_stiff_drug_binding_stays_finite(cep, gpu, oracle, precision):
    """A sample whose binding Hill coefficient (3.4) and concentration give a
    drug-binding rate of ~780 /ms: one forward-Euler step of the Markov chain
    is unstable at dt = 0.005 ms; the substepped update keeps it finite and
    on the oracle's trajectory."""
    hill = np.array([97.0292, 0.8377, 0.9136, 0.7587, 54.8446, 0.5487, 0.3744, 1.076, 0.8283, 2.6202,
                     0.1226, 3.6055, 0.0, 0.0, 375209.231, 0.0082, 3.4183, 40305.2473, -84.514, 3.5e-5])
    conc = 16.341988810388337
    b = cep.Batch("cipa2017", 1, precision)
    b.init(conc=conc, hill=hill, quirks=True)
    b.set_pacing(2000.0)
    b.run(80000)
    st = b.get_states()[0]
    assert np.isfinite(st).all() and b.status()[0] == cep.INST_RUNNING
    c = oracle.Cell("cipa2017", 0.0, conc, hill, quirks=True)
    c.set_pacing(2000.0)
    c.run(0.0, 0.005, 80000)
    tol = VM_TOL_FP64 if precision == "fp64" else 0.5
    assert abs(st[0] - c.states[0]) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["cipa2017", "ord2011"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_roles_kernel_matches_cell_kernel(cep, gpu, model, precision):
    """The warp-specialised kernels (4 or 2 warps per 32 cells) and the
    one-thread-per-cell kernel compute the same trajectory and biomarkers
    (the roles' contributions are added in the same order in both)."""
    conc, hill = cipa_population(20, 3, seed=21)  # 60 instances: two blocks, one partial
    if model == "ord2011":
        hill = hill[:, :14].copy()
    out = {}
    for kern in ("cell", "roles", "pairs"):
        b = cep.Batch(model, len(conc), precision)
        b.set_kernel(kern)
        b.init(conc=conc, hill=hill, quirks=True)
        b.set_pacing(1000.0)
        b.set_protocol(0.005, 2, 1, dt_write=1.0)
        b.run_to_end(30000)
        out[kern] = (b.get_states(), b.biomarkers())
    s0, b0 = out["cell"]
    tol = 1e-9 if precision == "fp64" else 1e-4
    for kern in ("roles", "pairs"):
        s1, b1 = out[kern]
        assert np.abs(s0[:, 0] - s1[:, 0]).max() <= tol, kern
        for key in ("apd90", "apd50", "cad90"):
            assert np.abs(b0[key] - b1[key]).max() <= 0.01, (kern, key)
        assert np.array_equal(b0["status"], b1["status"]), kern


@pytest.mark.gpu
def test_autotune_keeps_the_batch_state(cep, gpu):
    """cep_batch_autotune part-way through a protocol: the state, clocks and
    biomarker bookkeeping continue exactly where they were, and the run
    then ends within the mixed bars of a batch left on the default form."""
    conc, hill = cipa_population(100, 5, seed=4)

    def make():
        b = cep.Batch("cipa2017", len(conc), "mixed")
        b.init(conc=conc, hill=hill, quirks=True)
        b.set_pacing(1000.0)
        b.set_protocol(0.005, 2, 1, dt_write=1.0)
        return b

    a = make()
    a.run(30000)
    s0, clk0 = a.get_states(), a.clock(0)
    form, block = a.autotune(300)
    assert form in ("cell", "roles", "pairs") and block in (32, 64, 96, 128)
    assert np.array_equal(a.get_states(), s0) and a.clock(0) == clk0
    a.run_to_end(50000)
    ref = make()
    ref.run(30000)
    ref.run_to_end(50000)
    ba, br = a.biomarkers(), ref.biomarkers()
    assert (ba["status"] == cep.INST_DONE).all()
    rep = br["vm_valley"] < -80.0
    assert np.abs(ba["apd90"] - br["apd90"])[rep].max() <= APD_TOL_MIXED


@pytest.mark.gpu
def test_checkpoint_resume_is_bit_identical(cep, gpu):
    """A batch checkpointed mid-protocol (inside the evaluated beats, with
    the Ca ring part-filled) and restored into a fresh batch ends with the
    same states and biomarker records, bit for bit, as the run that was
    never interrupted."""
    conc, hill = cipa_population(50, 4, seed=6)
    n = len(conc)
    a = cep.Batch("cipa2017", n, "mixed")
    a.init(conc=conc, hill=hill, quirks=True)
    a.set_pacing(1000.0)
    a.set_protocol(0.005, 3, 1, dt_write=1.0)
    a.run(250000)
    blob = a.checkpoint()
    clk = a.clock(7)
    a.run_to_end(50000)
    ra, sa = a.biomarkers(), a.get_states()
    b = cep.Batch("cipa2017", n, "mixed")
    b.restore(blob)
    assert b.clock(7) == clk
    b.run_to_end(50000)
    rb, sb = b.biomarkers(), b.get_states()
    assert np.array_equal(sa, sb)
    for k in ra:
        assert np.array_equal(ra[k], rb[k], equal_nan=True), k
    with pytest.raises(cep.CepError):
        cep.Batch("cipa2017", n + 32, "mixed").restore(blob)
    with pytest.raises(cep.CepError):
        cep.Batch("cipa2017", n, "fp64").restore(blob)
    # a truncated blob is rejected before the batch changes: a restore of
    # the whole blob afterwards still resumes bit for bit
    c = cep.Batch("cipa2017", n, "mixed")
    with pytest.raises(cep.CepError):
        c.restore(blob[: len(blob) - 8])
    c.restore(blob)
    c.run_to_end(50000)
    rc = c.biomarkers()
    for k in ra:
        assert np.array_equal(ra[k], rc[k], equal_nan=True), k
