"""Protocol variants of the batched cell kernels: dynamic restitution
(CEPCell_NEO/modules/apdr_bench.cpp) and voltage-clamp replay
(CEPPatch/benchpatch.cpp). CPU tests pin the oracle's restatement by
properties of the protocols; GPU tests compare the device protocols with
the oracle record by record."""
from __future__ import annotations

import numpy as np
import pytest

# Restitution records: pace numbers, BCLs, recalibration flags and the
# segment clock are exact; APD90 and DI are quantised to the time step, and
# FP64 trajectories that agree to 1e-6 mV may cross a repolarisation band
# one step apart, so they agree within one dt.
DT = 0.01
APD_TOL_MIXED = 0.1
CLAMP_REL_FP64 = 1e-9
CLAMP_REL_MIXED = 2e-3


def _hill_rows(rng, n):
    rows = np.zeros((n, 14))
    for k in range(1, n):  # row 0: no drug
        rows[k, 0::2] = 10 ** rng.uniform(-1, 1, 7)
        rows[k, 1::2] = rng.uniform(0.6, 1.8, 7)
    return rows


def _records_equal(dev, ref, apd_tol):
    assert len(dev["pace"]) == len(ref["pace"])
    assert np.array_equal(dev["pace"], ref["pace"].astype(int))
    assert np.array_equal(dev["bcl"], ref["bcl"])
    assert np.array_equal(dev["t"], ref["t"])
    assert np.abs(dev["apd90"] - ref["apd90"]).max() <= apd_tol
    assert np.abs(dev["di"] - ref["di"]).max() <= apd_tol


# ------------------------------------------------------------------ oracle
def test_apdr_bcl_list(oracle):
    assert oracle.apdr_bcls(1000, 250, 100) == [1000.0, 900.0, 800.0, 700.0, 600.0, 500.0, 400.0, 300.0,
                                                290.0, 280.0, 270.0, 260.0, 250.0]
    assert oracle.apdr_bcls(500, 600, 50) == []


def test_oracle_restitution_properties(oracle, cep):
    bcls = [500.0, 300.0, 280.0]
    c = oracle.Cell("tt2004", mcell=True)
    r, st = c.restitution(bcls, 4, DT)
    assert st == 0
    assert len(r["pace"]) == cep.restitution_records(bcls, 4, DT) == 6
    # the first two paces of every BCL are not written (apdr_bench.cpp:209)
    assert list(r["pace"].astype(int)) == [3, 4, 7, 8, 11, 12]
    # apd90 + di spans one BCL: (t + start) - lo with lo = bcl*pace + start
    assert np.allclose(r["apd90"] + r["di"], r["bcl"], atol=1e-6)
    # 2:1 block at the short BCLs sends some paces through the search over the whole trace
    assert r["recal"].any() and not r["recal"].all()
    # the M cell (2004_a, g_Ks 0.062) repolarises later than the epicardial build
    e = oracle.Cell("tt2004")
    re_, _ = e.restitution([500.0], 4, DT)
    assert (r["apd90"][:2] > re_["apd90"]).all()


@pytest.mark.parametrize("model", ["ord2011", "cipa2017", "tt2006", "tt2004", "tomek2019"])
def test_oracle_clamp_replays_a_free_run(oracle, model):
    """Clamping V to the trace a free run produced reproduces that run
    (through the stimulus, so the upstroke is included)."""
    free = oracle.Cell(model)
    n, dt = 3000, 0.005
    v, cur = np.zeros(n), np.zeros((n, 2))
    t = 0.0
    for k in range(n):
        v[k] = free.y[0]
        c_ = free.step(t, dt)
        cur[k] = c_.ICaL, c_.IKr
        t += dt
    for j, idx in enumerate((3, 4)):
        c = oracle.Cell(model)
        out = c.clamp(v, 0.0, dt, idx)
        assert np.array_equal(out, cur[:, j])
        assert np.array_equal(c.states[1:], free.states[1:])
    assert v.max() > 0  # the stimulus fired inside the window


@pytest.mark.parametrize("bcls,n_pace,dt", [([500.0], 4, 0.03), ([410.0, 333.0], 3, 0.007), ([400.0], 2, 0.02),
                                            ([400.0], 1, 0.02)])
def test_oracle_restitution_record_count(oracle, cep, bcls, n_pace, dt):
    """The record count of the host formula (pace boundaries among
    iout = 1 .. (int)(n_pace*bcl/dt) + 1, minus two per BCL) against the
    oracle's loop, with bcl/dt not an integer and with n_pace <= 2."""
    r, st = oracle.Cell("tt2004").restitution(bcls, n_pace, dt)
    assert st == 0
    assert len(r["pace"]) == cep.restitution_records(bcls, n_pace, dt)


# --------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_restitution_fp64_matches_oracle(cep, gpu, oracle):
    rng = np.random.default_rng(21)
    n = 3
    hill = _hill_rows(rng, n)
    conc = np.array([0.0, 1.0, 3.0])
    bcls = [500.0, 300.0, 280.0]
    b = cep.Batch("tt2004", n, "fp64")
    b.init(conc=conc, hill=hill, mcell=True)
    dev = b.restitution(bcls, 4, DT, steps_per_launch=7000)
    n_recal = 0
    for i in range(n):
        c = oracle.Cell("tt2004", conc=conc[i], hill=hill[i], mcell=True)
        ref, st = c.restitution(bcls, 4, DT)
        assert st == 0
        _records_equal({f: dev[f][i] for f in dev}, ref, DT * 1.0001)
        assert np.array_equal(dev["recal"][i], ref["recal"].astype(int))
        n_recal += int(ref["recal"].sum())
        fin = b.get_states()[i]
        assert abs(fin[0] - c.y[0]) <= 1e-6
    assert n_recal > 0  # the recalibration search ran on the device


@pytest.mark.gpu
def test_restitution_mixed_and_other_models(cep, gpu, oracle):
    bcls = [600.0, 400.0]
    b = cep.Batch("tt2004", 2, "mixed")
    b.init(mcell=True)
    dev = b.restitution(bcls, 4, DT)
    ref, _ = oracle.Cell("tt2004", mcell=True).restitution(bcls, 4, DT)
    for i in range(2):
        _records_equal({f: dev[f][i] for f in dev}, ref, APD_TOL_MIXED)
    b = cep.Batch("tt2006", 1, "fp64")
    b.init()
    dev = b.restitution([800.0], 4, 0.02)
    ref, _ = oracle.Cell("tt2006").restitution([800.0], 4, 0.02)
    _records_equal({f: dev[f][0] for f in dev}, ref, 0.02 * 1.0001)


def _clamp_trace(n, dt):
    """Steps of a patch-clamp protocol: holding -85 mV, a test pulse to
    +10 mV, a ramp back, and a second pulse to -20 mV."""
    t = np.arange(n) * dt
    v = np.full(n, -85.0)
    v[(t >= 5) & (t < 150)] = 10.0
    ramp = (t >= 150) & (t < 250)
    v[ramp] = 10.0 - (t[ramp] - 150.0) * 0.95
    v[(t >= 300) & (t < 400)] = -20.0
    return v


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["ord2011", "cipa2017", "tomek2019"])
def test_clamp_matches_oracle(cep, gpu, oracle, model):
    dt = 0.005
    v = _clamp_trace(100000, dt)
    rng = np.random.default_rng(5)
    hill = _hill_rows(rng, 2)
    if model == "cipa2017":  # static hERG block off, dynamic hERG Kmax, Ku, n, halfmax, Vhalf, Kt
        hill[:, 12:14] = 0.0
        hill = np.hstack([hill, np.tile([2e4, 1e-3, 0.9, 1e4, -50.0, 3.5e-5], (2, 1))])
    for prec, tol in (("fp64", CLAMP_REL_FP64), ("mixed", CLAMP_REL_MIXED)):
        for cur in ("ICaL", "IKr"):
            b = cep.Batch(model, 2, prec)
            b.init(conc=np.array([0.0, 2.0]), hill=hill)
            dev = b.clamp(v, 0.0, dt, cur)
            for i in range(2):
                c = oracle.Cell(model, conc=[0.0, 2.0][i], hill=hill[i])
                ref = c.clamp(v, 0.0, dt, cep.CURRENTS.index(cur))
                scale = np.abs(ref).max()
                assert scale > 0
                assert np.abs(dev[:, i] - ref).max() <= tol * scale, (prec, cur, i)
