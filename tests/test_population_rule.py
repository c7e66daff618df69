"""The compliant mixed path's late-refinement rule (cep_population_late_mask,
the step-3 selection of cep_population_run in csrc/population.cpp): which
mixed records are re-run in FP64 after the run. Host code only, no device.

A record is re-run when its diastolic Vm is not below the threshold (a NaN
Vm included), its APD90 is above 0.9 BCL (the edge of 2:1 block), or its
rhythm is intermittent (some evaluated beats with an action potential at
the peak sample and some without). A cell with no action potential at the
peak sample in any evaluated beat (a strong sodium block) has no APD in
either precision and is not re-run."""
from __future__ import annotations

import numpy as np
import pytest


def _records(**cols):
    n = len(next(iter(cols.values())))
    base = {"vm_valley": np.full(n, -88.0), "apd90": np.full(n, 300.0), "n_eligible": np.full(n, 250, np.int32)}
    base.update({k: np.asarray(v) for k, v in cols.items()})
    return base


def test_late_mask_rule_cases(cep):
    nan = float("nan")
    recs = _records(
        vm_valley=[-88.0, -70.0, nan, -88.0, -88.0, -88.0, -88.0, -88.0, -80.0, -80.0000001],
        apd90=[300.0, 300.0, 300.0, 1850.0, 1800.0, 300.0, 300.0, 300.0, 300.0, 300.0],
        n_eligible=[250, 250, 250, 250, 250, 0, 249, 1, 250, 250],
    )
    got = cep.population_late_mask(recs, -80.0, 2000.0, 250)
    want = [False,  # repolarising, regular
            True,   # depolarised
            True,   # NaN Vm
            True,   # APD90 above 0.9 BCL
            False,  # APD90 at 0.9 BCL exactly
            False,  # no beat with an action potential at the peak sample
            True,   # intermittent: one beat without
            True,   # intermittent: one beat with
            True,   # diastolic Vm at the threshold (not below it)
            False]  # just below the threshold
    assert list(got) == want


def test_late_mask_short_protocols_and_bcl_scaling(cep):
    recs = _records(apd90=[440.0, 460.0], n_eligible=[0, 0])
    # no evaluated pace: n_eligible 0 is never intermittent
    assert list(cep.population_late_mask(recs, -80.0, 500.0, 0)) == [False, True]
    # the near-block bound scales with the BCL
    assert list(cep.population_late_mask(recs, -80.0, 1000.0, 0)) == [False, False]


def test_late_mask_matches_a_vectorised_restatement(cep):
    rng = np.random.default_rng(3)
    n = 5000
    bcl, thr, ev = 1000.0, -80.0, 250
    recs = _records(vm_valley=rng.uniform(-95.0, -60.0, n), apd90=rng.uniform(200.0, 1000.0, n),
                    n_eligible=rng.integers(0, ev + 1, n).astype(np.int32))
    recs["vm_valley"][::97] = np.nan
    got = cep.population_late_mask(recs, thr, bcl, ev)
    v, a, e = recs["vm_valley"], recs["apd90"], recs["n_eligible"]
    want = ~(v < thr) | (a > 0.9 * bcl) | ((e > 0) & (e < ev))
    assert np.array_equal(got, want)


def test_late_mask_argument_checks(cep):
    recs = _records(vm_valley=[-88.0])
    for bcl, ev in ((0.0, 10), (float("nan"), 10), (1000.0, -1)):
        with pytest.raises(cep.CepError) as e:
            cep.population_late_mask(recs, -80.0, bcl, ev)
        assert e.value.code == cep.ERR_ARG
    assert cep.population_late_mask(_records(vm_valley=np.zeros(0)), -80.0, 1000.0, 10).shape == (0,)
