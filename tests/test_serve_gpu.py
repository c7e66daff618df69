"""The screening-job server (continuous batching) on the GPU: a job's
results are identical alone and in a mix, they match a plain batch run,
admission waits for free slots, and bad jobs are rejected."""
from __future__ import annotations

import numpy as np
import pytest


def _job(seed: int, n_samples: int, n_conc: int):
    rng = np.random.default_rng(seed)
    hill = np.zeros((n_samples, 14))
    hill[:, 0::2] = 10 ** rng.uniform(-1, 2, (n_samples, 7))
    hill[:, 1::2] = rng.uniform(0.6, 1.8, (n_samples, 7))
    cmax = 10 ** rng.uniform(-2, 1)
    hill = np.repeat(hill, n_conc, axis=0)
    conc = np.tile(np.arange(n_conc) * cmax, n_samples)
    return conc, hill


FIELDS = ("apd90", "apd50", "cad90", "cad50", "qnet", "dvmdt_max", "dvmdt_repol", "vm_peak", "ca_peak",
          "steepest_pace", "status")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_job_alone_equals_job_in_mix(cep, gpu, precision):
    srv = cep.Server("ord2011", precision, capacity=512, dt=0.005, max_bcl=1000.0, steps_per_launch=7000)
    try:
        a_conc, a_hill = _job(1, 12, 3)
        ja = srv.submit(a_conc, a_hill, bcl=1000.0, n_pace=3, first_pace=1)
        srv.wait(ja, 600)
        alone, _ = srv.result(ja)
        assert (alone["status"] == cep.INST_DONE).all()
        # the same job again, arriving between others of other sizes, paces and BCLs
        b_conc, b_hill = _job(2, 40, 4)
        c_conc, c_hill = _job(3, 7, 2)
        jb = srv.submit(b_conc, b_hill, bcl=800.0, n_pace=4, first_pace=2)
        ja2 = srv.submit(a_conc, a_hill, bcl=1000.0, n_pace=3, first_pace=1)
        jc = srv.submit(c_conc, c_hill, bcl=1000.0, n_pace=2, first_pace=1)
        for j in (jb, ja2, jc):
            srv.wait(j, 600)
        mixed, _ = srv.result(ja2)
        for f in FIELDS:
            assert np.array_equal(alone[f], mixed[f]), f
        st = srv.stats()
        assert st["completed"] == 4 and st["slots_used"] == 0
    finally:
        srv.close()


@pytest.mark.gpu
def test_server_matches_batch_run(cep, gpu):
    """Biomarkers from the server equal a plain batch run of the same
    instances within the FP64 parity tolerance."""
    conc, hill = _job(4, 8, 2)
    srv = cep.Server("ord2011", "fp64", capacity=64, dt=0.005, max_bcl=1000.0, steps_per_launch=9000)
    try:
        j = srv.submit(conc, hill, bcl=1000.0, n_pace=2, first_pace=1)
        srv.wait(j, 600)
        res, times = srv.result(j)
    finally:
        srv.close()
    b = cep.Batch("ord2011", len(conc), "fp64")
    b.init(conc=conc, hill=hill)
    b.set_pacing(1000.0)
    b.set_protocol(0.005, 2, 1, dt_write=1.0)
    b.run_to_end(20000)
    ref = b.biomarkers()
    for f in ("apd90", "apd50", "cad90", "cad50"):
        assert np.abs(res[f] - ref[f]).max() <= 0.01, f
    assert times["latency_ms"] >= times["run_ms"] > 0
    assert times["cell_steps"] == len(conc) * 400000


@pytest.mark.gpu
def test_admission_waits_for_free_slots(cep, gpu):
    srv = cep.Server("ord2011", "mixed", capacity=100, dt=0.005, max_bcl=1000.0, steps_per_launch=10000)
    try:
        c1, h1 = _job(5, 30, 2)  # 60 slots
        c2, h2 = _job(6, 30, 2)  # 60 slots: cannot fit beside the first
        j1 = srv.submit(c1, h1, bcl=1000.0, n_pace=1, first_pace=0)
        j2 = srv.submit(c2, h2, bcl=1000.0, n_pace=1, first_pace=0)
        srv.wait(j1, 600)
        srv.wait(j2, 600)
        _, t1 = srv.result(j1)
        _, t2 = srv.result(j2)
        assert t2["queue_ms"] >= 0.5 * t1["run_ms"]
        with pytest.raises(cep.CepError) as e:
            srv.submit(np.zeros(101))  # larger than the pool
        assert e.value.code == cep.ERR_ARG
        with pytest.raises(cep.CepError) as e:
            srv.submit(np.zeros(4), bcl=2000.0, n_pace=2, first_pace=1)  # longer beat than max_bcl
        assert e.value.code == cep.ERR_ARG
        srv.release(j1)
        with pytest.raises(cep.CepError):
            srv.poll(j1)
    finally:
        srv.close()
