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


def _patch_alone(cep, nx, ny, steps, conc, hill, precision):
    """The same TT2006 patch run directly (cells + operator + tissue)."""
    n = nx * ny
    cells = cep.Batch("tt2006", n, precision)
    cells.init(conc=np.full(n, conc), hill=np.broadcast_to(hill, (n, 14)) if hill is not None else None)
    fem = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, 0.0013, fmt=cep.FEM_CLASSED).set_solver(1e-10)
    t = cep.Tissue(cells, fem, 0.01)
    mask = np.zeros((ny, nx), np.uint8)
    mask[:3, :3] = 1
    t.set_stimulus(mask.ravel(), 1000.0, 0.0, 1.0, 1)
    t.run(steps)
    return t.v(), t.activation()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tissue_jobs_alone_and_in_a_mix(cep, gpu, precision):
    """Tissue-patch jobs of different sizes, durations and drugs, running
    beside population jobs, give each patch's own result (V to the solver
    tolerance, activation times equal) and leave the population jobs'
    biomarkers bit-identical."""
    hill = np.zeros(14)
    hill[12], hill[13] = 0.4, 1.2
    patches = [(24, 18, 450, 0.0), (16, 30, 300, 0.5), (20, 20, 600, 1.5)]
    alone = [_patch_alone(cep, nx, ny, steps, c, hill, precision) for nx, ny, steps, c in patches]
    srv = cep.Server("ord2011", precision, capacity=256, dt=0.005, max_bcl=1000.0, steps_per_launch=7000)
    try:
        a_conc, a_hill = _job(5, 10, 3)
        ja = srv.submit(a_conc, a_hill, bcl=1000.0, n_pace=2, first_pace=1)
        srv.wait(ja, 600)
        pop_alone, _ = srv.result(ja)
        ids = [srv.submit_tissue(nx, ny, steps * 0.01, conc=c, hill=hill, stim=(3, 3), rtol=1e-10)
               for nx, ny, steps, c in patches]
        ja2 = srv.submit(a_conc, a_hill, bcl=1000.0, n_pace=2, first_pace=1)
        for j in ids + [ja2]:
            srv.wait(j, 600)
        for (v0, a0), j in zip(alone, ids):
            v, ta, tm = srv.tissue_result(j)
            assert np.abs(v - v0).max() <= 1e-6
            assert np.array_equal(ta, a0)
            assert tm["latency_ms"] >= tm["run_ms"] > 0
        pop_mix, _ = srv.result(ja2)
        for f in FIELDS:
            assert np.array_equal(pop_alone[f], pop_mix[f]), f
        with pytest.raises(cep.CepError):
            srv.result(ids[0])  # a tissue job has no biomarker records
    finally:
        srv.close()


@pytest.mark.gpu
def test_tissue_job_rejections(cep, gpu):
    srv = cep.Server("ord2011", "mixed", capacity=64, dt=0.005, max_bcl=1000.0, steps_per_launch=5000,
                     hbm_fraction=0.5)
    try:
        with pytest.raises(cep.CepError) as e:
            srv.submit_tissue(1, 10, 10.0)
        assert e.value.code == cep.ERR_ARG
        with pytest.raises(cep.CepError) as e:
            srv.submit_tissue(10, 10, -1.0)
        assert e.value.code == cep.ERR_ARG
        with pytest.raises(cep.CepError) as e:
            srv.submit_tissue(1 << 14, 1 << 14, 10.0)  # 2^28 nodes: over any HBM budget
        assert e.value.code in (cep.ERR_OOM, cep.ERR_ARG)
    finally:
        srv.close()


@pytest.mark.gpu
def test_cancel_queued_and_running_jobs(cep, gpu):
    """A queued job cancelled leaves at once; a running population job and
    a running patch job leave between launches, their slots and memory
    return, and the server goes on serving."""
    import time
    srv = cep.Server("ord2011", "mixed", capacity=64, dt=0.005, max_bcl=1000.0, steps_per_launch=2000)
    try:
        conc, hill = _job(5, 16, 3)  # 48 instances
        long_job = srv.submit(conc, hill, bcl=1000.0, n_pace=500, first_pace=499)
        queued = srv.submit(conc, hill, bcl=1000.0, n_pace=1, first_pace=0)  # cannot fit beside it
        assert srv.poll(queued) == cep.JOB_QUEUED
        srv.cancel(queued)
        assert srv.poll(queued) == cep.JOB_CANCELLED
        with pytest.raises(cep.CepError):
            srv.wait(queued, 5)
        patch = srv.submit_tissue(64, 64, 2000.0)
        t0 = time.time()
        while (srv.poll(long_job) != cep.JOB_RUNNING or srv.poll(patch) != cep.JOB_RUNNING) and time.time() - t0 < 60:
            time.sleep(0.01)
        srv.cancel(long_job)
        srv.cancel(patch)
        for j in (long_job, patch):
            with pytest.raises(cep.CepError):
                srv.wait(j, 120)
            assert srv.poll(j) == cep.JOB_CANCELLED
        c2, h2 = _job(6, 16, 4)  # the whole pool
        j = srv.submit(c2, h2, bcl=1000.0, n_pace=1, first_pace=0)
        srv.wait(j, 300)
        res, _ = srv.result(j)
        assert (res["status"] == cep.INST_DONE).all()
        assert srv.stats()["slots_used"] == 0
        with pytest.raises(cep.CepError):
            srv.cancel(j)
        for k in (long_job, queued, patch, j):
            srv.release(k)
    finally:
        srv.close()
