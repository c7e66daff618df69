"""The allocation-free PCG entry point (cep_fem_solve_csr_noalloc) against
the handle-based solve of the same CSR operator. Collected last so it also
runs after every other GPU test in the same process; it passes alone too."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest


def _field(n_elem, seed):
    rng = np.random.default_rng(seed)
    D = np.zeros((n_elem, 3))
    D[:, 0] = rng.uniform(5e-4, 2e-3, n_elem)
    D[:, 2] = rng.uniform(5e-4, 2e-3, n_elem)
    D[:, 1] = 0.3 * np.sqrt(D[:, 0] * D[:, 2]) * rng.uniform(-1, 1, n_elem)
    return D


@pytest.mark.gpu
def test_noalloc_solve_matches_handle_solve(cep, gpu, oracle):
    import torch
    nx, ny, dt, rtol, max_iter = 180, 130, 0.01, 1e-9, 500
    rp, ci, a, b = oracle.fem_assemble(2, nx, ny, 1, 0.025, dt, _field((nx - 1) * (ny - 1), 5))
    n = len(rp) - 1
    ref = cep.Fem.csr(rp, ci, a, b, dt, fmt=cep.FEM_CSR).set_solver(rtol, max_iter)
    d_rp, d_ci = torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda()
    d_a, d_b = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    lib = cep.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    for call in range(2):  # two calls in a row
        v = rng.uniform(-90, 30, n)
        xr, itr, _ = ref.solve(v)
        dv = torch.from_numpy(v.copy()).cuda()
        it = ctypes.c_int(-7)
        rc = lib.cep_fem_solve_csr_noalloc(n, d_rp.data_ptr(), d_ci.data_ptr(), d_a.data_ptr(), d_b.data_ptr(), dt,
                                           rtol, max_iter, dv.data_ptr(), stream, ctypes.byref(it))
        assert rc == cep.OK, lib.cep_last_error().decode()
        assert it.value == itr, (call, it.value, itr)
        assert np.array_equal(dv.cpu().numpy(), xr), call
    # asynchronous form: no status read, same result once the stream is done
    v = rng.uniform(-90, 30, n)
    xr, _, _ = ref.solve(v)
    dv = torch.from_numpy(v.copy()).cuda()
    rc = lib.cep_fem_solve_csr_noalloc(n, d_rp.data_ptr(), d_ci.data_ptr(), d_a.data_ptr(), d_b.data_ptr(), dt, rtol,
                                       max_iter, dv.data_ptr(), stream, None)
    assert rc == cep.OK
    torch.cuda.synchronize()
    assert np.array_equal(dv.cpu().numpy(), xr)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_and_reports_not_converged(cep, gpu, oracle):
    import torch
    lib = cep.lib()
    rp, ci, a, b = oracle.fem_assemble(2, 40, 30, 1, 0.025, 0.01, 0.0013)
    n = len(rp) - 1
    d = [torch.from_numpy(x).cuda() for x in (rp, ci, a, b)]
    v = torch.from_numpy(np.random.default_rng(0).uniform(-90, 30, n)).cuda()
    ptrs = [x.data_ptr() for x in d]
    big = cep.lib().cep_fem_solve_csr_noalloc(262144 + 1, *ptrs, 0.01, 1e-8, 100, v.data_ptr(), None, None)
    assert big == cep.ERR_ARG
    it = ctypes.c_int()
    rc = lib.cep_fem_solve_csr_noalloc(n, *ptrs, 0.01, 1e-15, 2, v.data_ptr(), None, ctypes.byref(it))
    assert rc == cep.ERR_NOT_CONVERGED and it.value == -2


@pytest.mark.gpu
def test_noalloc_on_a_second_stream_and_missing_diagonal(cep, gpu, oracle):
    """After a call on the default stream, a call on another stream gets the
    handle solve's result bit for bit (the per-device set-up is shared by
    every stream); a row without a diagonal entry is reported by the
    blocking form as an argument error."""
    import torch
    lib = cep.lib()
    dt, rtol, max_iter = 0.01, 1e-9, 500
    rp, ci, a, b = oracle.fem_assemble(2, 64, 48, 1, 0.025, dt, 0.0013)
    n = len(rp) - 1
    ref = cep.Fem.csr(rp, ci, a, b, dt, fmt=cep.FEM_CSR).set_solver(rtol, max_iter)
    d = [torch.from_numpy(x).cuda() for x in (rp, ci, a, b)]
    ptrs = [x.data_ptr() for x in d]
    rng = np.random.default_rng(3)
    it = ctypes.c_int()
    v0 = torch.from_numpy(rng.uniform(-90, 30, n)).cuda()
    assert lib.cep_fem_solve_csr_noalloc(n, *ptrs, dt, rtol, max_iter, v0.data_ptr(), None, ctypes.byref(it)) == 0
    side = torch.cuda.Stream()
    v = rng.uniform(-90, 30, n)
    xr, itr, _ = ref.solve(v)
    with torch.cuda.stream(side):
        dv = torch.from_numpy(v.copy()).to("cuda", non_blocking=False)
        side.synchronize()
        rc = lib.cep_fem_solve_csr_noalloc(n, *ptrs, dt, rtol, max_iter, dv.data_ptr(), side.cuda_stream,
                                           ctypes.byref(it))
        assert rc == cep.OK, lib.cep_last_error().decode()
    assert it.value == itr
    assert np.array_equal(dv.cpu().numpy(), xr)
    # drop the diagonal of row 5: its entry takes the left neighbour's column
    ci2 = ci.copy()
    k = rp[5] + int(np.flatnonzero(ci[rp[5]:rp[6]] == 5)[0])
    ci2[k] = ci[k - 1]
    d_ci2 = torch.from_numpy(ci2).cuda()
    dv = torch.from_numpy(v.copy()).cuda()
    rc = lib.cep_fem_solve_csr_noalloc(n, ptrs[0], d_ci2.data_ptr(), ptrs[2], ptrs[3], dt, rtol, max_iter,
                                       dv.data_ptr(), None, ctypes.byref(it))
    assert rc == cep.ERR_ARG
    assert "row 5" in lib.cep_last_error().decode()


@pytest.mark.gpu
def test_noalloc_reports_a_barrier_timeout(cep, gpu, oracle):
    """The blocking form reports a grid-barrier wait that ran out (forced by
    the wait test hook) as CEP_ERR_TIMEOUT, and the next call, with the hook
    reset, solves normally."""
    import torch
    lib = cep.lib()
    dt, rtol, max_iter = 0.01, 1e-9, 500
    rp, ci, a, b = oracle.fem_assemble(2, 400, 400, 1, 0.025, dt, 0.0013)
    n = len(rp) - 1
    ref = cep.Fem.csr(rp, ci, a, b, dt, fmt=cep.FEM_CSR).set_solver(rtol, max_iter)
    d = [torch.from_numpy(x).cuda() for x in (rp, ci, a, b)]
    ptrs = [x.data_ptr() for x in d]
    v = np.random.default_rng(9).uniform(-90, 30, n)
    it = ctypes.c_int()
    try:
        assert lib.cep_fem_set_wait_test(64, 5_000_000) == cep.OK
        dv = torch.from_numpy(v.copy()).cuda()
        rc = lib.cep_fem_solve_csr_noalloc(n, *ptrs, dt, rtol, max_iter, dv.data_ptr(), None, ctypes.byref(it))
        assert rc == cep.ERR_TIMEOUT
    finally:
        assert lib.cep_fem_set_wait_test(0, 0) == cep.OK
    xr, itr, _ = ref.solve(v)
    dv = torch.from_numpy(v.copy()).cuda()
    rc = lib.cep_fem_solve_csr_noalloc(n, *ptrs, dt, rtol, max_iter, dv.data_ptr(), None, ctypes.byref(it))
    assert rc == cep.OK and it.value == itr
    assert np.array_equal(dv.cpu().numpy(), xr)
