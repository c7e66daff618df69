"""The FEM oracle (test infrastructure) on CPU: element matrices, assembly
and Jacobi-PCG against closed-form properties and a direct solve.

The reference's FEM (fem.cpp) needs PETSc 3.1 and MPI, neither of which is
in the tree, so it cannot be compiled here; the oracle restates its element
routine and is checked through properties the operators must have.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla


@pytest.mark.parametrize("dim", [2, 3])
def test_element_matrices(oracle, dim):
    h, dt, D = 0.025, 0.01, 0.0013
    ae, be = oracle.fem_element(dim, h, dt, [D])
    vol = h ** dim
    # consistent mass integrates the constant exactly; stiffness kills constants
    assert abs(be.sum() - vol) < 1e-15 * max(1.0, vol) + 1e-18
    k = ae - be / dt
    assert np.abs(k.sum(axis=1)).max() < 1e-16
    assert np.abs(ae - ae.T).max() <= 1e-12 * np.abs(ae).max()
    # 2-point Gauss with the truncated 1/sqrt(3) (fem.cpp:231-271): the Q1
    # stiffness diagonal is D*(2/3) (2D) or D*h/3 (3D) up to that truncation
    expect = D * (2.0 / 3.0) if dim == 2 else D * h / 3.0
    assert abs(k[0, 0] - expect) / expect < 1e-4


def test_tensor_reduces_to_scalar(oracle):
    """An isotropic tensor gives the scalar element within a few ulp (the
    scalar form follows the reference's operation order, the tensor form is
    the anisotropic extension's grad . D grad)."""
    for dim, d6 in ((2, [0.001, 0, 0.001]), (3, [0.001, 0, 0, 0.001, 0, 0.001])):
        ae1, be1 = oracle.fem_element(dim, 0.02, 0.01, [0.001])
        ae6, be6 = oracle.fem_element(dim, 0.02, 0.01, d6)
        assert np.abs(ae1 - ae6).max() <= 4 * np.finfo(float).eps * np.abs(ae1).max()
        assert np.array_equal(be1, be6)


@pytest.mark.parametrize("dim,shape", [(2, (7, 5, 1)), (3, (4, 5, 3))])
def test_assembly_and_pcg(oracle, dim, shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(4)
    n_elem = (nx - 1) * (ny - 1) * ((nz - 1) if dim == 3 else 1)
    nd = 3 if dim == 2 else 6
    D = np.zeros((n_elem, nd))
    if dim == 2:
        D[:, 0] = rng.uniform(5e-4, 2e-3, n_elem)
        D[:, 2] = rng.uniform(5e-4, 2e-3, n_elem)
        D[:, 1] = 0.3 * np.sqrt(D[:, 0] * D[:, 2]) * rng.uniform(-1, 1, n_elem)
    else:
        for c in (0, 3, 5):
            D[:, c] = rng.uniform(5e-4, 2e-3, n_elem)
    rp, ci, a, b = oracle.fem_assemble(dim, nx, ny, nz, 0.025, 0.01, D)
    n = nx * ny * nz
    assert rp[-1] == len(ci) == (3 * nx - 2) * (3 * ny - 2) * ((3 * nz - 2) if dim == 3 else 1)
    for i in range(n):
        assert np.all(np.diff(ci[rp[i]:rp[i + 1]]) > 0)
    A = sp.csr_matrix((a, ci, rp), shape=(n, n))
    B = sp.csr_matrix((b, ci, rp), shape=(n, n))
    assert abs(A - A.T).max() < 1e-18
    assert abs(B.sum() - 0.025 ** dim * n_elem) < 1e-15
    v = rng.uniform(-90, 30, n)
    rhs = B @ v / 0.01
    x, it, res = oracle.pcg(rp, ci, a, rhs, 1e-12)
    assert it > 0 and res <= 1e-12
    ref = sla.spsolve(A.tocsc(), rhs)
    assert np.abs(x - ref).max() < 1e-8
    # unconverged: reports -max_iter
    _, it2, _ = oracle.pcg(rp, ci, a, rhs, 1e-14, max_iter=2)
    assert it2 == -2
    # zero right-hand side: x = 0 with no iterations
    x0, it0, _ = oracle.pcg(rp, ci, a, np.zeros(n), 1e-8)
    assert it0 == 0 and not x0.any()


def test_tissue_wave_propagates(oracle):
    """Corner S1 on a small TT2006 sheet activates the far corner later than
    the near one, and the wave is symmetric about the diagonal."""
    nx = ny = 16
    mask = np.zeros((ny, nx), np.uint8)
    mask[:3, :3] = 1
    v, its, tact = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, 0.01, 1200, mask.ravel(), 1000.0, 0.0,
                                     1.0, 1, rtol=1e-8)
    T = tact.reshape(ny, nx)
    assert (T > 0).all()
    assert T[0, 0] < T[0, -1] < T[-1, -1]
    assert np.abs(T - T.T).max() < 1e-9
    assert (its > 0).all()


def test_pseudo_ecg_oracle_properties(oracle):
    """The pseudo-ECG restatement: zero for a uniform V; for a linear ramp
    it is the element-centroid quadrature of w * int (D grad V) . r / |r|^3
    (w = 1/6); linear in V."""
    nx, ny, h, D = 20, 16, 0.025, 0.0013
    el = np.array([[0.2, 0.2, 1.0], [5.0, 0.2, 0.0]])
    assert np.abs(oracle.pseudo_ecg(2, nx, ny, 1, h, D, np.full(nx * ny, -80.0), el)).max() <= 1e-15
    x = (np.arange(nx * ny) % nx) * h
    got = oracle.pseudo_ecg(2, nx, ny, 1, h, D, 100.0 * x, el)
    ref = np.zeros(2)
    for ey in range(ny - 1):
        for ex in range(nx - 1):
            c = np.array([(ex + 0.5) * h, (ey + 0.5) * h, 0.0])
            for k in range(2):
                r = c - el[k]
                ref[k] += D * 100.0 * r[0] / np.linalg.norm(r) ** 3 * h * h / 6.0
    assert np.allclose(got, ref, rtol=1e-12, atol=0)
    rng = np.random.default_rng(3)
    v1, v2 = rng.normal(size=nx * ny), rng.normal(size=nx * ny)
    lhs = oracle.pseudo_ecg(2, nx, ny, 1, h, D, 2.0 * v1 - v2, el)
    rhs = 2.0 * oracle.pseudo_ecg(2, nx, ny, 1, h, D, v1, el) - oracle.pseudo_ecg(2, nx, ny, 1, h, D, v2, el)
    assert np.allclose(lhs, rhs, rtol=1e-12, atol=1e-18)
