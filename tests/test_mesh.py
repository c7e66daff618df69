"""Mesh files and unstructured P1 tetrahedra: the .inp reader/writer of the
reference's format, the VTK writer, the oracle's tetrahedral element
matrices against closed forms (CPU), and on the GPU the device assembly
(bit for bit) and a tissue on a tetrahedral mesh against the oracle."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

mesh = importlib.import_module("2ddrugsimulation_b200.mesh")


def _volumes(m):
    p = m.xyz[m.elements]
    return np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6.0


def test_inp_round_trip(tmp_path):
    m = mesh.box_tets(4, 3, 3, 0.025)
    m.targets = (0, 5, 35)
    for ct in (None, np.arange(len(m.xyz)) % 3):
        m.celltype = ct
        mesh.write_inp(tmp_path / "m.inp", m)
        r = mesh.read_inp(tmp_path / "m.inp")
        assert r.etype == "C3D4" and r.targets == m.targets
        assert np.array_equal(r.xyz, m.xyz) and np.array_equal(r.elements, m.elements)
        assert (r.celltype is None) == (ct is None)
        if ct is not None:
            assert np.array_equal(r.celltype, ct)


def test_box_tets_tile_the_box():
    m = mesh.box_tets(5, 4, 3, 0.1)
    v = _volumes(m)
    assert (v > 0).all() and np.isclose(v.sum(), 0.4 * 0.3 * 0.2)


def test_vtk_writer(tmp_path):
    m = mesh.box_tets(3, 3, 2, 0.1)
    mesh.write_vtk(tmp_path / "v.vtk", m, {"Voltage": np.linspace(-85, 20, len(m.xyz))})
    txt = (tmp_path / "v.vtk").read_text().splitlines()
    assert txt[0].startswith("# vtk DataFile") and f"POINTS {len(m.xyz)} float" in txt
    assert f"CELLS {len(m.elements)} {5 * len(m.elements)}" in txt and "SCALARS Voltage float" in txt


def test_oracle_tet_element_closed_forms(oracle):
    """Unit Gauss weights as the reference: B_e = 24 V (1 + delta_jk) / 20
    (the consistent mass times 24), K_e = 24 V grad phi_j . D grad phi_k;
    A = B/dt + K; symmetric; stiffness rows sum to 0."""
    rng = np.random.default_rng(2)
    x = np.array([[0, 0, 0], [0.03, 0.002, 0.001], [0.004, 0.025, 0.003], [0.002, 0.001, 0.028]]) + rng.normal(0, 1e-3, (4, 3))
    D = np.array([2e-3, 3e-4, -1e-4, 1.2e-3, 2e-4, 8e-4])
    dt = 0.01
    rp, ci, a, b = oracle.fem_assemble_tet(x, [[0, 1, 2, 3]], D[None, :], dt)
    A = np.zeros((4, 4))
    B = np.zeros((4, 4))
    for i in range(4):
        for q in range(rp[i], rp[i + 1]):
            A[i, ci[q]], B[i, ci[q]] = a[q], b[q]
    V = np.dot(np.cross(x[1] - x[0], x[2] - x[0]), x[3] - x[0]) / 6.0
    Bref = 24 * V * (np.ones((4, 4)) + np.eye(4)) / 20
    T = np.vstack([np.ones(4), x.T])
    G = np.linalg.inv(T)[:, 1:]  # rows: grad phi_j
    Dm = np.array([[D[0], D[1], D[2]], [D[1], D[3], D[4]], [D[2], D[4], D[5]]])
    Kref = 24 * V * G @ Dm @ G.T
    assert np.allclose(B, Bref, rtol=1e-12, atol=0)
    assert np.allclose(A - B / dt, Kref, rtol=1e-10, atol=1e-16)
    assert np.allclose(A, A.T, rtol=1e-12, atol=1e-18)


@pytest.mark.gpu
def test_tet_assembly_bitwise(cep, gpu, oracle):
    m = mesh.box_tets(6, 5, 4, 0.025)
    rng = np.random.default_rng(4)
    m.xyz = m.xyz + rng.uniform(-0.003, 0.003, m.xyz.shape)  # irregular, still positively oriented
    D = np.zeros((len(m.elements), 6))
    D[:, 0], D[:, 3], D[:, 5] = rng.uniform(5e-4, 2e-3, (3, len(m.elements)))
    D[:, 1] = 1e-4 * rng.uniform(-1, 1, len(m.elements))
    for d in (0.0013, D):
        f = cep.Fem.tet(m.xyz, m.elements, d, 0.01, fmt=cep.FEM_CSR)
        rp, ci, a, b = f.get_csr()
        orp, oci, oa, ob = oracle.fem_assemble_tet(m.xyz, m.elements, d, 0.01)
        assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
        assert np.array_equal(a, oa) and np.array_equal(b, ob)


@pytest.mark.gpu
def test_tissue_on_tet_mesh_matches_oracle(cep, gpu, oracle):
    m = mesh.box_tets(10, 8, 4, 0.025)
    n = len(m.xyz)
    mask = (m.xyz[:, 0] < 0.03).astype(np.uint8)
    cells = cep.Batch("tt2006", n, "fp64")
    cells.init()
    fem = cep.Fem.tet(m.xyz, m.elements, 0.0013, 0.01, fmt=cep.FEM_AUTO).set_solver(1e-10)
    t = cep.Tissue(cells, fem, 0.01)
    t.set_stimulus(mask, 1000.0, 0.0, 1.0, 1)
    t.run(800)
    rp, ci, a, b = oracle.fem_assemble_tet(m.xyz, m.elements, 0.0013, 0.01)
    vo, _, tao = oracle.tissue_run_csr("tt2006", rp, ci, a, b, 0.01, 800, mask, 1000.0, 0.0, 1.0, 1, rtol=1e-10)
    assert (tao > 0).any()
    assert np.abs(t.v() - vo).max() <= 1e-6
    assert np.array_equal(t.activation(), tao)
    with pytest.raises(cep.CepError):
        t.set_electrodes([[0.0, 0.0, 1.0]])  # no pseudo-ECG on unstructured operators


def test_output_and_states_files_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    st = rng.uniform(-90, 40, (7, 19))
    mesh.write_output(tmp_path / "output.0", 1234.5, st)
    first = (tmp_path / "output.0").read_text().splitlines()[0]
    assert first == "1234.500000 "
    t, back = mesh.read_output(tmp_path / "output.0", 19)
    assert t == 1234.5 and back.shape == (7, 19)
    assert np.abs(back - st).max() <= 5e-7  # six decimals, as the reference writes
    with pytest.raises(ValueError):
        mesh.read_output(tmp_path / "output.0", 18)
    y = rng.uniform(-1, 1, 41)
    mesh.write_states(tmp_path / "output_orudy.dat", y)
    assert np.abs(mesh.read_states(tmp_path / "output_orudy.dat") - y).max() <= 5e-7


@pytest.mark.gpu
def test_tissue_resumes_from_an_output_snapshot(cep, gpu, tmp_path):
    """iopt = 1: a TT2006 sheet resumed at 6 ms in a new tissue. From the
    exact states and clock the run continues bit for bit; from the
    output.<rank> file (six decimals) it stays close."""
    nx = ny = 24
    n = nx * ny
    mask = np.zeros((ny, nx), np.uint8)
    mask[:3, :3] = 1

    def make():
        cells = cep.Batch("tt2006", n, "fp64")
        cells.init()
        fem = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, 0.0013).set_solver(1e-10)
        t = cep.Tissue(cells, fem, 0.01)
        t.set_stimulus(mask.ravel(), 1000.0, 0.0, 1.0, 1)
        return cells, fem, t

    c1, f1, t1 = make()
    t1.run(600)
    clock, states = t1.stats()["time"], c1.get_states()
    mesh.write_output(tmp_path / "output.0", clock, states)
    t1.run(600)
    v_ref = t1.v()
    c2, f2, t2 = make()
    c2.set_states(states)
    t2.set_clock(clock)
    t2.run(600)
    assert np.array_equal(t2.v(), v_ref)
    c3, f3, t3 = make()
    time, st = mesh.read_output(tmp_path / "output.0", 19)
    c3.set_states(st)
    t3.set_clock(time)
    t3.run(600)
    d = np.abs(t3.v() - v_ref)
    assert np.median(d) <= 0.1, (np.median(d), d.max())


def test_grid_mesh_matches_the_grid_operator_numbering(tmp_path):
    m2 = mesh.grid_mesh(2, 5, 4, 1, 0.1)
    assert m2.etype == "S4" and m2.elements.shape == (12, 4) and len(m2.xyz) == 20
    p = m2.xyz[m2.elements]
    area = 0.5 * np.cross(p[:, 2] - p[:, 0], p[:, 1] - p[:, 3])[:, 2]  # quad diagonals
    assert np.allclose(np.abs(area), 0.01)
    assert np.array_equal(m2.xyz[7], [0.2, 0.1, 0.0])  # node i + nx*j
    m3 = mesh.grid_mesh(3, 4, 3, 3, 0.1)
    assert m3.etype == "C3D8I" and m3.elements.shape == (12, 8) and len(m3.xyz) == 36
    e = m3.xyz[m3.elements[0]]
    assert np.allclose(e[6] - e[0], [0.1, 0.1, 0.1]) and np.allclose(e[4] - e[0], [0, 0, 0.1])
    mesh.write_vtk(tmp_path / "g.vtk", m3, {"Voltage": np.arange(36.0)})
    text = (tmp_path / "g.vtk").read_text()
    assert "CELL_TYPES 12\n12\n" in text and "POINT_DATA 36" in text
