"""Monodomain FEM on the GPU against the oracle: device assembly (bit for
bit), SpMV, the persistent Jacobi-PCG solve, and a Godunov-split tissue run.

Tolerances: assembly is exact (the device builds each entry with the same
IEEE expression, summed over elements in the same order). SpMV rows use
FMA, so they agree to 1e-13 relative. The PCG's dot products are tree sums,
so iterates differ by rounding: iteration counts may differ by one at the
stopping boundary and converged solutions agree to the solver tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest


def _tensor_field(dim, n_elem, seed):
    rng = np.random.default_rng(seed)
    if dim == 2:
        D = np.zeros((n_elem, 3))
        D[:, 0] = rng.uniform(5e-4, 2e-3, n_elem)
        D[:, 2] = rng.uniform(5e-4, 2e-3, n_elem)
        D[:, 1] = 0.3 * np.sqrt(D[:, 0] * D[:, 2]) * rng.uniform(-1, 1, n_elem)
    else:
        D = np.zeros((n_elem, 6))
        for c in (0, 3, 5):
            D[:, c] = rng.uniform(5e-4, 2e-3, n_elem)
        D[:, 1] = 0.2 * np.sqrt(D[:, 0] * D[:, 3]) * rng.uniform(-1, 1, n_elem)
    return D


CASES = [(2, (13, 9, 1), "scalar"), (2, (11, 17, 1), "tensor"), (3, (6, 5, 4), "scalar"), (3, (7, 6, 5), "tensor")]


def _field(dim, shape, kind, seed=0):
    nx, ny, nz = shape
    n_elem = (nx - 1) * (ny - 1) * ((nz - 1) if dim == 3 else 1)
    if kind == "scalar":
        return np.random.default_rng(seed).uniform(5e-4, 2e-3, n_elem)
    return _tensor_field(dim, n_elem, seed)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,shape,kind", CASES)
def test_grid_assembly_bitwise(cep, gpu, oracle, dim, shape, kind):
    D = _field(dim, shape, kind)
    nx, ny, nz = shape
    f = cep.Fem.grid(dim, nx, ny, nz, 0.025, 0.01, D)
    rp, ci, a, b = f.get_csr()
    orp, oci, oa, ob = oracle.fem_assemble(dim, nx, ny, nz, 0.025, 0.01, D)
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    assert np.array_equal(a, oa), np.abs(a - oa).max()
    assert np.array_equal(b, ob), np.abs(b - ob).max()
    assert f.ell_width == (9 if dim == 2 else 27)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["csr", "ell", "stencil"])
@pytest.mark.parametrize("dim,shape,kind", CASES)
def test_spmv(cep, gpu, oracle, dim, shape, kind, fmt):
    D = _field(dim, shape, kind, seed=1)
    nx, ny, nz = shape
    f = cep.Fem.grid(dim, nx, ny, nz, 0.025, 0.01, D,
                     fmt={"csr": cep.FEM_CSR, "ell": cep.FEM_ELL, "stencil": cep.FEM_STENCIL}[fmt])
    rp, ci, a, b = oracle.fem_assemble(dim, nx, ny, nz, 0.025, 0.01, D)
    x = np.random.default_rng(2).uniform(-90, 30, f.n)
    for which, val in (("A", a), ("B", b)):
        y = f.spmv(x, which)
        ref = oracle.spmv(rp, ci, val, x)
        scale = oracle.spmv(rp, ci, np.abs(val), np.abs(x))
        assert np.all(np.abs(y - ref) <= 1e-13 * scale), (which, np.abs(y - ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precond_norm", [True, False])
@pytest.mark.parametrize("dim,shape,kind", CASES)
def test_pcg_matches_oracle(cep, gpu, oracle, dim, shape, kind, precond_norm):
    D = _field(dim, shape, kind, seed=3)
    nx, ny, nz = shape
    dt = 0.01
    f = cep.Fem.grid(dim, nx, ny, nz, 0.025, dt, D)
    rp, ci, a, b = oracle.fem_assemble(dim, nx, ny, nz, 0.025, dt, D)
    v = np.random.default_rng(5).uniform(-90, 30, f.n)
    rhs = oracle.spmv(rp, ci, b, v) / dt
    for rtol in (1e-5, 1e-8, 1e-12):
        f.set_solver(rtol, 1000, precond_norm)
        xg, itg, resg = f.solve(v)
        xo, ito, reso = oracle.pcg(rp, ci, a, rhs, rtol, 1000, precond_norm)
        assert abs(itg - ito) <= 1, (rtol, itg, ito)
        assert resg <= rtol
        tol = 1e-9 if itg == ito else 10 * rtol
        assert np.abs(xg - xo).max() <= tol * np.abs(xo).max(), (rtol, np.abs(xg - xo).max())


@pytest.mark.gpu
def test_pcg_from_user_csr_and_autotune(cep, gpu, oracle):
    nx, ny = 40, 33
    D = _field(2, (nx, ny, 1), "tensor", seed=9)
    rp, ci, a, b = oracle.fem_assemble(2, nx, ny, 1, 0.025, 0.01, D)
    g = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, D).set_solver(1e-10)
    u = cep.Fem.csr(rp, ci, a, b, 0.01, fmt=cep.FEM_AUTO).set_solver(1e-10)
    assert u.format in (cep.FEM_CSR, cep.FEM_ELL)
    v = np.random.default_rng(1).uniform(-90, 30, g.n)
    xg, itg, _ = g.solve(v)
    xu, itu, _ = u.solve(v)
    assert itg == itu and np.array_equal(xg, xu)  # same matrix, same order: bitwise
    with pytest.raises(cep.CepError) as e:
        u.set_format(cep.FEM_STENCIL)  # no grid behind a user CSR
    assert e.value.code == cep.ERR_ARG
    u.set_format(cep.FEM_CSR)
    xc, itc, _ = u.solve(v)
    assert itc == itg and np.abs(xc - xg).max() <= 1e-12 * np.abs(xg).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dim,shape,kind", CASES)
def test_formats_give_identical_solves(cep, gpu, dim, shape, kind):
    """ELL and the implicit-column stencil sum each row in the same order, so
    their solves are bit-identical; CSR rows agree to rounding."""
    D = _field(dim, shape, kind, seed=7)
    nx, ny, nz = shape
    f = cep.Fem.grid(dim, nx, ny, nz, 0.025, 0.01, D).set_solver(1e-10)
    v = np.random.default_rng(3).uniform(-90, 30, f.n)
    out = {}
    for fmt in (cep.FEM_ELL, cep.FEM_STENCIL, cep.FEM_CSR):
        f.set_format(fmt)
        out[fmt] = f.solve(v)
    assert out[cep.FEM_ELL][1] == out[cep.FEM_STENCIL][1]
    assert np.array_equal(out[cep.FEM_ELL][0], out[cep.FEM_STENCIL][0])
    assert np.abs(out[cep.FEM_CSR][0] - out[cep.FEM_ELL][0]).max() <= 1e-9 * np.abs(v).max()


def _layered_field(nx, ny, nz):
    """Fibre-rotated tensor that varies with depth only, so a 3D grid has a
    few distinct rows per plane (the classed format applies)."""
    n_elem = (nx - 1) * (ny - 1) * (nz - 1)
    D = np.zeros((n_elem, 6))
    z = np.repeat(np.arange(nz - 1), (nx - 1) * (ny - 1))
    th = np.deg2rad(-60 + 120 * z / max(nz - 2, 1))
    dl, dt = 2e-3, 6e-4
    D[:, 0] = dt + (dl - dt) * np.cos(th) ** 2
    D[:, 1] = (dl - dt) * np.cos(th) * np.sin(th)
    D[:, 3] = dt + (dl - dt) * np.sin(th) ** 2
    D[:, 5] = dt
    return D


CLASSED_CASES = [(2, (40, 33, 1), 0.0013), (3, (14, 12, 9), "layered")]


@pytest.mark.gpu
@pytest.mark.parametrize("dim,shape,field", CLASSED_CASES)
def test_classed_format_is_bitwise_stencil(cep, gpu, oracle, dim, shape, field):
    """Rows grouped into coefficient classes read the same coefficients in
    the same slot order as the stencil format: SpMV and solves are bit for
    bit the stencil's, and the SpMV matches the oracle's CSR product."""
    nx, ny, nz = shape
    D = _layered_field(nx, ny, nz) if field == "layered" else field
    f = cep.Fem.grid(dim, nx, ny, nz, 0.025, 0.01, D, fmt=cep.FEM_CLASSED).set_solver(1e-10)
    assert f.format == cep.FEM_CLASSED
    rp, ci, a, b = oracle.fem_assemble(dim, nx, ny, nz, 0.025, 0.01, D)
    x = np.random.default_rng(4).uniform(-90, 30, f.n)
    ys = {}
    for fmt in (cep.FEM_CLASSED, cep.FEM_STENCIL):
        f.set_format(fmt)
        ys[fmt] = (f.spmv(x, "A"), f.spmv(x, "B"), f.solve(x))
    for k in range(2):
        assert np.array_equal(ys[cep.FEM_CLASSED][k], ys[cep.FEM_STENCIL][k])
    assert ys[cep.FEM_CLASSED][2][1] == ys[cep.FEM_STENCIL][2][1]
    assert np.array_equal(ys[cep.FEM_CLASSED][2][0], ys[cep.FEM_STENCIL][2][0])
    for which, val in ((0, a), (1, b)):
        ref = oracle.spmv(rp, ci, val, x)
        scale = oracle.spmv(rp, ci, np.abs(val), np.abs(x))
        assert np.all(np.abs(ys[cep.FEM_CLASSED][which] - ref) <= 1e-13 * scale)


@pytest.mark.gpu
def test_classed_format_refused_for_irregular_fields(cep, gpu):
    """Per-element random conductivities leave nearly every row distinct:
    the operator keeps no class table and refuses the format."""
    nx, ny = 30, 20
    f = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, _field(2, (nx, ny, 1), "tensor", seed=2))
    with pytest.raises(cep.CepError) as e:
        f.set_format(cep.FEM_CLASSED)
    assert e.value.code == cep.ERR_ARG


@pytest.mark.gpu
def test_pcg_edge_cases(cep, gpu, oracle):
    f = cep.Fem.grid(2, 9, 7, 1, 0.025, 0.01, 0.0013)
    x, it, res = f.solve(np.zeros(f.n))
    assert it == 0 and not x.any()
    # uniform V is reproduced exactly up to rounding (K annihilates constants)
    x, it, _ = f.set_solver(1e-12).solve(np.full(f.n, -85.0))
    assert np.abs(x + 85.0).max() < 1e-9
    # a capped iteration count reports NOT_CONVERGED, and the counters say so
    f.set_solver(1e-15, 2)
    v = np.random.default_rng(0).uniform(-90, 30, f.n)
    with pytest.raises(cep.CepError) as e:
        f.solve(v)
    assert e.value.code == cep.ERR_NOT_CONVERGED
    st = f.stats()
    assert st["not_converged"] == 1 and st["last_iters"] == -2
    # deterministic reductions: repeated solves are bit-identical
    f.set_solver(1e-8)
    x1, _, _ = f.solve(v)
    x2, _, _ = f.solve(v)
    assert np.array_equal(x1, x2)


def _tissue(cep, precision, nx, ny, mask, conc=0.0, hill=None, rtol=1e-10):
    n = nx * ny
    cells = cep.Batch("tt2006", n, precision)
    cells.init(conc=np.full(n, conc), hill=hill)
    fem = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, 0.0013).set_solver(rtol)
    t = cep.Tissue(cells, fem, 0.01)
    t.set_stimulus(mask, 1000.0, 0.0, 1.0, 1)
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tissue_tt2006_matches_oracle(cep, gpu, oracle, precision):
    """20 x 16 TT2006 sheet, corner S1, 12 ms (1200 Godunov steps)."""
    nx, ny, steps = 20, 16, 1200
    mask = np.zeros((ny, nx), np.uint8)
    mask[:3, :3] = 1
    hill = np.zeros(14)
    hill[12], hill[13] = 0.5, 1.0  # IKr block
    vo, itso, tacto = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, 0.01, steps, mask.ravel(), 1000.0,
                                        0.0, 1.0, 1, conc=0.3, hill=hill, rtol=1e-10)
    t = _tissue(cep, precision, nx, ny, mask.ravel(), conc=0.3, hill=hill)
    t.run(steps)
    st = t.stats()
    assert st["steps"] == steps and st["not_converged"] == 0
    vg, tactg = t.v(), t.activation()
    assert (tacto > 0).all() and (tactg > 0).all()
    if precision == "fp64":
        assert np.abs(vg - vo).max() <= 1e-6, np.abs(vg - vo).max()
        assert np.array_equal(tactg, tacto)
        assert abs(st["cg_iters"] - int(itso.sum())) <= 0.02 * itso.sum()
    else:
        assert np.abs(tactg - tacto).max() <= 0.1 + 1e-9, np.abs(tactg - tacto).max()


def _sheet(cep, nx, ny, conc, hill, precision="fp64", rtol=1e-10, fmt=None):
    n = nx * ny
    cells = cep.Batch("tt2006", n, precision)
    cells.init(conc=np.full(n, conc), hill=hill)
    fem = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, 0.0013, **({} if fmt is None else {"fmt": fmt})).set_solver(rtol)
    t = cep.Tissue(cells, fem, 0.01)
    mask = np.zeros((ny, nx), np.uint8)
    mask[:2, :2] = 1
    t.set_stimulus(mask.ravel(), 1000.0, 0.0, 1.0, 1)
    return t


@pytest.mark.gpu
def test_tissue_group_of_one_equals_alone(cep, gpu):
    hill = np.zeros(14)
    a = _sheet(cep, 18, 14, 0.0, hill)
    b = _sheet(cep, 18, 14, 0.0, hill)
    a.run(600)
    g = cep.TissueGroup([b])
    g.run(600)
    b.sync()
    assert np.array_equal(a.v(), b.v())
    assert np.array_equal(a.activation(), b.activation())
    assert a.stats()["cg_iters"] == b.stats()["cg_iters"]


@pytest.mark.gpu
def test_tissue_group_uneven_sheets_match_individual_runs(cep, gpu, oracle):
    """Three sheets of different sizes and drug concentrations stepped as a
    group give each sheet's own result (solver tolerance; activation times
    equal) and the smallest one matches the oracle."""
    hill = np.zeros(14)
    hill[12], hill[13] = 0.5, 1.0
    shapes = [(20, 16, 0.0), (12, 9, 0.3), (26, 21, 1.0)]
    steps = 900
    alone = []
    for nx, ny, c in shapes:
        t = _sheet(cep, nx, ny, c, hill)
        t.run(steps)
        alone.append((t.v(), t.activation()))
    group = [_sheet(cep, nx, ny, c, hill) for nx, ny, c in shapes]
    g = cep.TissueGroup(group)
    g.run(steps)
    for (v0, a0), t in zip(alone, group):
        t.sync()
        assert np.abs(t.v() - v0).max() <= 1e-6
        assert np.array_equal(t.activation(), a0)
        assert t.stats()["not_converged"] == 0
    nx, ny, c = shapes[1]
    mask = np.zeros((ny, nx), np.uint8)
    mask[:2, :2] = 1
    vo, _, _ = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, 0.01, steps, mask.ravel(), 1000.0, 0.0, 1.0,
                                 1, conc=c, hill=hill, rtol=1e-10)
    assert np.abs(group[1].v() - vo).max() <= 1e-6


@pytest.mark.gpu
def test_tissue_group_classed_equals_stencil(cep, gpu):
    """A group of uniform sheets stepped on the classed format gives the
    stencil format's V and activation times bit for bit."""
    hill = np.zeros(14)
    out = {}
    for fmt in (cep.FEM_STENCIL, cep.FEM_CLASSED):
        sheets = [_sheet(cep, nx, ny, c, hill, fmt=fmt) for nx, ny, c in ((24, 18, 0.0), (16, 16, 0.5))]
        cep.TissueGroup(sheets).run(700)
        for t in sheets:
            t.sync()
        out[fmt] = [(t.v(), t.activation(), t.stats()["cg_iters"]) for t in sheets]
    for (v0, a0, i0), (v1, a1, i1) in zip(out[cep.FEM_STENCIL], out[cep.FEM_CLASSED]):
        assert np.array_equal(v0, v1) and np.array_equal(a0, a1) and i0 == i1


@pytest.mark.gpu
def test_tissue_group_phase_timing(cep, gpu):
    """Per-phase events change nothing in the results and cover every
    step run while timing is on."""
    hill = np.zeros(14)
    plain = [_sheet(cep, 20, 17, 0.0, hill), _sheet(cep, 15, 15, 0.2, hill)]
    timed = [_sheet(cep, 20, 17, 0.0, hill), _sheet(cep, 15, 15, 0.2, hill)]
    cep.TissueGroup(plain).run(400)
    g = cep.TissueGroup(timed)
    g.run(100)
    g.set_timing(True)
    g.run(300)
    tm = g.timing()
    assert tm["steps"] == 300 and tm["ionic_ms"] > 0 and tm["diffusion_ms"] > 0
    g.set_timing(False)
    assert g.timing()["steps"] == 0
    for a, b in zip(plain, timed):
        a.sync()
        b.sync()
        assert np.array_equal(a.v(), b.v())


@pytest.mark.gpu
def test_ord_slab_3d_anisotropic_matches_oracle(cep, gpu, oracle):
    """3D ORd slab with endo/M/epi layers (per-node celltypes, quirks off),
    a fibre-rotated conductivity tensor per element and an endocardial S1:
    FP64 V and activation times against the oracle's tissue loop."""
    import bench
    nx, ny, nz, steps = 10, 9, 6, 500
    ct, D, mask = bench.slab_fields(nx, ny, nz)
    hill = np.zeros(14)
    hill[12], hill[13] = 0.8, 1.1
    vo, _, tacto = oracle.tissue_run("ord2011", 3, nx, ny, nz, 0.025, D, 0.01, steps, mask, 1000.0, 0.0, 1.0, 1,
                                     conc=0.4, hill=hill, rtol=1e-10, celltype=ct)
    n = nx * ny * nz
    cells = cep.Batch("ord2011", n, "fp64")
    cells.init(celltype=ct, conc=np.full(n, 0.4), hill=hill, quirks=False)
    fem = cep.Fem.grid(3, nx, ny, nz, 0.025, 0.01, D).set_solver(1e-10)
    t = cep.Tissue(cells, fem, 0.01)
    t.set_stimulus(mask, 1000.0, 0.0, 1.0, 1)
    t.run(steps)
    assert t.stats()["not_converged"] == 0
    assert (tacto > 0).all()
    assert np.abs(t.v() - vo).max() <= 1e-6
    assert np.array_equal(t.activation(), tacto)


ELECTRODES = [[0.1, 0.2, 1.0], [0.5, -0.3, 0.4], [0.2, 0.1, -0.6], [2.0, 2.0, 0.0]]


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_pseudo_ecg_matches_oracle(cep, gpu, oracle, dim):
    """The pseudo-ECG recorded after each step equals the oracle's
    restatement of Cheart::Radiate on the same V (relative 1e-10)."""
    if dim == 2:
        nx, ny, nz = 21, 17, 1
        D = _tensor_field(2, (nx - 1) * (ny - 1), 11)
        n = nx * ny
        cells = cep.Batch("tt2006", n, "fp64")
        cells.init()
        mask = np.zeros((ny, nx), np.uint8)
        mask[:3, :3] = 1
        mask = mask.ravel()
    else:
        import bench
        nx, ny, nz = 9, 8, 6
        ct, D, mask = bench.slab_fields(nx, ny, nz)
        n = nx * ny * nz
        cells = cep.Batch("ord2011", n, "fp64")
        cells.init(celltype=ct, quirks=False)
    fem = cep.Fem.grid(dim, nx, ny, nz, 0.025, 0.01, D).set_solver(1e-10)
    t = cep.Tissue(cells, fem, 0.01)
    t.set_stimulus(mask, 1000.0, 0.0, 1.0, 1)
    t.set_electrodes(ELECTRODES * 5, every=1, max_records=100)  # 20 electrodes: two chunks
    t.run(120)
    rec = t.ecg()
    assert rec.shape == (100, 20)
    t.set_electrodes(ELECTRODES * 5, every=1, max_records=5)
    t.run(1)
    last = t.ecg()[0]
    ref = oracle.pseudo_ecg(dim, nx, ny, nz, 0.025, D, t.v(), np.array(ELECTRODES * 5))
    assert np.abs(ref).max() > 0
    assert np.all(np.abs(last - ref) <= 1e-10 * np.abs(ref).max()), np.abs(last - ref).max()


@pytest.mark.gpu
def test_pseudo_ecg_cadence_and_limits(cep, gpu, oracle):
    n = 12 * 10
    cells = cep.Batch("tt2006", n, "mixed")
    cells.init()
    fem = cep.Fem.grid(2, 12, 10, 1, 0.025, 0.01, 0.0013)
    t = cep.Tissue(cells, fem, 0.01)
    t.set_electrodes(ELECTRODES[:2], every=3, max_records=2)
    t.run(10)
    assert t.ecg().shape == (2, 2)
    t.set_electrodes([], every=1, max_records=0)
    t.run(3)
    assert t.ecg().shape == (0, 0)
    rp, ci, a, b = oracle.fem_assemble(2, 12, 10, 1, 0.025, 0.01, 0.0013)
    u = cep.Fem.csr(rp, ci, a, b, 0.01)
    cells2 = cep.Batch("tt2006", n, "mixed")
    cells2.init()
    t2 = cep.Tissue(cells2, u, 0.01)
    with pytest.raises(cep.CepError) as e:
        t2.set_electrodes(ELECTRODES[:1])
    assert e.value.code == cep.ERR_UNSUPPORTED


def _s2_sheet(cep, kind, region, target, thr, ecto_dur):
    nx = ny = 16
    n = nx * ny
    cells = cep.Batch("tt2006", n, "fp64")
    cells.init()
    fem = cep.Fem.grid(2, nx, ny, 1, 0.025, 0.01, 0.0013).set_solver(1e-10)
    t = cep.Tissue(cells, fem, 0.01)
    mask = np.zeros((ny, nx), np.uint8)
    mask[:, :2] = 1
    t.set_stimulus(mask.ravel(), 1000.0, 0.0, 1.0, 1)
    if kind:
        t.set_s2(kind, target, thr, region, ecto_dur)
    return t, mask


@pytest.mark.gpu
@pytest.mark.parametrize("kind,thr,steps", [(1, -45.0, 28500), (2, -75.0, 30500)])
def test_s1s2_protocols_match_oracle(cep, gpu, oracle, kind, thr, steps):
    """S1-S2 reset (kind 1) and ectopic (kind 2) protocols, triggered on the
    device by a monitored node's depolarisation and repolarisation in the
    last S1 pace: FP64 V within 1e-6 mV and activation times equal to the
    oracle's tissue loop, and the protocol changed the result."""
    nx = ny = 16
    region = np.zeros((ny, nx), np.uint8)
    region[:6, 8:] = 1
    target = 8 + nx * 8
    t, mask = _s2_sheet(cep, kind, region.ravel(), target, thr, 2.0)
    t.run(steps)
    vo, _, tao = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, 0.01, steps, mask.ravel(), 1000.0, 0.0,
                                   1.0, 1, rtol=1e-10, s2_kind=kind, s2_target=target, s2_thr=thr,
                                   s2_region=region.ravel(), ecto_dur=2.0)
    assert np.abs(t.v() - vo).max() <= 1e-6
    assert np.array_equal(t.activation(), tao)
    plain, _ = _s2_sheet(cep, 0, None, 0, 0.0, 0.0)
    plain.run(steps)
    assert np.abs(plain.v() - t.v())[region.ravel() == 1].max() > 10.0  # shortly after the protocol fired


@pytest.mark.gpu
def test_s1s2_argument_checks(cep, gpu):
    t, _ = _s2_sheet(cep, 0, None, 0, 0.0, 0.0)
    with pytest.raises(cep.CepError):
        t.set_s2(7, 0, -45.0, np.ones(256, np.uint8))
    with pytest.raises(cep.CepError):
        t.set_s2(cep.S2_RESET, 256, -45.0, np.ones(256, np.uint8))
    t.set_s2(cep.S2_NONE, 0, 0.0)


@pytest.mark.gpu
def test_pcg_barrier_wait_runs_out_and_recovers(cep, gpu):
    """The one device-side failure form that is safe to provoke: with the
    grid barrier's spin limit cut to 64 polls and block 0 held back for
    5 ms before its first barrier, the other blocks' waits run out; every
    block leaves, the solve reports CEP_ERR_TIMEOUT, and once the hook is
    reset the next solve of the same operator is bit-identical to one that
    never timed out (the context stays usable)."""
    nx = 400  # 160,000 rows: every SM holds a block of the cooperative grid
    rng = np.random.default_rng(12)
    v = rng.uniform(-90, 30, nx * nx)
    ref = cep.Fem.grid(2, nx, nx, 1, 0.025, 0.01, 0.0013).set_solver(1e-9)
    xr, itr, _ = ref.solve(v)
    f = cep.Fem.grid(2, nx, nx, 1, 0.025, 0.01, 0.0013).set_solver(1e-9)
    lib = cep.lib()
    try:
        assert lib.cep_fem_set_wait_test(64, 5_000_000) == cep.OK
        with pytest.raises(cep.CepError) as e:
            f.solve(v)
        assert e.value.code == cep.ERR_TIMEOUT
    finally:
        assert lib.cep_fem_set_wait_test(0, 0) == cep.OK
    x, it, _ = f.solve(v)
    assert it == itr and np.array_equal(x, xr)
    assert lib.cep_fem_set_wait_test(-1, 0) == cep.ERR_ARG
