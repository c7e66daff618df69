"""Slab parts on the GPU (csrc/slab.cu through 2ddrugsimulation_b200/
slab.py), K parts on one device with their halo planes and partial sums
moved as the multi-GPU path moves them: the parts' rows bit-equal to the
whole operator's, the split diffusion solve against the whole-operator
solve and against the oracle's split (oracle.SlabPart), and a slab tissue
against the single tissue and the oracle's tissue."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from test_slab import CASES, _tensor, _v0

slab = importlib.import_module("2ddrugsimulation_b200.slab")


def _parts(case, D, n_parts):
    return [slab.DevicePart(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D, k, n_parts)
            for k in range(n_parts)]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("n_parts", [1, 2, 3])
def test_part_rows_are_the_whole_operators_rows(cep, gpu, name, n_parts):
    case = CASES[name]
    D = _tensor(case)
    fem = cep.Fem.grid(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D)
    rp, ci, av, bv = fem.get_csr()
    for p in _parts(case, D, n_parts):
        prp, pci, pav, pbv = p.csr()
        r0, r1 = rp[p.row0], rp[p.row0 + p.n_own]
        assert np.array_equal(prp, rp[p.row0: p.row0 + p.n_own + 1] - r0)
        assert np.array_equal(pci, ci[r0:r1])
        assert np.array_equal(pav, av[r0:r1]) and np.array_equal(pbv, bv[r0:r1])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("n_parts", [2, 3])
def test_split_solve_matches_the_whole_solve_and_the_oracle_split(cep, gpu, oracle, name, n_parts):
    import torch
    case = CASES[name]
    D = _tensor(case)
    n = case["nx"] * case["ny"] * case["nz"]
    v = _v0(n)
    rtol = 1e-10
    fem = cep.Fem.grid(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D)
    fem.set_solver(rtol, 500)
    x_whole, it_whole, _ = fem.solve(v)
    parts = _parts(case, D, n_parts)
    s = slab.SlabSolver(parts, check_every=4).set_solver(rtol, 500)
    vs = [torch.tensor(v[p.row0: p.row0 + p.n_own], dtype=torch.float64, device="cuda") for p in parts]
    iters, res = s.solve(vs)
    x = np.concatenate([t.cpu().numpy() for t in vs])
    assert it_whole > 0 and abs(iters - it_whole) <= 1, (iters, it_whole)
    assert res <= rtol
    assert np.abs(x - x_whole).max() <= 1e-7 * np.abs(x_whole).max()
    ops = [oracle.SlabPart(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D, k, n_parts)
           for k in range(n_parts)]
    so = slab.SlabSolver(ops, check_every=4).set_solver(rtol, 500)
    vo = [v[p.row0: p.row0 + p.n_own].copy() for p in ops]
    it_o, _ = so.solve(vo)
    assert abs(iters - it_o) <= 1
    assert np.abs(x - np.concatenate(vo)).max() <= 1e-8 * np.abs(x).max()


@pytest.mark.gpu
def test_slab_tissue_matches_the_single_tissue_and_the_oracle(cep, gpu, oracle):
    """A 20 x 18 TT2006 sheet, corner S1, 12 ms, split into three slabs of
    rows (the wave crosses both boundaries): V within 1e-6 mV and activation
    times equal against the oracle's whole tissue, as the single tissue."""
    nx, ny, steps, dt = 20, 18, 1200, 0.01
    mask = np.zeros((ny, nx), np.uint8)
    mask[:3, :3] = 1
    hill = np.zeros(14)
    hill[12], hill[13] = 0.5, 1.0
    vo, _, tacto = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, dt, steps, mask.ravel(), 1000.0, 0.0, 1.0,
                                     1, conc=0.3, hill=hill, rtol=1e-10)
    parts = [slab.DevicePart(2, nx, ny, 1, 0.025, dt, 0.0013, k, 3) for k in range(3)]
    cells = []
    for p in parts:
        c = cep.Batch("tt2006", p.n_own, "fp64", stream=p.stream.cuda_stream)
        c.init(conc=np.full(p.n_own, 0.3), hill=hill)
        cells.append(c)
    t = slab.SlabTissue(parts, cells, dt)
    t.solver.set_solver(1e-10, 10000)
    t.set_stimulus([mask.ravel()[p.row0: p.row0 + p.n_own] for p in parts], 1000.0, 0.0, 1.0, 1)
    t.run(steps)
    v = np.concatenate([c.get_states()[:, 0] for c in cells])
    tact = np.concatenate([p.activation() for p in parts])
    assert min(t.iters) > 0
    assert (tacto > 0).all() and (tact > 0).all()
    assert np.abs(v - vo).max() <= 1e-6, np.abs(v - vo).max()
    assert np.array_equal(tact, tacto)
