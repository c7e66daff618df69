"""Slab decomposition of a grid tissue (2ddrugsimulation_b200/slab.py) on
the CPU: the plane split against the library's rule, the split Jacobi-PCG
over the oracle's restatement of the parts (oracle.SlabPart) in one process
against the oracle's whole-operator PCG, and the same split across two gloo
ranks (one and two parts per rank) reproducing the one-process result bit
for bit (the parts' partial sums are added in part order on every rank).
The per-part compute here is the oracle, standing in for each rank's GPU."""
from __future__ import annotations

import ctypes
import importlib
import os
import socket

import numpy as np
import pytest

slab = importlib.import_module("2ddrugsimulation_b200.slab")

CASES = {
    "sheet": dict(dim=2, nx=13, ny=11, nz=1, h=0.025, dt=0.02),
    "slab": dict(dim=3, nx=7, ny=6, nz=9, h=0.025, dt=0.02),
}


def _tensor(case):
    """A rotated anisotropic conductivity per element, varying in space."""
    dim, nx, ny, nz = case["dim"], case["nx"], case["ny"], case["nz"]
    n_elem = (nx - 1) * (ny - 1) * (nz - 1 if dim == 3 else 1)
    rng = np.random.default_rng(5)
    ang = rng.uniform(0, np.pi, n_elem)
    dl, dt_ = 0.0013, 0.0004
    if dim == 2:
        c, s = np.cos(ang), np.sin(ang)
        return np.stack([dt_ + (dl - dt_) * c * c, (dl - dt_) * c * s, dt_ + (dl - dt_) * s * s], 1)
    f = np.stack([np.cos(ang), np.sin(ang), 0.3 * np.ones(n_elem)], 1)
    f /= np.linalg.norm(f, axis=1, keepdims=True)
    o = lambda a, b: dt_ * (a == b) + (dl - dt_) * f[:, a] * f[:, b]
    return np.stack([o(0, 0), o(0, 1), o(0, 2), o(1, 1), o(1, 2), o(2, 2)], 1)


def _v0(n):
    x = np.linspace(0.0, 1.0, n)
    return -85.0 + 100.0 * np.exp(-((x - 0.3) / 0.05) ** 2)


def _oracle_parts(O, case, D, n_parts, which):
    return [O.SlabPart(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D, k, n_parts)
            for k in which]


def _split_solve(parts, v, rtol, dist=None):
    s = slab.SlabSolver(parts, dist, check_every=3).set_solver(rtol, 500)
    vs = [v[p.row0: p.row0 + p.n_own].copy() for p in parts]
    iters, res = s.solve(vs)
    return np.concatenate(vs), iters, res


@pytest.mark.parametrize("n_planes", [1, 2, 5, 11, 48])
def test_plane_split_rule_matches_the_library(cep, n_planes):
    f = cep.lib().cep_part_split
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    for n_parts in range(1, n_planes + 1):
        covered = 0
        for k in range(n_parts):
            a, b = ctypes.c_int(), ctypes.c_int()
            assert f(n_planes, n_parts, k, ctypes.byref(a), ctypes.byref(b)) == 0
            assert slab.split(n_planes, n_parts, k) == (a.value, b.value)
            assert a.value == covered and b.value >= 1
            covered += b.value
        assert covered == n_planes
    assert f(n_planes, n_planes + 1, 0, None, None) != 0
    with pytest.raises(ValueError):
        slab.split(n_planes, n_planes + 1, 0)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("n_parts", [1, 2, 3])
def test_split_pcg_in_one_process_matches_the_whole_operator(oracle, name, n_parts):
    case = CASES[name]
    D = _tensor(case)
    rp, ci, av, bv = oracle.fem_assemble(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D)
    n = len(rp) - 1
    v = _v0(n)
    rtol = 1e-10
    x_ref, it_ref, _ = oracle.pcg(rp, ci, av, oracle.spmv(rp, ci, bv, v) / case["dt"], rtol, 500)
    parts = _oracle_parts(oracle, case, D, n_parts, range(n_parts))
    # the parts' rows are the whole operator's rows
    for p in parts:
        lo = p.plane if p.has_lo else 0
        r0, r1 = rp[p.row0], rp[p.row0 + p.n_own]
        assert np.array_equal(p.ci + (p.row0 - lo), ci[r0:r1]) and np.array_equal(p.av, av[r0:r1])
    x, iters, res = _split_solve(parts, v, rtol)
    assert it_ref > 0 and abs(iters - it_ref) <= 1, (iters, it_ref)
    assert res <= rtol
    assert np.abs(x - x_ref).max() <= 1e-7 * np.abs(x_ref).max()


def _rank_main(rank, world, port, name, n_parts, path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sl = importlib.import_module("2ddrugsimulation_b200.slab")
    case = CASES[name]
    D = _tensor(case)
    n = case["nx"] * case["ny"] * case["nz"]
    parts = [O.SlabPart(case["dim"], case["nx"], case["ny"], case["nz"], case["h"], case["dt"], D, k, n_parts)
             for k in sl.rank_parts(n_parts, world, rank)]
    s = sl.SlabSolver(parts, dist, check_every=3).set_solver(1e-10, 500)
    vs = [_v0(n)[p.row0: p.row0 + p.n_own].copy() for p in parts]
    iters, res = s.solve(vs)
    local = np.concatenate(vs)
    out = [None] * world if rank == 0 else None
    dist.gather_object((parts[0].row0, local, iters, res), out, dst=0)
    if rank == 0:
        out.sort(key=lambda t: t[0])
        np.savez(path, v=np.concatenate([t[1] for t in out]), iters=np.array([t[2] for t in out]),
                 res=np.array([t[3] for t in out]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,n_parts", [("sheet", 2), ("slab", 4)])
def test_two_gloo_ranks_reproduce_the_one_process_split(tmp_path, oracle, name, n_parts):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    path = str(tmp_path / "slab.npz")
    mp.start_processes(_rank_main, args=(2, port, name, n_parts, path), nprocs=2, join=True, start_method="spawn")
    got = np.load(path)
    case = CASES[name]
    D = _tensor(case)
    n = case["nx"] * case["ny"] * case["nz"]
    parts = _oracle_parts(oracle, case, D, n_parts, range(n_parts))
    x, iters, res = _split_solve(parts, _v0(n), 1e-10)
    assert (got["iters"] == iters).all() and (got["res"] == res).all()
    assert np.array_equal(got["v"], x)
