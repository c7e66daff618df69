"""Instance sharding for the multi-GPU path (2ddrugsimulation_b200/shard.py):
balanced whole-sample ranges, and a world-size-2 gloo run on CPU whose
gathered records equal a single-process run. The per-rank compute here is
the oracle (test infrastructure standing in for each rank's GPU batch)."""
from __future__ import annotations

import importlib
import os
import socket

import numpy as np
import pytest

shard = importlib.import_module("2ddrugsimulation_b200.shard")


@pytest.mark.parametrize("n,world", [(1, 1), (7, 2), (8, 2), (2000, 8), (3, 4), (10, 3)])
def test_sample_ranges_partition(n, world):
    got = [shard.sample_range(n, world, r) for r in range(world)]
    assert got[0][0] == 0 and got[-1][1] == n
    for (a0, a1), (b0, b1) in zip(got, got[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in got]
    assert max(sizes) - min(sizes) <= 1
    i = [shard.instance_range(n, 5, world, r) for r in range(world)]
    assert i[0][0] == 0 and i[-1][1] == 5 * n and all(x[1] - x[0] == 5 * s for x, s in zip(i, sizes))


def test_bad_rank_rejected():
    with pytest.raises(ValueError):
        shard.sample_range(4, 2, 2)


def _population(n_samples, n_conc):
    rng = np.random.default_rng(17)
    hill = np.zeros((n_samples, 14))
    hill[:, 0::2] = 10 ** rng.uniform(-1, 2, (n_samples, 7))
    hill[:, 1::2] = rng.uniform(0.6, 1.8, (n_samples, 7))
    hill = np.repeat(hill, n_conc, axis=0)
    conc = np.tile(np.arange(n_conc) * 0.7, n_samples)
    return conc, hill


def _compute(conc, hill):
    from oracle import oracle as O
    out = {"apd90": [], "qnet": [], "cad90": []}
    for c, h in zip(conc, hill):
        cell = O.Cell("ord2011", 0.0, float(c), h, quirks=True)
        cell.set_pacing(1000.0)
        bm, _ = cell.run_biomarkers(0.005, 2, 1)
        for k in out:
            out[k].append(bm[k])
    return out


def _rank_main(rank, world, port, n_samples, n_conc, path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sh = importlib.import_module("2ddrugsimulation_b200.shard")
    conc, hill = _population(n_samples, n_conc)
    i0, i1 = sh.instance_range(n_samples, n_conc, world, rank)
    local = _compute(conc[i0:i1], hill[i0:i1])
    got = sh.gather_records(local, world, rank, dist)
    if rank == 0:
        np.savez(path, **got)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_gather_equals_single_process(tmp_path, oracle):
    import torch.multiprocessing as mp
    n_samples, n_conc = 3, 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    path = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(2, port, n_samples, n_conc, path), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(path)
    conc, hill = _population(n_samples, n_conc)
    ref = _compute(conc, hill)
    for k in ref:
        assert np.array_equal(got[k], np.array(ref[k])), k
