"""Instance sharding across ranks (one process per GPU).

A screening population is independent per instance, so the multi-GPU path
partitions it and needs no data-path collective: each rank runs whole
samples (a sample with all its concentrations stays on one rank, so the
qInward control of a sample is local, as the reference keeps it per MPI
rank: CEPCell_NEO/modules/cipa_drug_bench.cpp:127-132), and only the final
biomarker records are gathered to rank 0 (the reference's MPI_Reduce at
DrugSimulation/main.cpp:252 plays that role).
"""
from __future__ import annotations

import numpy as np


def sample_range(n_samples: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced range of samples owned by `rank` (sizes differ
    by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(n_samples, world)
    s0 = rank * base + min(rank, extra)
    return s0, s0 + base + (1 if rank < extra else 0)


def instance_range(n_samples: int, n_conc: int, world: int, rank: int) -> tuple[int, int]:
    """Instances [i0, i1) of a sample-major population (sample s, conc c at
    s * n_conc + c) owned by `rank`."""
    s0, s1 = sample_range(n_samples, world, rank)
    return s0 * n_conc, s1 * n_conc


def gather_records(local: dict, world: int, rank: int, pg=None) -> dict | None:
    """Concatenate every rank's per-instance arrays on rank 0 in rank order
    (None elsewhere). `pg` is torch.distributed (any backend) or None for a
    single process."""
    if pg is None or world == 1:
        return {k: np.asarray(v) for k, v in local.items()}
    parts = [None] * world if rank == 0 else None
    pg.gather_object({k: np.asarray(v) for k, v in local.items()}, parts, dst=0)
    if rank != 0:
        return None
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
