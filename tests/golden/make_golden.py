"""Generate the golden fixtures in tests/golden/ from the reference cell
models compiled from their own sources (oracle/_ref, built by
`make -C oracle ref` where the reference tree is present).

    python tests/golden/make_golden.py

Each fixture holds the inputs (celltype, concentration, Hill row, flags),
the reference's V trace sampled every `stride` steps of its explicit loop
(computeRates(t); solveAnalytical(dt); t += dt), its final STATES, and its
RATES at t = 0. The oracle and the GPU path are checked against these files
on machines where the reference itself is not available.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def hill_row(rng: np.random.Generator, skip: tuple[int, ...] = ()) -> np.ndarray:
    """Seeded Hill row: IC50 log-uniform in [0.1, 100] uM, h uniform in
    [0.6, 1.8] (the single-cell configuration's ranges)."""
    h = np.zeros(14)
    h[0::2] = 10 ** rng.uniform(-1, 2, 7)
    h[1::2] = rng.uniform(0.6, 1.8, 7)
    for ch in skip:
        h[2 * ch] = 0.0  # NA in the reference CSV -> 0 -> no block
    return h


def ord_cases():
    rng = np.random.default_rng(20240611)
    return [
        dict(name="ord_control", celltype=0.0, conc=0.0, hill=np.zeros(14), dutta=0),
        dict(name="ord_drug_dutta", celltype=0.0, conc=3.0, hill=hill_row(rng), dutta=1),
        dict(name="ord_drug_epi_skip", celltype=1.0, conc=10.0, hill=hill_row(rng, skip=(2,)), dutta=0),
        dict(name="ord_drug_mcell_dutta", celltype=2.0, conc=0.7, hill=hill_row(rng), dutta=1),
    ]


def make_ord(n_beats: int = 2, dt: float = 0.005, stride: int = 200, bcl: float = 1000.0):
    for c in ord_cases():
        r = O.RefCell("ord2011", c["celltype"], c["conc"], c["hill"], is_dutta=bool(c["dutta"]))
        r.consts[140] = bcl  # CONSTANTS[BCL]
        y0 = r.states.copy()
        r.L.ref_compute_rates(r.h, 0.0)
        rates0 = r.arr("rates", r.n).copy()
        n = int(round(n_beats * bcl / dt))
        t, v = r.run(0.0, dt, n, stride)
        np.savez_compressed(OUT / f"{c['name']}.npz", celltype=c["celltype"], conc=c["conc"], hill=c["hill"],
                            dutta=c["dutta"], dt=dt, stride=stride, bcl=bcl, n_steps=n, y0=y0, rates0=rates0,
                            v_trace=v, final_states=r.states.copy(), t_final=t)
        print("wrote", c["name"], "vmax", v.max())


if __name__ == "__main__":
    if not O.ref_available("ord2011"):
        sys.exit("reference models not built: run `make -C oracle ref` where the reference tree exists")
    make_ord()
