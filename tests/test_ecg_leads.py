"""Twelve-lead ECG derivation and file format of Cbspm::writeECG
(bspm.cpp:63-87)."""
from __future__ import annotations

import importlib

import numpy as np
import pytest

ecg = importlib.import_module("2ddrugsimulation_b200.ecg")


def test_leads_follow_the_wilson_terminal_definitions():
    rng = np.random.default_rng(2)
    phi = rng.normal(size=(5, 9))
    L = ecg.twelve_lead(phi)
    ra, la, ll = phi[:, 0], phi[:, 1], phi[:, 2]
    w = (ra + la + ll) / 3.0
    assert np.array_equal(L[:, 0], la - ra) and np.array_equal(L[:, 1], ll - ra) and np.array_equal(L[:, 2], ll - la)
    assert np.allclose(L[:, 0] + L[:, 2], L[:, 1])            # Einthoven: I + III = II
    assert np.allclose(L[:, 3] + L[:, 4] + L[:, 5], 0.0)        # aVR + aVL + aVF = 0
    assert np.array_equal(L[:, 6:], phi[:, 3:] - w[:, None])
    # a common offset on every electrode changes no lead
    assert np.allclose(ecg.twelve_lead(phi + 7.0), L)
    with pytest.raises(ValueError):
        ecg.twelve_lead(phi[:, :8])


def test_ecg_file_format(tmp_path):
    phi = np.arange(18, dtype=float).reshape(2, 9)
    ecg.write_ecg(tmp_path / "ecg.plt", [0.5, 1.0], phi)
    rows = [ln.split() for ln in (tmp_path / "ecg.plt").read_text().splitlines()]
    assert len(rows) == 2 and all(len(r) == 13 for r in rows)
    assert rows[0][0] == "0.500000" and float(rows[0][1]) == 1.0  # I = LA - RA
    assert (tmp_path / "ecg.plt").read_text().splitlines()[0].endswith(" ")
