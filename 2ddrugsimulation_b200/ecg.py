"""Twelve-lead ECG from the pseudo-ECG of nine electrodes, as
Cbspm::writeECG (bspm.cpp:63-87) derives and writes it.

Electrodes, in the order the reference keeps them (ecgl.vnode): RA, LA, LL,
V1 .. V6. With the Wilson central terminal W = (RA + LA + LL) / 3:
  I = LA - RA, II = LL - RA, III = LL - LA;
  aVR, aVL, aVF = 1.5 (RA - W), 1.5 (LA - W), 1.5 (LL - W);
  V1 .. V6 = Vk - W.
The electrode potentials come from cep_tissue_get_ecg (Tissue.ecg()).
"""
from __future__ import annotations

import numpy as np

LEADS = ("I", "II", "III", "aVR", "aVL", "aVF", "V1", "V2", "V3", "V4", "V5", "V6")


def twelve_lead(phi) -> np.ndarray:
    """[records, 9] electrode potentials -> [records, 12] leads, with the
    reference's operation order."""
    v = np.atleast_2d(np.asarray(phi, np.float64))
    if v.shape[1] != 9:
        raise ValueError("twelve_lead needs 9 electrodes: RA, LA, LL, V1..V6")
    w = (v[:, 0] + v[:, 1] + v[:, 2]) / 3.0
    out = np.empty((v.shape[0], 12))
    out[:, 0] = v[:, 1] - v[:, 0]
    out[:, 1] = v[:, 2] - v[:, 0]
    out[:, 2] = v[:, 2] - v[:, 1]
    for k in range(3):
        out[:, 3 + k] = 1.5 * (v[:, k] - w)
    for k in range(6):
        out[:, 6 + k] = v[:, 3 + k] - w
    return out


def write_ecg(path, times, phi) -> None:
    """One line per record: the time then the twelve leads, "%lf " each
    (bspm.cpp:81-85)."""
    leads = twelve_lead(phi)
    t = np.asarray(times, np.float64).reshape(-1)
    if len(t) != len(leads):
        raise ValueError("one time per record")
    with open(path, "w") as fh:
        for ti, row in zip(t, leads):
            fh.write("%f " % ti + "".join("%f " % x for x in row) + "\n")
