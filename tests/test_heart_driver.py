"""A heart.cpp-style tissue driver in C++ over the C ABI (tests/cpp/
heart_driver.cpp): it compiles against the header (CPU) and, on the GPU,
its final V, activation times and ECG match the oracle's tissue loop and
pseudo-ECG."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "heart_driver.cpp"
LIBDIR = ROOT / "2ddrugsimulation_b200" / "lib"


def _build(tmp: Path) -> Path:
    exe = tmp / "heart_driver"
    cuda = Path("/usr/local/cuda/lib64")
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           "-L", str(LIBDIR), "-lcep_b200", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath-link,{cuda}", "-L", str(cuda),
           f"-Wl,-rpath,{cuda}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def test_heart_driver_compiles(cep, tmp_path):
    cep.lib()
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_heart_driver_matches_oracle(cep, gpu, oracle, tmp_path):
    exe = _build(tmp_path)
    nx, ny, steps, conc, ic50, hh = 18, 14, 1500, 0.3, 0.5, 1.1
    out = subprocess.run([str(exe), str(nx), str(ny), str(steps), str(conc), str(ic50), str(hh)], capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    vals = np.array([float(x) for x in out.stdout.split()])
    n = nx * ny
    v, tact, ecg = vals[:n], vals[n:2 * n], vals[2 * n]
    mask = np.zeros((ny, nx), np.uint8)
    mask[:, :2] = 1
    hill = np.zeros(14)
    hill[12], hill[13] = ic50, hh
    vo, _, tao = oracle.tissue_run("tt2006", 2, nx, ny, 1, 0.025, 0.0013, 0.01, steps, mask.ravel(), 1000.0, 0.0, 1.0,
                                   1, conc=conc, hill=hill, rtol=1e-10)
    assert np.abs(v - vo).max() <= 1e-6
    assert np.array_equal(tact, tao)
    eo = oracle.pseudo_ecg(2, nx, ny, 1, 0.025, 0.0013, v, [[0.5 * (nx - 1) * 0.025, -0.5, 1.0]])[0]
    assert abs(ecg - eo) <= 1e-10 * abs(eo)
