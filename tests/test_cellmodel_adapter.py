"""The C++ Cellmodel adapter (include/cep_cellmodel.hpp): a reference-style
driver compiles against it (CPU) and, on the GPU, reproduces the oracle /
the reference's own traces."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "cellmodel_driver.cpp"
LIBDIR = ROOT / "2ddrugsimulation_b200" / "lib"


def _build(tmp: Path) -> Path:
    exe = tmp / "cellmodel_driver"
    cuda = Path("/usr/local/cuda/lib64")
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           "-L", str(LIBDIR), "-lcep_b200", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath-link,{cuda}", "-L", str(cuda),
           f"-Wl,-rpath,{cuda}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def test_adapter_driver_compiles(cep, tmp_path):
    cep.lib()  # the library is built
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_adapter_ord_loop_matches_oracle(cep, gpu, oracle, tmp_path):
    exe = _build(tmp_path)
    n, stride = 40000, 400
    out = subprocess.run([str(exe), "ord", str(n), str(stride), "800"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    v = np.array([float(x) for x in out.stdout.split()])
    hill = np.array([1.5, 0.9, 20.0, 1.1, 0, 0, 3.0, 1.3, 5.0, 0.8, 12.0, 1.0, 0.7, 1.2])
    c = oracle.Cell("ord2011", 0.0, 0.4, hill, quirks=True)
    c.set_pacing(800.0)
    _, vo = c.run(0.0, 0.005, n, stride)
    assert len(v) == len(vo)
    assert np.abs(v - vo).max() <= 1e-6


@pytest.mark.gpu
def test_adapter_tt2006_tissue_flag_matches_reference_golden(cep, gpu, tmp_path):
    exe = _build(tmp_path)
    g = np.load(ROOT / "tests" / "golden" / "tt2006_tissue.npz")
    out = subprocess.run([str(exe), "tt06_tissue", str(int(g["n_on"])), str(int(g["n_off"])), str(int(g["stride"]))],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    v = np.array([float(x) for x in out.stdout.split()])
    assert np.abs(v - g["v_trace"]).max() <= 1e-6


@pytest.mark.gpu
def test_adapter_full_rates_and_constants_writes(cep, gpu, oracle, tmp_path):
    """computeRates fills every RATES entry of CiPA-ORd (the CVODE
    right-hand side of the reference), and the bench's CONSTANTS writes
    (BCL, GNa *= gna_scale) reach the device: the trace follows an oracle
    cell with the same constants within 1e-6 mV, and the RATES at every
    printed state equal the oracle's rates at that state (1e-9 relative to
    the largest rate of the state, FP64 with a different division)."""
    exe = _build(tmp_path)
    n, stride = 60000, 3000
    out = subprocess.run([str(exe), "cipa_rates", str(n), str(stride), "1000"], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    rows = np.array([[float(x) for x in ln.split()] for ln in out.stdout.strip().splitlines()])
    ns = 49
    hill = np.array([1.5, 0.9, 20.0, 1.1, 0, 0, 3.0, 1.3, 5.0, 0.8, 12.0, 1.0, 0, 0, 5e3, 2e-3, 0.9, 1e4, -40.0,
                     3.5e-5])
    c = oracle.Cell("cipa2017", 0.0, 0.4, hill, quirks=True)
    c.set_pacing(1000.0)
    c.scale(cep.SCALE["gna"], 0.7)
    t = 0.0
    for r in rows:
        steps = int(round((r[-1] - t) / 0.005))
        c.run(t, 0.005, steps)
        t = r[-1]
        assert abs(r[0] - c.states[0]) <= 1e-6, (t, r[0], c.states[0])
        c.y[:ns] = r[:ns]  # the oracle's rates at the adapter's own state
        ro, _ = c.rates(t)
        scale = np.abs(ro).max()
        assert np.abs(r[ns:2 * ns] - ro).max() <= 1e-9 * scale, (t, np.abs(r[ns:2 * ns] - ro).max(), scale)
