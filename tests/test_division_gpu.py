"""The FP64 path's division and reciprocal (div64 / rcp64 in
csrc/cep_device.cuh: Newton-Raphson refinement of the hardware reciprocal
seed) against IEEE division.

Bound: within 1 ulp of the correctly rounded quotient (numpy's a / b) for
normal quotients and divisors of magnitude up to 2^1021; the IEEE result
exactly for zero, subnormal, infinite and NaN divisors, infinite and zero
dividends, and overflowing quotients; within 1 ulp of the smallest
subnormal for subnormal quotients. The test compiles a small kernel
(tests/cpp/div64_check.cu) against the library's own device header with
the library's flags."""
from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _lib(tmp: Path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    so = tmp / "libdiv64.so"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "--prec-div=false", "--prec-sqrt=false", "--ftz=true", "-I", str(ROOT / "2ddrugsimulation_b200" / "csrc"),
           "-o", str(so), str(ROOT / "tests" / "cpp" / "div64_check.cu")]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    L = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    L.div64_check.argtypes = [dp, dp, dp, dp, ctypes.c_int]
    return L, dp


def _ulps(x, y):
    """Distance in units in the last place (same sign, finite)."""
    xi = x.view(np.int64)
    yi = y.view(np.int64)
    return np.abs(xi - yi)


@pytest.mark.gpu
def test_div64_and_rcp64_against_ieee(gpu, tmp_path):
    L, dp = _lib(tmp_path)
    rng = np.random.default_rng(5)
    n = 1 << 20
    a = rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-300, 300, n)
    b = rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-300, 300, n)
    sub = np.array([5e-324, -5e-324, 1e-310, -2.2e-308, 1.5e-315])
    edges_b = np.concatenate([[0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0], sub, [2.0 ** -1021, 2.0 ** 1021]])
    edges_a = np.array([1.0, -3.5, 0.0, -0.0, np.inf, -np.inf, np.nan, 1e308, 1e-300, 7.0])
    ea, eb = np.meshgrid(edges_a, edges_b)
    a = np.concatenate([a, ea.ravel(), [1e300, 1e-300, 3e-310]])
    b = np.concatenate([b, eb.ravel(), [1e-300, 1e300, 7.0]])
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    q = np.zeros_like(a)
    r = np.zeros_like(a)
    assert L.div64_check(a.ctypes.data_as(dp), b.ctypes.data_as(dp), q.ctypes.data_as(dp), r.ctypes.data_as(dp),
                         len(a)) == 0
    with np.errstate(all="ignore"):
        qi = a / b
        ri = 1.0 / b
    for got, ref in ((q, qi), (r, ri)):
        nan = np.isnan(ref)
        assert np.array_equal(np.isnan(got), nan)
        fin = np.isfinite(ref) & ~nan
        inf = np.isinf(ref)
        assert np.array_equal(got[inf], ref[inf])  # overflow and division by zero: signed inf
        zero = fin & (ref == 0)
        assert (got[zero] == 0).all()
        normal = fin & (np.abs(ref) >= np.finfo(float).tiny)
        assert (np.sign(got[normal]) == np.sign(ref[normal])).all()
        assert _ulps(np.abs(got[normal]), np.abs(ref[normal])).max() <= 1
        tiny = fin & (ref != 0) & ~normal
        assert (np.abs(got[tiny] - ref[tiny]) <= 5e-324).all()
