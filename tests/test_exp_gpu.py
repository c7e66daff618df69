"""The FP64 policy's exponential (cep_device.cuh exp_tab: Tang's
table-driven method, N = 64) against CUDA's exp and against the host's
libm, over the argument ranges the models reach and the whole range of the
table path, plus the edges where it hands over to CUDA's exp.

Bars: within 1 ulp of CUDA's exp (itself within 1 ulp of e^x) and of the
host's exp everywhere; identical to CUDA's exp outside |x| < 707 and for
NaN and infinities."""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest


def _exp(cep, x: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    ref = np.empty_like(x)
    f = cep.lib().cep_internal_exp_f64
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    rc = f(x.ctypes.data, x.size, out.ctypes.data, ref.ctypes.data)
    assert rc == 0, cep.lib().cep_last_error()
    return out, ref


def _ulp_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|a - b| in units of the spacing at b (finite positive values)."""
    return np.abs(a - b) / np.spacing(b)


@pytest.mark.gpu
def test_exp_within_one_ulp_over_the_model_and_table_ranges(cep, gpu):
    rng = np.random.default_rng(5)
    x = np.concatenate([
        rng.uniform(-60.0, 60.0, 2_000_000),      # the models' arguments (V / k, a few 10s at most)
        rng.uniform(-706.999, 706.999, 2_000_000),  # the whole table path
        rng.uniform(-1e-3, 1e-3, 200_000),       # near 0: e^x - 1 dominated by r
        np.arange(-64 * 20, 64 * 20) * (math.log(2) / 64),  # table nodes (r near 0, j every value)
    ])
    out, ref = _exp(cep, x)
    assert np.isfinite(out).all() and (out > 0).all()
    d_cuda = _ulp_diff(out, ref)
    assert d_cuda.max() <= 1.0, (d_cuda.max(), x[d_cuda.argmax()])
    host = np.exp(x)
    d_host = _ulp_diff(out, host)
    assert d_host.max() <= 1.0, (d_host.max(), x[d_host.argmax()])
    # most results are the correctly rounded value CUDA's exp also returns
    assert (out == ref).mean() > 0.99


@pytest.mark.gpu
def test_exp_edges_hand_over_to_cuda(cep, gpu):
    edges = np.array([0.0, -0.0, 1e-300, -1e-300, 706.99, -706.99, 707.0, -707.0, 709.78, 709.79, -745.1, -745.2,
                      -708.5, 1000.0, -1000.0, np.inf, -np.inf, np.nan])
    out, ref = _exp(cep, edges)
    assert np.all(_ulp_diff(out[:6], ref[:6]) <= 1.0)  # the table path
    assert out[0] == 1.0 and out[1] == 1.0
    assert np.array_equal(out[6:], ref[6:], equal_nan=True)  # |x| >= 707, inf, NaN: CUDA's exp
