"""The oracle's seeded input generator (oracle/inputs_oracle.c) against the GPU
library's, and the accuracy of the series logarithm and sine / cosine both use.

The CPU baseline and the checker draw M from the oracle so that they never load the
product library; that is only sound if the two generators give the same bits. The
library's host generator runs on the CPU (no GPU call). The series functions are
checked against correctly rounded values (Python's decimal module, 50 digits):
ln within 3 ulp, sin / cos of 2 pi u within 2 ulp where |value| > 0.01 and within
2^-52 absolute everywhere. The GPU test compares the logarithm with CUDA's own.
"""
from decimal import Decimal, getcontext

import numpy as np
import pytest

import oracle
from project1_b200 import _lib
from project1_b200 import inputs

PI50 = Decimal("3.14159265358979323846264338327950288419716939937510")


def _library_cmatrix(seed, sid, rows, cols, col0, scale):
    import ctypes as C
    lib = _lib.load()
    out = np.empty((rows, cols), dtype=np.complex128, order="F")
    lib.spx_gen_cmatrix_host(C.c_uint64(seed), C.c_uint32(sid), rows, cols, rows, col0,
                             C.c_double(scale), C.c_void_p(out.ctypes.data))
    return out


@pytest.mark.parametrize("seed,sid,rows,cols,col0,scale", [
    (20261203, 1, 1000, 3, 0, 1.0), (20261203, 1, 4097, 2, 711, 0.0288675), (7, 9, 33, 5, 2, 2.5),
    (2**40 + 5, 3, 64, 1, 0, 1.0)])
def test_oracle_generator_is_bit_identical_to_the_library(seed, sid, rows, cols, col0, scale):
    a = oracle.gen_cmatrix(seed, sid, rows, cols, col0, scale)
    b = _library_cmatrix(seed, sid, rows, cols, col0, scale)
    assert a.tobytes(order="F") == b.tobytes(order="F")


def test_oracle_generator_matches_workload_columns():
    w = inputs.CONFIGS["c0"]
    a = oracle.gen_cmatrix(w.seed, w.stream_id, w.npair, 4, 396, w.m_scale)
    b = inputs.cprod_host(w, 396, 4)
    assert a.tobytes(order="F") == b.tobytes(order="F")


def _ulps(v: float, ref: Decimal) -> float:
    return float(abs(Decimal(v) - ref) / Decimal(np.spacing(abs(float(ref)))))


def test_series_log_within_3_ulp():
    getcontext().prec = 50
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(0, 1, 2000), np.exp(rng.uniform(-700, 700, 500)),
                        1 + rng.uniform(-1e-3, 1e-3, 300), [2.0 ** -53, 0.5, 2.0, 1e300]])
    y = oracle.series_log(x)
    worst = max(_ulps(v, Decimal(float(t)).ln()) for v, t in zip(y, x) if t != 1.0)
    assert worst <= 3.0, worst


def _sincos_turns_decimal(u: float):
    t = 2 * PI50 * Decimal(float(u))
    out = []
    for first, n0 in ((t, 1), (Decimal(1), 0)):
        acc, term, n = Decimal(0), first, n0
        while abs(term) > Decimal(10) ** -48:
            acc += term
            term = -term * t * t / ((n + 1) * (n + 2))
            n += 2
        out.append(acc)
    return out


def test_series_sincos_turns_accuracy():
    getcontext().prec = 50
    rng = np.random.default_rng(1)
    u = np.concatenate([rng.uniform(0, 1, 1500), np.arange(0, 1, 1 / 64), [1 - 2.0 ** -53]])
    s, c = oracle.series_sincos_turns(u)
    worst_ulp, worst_abs = 0.0, 0.0
    for uu, sv, cv in zip(u, s, c):
        rs, rc = _sincos_turns_decimal(uu)
        for v, r in ((sv, rs), (cv, rc)):
            worst_abs = max(worst_abs, float(abs(Decimal(v) - r)))
            if abs(r) > Decimal("0.01"):
                worst_ulp = max(worst_ulp, _ulps(v, r))
    assert worst_ulp <= 2.0 and worst_abs <= 2.0 ** -52, (worst_ulp, worst_abs)


@pytest.mark.gpu
def test_series_log_against_cuda_log():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(0, 1, 100000), np.exp(rng.uniform(-700, 700, 10000))])
    ours = oracle.series_log(x)
    cuda = torch.log(torch.from_numpy(x).to("cuda:0")).cpu().numpy()
    ulp = np.abs(ours - cuda) / np.spacing(np.abs(cuda))
    assert np.max(ulp) <= 4.0, np.max(ulp)   # 3 ulp of ours plus CUDA log's own 1 ulp
