"""CPU oracle for the SPEX polarisation hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline; the product never
imports it.

PARITY UNPINNED: the reference (SPEX 05.10, Fortran) cannot be compiled in this
image and ships no tests, golden vectors or fixtures for the path. The C
restatement (chi0_oracle.c, wfprod_oracle.c) follows the reference loops
line by line (citations in the C sources) and is cross-checked against an
independent numpy formulation (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        srcs = list(HERE.glob("*.c")) + [HERE / "Makefile"]
        if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
            build()
        lib = C.CDLL(str(LIB))
        P, I64, I32, D = C.c_void_p, C.c_int64, C.c_int32, C.c_double
        lib.oracle_weights.argtypes = [I64, P, P, D, I32, P, P]
        lib.oracle_chi0_faithful.argtypes = [I64, I32, P, I64, P, I32, P, C.c_int]
        lib.oracle_chi0_accurate.argtypes = [I64, I32, P, I64, P, I32, P, C.c_int]
        lib.oracle_chi0_element.argtypes = [I64, P, P, P, I32, P]
        lib.oracle_scale.argtypes = [P, I64, D]
        lib.oracle_max_threads.restype = C.c_int
        for name in ("oracle_weights", "oracle_chi0_faithful", "oracle_chi0_accurate",
                     "oracle_chi0_element", "oracle_scale"):
            getattr(lib, name).restype = None
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def weights(ediff, omega, wscale=None, scale_all: float = 1.0) -> np.ndarray:
    """w (npair, nw), Fortran order (src/susceptibility.f:950-975)."""
    ediff = np.ascontiguousarray(ediff, dtype=np.float64)
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    ws = None if wscale is None else np.ascontiguousarray(wscale, dtype=np.float64)
    w = np.zeros((ediff.shape[0], omega.shape[0]), dtype=np.float64, order="F")
    load().oracle_weights(ediff.shape[0], _p(ediff), _p(ws), scale_all, omega.shape[0], _p(omega), _p(w))
    return w


def chi0(cprod, w, accurate: bool = False, threads: int = 0, susceph=None) -> np.ndarray:
    """susceph (npack, nw) += body loop of src/susceptibility.f:1182-1240."""
    cprod = np.asfortranarray(cprod, dtype=np.complex128)
    w = np.asfortranarray(w, dtype=np.float64)
    npair, nbas = cprod.shape
    nw = w.shape[1]
    if susceph is None:
        susceph = np.zeros((nbas * (nbas + 1) // 2, nw), dtype=np.complex128, order="F")
    fn = load().oracle_chi0_accurate if accurate else load().oracle_chi0_faithful
    fn(npair, nbas, _p(cprod), npair, _p(w), nw, _p(susceph), threads)
    return susceph


def chi0_element(a, b, w) -> np.ndarray:
    """chi(i, j, :) for columns a = cprod(:, i), b = cprod(:, j); extended precision."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    w = np.asfortranarray(w, dtype=np.float64)
    out = np.zeros(w.shape[1], dtype=np.complex128)
    load().oracle_chi0_element(a.shape[0], _p(a), _p(b), _p(w), w.shape[1], _p(out))
    return out


def max_threads() -> int:
    return load().oracle_max_threads()
