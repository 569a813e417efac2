"""libspexgpu loads, exports the declared ABI, and validates arguments (no GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import project1_b200 as spx
from project1_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(spx_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_abi_version_and_strerror():
    lib = _lib.load()
    assert lib.spx_abi_version() == 1
    assert _lib.strerror(0) == "ok"
    assert "invalid" in _lib.strerror(-1)


def test_null_context_is_rejected():
    lib = _lib.load()
    assert lib.spx_chi0_accumulate(None, None, 0, 0, 0, None, None, 1.0, 0, None, 0, None, None) == _lib.SPX_EINVAL
    assert lib.spx_ctx_destroy(None) == _lib.SPX_EINVAL
    assert lib.spx_ctx_synchronize(None) == _lib.SPX_EINVAL


def test_ctx_create_without_gpu_reports_nodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.spx_ctx_create(0, None, C.byref(h)) == _lib.SPX_ENODEV


def test_host_generator_is_deterministic_and_normal():
    a = spx.gen_normal_host(7, 3, 0, 200000)
    b = spx.gen_normal_host(7, 3, 0, 200000)
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1) < 0.01
    # offsets address the same stream
    c = spx.gen_normal_host(7, 3, 1001, 10)
    assert np.array_equal(c, a[1001:1011])
    # different stream ids differ
    assert not np.array_equal(spx.gen_normal_host(7, 4, 0, 10), a[:10])


def test_cmatrix_columns_are_addressable():
    full = spx.gen_cmatrix_host(5, 1, 37, 9, scale=0.5)
    part = spx.gen_cmatrix_host(5, 1, 37, 3, col0=4, scale=0.5)
    assert np.array_equal(full[:, 4:7], part)
    z = spx.gen_normal_host(5, 1, 2 * 37 * 4, 2 * 37 * 3, 0.5)
    assert np.array_equal(part.reshape(-1, order="F").view(np.float64), z)


def test_packed_index_and_unpack():
    n = 6
    sp = np.zeros((spx.npack(n), 1), complex, order="F")
    for j in range(n):
        for i in range(j + 1):
            sp[spx.packed_index(i, j), 0] = i + 10 * j + 1j * (i - j)
    full = spx.unpack_hermitian(sp, n)[0]
    assert np.allclose(full, full.conj().T)
    assert full[2, 4] == 2 + 40 + 1j * (2 - 4)
