"""The allocation-free entry point (spx_chi0_accumulate_dev_noalloc) through the C ABI.

It serves callers that cannot call cudaMalloc (a Fortran host whose device memory
belongs to its offload runtime or a pool allocator): the call takes no context and
keeps its scratch in a static device array. Here it must give the same result as
the ordinary FP64 entry point on two calls in a row (the second call reuses the
scratch left by the first), and it must reject a frequency count that does not
fit its scratch.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import project1_b200 as spx
from project1_b200 import _lib, inputs
from chi0_util import normalized_error

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
FP64_TOL = 1e-10


def _p(t):
    return C.c_void_p(int(t.data_ptr())) if t is not None else None


def _case(nbas, npair, nw, seed):
    rng = np.random.default_rng(seed)
    m = (rng.standard_normal((nbas, npair)) + 1j * rng.standard_normal((nbas, npair))) / np.sqrt(nbas)
    d = rng.uniform(0.5, 50.0, npair)
    d[rng.choice(npair, max(1, npair // 100), replace=False)] = 1e-7
    return (torch.from_numpy(m).to(DEV), torch.from_numpy(d).to(DEV),
            torch.from_numpy(inputs.frequencies(nw)).to(DEV))


@pytest.mark.parametrize("nbas,npair,nw", [(70, 3001, 5), (200, 20000, 24)])
def test_noalloc_matches_fp64_entry_point_twice(nbas, npair, nw):
    lib = _lib.load()
    m, d, om = _case(nbas, npair, nw, seed=nbas + npair)
    npk = spx.npack(nbas)
    ref = torch.zeros((nw, npk), dtype=torch.complex128, device=DEV)
    with spx.Context(0) as ctx:
        ctx.chi0_accumulate_dev(m, d, om, ref, scale_all=0.5, precision="fp64")
        torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.zeros((nw, npk), dtype=torch.complex128, device=DEV)
        rc = lib.spx_chi0_accumulate_dev_noalloc(_p(m), npair, npair, nbas, _p(d), None, 0.5, nw,
                                                 _p(om), _p(out), C.c_void_p(stream))
        assert rc == 0, (call, _lib.strerror(rc))
        emax, fro = normalized_error(out.cpu().numpy().T, ref.cpu().numpy().T, nbas)
        assert emax <= FP64_TOL and fro <= 1e-12, (call, emax, fro)


def test_noalloc_several_slabs_with_pair_scales():
    """nw = 512 leaves room for 8192 pairs of weights in the scratch, so 9001 pairs
    run as two slabs (8192 + 809): each slab reuses the scratch, offsets cprod, ediff
    and wscale, and adds into the output."""
    lib = _lib.load()
    nbas, npair, nw = 40, 9001, 512
    m, d, om = _case(nbas, npair, nw, seed=17)
    ws = torch.from_numpy(np.random.default_rng(2).uniform(0.5, 1.5, npair)).to(DEV)
    npk = spx.npack(nbas)
    ref = torch.zeros((nw, npk), dtype=torch.complex128, device=DEV)
    with spx.Context(0) as ctx:
        ctx.chi0_accumulate_dev(m, d, om, ref, wscale=ws, scale_all=0.25, precision="fp64")
        torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.zeros((nw, npk), dtype=torch.complex128, device=DEV)
        rc = lib.spx_chi0_accumulate_dev_noalloc(_p(m), npair, npair, nbas, _p(d), _p(ws), 0.25, nw,
                                                 _p(om), _p(out), C.c_void_p(stream))
        assert rc == 0, (call, _lib.strerror(rc))
        emax, fro = normalized_error(out.cpu().numpy().T, ref.cpu().numpy().T, nbas)
        assert emax <= FP64_TOL and fro <= 1e-12, (call, emax, fro)


def test_noalloc_rejects_frequency_count_beyond_scratch():
    lib = _lib.load()
    m, d, om = _case(4, 16, 1, seed=1)
    out = torch.zeros((1, 10), dtype=torch.complex128, device=DEV)
    rc = lib.spx_chi0_accumulate_dev_noalloc(_p(m), 16, 16, 4, _p(d), None, 1.0, 262145, _p(om),
                                             _p(out), None)
    assert rc == _lib.SPX_EINVAL
