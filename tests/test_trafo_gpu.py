"""Transform to the Coulomb eigenbasis (src/susceptibility.f:806-832) against the
oracle's restatement of the reference's conj(matmul(conj(cprod), ctrafo))."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200.susceptibility import SpexGpuError

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-13   # max |error| / max |result|, FP64 DMMA


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _case(npair, nbas, dim, seed, ldc=None, ldt=None):
    rng = np.random.default_rng(seed)
    m = (rng.standard_normal((npair, nbas)) + 1j * rng.standard_normal((npair, nbas)))
    t = (rng.standard_normal((nbas, dim)) + 1j * rng.standard_normal((nbas, dim))) / np.sqrt(nbas)
    ldc = npair if ldc is None else ldc
    ldt = nbas if ldt is None else ldt
    md = torch.zeros((nbas, ldc), dtype=torch.complex128, device=DEV)
    md[:, :npair] = torch.from_numpy(np.ascontiguousarray(m.T))
    td = torch.zeros((dim, ldt), dtype=torch.complex128, device=DEV)
    td[:, :nbas] = torch.from_numpy(np.ascontiguousarray(t.T))
    return m, t, md, td


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("npair,nbas,dim", [(1000, 70, 50), (1, 1, 1), (333, 129, 130), (4097, 65, 64)])
def test_trafo_out_of_place(ctx, npair, nbas, dim):
    m, t, md, td = _case(npair, nbas, dim, seed=npair + nbas, ldc=npair + 3, ldt=nbas + 2)
    out = torch.full((dim, npair + 5), 7.0 + 0j, dtype=torch.complex128, device=DEV)
    ctx.trafo_dev(md, td, out, npair=npair)
    got = out.cpu().numpy()
    assert _rel(got[:, :npair].T, oracle.trafo(m, t)) <= TOL
    assert np.all(got[:, npair:] == 7.0)                     # rows past npair untouched


def test_trafo_in_place_several_chunks(ctx):
    """In place, as the reference does it, over more than one 65536-row chunk; the
    columns past dim keep their values."""
    npair, nbas, dim = 70000, 40, 24
    m, t, md, td = _case(npair, nbas, dim, seed=3)
    ctx.trafo_dev(md, td, None)
    got = md.cpu().numpy().T
    assert _rel(got[:, :dim], oracle.trafo(m, t)) <= TOL
    assert np.array_equal(got[:, dim:], m[:, dim:])


def test_trafo_rejects_bad_arguments(ctx):
    m, t, md, td = _case(100, 20, 10, seed=5)
    with pytest.raises(SpexGpuError):       # partial overlap of input and output
        rc = ctx.lib.spx_trafo_dev(ctx.handle, md.data_ptr(), 100, 100, 20, td.data_ptr(), 20, 10,
                                   md.data_ptr() + 16, 100, None)
        ctx._check(rc, "spx_trafo_dev")
    with pytest.raises(SpexGpuError):       # in place with another leading dimension
        rc = ctx.lib.spx_trafo_dev(ctx.handle, md.data_ptr(), 100, 100, 20, td.data_ptr(), 20, 10,
                                   md.data_ptr(), 101, None)
        ctx._check(rc, "spx_trafo_dev")


@pytest.mark.parametrize("inplace", [False, True])
def test_trafo_without_fullpw_matches_oracle(ctx, inplace):
    """The non-FULLPW branch (:814-824): interstitial rows of ctrafo multiplied by the
    plane-wave overlap (olapvec) before the transform; MT rows unchanged."""
    from project1_b200 import inputs
    from project1_b200.wavefproducts import PwDesc
    w = inputs.WFPROD_CONFIGS["c4"]
    basis = inputs.pw_basis(w)
    ng = 60
    gptm = basis["gptm"][:ng]
    pw = PwDesc(dict(basis, gptm=gptm))
    nbasp, npair, dim = 37, 3001, 90
    nbas = nbasp + ng
    m, t, md, td = _case(npair, nbas, dim, seed=12)
    ref = oracle.trafo_olap(m, t, nbasp, gptm, basis["cstep"], basis["step_radius"])
    if inplace:
        got = ctx.trafo_olap_dev(md, td, nbasp, pw)
        torch.cuda.synchronize()
        res = got.cpu().numpy()[:dim].T
    else:
        out = torch.zeros((dim, npair + 2), dtype=torch.complex128, device=DEV)
        ctx.trafo_olap_dev(md, td, nbasp, pw, out=out, npair=npair)
        torch.cuda.synchronize()
        res = out.cpu().numpy()[:, :npair].T
    assert _rel(res, ref) <= TOL
    # the overlap changes the result (it is not the FULLPW transform)
    assert _rel(oracle.trafo(m, t), ref) > 1e-3
