"""q -> 0 head and wings (src/susceptibility.f:1092-1157) in FP64 against the oracle's
restatement of the reference loops."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-12   # max |error| / max |value|


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("npair,dim,nw", [(40000, 70, 3), (1, 1, 1), (16385, 0, 2), (1100000, 8, 2)])
def test_headwings_match_oracle(ctx, npair, dim, nw):
    rng = np.random.default_rng(npair + dim)
    c = rng.standard_normal((npair, dim)) + 1j * rng.standard_normal((npair, dim))
    d = rng.standard_normal((npair, 3)) + 1j * rng.standard_normal((npair, 3))
    w = rng.standard_normal((npair, nw))
    h0 = rng.standard_normal((6, nw)) + 1j * rng.standard_normal((6, nw))
    g0 = rng.standard_normal((3, dim, nw)) + 1j * rng.standard_normal((3, dim, nw))
    href, gref = oracle.headwings(c, d, w)
    href, gref = href + h0, gref + g0                     # the call adds
    head = _d(h0.T)                                       # (nw, 6) == Fortran (6, nw)
    wing = _d(np.transpose(g0, (2, 1, 0)))                # (nw, dim, 3) == Fortran (3, dim, nw)
    cd = _d(c.T) if dim else torch.zeros((0, npair), dtype=torch.complex128, device=DEV)
    ctx.headwings_dev(cd, _d(d.T), _d(w.T), head, wing, npair=npair)
    assert _rel(head.cpu().numpy().T, href) <= TOL
    if dim:
        assert _rel(np.transpose(wing.cpu().numpy(), (2, 1, 0)), gref) <= TOL


def test_headwings_are_the_augmented_gram(ctx):
    """Head and wings are the rows k < 3 of the weighted Gram of [dcprod | cprod], the
    same sum the body accumulation forms: chi0 of the augmented panel agrees."""
    rng = np.random.default_rng(5)
    npair, dim, nw = 3000, 20, 2
    c = (rng.standard_normal((npair, dim)) + 1j * rng.standard_normal((npair, dim))) / 5
    d = (rng.standard_normal((npair, 3)) + 1j * rng.standard_normal((npair, 3))) / 5
    w = -np.abs(rng.standard_normal((npair, nw)))
    x = np.asfortranarray(np.hstack([d, c]))
    g = oracle.chi0(x, w, accurate=True)                 # packed (i <= j) over 3 + dim
    head = torch.zeros((nw, 6), dtype=torch.complex128, device=DEV)
    wing = torch.zeros((nw, dim, 3), dtype=torch.complex128, device=DEV)
    ctx.headwings_dev(_d(c.T), _d(d.T), _d(w.T), head, wing)
    h = head.cpu().numpy().T
    wg = np.transpose(wing.cpu().numpy(), (2, 1, 0))
    for k2 in range(3):
        for k1 in range(k2 + 1):
            assert np.allclose(h[k2 * (k2 + 1) // 2 + k1], g[k2 * (k2 + 1) // 2 + k1], rtol=1e-12, atol=1e-14)
        for i in range(dim):
            j = 3 + i
            assert np.allclose(wg[k2, i], np.conj(g[j * (j + 1) // 2 + k2]), rtol=1e-12, atol=1e-14)
