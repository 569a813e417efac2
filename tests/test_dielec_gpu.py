"""Dielectric matrix eps = 1 - v^1/2 chi v^1/2 and its inverse (src/correlation.f:614-636,
703-745) in FP64, against the oracle's restatement."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import inputs
from project1_b200.susceptibility import SpexGpuError, npack

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _chi(nbas, nw, seed):
    """A negative semi-definite packed chi from the HILBERT NONE body loop."""
    rng = np.random.default_rng(seed)
    P = 4 * nbas
    m = np.asfortranarray((rng.standard_normal((P, nbas)) + 1j * rng.standard_normal((P, nbas))) / np.sqrt(nbas))
    d = rng.uniform(0.5, 30.0, P)
    om = inputs.frequencies(nw)
    return oracle.chi0(m, oracle.weights(d, om, None, 1.0 / 4)), rng.uniform(0.1, 40.0, nbas)


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("nbas,nw,invert", [(50, 2, False), (50, 2, True), (300, 3, True), (1, 1, True), (129, 1, True),
                                            (64, 2, True), (700, 4, True)])
def test_dielec_matches_oracle(ctx, nbas, nw, invert):
    chi, coul = _chi(nbas, nw, seed=nbas)
    ref = oracle.dielec(chi, coul, invert)
    sus = _d(chi.T)
    ctx.dielec_dev(sus, _d(coul), invert=invert)
    got = sus.cpu().numpy().T
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_dielec_head_and_wings(ctx):
    nbas, nw = 20, 2
    chi, coul = _chi(nbas, nw, seed=3)
    rng = np.random.default_rng(1)
    head = rng.standard_normal((6, nw)) + 1j * rng.standard_normal((6, nw))
    wing = rng.standard_normal((3, nbas, nw)) + 1j * rng.standard_normal((3, nbas, nw))
    ref, href, gref = oracle.dielec(chi, coul, True, head, wing)
    sus, hd, wg = _d(chi.T), _d(head.T), _d(np.transpose(wing, (2, 1, 0)))
    ctx.dielec_dev(sus, _d(coul), invert=True, head=hd, wing=wg)
    assert np.allclose(sus.cpu().numpy().T, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    assert np.allclose(hd.cpu().numpy().T, href, rtol=1e-14, atol=1e-14)
    assert np.allclose(np.transpose(wg.cpu().numpy(), (2, 1, 0)), gref, rtol=1e-14, atol=1e-14)


def test_dielec_rejects_indefinite(ctx):
    """A positive chi large enough to make eps indefinite is reported, not inverted."""
    nbas = 16
    chi = np.zeros((npack(nbas), 2), complex, order="F")
    for j in range(nbas):
        chi[j * (j + 1) // 2 + j] = 3.0            # chi = 3 I, eps = 1 - 3 v
    sus = _d(chi.T)
    with pytest.raises(SpexGpuError, match="frequency 0"):
        ctx.dielec_dev(sus, _d(np.ones(nbas)), invert=True)


def test_dielec_reports_the_indefinite_frequency(ctx):
    """Only the second frequency's eps is indefinite (its pivot fails in a later block):
    the error names that frequency."""
    nbas = 150
    chi, coul = _chi(nbas, 2, seed=5)
    chi[:, 1] = 0.0
    for j in range(nbas):
        chi[j * (j + 1) // 2 + j, 1] = 0.0 if j < 100 else 3.0 / coul[j]     # eps_jj = 1 - 3 for j >= 100
    with pytest.raises(SpexGpuError, match="frequency 1"):
        ctx.dielec_dev(_d(chi.T), _d(coul), invert=True)
