"""Hilbert-mesh path on the imaginary axis: effective pair weights from tetrahedron
weights and getwghtS (src/susceptibility.f:996-1078, src/hilbert.f:193-300), and the
accumulation with caller-given weights."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import inputs
from project1_b200.susceptibility import npack
from chi0_util import normalized_error

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _d(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def test_hilbert_weights_match_oracle(ctx):
    rng = np.random.default_rng(4)
    P, S, nw = 5003, 60, 5
    wt = rng.uniform(0, 1, (P, S)) * (rng.uniform(0, 1, (P, S)) > 0.8)
    ws = rng.standard_normal((S, nw))
    ref = oracle.hilbert_weights(wt, ws, thr=0.05, scale_all=0.25)
    w = torch.zeros((nw, P + 3), dtype=torch.float64, device=DEV)
    ctx.weights_hilbert_dev(_d(wt.T), _d(ws.T), w, thr=0.05, scale_all=0.25, npair=P)
    got = w.cpu().numpy()[:, :P].T
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_accumulate_with_given_weights(ctx, precision, tol):
    """Weights of both signs (a real-axis style table), ragged sizes."""
    rng = np.random.default_rng(9)
    nbas, P, nw = 97, 40001, 3
    m = np.asfortranarray((rng.standard_normal((P, nbas)) + 1j * rng.standard_normal((P, nbas))) / np.sqrt(nbas))
    w = rng.standard_normal((P, nw))
    ref = oracle.chi0(m, w, accurate=True)
    out = torch.zeros((nw, npack(nbas)), dtype=torch.complex128, device=DEV)
    wd = torch.zeros((nw, P + 1), dtype=torch.float64, device=DEV)
    wd[:, :P] = _d(w.T)
    st = ctx.chi0_accumulate_w_dev(_d(m.T), wd, out, precision=precision, npair=P, stats=True)
    assert st["kernel_launches"] >= 1
    got = out.cpu().numpy().T
    # chi is no longer semidefinite: compare against the element scale sqrt(sum |M_i|^2 |M_j|^2 |w|)
    scale = np.sqrt(np.einsum("pi,pf->if", np.abs(m) ** 2, np.abs(w)))
    iu, ju = np.triu_indices(nbas)
    idx = ju * (ju + 1) // 2 + iu
    err = np.abs(got[idx] - ref[idx]) / (scale[iu] * scale[ju])
    assert err.max() <= tol, err.max()


def test_hilbert_path_reproduces_hilbert_none(ctx):
    """Pairs whose energy difference sits on a mesh point, each a unit-area hat on the
    mesh: the Hilbert path through the GPU gives the HILBERT NONE chi0 up to the mesh
    discretisation."""
    w = inputs.small("h", nbas=48, nk=2, nocc=4, nunocc=30, nw=4)
    frqs = np.concatenate([[0.0], np.geomspace(1e-2, 80.0, 300)])
    rng = np.random.default_rng(2)
    P = w.npair
    s0 = rng.integers(60, 290, P)                    # the pair's mesh point
    ediff = frqs[s0]
    omega = inputs.frequencies(w.nw)
    wr, _ = oracle.getwghtS(1j * omega, frqs, 0.0, 0, 0)
    wt = np.zeros((P, frqs.size))
    wt[np.arange(P), s0] = 2.0 / (frqs[s0 + 1] - frqs[s0 - 1])
    m = inputs.cprod_host(w)
    wd = torch.zeros((w.nw, P), dtype=torch.float64, device=DEV)
    ctx.weights_hilbert_dev(_d(wt.T), _d(wr.T), wd, scale_all=1.0 / w.nk)
    a = torch.zeros((w.nw, npack(w.nbas)), dtype=torch.complex128, device=DEV)
    ctx.chi0_accumulate_w_dev(_d(m.T), wd, a, precision="fp64", stats=True)
    b = torch.zeros_like(a)
    ctx.chi0_accumulate_dev(_d(m.T), _d(ediff), _d(omega), b, scale_all=1.0 / w.nk, stats=True)
    emax, _ = normalized_error(a.cpu().numpy().T, b.cpu().numpy().T, w.nbas)
    assert emax <= 5e-3, emax


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_real_frequency_suscepc_matches_oracle(ctx, precision, tol):
    """Real frequencies (suscepc): Hilbert weights wghtSr / wghtSi of real frequencies
    from getwghtS, contracted with tetrahedron weights on the device, then the full
    non-Hermitian matrix against the reference loop restated (:1182-1235)."""
    rng = np.random.default_rng(21)
    nbas, P, nw = 70, 3001, 4
    frqs = np.concatenate([[0.0], np.geomspace(0.05, 60.0, 120)])
    frqc = np.array([0.0, 1.3, 7.7, 25.0]) + 0j            # real frequencies
    wsr, wsi = oracle.getwghtS(frqc, frqs, 0.01, 0, 0)
    assert np.abs(wsi).max() > 0                            # the imaginary part matters
    wt = rng.uniform(0, 1, (P, frqs.size)) * (rng.uniform(0, 1, (P, frqs.size)) > 0.9)
    wr_ref = oracle.hilbert_weights(wt, wsr, scale_all=0.5)
    wi_ref = oracle.hilbert_weights(wt, wsi, scale_all=0.5)
    m = np.asfortranarray((rng.standard_normal((P, nbas)) + 1j * rng.standard_normal((P, nbas))) / np.sqrt(nbas))
    ref = oracle.chi0_realfreq(m, wr_ref, wi_ref)            # (nbas, nbas, nw)
    wrd = torch.zeros((nw, P), dtype=torch.float64, device=DEV)
    wid = torch.zeros((nw, P), dtype=torch.float64, device=DEV)
    ctx.weights_hilbert_dev(_d(wt.T), _d(wsr.T), wrd, scale_all=0.5)
    ctx.weights_hilbert_dev(_d(wt.T), _d(wsi.T), wid, scale_all=0.5)
    ldo = nbas + 3
    out = torch.zeros((nw, nbas, ldo), dtype=torch.complex128, device=DEV)
    st = ctx.chi0_accumulate_c_dev(_d(m.T), wrd, wid, out, precision=precision, stats=True)
    assert st["kernel_launches"] >= 3
    got = np.transpose(out.cpu().numpy()[:, :, :nbas], (2, 1, 0))   # (i, j, f)
    scale = np.sqrt(np.einsum("pi,pf->if", np.abs(m) ** 2, np.abs(wr_ref) + np.abs(wi_ref)))
    err = np.abs(got - ref) / (scale[:, None, :] * scale[None, :, :])
    assert err.max() <= tol, err.max()
    # the padding rows of suscepc are untouched
    assert out[:, :, nbas:].abs().max().item() == 0.0
