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


def _mom_case(seed=3, natom=2, lcut=3, nrad=2, nk=2, nocc=3, nunocc=5, ngpt=70):
    from project1_b200 import inputs
    rng = np.random.default_rng(seed)
    maxlm = (lcut + 1) ** 2 * nrad
    c1 = rng.standard_normal((nk, nocc, natom, maxlm)) + 1j * rng.standard_normal((nk, nocc, natom, maxlm))
    c2 = rng.standard_normal((nk, nunocc, natom, maxlm)) + 1j * rng.standard_normal((nk, nunocc, natom, maxlm))
    basis = inputs.pw_basis(inputs.WFPROD_CONFIGS["c4"])
    gpt = basis["gpt1"][:ngpt]
    p1 = rng.standard_normal((nk, nocc, ngpt)) + 1j * rng.standard_normal((nk, nocc, ngpt))
    p2 = rng.standard_normal((nk, nunocc, ngpt)) + 1j * rng.standard_normal((nk, nunocc, ngpt))
    m = dict(natom=natom, lcut=lcut, nrad=nrad, qmat1=rng.standard_normal((nrad, nrad, lcut + 1)),
             qmat2=rng.standard_normal((nrad, nrad, lcut + 1)), gpt=gpt,
             kpt=rng.uniform(-0.5, 0.5, (nk, 3)), rlat=2 * np.pi / 10.0 * (np.eye(3) + 0.1 * rng.standard_normal((3, 3))),
             cstep=basis["cstep"], step_radius=basis["step_radius"], vol=1000.0)
    return m, c1, c2, p1, p2


@pytest.mark.parametrize("with_ediff", [False, True])
def test_dcprod_matches_momentum_matrix_oracle(with_ediff):
    """dcprod from the MT and plane-wave coefficients against the restated
    momentum_matrix (src/dwavefproducts.f:89-330) and the scaling of
    src/susceptibility.f:858-869."""
    from project1_b200.wavefproducts import MomDesc, dcprod_dev
    m, c1, c2, p1, p2 = _mom_case()
    nk, nocc, nunocc = c1.shape[0], c1.shape[1], c2.shape[1]
    mom = oracle.momentum_matrix(c1, c2, p1, p2, m["lcut"], m["nrad"], m["qmat1"], m["qmat2"], m["gpt"],
                                 m["kpt"], m["rlat"], m["cstep"], m["step_radius"])
    npair = nk * nocc * nunocc
    ref = mom.reshape((npair, 3), order="F") / np.sqrt(m["vol"])
    ed = None
    if with_ediff:
        rng = np.random.default_rng(8)
        e = rng.uniform(0.5, 20.0, npair)
        e[5] = 1e-9                                 # |rdum| <= 1e-8: the element is dropped
        ref = ref / e[:, None]
        ref[5] = 0.0
        ed = torch.from_numpy(e).to(DEV)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)
    out = torch.full((3, npair + 4), 7.0 + 0j, dtype=torch.complex128, device=DEV)
    with spx.Context(0) as c:
        dcprod_dev(c, MomDesc(m), nk, nocc, nunocc, D(c1), D(c2), D(p1), D(p2), out, ediff=ed)
        torch.cuda.synchronize()
    got = out.cpu().numpy()[:, :npair].T
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(out.cpu().numpy()[:, npair:] == 7.0)          # padding untouched
