"""GPU mixed-product-basis projections (K4) against the product oracles, and the fused
products -> chi0 call against the chain oracle products -> oracle chi0."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import _lib, inputs
from project1_b200.wavefproducts import (MtDesc, PwDesc, chi0_from_coeffs, wavefproducts2_mt,
                                         wavefproducts2_pw)
from project1_b200.susceptibility import SpexGpuError, npack
from chi0_util import normalized_error
from wfprod_util import shifted_pw, small_workload

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
PROD_TOL = 1e-12          # max |error| / max |cprod|, FP64 products


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _cprod_dev(ncol, ldc, fill=0.0):
    return torch.full((ncol, ldc), fill, dtype=torch.complex128, device=DEV)


def _rel(got, ref):
    return np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)


@pytest.mark.parametrize("kw", [
    dict(), dict(natom=1, nunocc=1, nocc=1, nk=1), dict(nunocc=130, nocc=2, nk=1, lcutm=2),
    dict(lcut=4, nrad=3, lcutm=2, nradm=1, nunocc=65, nk=3)])
def test_mt_matches_oracle(ctx, kw):
    w = small_workload(**kw)
    mt = inputs.mt_basis(w)
    c1, c2 = inputs.mt_coeffs(w)
    ref = np.zeros((w.npair, w.nbasp), complex, order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, c1, c2, ref)
    cp = _cprod_dev(w.nbasp, w.npair)
    wavefproducts2_mt(ctx, mt, _dev(c1), _dev(c2), cp)
    got = cp.cpu().numpy().T
    assert _rel(got, ref) <= PROD_TOL


def test_mt_full_product_basis_few_bands(ctx):
    """The products workload's MT basis (lmax 8, 3 radial functions, 243 x 243 per atom, 5 % Gaunt)."""
    w = inputs.WfprodWorkload("c4sub", nk=1, nocc=3, nunocc=20)
    mt = inputs.mt_basis(w)
    c1, c2 = inputs.mt_coeffs(w)
    ref = np.zeros((w.npair, w.nbasp), complex, order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, c1, c2, ref)
    cp = _cprod_dev(w.nbasp, w.npair)
    wavefproducts2_mt(ctx, mt, _dev(c1), _dev(c2), cp)
    assert _rel(cp.cpu().numpy().T, ref) <= PROD_TOL


@pytest.mark.parametrize("kw,shifted", [
    (dict(), False), (dict(), True), (dict(nk=1, nocc=1, nunocc=1, ngptm=1), True),
    (dict(ngpt=150, ngptm=70, nunocc=100, step_radius=0), False),
    (dict(ngpt=120, ngptm=33, step_radius=4), True)])
def test_pw_matches_oracle(ctx, kw, shifted):
    w = small_workload(**kw)
    pw = shifted_pw(w) if shifted else inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = np.zeros((w.npair, w.ngptm), complex, order="F")
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, c1, c2, ref, 0)
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, pw, _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= PROD_TOL


def test_pw_full_basis_against_fft_branch(ctx):
    """The products workload's interstitial basis (3000 PW, 1014 MPB PW, 48^3 grid): checked against
    the numpy restatement of the reference's FFT branch on a few band pairs."""
    w = inputs.WfprodWorkload("c4sub", nk=1, nocc=2, nunocc=3)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = oracle.wfprod_pw_fft(pw, w.nk, w.nocc, w.nunocc, c1, c2, 48)
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, pw, _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= 1e-11


def test_products_respect_ldc_and_col0(ctx):
    """Padded leading dimension and a column offset: only the addressed block changes,
    and the products add to what is there."""
    w = small_workload(nk=2, nocc=2, nunocc=9)
    mt, pw = inputs.mt_basis(w), shifted_pw(w)
    m1, m2 = inputs.mt_coeffs(w)
    p1, p2 = inputs.pw_coeffs(w, pw)
    ldc, col0 = w.npair + 13, w.nbasp + 5
    ncol = col0 + w.ngptm + 3
    base = np.random.default_rng(1).standard_normal((ncol, ldc)) * (1 + 1j)
    cp = _dev(base)
    wavefproducts2_mt(ctx, mt, _dev(m1), _dev(m2), cp)
    wavefproducts2_pw(ctx, pw, _dev(p1), _dev(p2), cp, col0)
    got = cp.cpu().numpy()
    ref = base.T.copy(order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, m1, m2, ref, ldc)
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, p1, p2, ref, col0, ldc)
    assert _rel(got, ref.T) <= PROD_TOL
    assert np.array_equal(got[:, w.npair:], base[:, w.npair:])          # rows past npair
    assert np.array_equal(got[w.nbasp:col0], base[w.nbasp:col0])       # untouched columns
    assert np.array_equal(got[col0 + w.ngptm:], base[col0 + w.ngptm:])


def test_products_reject_bad_descriptors(ctx):
    w = small_workload(nk=1, nocc=1, nunocc=2)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    cp = _cprod_dev(w.ngptm, w.npair)
    bad = dict(pw, step_radius=5, cstep=np.zeros(11 ** 3, complex))
    with pytest.raises(SpexGpuError):
        wavefproducts2_pw(ctx, bad, _dev(c1), _dev(c2), cp, 0)
    with pytest.raises(SpexGpuError):
        wavefproducts2_pw(ctx, dict(pw, vol=0.0), _dev(c1), _dev(c2), cp, 0)
    with pytest.raises(SpexGpuError):   # ldc shorter than the pair count
        wavefproducts2_pw(ctx, pw, _dev(c1), _dev(c2), _cprod_dev(w.ngptm, w.npair - 1), 0)


def _fused_case(**kw):
    w = small_workload(**kw)
    mt, pw = inputs.mt_basis(w), shifted_pw(w)
    m1, m2 = inputs.mt_coeffs(w)
    p1, p2 = inputs.pw_coeffs(w, pw)
    rng = np.random.default_rng(5)
    ediff = rng.uniform(0.5, 40.0, w.npair)
    ediff[rng.choice(w.npair, max(1, w.npair // 100), replace=False)] = 3e-7
    omega = inputs.frequencies(3)
    return w, mt, pw, m1, m2, p1, p2, ediff, omega


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("split", 1e-6)])
def test_chi0_from_coeffs_matches_oracle_chain(ctx, precision, tol):
    w, mt, pw, m1, m2, p1, p2, ediff, omega = _fused_case(natom=1, lcut=2, lcutm=2, ngptm=30,
                                                         nk=2, nocc=4, nunocc=60)
    M = np.zeros((w.npair, w.nbas), complex, order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, m1, m2, M)
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, p1, p2, M, w.nbasp)
    ref = oracle.chi0(M, oracle.weights(ediff, omega, None, 0.5), accurate=True)
    sus = torch.zeros((len(omega), npack(w.nbas)), dtype=torch.complex128, device=DEV)
    st = chi0_from_coeffs(ctx, mt, pw, _dev(m1), _dev(m2), _dev(p1), _dev(p2), _dev(ediff),
                          _dev(omega), sus, scale_all=0.5, precision=precision, stats=True)
    got = sus.cpu().numpy().T
    emax, fro = normalized_error(got, ref, w.nbas)
    assert emax <= tol, (emax, fro)
    assert st["kernel_launches"] >= 5


@pytest.mark.parametrize("products", [_lib.SPX_PRODUCTS_FP64, _lib.SPX_PRODUCTS_SPLIT])
def test_chi0_from_coeffs_equals_products_then_accumulate(products):
    """The fused call is the composition of the three public calls, bit for bit, with
    the interstitial products in FP64 or on int8 slices alike."""
    ctx = spx.Context(0, products=products)
    w, mt, pw, m1, m2, p1, p2, ediff, omega = _fused_case(nk=1, nocc=3, nunocc=50)
    ldc = (w.npair + 15) // 16 * 16
    cp = _cprod_dev(w.nbas, ldc)
    wavefproducts2_mt(ctx, mt, _dev(m1), _dev(m2), cp)
    wavefproducts2_pw(ctx, pw, _dev(p1), _dev(p2), cp, w.nbasp)
    a = torch.zeros((len(omega), npack(w.nbas)), dtype=torch.complex128, device=DEV)
    ctx.chi0_accumulate_dev(cp, _dev(ediff), _dev(omega), a, precision="split", npair=w.npair,
                            stream=torch.cuda.current_stream().cuda_stream or 1)
    b = torch.zeros_like(a)
    chi0_from_coeffs(ctx, mt, pw, _dev(m1), _dev(m2), _dev(p1), _dev(p2), _dev(ediff),
                     _dev(omega), b, precision="split")
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    ctx.close()


# ---- FFT branch (src/wavefproducts.f:576-758) -------------------------------------

@pytest.mark.parametrize("kw,shifted,nfft", [
    (dict(), False, 24), (dict(), True, 24), (dict(nk=1, nocc=1, nunocc=1, ngptm=1), True, 20),
    (dict(ngpt=150, ngptm=70, nunocc=9, step_radius=0), False, 27),
    (dict(ngpt=120, ngptm=33, nunocc=5, step_radius=4), True, 30),
    # grid edges 16 r take the radix-16 x r line FFT
    (dict(), True, 16), (dict(ngpt=150, ngptm=70, nunocc=9), False, 64),
    (dict(nunocc=7), True, 48)])
def test_pw_fft_branch_matches_oracle(ctx, kw, shifted, nfft):
    w = small_workload(**kw)
    pw = shifted_pw(w) if shifted else inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = oracle.wfprod_pw_fft(pw, w.nk, w.nocc, w.nunocc, c1, c2, nfft)
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, dict(pw, nfft=nfft), _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= PROD_TOL


def test_pw_fft_branch_equals_explicit_without_aliasing(ctx):
    """On a grid that holds the whole product the two branches agree to rounding."""
    w = small_workload(nk=2, nocc=3, nunocc=40)
    pw = shifted_pw(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    a = _cprod_dev(w.ngptm, w.npair)
    b = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, pw, _dev(c1), _dev(c2), a, 0)
    wavefproducts2_pw(ctx, dict(pw, nfft=32), _dev(c1), _dev(c2), b, 0)
    assert _rel(b.cpu().numpy(), a.cpu().numpy()) <= PROD_TOL


def test_pw_fft_branch_aliasing_grid_follows_reference(ctx):
    """A grid too small for the product wraps around exactly as the reference's does."""
    w = small_workload(nk=1, nocc=2, nunocc=3, ngpt=100, ngptm=30)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = oracle.wfprod_pw_fft(pw, w.nk, w.nocc, w.nunocc, c1, c2, 9)
    exp = np.zeros((w.npair, w.ngptm), complex, order="F")
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, c1, c2, exp, 0)
    assert _rel(ref, exp) > 1e-6                                  # it does alias
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, dict(pw, nfft=9), _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= PROD_TOL


def test_pw_fft_branch_full_basis(ctx):
    """The products workload's interstitial basis on the 48^3 grid, a few band pairs."""
    w = inputs.WfprodWorkload("c4sub", nk=1, nocc=2, nunocc=3)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = oracle.wfprod_pw_fft(pw, w.nk, w.nocc, w.nunocc, c1, c2, 48)
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx, dict(pw, nfft=48), _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= 1e-11


def test_chi0_from_coeffs_fft_branch(ctx):
    w, mt, pw, m1, m2, p1, p2, ediff, omega = _fused_case(natom=1, lcut=2, lcutm=2, ngptm=30,
                                                         nk=2, nocc=3, nunocc=20)
    a = torch.zeros((len(omega), npack(w.nbas)), dtype=torch.complex128, device=DEV)
    b = torch.zeros_like(a)
    chi0_from_coeffs(ctx, mt, pw, _dev(m1), _dev(m2), _dev(p1), _dev(p2), _dev(ediff),
                     _dev(omega), a, precision="fp64")
    chi0_from_coeffs(ctx, mt, dict(pw, nfft=32), _dev(m1), _dev(m2), _dev(p1), _dev(p2),
                     _dev(ediff), _dev(omega), b, precision="fp64")
    emax, _ = normalized_error(b.cpu().numpy().T, a.cpu().numpy().T, w.nbas)
    assert emax <= 1e-10


def test_pw_fft_branch_rejects_bad_grids(ctx):
    w = small_workload(nk=1, nocc=1, nunocc=2)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    cp = _cprod_dev(w.ngptm, w.npair)
    with pytest.raises(SpexGpuError):
        wavefproducts2_pw(ctx, dict(pw, nfft=65), _dev(c1), _dev(c2), cp, 0)
    with pytest.raises(SpexGpuError):       # more than 16 distinct components per axis
        big = dict(pw, gptm=inputs._sphere(3000), nfft=48)
        wavefproducts2_pw(ctx, big, _dev(c1), _dev(c2), _cprod_dev(3000, w.npair), 0)


# ---- interstitial products on int8 digit slices (K4s) ---------------------------
# max |error| / max |cprod|. The slicing bound is 2^-17/127 * crest(A_m) * ||A_m|| ||B_col||
# (6e-8 times a crest factor of about 5-10 for the damped plane-wave rows); measured ~1e-7.
SPLIT_PROD_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx_split():
    c = spx.Context(0, products=_lib.SPX_PRODUCTS_SPLIT)
    yield c
    c.close()


@pytest.mark.parametrize("kw,shifted", [
    (dict(), False), (dict(), True), (dict(nk=1, nocc=1, nunocc=1, ngptm=1), True),
    (dict(ngpt=150, ngptm=70, nunocc=100, step_radius=0), False),
    (dict(ngpt=120, ngptm=33, nunocc=65, nk=3, step_radius=4), True)])
def test_pw_split_products_match_oracle(ctx_split, kw, shifted):
    w = small_workload(**kw)
    pw = shifted_pw(w) if shifted else inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ref = np.zeros((w.npair, w.ngptm), complex, order="F")
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, c1, c2, ref, 0)
    cp = _cprod_dev(w.ngptm, w.npair)
    wavefproducts2_pw(ctx_split, pw, _dev(c1), _dev(c2), cp, 0)
    assert _rel(cp.cpu().numpy().T, ref) <= SPLIT_PROD_TOL


def test_pw_split_products_full_basis(ctx, ctx_split):
    """The products workload's interstitial basis (3000 PW, 1014 MPB PW) against the FP64 GEMM,
    with a padded leading dimension and a column offset."""
    w = inputs.WfprodWorkload("c4sub", nk=2, nocc=3, nunocc=70)
    pw = inputs.pw_basis(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    ldc, col0 = w.npair + 7, 11
    a = _cprod_dev(col0 + w.ngptm, ldc, 0.5)
    b = _cprod_dev(col0 + w.ngptm, ldc, 0.5)
    wavefproducts2_pw(ctx, pw, _dev(c1), _dev(c2), a, col0)
    wavefproducts2_pw(ctx_split, pw, _dev(c1), _dev(c2), b, col0)
    a, b = a.cpu().numpy(), b.cpu().numpy()
    assert np.array_equal(b[:col0], a[:col0]) and np.array_equal(b[:, w.npair:], a[:, w.npair:])
    assert _rel(b - 0.5, a - 0.5) <= SPLIT_PROD_TOL
