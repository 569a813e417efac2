"""Product oracles (muffin tin, interstitial) against independent restatements, and the
synthetic product inputs. No GPU."""
import numpy as np

import oracle
from project1_b200 import inputs
from wfprod_util import mt_numpy, shifted_pw, small_workload


def test_mt_oracle_matches_closed_form_restatement():
    w = small_workload(nunocc=5)
    mt = inputs.mt_basis(w)
    c1, c2 = inputs.mt_coeffs(w)
    got = np.zeros((w.npair, w.nbasp), complex, order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, c1, c2, got)
    ref = mt_numpy(mt, w.nk, w.nocc, w.nunocc, c1, c2)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_mt_oracle_accumulates():
    w = small_workload(nunocc=4, natom=1)
    mt = inputs.mt_basis(w)
    c1, c2 = inputs.mt_coeffs(w)
    a = np.zeros((w.npair, w.nbasp), complex, order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, c1, c2, a)
    b = a.copy(order="F")
    oracle.wfprod_mt(mt, w.nk, w.nocc, w.nunocc, c1, c2, b)
    assert np.allclose(b, 2 * a, rtol=0, atol=1e-14 * np.abs(a).max())


def test_pw_explicit_oracle_matches_fft_path():
    """The explicit convolution (src/wavefproducts.f:760-997) and the FFT branch
    (:576-758) agree to rounding when the grid holds the product without aliasing."""
    w = small_workload(ngpt=80, ngptm=25, nk=2, nocc=2, nunocc=3)
    pw = shifted_pw(w)
    c1, c2 = inputs.pw_coeffs(w, pw)
    exp = np.zeros((w.npair, w.ngptm), complex, order="F")
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, c1, c2, exp, 0)
    fft = oracle.wfprod_pw_fft(pw, w.nk, w.nocc, w.nunocc, c1, c2, 24)
    assert np.abs(exp - fft).max() <= 1e-13 * np.abs(fft).max()


def test_pw_oracle_theta_one_is_plain_overlap():
    """With cstep = delta (theta = 1) the product is sum_G2 conj(c1(G2 - GM + g)) c2(G2)/sqrt(vol)."""
    w = small_workload(ngpt=60, ngptm=15, nk=1, nocc=2, nunocc=3, step_radius=1)
    pw = inputs.pw_basis(w)
    cs = np.zeros(27, complex)
    cs[13] = 1.0
    pw["cstep"] = cs
    c1, c2 = inputs.pw_coeffs(w, pw)
    got = np.zeros((w.npair, w.ngptm), complex, order="F")
    oracle.wfprod_pw(pw, w.nk, w.nocc, w.nunocc, c1, c2, got, 0)
    idx = {tuple(g): i for i, g in enumerate(pw["gpt1"])}
    ref = np.zeros_like(got)
    for n in range(w.nocc):
        for npr in range(w.nunocc):
            for ig, gm in enumerate(pw["gptm"]):
                s = 0
                for ig2, g2 in enumerate(pw["gpt2"]):
                    j = idx.get(tuple(g2 - gm + pw["gshift"]))
                    if j is not None:
                        s += c2[0, npr, ig2] * np.conj(c1[0, n, j])
                ref[npr + w.nunocc * n, ig] = s / np.sqrt(pw["vol"])
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()


def test_product_workload_shapes():
    w = inputs.WFPROD_CONFIGS["c4"]
    assert (w.maxlm, w.maxllm, w.nbasp, w.nbas, w.npair) == (243, 243, 486, 1500, 324000)
    pw = inputs.pw_basis(w)
    assert pw["gpt1"].shape == (3000, 3) and pw["gptm"].shape == (1014, 3)
    r1 = np.sqrt((pw["gpt1"].astype(float) ** 2).sum(1)).max()
    rm = np.sqrt((pw["gptm"].astype(float) ** 2).sum(1)).max()
    assert 8.5 < r1 < 9.5 and 6.0 < rm < 6.6
    # the step function is real in r space: cstep(-d) = conj(cstep(d))
    ns = 2 * w.step_radius + 1
    cs = pw["cstep"].reshape(ns, ns, ns, order="F")
    assert np.allclose(cs[::-1, ::-1, ::-1], np.conj(cs))
    # no aliasing on the 48^3 grid of the FFT branch
    span = 2 * np.abs(pw["gpt1"]).max() + w.step_radius + np.abs(pw["gptm"]).max()
    assert span < 48


def test_gaunt_table_density():
    w = inputs.WFPROD_CONFIGS["c4"]
    g = inputs.mt_basis(w)["gaunt"]
    L, Lm = w.lcut, w.lcutm
    valid = 0
    for LL in range(Lm + 1):
        for MM in range(-LL, LL + 1):
            for l in range(L + 1):
                for m in range(-l, l + 1):
                    for l1 in range(abs(l - LL), min(l + LL, L) + 1, 2):
                        valid += abs(m + MM) <= l1
    frac = np.count_nonzero(g) / valid
    assert 0.04 < frac < 0.06, frac


def test_batched_workload_draws():
    w = inputs.BATCHED_CONFIGS["c3"]
    qs = inputs.batched_qs(w)
    assert len(qs) == 32
    assert all(600 <= q.nbas <= 1800 and 20 <= q.nocc <= 60 and 150 <= q.nunocc <= 500 for q in qs)
    assert all(q.nk == 64 and q.nw == 24 for q in qs)
    assert len({q.seed for q in qs}) == 32
    assert qs == inputs.batched_qs(w)        # reproducible
    assert 5e15 < sum(q.flops for q in qs) < 1.2e16
