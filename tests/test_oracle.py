"""The CPU oracle against the independent numpy golden vectors (no GPU)."""
import numpy as np
import pytest

import oracle

G = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "chi0_golden.npz")
CASES = sorted({k.split("/")[0] for k in G.files if "/" in k})


def case(name):
    ws = G[f"{name}/wscale"] if f"{name}/wscale" in G.files else None
    return (G[f"{name}/cprod"], G[f"{name}/ediff"], G[f"{name}/omega"], ws,
            G[f"{name}/w"], G[f"{name}/susceph"])


@pytest.mark.parametrize("name", CASES)
def test_weights_match_golden(name):
    m, d, om, ws, w, _ = case(name)
    got = oracle.weights(d, om, ws, float(G["scale_all"]))
    np.testing.assert_allclose(got, w, rtol=1e-14, atol=0)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("accurate", [False, True])
def test_chi0_matches_golden(name, accurate):
    m, d, om, ws, w, ref = case(name)
    got = oracle.chi0(m, w, accurate=accurate, threads=2)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= 1e-13 * scale


def test_packet_split_invariance():
    """Accumulating MEM packets one after another gives the same chi (src/susceptibility.f:751-758)."""
    m, d, om, ws, w, ref = case("small_degenerate")
    acc = None
    for b, e in [(0, 13), (13, 40), (40, 60)]:
        acc = oracle.chi0(m[b:e], w[b:e], susceph=acc)
    assert np.max(np.abs(acc - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_hermitian_diagonal_real_and_negative():
    """Single-sign weights: chi(iw) is Hermitian negative semi-definite, so the diagonal is real <= 0."""
    m, d, om, ws, w, ref = case("ragged")
    n = m.shape[1]
    diag = np.array([j * (j + 1) // 2 + j for j in range(n)])
    assert np.all(np.abs(ref[diag].imag) <= 1e-15 * np.abs(ref[diag].real).max())
    assert np.all(ref[diag].real <= 0)
    for f in range(ref.shape[1]):
        full = np.zeros((n, n), complex)
        iu, ju = np.triu_indices(n)
        full[iu, ju] = ref[ju * (ju + 1) // 2 + iu, f]
        full[ju, iu] = np.conj(full[iu, ju])
        assert np.linalg.eigvalsh(full).max() <= 1e-14 * np.abs(full).max()


def test_element_sampler_matches_full():
    m, d, om, ws, w, ref = case("small_degenerate")
    for (i, j) in [(0, 0), (3, 17), (23, 23), (5, 6)]:
        got = oracle.chi0_element(m[:, i], m[:, j], w)
        np.testing.assert_allclose(got, ref[j * (j + 1) // 2 + i], rtol=1e-13, atol=1e-16)


def test_linearity_in_weights():
    m, d, om, ws, w, ref = case("tiny")
    a = oracle.chi0(m, 2.5 * w)
    np.testing.assert_allclose(a, 2.5 * ref, rtol=1e-13, atol=1e-17)


def test_trafo_oracle_is_the_reference_formula():
    """conj(conj(M) T) equals M conj(T): the two forms of src/susceptibility.f:806-832."""
    rng = np.random.default_rng(1)
    m = rng.standard_normal((30, 8)) + 1j * rng.standard_normal((30, 8))
    t = rng.standard_normal((8, 5)) + 1j * rng.standard_normal((8, 5))
    assert np.allclose(oracle.trafo(m, t), m @ np.conj(t), rtol=0, atol=1e-14)
    assert np.allclose(oracle.trafo(m, t, dim=3), (m @ np.conj(t))[:, :3], rtol=0, atol=1e-14)


def test_getwghtS_hat_reproduces_the_pole_weight():
    """A unit-area hat at a mesh point, transformed with the Hilbert weights of the
    imaginary axis (both branches), gives the HILBERT NONE weight -2D/(w^2+D^2)."""
    frqs = np.concatenate([[0.0], np.geomspace(1e-3, 60.0, 400)])
    omega = np.array([0.3, 2.0, 15.0])
    wr, wi = oracle.getwghtS(1j * omega, frqs, 0.0, 0, 0)
    for s0 in (120, 250, 330):
        D = frqs[s0]
        hat = 2.0 / (frqs[s0 + 1] - frqs[s0 - 1])
        w_eff = hat * wr[s0]
        exact = -2 * D / (omega ** 2 + D ** 2)
        assert np.allclose(w_eff, exact, rtol=2e-3, atol=0), (D, w_eff, exact)
        # the Hermitian part carries no imaginary weight on the imaginary axis
        assert np.abs(hat * wi[s0]).max() <= 1e-12 * np.abs(exact).max()


def test_hilbert_weights_threshold():
    rng = np.random.default_rng(0)
    wt = rng.uniform(0, 1, (50, 7)) * (rng.uniform(0, 1, (50, 7)) > 0.5)
    ws = rng.standard_normal((7, 3))
    a = oracle.hilbert_weights(wt, ws, thr=0.3, scale_all=0.5)
    b = 0.5 * np.where(wt > 0.3, wt, 0) @ ws
    assert np.allclose(a, b)


def test_realfreq_restatement_is_the_complex_weighted_gram():
    """The suscepc loop of the reference (two real sums per weight part, combined into
    (i,j) and (j,i)) equals sum_p M_i conj(M_j) (wr + i wi) for every i, j."""
    rng = np.random.default_rng(0)
    P, N, nw = 60, 9, 3
    m = rng.standard_normal((P, N)) + 1j * rng.standard_normal((P, N))
    wr, wi = rng.standard_normal((P, nw)), rng.standard_normal((P, nw))
    got = oracle.chi0_realfreq(m, wr, wi)
    direct = np.einsum("pi,pj,pf->ijf", m, np.conj(m), wr + 1j * wi)
    assert np.abs(got - direct).max() <= 1e-12 * np.abs(direct).max()


def test_real_restatement_matches_einsum():
    """The -DINV loop restated (real re(k) = cprod(k,i) cprod(k,j), :1197) is the real
    weighted Gram on the packed upper triangle."""
    rng = np.random.default_rng(3)
    m, w = rng.standard_normal((50, 6)), rng.standard_normal((50, 2))
    got = oracle.chi0_real(m, w)
    iu, ju = np.triu_indices(6)
    ref = np.einsum("pi,pj,pf->ijf", m, m, w)[iu, ju]
    assert np.abs(got[ju * (ju + 1) // 2 + iu] - ref).max() <= 1e-13
