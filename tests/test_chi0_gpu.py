"""FP64 band-pair accumulation on the GPU against the CPU oracle (parity tests)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import inputs
from project1_b200._lib import SPX_EINVAL, SpexGpuError
from chi0_util import normalized_error

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
FP64_TOL = 1e-10          # per-element normalised error, FP64 path
G = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "chi0_golden.npz")


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def to_dev_cprod(m):
    """Fortran (npair, nbas) -> torch (nbas, npair) contiguous == same memory order."""
    return torch.from_numpy(np.ascontiguousarray(m.T)).to(DEV)


def run_dev(ctx, m, d, om, ws=None, scale_all=1.0, precision="fp64", init=None):
    npair, nbas = m.shape
    nw = om.shape[0]
    out = torch.zeros((nw, nbas * (nbas + 1) // 2), dtype=torch.complex128, device=DEV)
    if init is not None:
        out.copy_(torch.from_numpy(np.ascontiguousarray(init.T)))
    ctx.chi0_accumulate_dev(to_dev_cprod(m), torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV), out,
                            wscale=None if ws is None else torch.from_numpy(ws).to(DEV),
                            scale_all=scale_all, precision=precision, stats=True)
    return out.cpu().numpy().T


def random_case(nbas, npair, nw, seed=0, degfrac=0.0):
    rng = np.random.default_rng(seed)
    m = np.asfortranarray((rng.standard_normal((npair, nbas)) + 1j * rng.standard_normal((npair, nbas)))
                          / np.sqrt(nbas))
    d = rng.uniform(0.5, 50.0, npair)
    if degfrac:
        sel = rng.choice(npair, max(1, int(degfrac * npair)), replace=False)
        d[sel] = rng.uniform(0, 1e-6, sel.size)
    return m, d, inputs.frequencies(nw)


def test_device_generator_matches_host(ctx):
    rows, cols = 1001, 7
    host = spx.gen_cmatrix_host(99, 2, rows, cols, col0=3, scale=0.25)
    dev = torch.empty((cols, rows + 5), dtype=torch.complex128, device=DEV)
    ctx.gen_cmatrix_dev(99, 2, dev, rows, col0=3, scale=0.25)
    assert np.array_equal(dev[:, :rows].cpu().numpy().T, host)


def test_weights_kernel_matches_oracle(ctx):
    m, d, om = random_case(4, 3001, 7, degfrac=0.05)
    ws = np.random.default_rng(1).uniform(0.5, 2, d.size)
    w = torch.empty((om.size, d.size), dtype=torch.float64, device=DEV)
    ctx.weights_dev(torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV), w,
                    wscale=torch.from_numpy(ws).to(DEV), scale_all=0.5)
    ref = oracle.weights(d, om, ws, 0.5)
    np.testing.assert_allclose(w.cpu().numpy().T, ref, rtol=1e-15, atol=0)


@pytest.mark.parametrize("name", sorted({k.split("/")[0] for k in G.files if "/" in k}))
def test_fp64_matches_golden(ctx, name):
    m, d, om = G[f"{name}/cprod"], G[f"{name}/ediff"], G[f"{name}/omega"]
    ws = G[f"{name}/wscale"] if f"{name}/wscale" in G.files else None
    ref = G[f"{name}/susceph"]
    got = run_dev(ctx, np.asfortranarray(m), d, om, ws, float(G["scale_all"]))
    emax, fro = normalized_error(got, ref, m.shape[1])
    assert emax <= FP64_TOL and fro <= 1e-12, (emax, fro)


@pytest.mark.parametrize("nbas,npair,nw", [
    (1, 1, 1), (7, 5, 3), (64, 16, 1), (65, 33, 2), (128, 17, 2), (130, 100, 3), (200, 1000, 5),
    (257, 64, 1)])
def test_fp64_matches_oracle_shapes(ctx, nbas, npair, nw):
    m, d, om = random_case(nbas, npair, nw, seed=nbas * 1000 + npair)
    ref = oracle.chi0(m, oracle.weights(d, om))
    got = run_dev(ctx, m, d, om)
    emax, fro = normalized_error(got, ref, nbas)
    assert emax <= FP64_TOL and fro <= 1e-12, (emax, fro)


def test_fp64_accumulates_into_existing_output(ctx):
    m, d, om = random_case(40, 50, 2, seed=5)
    init = np.asfortranarray(np.random.default_rng(3).standard_normal((40 * 41 // 2, 2)) + 0j)
    ref = oracle.chi0(m, oracle.weights(d, om), susceph=init.copy(order="F"))
    got = run_dev(ctx, m, d, om, init=init)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_fp64_c0_full_config(ctx):
    """c0: N_MB=400, 8 k, 20x80 bands, 12 frequencies, against the faithful loop."""
    w = inputs.CONFIGS["c0"]
    m = inputs.cprod_host(w)
    d = inputs.pair_ediff(w)
    om = inputs.frequencies(w.nw)
    ref = oracle.chi0(m, oracle.weights(d, om, None, 1.0 / w.nk))
    got = run_dev(ctx, m, d, om, None, 1.0 / w.nk)
    emax, fro = normalized_error(got, ref, w.nbas)
    assert emax <= FP64_TOL and fro <= 1e-12, (emax, fro)


@pytest.mark.parametrize("pinned", [False, True])
def test_host_path_streams_slabs(pinned):
    """Host-pointer drop-in with several streamed slabs equals the one-shot device result."""
    m, d, om = random_case(96, 1000, 3, seed=11)
    ref = oracle.chi0(m, oracle.weights(d, om, None, 0.25))
    with spx.Context(0, chunk_pairs=160) as c:
        out = np.zeros((96 * 97 // 2, 3), complex, order="F")
        if pinned:
            t = torch.from_numpy(np.ascontiguousarray(m.T)).pin_memory()
            st = c.chi0_accumulate_host_ptr(t.data_ptr(), 1000, 1000, 96, d, om, out, scale_all=0.25)
        else:
            st = c.chi0_accumulate(m, d, om, out, scale_all=0.25)
    assert st["h2d_bytes"] >= m.nbytes
    emax, fro = normalized_error(out, ref, 96)
    assert emax <= FP64_TOL, emax


def test_leading_dimension_padding(ctx):
    m, d, om = random_case(33, 40, 2, seed=2)
    big = np.zeros((48, 33), complex, order="F")
    big[:40] = m
    ref = oracle.chi0(m, oracle.weights(d, om))
    out = torch.zeros((2, 33 * 34 // 2), dtype=torch.complex128, device=DEV)
    ctx.chi0_accumulate_dev(to_dev_cprod(big), torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV),
                            out, npair=40)
    emax, _ = normalized_error(out.cpu().numpy().T, ref, 33)
    assert emax <= FP64_TOL


def test_susceptibility_mirror_spin_factor_and_packets(ctx):
    m, d, om = random_case(20, 60, 2, seed=8)
    frqh = 1j * om
    a = spx.susceptibility(ctx, m, d, frqh, nkpt=4)
    b = spx.susceptibility(ctx, m, d, frqh, nkpt=4, packets=[(0, 7), (7, 33), (33, 60)])
    ref = 2.0 * oracle.chi0(m, oracle.weights(d, om, None, 0.25))
    assert np.max(np.abs(a - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.max(np.abs(b - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_bad_arguments_raise(ctx):
    m, d, om = random_case(8, 10, 1)
    out = torch.zeros((1, 36), dtype=torch.complex128, device=DEV)
    with pytest.raises(SpexGpuError) as e:
        ctx.chi0_accumulate_dev(to_dev_cprod(m), torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV),
                                out, npair=11)
    assert e.value.status == SPX_EINVAL


def test_bounded_wait_reports_timeout_and_context_survives():
    """A device wait on a barrier phase that nothing completes runs out after its limit,
    is reported as SPX_ETIMEOUT with a message, and the context keeps working."""
    import time
    from project1_b200 import _lib
    with spx.Context(0) as c:
        t0 = time.perf_counter()
        rc = c.lib.spx_selftest_wait_dev(c.handle, 200)
        dt = time.perf_counter() - t0
        assert rc == _lib.SPX_ETIMEOUT
        assert "time limit" in c.lib.spx_last_error(c.handle).decode()
        assert 0.15 < dt < 5.0
        # the status word was cleared: ordinary work runs and is correct
        m, d, om = random_case(40, 200, 2, seed=1)
        ref = oracle.chi0(m, oracle.weights(d, om))
        out = np.zeros((40 * 41 // 2, 2), complex, order="F")
        c.chi0_accumulate(m, d, om, out)
        emax, _ = normalized_error(out, ref, 40)
        assert emax <= FP64_TOL


def test_measured_dmma_peak_is_plausible():
    """The FP64 tensor peak the bench divides by: B200's DMMA path is rated about
    40 TFLOP/s, so the measured value must lie in a plausible band."""
    with spx.Context(0) as c:
        v = c.measure_dmma_peak()
    print(f"measured DMMA peak: {v:.1f} TFLOP/s")
    assert 10.0 < v < 120.0, v


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("split", 1e-6)])
@pytest.mark.parametrize("nbas,npair,nw,ldpad", [(1, 3, 1, 0), (130, 5001, 3, 1), (257, 40000, 2, 0), (64, 64, 2, 3)])
def test_real_variant_matches_oracle(precision, tol, nbas, npair, nw, ldpad):
    """The -DINV build: real cprod (odd leading dimensions included), real packed chi."""
    rng = np.random.default_rng(nbas + npair)
    m = rng.standard_normal((npair, nbas)) / np.sqrt(nbas)
    d = rng.uniform(0.5, 40.0, npair)
    d[rng.choice(npair, max(1, npair // 100), replace=False)] = 3e-7
    om = inputs.frequencies(nw)
    w = oracle.weights(d, om, None, 0.5)
    ref = oracle.chi0_real(m, w)
    ldc = npair + ldpad
    cp = torch.zeros((nbas, ldc), dtype=torch.float64, device=DEV)
    cp[:, :npair] = torch.from_numpy(np.ascontiguousarray(m.T)).to(DEV)
    out = torch.zeros((nw, nbas * (nbas + 1) // 2), dtype=torch.float64, device=DEV)
    with spx.Context(0) as c:
        st = c.chi0_accumulate_real_dev(cp, torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV), out,
                                        scale_all=0.5, precision=precision, npair=npair, stats=True)
    assert st["kernel_launches"] >= 2
    got = out.cpu().numpy().T
    j = np.arange(nbas)
    dg = np.abs(ref[j * (j + 1) // 2 + j])
    iu, ju = np.triu_indices(nbas)
    idx = ju * (ju + 1) // 2 + iu
    err = np.abs(got[idx] - ref[idx]) / np.sqrt(dg[iu] * dg[ju])
    assert err.max() <= tol, err.max()


@pytest.mark.parametrize("nbas,npair", [(300, 9000), (161, 5000), (1200, 700)])
def test_real_wide_tiles_equal_square_tiles(nbas, npair):
    """The -DINV split path on 128 x 160 real tiles (N = 160 MMAs, the default) and on
    128 x 128 tiles (split variant 1) sums the same exact integers per element and
    slab: identical results, ragged column blocks included."""
    rng = np.random.default_rng(nbas * 7 + npair)
    m = rng.standard_normal((npair, nbas)) / np.sqrt(nbas)
    d = rng.uniform(0.5, 40.0, npair)
    om = inputs.frequencies(2)
    cp = torch.from_numpy(np.ascontiguousarray(m.T)).to(DEV)
    outs = []
    for variant in (0, 1):
        out = torch.zeros((2, nbas * (nbas + 1) // 2), dtype=torch.float64, device=DEV)
        with spx.Context(0, split_variant=variant) as c:
            c.chi0_accumulate_real_dev(cp, torch.from_numpy(d).to(DEV), torch.from_numpy(om).to(DEV), out,
                                       scale_all=0.5, precision="split", npair=npair)
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
