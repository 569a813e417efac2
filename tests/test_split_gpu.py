"""Split-precision (int8 digit slices on tcgen05) accumulation against the FP64 oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import inputs
from chi0_util import normalized_error
from test_chi0_gpu import DEV, G, random_case, run_dev

pytestmark = pytest.mark.gpu
SPLIT_TOL = 1e-6       # per-element error / sqrt(|chi_ii chi_jj|), split path
# Frobenius relative error, split path: the same bound. Three digits of both folded
# operands round at 2^-17/127 of the column scale and the dropped digit orders are of
# that size, so small or ragged slabs (crest factor near sqrt(P)) land at 1e-7..5e-7.
SPLIT_FRO = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted({k.split("/")[0] for k in G.files if "/" in k}))
def test_split_matches_golden(ctx, name):
    m, d, om = G[f"{name}/cprod"], G[f"{name}/ediff"], G[f"{name}/omega"]
    ws = G[f"{name}/wscale"] if f"{name}/wscale" in G.files else None
    ref = G[f"{name}/susceph"]
    got = run_dev(ctx, np.asfortranarray(m), d, om, ws, float(G["scale_all"]), precision="split")
    emax, fro = normalized_error(got, ref, m.shape[1])
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


@pytest.mark.parametrize("nbas,npair,nw,degfrac", [
    (1, 1, 1, 0.0), (7, 5, 3, 0.0), (64, 32, 1, 0.0), (65, 33, 2, 0.1), (130, 100, 3, 0.01),
    (200, 5000, 3, 0.01), (257, 64, 1, 0.0)])
def test_split_matches_oracle_shapes(ctx, nbas, npair, nw, degfrac):
    m, d, om = random_case(nbas, npair, nw, seed=7 * nbas + npair, degfrac=degfrac)
    ref = oracle.chi0(m, oracle.weights(d, om), accurate=True)
    got = run_dev(ctx, m, d, om, precision="split")
    emax, fro = normalized_error(got, ref, nbas)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


def test_split_several_slabs(ctx):
    """P above one exact int32 slab (32768 pairs): slabs are reduced in FP64."""
    m, d, om = random_case(80, 70000, 2, seed=3, degfrac=0.01)
    ref = oracle.chi0(m, oracle.weights(d, om, None, 1 / 64), accurate=True)
    got = run_dev(ctx, m, d, om, None, 1 / 64, precision="split")
    emax, fro = normalized_error(got, ref, 80)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


def test_split_c0_full_config(ctx):
    w = inputs.CONFIGS["c0"]
    m = inputs.cprod_host(w)
    d = inputs.pair_ediff(w)
    om = inputs.frequencies(w.nw)
    ref = oracle.chi0(m, oracle.weights(d, om, None, 1.0 / w.nk), accurate=True)
    got = run_dev(ctx, m, d, om, None, 1.0 / w.nk, precision="split")
    emax, fro = normalized_error(got, ref, w.nbas)
    print(f"c0 split: max normalised {emax:.3e}, Frobenius {fro:.3e}")
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


def test_split_degenerate_pairs_keep_fp64_weights(ctx):
    """Pairs with |e_n'-e_n| < 1e-6 eV carry weights ~1e-5 of the rest; they must still count."""
    rng = np.random.default_rng(4)
    nbas, npair = 48, 400
    m = np.asfortranarray((rng.standard_normal((npair, nbas)) + 1j * rng.standard_normal((npair, nbas))) / 7)
    d = rng.uniform(0, 1e-6, npair)          # every pair degenerate
    om = inputs.frequencies(3)
    ref = oracle.chi0(m, oracle.weights(d, om), accurate=True)
    got = run_dev(ctx, m, d, om, precision="split")
    emax, fro = normalized_error(got, ref, nbas)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


def test_split_host_path(ctx):
    m, d, om = random_case(96, 1000, 3, seed=11)
    ref = oracle.chi0(m, oracle.weights(d, om, None, 0.25), accurate=True)
    with spx.Context(0, chunk_pairs=320) as c:
        out = np.zeros((96 * 97 // 2, 3), complex, order="F")
        c.chi0_accumulate(m, d, om, out, scale_all=0.25, precision="split")
    emax, fro = normalized_error(out, ref, 96)
    assert emax <= SPLIT_TOL, emax


def test_split_accumulates(ctx):
    m, d, om = random_case(40, 50, 2, seed=5)
    init = np.asfortranarray(np.random.default_rng(3).standard_normal((40 * 41 // 2, 2)) * 1e-3 + 0j)
    ref = oracle.chi0(m, oracle.weights(d, om), accurate=True, susceph=init.copy(order="F"))
    got = run_dev(ctx, m, d, om, init=init, precision="split")
    assert np.max(np.abs(got - ref)) <= 1e-6 * np.max(np.abs(ref))


@pytest.mark.parametrize("nbas,npair,nw", [(65, 3000, 2), (200, 40000, 3), (130, 33, 1),
                                           (1200, 700, 2), (81, 5000, 1), (239, 2500, 2)])
def test_split_cta_pair_equals_single_cta(nbas, npair, nw):
    """The CTA-pair kernel (cta_group::2), the one-CTA kernel on 64 x 64 tiles and the
    one on 64 x 80 tiles (N = 160 MMAs) sum the same exact integers and add one FP64
    term per element per launch: results are identical (ragged 80-column blocks
    included)."""
    m, d, om = random_case(nbas, npair, nw, seed=nbas + 3 * npair, degfrac=0.01)
    outs = []
    for variant in (1, 2, 5):
        with spx.Context(0, split_variant=variant) as c:
            outs.append(run_dev(c, m, d, om, None, 0.5, precision="split"))
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])
    ref = oracle.chi0(m, oracle.weights(d, om, None, 0.5), accurate=True)
    emax, fro = normalized_error(outs[1], ref, nbas)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)


@pytest.mark.parametrize("nbas,npair,nw", [(65, 3000, 2), (200, 40000, 3)])
def test_split_persistent_single_call_equals_slab_kernels(nbas, npair, nw):
    """Variant 3 (one persistent kernel with its own preparation warps) adds the same
    slab sums in the same order as the slab kernels (32768-pair slabs for both): the
    results are identical."""
    m, d, om = random_case(nbas, npair, nw, seed=nbas * 5 + npair, degfrac=0.01)
    outs = []
    for variant in (1, 3):
        with spx.Context(0, split_variant=variant) as c:
            outs.append(run_dev(c, m, d, om, None, 0.5, precision="split"))
    ref = oracle.chi0(m, oracle.weights(d, om, None, 0.5), accurate=True)
    emax, fro = normalized_error(outs[1], ref, nbas)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)
    assert np.array_equal(outs[0], outs[1])


def test_split_host_ramp_equals_device_path(ctx):
    """With default chunking, the host-pointer call streams growing chunks whose
    boundaries fall on the exact slabs (32768 pairs untuned) of the split path, and it
    keeps one kernel for all chunks, so its result equals the device call's bit for
    bit (pinned source)."""
    nbas, npair = 72, 150000
    m, d, om = random_case(nbas, npair, 2, seed=21, degfrac=0.01)
    dev = run_dev(ctx, m, d, om, None, 0.5, precision="split")
    t = torch.from_numpy(np.ascontiguousarray(m.T)).pin_memory()
    out = np.zeros((nbas * (nbas + 1) // 2, 2), complex, order="F")
    with spx.Context(0) as c:
        st = c.chi0_accumulate_host_ptr(t.data_ptr(), npair, npair, nbas, d, om, out,
                                        scale_all=0.5, precision="split")
    assert st["h2d_bytes"] >= m.nbytes
    assert np.array_equal(out, dev)


@pytest.mark.parametrize("variant,slab", [(5, 8192), (5, 12288), (1, 16384), (3, 8192)])
def test_split_host_ramp_equals_device_path_tuned(tmp_path, variant, slab):
    """With a tuning entry (kernel and slab) for the array's shape, the host-pointer
    call cuts its chunks on that slab and runs that kernel for every chunk, so it
    still equals the device call bit for bit."""
    import json
    nbas, npair, nw = 72, 150000, 2
    m, d, om = random_case(nbas, npair, nw, seed=22, degfrac=0.01)
    table = tmp_path / "tune.json"
    table.write_text(json.dumps({"format": "spexgpu-tune-1", "entries": [
        {"nbas_bucket": 1, "npair_bucket": 2, "nw": nw, "variant": variant, "slab_pairs": slab,
         "tile": 64 + 3 * 256 if variant == 3 else 0, "tflops": 1.0}]}))
    with spx.Context(0) as c:
        c.tune_load(str(table))
        dev = run_dev(c, m, d, om, None, 0.5, precision="split")
        t = torch.from_numpy(np.ascontiguousarray(m.T)).pin_memory()
        out = np.zeros((nbas * (nbas + 1) // 2, nw), complex, order="F")
        c.chi0_accumulate_host_ptr(t.data_ptr(), npair, npair, nbas, d, om, out,
                                   scale_all=0.5, precision="split")
    assert np.array_equal(out, dev)


@pytest.mark.parametrize("variant", [5, 1])
def test_split_tuned_slab_below_one_slab_of_pairs(tmp_path, variant):
    """A tuned 8192-pair slab on 16000 pairs takes two buffers of 8192 pairs, more
    than one buffer of the 16000 pairs the untuned call needs: the call sizes its
    scratch for the slab it runs."""
    import json
    nbas, npair, nw = 100, 16000, 2
    m, d, om = random_case(nbas, npair, nw, seed=23, degfrac=0.01)
    table = tmp_path / "tune.json"
    table.write_text(json.dumps({"format": "spexgpu-tune-1", "entries": [
        {"nbas_bucket": 1, "npair_bucket": 0, "nw": nw, "variant": variant, "slab_pairs": 8192,
         "tile": 0, "tflops": 1.0}]}))
    ref = oracle.chi0(m, oracle.weights(d, om, None, 0.5), accurate=True)
    with spx.Context(0) as c:
        c.tune_load(str(table))
        got = run_dev(c, m, d, om, None, 0.5, precision="split")
    emax, fro = normalized_error(got, ref, nbas)
    assert emax <= SPLIT_TOL and fro <= SPLIT_FRO, (emax, fro)
