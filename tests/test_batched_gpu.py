"""Many q points in one launch (K7): the persistent split schedule, the per-slab
kernel schedule, and the autotuners."""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle
import project1_b200 as spx
from project1_b200 import _lib, inputs
from project1_b200.susceptibility import SpexGpuError, npack
from chi0_util import normalized_error

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
SPLIT_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = spx.Context(0)
    yield c
    c.close()


def _q(nbas, npair, nw, seed, generated, variant=2, slab=32768):
    rng = np.random.default_rng(seed)
    ed = rng.uniform(0.5, 40.0, npair)
    ed[rng.choice(npair, max(1, npair // 100), replace=False)] = 2e-7
    q = dict(nbas=nbas, npair=npair, variant=variant, slab_pairs=slab,
             ediff=torch.from_numpy(ed).to(DEV), scale_all=0.25,
             susceph=torch.zeros((nw, npack(nbas)), dtype=torch.complex128, device=DEV))
    if generated:
        q.update(seed=1000 + seed, stream_id=3, m_scale=1.0 / np.sqrt(nbas))
    else:
        m = spx.gen_cmatrix_host(1000 + seed, 3, npair, nbas, scale=1.0 / np.sqrt(nbas))
        ldc = npair + 5
        cp = torch.zeros((nbas, ldc), dtype=torch.complex128, device=DEV)
        cp[:, :npair] = torch.from_numpy(np.ascontiguousarray(m.T)).to(DEV)
        q.update(cprod=cp)
    return q


SHAPES = [(40, 300), (129, 5000), (200, 40000), (1, 7), (257, 33000)]


def _per_q_reference(ctx, q, omega, precision):
    """The same q through the single-q entry point on an explicit M."""
    nbas, npair = q["nbas"], q["npair"]
    if "cprod" in q:
        cp = q["cprod"]
    else:
        cp = torch.empty((nbas, npair), dtype=torch.complex128, device=DEV)
        ctx.gen_cmatrix_dev(q["seed"], q["stream_id"], cp, npair, scale=q["m_scale"])
        ctx.synchronize()
    out = torch.zeros_like(q["susceph"])
    torch.cuda.synchronize()   # the context stream does not wait for torch's
    ctx.chi0_accumulate_dev(cp, q["ediff"], omega, out, scale_all=q["scale_all"],
                            precision=precision, npair=npair, stats=True)
    return out


@pytest.mark.parametrize("generated", [False, True])
@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_batched_equals_per_q_calls(ctx, generated, precision):
    omega = torch.from_numpy(inputs.frequencies(3)).to(DEV)
    qs = [_q(n, p, 3, i, generated) for i, (n, p) in enumerate(SHAPES)]
    st = ctx.chi0_batched(qs, omega, precision=precision, stats=True)
    if precision == "split":
        assert st["kernel_launches"] == 1       # one persistent kernel for the whole batch
    else:
        assert st["kernel_launches"] > len(qs)
    for q in qs:
        ref = _per_q_reference(ctx, q, omega, precision)
        assert torch.equal(q["susceph"], ref), (q["nbas"], q["npair"])


def test_batched_matches_oracle(ctx):
    omega_h = inputs.frequencies(2)
    omega = torch.from_numpy(omega_h).to(DEV)
    qs = [_q(n, p, 2, 7 + i, True) for i, (n, p) in enumerate([(70, 900), (33, 2000), (150, 400)])]
    ctx.chi0_batched(qs, omega, stats=True)
    for q in qs:
        m = spx.gen_cmatrix_host(q["seed"], q["stream_id"], q["npair"], q["nbas"], scale=q["m_scale"])
        ref = oracle.chi0(m, oracle.weights(q["ediff"].cpu().numpy(), omega_h, None, q["scale_all"]),
                          accurate=True)
        emax, fro = normalized_error(q["susceph"].cpu().numpy().T, ref, q["nbas"])
        assert emax <= SPLIT_TOL, (emax, fro)


def test_graph_replay_repeats_the_result(ctx):
    omega = torch.from_numpy(inputs.frequencies(3)).to(DEV)
    qs = [_q(n, p, 3, 20 + i, True) for i, (n, p) in enumerate([(96, 3000), (300, 70000)])]
    ctx.chi0_batched(qs, omega, stats=True)           # captures the graph
    first = [q["susceph"].clone() for q in qs]
    for q in qs:
        q["susceph"].zero_()
    st = ctx.chi0_batched(qs, omega, stats=True)      # replays it
    assert st["kernel_launches"] > 0
    for q, a in zip(qs, first):
        assert torch.equal(q["susceph"], a)
    # without a graph: the same bits again
    for q in qs:
        q["susceph"].zero_()
    ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_NOGRAPH, stats=True)
    for q, a in zip(qs, first):
        assert torch.equal(q["susceph"], a)


def test_variants_and_slabs_agree(ctx):
    """Every tuning choice computes the same chi within the split bound."""
    omega_h = inputs.frequencies(2)
    omega = torch.from_numpy(omega_h).to(DEV)
    outs = []
    for variant, slab in [(1, 16384), (2, 16384), (1, 32768), (2, 4096)]:
        q = _q(180, 50000, 2, 99, True, variant=variant, slab=slab)
        ctx.chi0_batched([q], omega, stats=True)
        outs.append(q["susceph"].cpu().numpy().T)
    m = spx.gen_cmatrix_host(1099, 3, 50000, 180, scale=1 / np.sqrt(180))
    ref = oracle.chi0(m, oracle.weights(q["ediff"].cpu().numpy(), omega_h, None, 0.25), accurate=True)
    for o in outs:
        emax, _ = normalized_error(o, ref, 180)
        assert emax <= SPLIT_TOL


def test_autotune_table_roundtrip(ctx, tmp_path):
    e = ctx.autotune_split(200, 40000, 3)
    assert e["variant"] in (1, 2, 3, 5) and e["slab_pairs"] in (8192, 12288, 16384, 32768) and e["tflops"] > 0
    assert ctx.tune_lookup(200, 40000, 3) == e
    assert ctx.tune_lookup(200, 40000, 4) is None
    path = tmp_path / "tune.json"
    ctx.tune_save(path)
    doc = json.loads(path.read_text())
    assert doc["format"] == "spexgpu-tune-1" and len(doc["entries"]) >= 1
    other = spx.Context(0)
    try:
        assert other.tune_lookup(200, 40000, 3) is None
        other.tune_load(path)
        got = other.tune_lookup(200, 40000, 3)
        assert got["variant"] == e["variant"] and got["slab_pairs"] == e["slab_pairs"]
        bad = tmp_path / "bad.json"
        bad.write_text('{"format": "spexgpu-tune-1", "entries": [{"nbas_bucket": 2, "variant": 9}]}')
        with pytest.raises(SpexGpuError):
            other.tune_load(bad)
    finally:
        other.close()


def test_autotuned_batch(ctx):
    omega = torch.from_numpy(inputs.frequencies(2)).to(DEV)
    qs = [_q(n, p, 2, 40 + i, True, variant=0, slab=0) for i, (n, p) in enumerate([(260, 20000), (520, 9000)])]
    ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_AUTOTUNE, stats=True)
    for q in qs:
        t = ctx.tune_lookup_batched(q["nbas"], q["npair"], 2)
        assert t is not None and t["variant"] == 4 and t["tile"] in (64 + 3 * 256, 80 + 3 * 256, 32 + 4 * 256)
        assert torch.isfinite(torch.view_as_real(q["susceph"])).all()
        assert q["susceph"].abs().max() > 0


def test_batched_rejects_bad_descriptors(ctx):
    omega = torch.from_numpy(inputs.frequencies(2)).to(DEV)
    q = _q(40, 100, 2, 1, False)
    with pytest.raises(SpexGpuError):
        ctx.chi0_batched([dict(q, variant=3)], omega)
    with pytest.raises(SpexGpuError):
        ctx.chi0_batched([dict(q, npair=200)], omega)       # ldc 105 < npair
    with pytest.raises(SpexGpuError):
        ctx.chi0_batched([dict(q, nbas=50000)], omega)


def _force_tile(c, tmp_path, qs, nw, tile, slab):
    """Loads a tuning table that assigns `tile` and `slab` to the buckets of `qs`."""
    ents = []
    for q in qs:
        n, p = q["nbas"], q["npair"]
        ents.append({"nbas_bucket": (n + 127) // 128, "npair_bucket": 0 if p <= 16384 else (1 if p <= 32768 else 2),
                     "nw": nw, "variant": 4, "slab_pairs": slab, "tile": tile, "tflops": 1.0})
    path = tmp_path / f"tile{tile}.json"
    path.write_text(json.dumps({"format": "spexgpu-tune-1", "entries": ents}))
    c.tune_load(path)


@pytest.mark.parametrize("tile", [64 + 3 * 256, 32 + 3 * 256, 32 + 4 * 256, 80 + 3 * 256])
def test_persistent_tile_shapes_equal_per_q_calls(tmp_path, tile):
    """Every tile shape of the persistent schedule gives the per-q result bit for bit,
    with the slab ring reused many times (4096-pair slabs, 4 buffers) and a q whose
    weights change sign (negative energy differences)."""
    omega = torch.from_numpy(inputs.frequencies(3)).to(DEV)
    with spx.Context(0) as c:
        qs = [_q(n, p, 3, 60 + i, gen, slab=0) for i, (n, p, gen) in
              enumerate([(130, 60000, True), (65, 9000, False), (200, 20000, True)])]
        qs[1]["ediff"][::7] *= -1.0
        _force_tile(c, tmp_path, qs, 3, tile, 4096)
        st = c.chi0_batched(qs, omega, stats=True)
        assert st["kernel_launches"] == 1
        for q in qs:
            ref = torch.zeros_like(q["susceph"])
            cp = q.get("cprod")
            if cp is None:
                cp = torch.empty((q["nbas"], q["npair"]), dtype=torch.complex128, device=DEV)
                c.gen_cmatrix_dev(q["seed"], q["stream_id"], cp, q["npair"], scale=q["m_scale"])
            c.synchronize()
            torch.cuda.synchronize()
            with spx.Context(0, split_variant=1) as c1:
                for p0 in range(0, q["npair"], 4096):
                    # slab by slab, as the persistent schedule cuts them
                    n = min(4096, q["npair"] - p0)
                    c1.chi0_accumulate_dev(cp[:, p0:p0 + n].contiguous(), q["ediff"][p0:p0 + n].contiguous(),
                                           omega, ref, scale_all=q["scale_all"], precision="split", stats=True)
            assert torch.equal(q["susceph"], ref), (tile, q["nbas"], q["npair"])


def test_persistent_and_kernel_schedules_agree(ctx):
    omega = torch.from_numpy(inputs.frequencies(2)).to(DEV)
    qs = [_q(n, p, 2, 80 + i, True) for i, (n, p) in enumerate([(90, 40000), (300, 5000)])]
    ctx.chi0_batched(qs, omega, stats=True)
    a = [q["susceph"].clone() for q in qs]
    for q in qs:
        q["susceph"].zero_()
    st = ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_KERNELS, stats=True)
    assert st["kernel_launches"] > 1
    for q, x in zip(qs, a):
        assert torch.equal(q["susceph"], x)


def test_persistent_role_profile():
    """The role counters count every accumulation item of the batch (tiles x
    frequencies x slabs, 64 x 80 tiles untuned) and each role's waits fit inside
    the CTAs' cycles."""
    omega = torch.from_numpy(inputs.frequencies(2)).to(DEV)
    with spx.Context(0) as c:
        qs = [_q(n, p, 2, 80 + i, gen, slab=8192) for i, (n, p, gen) in
              enumerate([(200, 20000, True), (96, 9000, False)])]
        c.pb_profile_enable(True)
        c.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_NOGRAPH)
        prof = c.pb_profile_read()
        c.pb_profile_enable(False)

    def ntile80(n):   # 64-row blocks x 80-column blocks of the upper triangle
        nbr = (n + 63) // 64
        return sum(min((j * 80 + 79) // 64, nbr - 1) + 1 for j in range((n + 79) // 80))
    items = sum(ntile80(q["nbas"]) * 2 * -(-q["npair"] // 8192) for q in qs)
    assert prof["accumulation_items"] == items
    assert prof["preparation_items"] > 0 and prof["cta"] > 0
    for k, v in prof.items():
        if not k.endswith("_items"):
            assert 0 <= v <= prof["cta"], k
