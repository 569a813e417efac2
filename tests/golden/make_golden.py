"""Generates tests/golden/chi0_golden.npz: small HILBERT NONE polarisation cases
computed with an independent numpy formulation of the reference formulas

  w(p,f)   = -2 d_p / (omega_f^2 + d_p^2) * nkpts(k)/nkpt/nsym1   src/susceptibility.f:965
  chi(i,j) = sum_p cprod(p,i) conj(cprod(p,j)) w(p,f), i <= j      :1195-1230 + :1782-1783
  packed ij = j*(j+1)/2 + i (0-based)                             :1210

It does not use the C oracle, so it checks that restatement against a second,
independent one. Run: python tests/golden/make_golden.py
"""
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "chi0_golden.npz"

CASES = [
    # name, nbas, npair, nw, degenerate fraction, per-pair scale
    ("single_pair", 3, 1, 1, 0.0, False),
    ("tiny", 5, 7, 2, 0.0, False),
    ("ragged", 33, 17, 3, 0.0, True),
    ("small_degenerate", 24, 60, 4, 0.1, True),
]


def make_case(seed, nbas, npair, nw, degfrac, pscale):
    rng = np.random.default_rng(seed)
    m = (rng.standard_normal((npair, nbas)) + 1j * rng.standard_normal((npair, nbas))) / np.sqrt(nbas)
    d = rng.uniform(0.5, 50.0, npair)
    if degfrac > 0:
        sel = rng.choice(npair, size=max(1, int(degfrac * npair)), replace=False)
        d[sel] = rng.uniform(0.0, 1e-6, sel.size)
    x, _ = np.polynomial.legendre.leggauss(nw)
    omega = 50.0 * (x + 1.0)
    wscale = rng.uniform(0.5, 2.0, npair) if pscale else None
    s = (wscale if pscale else np.ones(npair)) * 0.125
    w = -2.0 * d[:, None] / (omega[None, :] ** 2 + d[:, None] ** 2) * s[:, None]
    full = np.einsum("pi,pj,pf->fij", m, np.conj(m), w)
    iu, ju = np.triu_indices(nbas)
    packed = np.stack([full[f][iu, ju] for f in range(nw)], axis=1)   # (npack, nw)
    order = np.argsort(ju * (ju + 1) // 2 + iu)
    packed = packed[order]
    return m, d, omega, wscale, w, packed


def main():
    arrays = {}
    for k, (name, nbas, npair, nw, degfrac, pscale) in enumerate(CASES):
        m, d, omega, wscale, w, packed = make_case(1000 + k, nbas, npair, nw, degfrac, pscale)
        arrays[f"{name}/cprod"] = m
        arrays[f"{name}/ediff"] = d
        arrays[f"{name}/omega"] = omega
        if wscale is not None:
            arrays[f"{name}/wscale"] = wscale
        arrays[f"{name}/w"] = w
        arrays[f"{name}/susceph"] = packed
    arrays["scale_all"] = np.array(0.125)
    np.savez_compressed(OUT, **arrays)
    print(OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
