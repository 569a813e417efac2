"""Seeded synthetic inputs for the polarisation workloads.

The reference computes cprod from DFT wave functions; no public dataset is
involved. The workloads use seeded stand-ins with the stated shapes and
distributions:
  * M_I,p = (N(0,1) + i N(0,1)) / sqrt(N_MB), from the library's Philox4x32-10
    stream (identical bits on host and device);
  * occupied energies U[-10, 0] eV, unoccupied U[0.5, 40] eV, sorted per k;
  * frequencies: Gauss-Legendre nodes on [-1, 1] mapped linearly to [0, 100] eV;
  * pair weights nkpts(k)/nkpt/nsym1 = 1/nk;
  * optionally a fraction of near-degenerate pairs with |e_n' - e_n| < 1e-6 eV.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

SEED = 20261203


@dataclass
class Chi0Workload:
    name: str
    nbas: int          # N_MB
    nk: int            # k points
    nocc: int          # occupied bands
    nunocc: int        # unoccupied bands
    nw: int            # imaginary frequencies
    degenerate_frac: float = 0.0
    seed: int = SEED
    stream_id: int = 1

    @property
    def npair(self) -> int:
        return self.nk * self.nocc * self.nunocc

    @property
    def flops(self) -> float:
        """Algorithmic real flops of the full complex Gram, 8 N^2 P Nw."""
        return 8.0 * self.nbas ** 2 * self.npair * self.nw

    @property
    def flops_hermitian(self) -> float:
        """Flops of the upper triangle only, 4 N (N+1) P Nw."""
        return 4.0 * self.nbas * (self.nbas + 1) * self.npair * self.nw

    @property
    def m_scale(self) -> float:
        return 1.0 / np.sqrt(self.nbas)


CONFIGS = {
    # plain FP64, small (CPU-runnable reference routine)
    "c0": Chi0Workload("c0", nbas=400, nk=8, nocc=20, nunocc=80, nw=12),
    # plain FP64 GPU drop-in timing anchor
    "c1": Chi0Workload("c1", nbas=1200, nk=64, nocc=40, nunocc=400, nw=24),
    # split precision, c1 shape, 1% degenerate pairs
    "c2": Chi0Workload("c2", nbas=1200, nk=64, nocc=40, nunocc=400, nw=24, degenerate_frac=0.01),
}


def frequencies(nw: int, lo: float = 0.0, hi: float = 100.0) -> np.ndarray:
    """Gauss-Legendre nodes on [-1, 1] mapped linearly to [lo, hi] (imaginary-axis magnitudes)."""
    x, _ = np.polynomial.legendre.leggauss(nw)
    return (lo + (x + 1.0) * 0.5 * (hi - lo)).astype(np.float64)


def energies(w: Chi0Workload):
    """(e_occ (nk, nocc), e_unocc (nk, nunocc)) sorted per k point."""
    rng = np.random.default_rng([w.seed, 7])
    e_occ = np.sort(rng.uniform(-10.0, 0.0, size=(w.nk, w.nocc)), axis=1)
    e_unocc = np.sort(rng.uniform(0.5, 40.0, size=(w.nk, w.nunocc)), axis=1)
    return e_occ, e_unocc


def pair_ediff(w: Chi0Workload) -> np.ndarray:
    """ediff[p] = e_n'(k+q) - e_n(k) with p = n' + nu*(n + no*k); degenerate pairs injected."""
    e_occ, e_unocc = energies(w)
    d = (e_unocc[:, None, :] - e_occ[:, :, None]).reshape(-1)  # k outer, n, then n' fastest
    if w.degenerate_frac > 0:
        rng = np.random.default_rng([w.seed, 11])
        ndeg = int(round(w.degenerate_frac * d.size))
        sel = rng.choice(d.size, size=ndeg, replace=False)
        d[sel] = rng.uniform(0.0, 1e-6, size=ndeg)
    return d.astype(np.float64)


def cprod_host(w: Chi0Workload, col0: int = 0, ncol: Optional[int] = None) -> np.ndarray:
    """Columns [col0, col0+ncol) of M as a Fortran (npair, ncol) complex128 array."""
    from .susceptibility import gen_cmatrix_host
    ncol = w.nbas - col0 if ncol is None else ncol
    return gen_cmatrix_host(w.seed, w.stream_id, w.npair, ncol, col0=col0, scale=w.m_scale)


def small(name: str, nbas: int, nk: int, nocc: int, nunocc: int, nw: int,
          degenerate_frac: float = 0.0, seed: int = SEED) -> Chi0Workload:
    return Chi0Workload(name, nbas, nk, nocc, nunocc, nw, degenerate_frac, seed)
