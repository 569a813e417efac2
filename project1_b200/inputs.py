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


# ---------------------------------------------------------------------------
# wave-function products workload: 2 atoms, lmax 8, 3 radial functions per l,
# seeded sparse Gaunt table (5 % of the valid entries), seeded radial integrals;
# 3000 plane waves per k damped by exp(-|G|^2/50); 1014 mixed-basis plane waves.

@dataclass
class WfprodWorkload:
    name: str
    natom: int = 2
    lcut: int = 8
    nrad: int = 3
    lcutm: int = 8
    nradm: int = 3
    ngpt: int = 3000
    ngptm: int = 1014
    nk: int = 27
    nocc: int = 40
    nunocc: int = 300
    nw: int = 24
    step_radius: int = 2
    vol: float = 1000.0
    gaunt_density: float = 0.05
    seed: int = SEED + 4

    @property
    def maxlm(self) -> int:
        return (self.lcut + 1) ** 2 * self.nrad

    @property
    def maxllm(self) -> int:
        return (self.lcutm + 1) ** 2 * self.nradm

    @property
    def nbasp(self) -> int:
        return self.natom * self.maxllm

    @property
    def nbas(self) -> int:
        return self.nbasp + self.ngptm

    @property
    def npair(self) -> int:
        return self.nk * self.nocc * self.nunocc

    @property
    def flops(self) -> float:
        return 8.0 * self.nbas ** 2 * self.npair * self.nw


WFPROD_CONFIGS = {"c4": WfprodWorkload("c4")}


def mt_basis(w: WfprodWorkload) -> dict:
    rng = np.random.default_rng([w.seed, 1])
    L, Lm = w.lcut, w.lcutm
    g = np.zeros((L + 1, L + 1, Lm + 1, 2 * L + 1, 2 * Lm + 1), order="F")
    for LL in range(Lm + 1):
        for MM in range(-LL, LL + 1):
            for l in range(L + 1):
                for m in range(-l, l + 1):
                    for l1 in range(abs(l - LL), min(l + LL, L) + 1, 2):
                        if abs(m + MM) <= l1 and rng.random() < w.gaunt_density:
                            g[l1, l, LL, m + L, MM + Lm] = rng.standard_normal() * 0.3
    nln = (L + 1) * w.nrad
    integral = np.asfortranarray(rng.standard_normal((nln, nln, (Lm + 1) * w.nradm)) * 0.2)
    phase = rng.uniform(0, 1, w.natom)
    cexp = np.exp(-2j * np.pi * phase)
    return dict(natom=w.natom, lcut=L, nrad=w.nrad, lcutm=Lm, nradm=w.nradm, gaunt=g,
                integral=integral, cexp=cexp)


def _sphere(n: int) -> np.ndarray:
    r = int(np.ceil((3 * n / (4 * np.pi)) ** (1 / 3))) + 2
    ax = np.arange(-r, r + 1)
    G = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    order = np.lexsort((G[:, 2], G[:, 1], G[:, 0], (G ** 2).sum(1)))
    return np.ascontiguousarray(G[order[:n]].astype(np.int32))


def pw_basis(w: WfprodWorkload) -> dict:
    rng = np.random.default_rng([w.seed, 2])
    sr = w.step_radius
    ns = 2 * sr + 1
    cs = np.zeros((ns, ns, ns), complex)
    for d0 in range(-sr, sr + 1):
        for d1 in range(-sr, sr + 1):
            for d2 in range(-sr, sr + 1):
                if (d0, d1, d2) < (0, 0, 0):
                    continue
                v = 0.8 if (d0, d1, d2) == (0, 0, 0) else 0.05 * (rng.standard_normal() + 1j * rng.standard_normal())
                cs[d0 + sr, d1 + sr, d2 + sr] = v
                cs[-d0 + sr, -d1 + sr, -d2 + sr] = np.conj(v)  # real step function
    cs[sr, sr, sr] = 0.8
    g = _sphere(w.ngpt)
    return dict(gpt1=g, gpt2=g.copy(), gptm=_sphere(w.ngptm), gshift=np.zeros(3, np.int32),
                step_radius=sr, cstep=np.asfortranarray(cs).reshape(-1, order="F"), vol=w.vol)


def mt_coeffs(w: WfprodWorkload):
    """cmt_occ (nk, nocc, natom, maxlm) and cmt_unocc (nk, nunocc, natom, maxlm), C order."""
    rng = np.random.default_rng([w.seed, 3])
    sh1 = (w.nk, w.nocc, w.natom, w.maxlm)
    sh2 = (w.nk, w.nunocc, w.natom, w.maxlm)
    c1 = rng.standard_normal(sh1) + 1j * rng.standard_normal(sh1)
    c2 = rng.standard_normal(sh2) + 1j * rng.standard_normal(sh2)
    return c1, c2


def pw_coeffs(w: WfprodWorkload, pw: dict):
    """cpw_occ (nk, nocc, ngpt1) and cpw_unocc (nk, nunocc, ngpt2), damped exp(-|G|^2/50)."""
    rng = np.random.default_rng([w.seed, 5])
    n1, n2 = pw["gpt1"].shape[0], pw["gpt2"].shape[0]
    d1 = np.exp(-(pw["gpt1"].astype(float) ** 2).sum(1) / 50.0)
    d2 = np.exp(-(pw["gpt2"].astype(float) ** 2).sum(1) / 50.0)
    c1 = (rng.standard_normal((w.nk, w.nocc, n1)) + 1j * rng.standard_normal((w.nk, w.nocc, n1))) * d1
    c2 = (rng.standard_normal((w.nk, w.nunocc, n2)) + 1j * rng.standard_normal((w.nk, w.nunocc, n2))) * d2
    return c1, c2


# ---------------------------------------------------------------------------
# batched uneven q-point workload: 32 q with N_MB ~ U{600..1800}, band windows
# occ ~ U{20..60} x unocc ~ U{150..500}, 64 k points, 24 frequencies, M generated
# per q from its own Philox stream.

@dataclass
class BatchedWorkload:
    name: str
    nq: int = 32
    nk: int = 64
    nw: int = 24
    nbas_range: tuple = (600, 1800)
    occ_range: tuple = (20, 60)
    unocc_range: tuple = (150, 500)
    seed: int = SEED + 3


BATCHED_CONFIGS = {"c3": BatchedWorkload("c3")}


def batched_qs(w: BatchedWorkload) -> list:
    """The per-q workloads, drawn once from the batch seed (inclusive ranges)."""
    rng = np.random.default_rng([w.seed, 31])
    out = []
    for q in range(w.nq):
        nbas = int(rng.integers(w.nbas_range[0], w.nbas_range[1] + 1))
        nocc = int(rng.integers(w.occ_range[0], w.occ_range[1] + 1))
        nunocc = int(rng.integers(w.unocc_range[0], w.unocc_range[1] + 1))
        out.append(Chi0Workload(f"{w.name}q{q}", nbas, w.nk, nocc, nunocc, w.nw,
                                seed=w.seed * 1000 + q, stream_id=1))
    return out
