"""Shared helpers for the polarisation parity tests."""
import numpy as np


def diag_index(n):
    j = np.arange(n)
    return j * (j + 1) // 2 + j


def normalized_error(got, ref, nbas):
    """max over (i<=j, f) of |got-ref| / sqrt(|ref_ii ref_jj|), and the Frobenius relative error.

    With single-sign weights chi(iw) is negative semi-definite, so |chi_ij| <= sqrt(chi_ii chi_jj);
    this is the per-element scale of every entry.
    """
    got = np.asarray(got)
    ref = np.asarray(ref)
    iu, ju = np.triu_indices(nbas)
    idx = ju * (ju + 1) // 2 + iu
    d = np.abs(ref[diag_index(nbas)].real)                         # (nbas, nw)
    scale = np.sqrt(d[iu] * d[ju])                                  # (npack', nw)
    err = np.abs(got[idx] - ref[idx])
    tiny = np.finfo(float).tiny
    emax = float(np.max(err / np.maximum(scale, tiny))) if err.size else 0.0
    fro = float(np.linalg.norm(got - ref) / max(np.linalg.norm(ref), tiny))
    return emax, fro
