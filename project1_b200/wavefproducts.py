"""Host-side mirror of SPEX's `wavefproducts2_mt` / `wavefproducts2_pw` on libspexgpu.

Reference: src/wavefproducts.f:95-431 (muffin tin), :760-997 (interstitial,
explicit convolution with the step function). The Fortran routines read the
wave-function coefficients from module state (`wavefunction_mt/pw`,
src/trafo.f:514-569); here they are explicit device arrays:

  cmt_occ   complex128 (nk, nocc, natom, maxlm)     coefficients of the occupied bands at k
  cmt_unocc complex128 (nk, nunocc, natom, maxlm)   unoccupied bands at k+q
  cpw_occ   complex128 (nk, nocc, ngpt1)
  cpw_unocc complex128 (nk, nunocc, ngpt2)
  cprod     complex128 (ncol, ldc) row-major == Fortran (ldc, ncol); rows
            p = n' + nunocc*(n + nocc*k), as src/susceptibility.f:861-865 orders them.

Both calls ADD into cprod. Calls on torch tensors are ordered on torch's current
stream unless a stream is given. Descriptors are dicts as built by
project1_b200.inputs.mt_basis / pw_basis.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .susceptibility import PRECISIONS, Context, _ptr, _stats, torch_stream


class MtDesc:
    """spx_mt_desc over host arrays kept alive by this object."""

    def __init__(self, mt: dict):
        self.gaunt = np.asfortranarray(mt["gaunt"], dtype=np.float64)
        self.integral = np.asfortranarray(mt["integral"], dtype=np.float64)
        self.cexp = np.ascontiguousarray(mt["cexp"], dtype=np.complex128)
        self.natom, self.lcut, self.nrad = mt["natom"], mt["lcut"], mt["nrad"]
        self.lcutm, self.nradm = mt["lcutm"], mt["nradm"]
        self.maxlm = (self.lcut + 1) ** 2 * self.nrad
        self.maxllm = (self.lcutm + 1) ** 2 * self.nradm
        self.c = _lib.spx_mt_desc(self.natom, self.lcut, self.nrad, self.lcutm, self.nradm,
                                  self.integral.shape[1], self.gaunt.ctypes.data,
                                  self.integral.ctypes.data, self.cexp.ctypes.data)


class PwDesc:
    """spx_pw_desc over host arrays kept alive by this object."""

    def __init__(self, pw: dict):
        self.gpt1 = np.ascontiguousarray(pw["gpt1"], dtype=np.int32)
        self.gpt2 = np.ascontiguousarray(pw["gpt2"], dtype=np.int32)
        self.gptm = np.ascontiguousarray(pw["gptm"], dtype=np.int32)
        self.cstep = np.ascontiguousarray(pw["cstep"], dtype=np.complex128)
        self.ngptm = self.gptm.shape[0]
        gs = (C.c_int32 * 3)(*[int(x) for x in pw["gshift"]])
        self.c = _lib.spx_pw_desc(self.gpt1.shape[0], self.gpt2.shape[0], self.ngptm,
                                  int(pw["step_radius"]), self.gpt1.ctypes.data,
                                  self.gpt2.ctypes.data, self.gptm.ctypes.data, gs,
                                  int(pw.get("nfft", 0)),
                                  self.cstep.ctypes.data, float(pw["vol"]))


_stream = torch_stream


def wavefproducts2_mt(ctx: Context, mt, cmt_occ, cmt_unocc, cprod, stream=None) -> None:
    """cprod[:natom*maxllm] += MT projections (torch CUDA tensors)."""
    d = mt if isinstance(mt, MtDesc) else MtDesc(mt)
    nk, nocc = cmt_occ.shape[0], cmt_occ.shape[1]
    nunocc = cmt_unocc.shape[1]
    if cmt_occ.shape[2:] != (d.natom, d.maxlm) or cmt_unocc.shape[2:] != (d.natom, d.maxlm):
        raise ValueError("coefficient arrays must be (nk, nb, natom, maxlm)")
    rc = ctx.lib.spx_wfprod_mt_dev(ctx.handle, C.byref(d.c), nk, nocc, nunocc, _ptr(cmt_occ),
                                   _ptr(cmt_unocc), _ptr(cprod), cprod.shape[1], _stream(stream, cprod))
    ctx._check(rc, "spx_wfprod_mt_dev")


def wavefproducts2_pw(ctx: Context, pw, cpw_occ, cpw_unocc, cprod, col0: int,
                      stream=None) -> None:
    """cprod[col0:col0+ngptm] += interstitial projections (torch CUDA tensors)."""
    d = pw if isinstance(pw, PwDesc) else PwDesc(pw)
    nk, nocc = cpw_occ.shape[0], cpw_occ.shape[1]
    nunocc = cpw_unocc.shape[1]
    rc = ctx.lib.spx_wfprod_pw_dev(ctx.handle, C.byref(d.c), nk, nocc, nunocc, _ptr(cpw_occ),
                                   _ptr(cpw_unocc), _ptr(cprod), cprod.shape[1], col0,
                                   _stream(stream, cprod))
    ctx._check(rc, "spx_wfprod_pw_dev")


def chi0_from_coeffs(ctx: Context, mt, pw, cmt_occ, cmt_unocc, cpw_occ, cpw_unocc, ediff,
                     omega, susceph, wscale=None, scale_all: float = 1.0,
                     precision: str = "split", stream=None, stats: bool = False) -> Optional[dict]:
    """susceph += chi0 of the products of the given coefficients; M never leaves the device."""
    dm = mt if isinstance(mt, MtDesc) else MtDesc(mt)
    dp = pw if isinstance(pw, PwDesc) else PwDesc(pw)
    nk, nocc = cmt_occ.shape[0], cmt_occ.shape[1]
    nunocc = cmt_unocc.shape[1]
    st = _lib.spx_chi0_stats() if stats else None
    rc = ctx.lib.spx_chi0_from_coeffs_dev(
        ctx.handle, C.byref(dm.c), C.byref(dp.c), nk, nocc, nunocc, _ptr(cmt_occ),
        _ptr(cmt_unocc), _ptr(cpw_occ), _ptr(cpw_unocc), _ptr(ediff), _ptr(wscale), scale_all,
        omega.shape[0], _ptr(omega), PRECISIONS[precision], _ptr(susceph), _stream(stream, susceph),
        C.byref(st) if st is not None else None)
    ctx._check(rc, "spx_chi0_from_coeffs_dev")
    return _stats(st) if st is not None else None


class MomDesc:
    """spx_mom_desc over host arrays kept alive by this object (momentum matrix of the
    q -> 0 head and wings)."""

    def __init__(self, m: dict):
        self.qmat1 = np.asfortranarray(m["qmat1"], dtype=np.float64)
        self.qmat2 = np.asfortranarray(m["qmat2"], dtype=np.float64)
        self.gpt = np.ascontiguousarray(m["gpt"], dtype=np.int32)
        self.kpt = np.ascontiguousarray(m["kpt"], dtype=np.float64)
        self.rlat = np.asfortranarray(m["rlat"], dtype=np.float64)
        self.cstep = np.ascontiguousarray(m["cstep"], dtype=np.complex128)
        self.c = _lib.spx_mom_desc(int(m["natom"]), int(m["lcut"]), int(m["nrad"]), self.gpt.shape[0],
                                   self.qmat1.ctypes.data, self.qmat2.ctypes.data, self.gpt.ctypes.data,
                                   self.kpt.ctypes.data, self.rlat.ctypes.data, self.cstep.ctypes.data,
                                   int(m["step_radius"]), 0, float(m["vol"]))


def dcprod_dev(ctx: Context, mom: MomDesc, nk: int, nocc: int, nunocc: int, cmt_occ, cmt_unocc,
               cpw_occ, cpw_unocc, dcprod, ediff=None, stream=None) -> None:
    """dcprod (3, ldd) complex128 == Fortran (ldd, 3): momentum / sqrt(vol) / ediff
    (src/dwavefproducts.f:89-330, src/susceptibility.f:848-870)."""
    ldd = dcprod.shape[1]
    rc = ctx.lib.spx_dcprod_dev(ctx.handle, C.byref(mom.c), nk, nocc, nunocc, _ptr(cmt_occ), _ptr(cmt_unocc),
                                _ptr(cpw_occ), _ptr(cpw_unocc), _ptr(ediff), _ptr(dcprod), ldd,
                                torch_stream(stream, dcprod))
    ctx._check(rc, "spx_dcprod_dev")
