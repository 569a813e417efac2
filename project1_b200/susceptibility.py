"""Host-side mirror of SPEX's `susceptibility` call surface for the HILBERT NONE
imaginary-frequency polarisation, running on libspexgpu.

Reference: src/susceptibility.f:100-102 (signature), :211-223 (outputs zeroed on
entry), :751-1276 (packet loop: products, weights, body accumulation),
:1331-1343 (spin factor 2). The Fortran routine reads its band-pair products
from module state after `wavefproducts2_*`; here they are explicit arguments.

Array conventions (those of the Fortran caller):
  cprod    complex128 (npair, nbas), Fortran order: column I holds M_I,p for all
           band pairs p = n' + nu*(n + no*k)          (src/susceptibility.f:861-865)
  ediff    float64 (npair,) e_n'(k+q) - e_n(k)
  frqh     complex128 (nw,) imaginary frequencies i*omega (frqh/img = omega)
  susceph  complex128 (nbas*(nbas+1)/2, nw), Fortran order, packed upper triangle
           ij = j*(j+1)/2 + i (0-based, i <= j)        (src/susceptibility.f:1210)
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import SPX_FP64, SPX_SPLIT, SpexGpuError

PRECISIONS = {"fp64": SPX_FP64, "split": SPX_SPLIT}


def _ptr(a) -> C.c_void_p:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(int(a.data_ptr()))  # torch tensor


def npack(nbas: int) -> int:
    return nbas * (nbas + 1) // 2


def packed_index(i: int, j: int) -> int:
    """0-based packed upper-triangle index of (i, j), i <= j."""
    return j * (j + 1) // 2 + i


def unpack_hermitian(susceph: np.ndarray, nbas: int) -> np.ndarray:
    """Packed (npack, nw) -> full Hermitian (nw, nbas, nbas)."""
    sp = np.asarray(susceph)
    nw = sp.shape[1]
    out = np.zeros((nw, nbas, nbas), dtype=np.complex128)
    iu, ju = np.triu_indices(nbas)
    idx = ju * (ju + 1) // 2 + iu
    for f in range(nw):
        out[f, iu, ju] = sp[idx, f]
        out[f, ju, iu] = np.conj(sp[idx, f])
    return out


class Context:
    """One libspexgpu context: a device, its streams and workspace."""

    def __init__(self, device: int = 0, workspace_limit: int = 0, chunk_pairs: int = 0,
                 timeout_ms: int = 0, pinned_limit: int = 0, split_variant: int = 0,
                 products: int = 0):
        self.lib = _lib.load()
        opt = _lib.spx_options(C.sizeof(_lib.spx_options), 0, workspace_limit, pinned_limit,
                               chunk_pairs, timeout_ms, split_variant, products)
        h = C.c_void_p()
        rc = self.lib.spx_ctx_create(device, C.byref(opt), C.byref(h))
        if rc != 0:
            raise SpexGpuError(rc, f"spx_ctx_create: {_lib.strerror(rc)}")
        self.handle = h
        self.device = device
        self.split_variant = split_variant

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.spx_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            msg = self.lib.spx_last_error(self.handle).decode()
            raise SpexGpuError(rc, f"{what}: {_lib.strerror(rc)}: {msg}")

    def synchronize(self) -> None:
        self._check(self.lib.spx_ctx_synchronize(self.handle), "spx_ctx_synchronize")

    # ---- band-pair accumulation ------------------------------------------------

    def chi0_accumulate(self, cprod: np.ndarray, ediff: np.ndarray, omega: np.ndarray,
                        susceph: np.ndarray, wscale: Optional[np.ndarray] = None,
                        scale_all: float = 1.0, precision: str = "fp64") -> dict:
        """susceph += sum_p cprod(p,i) conj(cprod(p,j)) w(p,f) on host arrays (drop-in)."""
        cprod = np.asarray(cprod)
        if cprod.dtype != np.complex128 or not cprod.flags.f_contiguous:
            raise ValueError("cprod must be a Fortran-ordered complex128 (npair, nbas) array")
        if susceph.dtype != np.complex128 or not susceph.flags.f_contiguous:
            raise ValueError("susceph must be a Fortran-ordered complex128 (npack, nw) array")
        npair, nbas = cprod.shape
        ediff = np.ascontiguousarray(ediff, dtype=np.float64)
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        ws = None if wscale is None else np.ascontiguousarray(wscale, dtype=np.float64)
        st = _lib.spx_chi0_stats()
        rc = self.lib.spx_chi0_accumulate(self.handle, _ptr(cprod), npair, npair, nbas, _ptr(ediff),
                                          _ptr(ws), scale_all, len(omega), _ptr(omega),
                                          PRECISIONS[precision], _ptr(susceph), C.byref(st))
        self._check(rc, "spx_chi0_accumulate")
        return _stats(st)

    def chi0_accumulate_host_ptr(self, cprod_ptr: int, ldc: int, npair: int, nbas: int,
                                 ediff: np.ndarray, omega: np.ndarray, susceph: np.ndarray,
                                 wscale: Optional[np.ndarray] = None, scale_all: float = 1.0,
                                 precision: str = "fp64") -> dict:
        """Same as chi0_accumulate on a raw host pointer (e.g. pinned torch memory)."""
        ediff = np.ascontiguousarray(ediff, dtype=np.float64)
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        ws = None if wscale is None else np.ascontiguousarray(wscale, dtype=np.float64)
        st = _lib.spx_chi0_stats()
        rc = self.lib.spx_chi0_accumulate(self.handle, C.c_void_p(cprod_ptr), ldc, npair, nbas,
                                          _ptr(ediff), _ptr(ws), scale_all, len(omega), _ptr(omega),
                                          PRECISIONS[precision], _ptr(susceph), C.byref(st))
        self._check(rc, "spx_chi0_accumulate")
        return _stats(st)

    def chi0_accumulate_dev(self, cprod, ediff, omega, susceph, wscale=None, scale_all: float = 1.0,
                            precision: str = "fp64", stream=None, npair: Optional[int] = None,
                            stats: bool = False) -> Optional[dict]:
        """Device form on torch CUDA tensors, ordered on torch's current stream unless
        `stream` is given.

        cprod: complex128 (nbas, ldc) row-major == Fortran (ldc, nbas); npair <= ldc.
        susceph: complex128 (nw, npack) row-major == Fortran (npack, nw).
        """
        nbas, ldc = cprod.shape
        npair = ldc if npair is None else npair
        nw = omega.shape[0]
        st = _lib.spx_chi0_stats() if stats else None
        rc = self.lib.spx_chi0_accumulate_dev(
            self.handle, _ptr(cprod), ldc, npair, nbas, _ptr(ediff), _ptr(wscale), scale_all, nw,
            _ptr(omega), PRECISIONS[precision], _ptr(susceph), torch_stream(stream, susceph),
            C.byref(st) if st is not None else None)
        self._check(rc, "spx_chi0_accumulate_dev")
        return _stats(st) if st is not None else None

    def weights_dev(self, ediff, omega, w, wscale=None, scale_all: float = 1.0, stream=None) -> None:
        rc = self.lib.spx_weights_dev(self.handle, ediff.shape[0], _ptr(ediff), _ptr(wscale), scale_all,
                                      omega.shape[0], _ptr(omega), _ptr(w),
                                      torch_stream(stream, w))
        self._check(rc, "spx_weights_dev")

    def scale_dev(self, z, factor: float, stream=None) -> None:
        rc = self.lib.spx_scale_dev(self.handle, _ptr(z), z.numel(), factor, torch_stream(stream, z))
        self._check(rc, "spx_scale_dev")

    # ---- Hilbert-mesh weights and caller-given weights ----------------------------

    def weights_hilbert_dev(self, wtetra, wghtSr, w, thr: float = 0.0, scale_all: float = 1.0,
                            npair: Optional[int] = None, stream=None) -> None:
        """w(p, f) = scale_all sum_s [wtetra > thr] wtetra(p, s) wghtSr(s, f).

        wtetra: float64 (nfrqs, ldt) == Fortran (ldt, nfrqs); wghtSr: (nw, nfrqs) ==
        Fortran (nfrqs, nw); w: (nw, ldw) == Fortran (ldw, nw)."""
        nfrqs, ldt = wtetra.shape
        nw, ldw = w.shape
        npair = ldt if npair is None else npair
        rc = self.lib.spx_weights_hilbert_dev(self.handle, npair, nfrqs, _ptr(wtetra), ldt, thr, nw,
                                              _ptr(wghtSr), scale_all, _ptr(w), ldw, torch_stream(stream, w))
        self._check(rc, "spx_weights_hilbert_dev")

    def chi0_accumulate_real_dev(self, cprod, ediff, omega, susceph, wscale=None,
                                 scale_all: float = 1.0, precision: str = "fp64", stream=None,
                                 npair: Optional[int] = None, stats: bool = False) -> Optional[dict]:
        """The -DINV form: cprod float64 (nbas, ldc) == Fortran real (ldc, nbas), susceph
        float64 (nw, npack) == Fortran real (npack, nw)."""
        nbas, ldc = cprod.shape
        npair = ldc if npair is None else npair
        nw = omega.shape[0]
        st = _lib.spx_chi0_stats() if stats else None
        rc = self.lib.spx_chi0_accumulate_real_dev(
            self.handle, _ptr(cprod), ldc, npair, nbas, _ptr(ediff), _ptr(wscale), scale_all, nw,
            _ptr(omega), PRECISIONS[precision], _ptr(susceph), torch_stream(stream, susceph),
            C.byref(st) if st is not None else None)
        self._check(rc, "spx_chi0_accumulate_real_dev")
        return _stats(st) if st is not None else None

    def chi0_accumulate_w_dev(self, cprod, w, susceph, precision: str = "fp64",
                              npair: Optional[int] = None, stream=None, stats: bool = False):
        """susceph += sum_p cprod(p,i) conj(cprod(p,j)) w(p,f) with given weights w (nw, ldw)."""
        nbas, ldc = cprod.shape
        nw, ldw = w.shape
        npair = ldc if npair is None else npair
        st = _lib.spx_chi0_stats() if stats else None
        rc = self.lib.spx_chi0_accumulate_w_dev(self.handle, _ptr(cprod), ldc, npair, nbas, _ptr(w), ldw,
                                                nw, PRECISIONS[precision], _ptr(susceph),
                                                torch_stream(stream, susceph),
                                                C.byref(st) if st is not None else None)
        self._check(rc, "spx_chi0_accumulate_w_dev")
        return _stats(st) if st is not None else None

    def chi0_accumulate_c_dev(self, cprod, wr, wi, suscepc, precision: str = "fp64",
                              npair: Optional[int] = None, stream=None, stats: bool = False):
        """Real-frequency suscepc += sum_p cprod(p,i) conj(cprod(p,j)) (wr + i wi)(p,f), full
        matrix: suscepc complex128 (nw, nbas, ldo) row-major == Fortran (ldo, nbas, nw);
        wr, wi (nw, ldw)."""
        nbas, ldc = cprod.shape
        nw, ldw = wr.shape
        ldo = suscepc.shape[2]
        npair = ldc if npair is None else npair
        st = _lib.spx_chi0_stats() if stats else None
        rc = self.lib.spx_chi0_accumulate_c_dev(self.handle, _ptr(cprod), ldc, npair, nbas, _ptr(wr),
                                                _ptr(wi), ldw, nw, PRECISIONS[precision], _ptr(suscepc),
                                                ldo, torch_stream(stream, suscepc),
                                                C.byref(st) if st is not None else None)
        self._check(rc, "spx_chi0_accumulate_c_dev")
        return _stats(st) if st is not None else None

    # ---- q -> 0 head and wings -------------------------------------------------------

    def headwings_dev(self, cprod, dcprod, w, head, wing, npair: Optional[int] = None,
                      stream=None) -> None:
        """head (nw, 6) and wing (nw, dim, 3) complex, row-major == Fortran (6, nw) and
        (3, dim, nw); cprod (dim, ldc), dcprod (3, ldd), w (nw, ldw)."""
        dim, ldc = cprod.shape
        ldd = dcprod.shape[1]
        nw, ldw = w.shape
        npair = ldd if npair is None else npair
        rc = self.lib.spx_headwings_dev(self.handle, _ptr(cprod), ldc, npair, dim, _ptr(dcprod), ldd,
                                        _ptr(w), ldw, nw, _ptr(head), _ptr(wing), torch_stream(stream, head))
        self._check(rc, "spx_headwings_dev")

    # ---- dielectric matrix ----------------------------------------------------------

    def dielec_dev(self, susceph, coul, invert: bool = True, head=None, wing=None,
                   stream=None) -> None:
        """In place: susceph (nw, npack) -> eps = 1 - v^1/2 chi v^1/2, inverted if asked
        (src/correlation.f:614-636, :703-745); head (nw, 6), wing (nw, nbas, 3) optional."""
        nw, npk = susceph.shape
        nbas = int(round((np.sqrt(8 * npk + 1) - 1) / 2))
        rc = self.lib.spx_dielec_dev(self.handle, nbas, nw, _ptr(susceph), _ptr(coul), int(invert),
                                     _ptr(head), _ptr(wing), torch_stream(stream, susceph))
        self._check(rc, "spx_dielec_dev")

    # ---- transform to the Coulomb eigenbasis -----------------------------------------

    def trafo_dev(self, cprod, ctrafo, out=None, npair: Optional[int] = None, stream=None):
        """out(p, j) = sum_i cprod(p, i) conj(ctrafo(i, j)) (src/susceptibility.f:806-832).

        cprod: complex128 (nbas, ldc) == Fortran (ldc, nbas); ctrafo: (dim, ldt) ==
        Fortran (ldt, dim); out: (dim, ldo) or None for in place (then dim <= nbas)."""
        nbas, ldc = cprod.shape
        dim, ldt = ctrafo.shape
        npair = ldc if npair is None else npair
        o = cprod if out is None else out
        rc = self.lib.spx_trafo_dev(self.handle, _ptr(cprod), ldc, npair, nbas, _ptr(ctrafo), ldt,
                                    dim, _ptr(o), o.shape[1], torch_stream(stream, cprod))
        self._check(rc, "spx_trafo_dev")
        return o

    def trafo_olap_dev(self, cprod, ctrafo, nbasp: int, pw, out=None, npair: Optional[int] = None,
                       stream=None):
        """The transform without FULLPW (src/susceptibility.f:814-824): the interstitial
        rows of ctrafo are first multiplied by the plane-wave overlap built from
        pw (a wavefproducts.PwDesc: gptm and cstep). Shapes as trafo_dev."""
        nbas, ldc = cprod.shape
        dim, ldt = ctrafo.shape
        npair = ldc if npair is None else npair
        o = cprod if out is None else out
        rc = self.lib.spx_trafo_olap_dev(self.handle, _ptr(cprod), ldc, npair, nbas, nbasp, _ptr(ctrafo),
                                         ldt, dim, C.byref(pw.c), _ptr(o), o.shape[1],
                                         torch_stream(stream, cprod))
        self._check(rc, "spx_trafo_olap_dev")
        return o

    # ---- many q points in one launch ---------------------------------------------

    def chi0_batched(self, qs, omega, precision: str = "split", flags: int = 0, stream=None,
                     stats: bool = False) -> Optional[dict]:
        """Accumulates every q of `qs` (dicts, see below) in one launch of a cached graph.

        Each dict: nbas, npair, ediff (device float64), susceph (device complex128
        (nw, npack)), optionally cprod (device (nbas, ldc)) or seed/stream_id/m_scale
        for on-device generation, wscale, scale_all, variant, slab_pairs.
        Ordered on torch's current stream unless `stream` is given."""
        arr = (_lib.spx_q_desc * max(len(qs), 1))()
        for i, q in enumerate(qs):
            d = arr[i]
            d.nbas, d.npair = int(q["nbas"]), int(q["npair"])
            d.variant, d.slab_pairs = int(q.get("variant", 0)), int(q.get("slab_pairs", 0))
            cp = q.get("cprod")
            d.cprod = None if cp is None else int(cp.data_ptr())
            d.ldc = 0 if cp is None else int(cp.shape[1])
            d.seed, d.stream_id = int(q.get("seed", 0)), int(q.get("stream_id", 0))
            d.m_scale = float(q.get("m_scale", 1.0))
            d.ediff = int(q["ediff"].data_ptr())
            ws = q.get("wscale")
            d.wscale = None if ws is None else int(ws.data_ptr())
            d.scale_all = float(q.get("scale_all", 1.0))
            d.susceph = int(q["susceph"].data_ptr())
        st = _lib.spx_chi0_stats() if stats else None
        rc = self.lib.spx_chi0_batched(self.handle, len(qs), arr, omega.shape[0], _ptr(omega),
                                       PRECISIONS[precision], flags, torch_stream(stream, omega),
                                       C.byref(st) if st is not None else None)
        self._check(rc, "spx_chi0_batched")
        return _stats(st) if st is not None else None

    def measure_dmma_peak(self) -> float:
        """The device's FP64 tensor (DMMA) peak in TFLOP/s, measured by the library."""
        v = C.c_double()
        self._check(self.lib.spx_measure_dmma_peak(self.handle, C.byref(v)), "spx_measure_dmma_peak")
        return v.value

    def autotune_split(self, nbas: int, npair: int, nw: int) -> dict:
        e = _lib.spx_tune_entry()
        self._check(self.lib.spx_autotune_split(self.handle, nbas, npair, nw, C.byref(e)),
                    "spx_autotune_split")
        return _stats(e)

    def tune_lookup(self, nbas: int, npair: int, nw: int) -> Optional[dict]:
        e = _lib.spx_tune_entry()
        rc = self.lib.spx_tune_lookup(self.handle, nbas, npair, nw, C.byref(e))
        return _stats(e) if rc == 0 else None

    def autotune_batched(self, nbas: int, npair: int, nw: int) -> dict:
        e = _lib.spx_tune_entry()
        self._check(self.lib.spx_autotune_batched(self.handle, nbas, npair, nw, C.byref(e)),
                    "spx_autotune_batched")
        return _stats(e)

    def tune_lookup_batched(self, nbas: int, npair: int, nw: int) -> Optional[dict]:
        e = _lib.spx_tune_entry()
        rc = self.lib.spx_tune_lookup_batched(self.handle, nbas, npair, nw, C.byref(e))
        return _stats(e) if rc == 0 else None

    PB_PROFILE_FIELDS = ("cta", "tma_wait_planes", "tma_wait_stage", "mma_wait_operands",
                         "mma_wait_epilogue", "mma_wait_item", "epilogue_wait_tile",
                         "epilogue_wait_order", "prep_wait", "prep_m", "prep_weights",
                         "prep_planes", "accumulation_items", "preparation_items")

    def pb_profile_enable(self, on: bool = True) -> None:
        """Role cycle counters of the persistent schedule: zeroed and switched on (or off)."""
        self._check(self.lib.spx_pb_profile_enable(self.handle, 1 if on else 0), "spx_pb_profile_enable")

    def pb_profile_read(self) -> dict:
        """The counters summed since the last enable (waits for the device)."""
        n = len(self.PB_PROFILE_FIELDS)
        out = (C.c_double * n)()
        self._check(self.lib.spx_pb_profile_read(self.handle, out, n), "spx_pb_profile_read")
        return dict(zip(self.PB_PROFILE_FIELDS, list(out)))

    def tune_save(self, path: str) -> None:
        self._check(self.lib.spx_tune_save(self.handle, str(path).encode()), "spx_tune_save")

    def tune_load(self, path: str) -> None:
        self._check(self.lib.spx_tune_load(self.handle, str(path).encode()), "spx_tune_load")

    def gen_cmatrix_dev(self, seed: int, stream_id: int, out, rows: int, col0: int = 0,
                        scale: float = 1.0, stream=None) -> None:
        """Fills torch complex128 (cols, ld) with the seeded normal matrix (see spx_gen_cmatrix_host)."""
        cols, ld = out.shape
        rc = self.lib.spx_gen_cmatrix_dev(self.handle, seed, stream_id, rows, cols, ld, col0, scale,
                                          _ptr(out), torch_stream(stream, out))
        self._check(rc, "spx_gen_cmatrix_dev")


def torch_stream(stream, like=None):
    """The stream a call is ordered on: the given one, else torch's current stream of
    the tensor `like` (so the call is ordered after the torch work that made its inputs)."""
    if stream is None and like is not None and hasattr(like, "is_cuda") and like.is_cuda:
        import torch
        stream = torch.cuda.current_stream(like.device).cuda_stream
    if stream is None:
        return None
    # handle 0 is the legacy default stream (torch's default stream), which the C ABI
    # would read as "the context stream": name it as cudaStreamLegacy (handle 1)
    return C.c_void_p(int(stream) or 1)


def _stats(st) -> dict:
    return {k: getattr(st, k) for k, _ in st._fields_}


def gen_cmatrix_host(seed: int, stream_id: int, rows: int, cols: int, col0: int = 0,
                     scale: float = 1.0) -> np.ndarray:
    """Seeded complex normal matrix (rows, cols), Fortran order; identical bits to the device form."""
    out = np.empty((rows, cols), dtype=np.complex128, order="F")
    _lib.load().spx_gen_cmatrix_host(seed, stream_id, rows, cols, rows, col0, scale, _ptr(out))
    return out


def gen_normal_host(seed: int, stream_id: int, offset: int, n: int, scale: float = 1.0) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    _lib.load().spx_gen_normal_host(seed, stream_id, offset, n, scale, _ptr(out))
    return out


def susceptibility(ctx: Context, cprod: np.ndarray, ediff: np.ndarray, frqh: np.ndarray, nkpt: int,
                   nsym1: int = 1, nkpts: Optional[np.ndarray] = None, nspin: int = 1,
                   l_soc: bool = False, precision: str = "fp64",
                   packets: Optional[list] = None) -> np.ndarray:
    """HILBERT NONE susceph for one q point and spin, as `susceptibility` returns it.

    `nkpts` (per pair) is the weight of the k point of each pair; the pair weight
    is nkpts(k)/nkpt/nsym1 (src/susceptibility.f:965). `packets` optionally
    lists (p_begin, p_end) band-pair ranges accumulated one after another, as the
    reference's MEM packets are (:751-758); the result does not depend on them.
    """
    cprod = np.asfortranarray(cprod, dtype=np.complex128)
    npair, nbas = cprod.shape
    omega = np.asarray(np.asarray(frqh) / 1j).real.astype(np.float64)
    nw = omega.shape[0]
    susceph = np.zeros((npack(nbas), nw), dtype=np.complex128, order="F")   # intent(out), zeroed
    wscale = None if nkpts is None else np.asarray(nkpts, dtype=np.float64)
    scale_all = 1.0 / nkpt / nsym1
    for (b, e) in (packets or [(0, npair)]):
        ctx.chi0_accumulate(np.asfortranarray(cprod[b:e]), ediff[b:e], omega, susceph,
                            wscale=None if wscale is None else wscale[b:e], scale_all=scale_all,
                            precision=precision)
    if not l_soc and nspin == 1:
        susceph *= 2.0                                                        # :1336
    return susceph
