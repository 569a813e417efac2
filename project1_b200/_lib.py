"""ctypes binding of libspexgpu.so (the C ABI in include/spexgpu.h).

The library is the product; this module only declares its signatures. There is
no fallback: importing a function whose library is missing raises at once.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libspexgpu.so"

SPX_OK, SPX_EINVAL, SPX_ENOMEM, SPX_ECUDA, SPX_ETIMEOUT, SPX_ENOTSUP, SPX_ENODEV = 0, -1, -2, -3, -4, -5, -6
SPX_FP64, SPX_SPLIT = 0, 1
SPX_PRODUCTS_AUTO, SPX_PRODUCTS_FP64, SPX_PRODUCTS_SPLIT = 0, 1, 2


class SpexGpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class spx_options(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("verbose", C.c_int32),
        ("workspace_limit", C.c_int64),
        ("pinned_limit", C.c_int64),
        ("chunk_pairs", C.c_int32),
        ("timeout_ms", C.c_int32),
        ("split_variant", C.c_int32),
        ("products", C.c_int32),
    ]


class spx_chi0_stats(C.Structure):
    _fields_ = [
        ("ms_total", C.c_double),
        ("ms_gram", C.c_double),
        ("ms_prep", C.c_double),
        ("flops", C.c_double),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("kernel_launches", C.c_int32),
        ("precision", C.c_int32),
    ]


class spx_mom_desc(C.Structure):
    _fields_ = [
        ("natom", C.c_int32), ("lcut", C.c_int32), ("nrad", C.c_int32), ("ngpt", C.c_int32),
        ("qmat1", C.c_void_p), ("qmat2", C.c_void_p), ("gpt", C.c_void_p), ("kpt", C.c_void_p),
        ("rlat", C.c_void_p), ("cstep", C.c_void_p), ("step_radius", C.c_int32),
        ("reserved", C.c_int32), ("vol", C.c_double),
    ]


class spx_mt_desc(C.Structure):
    _fields_ = [
        ("natom", C.c_int32), ("lcut", C.c_int32), ("nrad", C.c_int32),
        ("lcutm", C.c_int32), ("nradm", C.c_int32), ("ld1", C.c_int32),
        ("gaunt", C.c_void_p), ("integral", C.c_void_p), ("cexp", C.c_void_p),
    ]


class spx_pw_desc(C.Structure):
    _fields_ = [
        ("ngpt1", C.c_int32), ("ngpt2", C.c_int32), ("ngptm", C.c_int32),
        ("step_radius", C.c_int32),
        ("gpt1", C.c_void_p), ("gpt2", C.c_void_p), ("gptm", C.c_void_p),
        ("gshift", C.c_int32 * 3), ("nfft", C.c_int32),
        ("cstep", C.c_void_p), ("vol", C.c_double),
    ]


class spx_q_desc(C.Structure):
    _fields_ = [
        ("nbas", C.c_int32), ("variant", C.c_int32), ("npair", C.c_int64),
        ("slab_pairs", C.c_int32), ("reserved0", C.c_int32),
        ("cprod", C.c_void_p), ("ldc", C.c_int64),
        ("seed", C.c_uint64), ("stream_id", C.c_uint32), ("reserved1", C.c_int32),
        ("m_scale", C.c_double), ("ediff", C.c_void_p), ("wscale", C.c_void_p),
        ("scale_all", C.c_double), ("susceph", C.c_void_p),
    ]


class spx_tune_entry(C.Structure):
    _fields_ = [
        ("nbas_bucket", C.c_int32), ("npair_bucket", C.c_int32), ("nw", C.c_int32),
        ("variant", C.c_int32), ("slab_pairs", C.c_int32), ("tile", C.c_int32),
        ("tflops", C.c_double),
    ]


SPX_BATCH_AUTOTUNE, SPX_BATCH_NOGRAPH, SPX_BATCH_KERNELS = 1, 2, 4

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64 = C.c_int64
_I32 = C.c_int32

# name -> (restype, argtypes); every symbol declared in include/spexgpu.h
SIGNATURES = {
    "spx_abi_version": (C.c_int, []),
    "spx_strerror": (C.c_char_p, [C.c_int]),
    "spx_ctx_create": (C.c_int, [C.c_int, C.POINTER(spx_options), C.POINTER(_P)]),
    "spx_ctx_destroy": (C.c_int, [_P]),
    "spx_last_error": (C.c_char_p, [_P]),
    "spx_ctx_synchronize": (C.c_int, [_P]),
    "spx_weights_dev": (C.c_int, [_P, _I64, _P, _P, C.c_double, _I32, _P, _P, _P]),
    "spx_chi0_accumulate": (
        C.c_int,
        [_P, _P, _I64, _I64, _I32, _P, _P, C.c_double, _I32, _P, _I32, _P, C.POINTER(spx_chi0_stats)],
    ),
    "spx_chi0_accumulate_dev": (
        C.c_int,
        [_P, _P, _I64, _I64, _I32, _P, _P, C.c_double, _I32, _P, _I32, _P, _P, C.POINTER(spx_chi0_stats)],
    ),
    "spx_chi0_accumulate_real_dev": (
        C.c_int,
        [_P, _P, _I64, _I64, _I32, _P, _P, C.c_double, _I32, _P, _I32, _P, _P, C.POINTER(spx_chi0_stats)],
    ),
    "spx_scale_dev": (C.c_int, [_P, _P, _I64, C.c_double, _P]),
    "spx_chi0_accumulate_dev_noalloc": (
        C.c_int, [_P, _I64, _I64, _I32, _P, _P, C.c_double, _I32, _P, _P, _P]),
    "spx_wfprod_mt_dev": (
        C.c_int, [_P, C.POINTER(spx_mt_desc), _I32, _I32, _I32, _P, _P, _P, _I64, _P]),
    "spx_wfprod_pw_dev": (
        C.c_int, [_P, C.POINTER(spx_pw_desc), _I32, _I32, _I32, _P, _P, _P, _I64, _I32, _P]),
    "spx_chi0_from_coeffs_dev": (
        C.c_int,
        [_P, C.POINTER(spx_mt_desc), C.POINTER(spx_pw_desc), _I32, _I32, _I32, _P, _P, _P, _P,
         _P, _P, C.c_double, _I32, _P, _I32, _P, _P, C.POINTER(spx_chi0_stats)],
    ),
    "spx_weights_hilbert_dev": (
        C.c_int, [_P, _I64, _I32, _P, _I64, C.c_double, _I32, _P, C.c_double, _P, _I64, _P]),
    "spx_chi0_accumulate_w_dev": (
        C.c_int, [_P, _P, _I64, _I64, _I32, _P, _I64, _I32, _I32, _P, _P, C.POINTER(spx_chi0_stats)]),
    "spx_chi0_accumulate_c_dev": (
        C.c_int, [_P, _P, _I64, _I64, _I32, _P, _P, _I64, _I32, _I32, _P, _I64, _P,
                  C.POINTER(spx_chi0_stats)]),
    "spx_headwings_dev": (
        C.c_int, [_P, _P, _I64, _I64, _I32, _P, _I64, _P, _I64, _I32, _P, _P, _P]),
    "spx_dielec_dev": (C.c_int, [_P, _I32, _I32, _P, _P, _I32, _P, _P, _P]),
    "spx_selftest_wait_dev": (C.c_int, [_P, _I32]),
    "spx_measure_dmma_peak": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "spx_trafo_dev": (C.c_int, [_P, _P, _I64, _I64, _I32, _P, _I64, _I32, _P, _I64, _P]),
    "spx_dcprod_dev": (C.c_int, [_P, C.POINTER(spx_mom_desc), _I32, _I32, _I32, _P, _P, _P, _P, _P,
                                 _P, _I64, _P]),
    "spx_trafo_olap_dev": (C.c_int, [_P, _P, _I64, _I64, _I32, _I32, _P, _I64, _I32,
                                     C.POINTER(spx_pw_desc), _P, _I64, _P]),
    "spx_chi0_batched": (
        C.c_int, [_P, _I32, C.POINTER(spx_q_desc), _I32, _P, _I32, _I32, _P, C.POINTER(spx_chi0_stats)]),
    "spx_autotune_split": (C.c_int, [_P, _I32, _I64, _I32, C.POINTER(spx_tune_entry)]),
    "spx_tune_lookup": (C.c_int, [_P, _I32, _I64, _I32, C.POINTER(spx_tune_entry)]),
    "spx_autotune_batched": (C.c_int, [_P, _I32, _I64, _I32, C.POINTER(spx_tune_entry)]),
    "spx_tune_lookup_batched": (C.c_int, [_P, _I32, _I64, _I32, C.POINTER(spx_tune_entry)]),
    "spx_tune_save": (C.c_int, [_P, C.c_char_p]),
    "spx_pb_profile_enable": (C.c_int, [_P, _I32]),
    "spx_pb_profile_read": (C.c_int, [_P, _P, _I32]),
    "spx_tune_load": (C.c_int, [_P, C.c_char_p]),
    "spx_gen_normal_host": (None, [C.c_uint64, C.c_uint32, _I64, _I64, C.c_double, _P]),
    "spx_gen_normal_dev": (C.c_int, [_P, C.c_uint64, C.c_uint32, _I64, _I64, C.c_double, _P, _P]),
    "spx_gen_cmatrix_host": (None, [C.c_uint64, C.c_uint32, _I64, _I64, _I64, _I64, C.c_double, _P]),
    "spx_gen_cmatrix_dev": (
        C.c_int,
        [_P, C.c_uint64, C.c_uint32, _I64, _I64, _I64, _I64, C.c_double, _P, _P],
    ),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libspexgpu.so and binds every declared entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python -m project1_b200.build` "
            "(there is no CPU fallback for this library)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def strerror(status: int) -> str:
    return load().spx_strerror(status).decode()
