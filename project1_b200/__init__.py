"""spexgpu: B200-native (sm_100a) Kohn-Sham polarisation for SPEX 05.10.

The compute path is libspexgpu.so (hand-written CUDA + a C ABI, include/spexgpu.h);
this package binds it and mirrors the reference's `susceptibility` call surface.
"""
from ._lib import SPX_FP64, SPX_SPLIT, SpexGpuError, load  # noqa: F401
from .susceptibility import (Context, gen_cmatrix_host, gen_normal_host, npack,  # noqa: F401
                             packed_index, susceptibility, unpack_hermitian)

__all__ = ["Context", "SpexGpuError", "susceptibility", "npack", "packed_index",
           "unpack_hermitian", "gen_cmatrix_host", "gen_normal_host", "load",
           "SPX_FP64", "SPX_SPLIT"]
