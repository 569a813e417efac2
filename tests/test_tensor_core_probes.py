"""Self-checking probes of the two tensor-core facts the kernels rely on (GPU).

1. mma.sync f64 fragment layouts (m16n8k4/k8/k16) used by the FP64 kernel.
2. How tcgen05.mma kind::f16 (BF16 in, FP32 accumulate) rounds: products are
   aligned to the largest term and truncated toward zero. This is why the split
   path slices into int8 digits with exact int32 accumulation instead of BF16.
Both probes are single-CTA, in-bounds programs compiled here with nvcc.
"""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
HERE = Path(__file__).resolve().parent / "probes"


def build_and_run(src: str, tmp_path) -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / Path(src).stem
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-o", str(exe),
                    str(HERE / src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


def test_dmma_fragment_layouts(tmp_path):
    out = build_and_run("dmma_layout.cu", tmp_path)
    assert out.count("layout ok") == 3


def test_tcgen05_bf16_accumulation_truncates(tmp_path):
    out = build_and_run("tcgen05_rounding.cu", tmp_path)
    assert "single MMA 128x256x16 bf16->f32: ok" in out
    ulp = {int(m.group(1)): float(m.group(2)) for m in re.finditer(r"^t(\d+)\s.*->\s+1 \+ (-?[\d.]+) ulp", out, re.M)}
    assert ulp[0] == 0.0      # 1 + 0.75 ulp stays 1: truncation, not round-to-nearest
    assert ulp[4] == 0.0      # -1 - 0.75 ulp stays -1: toward zero
    assert ulp[5] == 0.0      # 15 products of 0.125 ulp inside one MMA are all lost
