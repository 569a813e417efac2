"""Regression check of the tensor-core fact the FP64 kernels rely on (GPU): the
mma.sync f64 fragment layouts (m16n8k4/k8/k16). The probe is a single-CTA,
in-bounds program compiled here with nvcc.
"""
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

