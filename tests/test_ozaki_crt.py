"""CPU check of the Ozaki path's CRT weights and reconstruction arithmetic
(tests/cpp/test_crt.cu, compiled with nvcc for the host)."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("nvcc") is None and not Path("/usr/local/cuda/bin/nvcc").exists(),
                    reason="nvcc not available")
def test_crt_reconstruction(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "test_crt"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-o", str(exe), str(HERE / "cpp" / "test_crt.cu")],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK")
