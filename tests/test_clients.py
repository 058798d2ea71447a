"""Applications written against the reference's interfaces build against
include/ and link with libspla.so unchanged: a C client (tests/cpp/client_c.c:
complex double pgemm_ssb, float pgemm_ssbtr, double pgemm_sbs) and a C++ client
(tests/cpp/client_cpp.cpp: Context, MatrixDistribution, complex float
pgemm_ssb, double pgemm_ssbtr with offsets, gemm over all op pairs, the
exception of an invalid call). Building and linking is checked on the CPU;
running them (each checks its results against long-double loops) needs a GPU."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
INC = ["-I", str(ROOT / "include"), "-I", str(ROOT / "spla_b200" / "csrc" / "mpi_single_rank")]


def _build(spla_lib, tmp_path, src, compiler, std):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not available")
    exe = tmp_path / Path(src).stem
    libdir = str(Path(spla_lib.LIB_PATH).parent)
    cmd = [compiler, std, "-O2", "-o", str(exe), str(ROOT / "tests" / "cpp" / src)] + INC + [
        "-L", libdir, "-lspla", f"-Wl,-rpath,{libdir}", "-lm"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


@pytest.mark.parametrize("src,compiler,std", [("client_c.c", "gcc", "-std=c11"),
                                              ("client_cpp.cpp", "g++", "-std=c++17")])
def test_client_builds_and_links(spla_lib, tmp_path, src, compiler, std):
    _build(spla_lib, tmp_path, src, compiler, std)


@pytest.mark.gpu
@pytest.mark.parametrize("src,compiler,std", [("client_c.c", "gcc", "-std=c11"),
                                              ("client_cpp.cpp", "g++", "-std=c++17")])
def test_client_runs(spla_lib, tmp_path, src, compiler, std):
    exe = _build(spla_lib, tmp_path, src, compiler, std)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip().endswith("OK"), out.stdout + out.stderr
