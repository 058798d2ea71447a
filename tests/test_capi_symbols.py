"""The product library loads and exports every function the public headers
declare (include/*.h and include/spla/*.h), plus the C++ interface. CPU only:
no compute call is made."""
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_c_functions():
    names = set()
    for h in list((ROOT / "include").glob("*.h")) + list((ROOT / "include" / "spla").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"(?:SPLA_EXPORT|SPLAB_API)\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_headers_declare_reference_abi():
    """Every C symbol the reference library exports (tests/golden/ref_symbols.txt,
    taken from the reference build) is declared, plus spla_ctx_processing_unit,
    which the reference declares (include/spla/context.h:70) but never defines."""
    names = declared_c_functions()
    ref = set((ROOT / "tests" / "golden" / "ref_symbols.txt").read_text().split())
    assert ref, "empty reference symbol list"
    assert not sorted(ref - names)
    ours = {n for n in names if n.startswith("spla_") and not n.startswith("spla_b200")}
    assert ours - ref == {"spla_ctx_processing_unit"}
    for n in ["splab_gemm", "splab_block_cyclic_info", "splab_gemm_workspace_size"]:
        assert n in names, n


def test_library_exports_every_declared_symbol(spla_lib):
    syms = exported(spla_lib.LIB_PATH)
    missing = sorted(declared_c_functions() - syms)
    assert not missing, missing


def test_library_exports_cpp_interface(spla_lib):
    out = subprocess.run(["nm", "-DC", "--defined-only", str(spla_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    for sig in ["spla::pgemm_ssb(int, int, int, SplaOperation, std::complex<double>",
                "spla::pgemm_ssbtr(int, int, int, SplaOperation, float",
                "spla::pgemm_sbs(int, int, int, double",
                "spla::gemm(SplaOperation, SplaOperation, int, int, int, std::complex<float>",
                "spla::Context::Context(SplaProcessingUnit)",
                "spla::MatrixDistribution::create_blacs_block_cyclic(int, char, int, int, int, int)"]:
        assert sig in out, sig


def test_library_loads_via_ctypes(spla_lib):
    lib = spla_lib.lib()
    assert lib.splab_status_string(0) == b"ok"
