"""The drop-in boundary without a GPU.

The reference's headers declare its entry points with C++ linkage (no
extern "C": Release_CBCT_Projection_CM/reprojectionOnGPU.h:1-19,
lengthproj.h, IR_ImageCBCT.h, Release_recon_from_forward_pro_float_CM/
filterSinogram.h:1-6, reconstructImage.h:1-5), so a driver compiled against
them asks the linker for the mangled names.  libvcbct must define exactly
those; a program that includes the reference's own headers and calls every
entry point must link against -lvcbct alone; and the reference's unmodified
programs built by oracle/Makefile against -lvcbct must resolve every symbol.
"""
import os
import subprocess

import pytest

from oracle.refpath import reference_path

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
LIB = os.path.join(ROOT, "virtualcbct_b200", "libvcbct.so")
REF = os.path.join(ROOT, "oracle", "_ref")

# The Itanium C++ ABI names of the reference's prototypes.
MANGLED = {
    "initializeGPU": "_Z13initializeGPUididiiiPdS_S_S_dddddddi",
    "terminateGPU": "_Z12terminateGPUv",
    "reprojectionOnGPU": "_Z17reprojectionOnGPUiiiPtPfS0_S0_ddiiiiPdS1_S1_S1_S1_dS1_dddddddS0_S0_iiPc",
    "lengthproj": "_Z10lengthprojiiiPsPtPfS0_ddiiiiPdS2_S2_S2_S2_dS2_ddddddd",
    "IR_ImageCBCT": "_Z12IR_ImageCBCTiiidPsPfS0_S0_dddi",
    "prepareConstMap": "_Z15prepareConstMapid",
    "filterSinogram": "_Z14filterSinogramiiiPPPfS1_PPdS2_S2_d",
    "reconstructImage": "_Z16reconstructImageiiiddPPPdPPciiiPPPfiS_S_S_S_d",
}


def _exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_reference_names_exported_with_cpp_linkage():
    names = _exported()
    missing = [k for k, m in MANGLED.items() if m not in names]
    assert not missing, missing
    # the C twins serve C and ctypes callers; the bare C names are not exported
    for k in MANGLED:
        assert "vcbct_" + k in names
        assert k not in names


def test_program_using_the_reference_headers_links(tmp_path):
    """Compile a caller of all eight entry points against the reference's own
    headers and link it against libvcbct only (no reference objects)."""
    P = reference_path("Release_CBCT_Projection_CM")
    R = reference_path("Release_recon_from_forward_pro_float_CM")
    if not os.path.isdir(P):
        pytest.skip("reference tree not available")
    src = tmp_path / "caller.cpp"
    src.write_text(
        '#include "reprojectionOnGPU.h"\n#include "lengthproj.h"\n#include "IR_ImageCBCT.h"\n'
        '#include "filterSinogram.h"\n#include "reconstructImage.h"\n'
        "int main(int argc, char**) {\n"
        "  if (argc > 100) {\n"
        "    initializeGPU(0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0);\n"
        "    reprojectionOnGPU(0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0);\n"
        "    terminateGPU();\n"
        "    lengthproj(0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0);\n"
        "    IR_ImageCBCT(0,0,0,0,0,0,0,0,0,0,0,0);\n"
        "    double** m = prepareConstMap(0, 0);\n"
        "    filterSinogram(0,0,0,0,0,m,0,0,0);\n"
        "    reconstructImage(0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0,0);\n"
        "  }\n  return 0;\n}\n")
    exe = tmp_path / "caller"
    r = subprocess.run(["g++", "-std=c++17", "-w", f"-I{P}", f"-I{R}", str(src), "-o", str(exe),
                        f"-L{os.path.dirname(LIB)}", "-lvcbct", f"-Wl,-rpath,{os.path.dirname(LIB)}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_our_reference_header_matches_the_exports(tmp_path):
    """include/vcbct_reference.h declares the same functions the library
    defines (a caller compiled against it links)."""
    src = tmp_path / "caller.cpp"
    src.write_text('#include "vcbct_reference.h"\n#include "vcbct.h"\n'
                   "int main(int argc, char**) { if (argc > 100) { terminateGPU();"
                   " double** m = prepareConstMap(4, 0.1); vcbct_free_const_map(m, 4); } return 0; }\n")
    exe = tmp_path / "caller"
    r = subprocess.run(["g++", "-std=c++17", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe),
                        f"-L{os.path.dirname(LIB)}", "-lvcbct", f"-Wl,-rpath,{os.path.dirname(LIB)}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.parametrize("prog", ["proj_dropin", "cbct2_dropin"])
def test_prebuilt_dropins_resolve_every_symbol(prog):
    path = os.path.join(REF, prog)
    if not os.path.exists(path):
        pytest.skip(f"{prog} not built (make -C oracle where the reference tree is present)")
    r = subprocess.run(["ldd", "-r", path], capture_output=True, text=True)
    assert "undefined symbol" not in r.stdout + r.stderr, r.stdout + r.stderr
    assert "libvcbct.so" in r.stdout
