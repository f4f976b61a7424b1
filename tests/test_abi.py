"""The C ABI library loads and exports every entry point declared in
include/*.h; error paths work without a GPU."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(hdr).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(tosp_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_all_declared_symbols():
    import tosp
    lib = C.CDLL(tosp.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n


def test_version_and_defaults():
    import tosp
    assert "sm_100a" in tosp.version()
    mg = tosp.default_mg()
    # reference defaults of I/TopOpt3D.m:171-190
    assert (mg.ngrids, mg.cycle, mg.smoother, mg.omega, mg.smoothiter1, mg.smoothiter2) == (3, 1, 0, 0.5, 1, 1)
    assert (mg.tolMG, mg.maxiterMG, mg.nmaxchol) == (1e-8, 5000, 60000)


def test_create_reports_error_without_gpu():
    if gpu_available():
        pytest.skip("a GPU is present")
    import tosp
    from tosp import problems as P
    with pytest.raises(tosp.TospError) as ei:
        tosp.Solver(P.cantilever(4, 2, 2))
    assert ei.value.code in (-2, -3)


def test_python_binding_names_mirror_reference():
    import tosp
    for name in ("SetupGMG", "SolveMG", "KelemProd", "Grad", "ApplyFilter", "MGCycle"):
        assert hasattr(tosp.Solver, name)
    assert callable(tosp.ElemStiffMatrixGQMR)


def test_pointer_rule_refuses_other_gpus_memory(tmp_path):
    """Where a pointer argument lives, from faked cudaPointerGetAttributes
    results (csrc/ptr_kind.h compiled with g++; no GPU needed): device memory
    of the handle's GPU is used in place, another GPU's device memory is
    refused (the kernels would fault on it), host and managed memory work."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    src = tmp_path / "ptr_rule.cpp"
    src.write_text(
        '#include <cstdio>\n#include "ptr_kind.h"\n'
        "using namespace tosp;\n"
        "int main() {\n"
        "  int bad = 0;\n"
        "  bad += classify_ptr(true, MEMTYPE_DEVICE, 0, 0) != PTR_DEVICE;\n"
        "  bad += classify_ptr(true, MEMTYPE_DEVICE, 1, 0) != PTR_OTHER_DEVICE;\n"
        "  bad += classify_ptr(true, MEMTYPE_DEVICE, 0, 3) != PTR_OTHER_DEVICE;\n"
        "  bad += classify_ptr(true, MEMTYPE_MANAGED, 2, 0) != PTR_DEVICE;\n"
        "  bad += classify_ptr(true, MEMTYPE_HOST, 0, 0) != PTR_HOST;\n"
        "  bad += classify_ptr(true, MEMTYPE_UNREGISTERED, -2, 0) != PTR_HOST;\n"
        "  bad += classify_ptr(false, 0, 0, 0) != PTR_HOST;\n"
        '  std::printf("%d\\n", bad);\n  return bad;\n}\n')
    exe = tmp_path / "ptr_rule"
    inc = os.path.join(ROOT, "topopt-slp-3d_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-I" + inc, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "0", r.stdout
