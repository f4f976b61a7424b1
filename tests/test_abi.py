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
