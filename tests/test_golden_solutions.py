"""The committed golden solutions (tests/golden/solutions.npz, made by
tests/golden/make_solutions.py from the NumPy/SciPy oracle) are reproduced by
the oracle and by its C/OpenMP restatement of the assembled path, so a change
to either is caught before the GPU tests compare the CUDA path with them."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_solutions as MS  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "solutions.npz"))


def golden(name):
    return {k.split("/", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(name + "/")}


@pytest.mark.parametrize("name", list(MS.CASES))
def test_oracle_reproduces_golden(name):
    r = MS.solve_case(name, MS.CASES[name])
    gd = golden(name)
    assert int(r["it"][0]) == int(gd["it"][0])
    assert np.abs(r["u"] - gd["u"]).max() <= 1e-12 * np.abs(gd["u"]).max()
    assert np.abs(r["g"] - gd["g"]).max() <= 1e-12 * np.abs(gd["g"]).max()
    assert gd["relres"][0] <= 1e-8


@pytest.mark.parametrize("name", list(MS.CASES))
def test_assembled_port_reproduces_golden(name):
    pytest.importorskip("oracle.cpu_assembled")
    from oracle_solver import AssembledOracleSolver
    spec = MS.CASES[name]
    pb = MS.case_problem(name)
    gd = golden(name)
    n = spec["n"]
    dens = gd["dens"] if "dens" in gd else np.full(pb.nelem * n ** 3, 0.3)
    s = AssembledOracleSolver(pb, n=n, ngrids=MS.NGRIDS, omega=spec["omega"], rmin=spec["rmin"], nthreads=4)
    s.SetupGMG(dens)
    u, it, nr, _ = s.SolveMG(np.zeros(pb.f.size), pb.f)
    assert it == int(gd["it"][0]) and nr <= 1e-8
    assert abs(pb.f @ u - gd["F"][0]) <= 1e-11 * abs(gd["F"][0])
    assert np.abs(u - gd["u"]).max() <= 1e-10 * np.abs(gd["u"]).max()
    uf = np.zeros(3 * pb.nnodes)
    uf[pb.freedofs] = u
    g = s.Grad(uf)
    assert np.abs(g - gd["g"]).max() <= 1e-10 * np.abs(gd["g"]).max()
