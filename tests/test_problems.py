"""Problem builders against the reference's saved fixtures (golden vectors
extracted from Implementation/Tests/*.mat by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from tosp import problems as P

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "fixtures.npz"))
NAMES = sorted({k.split("/")[0] for k in GOLD.files})


@pytest.mark.parametrize("name", NAMES)
def test_supports_loads_regions_bit_exact(name):
    nelx, nely, nelz = [int(v) for v in GOLD[name + "/dims"]]
    el, eh, ew, E, nu = GOLD[name + "/sizes"]
    fix = GOLD[name + "/fix"] if (name + "/fix") in GOLD.files else None
    pb = P.build(nelx, nely, nelz, GOLD[name + "/supp"], GOLD[name + "/loads"], fix=fix, el=el, eh=eh, ew=ew,
                 E=E, nu=nu)
    mask = np.unpackbits(GOLD[name + "/freemask"])[: 3 * pb.nnodes].astype(bool)
    assert np.array_equal(pb.freedofs, np.nonzero(mask)[0])
    assert pb.freedofs.size == int(GOLD[name + "/nfree"][0])
    f_free = np.zeros(pb.freedofs.size)      # str.f is stored on the free dofs
    f_free[GOLD[name + "/f_idx"]] = GOLD[name + "/f_val"]
    assert np.array_equal(pb.f, f_free)                       # bit-exact
    if fix is not None:
        assert np.array_equal(pb.fixed_dens, GOLD[name + "/fixedDens"])
        assert np.array_equal(pb.fixed_dens_val, GOLD[name + "/fixedDensVal"])


def test_synthetic_workloads():
    cb = P.cantilever(48, 24, 24)
    assert cb.f.sum() == pytest.approx(-1.0)
    assert cb.freedofs.size == 3 * cb.nnodes - 3 * 25 * 25
    br = P.bridge(16, 8, 4)
    assert br.f.sum() == pytest.approx(-1.0)
    to = P.torsion(8, 4, 4)
    assert abs(to.f.sum()) < 1e-12


def test_empty_and_ragged_edge_cases():
    # a support box that rounds to a single node layer and a zero-length line load
    pb = P.build(3, 2, 1, [[0, 0.4, 0, 0, 0, 0, 1, 1, 1]], [[3, 3, 2, 2, 0, 0, 0, 0, 0]])
    assert pb.freedofs.size == 3 * pb.nnodes - 3
    assert not pb.f.any()
