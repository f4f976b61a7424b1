"""tosp_kelem_prod_noalloc: the allocation-free KelemProd.

Callers that cannot allocate device memory when they need the product (a
stream capture in progress, a host that pools the GPU memory itself, or a
multi-stream pipeline that cudaMalloc would synchronise) use this entry point;
its scratch is a fixed array inside the library.  The test checks it against
tosp_kelem_prod on two calls in a row (the array keeps the previous call's
contents, so the second call shows that what must start at zero is cleared),
and that a problem above the scratch limit is refused with a clear error.
Kept in a file of its own that pytest collects last.
"""
import numpy as np
import pytest

from tosp import problems as P

pytestmark = pytest.mark.gpu


def test_noalloc_matches_kelem_prod_twice(tosp_mod):
    torch = pytest.importorskip("torch")
    import ctypes as C
    pb = P.cantilever(16, 8, 8)
    n = 2
    dens = np.random.default_rng(5).uniform(0.001, 1.0, pb.nelem * n ** 3)
    s = tosp_mod.Solver(pb, tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6), mr_n=n, p=3.0, emin=1e-9, rmin=1.0)
    s.SetupGMG(dens)
    rng = np.random.default_rng(11)
    for call in range(2):
        x = rng.standard_normal(pb.freedofs.size)
        y_ref = s.KelemProd(x)                                   # existing entry point
        xd = torch.tensor(x, dtype=torch.float64, device="cuda")
        yd = torch.full_like(xd, float("nan"))
        rc = tosp_mod._lib.tosp_kelem_prod_noalloc(s.h, xd.data_ptr(), yd.data_ptr(), C.c_int64(x.size))
        assert rc == 0, tosp_mod._lib.tosp_last_error(s.h).decode()
        y = yd.cpu().numpy()
        # same kernel; only the order of the atomic additions can differ
        assert np.abs(y - y_ref).max() <= 1e-13 * np.abs(y_ref).max(), call
    s.close()


def test_noalloc_rejects_problems_above_the_limit(tosp_mod):
    torch = pytest.importorskip("torch")
    import ctypes as C
    pb = P.cantilever(72, 72, 72)                                 # 1,167,051 dofs > 1,048,576
    s = tosp_mod.Solver(pb, tosp_mod.default_mg(ngrids=3), mr_n=1)
    xd = torch.zeros(pb.freedofs.size, dtype=torch.float64, device="cuda")
    yd = torch.zeros_like(xd)
    rc = tosp_mod._lib.tosp_kelem_prod_noalloc(s.h, xd.data_ptr(), yd.data_ptr(), C.c_int64(xd.numel()))
    assert rc == -1
    assert "limit" in tosp_mod._lib.tosp_last_error(s.h).decode()
    s.close()
