"""tosp_kelem_prod_noalloc: the allocation-free KelemProd.

Callers that cannot allocate device memory when they need the product (a
host whose GPU memory belongs to its own pooling allocator, such as a MATLAB
gpuArray session, or a pipeline with work in flight on several streams that
a cudaMalloc/cudaFree would synchronise) use this entry point; its scratch is
a fixed array inside the library, shared by every call.

The test checks it against tosp_kelem_prod, call after call.  Between two
calls on one handle it calls the entry point on a second handle whose fixed
dofs differ (a bridge instead of a cantilever on the same mesh), which leaves
non-zero values in the shared array where the first handle's fixed dofs are;
the next call on the first handle must clear them.  A problem above the
scratch limit is refused with a clear error.  Kept in a file of its own that
pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from tosp import problems as P

pytestmark = pytest.mark.gpu


def _noalloc(tosp_mod, s, x):
    torch = pytest.importorskip("torch")
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    yd = torch.full_like(xd, float("nan"))
    rc = tosp_mod._lib.tosp_kelem_prod_noalloc(s.h, xd.data_ptr(), yd.data_ptr(), C.c_int64(x.size))
    assert rc == 0, tosp_mod._lib.tosp_last_error(s.h).decode()
    return yd.cpu().numpy()


def test_noalloc_matches_kelem_prod_across_calls_and_handles(tosp_mod):
    n = 2
    pa, pb = P.cantilever(16, 8, 8), P.bridge(16, 8, 8)
    assert 3 * pa.nnodes == 3 * pb.nnodes
    assert not np.array_equal(pa.freedofs, pb.freedofs)
    mg = tosp_mod.default_mg(ngrids=3, cycle=0, omega=0.6)
    rng = np.random.default_rng(11)
    sa = tosp_mod.Solver(pa, mg, mr_n=n, p=3.0, emin=1e-9, rmin=1.0)
    sb = tosp_mod.Solver(pb, mg, mr_n=n, p=3.0, emin=1e-9, rmin=1.0)
    sa.SetupGMG(rng.uniform(0.001, 1.0, pa.nelem * n ** 3))
    sb.SetupGMG(rng.uniform(0.001, 1.0, pb.nelem * n ** 3))
    for call, (s, pr) in enumerate([(sa, pa), (sb, pb), (sa, pa)]):
        x = rng.standard_normal(pr.freedofs.size)
        y_ref = s.KelemProd(x)                                   # existing entry point
        y = _noalloc(tosp_mod, s, x)
        # same kernel; only the order of the atomic additions can differ
        assert np.abs(y - y_ref).max() <= 1e-13 * np.abs(y_ref).max(), call
    sa.close()
    sb.close()


def test_noalloc_rejects_problems_above_the_limit(tosp_mod):
    torch = pytest.importorskip("torch")
    pb = P.cantilever(72, 72, 72)                                 # 1,167,051 dofs > 1,048,576
    s = tosp_mod.Solver(pb, tosp_mod.default_mg(ngrids=3), mr_n=1)
    xd = torch.zeros(pb.freedofs.size, dtype=torch.float64, device="cuda")
    yd = torch.zeros_like(xd)
    rc = tosp_mod._lib.tosp_kelem_prod_noalloc(s.h, xd.data_ptr(), yd.data_ptr(), C.c_int64(xd.numel()))
    assert rc == -1
    assert "limit" in tosp_mod._lib.tosp_last_error(s.h).decode()
    s.close()
