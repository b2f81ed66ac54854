"""Plan solves of many right-hand sides in 2D Helmholtz (Plan2D.zhfmm2d with
nd >= 2): the upward and downward passes run per right-hand side, the M2L of
groups of up to 64 right-hand sides at once, on the tcgen05 tensor cores
(TF32 three-term split, FP32 accumulation) when eps >= 1e-7 and in FP64
below.  Every right-hand side must match the single zhfmm2d call (FP64
throughout) to 10 eps at eps = 1e-6, and to rounding on the FP64 path; the
single calls themselves match the oracle (test_gpu_helm2d.py)."""
import numpy as np
import pytest

from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def cn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("eps,nd,tol", [(1e-6, 20, 1e-5), (1e-6, 70, 1e-5), (1e-9, 9, 1e-13)])
def test_batched_rhs_match_single_solves(eps, nd, tol):
    import zfmm_b200
    w = W.curve2d(30000, seed=31)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(7)
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    zk = 40 + 0.5j
    plan = zfmm_b200.Plan2D(eps, n, zs, n, zs)
    p, g = plan.zhfmm2d(zk, nd, 1, q, 1, ds, w["dipvec"], 2)
    for r in sorted({0, 1, nd // 2, nd - 1}):
        p1, g1 = zfmm_b200.zhfmm2d(eps, zk, n, zs, 1, q[r], 1, ds[r], w["dipvec"], n, zs, 2, 1)
        assert rel(p[r], p1) < tol, (r, rel(p[r], p1))
        assert rel(g[r], g1) < tol, (r, rel(g[r], g1))
    plan.close()


def test_batched_rhs_charges_only_and_two_wavenumbers():
    import zfmm_b200
    eps = 1e-6
    w = W.curve2d(12000, seed=33)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(8)
    nd = 16
    q = cn(rng, nd, n)
    plan = zfmm_b200.Plan2D(eps, n, zs, n, zs)
    for zk in (40 + 0.5j, 15 + 0.2j):
        p, _ = plan.zhfmm2d(zk, nd, 1, q, 0, None, None, 1)
        for r in (0, nd - 1):
            p1, _ = zfmm_b200.zhfmm2d(eps, zk, n, zs, 1, q[r], 0, None, None, n, zs, 1, 1)
            assert rel(p[r], p1) < 1e-5, (zk, r)
    plan.close()
