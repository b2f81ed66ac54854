"""2D plans (zfmm_plan2d_*, Plan2D): one quadtree reused by solves of several
right-hand sides and wavenumbers (the two-wavenumber matvecs of a
transmission-problem GMRES).  Every right-hand side runs the single-solve
passes on the plan's tree, so each column must equal the single zlfmm2d /
zhfmm2d call on the same points to rounding."""
import numpy as np
import pytest

from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def cn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_helmholtz_plan_two_wavenumbers():
    import zfmm_b200
    eps = 1e-9
    w = W.curve2d(20000, seed=21)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(3)
    nd = 3
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan2D(eps, n, zs, n, zs)
    nb, nl = plan.info()
    assert nb > 1 and nl >= 2
    for zk in (40 + 0.5j, 20 + 0.3j):
        for ifc, ifd, ifpgh in [(1, 1, 2), (0, 1, 1)]:
            p, g = plan.zhfmm2d(zk, nd, ifc, q, ifd, ds, w["dipvec"], ifpgh)
            assert p.shape == (nd, n) and g.shape == (nd, 2, n)
            for r in range(nd):
                p1, g1 = zfmm_b200.zhfmm2d(eps, zk, n, zs, ifc, q[r], ifd, ds[r], w["dipvec"], n,
                                           zs, ifpgh, 1)
                assert rel(p[r], p1) < 1e-13, (zk, ifc, r)
                if ifpgh == 2:
                    assert rel(g[r], g1) < 1e-13, (zk, ifc, r)
    plan.close()


def test_laplace_plan_separate_targets_and_torch():
    import torch
    import zfmm_b200
    eps = 1e-9
    w = W.lap2d_uniform(12000, seed=22)
    t = W.lap2d_uniform(5000, seed=23)["zsrc"]
    zs = w["zsrc"]
    n, nt = zs.shape[1], t.shape[1]
    rng = np.random.default_rng(4)
    nd = 2
    q = cn(rng, nd, n)
    plan = zfmm_b200.Plan2D(eps, n, zs, nt, t)
    p, g = plan.zlfmm2d(nd, 1, q, 0, None, None, 2)
    for r in range(nd):
        p1, g1 = zfmm_b200.zlfmm2d(eps, n, zs, 1, q[r], 0, None, None, nt, t, 2, 1)
        assert rel(p[r], p1) < 1e-13, r
        assert rel(g[r], g1) < 1e-13, r
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    plan_t = zfmm_b200.Plan2D(eps, n, T(zs.T), nt, T(t.T))
    pt, gt = plan_t.zlfmm2d(nd, 1, T(q.T), 0, None, None, 2)
    torch.cuda.synchronize()
    assert rel(pt.cpu().numpy(), p) < 1e-13
    assert rel(gt.cpu().numpy(), g) < 1e-13
