"""3D plans: one geometry, many right-hand sides (zfmm_plan3d_*, Plan3D).

A plan solve runs the same algorithm on the same tree as the single-solve
zlfmm3d, with each right-hand side's expansions formed and translated by the
batched kernels; right-hand side by right-hand side it must match the single
solve (itself pinned to the oracle) to 10*eps relative L2, the parity bar of
the FMMs.  One small case goes straight against the oracle.  The cases cover
one and many right-hand sides (a ragged last pass of 32), charges and dipoles,
ifpgh 1 and 2, adaptive trees with lists 3 and 4, plan reuse, and the device
(torch) entry point.  Fewer than 4 right-hand sides, or orders whose batched
working set exceeds shared memory (eps below ~3e-10), run the single-solve
passes per right-hand side on the plan's tree.  Helmholtz plan solves with 4
or more right-hand sides batch the translations (P2M, P2L, P2P and the
evaluations run per right-hand side) and must match the single zhfmm3d solves
to 10*eps; with fewer they run the single-solve passes on the plan's tree and
equal the single solves to rounding."""
import numpy as np
import pytest

import oracle_lib as O
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def single(eps, zs, q, ifd, ds, dv, ifpgh):
    import zfmm_b200
    n = zs.shape[1]
    return zfmm_b200.zlfmm3d(eps, n, zs, 1 if q is not None else 0, q, ifd, ds, dv, n, zs,
                             ifpgh, 1)


def cn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_plan_one_rhs_matches_single():
    import zfmm_b200
    eps = 1e-9
    w = W.lap3d_uniform(20000, seed=11)
    zs = w["zsrc"]
    plan = zfmm_b200.Plan3D(eps, zs.shape[1], zs, zs.shape[1], zs)
    nb, nl = plan.info()
    assert nb > 1 and nl >= 2
    p, g = plan.zlfmm3d(1, 1, w["charge"][None, :], 1, w["dipstr"][None, :], w["dipvec"], 2)
    p1, g1 = single(eps, zs, w["charge"], 1, w["dipstr"], w["dipvec"], 2)
    assert rel(p[0], p1) < 10 * eps
    assert rel(g[0], g1) < 10 * eps
    plan.close()


def test_plan_many_rhs_columns():
    import zfmm_b200
    eps = 1e-9
    nd = 40  # one full pass of 32 and a ragged one
    w = W.lap3d_uniform(12000, seed=12, nrhs=nd)
    zs = w["zsrc"]
    n = zs.shape[1]
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zlfmm3d(nd, 1, w["charge"], 0, None, None, 2)
    assert p.shape == (nd, n) and g.shape == (nd, 3, n)
    for r in [0, 17, 31, 32, 39]:
        p1, g1 = single(eps, zs, w["charge"][r], 0, None, None, 2)
        assert rel(p[r], p1) < 10 * eps, r
        assert rel(g[r], g1) < 10 * eps, r


def test_plan_dipoles_adaptive_tree():
    import zfmm_b200
    eps = 1e-9
    w = W.clustered3d(9000, seed=13)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(5)
    nd = 5
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    for ifc, ifd, ifpgh in [(1, 1, 2), (0, 1, 1), (1, 0, 2)]:
        p, g = plan.zlfmm3d(nd, ifc, q, ifd, ds, w["dipvec"], ifpgh)
        for r in range(nd):
            p1, g1 = single(eps, zs, q[r] if ifc else None, ifd, ds[r], w["dipvec"], ifpgh)
            assert rel(p[r], p1) < 10 * eps, (ifc, ifd, r)
            if ifpgh == 2:
                assert rel(g[r], g1) < 10 * eps, (ifc, ifd, r)
            else:
                assert not np.any(g[r])


def test_plan_against_oracle():
    import zfmm_b200
    eps = 1e-6
    w = W.clustered3d(3000, seed=14)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(6)
    nd = 4
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zlfmm3d(nd, 1, q, 1, ds, w["dipvec"], 2)
    for r in range(nd):
        po, go = O.zlfmm3d(eps, zs.T, q[r], ds[r], w["dipvec"].T, zs.T, ifpgh=2)
        assert rel(p[r], po) < 10 * eps, r
        assert rel(g[r], go.T) < 10 * eps, r


def test_plan_reuse_and_separate_targets():
    import zfmm_b200
    eps = 1e-9
    w = W.lap3d_uniform(8000, seed=15)
    t = W.lap3d_uniform(3000, seed=16)["zsrc"]
    zs = w["zsrc"]
    rng = np.random.default_rng(7)
    plan = zfmm_b200.Plan3D(eps, zs.shape[1], zs, t.shape[1], t)
    for k in range(2):
        q = cn(rng, 2, zs.shape[1])
        p, g = plan.zlfmm3d(2, 1, q, 0, None, None, 2)
        for r in range(2):
            p1, g1 = zfmm_b200.zlfmm3d(eps, zs.shape[1], zs, 1, q[r], 0, None, None, t.shape[1],
                                       t, 2, 1)
            assert rel(p[r], p1) < 10 * eps, (k, r)
            assert rel(g[r], g1) < 10 * eps, (k, r)


def test_plan_device_entry_point():
    import torch
    import zfmm_b200
    eps = 1e-9
    nd = 5
    w = W.lap3d_uniform(10000, seed=17, nrhs=nd)
    zs = w["zsrc"]
    n = zs.shape[1]
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zlfmm3d(nd, 1, w["charge"], 0, None, None, 2)
    zt = torch.from_numpy(np.ascontiguousarray(zs.T)).cuda()
    qt = torch.from_numpy(np.ascontiguousarray(w["charge"].T)).cuda()  # (n, nd)
    plan_t = zfmm_b200.Plan3D(eps, n, zt, n, zt)
    pt, gt = plan_t.zlfmm3d(nd, 1, qt, 0, None, None, 2)
    torch.cuda.synchronize()
    assert tuple(pt.shape) == (nd, n) and tuple(gt.shape) == (nd, 3, n)
    assert rel(pt.cpu().numpy(), p) < 1e-13
    assert rel(gt.cpu().numpy(), g) < 1e-13


def test_helmholtz_plan_matches_single_two_wavenumbers():
    import zfmm_b200
    eps = 1e-9
    w = W.sphere3d(15000, seed=18)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(8)
    nd = 3
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    for zk in (10 + 0.2j, 4 - 0.1j):
        for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1)]:
            p, g = plan.zhfmm3d(zk, nd, ifc, q, ifd, ds, w["dipvec"], ifpgh)
            for r in range(nd):
                p1, g1 = zfmm_b200.zhfmm3d(eps, zk, n, zs, ifc, q[r], ifd, ds[r], w["dipvec"],
                                           n, zs, ifpgh, 1)
                assert rel(p[r], p1) < 1e-13, (zk, ifc, ifd, r)
                if ifpgh == 2:
                    assert rel(g[r], g1) < 1e-13, (zk, ifc, ifd, r)


def test_plan_small_eps_runs_per_rhs():
    import zfmm_b200
    eps = 1e-11  # order 46: beyond the batched translation's shared memory
    nd = 6
    w = W.clustered3d(6000, seed=19)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(9)
    q = cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zlfmm3d(nd, 1, q, 0, None, None, 2)
    for r in (0, nd - 1):
        p1, g1 = single(eps, zs, q[r], 0, None, None, 2)
        assert rel(p[r], p1) < 1e-13, r
        assert rel(g[r], g1) < 1e-13, r


def hsingle(eps, zk, zs, q, ifd, ds, dv, ifpgh, zt=None):
    import zfmm_b200
    n = zs.shape[1]
    zt = zs if zt is None else zt
    return zfmm_b200.zhfmm3d(eps, zk, n, zs, 1 if q is not None else 0, q, ifd, ds, dv,
                             zt.shape[1], zt, ifpgh, 1)


def test_helmholtz_batched_matches_single():
    # 4 or more right-hand sides: the batched translations (one ragged pass of 32)
    import zfmm_b200
    eps = 1e-9
    w = W.sphere3d(15000, seed=21)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(21)
    nd = 37
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    zk = 10 + 0.2j
    p, g = plan.zhfmm3d(zk, nd, 1, q, 1, ds, w["dipvec"], 2)
    assert p.shape == (nd, n) and g.shape == (nd, 3, n)
    for r in [0, 13, 31, 32, 36]:
        p1, g1 = hsingle(eps, zk, zs, q[r], 1, ds[r], w["dipvec"], 2)
        assert rel(p[r], p1) < 10 * eps, r
        assert rel(g[r], g1) < 10 * eps, r


def test_helmholtz_batched_adaptive_kinds():
    # adaptive tree (lists 3 and 4), charges only / dipoles only, ifpgh 1 and 2,
    # two wavenumbers on one plan
    import zfmm_b200
    eps = 1e-8
    w = W.clustered3d(9000, seed=22)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(22)
    nd = 6
    q, ds = cn(rng, nd, n), cn(rng, nd, n)
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    for zk in (6 + 0.1j, 2.5 - 0.05j):
        for ifc, ifd, ifpgh in [(1, 0, 2), (0, 1, 1)]:
            p, g = plan.zhfmm3d(zk, nd, ifc, q, ifd, ds, w["dipvec"], ifpgh)
            for r in (0, nd - 1):
                p1, g1 = hsingle(eps, zk, zs, q[r] if ifc else None, ifd, ds[r], w["dipvec"],
                                 ifpgh)
                assert rel(p[r], p1) < 10 * eps, (zk, ifc, ifd, r)
                if ifpgh == 2:
                    assert rel(g[r], g1) < 10 * eps, (zk, ifc, ifd, r)


def test_helmholtz_batched_separate_targets_and_oracle():
    import zfmm_b200
    eps = 1e-6
    w = W.clustered3d(2500, seed=23)
    zs = w["zsrc"]
    t = W.clustered3d(900, seed=24)["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(23)
    nd = 4
    q = cn(rng, nd, n)
    zk = 3 + 0.1j
    plan = zfmm_b200.Plan3D(eps, n, zs, t.shape[1], t)
    p, g = plan.zhfmm3d(zk, nd, 1, q, 0, None, None, 2)
    for r in range(nd):
        po, go = O.zhfmm3d(eps, zk, zs.T, q[r], None, None, t.T, ifpgh=2)
        assert rel(p[r], po) < 10 * eps, r
        assert rel(g[r], go.T) < 10 * eps, r


def test_helmholtz_batched_device_entry_point():
    import torch
    import zfmm_b200
    eps = 1e-9
    nd = 5
    w = W.sphere3d(8000, seed=25)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(25)
    q = cn(rng, nd, n)
    zk = 8 + 0.1j
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zhfmm3d(zk, nd, 1, q, 0, None, None, 2)
    zt = torch.from_numpy(np.ascontiguousarray(zs.T)).cuda()
    qt = torch.from_numpy(np.ascontiguousarray(q.T)).cuda()
    plan_t = zfmm_b200.Plan3D(eps, n, zt, n, zt)
    pt, gt = plan_t.zhfmm3d(zk, nd, 1, qt, 0, None, None, 2)
    torch.cuda.synchronize()
    assert rel(pt.cpu().numpy(), p) < 1e-13
    assert rel(gt.cpu().numpy(), g) < 1e-13


def test_helmholtz_plan_small_eps_runs_per_rhs():
    # orders above the batched kernels' shared memory (p > 40): every pass per
    # right-hand side on the plan's tree, equal to the single solves to rounding
    import zfmm_b200
    eps = 1e-12
    nd = 5
    w = W.sphere3d(4000, seed=26)
    zs = w["zsrc"]
    n = zs.shape[1]
    rng = np.random.default_rng(26)
    q = cn(rng, nd, n)
    zk = 10 + 0.2j
    # level-2 boxes of the unit sphere's tree: a quarter of the ~2.2 root box
    assert zfmm_b200.h3dterms(0.25, zk * 2.2, eps) > 40
    plan = zfmm_b200.Plan3D(eps, n, zs, n, zs)
    p, g = plan.zhfmm3d(zk, nd, 1, q, 0, None, None, 2)
    for r in (0, nd - 1):
        p1, g1 = hsingle(eps, zk, zs, q[r], 0, None, None, 2)
        assert rel(p[r], p1) < 1e-13, r
        assert rel(g[r], g1) < 1e-13, r
