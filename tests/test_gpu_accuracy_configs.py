"""The stated configurations at their stated accuracy, against the oracle and
the FP64 direct sum.

1. zhfmm3d on the many-instance configuration's geometry (points on the unit
   sphere displaced by 0.1i times the normal scaled by a degree-4 field,
   zk = 10+0.2i, charges and dipoles, pot + grad) at eps = 1e-9: the device
   FMM matches the oracle (the reference algorithm restated) to 10 eps.
2. Attribution of the distance to the direct sum.  On the batched 3D Laplace
   configuration's geometry (uniform cube, imaginary parts 0.05 sin(2 pi .))
   and on the sphere above, the reference algorithm itself misses the FP64
   direct sum by more than eps (expansions about complex box centres; the
   zylgndrf branch of zl3devalloc / zh3devalloc).  The tests measure the
   oracle's error and the device FMM's error against the direct sum on the
   same seeded subset of targets and require them to be equal to 1e-8: the
   device reproduces the reference algorithm's error, it does not add one.
"""
import numpy as np
import pytest

import oracle_lib as O
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def subset(n, m, seed):
    return np.sort(np.random.default_rng(seed).choice(n, m, replace=False))


def test_zhfmm3d_sphere_eps1e9_matches_oracle_and_attribution():
    import zfmm_b200
    eps, zk = 1e-9, 10 + 0.2j
    w = W.sphere3d(20000, seed=41)
    zs = w["zsrc"]
    n = zs.shape[1]
    p, g = zfmm_b200.zhfmm3d(eps, zk, n, zs, 1, w["charge"], 1, w["dipstr"], w["dipvec"], n, zs,
                             2, 1)
    po, go = O.zhfmm3d(eps, zk, zs.T, w["charge"], w["dipstr"], w["dipvec"].T, ifpgh=2)
    go = go.T
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps
    # FP64 direct sum on 2,000 seeded targets (self term excluded as in the FMM)
    idx = subset(n, 2000, 5)
    pd, gd = O.zh3ddirect(zk, zs.T, w["charge"], w["dipstr"], w["dipvec"].T, ztarg=zs.T[idx],
                          ifpgh=2)
    e_dev, e_or = rel(p[idx], pd), rel(po[idx], pd)
    assert abs(e_dev - e_or) < 1e-8, (e_dev, e_or)
    assert abs(rel(g[:, idx], gd.T) - rel(go[:, idx], gd.T)) < 1e-8


def test_zlfmm3d_batched_geometry_attribution():
    import zfmm_b200
    eps = 1e-9
    w = W.lap3d_uniform(20000, seed=31)  # imaginary amplitude 0.05 of the batched configuration
    zs = w["zsrc"]
    n = zs.shape[1]
    q = w["charge"][0] if w["charge"].ndim == 2 else w["charge"]
    p, g = zfmm_b200.zlfmm3d(eps, n, zs, 1, q, 0, None, None, n, zs, 2, 1)
    po, go = O.zlfmm3d(eps, zs.T, q, ifpgh=2)
    go = go.T
    idx = subset(n, 2000, 6)
    pd, gd = O.zl3ddirect(zs.T, q, ztarg=zs.T[idx], ifpgh=2)
    e_dev, e_or = rel(p[idx], pd), rel(po[idx], pd)
    assert abs(e_dev - e_or) < 1e-8, (e_dev, e_or)
    assert abs(rel(g[:, idx], gd.T) - rel(go[:, idx], gd.T)) < 1e-8
    # and everywhere the device agrees with the reference algorithm far below
    # that common error
    assert rel(p, po) < 1e-2 * max(e_or, 10 * eps)
