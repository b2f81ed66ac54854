"""zhfmm2d / zh2devaldirect on the GPU against the CPU oracle.

The FMM must match the oracle's FMM (the reference algorithm restated) to
10*eps relative L2 for pot and grad; the direct sum is FP64 pair arithmetic
including H0/H1 of complex argument: 1e-12 relative (the Hankel functions are
accurate to ~2.5e-14 relative, summed over thousands of pairs)."""
import json
import os

import numpy as np
import pytest

import oracle_lib as O
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
G = json.load(open(os.path.join(GOLD, "golden.json")))
EPS12 = float(np.float32(1e-12))


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def run_gpu(eps, zk, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    import zfmm_b200
    zs = w["zsrc"]
    zt = zs if zt is None else zt
    return zfmm_b200.zhfmm2d(eps, zk, zs.shape[1], zs, ifc, w["charge"], ifd, w["dipstr"],
                             w["dipvec"], zt.shape[1], zt, ifpgh, isep)


def run_oracle(eps, zk, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    zs = w["zsrc"].T
    zt = zs if zt is None else zt.T
    p, g = O.zhfmm2d(eps, zk, zs, w["charge"] if ifc else None, w["dipstr"] if ifd else None,
                     w["dipvec"].T if ifd else None, zt, ifpgh=ifpgh, isep=isep)
    return p, g.T


def test_direct_matches_oracle():
    import zfmm_b200
    w = W.curve2d(3000, seed=4)
    t = W.curve2d(700, seed=5)["zsrc"]
    for zk in [40 + 0.5j, 3 * np.pi, 0.3 + 2j]:
        for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1), (0, 1, 2)]:
            pd, gd = zfmm_b200.zh2devaldirect(zk, 700, t, 3000, w["zsrc"], w["charge"],
                                              w["dipstr"], w["dipvec"], ifc, ifd, ifpgh)
            po, go = O.zh2ddirect(zk, w["zsrc"].T, w["charge"] if ifc else None,
                                  w["dipstr"] if ifd else None, w["dipvec"].T if ifd else None,
                                  ztarg=t.T, ifpgh=ifpgh)
            assert rel(pd, po) < 1e-12, (zk, ifc, ifd)
            if ifpgh == 2:
                assert rel(gd, go.T) < 1e-12, (zk, ifc, ifd)


def test_direct_golden_first12():
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture2d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    pd, _ = zfmm_b200.zh2devaldirect(3 * np.pi, 12, z[:, :12], n, z, q, None, None, 1, 0, 1)
    for p, (re, im) in zip(pd, G["2d_helmholtz"]["pot0"]):
        for a, b in [(p.real, re), (p.imag, im)]:
            e = np.floor(np.log10(abs(b))) + 1
            assert abs(a - b) <= 0.5e-5 * 10.0 ** e * 1.0001


@pytest.mark.parametrize("eps", [1e-6, 1e-9, 1e-12])
def test_fmm_matches_oracle_curve(eps):
    w = W.curve2d(20000, seed=1)
    zk = 40 + 0.5j
    p, g = run_gpu(eps, zk, w)
    po, go = run_oracle(eps, zk, w)
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps


def test_fmm_fixture_reference_case():
    """The reference's Helmholtz test: fixture, zk = 3 pi, eps = 1E-12, charges, pot."""
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture2d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    p, _ = zfmm_b200.zhfmm2d(EPS12, 3 * np.pi, n, z, 1, q, 0, None, None, n, z, 1, 1)
    po, _ = O.zhfmm2d(EPS12, 3 * np.pi, z.T, q)
    assert rel(p, po) < 1e-11


def test_fmm_flags_targets_and_zk():
    w = W.clustered2d(5000, seed=7)
    t = W.lap2d_uniform(2000, seed=8)["zsrc"]
    for zk, ifc, ifd, ifpgh in [(10 + 1j, 1, 0, 1), (2 + 0.1j, 0, 1, 2), (25.0, 1, 1, 2)]:
        p, g = run_gpu(1e-9, zk, w, ifc, ifd, ifpgh, zt=t)
        po, go = run_oracle(1e-9, zk, w, ifc, ifd, ifpgh, zt=t)
        assert rel(p, po) < 1e-8, (zk, ifc, ifd)
        if ifpgh == 2:
            assert rel(g, go) < 1e-8, (zk, ifc, ifd)
