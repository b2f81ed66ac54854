"""zhfmm3d / zh3devaldirect on the GPU against the CPU oracle.

The FMM must match the oracle's FMM (the reference algorithm restated) to
10*eps relative L2 for pot and grad: uniform points (complete octree),
deeper adaptive trees (lists 3 and 4), points on a complex-displaced sphere,
and the reference's own test geometry (eps = 1e-12, zk = pi, expansion orders
large enough to need the global-memory translation workspace) where the
first 12 potentials of its log are reproduced; the direct sum is FP64 pair
arithmetic: 1e-13 relative."""
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


def close5(a, b):
    e = np.floor(np.log10(abs(b))) + 1
    return abs(a - b) <= 0.5e-5 * 10.0 ** e * 1.0001


def run_gpu(eps, zk, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    import zfmm_b200
    zs = w["zsrc"]
    zt = zs if zt is None else zt
    return zfmm_b200.zhfmm3d(eps, zk, zs.shape[1], zs, ifc, w["charge"], ifd, w["dipstr"],
                             w["dipvec"], zt.shape[1], zt, ifpgh, isep)


def run_oracle(eps, zk, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    zs = w["zsrc"].T
    zt = zs if zt is None else zt.T
    p, g = O.zhfmm3d(eps, zk, zs, w["charge"] if ifc else None, w["dipstr"] if ifd else None,
                     w["dipvec"].T if ifd else None, zt, ifpgh=ifpgh, isep=isep)
    return p, g.T


def test_direct_matches_oracle():
    import zfmm_b200
    w = W.sphere3d(3000, seed=4)
    t = W.lap3d_uniform(700, seed=5)["zsrc"]
    for zk in [10 + 0.2j, np.pi, 0.5 + 2j]:
        for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1), (0, 1, 2)]:
            pd, gd = zfmm_b200.zh3devaldirect(zk, 700, t, 3000, w["zsrc"], w["charge"],
                                              w["dipstr"], w["dipvec"], ifc, ifd, ifpgh)
            po, go = O.zh3ddirect(zk, w["zsrc"].T, w["charge"] if ifc else None,
                                  w["dipstr"] if ifd else None, w["dipvec"].T if ifd else None,
                                  ztarg=t.T, ifpgh=ifpgh)
            assert rel(pd, po) < 1e-13, (zk, ifc, ifd)
            if ifpgh == 2:
                assert rel(gd, go.T) < 1e-13, (zk, ifc, ifd)


def test_direct_golden_first12():
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture3d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    pd, _ = zfmm_b200.zh3devaldirect(np.pi, 12, z[:, :12], n, z, q, None, None, 1, 0, 1)
    for p, (re, im) in zip(pd, G["3d_helmholtz"]["pot0"]):
        assert close5(p.real, re) and close5(p.imag, im)


@pytest.mark.parametrize("eps,zk", [(1e-3, 10 + 0.2j), (1e-6, 10 + 0.2j), (1e-9, 5 + 0.1j)])
def test_fmm_matches_oracle_uniform(eps, zk):
    w = W.lap3d_uniform(20000 if eps > 1e-9 else 12000, seed=1, amp=0.01)
    p, g = run_gpu(eps, zk, w)
    po, go = run_oracle(eps, zk, w)
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps


def test_fmm_matches_oracle_sphere():
    w = W.sphere3d(20000, seed=2)
    p, g = run_gpu(1e-6, 10 + 0.2j, w)
    po, go = run_oracle(1e-6, 10 + 0.2j, w)
    assert rel(p, po) < 1e-5
    assert rel(g, go) < 1e-5


def test_fmm_flags_and_separate_targets():
    w = W.clustered3d(8000, seed=3)
    zt = W.lap3d_uniform(3000, seed=7, amp=0.01)["zsrc"] * 0.8
    for ifc, ifd, ifpgh in [(1, 0, 1), (0, 1, 2), (1, 1, 1)]:
        p, g = run_gpu(1e-6, 3 + 0.1j, w, ifc, ifd, ifpgh, zt=zt)
        po, go = run_oracle(1e-6, 3 + 0.1j, w, ifc, ifd, ifpgh, zt=zt)
        assert rel(p, po) < 1e-5, (ifc, ifd, ifpgh)
        if ifpgh == 2:
            assert rel(g, go) < 1e-5
        else:
            assert not np.any(g)


def test_fmm_vs_direct_subset():
    import zfmm_b200
    w = W.sphere3d(30000, seed=9)
    zk = 10 + 0.2j
    p, g = run_gpu(1e-9, zk, w)
    idx = np.random.default_rng(0).choice(30000, 400, replace=False)
    pd, gd = zfmm_b200.zh3devaldirect(zk, 400, w["zsrc"][:, idx], 30000, w["zsrc"], w["charge"],
                                      w["dipstr"], w["dipvec"], 1, 1, 2)
    assert rel(p[idx], pd) < 1e-7
    assert rel(g[:, idx], gd) < 1e-7


def test_torch_device_path():
    import torch
    import zfmm_b200
    w = W.sphere3d(20000, seed=11)
    d = torch.device("cuda:0")
    zs = torch.from_numpy(np.ascontiguousarray(w["zsrc"].T)).to(d)
    q = torch.from_numpy(w["charge"]).to(d)
    p, g = zfmm_b200.zhfmm3d(1e-6, 10 + 0.2j, 20000, zs, 1, q, 0, None, None, 20000, zs, 2)
    ph, gh = run_gpu(1e-6, 10 + 0.2j, w, ifd=0)
    assert rel(p.cpu().numpy(), ph) < 1e-14
    assert rel(g.cpu().numpy(), gh) < 1e-14


def test_fmm_fixture_reference_case():
    """The reference's own 3D Helmholtz test: zk = pi, eps = 1e-12, charges,
    pot only (a box ~25 wavelengths wide: orders up to ~70, run on the
    global-memory translation workspace).  At this size the FMM result is
    rounding-limited near 2.5e-9: the oracle compiled with and without
    fused multiply-adds differs from itself by 7e-10, and the reference's log
    and the oracle differ at the same level.  So the checks are the
    reference's own: the first 12 potentials of its log, its error metric
    err / (|pot0| + |q|) (8.8576e-10 in the log) within a factor 3, and
    agreement with the oracle's FMM at that accuracy."""
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture3d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    p, _ = zfmm_b200.zhfmm3d(EPS12, np.pi, n, z, 1, q, 0, None, None, n, z, 1)
    for a, (re, im) in zip(p[:12], G["3d_helmholtz"]["pot"]):
        assert close5(a.real, re) and close5(a.imag, im)
    pd, _ = zfmm_b200.zh3devaldirect(np.pi, n, z, n, z, q, None, None, 1, 0, 1)
    assert close5(np.linalg.norm(pd), G["3d_helmholtz"]["pot0_norm"][0])
    err = np.linalg.norm(p - pd) / (np.linalg.norm(pd) + np.linalg.norm(q))
    assert err < 3 * 8.8576e-10
    po, _ = O.zhfmm3d(EPS12, np.pi, z.T, q, ifpgh=1)
    assert rel(p, po) < 1e-8
