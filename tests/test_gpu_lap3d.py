"""zlfmm3d / zl3devaldirect on the GPU against the CPU oracle.

The FMM must match the oracle's FMM (the reference algorithm restated) to
10*eps relative L2 for pot and grad, on uniform (complete octree) and
clustered (adaptive octree, non-empty lists 3 and 4) inputs, and reproduce the
reference's logged potentials on its own test geometry; the direct sum is FP64
pair arithmetic: 1e-13 relative."""
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


def run_gpu(eps, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    import zfmm_b200
    zs = w["zsrc"]
    zt = zs if zt is None else zt
    return zfmm_b200.zlfmm3d(eps, zs.shape[1], zs, ifc, w["charge"], ifd, w["dipstr"],
                             w["dipvec"], zt.shape[1], zt, ifpgh, isep)


def run_oracle(eps, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    zs = w["zsrc"].T
    zt = zs if zt is None else zt.T
    p, g = O.zlfmm3d(eps, zs, w["charge"] if ifc else None, w["dipstr"] if ifd else None,
                     w["dipvec"].T if ifd else None, zt, ifpgh=ifpgh, isep=isep)
    return p, g.T


def test_direct_matches_oracle():
    import zfmm_b200
    w = W.clustered3d(3000, seed=4)
    t = W.lap3d_uniform(700, seed=5)["zsrc"]
    for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1), (0, 1, 2), (1, 0, 2)]:
        pd, gd = zfmm_b200.zl3devaldirect(700, t, 3000, w["zsrc"], w["charge"], w["dipstr"],
                                          w["dipvec"], ifc, ifd, ifpgh)
        po, go = O.zl3ddirect(w["zsrc"].T, w["charge"] if ifc else None,
                              w["dipstr"] if ifd else None, w["dipvec"].T if ifd else None,
                              ztarg=t.T, ifpgh=ifpgh)
        assert rel(pd, po) < 1e-13, (ifc, ifd)
        if ifpgh == 2:
            assert rel(gd, go.T) < 1e-13, (ifc, ifd)


def test_direct_golden_first12():
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture3d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    pd, _ = zfmm_b200.zl3devaldirect(12, z[:, :12], n, z, q, None, None, 1, 0, 1)
    for p, (re, im) in zip(pd, G["3d_laplace"]["pot0"]):
        assert close5(p.real, re) and close5(p.imag, im)


@pytest.mark.parametrize("eps,n", [(1e-3, 20000), (1e-6, 20000), (1e-9, 12000)])
def test_fmm_matches_oracle_uniform(eps, n):
    w = W.lap3d_uniform(n, seed=1)
    p, g = run_gpu(eps, w)
    po, go = run_oracle(eps, w)
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
def test_fmm_matches_oracle_clustered(eps):
    w = W.clustered3d(20000, seed=2)
    p, g = run_gpu(eps, w)
    po, go = run_oracle(eps, w)
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps


def test_fmm_flags_and_separate_targets():
    w = W.clustered3d(8000, seed=3)
    zt = W.lap3d_uniform(3000, seed=7)["zsrc"] * 0.8
    for ifc, ifd, ifpgh in [(1, 0, 1), (0, 1, 2), (1, 1, 1)]:
        p, g = run_gpu(1e-6, w, ifc, ifd, ifpgh, zt=zt)
        po, go = run_oracle(1e-6, w, ifc, ifd, ifpgh, zt=zt)
        assert rel(p, po) < 1e-5, (ifc, ifd, ifpgh)
        if ifpgh == 2:
            assert rel(g, go) < 1e-5
        else:
            assert not np.any(g)


def test_fmm_isep2():
    w = W.lap3d_uniform(20000, seed=8)
    p, g = run_gpu(1e-3, w, isep=2)
    po, go = run_oracle(1e-3, w, isep=2)
    assert rel(p, po) < 1e-2 and rel(g, go) < 1e-2


def test_fmm_fixture_reference_case():
    """The reference's own 3D Laplace test geometry at eps = 1e-12 (charges,
    pot only): the first 12 potentials of the log and the oracle's FMM."""
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture3d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    p, _ = zfmm_b200.zlfmm3d(EPS12, n, z, 1, q, 0, None, None, n, z, 1)
    po, _ = O.zlfmm3d(EPS12, z.T, q, ifpgh=1)
    assert rel(p, po) < 10 * EPS12
    for a, (re, im) in zip(p[:12], G["3d_laplace"]["pot"]):
        assert close5(a.real, re) and close5(a.imag, im)


def test_fmm_vs_direct_subset():
    """FMM against the FP64 direct sum.  Imaginary amplitude 0.01: from about
    0.02 on (at this density), some targets lie where Re((x-cx)^2 + (y-cy)^2) < 0 about their
    box's complex centre, and the reference's local-expansion evaluation
    (zylgndrf's u = -sqrt(1-ct^2) against zcart2sph's sin(theta)) takes
    opposite square-root branches there; the oracle shows the same ~1e-4
    deviation from the direct sum, and test_fmm_matches_oracle_uniform covers
    that regime for parity."""
    import zfmm_b200
    w = W.lap3d_uniform(30000, seed=9, amp=0.01)
    p, g = run_gpu(1e-9, w, ifd=0)
    idx = np.random.default_rng(0).choice(30000, 500, replace=False)
    pd, gd = zfmm_b200.zl3devaldirect(500, w["zsrc"][:, idx], 30000, w["zsrc"], w["charge"],
                                      None, None, 1, 0, 2)
    assert rel(p[idx], pd) < 1e-8
    assert rel(g[:, idx], gd) < 1e-8


def test_small_and_empty():
    import zfmm_b200
    w = W.lap3d_uniform(50, seed=10)
    p, g = run_gpu(1e-6, w)
    po, go = run_oracle(1e-6, w)
    assert rel(p, po) < 1e-12 and rel(g, go) < 1e-12  # one leaf: direct sums only
    p0, g0 = zfmm_b200.zlfmm3d(1e-6, 50, w["zsrc"], 1, w["charge"], 0, None, None, 0,
                               np.zeros((3, 0), complex), 2)
    assert p0.size == 0


def test_torch_device_path():
    import torch
    import zfmm_b200
    w = W.lap3d_uniform(20000, seed=11)
    d = torch.device("cuda:0")
    zs = torch.from_numpy(np.ascontiguousarray(w["zsrc"].T)).to(d)
    q = torch.from_numpy(w["charge"]).to(d)
    p, g = zfmm_b200.zlfmm3d(1e-6, 20000, zs, 1, q, 0, None, None, 20000, zs, 2)
    ph, gh = run_gpu(1e-6, w, ifd=0)
    assert rel(p.cpu().numpy(), ph) < 1e-14
    assert rel(g.cpu().numpy(), gh) < 1e-14
