"""zlfmm2d / zl2devaldirect on the GPU against the CPU oracle.

Tolerances: the FMM must agree with the oracle's FMM (the reference algorithm
restated) to 10*eps relative L2 over all targets, for pot and for grad, and
with the FP64 direct sum to the accuracy the reference itself reaches.  The
direct sum is pure FP64 pair arithmetic: 1e-13 relative."""
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


def run_gpu(eps, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    import zfmm_b200
    zs = w["zsrc"]
    zt = zs if zt is None else zt
    return zfmm_b200.zlfmm2d(eps, zs.shape[1], zs, ifc, w["charge"], ifd, w["dipstr"],
                             w["dipvec"], zt.shape[1], zt, ifpgh, isep)


def run_oracle(eps, w, ifc=1, ifd=1, ifpgh=2, zt=None, isep=1):
    zs = w["zsrc"].T
    zt = zs if zt is None else zt.T
    p, g = O.zlfmm2d(eps, zs, w["charge"] if ifc else None, w["dipstr"] if ifd else None,
                     w["dipvec"].T if ifd else None, zt, ifpgh=ifpgh, isep=isep)
    return p, g.T


@pytest.mark.parametrize("eps", [1e-6, 1e-9, 1e-12])
def test_fmm_matches_oracle_uniform(eps):
    w = W.lap2d_uniform(20000, seed=1)
    p, g = run_gpu(eps, w)
    po, go = run_oracle(eps, w)
    assert rel(p, po) < 10 * eps
    assert rel(g, go) < 10 * eps


def test_fmm_flags_and_separate_targets():
    w = W.clustered2d(6000, seed=7)
    t = W.lap2d_uniform(3000, seed=8)["zsrc"]
    for ifc, ifd, ifpgh in [(1, 0, 1), (0, 1, 2), (1, 1, 1)]:
        p, g = run_gpu(1e-9, w, ifc, ifd, ifpgh, zt=t)
        po, go = run_oracle(1e-9, w, ifc, ifd, ifpgh, zt=t)
        assert rel(p, po) < 1e-8
        if ifpgh == 2:
            assert rel(g, go) < 1e-8
        else:
            assert not np.any(g)


def test_fmm_isep2():
    w = W.clustered2d(8000, seed=9)
    p, g = run_gpu(1e-9, w, isep=2)
    po, go = run_oracle(1e-9, w, isep=2)
    assert rel(p, po) < 1e-8 and rel(g, go) < 1e-8


def test_fmm_vs_direct_sum():
    """With real coordinates the FMM reaches eps against the direct sum.  With
    the complex stretch of the uniform benchmark case the reference algorithm
    itself stops converging at deep levels (its README: eps is only guaranteed
    for real locations); there the GPU FMM must show the same error as the
    oracle's FMM."""
    import zfmm_b200
    n = 20000
    sub = np.arange(0, n, 5)
    for stretch in [0.0, 1.0]:
        w = W.lap2d_uniform(n, seed=2)
        w["zsrc"] = w["zsrc"].real + 1j * stretch * w["zsrc"].imag
        p, g = run_gpu(1e-9, w)
        zt = w["zsrc"][:, sub]
        pd, gd = zfmm_b200.zl2devaldirect(len(sub), zt, n, w["zsrc"], w["charge"], w["dipstr"],
                                          w["dipvec"], 1, 1, 2)
        ep, eg = rel(p[sub] * 2 * np.pi, pd), rel(g[:, sub] * 2 * np.pi, gd)
        if stretch == 0.0:
            assert ep < 1e-8 and eg < 1e-8
        else:
            po, go = run_oracle(1e-9, w)
            eop, eog = rel(po[sub] * 2 * np.pi, pd), rel(go[:, sub] * 2 * np.pi, gd)
            assert abs(ep - eop) < 1e-8 and abs(eg - eog) < 1e-8


def test_direct_matches_oracle():
    import zfmm_b200
    w = W.clustered2d(3000, seed=4)
    t = W.lap2d_uniform(1000, seed=5)["zsrc"]
    for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1), (0, 1, 2)]:
        pd, gd = zfmm_b200.zl2devaldirect(1000, t, 3000, w["zsrc"], w["charge"], w["dipstr"],
                                          w["dipvec"], ifc, ifd, ifpgh)
        po, go = O.zl2ddirect(w["zsrc"].T, w["charge"] if ifc else None,
                              w["dipstr"] if ifd else None, w["dipvec"].T if ifd else None,
                              ztarg=t.T, ifpgh=ifpgh)
        assert rel(pd, po) < 1e-13
        if ifpgh == 2:
            assert rel(gd, go.T) < 1e-13


def test_fixture_golden_values():
    """Reference test5.f case: fixture, eps=1E-12, charges, pot only."""
    import zfmm_b200
    f = np.load(os.path.join(GOLD, "fixture2d.npz"))
    z, q = f["zsrc"].T, f["charge"]
    n = z.shape[1]
    p, _ = zfmm_b200.zlfmm2d(EPS12, n, z, 1, q, 0, None, None, n, z, 1, 1)
    po, _ = O.zlfmm2d(EPS12, z.T, q)
    assert rel(p, po) < 1e-11
    for v, (re, im) in zip(p[:12] * 2 * np.pi, G["2d_laplace"]["pot0"]):
        assert abs(v.real - re) <= 0.5e-4 * 10 ** np.ceil(np.log10(abs(re)))
        assert abs(v.imag - im) <= 0.5e-4 * 10 ** np.ceil(np.log10(abs(im)))
    pd, _ = zfmm_b200.zl2devaldirect(12, z[:, :12], n, z, q, None, None, 1, 0, 1)
    assert rel(p[:12] * 2 * np.pi, pd) < 1e-11


def test_edge_cases():
    import zfmm_b200
    rng = np.random.default_rng(0)
    # single source and target, coincident (excluded pair) and distinct.  The
    # reference returns NaN for the coincident case (its L2T divides by the
    # zero box size of the root); the local expansion of a level-0 box is
    # identically zero, so the device path skips it and returns 0.
    z = np.array([[0.1 + 0.01j], [0.2 - 0.02j]])
    p, g = zfmm_b200.zlfmm2d(1e-9, 1, z, 1, np.array([1.0 + 0j]), 0, None, None, 1, z, 2, 1)
    assert p[0] == 0 and not np.any(g)
    t = z + 0.5
    p, g = zfmm_b200.zlfmm2d(1e-9, 1, z, 1, np.array([1.0 + 0j]), 0, None, None, 1, t, 2, 1)
    r = np.sqrt(np.sum((t - z) ** 2))
    assert abs(p[0] - np.log(r) / (2 * np.pi)) < 1e-14
    # no sources: zero potential
    p, g = zfmm_b200.zlfmm2d(1e-9, 0, np.zeros((2, 0)), 1, np.zeros(0), 0, None, None, 1, t, 2, 1)
    assert p[0] == 0
    # out-of-range flags are clamped like the reference (ifpgh=7 -> 1)
    w = W.lap2d_uniform(500, seed=3)
    p1, g1 = run_gpu(1e-9, w, 1, 0, 7)
    p2, _ = run_gpu(1e-9, w, 1, 0, 1)
    assert np.array_equal(p1, p2) and not np.any(g1)


def test_torch_device_path():
    import torch
    import zfmm_b200
    w = W.lap2d_uniform(5000, seed=6)
    dev = torch.device("cuda:0")
    zs = torch.from_numpy(np.ascontiguousarray(w["zsrc"].T)).to(dev)
    q = torch.from_numpy(w["charge"]).to(dev)
    ds = torch.from_numpy(w["dipstr"]).to(dev)
    dv = torch.from_numpy(np.ascontiguousarray(w["dipvec"].T)).to(dev)
    p, g = zfmm_b200.zlfmm2d(1e-9, 5000, zs, 1, q, 1, ds, dv, 5000, zs, 2, 1)
    ph, gh = run_gpu(1e-9, w)
    assert rel(p.cpu().numpy(), ph) < 1e-14
    assert rel(g.cpu().numpy(), gh) < 1e-14
