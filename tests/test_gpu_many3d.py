"""Many independent 3D FMMs in one call (zfmm_z?fmm3d_many): every instance
must equal its own single call (the same passes run on each instance's own
tree, concurrently on several streams), for instances of very different sizes,
with charges and dipoles, shared or separate targets, and any number of
worker streams; completion times are reported for every instance."""
import numpy as np
import pytest

from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def test_helmholtz_instances_match_single_calls():
    import zfmm_b200
    eps, zk = 1e-9, 10 + 0.2j
    sizes = [1500, 12000, 3000, 25000, 700, 8000]
    inst = [W.sphere3d(n, seed=30 + i) for i, n in enumerate(sizes)]
    outs, done = zfmm_b200.zhfmm3d_many(eps, zk, inst, 1, 1, 2, 1, nstreams=3)
    assert np.all(done > 0) and len(done) == len(sizes)
    for w, (p, g) in zip(inst, outs):
        n = w["zsrc"].shape[1]
        p1, g1 = zfmm_b200.zhfmm3d(eps, zk, n, w["zsrc"], 1, w["charge"], 1, w["dipstr"],
                                   w["dipvec"], n, w["zsrc"], 2, 1)
        assert rel(p, p1) < 1e-14
        assert rel(g, g1) < 1e-14


def test_laplace_instances_separate_targets():
    import zfmm_b200
    eps = 1e-9
    inst = []
    for i, n in enumerate([5000, 900, 16000]):
        w = W.clustered3d(n, seed=40 + i)
        w["ztarg"] = W.lap3d_uniform(n // 2 + 100, seed=50 + i)["zsrc"]
        inst.append(w)
    for nstreams in (1, 4):
        outs, done = zfmm_b200.zlfmm3d_many(eps, inst, 1, 1, 2, 1, nstreams=nstreams)
        for w, (p, g) in zip(inst, outs):
            n, t = w["zsrc"].shape[1], w["ztarg"]
            p1, g1 = zfmm_b200.zlfmm3d(eps, n, w["zsrc"], 1, w["charge"], 1, w["dipstr"],
                                       w["dipvec"], t.shape[1], t, 2, 1)
            assert rel(p, p1) < 1e-14, nstreams
            assert rel(g, g1) < 1e-14, nstreams
