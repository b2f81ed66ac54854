"""The MATLAB gateway on the GPU: every routine called with the mwrap
argument protocol returns what the library's own entry points return for the
same inputs (same device path: bit-identical), including the inout semantics
of the direct sums (they add into the pot / grad passed in)."""
import numpy as np
import pytest

import mex_gateway as G
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,d,zk", [("zlfmm2d", 2, None), ("zhfmm2d", 2, 20 + 0.5j),
                                       ("zlfmm3d", 3, None), ("zhfmm3d", 3, 10 + 0.2j)])
def test_gateway_fmm_matches_library(tmp_path, name, d, zk):
    import zfmm_b200
    L = G.build(tmp_path)
    w = W.lap2d_uniform(4000, seed=91) if d == 2 else W.sphere3d(4000, seed=92)
    zs, n = w["zsrc"], w["zsrc"].shape[1]
    t = zs[:, :1500]
    nt = t.shape[1]
    pot0, grad0 = np.zeros(nt, np.complex128), np.zeros((d, nt), np.complex128)
    head = [1e-9] + ([zk] if zk is not None else [])
    args = head + [n, zs, 1, w["charge"], 1, w["dipstr"], w["dipvec"], pot0, grad0, nt, t, 2, 1,
                   0]
    (pot, grad), err = G.call(L, name, args)
    assert err is None, err
    f = getattr(zfmm_b200, name)
    if zk is None:
        pr, gr = f(1e-9, n, zs, 1, w["charge"], 1, w["dipstr"], w["dipvec"], nt, t, 2, 1)
    else:
        pr, gr = f(1e-9, zk, n, zs, 1, w["charge"], 1, w["dipstr"], w["dipvec"], nt, t, 2, 1)
    assert np.array_equal(pot[:, 0], pr)
    assert np.array_equal(grad, gr)


@pytest.mark.parametrize("name,d,zk", [("zl2devaldirect", 2, None), ("zh2devaldirect", 2, 3 + 0.1j),
                                       ("zl3devaldirect", 3, None), ("zh3devaldirect", 3, 3 + 0.1j)])
def test_gateway_direct_adds_into_inout(tmp_path, name, d, zk):
    import zfmm_b200
    L = G.build(tmp_path)
    w = W.lap2d_uniform(800, seed=93) if d == 2 else W.sphere3d(800, seed=94)
    zs, n = w["zsrc"], w["zsrc"].shape[1]
    t = zs[:, :300] + 0.01
    nt = t.shape[1]
    pot0 = np.full(nt, 1.0 + 2.0j)
    grad0 = np.full((d, nt), -1.0 + 0.5j)
    head = [zk] if zk is not None else []
    args = head + [nt, t, n, zs, w["charge"], w["dipstr"], w["dipvec"], 1, pot0, grad0, 1, 2]
    (pot, grad), err = G.call(L, name, args)
    assert err is None, err
    f = getattr(zfmm_b200, name)
    rest = (nt, t, n, zs, w["charge"], w["dipstr"], w["dipvec"], 1, 1, 2)
    pr, gr = f(zk, *rest) if zk is not None else f(*rest)
    assert np.allclose(pot[:, 0], pr + pot0, rtol=1e-14, atol=0)
    assert np.allclose(grad, gr + grad0, rtol=1e-14, atol=0)


def test_gateway_error_carries_status(tmp_path):
    L = G.build(tmp_path)
    w = W.lap2d_uniform(500, seed=95)
    zs, n = w["zsrc"], 500
    args = [1e-6, n, zs, 1, w["charge"], 0, w["dipstr"], zs, np.zeros(n), np.zeros((2, n)), n, zs,
            1, 0, 0]  # isep = 0
    _, err = G.call(L, "zlfmm2d", args)
    assert err is not None and "status 1" in err and "isep" in err
