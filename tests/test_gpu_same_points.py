"""Targets passed as the source array itself (one pointer for zsrc and ztarg,
the sources being their own targets): the set-up then assigns, sorts and centres the
points once and copies the target side.  The result must be bit-identical to
the same call with the targets in a separate copy of the array, through the
host-array entry points, the device entry points and the plans."""
import numpy as np
import pytest
import torch

import zfmm_b200 as zf

pytestmark = pytest.mark.gpu

CASES = [
    ("zlfmm2d", 2, None),
    ("zhfmm2d", 2, 3.0 + 0.1j),
    ("zlfmm3d", 3, None),
    ("zhfmm3d", 3, 2.0 + 0.05j),
]


def _inputs(d, n, seed):
    rng = np.random.default_rng(seed)
    z = rng.random((d, n)) + 0.05j * rng.standard_normal((d, n))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ds = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    dv = rng.standard_normal((d, n)) + 1j * rng.standard_normal((d, n))
    return np.asfortranarray(z), q, ds, np.asfortranarray(dv)


def _call(name, zk, eps, n, zs, q, ds, dv, zt):
    f = getattr(zf, name)
    if zk is None:
        return f(eps, n, zs, 1, q, 1, ds, dv, n, zt, 2)
    return f(eps, zk, n, zs, 1, q, 1, ds, dv, n, zt, 2)


@pytest.mark.parametrize("name,d,zk", CASES)
def test_host_same_array(name, d, zk):
    n = 6000
    z, q, ds, dv = _inputs(d, n, 11)
    p1, g1 = _call(name, zk, 1e-9, n, z, q, ds, dv, z)
    p2, g2 = _call(name, zk, 1e-9, n, z, q, ds, dv, z.copy(order="F"))
    assert np.array_equal(p1, p2)
    assert np.array_equal(g1, g2)


@pytest.mark.parametrize("name,d,zk", CASES)
def test_device_same_tensor(name, d, zk):
    n = 6000
    z, q, ds, dv = _inputs(d, n, 12)
    dev = torch.device("cuda:0")
    tz = torch.from_numpy(np.ascontiguousarray(z.T)).to(dev)
    tq = torch.from_numpy(q).to(dev)
    tds = torch.from_numpy(ds).to(dev)
    tdv = torch.from_numpy(np.ascontiguousarray(dv.T)).to(dev)
    p1, g1 = _call(name, zk, 1e-9, n, tz, tq, tds, tdv, tz)
    p2, g2 = _call(name, zk, 1e-9, n, tz, tq, tds, tdv, tz.clone())
    torch.cuda.synchronize()
    assert torch.equal(p1, p2)
    assert torch.equal(g1, g2)
    # the device and host entry points give the same bits
    p_host, _ = _call(name, zk, 1e-9, n, z, q, ds, dv, z)
    assert np.array_equal(p1.cpu().numpy(), p_host)


@pytest.mark.parametrize("D", [2, 3])
def test_plan_same_array(D):
    n = 5000
    z, q, ds, dv = _inputs(D, n, 13)
    P = zf.Plan2D if D == 2 else zf.Plan3D
    a = P(1e-9, n, z, n, z)
    b = P(1e-9, n, z, n, z.copy(order="F"))
    try:
        fa = a.zlfmm2d if D == 2 else a.zlfmm3d
        fb = b.zlfmm2d if D == 2 else b.zlfmm3d
        pa, ga = fa(1, 1, q, 1, ds, dv, 2)
        pb, gb = fb(1, 1, q, 1, ds, dv, 2)
        assert np.array_equal(pa, pb)
        assert np.array_equal(ga, gb)
    finally:
        a.close()
        b.close()
