"""The eight Fortran-callable symbols on the GPU, called by reference as a
Fortran program calls them (tests/fortran_abi.py): results equal to the
status-returning C entry points on the same inputs (same device path, so
bit-identical), the flags clamped in place, and on a failing call pot and
grad zero with the reason in zfmm_last_error()."""
import numpy as np
import pytest

import fortran_abi as F
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _inputs(d, n, seed):
    w = W.lap2d_uniform(n, seed=seed) if d == 2 else W.sphere3d(n, seed=seed)
    return w


@pytest.mark.parametrize("d,zk", [(2, None), (2, 20 + 0.5j), (3, None), (3, 10 + 0.2j)])
def test_fmm_symbols_match_c_entry_points(d, zk):
    import zfmm_b200
    w = _inputs(d, 6000, 51 + d)
    zs = w["zsrc"]
    t = zs[:, :2500]
    n = zs.shape[1]
    for ifc, ifd, ifpgh in [(1, 1, 2), (1, 0, 1), (0, 1, 2)]:
        flags = []
        pf, gf = F.fmm(d, 1e-9, zk, zs, ifc, w["charge"], ifd, w["dipstr"], w["dipvec"], t, ifpgh,
                       flags_out=flags)
        assert flags == [ifc, ifd, ifpgh]
        fn = {(2, False): zfmm_b200.zlfmm2d, (3, False): zfmm_b200.zlfmm3d}
        if zk is None:
            pc, gc = fn[(d, False)](1e-9, n, zs, ifc, w["charge"], ifd, w["dipstr"], w["dipvec"],
                                   t.shape[1], t, ifpgh, 1)
        else:
            f = zfmm_b200.zhfmm2d if d == 2 else zfmm_b200.zhfmm3d
            pc, gc = f(1e-9, zk, n, zs, ifc, w["charge"], ifd, w["dipstr"], w["dipvec"],
                       t.shape[1], t, ifpgh, 1)
        assert np.array_equal(pf, pc), (ifc, ifd, ifpgh)
        if ifpgh == 2:
            assert np.array_equal(gf, gc), (ifc, ifd, ifpgh)
        else:
            assert np.all(gf == 0)


@pytest.mark.parametrize("d,zk", [(2, None), (2, 20 + 0.5j), (3, None), (3, 10 + 0.2j)])
def test_direct_symbols_match_c_entry_points(d, zk):
    import zfmm_b200
    w = _inputs(d, 3000, 61 + d)
    zs = w["zsrc"]
    t = zs[:, :700] + 0.01
    n = zs.shape[1]
    for ifc, ifd, ifpgh in [(1, 1, 2), (0, 1, 1)]:
        pf, gf = F.direct(d, zk, t, zs, w["charge"], w["dipstr"], w["dipvec"], ifc, ifd, ifpgh)
        args = (t.shape[1], t, n, zs, w["charge"], w["dipstr"], w["dipvec"], ifc, ifd, ifpgh)
        if zk is None:
            f = zfmm_b200.zl2devaldirect if d == 2 else zfmm_b200.zl3devaldirect
            pc, gc = f(*args)
        else:
            f = zfmm_b200.zh2devaldirect if d == 2 else zfmm_b200.zh3devaldirect
            pc, gc = f(zk, *args)
        assert np.array_equal(pf, pc)
        if ifpgh == 2:
            assert np.array_equal(gf, gc)


@pytest.mark.parametrize("d,zk", [(2, None), (2, 20 + 0.5j), (3, None), (3, 10 + 0.2j)])
def test_out_of_range_flags_clamped_like_the_reference(d, zk):
    import zfmm_b200
    w = _inputs(d, 3000, 71 + d)
    zs = w["zsrc"]
    n = zs.shape[1]
    flags = []
    pf, gf = F.fmm(d, 1e-6, zk, zs, 5, w["charge"], 2, w["dipstr"], w["dipvec"], zs, 3,
                   flags_out=flags)
    # zlfmm2d.f:58-68: ifcharge -> 1, ifdipole -> 0, ifpgh -> 1 when out of range
    assert flags == [1, 0, 1]
    if zk is None:
        f = zfmm_b200.zlfmm2d if d == 2 else zfmm_b200.zlfmm3d
        pc, _ = f(1e-6, n, zs, 1, w["charge"], 0, None, None, n, zs, 1, 1)
    else:
        f = zfmm_b200.zhfmm2d if d == 2 else zfmm_b200.zhfmm3d
        pc, _ = f(1e-6, zk, n, zs, 1, w["charge"], 0, None, None, n, zs, 1, 1)
    assert np.array_equal(pf, pc)
    assert np.all(gf == 0)


@pytest.mark.parametrize("d,zk", [(2, None), (2, 20 + 0.5j), (3, None), (3, 10 + 0.2j)])
def test_failing_call_zeroes_outputs_and_reports(d, zk):
    from zfmm_b200 import _capi
    w = _inputs(d, 2000, 81 + d)
    zs = w["zsrc"]
    pot, grad = F.fmm(d, 1e-6, zk, zs, 1, w["charge"], 0, None, None, zs, 2, isep=0)
    assert np.all(pot == 0) and np.all(grad == 0)
    assert b"isep" in _capi.lib().zfmm_last_error()
    # a NaN coordinate cannot be placed in a tree: refused, outputs zero
    bad = zs.copy()
    bad[0, 17] = np.nan
    pot, grad = F.fmm(d, 1e-6, zk, bad, 1, w["charge"], 0, None, None, bad, 2)
    assert np.all(pot == 0) and np.all(grad == 0)
    assert b"finite" in _capi.lib().zfmm_last_error()
