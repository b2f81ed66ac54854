"""The autotuner on the GPU: with tuning on, the first solve times the
candidate block sizes of the tunable 2D Helmholtz kernels (filling the
table), and every solve, tuned or not, gives bit-identical results."""
import numpy as np
import pytest

from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_tuned_solves_are_identical():
    import zfmm_b200
    from zfmm_b200 import _capi
    L = _capi.lib()
    w = W.curve2d(40000, seed=61)
    zs, n = w["zsrc"], 40000
    args = (1e-9, 40 + 0.5j, n, zs, 1, w["charge"], 1, w["dipstr"], w["dipvec"], n, zs, 2, 1)
    p0, g0 = zfmm_b200.zhfmm2d(*args)
    L.zfmm_set_autotune(1)
    try:
        n0 = L.zfmm_autotune_entries()
        p1, g1 = zfmm_b200.zhfmm2d(*args)
        assert L.zfmm_autotune_entries() >= n0 + 5
        p2, g2 = zfmm_b200.zhfmm2d(*args)
    finally:
        L.zfmm_set_autotune(0)
    for p, g in ((p1, g1), (p2, g2)):
        assert np.array_equal(p, p0) and np.array_equal(g, g0)
