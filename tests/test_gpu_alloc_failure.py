"""Device-allocation failure in the middle of a solve (injected on the host
through zfmm_fail_alloc_after, no GPU fault): the call reports status 3
(out of memory) with the allocator's message, returns what it had taken, and
the next call on the same process gives the same result as before."""
import numpy as np
import pytest
import torch

import zfmm_b200 as zf
from zfmm_b200 import workloads as W
from zfmm_b200._capi import ZfmmError, lib

pytestmark = pytest.mark.gpu


def _solve2d(w, n):
    return zf.zhfmm2d(1e-9, 40 + 0.5j, n, w["zsrc"], 1, w["charge"], 1, w["dipstr"],
                      w["dipvec"], n, w["zsrc"], 2, 1)


def _solve3d(w, n):
    return zf.zhfmm3d(1e-6, 3.0 + 0.1j, n, w["zsrc"], 1, w["charge"], 1, w["dipstr"],
                      w["dipvec"], n, w["zsrc"], 2, 1)


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_failed_allocation_then_recovery(kind):
    n = 4000
    w = W.curve2d(n, seed=21) if kind == "2d" else W.sphere3d(n, seed=21)
    solve = _solve2d if kind == "2d" else _solve3d
    L = lib()
    p0, g0 = solve(w, n)
    failed = 0
    try:
        for k in [0, 1, 2, 3, 5, 8, 13, 21, 34, 55, 89, 144]:
            L.zfmm_fail_alloc_after(k)
            try:
                solve(w, n)
            except ZfmmError as e:
                assert "status 3" in str(e), str(e)
                failed += 1
            L.zfmm_fail_alloc_after(-1)
            p, g = solve(w, n)
            assert np.array_equal(p, p0) and np.array_equal(g, g0)
    finally:
        L.zfmm_fail_alloc_after(-1)
    assert failed >= 6  # a solve makes many allocations: the early ones all fail it


def test_failed_allocation_device_path():
    n = 4000
    w = W.curve2d(n, seed=22)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    zs, q, ds, dv = t(w["zsrc"].T), t(w["charge"]), t(w["dipstr"]), t(w["dipvec"].T)
    run = lambda: zf.zhfmm2d(1e-9, 40 + 0.5j, n, zs, 1, q, 1, ds, dv, n, zs, 2, 1)
    p0, _ = run()
    L = lib()
    try:
        L.zfmm_fail_alloc_after(7)
        with pytest.raises(ZfmmError, match="status 3"):
            run()
    finally:
        L.zfmm_fail_alloc_after(-1)
    p1, _ = run()
    torch.cuda.synchronize()
    assert torch.equal(p0, p1)
