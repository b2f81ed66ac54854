"""Allocation-free direct sum (zfmm_zl2devaldirect_dev_noalloc).

This entry point serves callers that cannot allocate device memory during a
solve (their GPU memory is owned by another allocator, or they run under a
fixed budget): it keeps the partial sums of its source-split kernel in a fixed
device array of the library instead of taking scratch memory.  The test calls
it through the C ABI and compares it with the allocating entry point
zfmm_zl2devaldirect_dev on the same device inputs, twice in a row (the array
keeps the previous call's contents, which must not leak into the next
result), at the tolerance of the direct-sum tests (1e-13 relative).  The sizes
(1,000 targets, 40,000 sources) make the kernel split the sources, so the
fixed array is really used.  The file name sorts last so that a run stopping
at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, torch, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def test_noalloc_direct_matches_allocating_entry_point():
    import torch

    from zfmm_b200 import _capi
    from zfmm_b200 import workloads as W

    L = _capi.lib()
    dev = torch.device("cuda:0")
    ns, nt = 40000, 1000
    w = W.clustered2d(ns, seed=21)
    t = W.lap2d_uniform(nt, seed=22)["zsrc"]
    zs = _dev(w["zsrc"].T, torch, dev)
    zt = _dev(t.T, torch, dev)
    q = _dev(w["charge"], torch, dev)
    ds = _dev(w["dipstr"], torch, dev)
    dv = _dev(w["dipvec"].T, torch, dev)
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    assert L.zfmm_zl2devaldirect_noalloc_capacity() == 8 << 20

    def run(fn):
        pot = torch.zeros(nt, dtype=torch.complex128, device=dev)
        grad = torch.zeros((nt, 2), dtype=torch.complex128, device=dev)
        _capi.check(fn(nt, P(zt), ns, P(zs), P(q), P(ds), P(dv), 1, P(pot), P(grad), 1, 2,
                       stream))
        return pot.cpu().numpy(), grad.cpu().numpy()

    p_ref, g_ref = run(L.zfmm_zl2devaldirect_dev)
    for _ in range(2):
        p, g = run(L.zfmm_zl2devaldirect_dev_noalloc)
        assert np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref) < 1e-13
        assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 1e-13
