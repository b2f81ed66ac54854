"""The tcgen05 TF32 building block of the batched translations
(zfmm_tc_selftest): D = A B^T through the tensor cores with the three-term
split must match the FP64 product to the split's accuracy (about 1e-6
relative, FP32 accumulation) for operand shapes used by the translations."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(64, 128), (16, 8), (128, 72), (256, 40), (48, 104)])
def test_tf32x3_product_matches_fp64(N, K):
    import torch

    from zfmm_b200 import _capi
    L = _capi.lib()
    rng = np.random.default_rng(N * 1000 + K)
    a = rng.standard_normal((128, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    dev = torch.device("cuda:0")
    A, B = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    D = torch.zeros((128, N), dtype=torch.float32, device=dev)
    s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    rc = L.zfmm_tc_selftest(N, K, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
                            ctypes.c_void_p(D.data_ptr()), s)
    assert rc == 0
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    err = np.abs(D.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
    # the one-term TF32 product would be ~1e-3: the split is in effect
    assert err < 1e-5


def test_selftest_rejects_bad_shapes():
    from zfmm_b200 import _capi
    L = _capi.lib()
    assert L.zfmm_tc_selftest(20, 8, None, None, None, None) == 1
    assert L.zfmm_tc_selftest(64, 12, None, None, None, None) == 1
