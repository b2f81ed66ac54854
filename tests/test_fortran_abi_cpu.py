"""The Fortran-callable symbols on a machine without a GPU: the flags are
clamped in place before anything else (zlfmm2d.f:58-68), and a call that
cannot run leaves pot and grad zero and the reason in zfmm_last_error()
(no status is returned to a Fortran caller, as in the reference)."""
import numpy as np
import pytest

import fortran_abi as F


def _no_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present: the failure path is covered by test_gpu_fortran_abi")


@pytest.mark.parametrize("d,zk", [(2, None), (2, 3 + 0.1j), (3, None), (3, 3 + 0.1j)])
def test_flags_clamped_in_place_and_failure_zeroes_outputs(d, zk):
    _no_gpu()
    from zfmm_b200 import _capi
    z = np.zeros((d, 5), np.complex128)
    z[0] = np.arange(5)
    flags = []
    pot, grad = F.fmm(d, 1e-6, zk, z, 7, np.ones(5), -3, np.ones(5), np.ones((d, 5)), z, 9,
                      flags_out=flags)
    # out-of-range flags are rewritten as the reference does:
    # ifcharge -> 1, ifdipole -> 0, ifpgh -> 1
    assert flags == [1, 0, 1]
    assert np.all(pot == 0) and np.all(grad == 0)
    assert b"no CUDA device" in _capi.lib().zfmm_last_error()
