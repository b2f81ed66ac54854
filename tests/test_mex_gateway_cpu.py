"""The MATLAB gateway on a machine without a GPU or MATLAB: it compiles
against the MEX API, checks argument sizes the way mwrap gateways do, and a
library failure (here: no GPU, status 5) becomes a MATLAB error carrying the
library's message instead of a crash or a silent fallback."""
import numpy as np
import pytest

import mex_gateway as G


def _args2d(n=5):
    z = np.zeros((2, n), np.complex128)
    z[0] = np.arange(n)
    one = np.ones(n, np.complex128)
    return [1e-6, n, z, 1, one, 0, one, z, np.zeros(n, np.complex128),
            np.zeros((2, n), np.complex128), n, z, 1, 1, 0]


def test_gateway_reports_library_failure_as_matlab_error(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present: covered by test_gpu_mex_gateway")
    L = G.build(tmp_path)
    outs, err = G.call(L, "zlfmm2d", _args2d())
    assert err is not None and "status 5" in err and "no CUDA device" in err


def test_gateway_checks_sizes_and_identifiers(tmp_path):
    L = G.build(tmp_path)
    a = _args2d()
    dims = [1, 1, 2, 4, 1, 5, 1, 5, 2, 5, 5, 2, 5, 1, 2, 5, 1, 1, 1]  # zsrc declared 2 x 4
    _, err = G.call(L, "zlfmm2d", a, dims=dims)
    assert err == "Bad argument size: zsrc"
    _, err = G.call(L, "zlfmm2d", a, spec="d i m i v i v m v m i m i i")  # 14 arguments
    assert err is not None and "does not match" in err
    _, err = G.call(L, "zqfmm2d", a, spec=G.SPECS["zlfmm2d"])
    assert err == "Unknown identifier"
