"""CPU-side checks of the product library: it is built, loads without a GPU,
exports every entry point declared in include/zfmm.h, and fails loudly (a
status, no crash, no silent CPU fallback) when no GPU is present."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "zfmm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|long|double|char)\s*\*?\s*(\w+)\s*\(", src,
                       flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["zlfmm2d_", "zl2devaldirect_", "zfmm_zlfmm2d", "zfmm_zlfmm2d_dev",
              "zfmm_zl2devaldirect", "zfmm_last_error"]:
        assert n in names


def test_library_loads_and_exports_all_symbols():
    from zfmm_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        import zfmm_b200.build as b
        b.build(verbose=False)
    L = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding declares a signature for every exported C function
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_version_string():
    import zfmm_b200
    assert "sm_100a" in zfmm_b200.version()


def test_no_gpu_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import zfmm_b200
    z = np.zeros((2, 4), np.complex128)
    z[0] = np.arange(4)
    with pytest.raises(zfmm_b200.ZfmmError, match="status 5"):
        zfmm_b200.zlfmm2d(1e-6, 4, z, 1, np.ones(4), 0, None, None, 4, z, 1, 1)


def test_argument_errors_are_reported():
    import zfmm_b200
    z = np.zeros((2, 4), np.complex128)
    with pytest.raises(ValueError):
        zfmm_b200.zlfmm2d(1e-6, 4, z[:, :3], 1, np.ones(4), 0, None, None, 4, z, 1, 1)
    L = zfmm_b200.lib()
    rc = L.zfmm_zlfmm2d(1e-6, -1, None, 1, None, 0, None, None, None, None, 1, None, 1, 1, 0)
    assert rc == 1
    assert b"ns and nt" in L.zfmm_last_error()


def test_h2dterms_matches_reference_log():
    """The library's host-side h2dterms against the per-level expansion orders
    of the reference's Helmholtz test (zfmm2d/test/helmholtz/fort.13:22-24)."""
    import json
    import zfmm_b200
    gold = os.path.join(os.path.dirname(__file__), "golden")
    g = json.load(open(os.path.join(gold, "golden.json")))["2d_helmholtz"]
    z = np.load(os.path.join(gold, "fixture2d.npz"))["zsrc"].real
    bs0 = max(np.ptp(z[:, 0]), np.ptp(z[:, 1]))
    zk = np.array([3 * np.pi, 0.0])
    L = zfmm_b200.lib()
    got = [L.zfmm_h2dterms(bs0 / 2 ** l, zk.ctypes.data, float(np.float32(1e-12)), 1)
           for l in range(11)]
    assert got == g["nterms"]


def test_no_gpu_plans_and_batches_are_errors():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import zfmm_b200
    z = np.zeros((3, 5), np.complex128)
    z[0] = np.arange(5)
    with pytest.raises(zfmm_b200.ZfmmError, match="status 5"):
        zfmm_b200.Plan3D(1e-6, 5, z, 5, z)
    inst = [dict(zsrc=z, charge=np.ones(5))]
    with pytest.raises(zfmm_b200.ZfmmError, match="status 5"):
        zfmm_b200.zhfmm3d_many(1e-6, 1.0, inst, nstreams=2)


def test_misaligned_device_pointer_is_refused_before_launch():
    """Device entry points read complex values as 16-byte pairs: a pointer that
    is 8-byte but not 16-byte aligned is refused with status 1 (checked before
    the device is touched, so this runs without a GPU)."""
    import zfmm_b200
    L = zfmm_b200.lib()
    good, bad = ctypes.c_void_p(0x10000), ctypes.c_void_p(0x10008)
    stream = ctypes.c_void_p(0)
    rc = L.zfmm_zlfmm2d_dev(1e-6, 4, bad, 1, good, 0, None, None, good, good, 4, good, 1, 1,
                            stream)
    assert rc == 1 and b"16-byte aligned" in L.zfmm_last_error()
    rc = L.zfmm_zhfmm3d_dev(1e-6, np.array([1.0, 0.0]).ctypes.data, 4, good, 1, bad, 0, None,
                            None, good, good, 4, good, 1, 1, stream)
    assert rc == 1 and b"16-byte aligned" in L.zfmm_last_error()
    rc = L.zfmm_zl2devaldirect_dev_noalloc(4, good, 4, good, good, None, None, 1, bad, None, 0,
                                           1, stream)
    assert rc == 1 and b"16-byte aligned" in L.zfmm_last_error()
    # an unused array (flag off) is not checked
    rc = L.zfmm_zl2devaldirect_dev(4, good, 4, good, good, bad, bad, 1, good, None, 0, 1, stream)
    assert b"16-byte aligned" not in L.zfmm_last_error()


def test_torch_inputs_are_checked_before_any_pointer_is_used():
    """Strengths passed as torch tensors must be complex128 CUDA tensors of the
    right length; anything else is a ValueError, never a raw pointer handed to
    a kernel (checked here with CPU tensors, which no device entry point may
    receive)."""
    import torch
    import zfmm_b200
    z = torch.zeros((4, 2), dtype=torch.complex128)
    with pytest.raises(ValueError, match="CUDA tensor"):
        zfmm_b200.zlfmm2d(1e-6, 4, z, 1, torch.ones(4, dtype=torch.complex128), 0, None, None,
                          4, z, 1, 1)
    with pytest.raises(ValueError, match="CUDA tensor"):
        zfmm_b200._torch_vec(torch.ones(4, dtype=torch.complex64), 4, "charge",
                             torch.device("cpu"))
    with pytest.raises(ValueError, match="CUDA tensor"):
        zfmm_b200._torch_vec(np.ones(4, np.complex128), 4, "charge", torch.device("cpu"))


def test_adjoint_inputs_are_checked():
    import torch
    from zfmm_b200.adjoint import zhfmm2d_curves
    xr = torch.zeros((4, 2), dtype=torch.float64)
    with pytest.raises(ValueError, match="CUDA tensor"):
        zhfmm2d_curves(1e-6, 1.0, xr, xr, torch.zeros(4, dtype=torch.int64),
                       torch.zeros(1, dtype=torch.float64), torch.ones(4, dtype=torch.complex128))
