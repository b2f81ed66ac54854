"""Plan files (zfmm_plan2d_save / load, zfmm_plan3d_save / load): a plan
written to disk and read back solves exactly as the original plan (same
geometry arrays, so bit-identical results), and files of the wrong kind,
truncated files or other data are refused with status 1."""
import numpy as np
import pytest

from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def cn(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_plan2d_file_roundtrip(tmp_path):
    import zfmm_b200
    w = W.curve2d(15000, seed=41)
    zs = w["zsrc"]
    n = zs.shape[1]
    q, ds = cn(np.random.default_rng(1), 2, n), cn(np.random.default_rng(2), 2, n)
    plan = zfmm_b200.Plan2D(1e-9, n, zs, n, zs)
    f = tmp_path / "curve.zfmmplan"
    plan.save(f)
    p0, g0 = plan.zhfmm2d(40 + 0.5j, 2, 1, q, 1, ds, w["dipvec"], 2)
    plan.close()
    back = zfmm_b200.Plan2D.load(f)
    assert (back.ns, back.nt) == (n, n)
    p1, g1 = back.zhfmm2d(40 + 0.5j, 2, 1, q, 1, ds, w["dipvec"], 2)
    assert np.array_equal(p0, p1) and np.array_equal(g0, g1)
    pl, _ = back.zlfmm2d(1, 1, q[0], 0, None, None, 1)
    pr, _ = zfmm_b200.zlfmm2d(1e-9, n, zs, 1, q[0], 0, None, None, n, zs, 1, 1)
    assert np.array_equal(pl[0], pr)
    back.close()


def test_plan3d_file_roundtrip_and_refusals(tmp_path):
    import zfmm_b200
    w = W.sphere3d(12000, seed=42)
    zs = w["zsrc"]
    n = zs.shape[1]
    q = cn(np.random.default_rng(3), 5, n)
    plan = zfmm_b200.Plan3D(1e-9, n, zs, n, zs)
    f = tmp_path / "sphere.zfmmplan"
    plan.save(f)
    p0, g0 = plan.zhfmm3d(10 + 0.2j, 5, 1, q, 0, None, None, 2)
    plan.close()
    back = zfmm_b200.Plan3D.load(f)
    p1, g1 = back.zhfmm3d(10 + 0.2j, 5, 1, q, 0, None, None, 2)
    assert np.array_equal(p0, p1) and np.array_equal(g0, g1)
    back.close()
    with pytest.raises(zfmm_b200.ZfmmError, match="status 1"):
        zfmm_b200.Plan2D.load(f)  # a 3D plan file
    raw = f.read_bytes()
    short = tmp_path / "short.zfmmplan"
    short.write_bytes(raw[: len(raw) // 2])
    with pytest.raises(zfmm_b200.ZfmmError, match="status 1"):
        zfmm_b200.Plan3D.load(short)
    junk = tmp_path / "junk.bin"
    junk.write_bytes(b"not a plan" * 10)
    with pytest.raises(zfmm_b200.ZfmmError, match="status 1"):
        zfmm_b200.Plan3D.load(junk)
