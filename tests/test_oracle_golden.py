"""Pin the CPU oracle against the reference's own golden outputs.

The golden values come from the reference test logs (fort.13) for the binary
fixtures (see tests/golden/make_fixtures.py):
  * tree statistics: zfmm2d/test/helmholtz/fort.13:9-58 (same tree as the
    Laplace test, same ndiv), zfmm3d/test/laplace/fort.13:1-38;
  * first 12 direct-sum potentials: zfmm2d/test/laplace/fort.13:54-58 (unscaled
    zl2devaldirect), printed to 5 significant digits.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
G = json.load(open(os.path.join(GOLD, "golden.json")))
EPS12 = float(np.float32(1e-12))  # the tests assign the REAL*4 literal 1E-12


def fx(name):
    f = np.load(os.path.join(GOLD, name))
    return f["zsrc"], f["charge"]


def close5(a, b):
    """prini prints E11.5: 0.ddddd x 10^e, so the printed value is within
    half a unit of the fifth mantissa digit."""
    a, b = float(a), float(b)
    if b == 0.0:
        return abs(a) < 1e-300
    e = np.floor(np.log10(abs(b))) + 1
    return abs(a - b) <= 0.5e-5 * 10.0 ** e * 1.0001


def test_tree2d_matches_reference_log():
    z, _ = fx("fixture2d.npz")
    g = G["2d_helmholtz"]
    info = O.tree_info(2, g["ndiv"], z)
    assert info["nboxes"] == g["nboxes"] == G["2d_laplace"]["nboxes"]
    assert info["nlevels"] == g["nlevels"]
    assert (info["laddr"] + 1).tolist() == g["laddr"]
    assert info["mnlist"] == [g["mnlist1"], g["mnlist2"], g["mnlist3"], g["mnlist4"]]


def test_tree3d_matches_reference_log():
    z, _ = fx("fixture3d.npz")
    g = G["3d_laplace"]
    info = O.tree_info(3, g["ndiv"], z)
    assert info["nboxes"] == g["nboxes"]
    assert info["nlevels"] == g["nlevels"]
    assert (info["laddr"] + 1).tolist() == g["laddr"]
    assert info["mnlist"] == [g["mnlist1"], g["mnlist2"], g["mnlist3"], g["mnlist4"]]


def test_ndiv_and_nterms_tables():
    g = G["2d_laplace"]
    ndiv = O.lib().o_lndiv2d
    import ctypes
    a, b = ctypes.c_int(), ctypes.c_int()
    ndiv.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                     ctypes.POINTER(ctypes.c_int)]
    ndiv(EPS12, 1, 1, ctypes.byref(a), ctypes.byref(b))
    assert a.value == g["ndiv"] and b.value == 0
    f = O.lib().o_l2dterms
    f.argtypes = [ctypes.c_double]
    assert f(EPS12) == g["nterms"][0] == 37
    assert f(1e-9) == 28


def test_direct2d_laplace_first12():
    z, q = fx("fixture2d.npz")
    pot, _ = O.zl2ddirect(z, q, ztarg=z[:12])
    for p, (re, im) in zip(pot, G["2d_laplace"]["pot0"]):
        assert close5(p.real, re) and close5(p.imag, im)


def test_fmm2d_laplace_fixture_matches_direct():
    z, q = fx("fixture2d.npz")
    pot, _ = O.zlfmm2d(EPS12, z, q)
    # the log's FMM values are unscaled (they predate the 1/(2 pi) line)
    for p, (re, im) in zip(pot[:12] * 2 * np.pi, G["2d_laplace"]["pot"]):
        assert close5(p.real, re) and close5(p.imag, im)
    sub = np.arange(0, z.shape[0], 7)
    pd, _ = O.zl2ddirect(z, q, ztarg=z[sub])
    err = np.linalg.norm(pot[sub] * 2 * np.pi - pd) / np.linalg.norm(pd)
    assert err < 1e-11


def test_direct3d_laplace_first12():
    z, q = fx("fixture3d.npz")
    pot, _ = O.zl3ddirect(z, q, ztarg=z[:12])
    for p, (re, im) in zip(pot, G["3d_laplace"]["pot0"]):
        assert close5(p.real, re) and close5(p.imag, im)


def test_fmm3d_laplace_fixture_matches_log():
    """The reference's 3D Laplace test (test9.f:78-133): eps = 1e-12, charges,
    pot only; its log shows the first 12 potentials and err/(|pot0|+|q|) =
    1.4130e-10 (fort.13:57-76)."""
    z, q = fx("fixture3d.npz")
    pot, _ = O.zlfmm3d(EPS12, z, q)
    for p, (re, im) in zip(pot[:12], G["3d_laplace"]["pot"]):
        assert close5(p.real, re) and close5(p.imag, im)
    pd, _ = O.zl3ddirect(z, q)
    err = np.linalg.norm(pot - pd)
    assert close5(np.linalg.norm(pd), G["3d_laplace"]["pot0_norm"][0])
    assert close5(np.linalg.norm(q), G["3d_laplace"]["charge_norm"][0])
    rel = err / (np.linalg.norm(pd) + np.linalg.norm(q))
    assert rel < 3 * 1.4130e-10


def test_direct3d_helmholtz_first12():
    z, q = fx("fixture3d.npz")
    g = G["3d_helmholtz"]
    assert abs(complex(*g["zk"]) - np.pi) < 1e-4
    pot, _ = O.zh3ddirect(np.pi, z, q, ztarg=z[:12])  # test9.f: zk = pi
    for p, (re, im) in zip(pot, g["pot0"]):
        assert close5(p.real, re) and close5(p.imag, im)


def test_fmm3d_helmholtz_fixture_matches_log():
    """The reference's 3D Helmholtz test: zk = pi, eps = 1e-12, charges, pot
    only; its log shows the first 12 potentials, |pot0| = 13.215 and
    err/(|pot0|+|q|) = 8.8576e-10 (zfmm3d/test/helmholtz/fort.13:1-40)."""
    z, q = fx("fixture3d.npz")
    g = G["3d_helmholtz"]
    zk = complex(*g["zk"])
    assert abs(zk - np.pi) < 1e-4
    zk = np.pi  # test9.f: zk = pi (the log prints 5 digits)
    pot, _ = O.zhfmm3d(EPS12, zk, z, q)
    for p, (re, im) in zip(pot[:12], g["pot"]):
        assert close5(p.real, re) and close5(p.imag, im)
    pd, _ = O.zh3ddirect(zk, z, q)
    assert close5(np.linalg.norm(pd), g["pot0_norm"][0])
    rel = np.linalg.norm(pot - pd) / (np.linalg.norm(pd) + np.linalg.norm(q))
    assert rel < 3 * 8.8576e-10


def test_h3dterms_levels_and_quadrature():
    """h3dterms on the rescaled boxes of the fixture run, and the Gauss-Legendre
    rule of the z-shifts against numpy's."""
    import numpy.polynomial.legendre as leg
    for n in [5, 30, 92, 125]:
        x, w = O.gauss_legendre(n)
        xr, wr = leg.leggauss(n)
        assert np.abs(x - xr).max() < 1e-14 and np.abs(w - wr).max() < 1e-13
    p = [O.h3dterms(2.0 ** -l, np.pi * G["3d_laplace"]["b0"][0], EPS12) for l in range(4)]
    assert min(p) > 10 and max(p) < 200
