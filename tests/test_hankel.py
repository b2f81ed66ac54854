"""H0/H1 of complex argument and the 2D Helmholtz sizing, pinned against
independent high-precision values (mpmath, 160 digits) and the reference logs.

The reference computes H0, H1 with hank101/hank103
(zfmm2d/src/helmholtz/hank103.f:131-263): principal branch, a zero imaginary
part counting as +0.  The oracle and the device code compute the same
functions from the mathematics (hank2d.cuh); this file checks the oracle."""
import json
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
G = json.load(open(os.path.join(GOLD, "golden.json")))
EPS12 = float(np.float32(1e-12))


def test_hankel_against_mpmath():
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 160
    worst = 0.0
    for R in [1e-3, 0.5, 1.99, 2.01, 5, 12, 40]:
        for th in np.linspace(-np.pi + 0.05, np.pi, 13):
            z = R * np.exp(1j * th)
            h0, h1 = O.hank103(z)
            zz = mp.mpc(z.real, z.imag)
            r0 = complex(mp.hankel1(0, zz))
            r1 = complex(mp.hankel1(1, zz))
            worst = max(worst, abs(h0 - r0) / abs(r0), abs(h1 - r1) / abs(r1))
    assert worst < 5e-14


def test_hankel_negative_real_axis_is_upper_side():
    # -0 imaginary part is treated as +0 (the reference's upper-half-plane test)
    a = O.hank103(complex(-3.0, 0.0))
    b = O.hank103(complex(-3.0, -0.0))
    assert a == b
    mp = pytest.importorskip("mpmath")
    r = complex(mp.hankel1(0, mp.mpc(-3.0, 1e-300)))
    assert abs(a[0] - r) / abs(r) < 1e-14


def test_h2dterms_matches_reference_log():
    """nterms per level of the Helmholtz test (zk = 3 pi, eps = 1E-12):
    zfmm2d/test/helmholtz/fort.13:22-24."""
    z = np.load(os.path.join(GOLD, "fixture2d.npz"))["zsrc"]
    x = z.real
    bs0 = max(np.ptp(x[:, 0]), np.ptp(x[:, 1]))
    got = [O.h2dterms(bs0 / 2 ** l, complex(3 * np.pi), EPS12) for l in range(11)]
    assert got == G["2d_helmholtz"]["nterms"]


def test_direct2d_helmholtz_first12():
    """zh2devaldirect on the fixture, zk = 3 pi: zfmm2d/test/helmholtz/fort.13:82-86."""
    f = np.load(os.path.join(GOLD, "fixture2d.npz"))
    z, q = f["zsrc"], f["charge"]
    pot, _ = O.zh2ddirect(3 * np.pi, z, q, ztarg=z[:12])
    for p, (re, im) in zip(pot, G["2d_helmholtz"]["pot0"]):
        for a, b in [(p.real, re), (p.imag, im)]:
            e = np.floor(np.log10(abs(b))) + 1
            assert abs(a - b) <= 0.5e-5 * 10.0 ** e * 1.0001


def test_fmm2d_helmholtz_fixture_matches_direct():
    f = np.load(os.path.join(GOLD, "fixture2d.npz"))
    z, q = f["zsrc"], f["charge"]
    pot, _ = O.zhfmm2d(EPS12, 3 * np.pi, z, q)
    sub = np.arange(0, z.shape[0], 97)
    pd, _ = O.zh2ddirect(3 * np.pi, z, q, ztarg=z[sub])
    err = np.linalg.norm(pot[sub] - 0.25j * pd) / np.linalg.norm(0.25j * pd)
    assert err < 1e-11
