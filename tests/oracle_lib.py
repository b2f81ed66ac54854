"""ctypes access to the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: used by tests/, __graft_entry__.smoke() and the CPU
legs of bench.py as the checker, never by the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = ctypes.CDLL(ORACLE_SO)
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.c_void_p)


def c128(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128))
    if shape is not None:
        a = a.reshape(shape)
    return a


def zlfmm2d(eps, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1, isep=1):
    """Oracle zlfmm2d with the reference argument meaning; arrays (n,2) complex."""
    zsrc = c128(zsrc)
    ns = zsrc.shape[0]
    ztarg = zsrc if ztarg is None else c128(ztarg)
    nt = ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 2), np.complex128)
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 2), np.complex128)
    f = lib().o_zlfmm2d
    f.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int]
    rc = f(eps, ns, _p(zsrc), ifc, _p(q), ifd, _p(ds), _p(dv), _p(pot), _p(grad), nt, _p(ztarg),
           ifpgh, isep, 0)
    assert rc == 0
    return pot, grad


def zl2ddirect(zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1):
    """Unscaled zl2devaldirect (no 1/2pi), as in the reference."""
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    ns, nt = zsrc.shape[0], ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 2), np.complex128)
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 2), np.complex128)
    f = lib().o_zl2devaldirect
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    f(nt, _p(ztarg), ns, _p(zsrc), _p(q), _p(ds), _p(dv), ifc, _p(pot), _p(grad), ifd, ifpgh)
    return pot, grad


def tree_info(D, ndiv, zsrc, ztarg=None, isep=1):
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    nlev = ctypes.c_int(0)
    laddr = np.zeros(2 * 64, np.int32)
    mnl = np.zeros(4, np.int32)
    f = lib().o_tree_info
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    nb = f(D, 0.0, ndiv, _p(zsrc), zsrc.shape[0], _p(ztarg), ztarg.shape[0], isep,
           ctypes.byref(nlev), _p(laddr), laddr.size, _p(mnl))
    L = nlev.value
    return {"nboxes": nb, "nlevels": L, "laddr": laddr[:2 * (L + 1)].reshape(L + 1, 2),
            "mnlist": mnl.tolist()}


def tree_dump(D, ndiv, zsrc, ztarg=None, isep=1):
    """Full tree: per-box arrays, sort permutations/ranges and lists (0-based)."""
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    info = tree_info(D, ndiv, zsrc, ztarg, isep)
    nb = info["nboxes"]
    NC = 1 << D
    ns, nt = zsrc.shape[0], ztarg.shape[0]
    out = dict(ilevel=np.zeros(nb, np.int32), iparent=np.zeros(nb, np.int32),
               nchild=np.zeros(nb, np.int32), ichild=np.zeros((nb, NC), np.int32),
               centers=np.zeros((nb, D)), isrc=np.zeros(ns, np.int32),
               isrcse=np.zeros((nb, 2), np.int32), itarg=np.zeros(nt, np.int32),
               itargse=np.zeros((nb, 2), np.int32), nlist=np.zeros((4, nb), np.int32))
    cap = 400 * nb + 1000
    flat = np.zeros(cap, np.int32)
    f = lib().o_tree_dump
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 11 + [ctypes.c_int]
    n = f(D, ndiv, _p(zsrc), ns, _p(ztarg), nt, isep, _p(out["ilevel"]), _p(out["iparent"]),
          _p(out["nchild"]), _p(out["ichild"]), _p(out["centers"]), _p(out["isrc"]),
          _p(out["isrcse"]), _p(out["itarg"]), _p(out["itargse"]), _p(out["nlist"]), _p(flat),
          cap)
    assert 0 <= n <= cap
    out["lists_flat"] = flat[:n]
    out.update(info)
    return out


def hank103(z):
    f = lib().o_hank103
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    a = np.zeros(2)
    b = np.zeros(2)
    f(float(np.real(z)), float(np.imag(z)), _p(a), _p(b))
    return a[0] + 1j * a[1], b[0] + 1j * b[1]


def h2dterms(bsize, zk, eps, isep=1):
    f = lib().o_h2dterms
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    f.restype = ctypes.c_int
    return f(bsize, zk.real, zk.imag, eps, isep)


def jbessel2d(nterms, z, rscale, ifder=0):
    f = lib().o_jbessel2d
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p]
    a = np.zeros(nterms + 2, np.complex128)
    d = np.zeros(nterms + 2, np.complex128)
    f(nterms, z.real, z.imag, rscale, _p(a), ifder, _p(d))
    return a[:nterms + 1], d[:nterms + 1]


def h2dall(nterms, z, rscale, ifder=0):
    f = lib().o_h2dall
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p]
    a = np.zeros(nterms + 2, np.complex128)
    d = np.zeros(nterms + 2, np.complex128)
    f(nterms, z.real, z.imag, rscale, _p(a), ifder, _p(d))
    return a[:nterms + 1], d[:nterms + 1]


def zhfmm2d(eps, zk, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1, isep=1):
    """Oracle zhfmm2d (scaled by i/4 like the reference); arrays (n,2) complex."""
    zsrc = c128(zsrc)
    ns = zsrc.shape[0]
    ztarg = zsrc if ztarg is None else c128(ztarg)
    nt = ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 2), np.complex128)
    zkv = np.array([complex(zk).real, complex(zk).imag])
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 2), np.complex128)
    f = lib().o_zhfmm2d
    f.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int]
    rc = f(eps, _p(zkv), ns, _p(zsrc), ifc, _p(q), ifd, _p(ds), _p(dv), _p(pot), _p(grad), nt,
           _p(ztarg), ifpgh, isep, 0)
    assert rc == 0
    return pot, grad


def zh2ddirect(zk, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1):
    """Unscaled zh2devaldirect (no i/4), as in the reference."""
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    ns, nt = zsrc.shape[0], ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 2), np.complex128)
    zkv = np.array([complex(zk).real, complex(zk).imag])
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 2), np.complex128)
    f = lib().o_zh2devaldirect
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    f(_p(zkv), nt, _p(ztarg), ns, _p(zsrc), _p(q), _p(ds), _p(dv), ifc, _p(pot), _p(grad), ifd,
      ifpgh)
    return pot, grad


def zlfmm3d(eps, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1, isep=1):
    """Oracle zlfmm3d; arrays (n,3) complex."""
    zsrc = c128(zsrc)
    ns = zsrc.shape[0]
    ztarg = zsrc if ztarg is None else c128(ztarg)
    nt = ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 3), np.complex128)
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 3), np.complex128)
    f = lib().o_zlfmm3d
    f.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_int]
    rc = f(eps, ns, _p(zsrc), ifc, _p(q), ifd, _p(ds), _p(dv), _p(pot), _p(grad), nt, _p(ztarg),
           ifpgh, isep, 0)
    assert rc == 0
    return pot, grad


def zl3ddirect(zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1):
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    ns, nt = zsrc.shape[0], ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 3), np.complex128)
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 3), np.complex128)
    f = lib().o_zl3devaldirect
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    f(nt, _p(ztarg), ns, _p(zsrc), _p(q), _p(ds), _p(dv), ifc, _p(pot), _p(grad), ifd, ifpgh)
    return pot, grad


def h3dterms(size, zk, eps, isep=1):
    f = lib().o_h3dterms
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    f.restype = ctypes.c_int
    zk = complex(zk)
    return f(size, zk.real, zk.imag, eps, isep)


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    f = lib().o_gauss_legendre
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f(n, _p(x), _p(w))
    return x, w


def zhfmm3d(eps, zk, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1, isep=1):
    """Oracle zhfmm3d; arrays (n,3) complex."""
    zsrc = c128(zsrc)
    ns = zsrc.shape[0]
    ztarg = zsrc if ztarg is None else c128(ztarg)
    nt = ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 3), np.complex128)
    k = np.array([complex(zk).real, complex(zk).imag])
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 3), np.complex128)
    f = lib().o_zhfmm3d
    f.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int]
    rc = f(eps, _p(k), ns, _p(zsrc), ifc, _p(q), ifd, _p(ds), _p(dv), _p(pot), _p(grad), nt,
           _p(ztarg), ifpgh, isep, 0)
    assert rc == 0
    return pot, grad


def zh3ddirect(zk, zsrc, charge=None, dipstr=None, dipvec=None, ztarg=None, ifpgh=1):
    zsrc = c128(zsrc)
    ztarg = zsrc if ztarg is None else c128(ztarg)
    ns, nt = zsrc.shape[0], ztarg.shape[0]
    ifc = 0 if charge is None else 1
    ifd = 0 if dipstr is None else 1
    q = c128(charge) if ifc else np.zeros(1, np.complex128)
    ds = c128(dipstr) if ifd else np.zeros(1, np.complex128)
    dv = c128(dipvec) if ifd else np.zeros((1, 3), np.complex128)
    k = np.array([complex(zk).real, complex(zk).imag])
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((nt, 3), np.complex128)
    f = lib().o_zh3devaldirect
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    f(_p(k), nt, _p(ztarg), ns, _p(zsrc), _p(q), _p(ds), _p(dv), ifc, _p(pot), _p(grad), ifd,
      ifpgh)
    return pot, grad
