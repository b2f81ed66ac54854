"""Calls of the Fortran-callable symbols (zlfmm2d_ ... zh3devaldirect_) the
way a Fortran caller makes them: every argument by reference, INTEGER*4
scalars, `complex*16 zk` as one (re, im) pair, arrays in column-major order
(the reference's test drivers zfmm2d/test/laplace/test5.f:97-107 and
zfmm3d/test/laplace/test9.f:80-90 call the subroutines like this)."""
import ctypes

import numpy as np

from zfmm_b200 import _capi


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


def _a(x):
    return None if x is None else x.ctypes.data_as(ctypes.c_void_p)


def _cm(z, d, n):
    """(d, n) complex -> Fortran-ordered complex*16 array."""
    return np.asfortranarray(np.asarray(z, np.complex128).reshape(d, n))


def fmm(d, eps, zk, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, ztarg, ifpgh, isep=1,
        flags_out=None):
    """call z{l,h}fmm{d}d(eps,[zk,]ns,zsrc,ifcharge,charge,ifdipole,dipstr,dipvec,
    pot,grad,nt,ztarg,ifpgh,isep,ifprint); returns pot (nt,), grad (d, nt) and
    the flags as the library left them (it may clamp them in place)."""
    L = _capi.lib()
    ns, nt = zsrc.shape[1], ztarg.shape[1]
    zs, zt = _cm(zsrc, d, ns), _cm(ztarg, d, nt)
    q = np.ascontiguousarray(charge, np.complex128) if charge is not None else None
    ds = np.ascontiguousarray(dipstr, np.complex128) if dipstr is not None else None
    dv = _cm(dipvec, d, ns) if dipvec is not None else None
    pot = np.full(nt, 7.0 + 7.0j)  # the library zeroes pot and grad before it writes them
    grad = np.asfortranarray(np.full((d, nt), 7.0 + 7.0j))
    fc, fd, fp = ctypes.c_int(ifcharge), ctypes.c_int(ifdipole), ctypes.c_int(ifpgh)
    args = [_d(eps)]
    if zk is not None:
        k = np.array([complex(zk)], np.complex128)
        args.append(_a(k))
    args += [_i(ns), _a(zs), ctypes.byref(fc), _a(q), ctypes.byref(fd), _a(ds), _a(dv), _a(pot),
             _a(grad), _i(nt), _a(zt), ctypes.byref(fp), _i(isep), _i(0)]
    name = ("zl" if zk is None else "zh") + f"fmm{d}d_"
    getattr(L, name)(*args)
    if flags_out is not None:
        flags_out.extend([fc.value, fd.value, fp.value])
    return pot, grad


def direct(d, zk, ztarg, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh):
    """call z{l,h}{d}devaldirect([zk,]nt,ztarg,ns,zsrc,charge,dipstr,dipvec,ifcharge,
    pot,grad,ifdipole,ifpgh) on zero-initialised pot/grad (the routines add)."""
    L = _capi.lib()
    ns, nt = zsrc.shape[1], ztarg.shape[1]
    zs, zt = _cm(zsrc, d, ns), _cm(ztarg, d, nt)
    q = np.ascontiguousarray(charge, np.complex128) if charge is not None else None
    ds = np.ascontiguousarray(dipstr, np.complex128) if dipstr is not None else None
    dv = _cm(dipvec, d, ns) if dipvec is not None else None
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((d, nt), np.complex128, order="F")
    args = []
    if zk is not None:
        k = np.array([complex(zk)], np.complex128)
        args.append(_a(k))
    args += [_i(nt), _a(zt), _i(ns), _a(zs), _a(q), _a(ds), _a(dv), _i(ifcharge), _a(pot),
             _a(grad), _i(ifdipole), _i(ifpgh)]
    name = ("zl" if zk is None else "zh") + f"{d}devaldirect_"
    getattr(L, name)(*args)
    return pot, grad
