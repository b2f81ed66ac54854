"""zfmm_b200: complex-coordinate fast multipole methods on NVIDIA B200 (sm_100a).

Python mirror of the reference's MATLAB/mwrap interface
(zfmm2d/matlab_linux/zlfmm2d.mw:1, zl2devaldirect.mw:1): same names, same
argument order and meaning, arrays in the reference's shapes:

    pot, grad = zlfmm2d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr,
                        dipvec, nt, ztarg, ifpgh, isep)

zsrc/ztarg/dipvec are (2, n) complex arrays (MATLAB column layout), charge and
dipstr (n,) complex, pot (nt,), grad (2, nt).  numpy inputs run through the
host-array C entry point; torch CUDA tensors (complex128, shaped (n, 2) or
(2, n) in Fortran order) run through the device entry point on the current
stream.  Everything executes on the GPU; there is no CPU fallback.
"""
import ctypes

import numpy as np

from ._capi import ZfmmError, check, lib

__all__ = ["zlfmm2d", "zl2devaldirect", "zhfmm2d", "zh2devaldirect", "zlfmm3d", "zl3devaldirect",
           "zhfmm3d", "zh3devaldirect", "zl3dterms", "h3dterms", "tree_dump", "ZfmmError",
           "set_step_timing", "last_step_times", "last_counts", "version", "Plan3D", "Plan2D",
           "zlfmm3d_many", "zhfmm3d_many"]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _pts(z, d, n, name):
    """(d, n) complex -> Fortran-ordered complex128 array (memory of zsrc(d,n))."""
    a = np.asarray(z, dtype=np.complex128)
    if a.shape == (n, d) and d != n:
        a = a.T
    if a.shape != (d, n):
        raise ValueError(f"{name} must have shape ({d}, {n}), got {a.shape}")
    return np.asfortranarray(a)


def _vec(v, n, name):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.complex128).reshape(-1))
    if a.size != n:
        raise ValueError(f"{name} must have {n} entries, got {a.size}")
    return a


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _torch_pts(x, d, n, name, device=None):
    import torch
    if not isinstance(x, torch.Tensor) or x.dtype != torch.complex128 or not x.is_cuda:
        raise ValueError(f"{name} must be a complex128 CUDA tensor")
    if device is not None and x.device != device:
        raise ValueError(f"{name} is on {x.device}, the solve runs on {device}")
    x = x.resolve_conj()  # the C entry points read raw memory: no lazy conjugate views
    if tuple(x.shape) == (n, d):
        x = x.contiguous()
    elif tuple(x.shape) == (d, n):
        x = x.t().contiguous()
    else:
        raise ValueError(f"{name} must have shape ({n}, {d}) or ({d}, {n})")
    return x


def _torch_vec(x, n, name, device):
    """A complex128 CUDA tensor of n entries on `device`, as contiguous memory
    (the device entry points read n complex values from its data pointer, so a
    wrong dtype, device or length must be refused here, not read past)."""
    import torch
    if not isinstance(x, torch.Tensor) or x.dtype != torch.complex128 or not x.is_cuda:
        raise ValueError(f"{name} must be a complex128 CUDA tensor")
    if x.device != device:
        raise ValueError(f"{name} is on {x.device}, the solve runs on {device}")
    if x.numel() != n:
        raise ValueError(f"{name} must have {n} entries, got {x.numel()}")
    return x.resolve_conj().contiguous()


def _zk(zk):
    z = complex(zk)
    return np.array([z.real, z.imag], np.float64)


def _fmm2d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh,
           isep):
    if _is_torch(zsrc):
        return _fmm2d_torch(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt,
                            ztarg, ifpgh, isep)
    ns, nt = int(ns), int(nt)
    zs = _pts(zsrc, 2, ns, "zsrc")
    zt = zs if ztarg is zsrc and nt == ns else _pts(ztarg, 2, nt, "ztarg")
    q = _vec(charge, ns, "charge") if ifcharge == 1 else None
    ds = _vec(dipstr, ns, "dipstr") if ifdipole == 1 else None
    dv = _pts(dipvec, 2, ns, "dipvec") if ifdipole == 1 else None
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((2, nt), np.complex128, order="F")
    if zk is None:
        check(lib().zfmm_zlfmm2d(float(eps), ns, _ptr(zs), int(ifcharge), _ptr(q), int(ifdipole),
                                 _ptr(ds), _ptr(dv), _ptr(pot), _ptr(grad), nt, _ptr(zt),
                                 int(ifpgh), int(isep), 0))
    else:
        k = _zk(zk)
        check(lib().zfmm_zhfmm2d(float(eps), _ptr(k), ns, _ptr(zs), int(ifcharge), _ptr(q),
                                 int(ifdipole), _ptr(ds), _ptr(dv), _ptr(pot), _ptr(grad), nt,
                                 _ptr(zt), int(ifpgh), int(isep), 0))
    return pot, grad


def zlfmm2d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh=1,
            isep=1):
    """2D Laplace FMM with complex coordinates (reference zlfmm2d.f:14-234).

    pot(i) = sum_j charge_j log(R_ij)/(2 pi) - dipstr_j <dipvec_j, grad_y log R_ij>/(2 pi),
    R = sqrt((x1-y1)^2 + (x2-y2)^2) on the principal branch.  Returns (pot, grad).
    """
    return _fmm2d(eps, None, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                  ifpgh, isep)


def zhfmm2d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh=1,
            isep=1):
    """2D Helmholtz FMM with complex coordinates (reference zhfmm2d.f:14-227).

    pot(i) = sum_j (i/4) charge_j H0(zk R_ij) + dipole terms, R as in zlfmm2d,
    H0 = H0^(1) on its principal branch.  Argument order of zhfmm2d.mw:1.
    """
    return _fmm2d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                  ifpgh, isep)


def _fmm2d_torch(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh,
                 isep):
    import torch
    zs = _torch_pts(zsrc, 2, ns, "zsrc")
    dev = zs.device
    zt = zs if ztarg is zsrc and nt == ns else _torch_pts(ztarg, 2, nt, "ztarg", dev)
    q = _torch_vec(charge, ns, "charge", dev) if ifcharge == 1 else None
    ds = _torch_vec(dipstr, ns, "dipstr", dev) if ifdipole == 1 else None
    dv = _torch_pts(dipvec, 2, ns, "dipvec", dev) if ifdipole == 1 else None
    pot = torch.empty(nt, dtype=torch.complex128, device=dev)
    grad = torch.empty((nt, 2), dtype=torch.complex128, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
    if zk is None:
        check(lib().zfmm_zlfmm2d_dev(float(eps), int(ns), p(zs), int(ifcharge), p(q),
                                     int(ifdipole), p(ds), p(dv), p(pot), p(grad), int(nt), p(zt),
                                     int(ifpgh), int(isep), stream))
    else:
        k = _zk(zk)
        check(lib().zfmm_zhfmm2d_dev(float(eps), _ptr(k), int(ns), p(zs), int(ifcharge), p(q),
                                     int(ifdipole), p(ds), p(dv), p(pot), p(grad), int(nt), p(zt),
                                     int(ifpgh), int(isep), stream))
    return pot, grad.t()


def _direct2d(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh):
    ns, nt = int(ns), int(nt)
    zs = _pts(zsrc, 2, ns, "zsrc")
    zt = _pts(ztarg, 2, nt, "ztarg")
    q = _vec(charge, ns, "charge") if ifcharge == 1 else None
    ds = _vec(dipstr, ns, "dipstr") if ifdipole == 1 else None
    dv = _pts(dipvec, 2, ns, "dipvec") if ifdipole == 1 else None
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((2, nt), np.complex128, order="F")
    if zk is None:
        check(lib().zfmm_zl2devaldirect(nt, _ptr(zt), ns, _ptr(zs), _ptr(q), _ptr(ds), _ptr(dv),
                                        int(ifcharge), _ptr(pot), _ptr(grad), int(ifdipole),
                                        int(ifpgh)))
    else:
        k = _zk(zk)
        check(lib().zfmm_zh2devaldirect(_ptr(k), nt, _ptr(zt), ns, _ptr(zs), _ptr(q), _ptr(ds),
                                        _ptr(dv), int(ifcharge), _ptr(pot), _ptr(grad),
                                        int(ifdipole), int(ifpgh)))
    return pot, grad


def zl2devaldirect(nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh=1):
    """Unscaled 2D Laplace direct sum (reference zlfmm2d.f:600-654; no 1/(2 pi))."""
    return _direct2d(None, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh)


def zh2devaldirect(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh=1):
    """Unscaled 2D Helmholtz direct sum (reference zhfmm2d.f:773-838; no i/4)."""
    return _direct2d(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh)


def _fmm3d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh,
           isep):
    if _is_torch(zsrc):
        import torch
        zs = _torch_pts(zsrc, 3, ns, "zsrc")
        zt = (zs if ztarg is zsrc and nt == ns
              else _torch_pts(ztarg, 3, nt, "ztarg", zs.device))
        q = _torch_vec(charge, ns, "charge", zs.device) if ifcharge == 1 else None
        ds = _torch_vec(dipstr, ns, "dipstr", zs.device) if ifdipole == 1 else None
        dv = _torch_pts(dipvec, 3, ns, "dipvec", zs.device) if ifdipole == 1 else None
        pot = torch.empty(nt, dtype=torch.complex128, device=zs.device)
        grad = torch.empty((nt, 3), dtype=torch.complex128, device=zs.device)
        stream = ctypes.c_void_p(torch.cuda.current_stream(zs.device).cuda_stream)
        p = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        if zk is None:
            check(lib().zfmm_zlfmm3d_dev(float(eps), int(ns), p(zs), int(ifcharge), p(q),
                                         int(ifdipole), p(ds), p(dv), p(pot), p(grad), int(nt),
                                         p(zt), int(ifpgh), int(isep), stream))
        else:
            k = _zk(zk)
            check(lib().zfmm_zhfmm3d_dev(float(eps), _ptr(k), int(ns), p(zs), int(ifcharge),
                                         p(q), int(ifdipole), p(ds), p(dv), p(pot), p(grad),
                                         int(nt), p(zt), int(ifpgh), int(isep), stream))
        return pot, grad.t()
    ns, nt = int(ns), int(nt)
    zs = _pts(zsrc, 3, ns, "zsrc")
    zt = zs if ztarg is zsrc and nt == ns else _pts(ztarg, 3, nt, "ztarg")
    q = _vec(charge, ns, "charge") if ifcharge == 1 else None
    ds = _vec(dipstr, ns, "dipstr") if ifdipole == 1 else None
    dv = _pts(dipvec, 3, ns, "dipvec") if ifdipole == 1 else None
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((3, nt), np.complex128, order="F")
    if zk is None:
        check(lib().zfmm_zlfmm3d(float(eps), ns, _ptr(zs), int(ifcharge), _ptr(q), int(ifdipole),
                                 _ptr(ds), _ptr(dv), _ptr(pot), _ptr(grad), nt, _ptr(zt),
                                 int(ifpgh), int(isep), 0))
    else:
        k = _zk(zk)
        check(lib().zfmm_zhfmm3d(float(eps), _ptr(k), ns, _ptr(zs), int(ifcharge), _ptr(q),
                                 int(ifdipole), _ptr(ds), _ptr(dv), _ptr(pot), _ptr(grad), nt,
                                 _ptr(zt), int(ifpgh), int(isep), 0))
    return pot, grad


def zlfmm3d(eps, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh=1,
            isep=1):
    """3D Laplace FMM with complex coordinates (reference zlfmm3d.f:14-245).

    pot(i) = sum_j charge_j / (4 pi R_ij) + dipole terms, R = sqrt(sum_k (x_k - y_k)^2)
    on the principal branch.  zsrc, ztarg, dipvec: (3, n) or (n, 3) complex.
    Returns (pot, grad) with grad of shape (3, nt).  numpy inputs run through the
    host-array entry point, complex128 CUDA tensors through the device entry point
    on the current stream (grad then is a (3, nt) view).
    """
    return _fmm3d(eps, None, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                  ifpgh, isep)


def zhfmm3d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg, ifpgh=1,
            isep=1):
    """3D Helmholtz FMM with complex coordinates (reference zhfmm3d.f:1-249).

    pot(i) = sum_j charge_j e^{i zk R_ij} / (4 pi R_ij) + dipole terms, R as in
    zlfmm3d.  Same layouts and return values as zlfmm3d.
    """
    return _fmm3d(eps, zk, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                  ifpgh, isep)


def _direct3d(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh):
    ns, nt = int(ns), int(nt)
    zs = _pts(zsrc, 3, ns, "zsrc")
    zt = _pts(ztarg, 3, nt, "ztarg")
    q = _vec(charge, ns, "charge") if ifcharge == 1 else None
    ds = _vec(dipstr, ns, "dipstr") if ifdipole == 1 else None
    dv = _pts(dipvec, 3, ns, "dipvec") if ifdipole == 1 else None
    pot = np.zeros(nt, np.complex128)
    grad = np.zeros((3, nt), np.complex128, order="F")
    if zk is None:
        check(lib().zfmm_zl3devaldirect(nt, _ptr(zt), ns, _ptr(zs), _ptr(q), _ptr(ds), _ptr(dv),
                                        int(ifcharge), _ptr(pot), _ptr(grad), int(ifdipole),
                                        int(ifpgh)))
    else:
        k = _zk(zk)
        check(lib().zfmm_zh3devaldirect(_ptr(k), nt, _ptr(zt), ns, _ptr(zs), _ptr(q), _ptr(ds),
                                        _ptr(dv), int(ifcharge), _ptr(pot), _ptr(grad),
                                        int(ifdipole), int(ifpgh)))
    return pot, grad


def zl3devaldirect(nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh=1):
    """3D Laplace direct sum with 1/(4 pi) (reference zlfmm3d.f:628-683)."""
    return _direct3d(None, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh)


def zh3devaldirect(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh=1):
    """3D Helmholtz direct sum with 1/(4 pi) (reference zhfmm3d.f:626-693)."""
    return _direct3d(zk, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, ifdipole, ifpgh)


def _mat(v, nd, n, name):
    """(nd, n) complex, right-hand side fastest in memory (Fortran order)."""
    a = np.asarray(v, dtype=np.complex128)
    if nd == 1 and a.ndim == 1:
        a = a.reshape(1, -1)
    if a.shape != (nd, n):
        raise ValueError(f"{name} must have shape ({nd}, {n}), got {a.shape}")
    return np.asfortranarray(a)


class _Plan:
    """Geometry of a complex-coordinate FMM built once and reused (base of
    Plan2D / Plan3D)."""

    D = 3
    _fn = {}

    def __init__(self, eps, ns, zsrc, nt, ztarg, isep=1):
        self._h = ctypes.c_void_p()
        self.ns, self.nt, self.eps = int(ns), int(nt), float(eps)
        d = self.D
        if _is_torch(zsrc):
            import torch
            zs = _torch_pts(zsrc, d, self.ns, "zsrc")
            zt = (zs if ztarg is zsrc and self.nt == self.ns
                  else _torch_pts(ztarg, d, self.nt, "ztarg", zs.device))
            self.device = zs.device
            stream = ctypes.c_void_p(torch.cuda.current_stream(zs.device).cuda_stream)
            check(getattr(lib(), self._fn["create_dev"])(
                self.eps, self.ns, ctypes.c_void_p(zs.data_ptr()), self.nt,
                ctypes.c_void_p(zt.data_ptr()), int(isep), stream, ctypes.byref(self._h)))
        else:
            self.device = None
            zs = _pts(zsrc, d, self.ns, "zsrc")
            zt = zs if ztarg is zsrc and self.nt == self.ns else _pts(ztarg, d, self.nt, "ztarg")
            check(getattr(lib(), self._fn["create"])(self.eps, self.ns, _ptr(zs), self.nt,
                                                     _ptr(zt), int(isep), ctypes.byref(self._h)))

    def save(self, path):
        """Write the plan's geometry (tree, point order, centres, lists) to a
        plan file that load() reads back in a later process."""
        import os
        check(getattr(lib(), self._fn["save"])(self._h, os.fsencode(str(path))))

    @classmethod
    def load(cls, path):
        """A plan read from a file written by save(), on the current device."""
        import os
        self = cls.__new__(cls)
        self._h = ctypes.c_void_p()
        check(getattr(lib(), cls._fn["load"])(os.fsencode(str(path)), ctypes.byref(self._h)))
        nb, nl, ns, nt = (ctypes.c_int() for _ in range(4))
        check(getattr(lib(), cls._fn["info"])(self._h, ctypes.byref(nb), ctypes.byref(nl),
                                              ctypes.byref(ns), ctypes.byref(nt)))
        self.ns, self.nt, self.eps = ns.value, nt.value, None
        self.device = None
        try:
            import torch
            if torch.cuda.is_available():
                self.device = torch.device("cuda", torch.cuda.current_device())
        except ImportError:
            pass
        return self

    def info(self):
        """(nboxes, nlevels) of the plan's tree."""
        nb, nl, a, b = (ctypes.c_int() for _ in range(4))
        check(getattr(lib(), self._fn["info"])(self._h, ctypes.byref(nb), ctypes.byref(nl),
                                               ctypes.byref(a), ctypes.byref(b)))
        return nb.value, nl.value

    def _solve(self, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh):
        nd, ns, nt, d = int(nd), self.ns, self.nt, self.D
        k = None if zk is None else _zk(zk)
        L = lib()
        if _is_torch(charge if ifcharge == 1 else dipstr):
            import torch
            dev = self.device
            if dev is None:
                raise ValueError("this plan was built from host arrays: pass numpy strengths")
            q = _torch_vec(charge, ns * nd, "charge", dev) if ifcharge == 1 else None
            ds = _torch_vec(dipstr, ns * nd, "dipstr", dev) if ifdipole == 1 else None
            dv = _torch_pts(dipvec, d, ns, "dipvec", dev) if ifdipole == 1 else None
            pot = torch.empty((nt, nd), dtype=torch.complex128, device=dev)
            grad = torch.empty((nt, d, nd), dtype=torch.complex128, device=dev)
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            p = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
            if k is None:
                check(getattr(L, self._fn["lap_dev"])(self._h, nd, int(ifcharge), p(q),
                                                      int(ifdipole), p(ds), p(dv), int(ifpgh),
                                                      p(pot), p(grad), stream))
            else:
                check(getattr(L, self._fn["helm_dev"])(self._h, _ptr(k), nd, int(ifcharge), p(q),
                                                       int(ifdipole), p(ds), p(dv), int(ifpgh),
                                                       p(pot), p(grad), stream))
            return pot.t(), grad.permute(2, 1, 0)
        q = _mat(charge, nd, ns, "charge") if ifcharge == 1 else None
        ds = _mat(dipstr, nd, ns, "dipstr") if ifdipole == 1 else None
        dv = _pts(dipvec, d, ns, "dipvec") if ifdipole == 1 else None
        pot = np.zeros((nd, nt), np.complex128, order="F")
        grad = np.zeros((nd, d, nt), np.complex128, order="F")
        if k is None:
            check(getattr(L, self._fn["lap"])(self._h, nd, int(ifcharge), _ptr(q), int(ifdipole),
                                              _ptr(ds), _ptr(dv), int(ifpgh), _ptr(pot),
                                              _ptr(grad)))
        else:
            check(getattr(L, self._fn["helm"])(self._h, _ptr(k), nd, int(ifcharge), _ptr(q),
                                               int(ifdipole), _ptr(ds), _ptr(dv), int(ifpgh),
                                               _ptr(pot), _ptr(grad)))
        return pot, grad

    def close(self):
        if self._h:
            check(getattr(lib(), self._fn["destroy"])(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan3D(_Plan):
    """Geometry of a 3D complex-coordinate FMM built once and reused.

    The octree on the real parts, the sorted and rescaled points, the complex
    box centres and the interaction lists (the set-up of zlfmm3d.f:60-200) are
    built on the GPU when the plan is created; every solve then only forms,
    translates and evaluates expansions, for nd right-hand sides at a time.

        plan = Plan3D(eps, ns, zsrc, nt, ztarg, isep=1)
        pot, grad = plan.zlfmm3d(nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh)

    numpy: zsrc (3, ns), ztarg (3, nt); charge and dipstr (nd, ns); dipvec (3, ns),
    shared by the right-hand sides; returns pot (nd, nt) and grad (nd, 3, nt).
    torch (complex128 CUDA): zsrc (ns, 3), charge (ns, nd) contiguous; returns
    views shaped (nd, nt) and (nd, 3, nt) of right-hand-side-fastest storage.
    """

    D = 3
    _fn = dict(create="zfmm_plan3d_create", create_dev="zfmm_plan3d_create_dev",
               save="zfmm_plan3d_save", load="zfmm_plan3d_load",
               info="zfmm_plan3d_info", destroy="zfmm_plan3d_destroy", lap="zfmm_zlfmm3d_plan",
               lap_dev="zfmm_zlfmm3d_plan_dev", helm="zfmm_zhfmm3d_plan",
               helm_dev="zfmm_zhfmm3d_plan_dev")

    def zlfmm3d(self, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh=1):
        """3D Laplace FMM of nd right-hand sides on the plan's points."""
        return self._solve(None, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh)

    def zhfmm3d(self, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh=1):
        """3D Helmholtz FMM (wavenumber zk) of nd right-hand sides on the plan's points."""
        return self._solve(zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh)


class Plan2D(_Plan):
    """Geometry of a 2D complex-coordinate FMM (quadtree, sorted points,
    complex centres, lists; zlfmm2d.f:70-200) built once and reused by solves
    of nd right-hand sides at any wavenumber, as Plan3D with d = 2: charge and
    dipstr (nd, ns), dipvec (2, ns) shared, pot (nd, nt), grad (nd, 2, nt)."""

    D = 2
    _fn = dict(create="zfmm_plan2d_create", create_dev="zfmm_plan2d_create_dev",
               save="zfmm_plan2d_save", load="zfmm_plan2d_load",
               info="zfmm_plan2d_info", destroy="zfmm_plan2d_destroy", lap="zfmm_zlfmm2d_plan",
               lap_dev="zfmm_zlfmm2d_plan_dev", helm="zfmm_zhfmm2d_plan",
               helm_dev="zfmm_zhfmm2d_plan_dev")

    def zlfmm2d(self, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh=1):
        """2D Laplace FMM of nd right-hand sides on the plan's points."""
        return self._solve(None, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh)

    def zhfmm2d(self, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh=1):
        """2D Helmholtz FMM (wavenumber zk) of nd right-hand sides on the plan's points."""
        return self._solve(zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh)


def _many(eps, zk, instances, ifcharge, ifdipole, ifpgh, isep, nstreams):
    n = len(instances)
    keep = []
    ns = np.zeros(n, np.int32)
    nt = np.zeros(n, np.int32)
    P = lambda: (ctypes.c_void_p * n)()
    zs, zt, q, ds, dv, pot, grad = P(), P(), P(), P(), P(), P(), P()
    outs = []
    for i, inst in enumerate(instances):
        a = _pts(inst["zsrc"], 3, np.asarray(inst["zsrc"]).shape[-1], "zsrc")
        ns[i] = a.shape[1]
        t = _pts(inst["ztarg"], 3, np.asarray(inst["ztarg"]).shape[-1], "ztarg") \
            if inst.get("ztarg") is not None else a
        nt[i] = t.shape[1]
        zs[i], zt[i] = _ptr(a), _ptr(t)
        keep += [a, t]
        if ifcharge == 1:
            c = _vec(inst["charge"], ns[i], "charge")
            q[i] = _ptr(c)
            keep.append(c)
        if ifdipole == 1:
            d = _vec(inst["dipstr"], ns[i], "dipstr")
            v = _pts(inst["dipvec"], 3, ns[i], "dipvec")
            ds[i], dv[i] = _ptr(d), _ptr(v)
            keep += [d, v]
        po = np.zeros(nt[i], np.complex128)
        gr = np.zeros((3, nt[i]), np.complex128, order="F")
        pot[i], grad[i] = _ptr(po), _ptr(gr)
        outs.append((po, gr))
    done = np.zeros(n, np.float64)
    if zk is None:
        check(lib().zfmm_zlfmm3d_many(n, float(eps), _ptr(ns), zs, int(ifcharge), q,
                                      int(ifdipole), ds, dv, _ptr(nt), zt, int(ifpgh), int(isep),
                                      pot, grad, int(nstreams), _ptr(done)))
    else:
        k = _zk(zk)
        check(lib().zfmm_zhfmm3d_many(n, float(eps), _ptr(k), _ptr(ns), zs, int(ifcharge), q,
                                      int(ifdipole), ds, dv, _ptr(nt), zt, int(ifpgh), int(isep),
                                      pot, grad, int(nstreams), _ptr(done)))
    return outs, done


def zlfmm3d_many(eps, instances, ifcharge=1, ifdipole=0, ifpgh=1, isep=1, nstreams=8):
    """Many independent zlfmm3d solves in one call.  instances: list of dicts
    with zsrc (3, ns), charge, dipstr, dipvec (3, ns) and optional ztarg
    (default: the sources).  Returns ([(pot, grad), ...], done_ms): each
    instance's outputs as zlfmm3d's and its completion time (ms after the call
    started)."""
    return _many(eps, None, instances, ifcharge, ifdipole, ifpgh, isep, nstreams)


def zhfmm3d_many(eps, zk, instances, ifcharge=1, ifdipole=0, ifpgh=1, isep=1, nstreams=8):
    """Many independent zhfmm3d solves (shared zk) in one call; as zlfmm3d_many."""
    return _many(eps, zk, instances, ifcharge, ifdipole, ifpgh, isep, nstreams)


def h3dterms(size, zk, eps, isep=1):
    """Expansion order of the 3D Helmholtz FMM (reference h3dterms.f:16-75)."""
    k = _zk(zk)
    return int(lib().zfmm_h3dterms(float(size), _ptr(k), float(eps), int(isep)))


def zl3dterms(eps):
    """Expansion order of the 3D Laplace FMM (reference zlfmm3d.f:1283-1321)."""
    return int(lib().zfmm_zl3dterms(float(eps)))


def tree_dump(D, ndiv, zsrc, ztarg=None, isep=1):
    """Device tree, sort and lists for the real parts of zsrc/ztarg ((n, D) complex)."""
    zs = np.ascontiguousarray(np.asarray(zsrc, np.complex128))
    zt = zs if ztarg is None else np.ascontiguousarray(np.asarray(ztarg, np.complex128))
    ns, nt = zs.shape[0], zt.shape[0]
    nb, nl, tot = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    mnl = np.zeros(4, np.int32)
    L = lib()
    z = [None] * 12
    check(L.zfmm_tree_dump(D, ndiv, isep, ns, _ptr(zs), nt, _ptr(zt), 0, 0, ctypes.byref(nb),
                           ctypes.byref(nl), *z, ctypes.byref(tot), _ptr(mnl)))
    n, NC = nb.value, 1 << D
    o = dict(laddr=np.zeros(2 * (nl.value + 1), np.int32), ilevel=np.zeros(n, np.int32),
             iparent=np.zeros(n, np.int32), nchild=np.zeros(n, np.int32),
             ichild=np.zeros((n, NC), np.int32), centers=np.zeros((n, D)),
             isrc=np.zeros(ns, np.int32), isrcse=np.zeros((n, 2), np.int32),
             itarg=np.zeros(nt, np.int32), itargse=np.zeros((n, 2), np.int32),
             nlist=np.zeros((4, n), np.int32))
    cap = 400 * n + 1000
    flat = np.zeros(cap, np.int32)
    check(L.zfmm_tree_dump(D, ndiv, isep, ns, _ptr(zs), nt, _ptr(zt), n, cap, ctypes.byref(nb),
                           ctypes.byref(nl), _ptr(o["laddr"]), _ptr(o["ilevel"]),
                           _ptr(o["iparent"]), _ptr(o["nchild"]), _ptr(o["ichild"]),
                           _ptr(o["centers"]), _ptr(o["isrc"]), _ptr(o["isrcse"]),
                           _ptr(o["itarg"]), _ptr(o["itargse"]), _ptr(o["nlist"]), _ptr(flat),
                           ctypes.byref(tot), _ptr(mnl)))
    o["lists_flat"] = flat[:tot.value]
    o["nboxes"] = n
    o["nlevels"] = nl.value
    o["laddr"] = o["laddr"].reshape(-1, 2)
    o["mnlist"] = mnl.tolist()
    return o


def set_step_timing(on=True):
    lib().zfmm_set_step_timing(1 if on else 0)


def last_step_times():
    ms = np.zeros(7)
    nb, nl, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().zfmm_last_step_times(_ptr(ms), ctypes.byref(nb), ctypes.byref(nl), ctypes.byref(nt))
    names = ["setup", "p2m", "m2m", "m2l_p2l", "l2l", "eval", "unsort"]
    return dict(zip(names, ms.tolist())), dict(nboxes=nb.value, nlevels=nl.value,
                                                 nterms=nt.value)


def last_counts():
    """Interaction counts and kernel launches of the last timed FMM call."""
    c = np.zeros(16, np.int64)
    nl = ctypes.c_long()
    lib().zfmm_last_counts(_ptr(c), ctypes.byref(nl))
    names = ["p2p_pairs", "m2t", "l2t", "m2l_pairs", "p2l", "m2m_pairs", "l2l_pairs", "p2m"]
    d = dict(zip(names, c[:8].tolist()))
    d.update({k + "_P": v for k, v in zip(names, c[8:].tolist()) if k != "p2p_pairs"})
    return d, nl.value


def last_level_counts():
    """Per-level interaction counts and expansion orders of the last 3D FMM
    call made with set_step_timing(2): ({name: [count per level]}, [order per
    level])."""
    c = np.zeros(8 * 64, np.int64)
    o = np.zeros(64, np.int32)
    nl = ctypes.c_int()
    lib().zfmm_last_level_counts(_ptr(c), _ptr(o), ctypes.byref(nl))
    L = nl.value + 1
    names = ["p2p_pairs", "m2t", "l2t", "m2l_pairs", "p2l", "m2m_pairs", "l2l_pairs", "p2m"]
    c = c.reshape(8, 64)
    return {k: c[i, :L].tolist() for i, k in enumerate(names)}, o[:L].tolist()


def version():
    return lib().zfmm_version().decode()
