"""Reverse-mode (adjoint) 2D Helmholtz FMM on complex-deformed curves.

The forward map is zhfmm2d with sources = targets (reference
zfmm2d/src/helmholtz/zhfmm2d.f:14-227), on points

    z_i = xr_i + 1j * a[curve_i] * disp_i        (xr, disp real (n, 2))

whose imaginary displacement amplitude a[c] is a learnable real parameter per
curve, with charges q and dipole strengths ds (complex), dipole vectors v:

    pot_i = sum_{j != i} q_j G(z_i - z_j) + ds_j (v_j . grad) G(z_i - z_j),
    G(x) = (i/4) H0(zk |x|).

`zhfmm2d_curves` wraps it as a torch.autograd.Function.  The backward pass is
a second FMM run on the transposed problem (G is even, so the transpose is the
same FMM with the roles of sources and targets exchanged), expressed through
the two FMM evaluations with dipole sources of strengths w = conj(grad_pot)
and dipole vectors e+- = (1, +-i):

    F+-(y) = sum_i w_i (e+- . grad_y) G(y - z_i) = D+- u(y),
    u(y) = sum_i w_i G(y - z_i),  D+- = d/dy1 +- i d/dy2,

at the targets y = z_j (i != j, as in the forward).  Their values and
gradients give u = -(D-D+ u)/zk^2 (Helmholtz equation), grad u, D+D+ u and
D-D- u, from which (torch's convention grad = dL/dRe + i dL/dIm):

    dL/dq_j    = conj(u_j)
    dL/dds_j   = conj(-v_j . grad u_j)
    dL/da_c    = Re[ sum_{i in c} w_i zd_i . grad pot_i
                     + sum_{j in c} q_j zd_j . grad u_j - ds_j zd_j^T H_j v_j ]

with zd = dz/da = 1j * disp and zd^T H v = (1/4)[zd- v- D+D+u
+ (zd- v+ + zd+ v-) Du + zd+ v+ D-D-u], x+- = x1 +- i x2, Du = -zk^2 u.  The
target-motion term uses the forward's gradient, so the forward runs with
ifpgh = 2 when a requires a gradient.  The backward costs two FMMs with dipole
sources (about twice a forward solve); the forward and both backward solves
run on one 2D plan (one tree build).

direct=True evaluates every sum above by the FP64 direct sum (zh2devaldirect)
instead of the FMM: the reference gradient of the tests (small n only).
"""
import numpy as np
import torch

from . import Plan2D, zh2devaldirect

__all__ = ["zhfmm2d_curves", "points"]


def points(xr, disp, curve, a):
    """Complex coordinates (n, 2) of the deformed curves."""
    return xr.to(torch.complex128) + 1j * (a[curve].unsqueeze(1) * disp).to(torch.complex128)


def _eval(plan, zk, src, q, ds, dv, tgt, ifpgh, direct):
    """pot (nt,) and grad (2, nt) of sources src (n, 2) at targets tgt (nt, 2),
    scaled as zhfmm2d (i/4 included); through the plan on src (the forward and
    both backward solves share one tree) unless direct."""
    n, nt = src.shape[0], tgt.shape[0]
    ifc = 1 if q is not None else 0
    ifd = 1 if ds is not None else 0
    if not direct:
        pot, grad = plan.zhfmm2d(zk, 1, ifc, q, ifd, ds, dv, ifpgh)
        return pot[0], grad[0]
    c = lambda t: None if t is None else t.detach().cpu().numpy()
    zs = c(src).T
    zt = c(tgt).T
    p, g = zh2devaldirect(zk, nt, zt, n, zs, c(q), c(ds), None if dv is None else c(dv).T, ifc,
                          ifd, ifpgh)
    dev = src.device
    return (torch.from_numpy(p * 0.25j).to(dev),
            torch.from_numpy(np.ascontiguousarray(g * 0.25j)).to(dev))


class _Curves(torch.autograd.Function):
    @staticmethod
    def forward(ctx, charge, dipstr, a, xr, disp, curve, dipvec, eps, zk, direct):
        z = points(xr, disp, curve, a)
        need_g = a.requires_grad
        plan = None if direct else Plan2D(eps, z.shape[0], z, z.shape[0], z)
        pot, grad = _eval(plan, zk, z, charge, dipstr, dipvec, z, 2 if need_g else 1, direct)
        ctx.save_for_backward(charge, dipstr, a, xr, disp, curve, dipvec, z,
                              grad if need_g else torch.empty(0))
        ctx.cfg = (eps, zk, direct, charge is not None, dipstr is not None)
        ctx.plan = plan
        return pot

    @staticmethod
    def backward(ctx, gpot):
        charge, dipstr, a, xr, disp, curve, dipvec, z, gfwd = ctx.saved_tensors
        eps, zk, direct, has_q, has_d = ctx.cfg
        zk = complex(zk)
        n = z.shape[0]
        w = torch.conj_physical(gpot).contiguous()
        dev = z.device
        ep = torch.zeros((n, 2), dtype=torch.complex128, device=dev)
        ep[:, 0] = 1.0
        ep[:, 1] = 1j
        em = torch.conj_physical(ep)
        plan = ctx.plan
        if plan is None and not direct:
            # a second backward over the same graph (retain_graph=True): the
            # first one released the plan, so the tree is built again
            plan = Plan2D(eps, n, z, n, z)
        Fp, Gp = _eval(plan, zk, z, None, w, ep, z, 2, direct)
        Fm, Gm = _eval(plan, zk, z, None, w, em, z, 2, direct)
        ctx.plan = None
        dpdp = Gp[0] + 1j * Gp[1]
        dmdm = Gm[0] - 1j * Gm[1]
        lap = 0.5 * ((Gp[0] - 1j * Gp[1]) + (Gm[0] + 1j * Gm[1]))
        u = -lap / (zk * zk)
        gu1 = 0.5 * (Fp + Fm)
        gu2 = (Fp - Fm) / 2j
        gq = gds = ga = None
        if has_q and ctx.needs_input_grad[0]:
            gq = torch.conj(u)
        if has_d and ctx.needs_input_grad[1]:
            gds = torch.conj(-(dipvec[:, 0] * gu1 + dipvec[:, 1] * gu2))
        if ctx.needs_input_grad[2]:
            zd = 1j * disp.to(torch.complex128)
            zdm, zdp = zd[:, 0] - 1j * zd[:, 1], zd[:, 0] + 1j * zd[:, 1]
            term = w * (zd[:, 0] * gfwd[0] + zd[:, 1] * gfwd[1])
            if has_q:
                term = term + charge * (zd[:, 0] * gu1 + zd[:, 1] * gu2)
            if has_d:
                vm = dipvec[:, 0] - 1j * dipvec[:, 1]
                vp = dipvec[:, 0] + 1j * dipvec[:, 1]
                hess = 0.25 * (zdm * vm * dpdp + (zdm * vp + zdp * vm) * lap + zdp * vp * dmdm)
                term = term - dipstr * hess
            ga = torch.zeros_like(a)
            ga.index_add_(0, curve, term.real)
        return gq, gds, ga, None, None, None, None, None, None, None


def _check_curves(xr, disp, curve, a, charge, dipstr, dipvec):
    """Refuse inputs whose dtype, device or shape the device entry points would
    misread (they take raw data pointers of n complex128 values)."""
    if not isinstance(xr, torch.Tensor) or not xr.is_cuda:
        raise ValueError("xr must be a CUDA tensor")
    dev = xr.device
    if xr.dim() != 2 or xr.shape[1] != 2:
        raise ValueError(f"xr must have shape (n, 2), got {tuple(xr.shape)}")
    n = xr.shape[0]

    def want(t, name, dtype, shape):
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{name} must be a tensor")
        if t.dtype != dtype:
            raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
        if t.device != dev:
            raise ValueError(f"{name} is on {t.device}, xr on {dev}")
        if tuple(t.shape) != shape:
            raise ValueError(f"{name} must have shape {shape}, got {tuple(t.shape)}")

    want(xr, "xr", torch.float64, (n, 2))
    want(disp, "disp", torch.float64, (n, 2))
    want(curve, "curve", torch.int64, (n,))
    if not isinstance(a, torch.Tensor) or a.dim() != 1:
        raise ValueError("a must be a 1-D tensor")
    want(a, "a", torch.float64, (a.shape[0],))
    if charge is None and dipstr is None:
        raise ValueError("charge or dipstr is required")
    if charge is not None:
        want(charge, "charge", torch.complex128, (n,))
    if dipstr is not None:
        want(dipstr, "dipstr", torch.complex128, (n,))
        want(dipvec, "dipvec", torch.complex128, (n, 2))


def zhfmm2d_curves(eps, zk, xr, disp, curve, a, charge, dipstr=None, dipvec=None,
                   direct=False):
    """pot at the points z = xr + 1j a[curve] disp from charges / dipoles at the
    same points (zhfmm2d, sources = targets); differentiable in charge,
    dipstr and the per-curve amplitudes a.  Tensors on one CUDA device:
    xr, disp (n, 2) float64, curve (n,) int64, a (ncurves,) float64, charge
    and dipstr (n,) complex128, dipvec (n, 2) complex128."""
    if zk is None or complex(zk) == 0:
        raise ValueError("zk must be nonzero")
    _check_curves(xr, disp, curve, a, charge, dipstr, dipvec)
    return _Curves.apply(charge, dipstr, a, xr, disp, curve, dipvec, float(eps), complex(zk),
                         bool(direct))
