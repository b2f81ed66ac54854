"""Layer-potential operators on a fixed geometry, for Krylov solvers.

A boundary-integral solve applies the same FMM to new densities in every
iteration: the reference's transmission-problem demo calls zhfmm2d once for
the single-layer and once for the double-layer part of every GMRES matvec
(zfmm2d/demos, solver_apply_A_fmm.m).  `Helm2DLayerOperator` builds the
geometry once (a `Plan2D`) and applies

    (A x)_i = sum_j [ alpha x_j (i/4) H0(zk R_ij)
                      + beta  x_j (dipole term of zhfmm2d with dipvec_j) ]

(the potentials of zhfmm2d with charge alpha x and dipole strength beta x,
the self-pair left out as zhfmm2d leaves it out), so a combined-field
operator costs one FMM per matvec.  `matmat` applies it to k densities at
once through the plan's batched right-hand-side path.  Host arrays (numpy)
or complex128 CUDA tensors work alike; `as_linear_operator()` gives a
`scipy.sparse.linalg.LinearOperator` for scipy's Krylov solvers.
"""
import numpy as np

from . import Plan2D

__all__ = ["Helm2DLayerOperator"]


def _is_torch(x):
    return type(x).__module__.startswith("torch")


class Helm2DLayerOperator:
    """alpha S + beta D of zhfmm2d on the points zsrc (complex, (2, n) or
    (n, 2)), evaluated at ztarg (default: the sources themselves)."""

    def __init__(self, eps, zk, zsrc, dipvec=None, alpha=1.0, beta=0.0, ztarg=None, isep=1):
        self.zk = complex(zk)
        self.alpha, self.beta = complex(alpha), complex(beta)
        if self.beta != 0 and dipvec is None:
            raise ValueError("a double-layer part (beta != 0) needs dipvec")
        self._torch = _is_torch(zsrc)
        ns = zsrc.shape[-1] if tuple(zsrc.shape)[0] == 2 and zsrc.shape[-1] != 2 else zsrc.shape[0]
        if ztarg is None:
            ztarg, nt = zsrc, ns
        else:
            nt = ztarg.shape[-1] if tuple(ztarg.shape)[0] == 2 and ztarg.shape[-1] != 2 \
                else ztarg.shape[0]
        self.ns, self.nt = int(ns), int(nt)
        self.dipvec = dipvec
        self.plan = Plan2D(eps, self.ns, zsrc, self.nt, ztarg, isep)

    @property
    def shape(self):
        return (self.nt, self.ns)

    dtype = np.complex128

    def _apply(self, X, k):
        """X: (k, ns) densities -> (k, nt) potentials."""
        ifc = 1 if self.alpha != 0 else 0
        ifd = 1 if self.beta != 0 else 0
        if not ifc and not ifd:
            return X.new_zeros(k, self.nt) if self._torch else np.zeros((k, self.nt), np.complex128)
        # the plan's device path reads right-hand sides fastest: (ns, k) rows
        lay = (lambda Y: Y.t().contiguous()) if self._torch else (lambda Y: Y)
        q = lay(self.alpha * X) if ifc else None
        ds = lay(self.beta * X) if ifd else None
        pot, _ = self.plan.zhfmm2d(self.zk, k, ifc, q, ifd, ds, self.dipvec if ifd else None, 1)
        return pot

    def matvec(self, x):
        """A x for one density of ns entries; returns nt potentials."""
        X = x.reshape(1, -1)
        if X.shape[1] != self.ns:
            raise ValueError(f"x must have {self.ns} entries, got {X.shape[1]}")
        return self._apply(X, 1).reshape(-1)

    def matmat(self, X):
        """A X for an (ns, k) block of densities; returns (nt, k).  The k
        densities share one pass of the FMM (batched right-hand sides)."""
        if X.shape[0] != self.ns:
            raise ValueError(f"X must have {self.ns} rows, got {X.shape[0]}")
        k = X.shape[1]
        Xt = X.T.contiguous() if self._torch else np.ascontiguousarray(X.T)
        return self._apply(Xt, k).T

    def as_linear_operator(self):
        """The operator as a scipy.sparse.linalg.LinearOperator (host arrays)."""
        from scipy.sparse.linalg import LinearOperator
        if self._torch:
            raise ValueError("built from CUDA tensors: scipy needs a host-array operator")
        return LinearOperator(self.shape, matvec=lambda x: self.matvec(np.asarray(x)),
                              matmat=lambda X: self.matmat(np.asarray(X)),
                              dtype=np.complex128)

    def close(self):
        self.plan.close()
