"""Layer-potential operator for Krylov solvers (zfmm_b200.operator): one
matvec equals the zhfmm2d potentials of charge alpha x and dipole strength
beta x (checked against the FP64 direct sum), a block of densities through
matmat equals the same number of matvecs, the CUDA-tensor operator equals the
host one, and scipy's GMRES solves a system with it."""
import numpy as np
import pytest
import torch

import zfmm_b200 as zf
from zfmm_b200 import workloads as W
from zfmm_b200.operator import Helm2DLayerOperator

pytestmark = pytest.mark.gpu

ZK = 12.0 + 0.2j


def _geometry(n, seed):
    w = W.curve2d(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return np.asfortranarray(w["zsrc"]), np.asfortranarray(w["dipvec"]), x


def test_matvec_against_direct_sum():
    n = 4000
    z, dv, x = _geometry(n, 3)
    A = Helm2DLayerOperator(1e-12, ZK, z, dipvec=dv, alpha=1.0, beta=0.5)
    try:
        y = A.matvec(x)
    finally:
        A.close()
    pd, _ = zf.zh2devaldirect(ZK, n, z, n, z, x, 0.5 * x, dv, 1, 1, 1)
    pd = 0.25j * pd  # the direct sum leaves out the factor i/4
    assert np.linalg.norm(y - pd) / np.linalg.norm(pd) < 1e-10


def test_matmat_equals_matvecs():
    n = 3000
    z, dv, _ = _geometry(n, 4)
    rng = np.random.default_rng(5)
    X = rng.standard_normal((n, 6)) + 1j * rng.standard_normal((n, 6))
    A = Helm2DLayerOperator(1e-10, ZK, z, dipvec=dv, alpha=1.0, beta=-0.3j)
    try:
        Y = A.matmat(X)
        cols = np.stack([A.matvec(X[:, j]) for j in range(6)], axis=1)
    finally:
        A.close()
    assert Y.shape == (n, 6)
    assert np.linalg.norm(Y - cols) / np.linalg.norm(cols) < 1e-12


def test_cuda_tensor_operator_equals_host():
    n = 3000
    z, dv, x = _geometry(n, 6)
    dev = torch.device("cuda:0")
    A = Helm2DLayerOperator(1e-10, ZK, z, dipvec=dv, alpha=0.7, beta=1.0)
    At = Helm2DLayerOperator(1e-10, ZK, torch.from_numpy(np.ascontiguousarray(z.T)).to(dev),
                             dipvec=torch.from_numpy(np.ascontiguousarray(dv.T)).to(dev),
                             alpha=0.7, beta=1.0)
    try:
        y = A.matvec(x)
        yt = At.matvec(torch.from_numpy(x).to(dev)).cpu().numpy()
        X = np.stack([x, 2 * x, 1j * x], axis=1)
        Yt = At.matmat(torch.from_numpy(X).to(dev)).cpu().numpy()
    finally:
        A.close()
        At.close()
    assert np.linalg.norm(yt - y) / np.linalg.norm(y) < 1e-13
    assert np.linalg.norm(Yt[:, 1] - 2 * y) / np.linalg.norm(y) < 1e-12


def test_gmres_solve():
    from scipy.sparse.linalg import LinearOperator, gmres
    n = 2000
    z, dv, _ = _geometry(n, 7)
    rng = np.random.default_rng(8)
    A = Helm2DLayerOperator(1e-10, ZK, z, dipvec=dv, alpha=1.0, beta=0.5)
    try:
        L = A.as_linear_operator()
        # scale so that c A is a small perturbation of the identity
        v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        c = 0.05 * np.linalg.norm(v) / np.linalg.norm(L.matvec(v))
        M = LinearOperator((n, n), matvec=lambda u: u + c * L.matvec(u), dtype=np.complex128)
        b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        sol, info = gmres(M, b, rtol=1e-10, atol=0.0, restart=50, maxiter=20)
        assert info == 0
        res = np.linalg.norm(M.matvec(sol) - b) / np.linalg.norm(b)
        assert res < 1e-9
    finally:
        A.close()
