"""Adjoint 2D Helmholtz FMM (zfmm_b200.adjoint) on two complex-deformed curves.

The inner curve is the outer one scaled 0.3 and shifted by (0.2, 0.1), with an
imaginary amplitude scaled alike: with the two amplitudes equal, or the copy
scaled 0.6 and crossing the outer curve, the reference algorithm itself (the
oracle) misses the direct sum by orders of magnitude (expansions about
complex centres of boxes that hold both curves), so no gradient could be
checked there.

The gradients of loss = mean |pot - ref|^2 with respect to the charges, the
dipole strengths and the two imaginary-displacement amplitudes must agree with
(1) the same adjoint formulas evaluated by the FP64 direct sum, and (2) central
finite differences of the FMM loss (h = 1e-6 for the amplitudes); torch's convention for complex
leaves is grad = dL/dRe + i dL/dIm."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def two_curves(n, seed):
    rng = np.random.default_rng(seed)
    m = n // 2
    xr, disp, curve = [], [], []
    for c, (sc, sh) in enumerate([(1.0, (0.0, 0.0)), (0.3, (0.2, 0.1))]):
        t = rng.uniform(0, 2 * np.pi, m)
        r = 1.0 + 0.3 * np.cos(5 * t)
        xr.append(np.stack([sc * r * np.cos(t) + sh[0], sc * r * np.sin(t) + sh[1]], 1))
        disp.append(np.stack([np.cos(3 * t), np.sin(3 * t)], 1))
        curve.append(np.full(m, c))
    cn = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return (np.concatenate(xr), np.concatenate(disp), np.concatenate(curve), cn(2 * m),
            cn(2 * m), cn(2 * m, 2), cn(2 * m))


def setup(n, seed=3):
    import torch
    xr, disp, curve, q, ds, dv, ref = two_curves(n, seed)
    T = lambda x, **k: torch.tensor(x, device="cuda", **k)
    return dict(xr=T(xr), disp=T(disp), curve=T(curve), q=T(q), ds=T(ds), dv=T(dv), ref=T(ref))


def loss_and_grads(D, eps, zk, a0, direct=False, grads=True):
    import torch
    from zfmm_b200.adjoint import zhfmm2d_curves
    q = D["q"].clone().requires_grad_(grads)
    ds = D["ds"].clone().requires_grad_(grads)
    a = torch.tensor(a0, device="cuda", dtype=torch.float64, requires_grad=grads)
    pot = zhfmm2d_curves(eps, zk, D["xr"], D["disp"], D["curve"], a, q, ds, D["dv"],
                         direct=direct)
    L = torch.mean(torch.abs(pot - D["ref"]) ** 2)
    if not grads:
        return float(L)
    L.backward()
    return float(L.detach()), q.grad.cpu().numpy(), ds.grad.cpu().numpy(), a.grad.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def test_adjoint_matches_direct_sum_gradient():
    eps, zk = 1e-10, 20 + 0.3j
    D = setup(3000)
    a0 = [0.05, 0.015]
    L, gq, gds, ga = loss_and_grads(D, eps, zk, a0)
    Ld, gqd, gdsd, gad = loss_and_grads(D, eps, zk, a0, direct=True)
    assert abs(L - Ld) / Ld < 1e-8
    assert rel(gq, gqd) < 1e-7
    assert rel(gds, gdsd) < 1e-7
    assert rel(ga, gad) < 1e-6


def test_adjoint_matches_finite_differences():
    eps, zk, h = 1e-10, 20 + 0.3j, 1e-6
    D = setup(3000, seed=4)
    a0 = [0.05, 0.012]
    L, gq, gds, ga = loss_and_grads(D, eps, zk, a0)
    for c in range(2):
        ap, am = list(a0), list(a0)
        ap[c] += h
        am[c] -= h
        fd = (loss_and_grads(D, eps, zk, ap, grads=False)
              - loss_and_grads(D, eps, zk, am, grads=False)) / (2 * h)
        assert abs(fd - ga[c]) <= 1e-5 * abs(ga[c]), (c, fd, ga[c])
    # the loss is quadratic in the strengths, so central differences are exact
    # there for any step; a step of 1e-2 keeps the difference far above the
    # rounding of the loss
    hq = 1e-2
    for key, g in (("q", gq), ("ds", gds)):
        for k in (0, 1234):
            for part, unit in ((0, 1.0), (1, 1j)):
                Dp = dict(D)
                Dm = dict(D)
                Dp[key] = D[key].clone()
                Dm[key] = D[key].clone()
                Dp[key][k] += hq * unit
                Dm[key][k] -= hq * unit
                fd = (loss_and_grads(Dp, eps, zk, a0, grads=False)
                      - loss_and_grads(Dm, eps, zk, a0, grads=False)) / (2 * hq)
                want = g[k].real if part == 0 else g[k].imag
                assert abs(fd - want) <= 1e-5 * abs(g[k]), (key, k, part, fd, want)
