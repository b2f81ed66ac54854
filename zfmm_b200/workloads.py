"""Seeded synthetic inputs with the shapes and distributions of the benchmark
configurations (no external data).  Arrays are returned in the reference's
layouts: points (d, n) complex, strengths (n,) complex.
"""
import numpy as np


def cnormal(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)


def lap2d_uniform(n=20000, seed=0):
    """zlfmm2d plain solve: real parts U[-1,1]^2, imaginary parts
    0.1*sin(pi x1)*cos(pi x2) on each coordinate, complex normal charges and
    dipole strengths, real unit dipole vectors at uniform angles."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=(2, n))
    im = 0.1 * np.sin(np.pi * x[0]) * np.cos(np.pi * x[1])
    z = x + 1j * im[None, :]
    q = cnormal(rng, n)
    ds = cnormal(rng, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    dv = np.stack([np.cos(phi), np.sin(phi)]).astype(np.complex128)
    return dict(zsrc=z, charge=q, dipstr=ds, dipvec=dv)


def curve2d(n=2_000_000, seed=0, scale=1.0, shift=(0.0, 0.0), amp=0.05):
    """Complex-deformed closed curve r(t) = (1+0.3cos5t)(cos t, sin t)
    + amp*i*(cos3t, sin3t), t uniform on [0, 2pi)."""
    rng = np.random.default_rng(seed)
    t = rng.uniform(0.0, 2 * np.pi, n)
    r = 1.0 + 0.3 * np.cos(5 * t)
    z = np.stack([scale * r * np.cos(t) + shift[0], scale * r * np.sin(t) + shift[1]]) \
        + 1j * amp * np.stack([np.cos(3 * t), np.sin(3 * t)])
    return dict(zsrc=z.astype(np.complex128), charge=cnormal(rng, n), dipstr=cnormal(rng, n),
                dipvec=cnormal(rng, 2, n))


def clustered2d(n, seed=0, nclusters=5):
    """Strongly non-uniform points (Gaussian clusters of different widths):
    exercises deep adaptive refinement and the level-restriction passes."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, size=(nclusters, 2))
    w = 10.0 ** rng.uniform(-3, -1, nclusters)
    k = rng.integers(0, nclusters, n)
    x = c[k].T + w[k][None, :] * rng.standard_normal((2, n))
    im = 0.05 * np.sin(3 * x[0]) * np.cos(2 * x[1])
    z = x + 1j * im[None, :]
    return dict(zsrc=z, charge=cnormal(rng, n), dipstr=cnormal(rng, n), dipvec=cnormal(rng, 2, n))


def lap3d_uniform(n=1_000_000, seed=0, nrhs=1, amp=0.05):
    """zlfmm3d batched solve: real parts U[-1,1]^3, imaginary parts
    amp*(sin 2pi x2, sin 2pi x3, sin 2pi x1) (amp = 0.05 in the benchmark); nrhs complex normal charge
    vectors (charge has shape (n,) for nrhs == 1, else (nrhs, n)); dipole
    strengths complex normal and real unit dipole vectors for the tests that
    use them."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=(3, n))
    im = amp * np.stack([np.sin(2 * np.pi * x[1]), np.sin(2 * np.pi * x[2]),
                         np.sin(2 * np.pi * x[0])])
    z = x + 1j * im
    q = cnormal(rng, n) if nrhs == 1 else cnormal(rng, nrhs, n)
    ds = cnormal(rng, n)
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0, keepdims=True)
    return dict(zsrc=z, charge=q, dipstr=ds, dipvec=v.astype(np.complex128))


def clustered3d(n, seed=0, nclusters=4):
    """Gaussian clusters of different widths in 3D (adaptive octree with
    non-empty lists 3 and 4), small smooth imaginary parts, complex dipoles."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, size=(nclusters, 3))
    w = 10.0 ** rng.uniform(-2, -0.5, nclusters)
    k = rng.integers(0, nclusters, n)
    x = c[k].T + w[k][None, :] * rng.standard_normal((3, n))
    im = 0.03 * np.stack([np.sin(3 * x[1]), np.cos(2 * x[2]), np.sin(x[0] + x[1])])
    z = x + 1j * im
    return dict(zsrc=z, charge=cnormal(rng, n), dipstr=cnormal(rng, n), dipvec=cnormal(rng, 3, n))


def sphere3d(n, seed=0, amp=0.1):
    """Points uniform on the unit sphere, displaced by amp*i times the outward
    normal scaled by a random smooth field of degree 4 (a seeded polynomial
    of degree <= 4 in x, y, z, normalised to max |f| = 1 on the points);
    complex normal charges and dipole strengths, complex normal dipole
    vectors."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0, keepdims=True)
    f = np.zeros(n)
    for a in range(5):
        for b in range(5 - a):
            for c in range(5 - a - b):
                f += rng.standard_normal() * v[0] ** a * v[1] ** b * v[2] ** c
    f /= np.abs(f).max()
    z = v + 1j * amp * f[None, :] * v
    return dict(zsrc=z, charge=cnormal(rng, n), dipstr=cnormal(rng, n), dipvec=cnormal(rng, 3, n))
