"""A Fortran program using the library through include/zfmm.f90 (compiled
with gfortran where one is installed; skipped otherwise): the module compiles,
the program links against libzfmm_b200, and on a GPU its results equal the
Python binding's, the out-of-range flag comes back clamped, and a bad call
returns status 1 with the library's message."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "zfmm_b200")


def _build(tmp_path):
    fc = shutil.which("gfortran")
    if fc is None:
        pytest.skip("no Fortran compiler on this machine")
    exe = os.path.join(str(tmp_path), "drop_in")
    subprocess.run([fc, "-c", os.path.join(ROOT, "include", "zfmm.f90"), "-J", str(tmp_path),
                    "-o", os.path.join(str(tmp_path), "zfmm.o")], check=True)
    subprocess.run([fc, "-I", str(tmp_path), os.path.join(ROOT, "tests", "fortran", "drop_in.f90"),
                    os.path.join(str(tmp_path), "zfmm.o"), "-L" + PKG, "-lzfmm_b200",
                    "-Wl,-rpath," + PKG, "-o", exe], check=True)
    return exe


def test_fortran_module_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_fortran_program_matches_python_binding(tmp_path):
    import zfmm_b200
    exe = _build(tmp_path)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    n = 2000
    t = 2 * np.pi * np.arange(n) / n
    zs = np.stack([np.cos(t) + 0.05j * np.sin(3 * t), np.sin(t) + 0.05j * np.cos(3 * t)])
    q = np.cos(7 * t) + 1j * np.sin(5 * t)
    ds = np.sin(2 * t) + 1j
    dv = np.stack([np.cos(t), np.sin(t)]).astype(np.complex128)
    p, _ = zfmm_b200.zlfmm2d(1e-9, n, zs, 1, q, 1, ds, dv, n, zs, 2, 1)
    v = [float(x) for x in out[0].split()[1:]]
    assert np.allclose([p[0].real, p[0].imag, p[-1].real, p[-1].imag], v, rtol=1e-12, atol=0)
    z3 = np.concatenate([zs, (0.1 * (np.arange(n) + 1) / n)[None, :].astype(np.complex128)])
    p3, _ = zfmm_b200.zhfmm3d(1e-9, 10 + 0.2j, n, z3, 1, q, 1, ds, np.ones((3, n)), n, z3, 1, 1)
    f = out[1].split()
    assert int(f[1]) == 1
    v = [float(x) for x in f[2:]]
    assert np.allclose([p3[0].real, p3[0].imag, p3[-1].real, p3[-1].imag], v, rtol=1e-12, atol=0)
    assert out[2].split()[1] == "1" and "isep" in out[2]
