"""Drives the MATLAB gateway (zfmm_b200/matlab/zfmm_b200_mex.c) without
MATLAB: the gateway is compiled with gcc against the test stand-in of the MEX
API (tests/mex_shim) and called through ctypes with the argument lists the
mwrap-generated .m wrappers pass (mex_id_, the .mw FORTRAN arguments, then
one size per [x] argument and two per [xx] argument)."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "zfmm_b200")


def build(outdir):
    so = os.path.join(str(outdir), "zfmm_mexgw.so")
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", so,
                    os.path.join(PKG, "matlab", "zfmm_b200_mex.c"),
                    os.path.join(ROOT, "tests", "mex_shim", "mex_shim.c"),
                    "-I" + os.path.join(ROOT, "tests", "mex_shim"),
                    "-I" + os.path.join(ROOT, "include"), "-L" + PKG, "-lzfmm_b200",
                    "-Wl,-rpath," + PKG], check=True)
    L = ctypes.CDLL(so)
    vp = ctypes.c_void_p
    for name, res, args in [("shim_real", vp, [ctypes.c_size_t, ctypes.c_size_t, vp]),
                            ("shim_complex", vp, [ctypes.c_size_t, ctypes.c_size_t, vp]),
                            ("shim_string", vp, [ctypes.c_char_p]),
                            ("shim_data", vp, [vp]), ("shim_m", ctypes.c_size_t, [vp]),
                            ("shim_n", ctypes.c_size_t, [vp]), ("shim_free", None, [vp]),
                            ("shim_is_complex", ctypes.c_int, [vp]),
                            ("shim_error", ctypes.c_char_p, []),
                            ("shim_call", ctypes.c_int, [ctypes.c_int, vp, ctypes.c_int, vp])]:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


# .mw FORTRAN argument specs: (name, kind) with kind 'd' double[1], 'i' int[1],
# 'z' dcomplex[1], 'v' dcomplex[n] (vector), 'm' dcomplex[d, n]
SPECS = {
    "zlfmm2d": "d i m i v i v m v m i m i i i",
    "zhfmm2d": "d z i m i v i v m v m i m i i i",
    "zlfmm3d": "d i m i v i v m v m i m i i i",
    "zhfmm3d": "d z i m i v i v m v m i m i i i",
    "zl2devaldirect": "i m i m v v m i v m i i",
    "zh2devaldirect": "z i m i m v v m i v m i i",
    "zl3devaldirect": "i m i m v v m i v m i i",
    "zh3devaldirect": "z i m i m v v m i v m i i",
}
WORD = {"d": "i double[x]", "i": "i int[x]", "z": "i dcomplex[x]", "v": "i dcomplex[x]",
        "m": "i dcomplex[xx]"}


def call(L, name, args, nlhs=2, spec=None, dims=None):
    """[outs...] = gateway(mex_id_, args..., dims...) -> (outputs, error or None).
    args are numpy arrays / numbers in .mw order; dims are derived from their
    shapes unless given."""
    kinds = (spec or SPECS[name]).split()
    mex_id = name + "(" + ", ".join(WORD[k] for k in kinds) + ")"
    keep, prhs = [], []
    s = L.shim_string(mex_id.encode())
    prhs.append(s)
    auto = []
    for k, a in zip(kinds, args):
        a = np.asarray(a)
        if k in "di":
            arr = L.shim_real(1, 1, np.array([float(a)]).ctypes.data)
            auto.append(1)
        else:
            c = np.asfortranarray(np.asarray(a, np.complex128))
            if c.ndim == 0:
                c = c.reshape(1, 1)
            elif c.ndim == 1:
                c = c.reshape(-1, 1, order="F")
            keep.append(c)
            arr = L.shim_complex(c.shape[0], c.shape[1], c.ctypes.data)
            auto += [c.shape[0] * c.shape[1]] if k in "zv" else [c.shape[0], c.shape[1]]
        prhs.append(arr)
    for v in (dims if dims is not None else auto):
        prhs.append(L.shim_real(1, 1, np.array([float(v)]).ctypes.data))
    P = (ctypes.c_void_p * len(prhs))(*prhs)
    O = (ctypes.c_void_p * max(nlhs, 1))()
    rc = L.shim_call(nlhs, O, len(prhs), P)
    err = L.shim_error().decode() if rc else None
    outs = []
    if not rc:
        for i in range(nlhs):
            o = O[i]
            m, n = L.shim_m(o), L.shim_n(o)
            buf = (ctypes.c_double * (2 * m * n)).from_address(L.shim_data(o))
            v = np.frombuffer(buf, np.float64).copy().view(np.complex128).reshape((m, n), order="F")
            outs.append(v)
            L.shim_free(o)
    for p in prhs:
        L.shim_free(p)
    return outs, err
