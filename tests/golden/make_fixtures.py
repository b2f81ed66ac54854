"""Generate the golden fixtures used by the parity tests.

Run once, in a checkout that can see the reference tree (its root is given by
the required --ref argument); the outputs are committed, so the tests never
read the reference at run time.

Inputs (reference test data and logs):
  zfmm2d/test/laplace/test_data_2d.bin   read by zfmm2d/test/laplace/test5.f:31-78
  zfmm3d/test/laplace/test_data.bin      read by zfmm3d/test/laplace/test9.f
  zfmm2d/test/{laplace,helmholtz}/fort.13, zfmm3d/test/{laplace,helmholtz}/fort.13
      logs printed by those tests (prini unit 13)

The .bin layout is an int32 point count followed by float64 arrays in Fortran
column-major order: zsrc_re(d,n), zsrc_im(d,n), ztarg_re, ztarg_im,
charge_re(n), charge_im(n), dipvec_re(d,n), dipvec_im(d,n), dipstr_re(n),
dipstr_im(n).  The tests set targets = sources, so only sources and charges
are kept (the 3D dipoles are kept too for a dipole smoke case).

Outputs: fixture2d.npz, fixture3d.npz, golden.json (tree statistics, expansion
orders and the first 12 potentials, as printed in the logs).
"""
import argparse
import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_bin(path, d):
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    a = np.frombuffer(raw[4:], dtype=np.float64)
    off = 0
    out = {}
    for name, s in [("zsrc_re", d), ("zsrc_im", d), ("ztarg_re", d), ("ztarg_im", d),
                    ("charge_re", 1), ("charge_im", 1), ("dipvec_re", d), ("dipvec_im", d),
                    ("dipstr_re", 1), ("dipstr_im", 1)]:
        x = a[off:off + s * n]
        off += s * n
        out[name] = x.reshape(n, s) if s > 1 else x.copy()
    assert off == a.size
    return n, out


def parse_log(path):
    """prini log: 'name=' line followed by whitespace separated numbers."""
    vals = {}
    cur = None
    for line in open(path):
        s = line.strip()
        if not s:
            continue
        m = re.match(r"^([A-Za-z0-9_ ]+?)\s*=?\s*$", s)
        if m and not re.match(r"^[-+0-9.]", s):
            cur = m.group(1).strip()
            vals.setdefault(cur, [])
            vals[cur].append([])
            continue
        if cur is None:
            continue
        nums = [float(x.replace("D", "E")) for x in s.split()]
        vals[cur][-1].extend(nums)
    return vals


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True,
                    help="root of a checkout of the reference (wangyuguan/zfmm)")
    args = ap.parse_args()
    ref = args.ref

    n2, f2 = read_bin(os.path.join(ref, "zfmm2d/test/laplace/test_data_2d.bin"), 2)
    z2 = f2["zsrc_re"] + 1j * f2["zsrc_im"]
    q2 = f2["charge_re"] + 1j * f2["charge_im"]
    np.savez_compressed(os.path.join(HERE, "fixture2d.npz"), zsrc=z2, charge=q2)

    n3, f3 = read_bin(os.path.join(ref, "zfmm3d/test/laplace/test_data.bin"), 3)
    z3 = f3["zsrc_re"] + 1j * f3["zsrc_im"]
    q3 = f3["charge_re"] + 1j * f3["charge_im"]
    np.savez_compressed(os.path.join(HERE, "fixture3d.npz"), zsrc=z3, charge=q3)

    g = {}
    for key, rel in [("2d_laplace", "zfmm2d/test/laplace/fort.13"),
                     ("2d_helmholtz", "zfmm2d/test/helmholtz/fort.13"),
                     ("3d_laplace", "zfmm3d/test/laplace/fort.13"),
                     ("3d_helmholtz", "zfmm3d/test/helmholtz/fort.13")]:
        v = parse_log(os.path.join(ref, rel))
        ent = {"source": rel}
        for name in ["nboxes", "nlevels", "ndiv", "mnlist1", "mnlist2", "mnlist3", "mnlist4",
                     "nmax"]:
            if name in v:
                ent[name] = int(v[name][0][0])
        if "nterms" in v:
            ent["nterms"] = [int(x) for x in v["nterms"][0]]
        if "laddr" in v:
            ent["laddr"] = [[int(a) for a in x] for x in v["laddr"]]
        for name in ["pot", "pot0"]:
            if name in v:
                x = v[name][0]
                ent[name] = [[x[2 * i], x[2 * i + 1]] for i in range(len(x) // 2)]
        for name in ["pot0_norm", "charge_norm", "charge norm", "err", "pot_err", "rscales",
                     "zk", "b0"]:
            if name in v:
                ent[name.replace(" ", "_")] = v[name][0]
        g[key] = ent
    g["npt_2d"] = n2
    g["npt_3d"] = n3
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(g, fh, indent=1)
    print("wrote fixtures:", n2, n3)


if __name__ == "__main__":
    main()
