"""Build libzfmm_b200.so (sm_100a) in-tree with nvcc.

Usage: python -m zfmm_b200.build [--force]
Objects go to zfmm_b200/_build/, the shared library to zfmm_b200/libzfmm_b200.so.
tree.cu is compiled with --fmad=false: the tree's distance tests must see the
same roundings as the reference (no contracted multiply-adds).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libzfmm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]
NO_FMAD = {"tree.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "zfmm.h"))
    return max(os.path.getmtime(h) for h in hs if os.path.exists(h))


def build(force=False, verbose=True, extra=None):
    os.makedirs(BUILD, exist_ok=True)
    hm = headers_mtime()
    objs = []
    jobs = []
    for f in sources():
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f[:-3] + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hm):
            continue
        cmd = [NVCC] + ARCH + COMMON + (extra or [])
        if f in NO_FMAD:
            cmd.append("--fmad=false")
        cmd += ["-c", src, "-o", obj]
        jobs.append((f, cmd))
    procs = []
    for f, cmd in jobs:
        if verbose:
            print("nvcc", f, flush=True)
        procs.append((f, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for f, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed = True
            print(out)
        elif verbose and out.strip():
            print(out)
    if failed:
        raise RuntimeError("nvcc failed")
    newest = max(os.path.getmtime(o) for o in objs)
    if force or jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
        if verbose:
            print("linked", LIB, flush=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
