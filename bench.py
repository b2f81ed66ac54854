#!/usr/bin/env python
"""Benchmark of the complex-coordinate FMM on B200: targets/sec at eps=1e-9.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--workload NAME]

One step = one FMM solve (tree, lists, all eight passes, unsort) of the
workload's synthetic inputs.  `value` is measured through the device-pointer C
entry point with the inputs resident in HBM; `e2e` through the host-array C
entry point (the drop-in call) with the inputs in pinned host memory, so each
step includes the host->device copy of the inputs and the device->host copy of
pot/grad.  Between timed steps L2 is flushed by writing a 256 MiB buffer
(outside the timed events).  Multi-GPU: one process per GPU, each solving an
independent replica (a single FMM is not sharded), value = all ranks' targets
/ max-over-ranks time; scaling "weak".

--impl reference times the reference algorithm on the host cores: the
reference Fortran cannot be built on this image (no Fortran compiler), so it
runs the C restatement in oracle/ with all host threads (OpenMP), on a bounded
sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # zlfmm2d plain single solve, 20,000 points (sources = targets), charges +
    # dipoles, pot + grad, isep=1, eps=1e-9
    "zlfmm2d_uniform_20k": dict(kind="lap2d", n=20000, eps=1e-9, ifpgh=2, isep=1, cpu_n=20000),
    # zhfmm2d single solve, 2,000,000 points on the complex-deformed curve,
    # zk = 40+0.5i, charges + dipoles, pot + grad, isep=1, eps=1e-9
    "zhfmm2d_curve_2m": dict(kind="helm2d", n=2_000_000, eps=1e-9, zk=40 + 0.5j, ifpgh=2, isep=1,
                             cpu_n=200_000),
    # smaller case of the same distribution, for kernel-level profiling
    "zhfmm2d_curve_500k": dict(kind="helm2d", n=500_000, eps=1e-9, zk=40 + 0.5j, ifpgh=2, isep=1,
                               cpu_n=200_000),
    "zhfmm2d_curve_2m_eps1e-6": dict(kind="helm2d", n=2_000_000, eps=1e-6, zk=40 + 0.5j, ifpgh=2,
                                     isep=1, cpu_n=200_000),
    # zhfmm2d plan solve of 64 right-hand sides on the curve of the 2M case
    # (500,000 points, zk = 40+0.5i, charges + dipoles, pot + grad): at eps
    # 1e-6 the M2L runs on the tensor cores, at 1e-9 in FP64
    "zhfmm2d_batched_500k_64_eps1e-6": dict(kind="helm2d", n=500_000, nrhs=64, eps=1e-6,
                                            zk=40 + 0.5j, ifpgh=2, isep=1, cpu_n=50_000),
    "zhfmm2d_batched_500k_64": dict(kind="helm2d", n=500_000, nrhs=64, eps=1e-9, zk=40 + 0.5j,
                                    ifpgh=2, isep=1, cpu_n=50_000),
    "zhfmm2d_curve_2m_eps1e-12": dict(kind="helm2d", n=2_000_000, eps=1e-12, zk=40 + 0.5j,
                                      ifpgh=2, isep=1, cpu_n=200_000),
    # zlfmm3d single solve on the geometry of the batched configuration:
    # 1,000,000 points U[-1,1]^3 with imaginary parts 0.05 sin(2 pi .), one
    # charge vector, charges only, pot + grad, eps=1e-9
    "zlfmm3d_uniform_1m": dict(kind="lap3d", n=1_000_000, eps=1e-9, ifpgh=2, isep=1,
                               cpu_n=30_000, dipoles=False),
    "zlfmm3d_uniform_200k": dict(kind="lap3d", n=200_000, eps=1e-9, ifpgh=2, isep=1,
                                 cpu_n=30_000, dipoles=False),
    # zhfmm3d single instance at the largest size of the batched configuration:
    # 500,000 points on the unit sphere displaced by 0.1i times the normal
    # scaled by a degree-4 field, zk = 10+0.2i, charges + dipoles, pot + grad
    "zhfmm3d_sphere_500k": dict(kind="helm3d", n=500_000, eps=1e-9, zk=10 + 0.2j, ifpgh=2,
                                isep=1, cpu_n=30_000),
    "zhfmm3d_sphere_100k": dict(kind="helm3d", n=100_000, eps=1e-9, zk=10 + 0.2j, ifpgh=2,
                                isep=1, cpu_n=30_000),
    # zlfmm3d batched right-hand sides: one geometry of 1,000,000 points (the
    # distribution above), 64 complex normal charge vectors, charges only,
    # pot + grad, eps=1e-9; one step = plan (tree, lists, centres) + one
    # 64-right-hand-side solve
    "zlfmm3d_batched_1m_64": dict(kind="lap3d", n=1_000_000, nrhs=64, eps=1e-9, ifpgh=2, isep=1,
                                  cpu_n=30_000, dipoles=False),
    "zlfmm3d_batched_200k_64": dict(kind="lap3d", n=200_000, nrhs=64, eps=1e-9, ifpgh=2,
                                    isep=1, cpu_n=30_000, dipoles=False),
    # small case of the same distribution for kernel profiles (one 32-right-hand-side pass)
    "zlfmm3d_batched_30k_32": dict(kind="lap3d", n=30_000, nrhs=32, eps=1e-9, ifpgh=2,
                                   isep=1, cpu_n=30_000, dipoles=False),
    # zhfmm3d batched right-hand sides: one geometry of 200,000 points on the
    # unit sphere displaced by 0.1i times the normal scaled by a degree-4 field
    # (the instance distribution below), 64 complex normal charge and dipole
    # strength vectors with shared complex dipole vectors, zk = 10+0.2i,
    # pot + grad, eps=1e-9; one step = plan + one 64-right-hand-side solve
    # zhfmm3d batched right-hand sides on the batched zlfmm3d geometry (1,000,000
    # points U[-1,1]^3 with imaginary parts 0.05 sin(2 pi .)), zk = 10+0.2i, 64
    # complex normal charge vectors, charges only, pot + grad, eps=1e-9: the
    # batched-vs-plain per-right-hand-side speed-up of this case is the
    # north-star target line (also carried by the default line)
    "zhfmm3d_batched_1m_64": dict(kind="helm3d", geometry="cube", n=1_000_000, nrhs=64,
                                  eps=1e-9, zk=10 + 0.2j, ifpgh=2, isep=1, cpu_n=30_000,
                                  dipoles=False),
    "zhfmm3d_batched_200k_64": dict(kind="helm3d", n=200_000, nrhs=64, eps=1e-9, zk=10 + 0.2j,
                                    ifpgh=2, isep=1, cpu_n=30_000, dipoles=True),
    "zhfmm3d_batched_30k_32": dict(kind="helm3d", n=30_000, nrhs=32, eps=1e-9, zk=10 + 0.2j,
                                   ifpgh=2, isep=1, cpu_n=30_000, dipoles=True),
    # zhfmm3d batched uneven instances: 200 independent FMMs, point counts
    # log-uniform in [2,000, 500,000], points on unit spheres displaced by 0.1i
    # times the normal scaled by a degree-4 field, zk = 10+0.2i, charges +
    # dipoles, pot + grad, eps=1e-9; one step = all 200 solves in one call
    # zhfmm2d adjoint: forward + reverse pass on 200,000 points of a two-curve
    # interface (the curve above plus a copy scaled 0.3, imaginary part
    # included, and shifted by (0.2, 0.1)), imaginary displacement amplitudes
    # (0.05, 0.015) as learnable parameters, zk = 20+0.3i, charges + dipoles,
    # loss = mean |pot - ref|^2,
    # eps=1e-10; one step = forward (pot and grad) + backward (gradients for
    # charges, dipole strengths and both amplitudes)
    "zhfmm2d_adjoint_200k": dict(kind="helm2d", adjoint=True, n=200_000, eps=1e-10,
                                 zk=20 + 0.3j, ifpgh=2, isep=1, cpu_n=100_000),
    "zhfmm3d_instances_200": dict(kind="helm3d", instances=200, nmin=2000, nmax=500_000,
                                  n=500_000, eps=1e-9, zk=10 + 0.2j, ifpgh=2, isep=1,
                                  cpu_n=30_000, nstreams=8),
}
for _k, _v in WORKLOADS.items():
    _v["name"] = _k
DEFAULT_WORKLOAD = "zhfmm2d_curve_2m"
# the batched case reported beside the default line (batched_rhs key)
BATCHED_KEY_WORKLOAD = "zhfmm3d_batched_1m_64"
# wall-clock bound of the reference arm's timed solves at full size
REF_BUDGET_S = 600.0

def m2l3d_flops(p):
    """Real flops of one point-and-shoot 3D Laplace translation at order p, as
    implemented: two y-rotations, each sampling 2p+1 meridian points with 92
    flops per (n, m >= 0, sample) and projecting with (p+1)^2 (2p+1) complex
    MACs, plus the axial shift (one complex MAC per term of its Toeplitz sums)."""
    ns = 2 * p + 1
    sample = 92 * ns * (p + 1) * (p + 2) // 2
    project = 8 * (p + 1) ** 2 * ns
    shift = 8 * sum(p + 1 - abs(k) for j in range(p + 1) for k in range(-j, j + 1))
    return 2 * (sample + project) + shift


def rot3d_flops(p):
    """One point-and-shoot y-rotation of order p: 2p+1 meridian samples with 92
    flops per (n, m >= 0, sample), then the (p+1)^2 (2p+1) complex-MAC DFT
    projection."""
    ns = 2 * p + 1
    return 92 * ns * (p + 1) * (p + 2) // 2 + 8 * (p + 1) ** 2 * ns


def h3d_trans_flops(p1, p2):
    """One 3D Helmholtz translation (order p1 -> p2) as implemented: the two
    rotations plus the quadrature z-shift at nquad = 2.5 p2 nodes: 70 flops per
    (node, n, m >= 0) for the value/derivative sums, 5 per projection Legendre
    term and 8 per (node, output coefficient) for the projection."""
    nq = int(2.5 * p2)
    quad = nq * (70 * (p1 + 1) * (p1 + 2) // 2 + 5 * (p2 + 1) * (p2 + 2) // 2
                 + 8 * (p2 + 1) ** 2)
    return rot3d_flops(p1) + rot3d_flops(p2) + quad


def flop_model3d(kind, lvl, orders):
    """Per-step flops from the per-level interaction counts (last_level_counts)
    and the order of each level.  Per source (P2M/P2L) 42 (Laplace) or 50
    (Helmholtz) flops per (n, m >= 0); per target and expansion (M2T/L2T with
    gradient) 80; P2P pair 90 (Laplace) or 130 (Helmholtz)."""
    L = len(orders)
    nm = lambda p: (p + 1) * (p + 2) // 2
    helm = kind == "helm3d"
    src, pair = (50, 130) if helm else (42, 90)
    tr = h3d_trans_flops if helm else (lambda p1, p2: m2l3d_flops(p1))
    steps = {"p2m": 0, "m2m": 0, "m2l_p2l": 0, "l2l": 0, "eval": 0}
    for l in range(L):
        p = orders[l]
        pc = orders[min(l + 1, L - 1)]
        pp = orders[max(l - 1, 0)]
        steps["p2m"] += src * nm(p) * lvl["p2m"][l]
        steps["m2m"] += tr(pc, p) * lvl["m2m_pairs"][l]
        steps["m2l_p2l"] += tr(p, p) * lvl["m2l_pairs"][l] + src * nm(p) * lvl["p2l"][l]
        steps["l2l"] += tr(pp, p) * lvl["l2l_pairs"][l]
        steps["eval"] += (pair * lvl["p2p_pairs"][l] + 80 * nm(pc) * lvl["m2t"][l]
                          + 80 * nm(p) * lvl["l2t"][l])
    pm = max(orders) if orders else 0
    per = {"p2p_pair": pair, "translation_at_pmax": tr(pm, pm),
           "p2m_p2l_per_source_per_nm": src, "m2t_l2t_per_target_per_nm": 80,
           "orders_per_level": orders}
    return steps, per


def nd_trans3_flops(p, nd, kind=1):
    """Real flops of one batched 3D Laplace translation of nd right-hand sides
    at order p, as implemented: per 32-right-hand-side pass and rotation, the
    (angle >= 0, order) recurrences and sample coefficients (100 flops per
    angle, n, m >= 0); per right-hand side and rotation, the sample product on
    sums / differences (2 (p+1) sum_n (n+1) complex MACs) and the cosine / sine
    projection (2 (p+1) sum_n (n+1) real-by-complex MACs); per right-hand side
    the axial shift (M2L: sum_m (p+1-|m|)^2 complex MACs, M2M / L2L half)."""
    L = p + 1
    tri = L * (L + 1) // 2
    passes = -(-nd // 32)
    gen = 2 * passes * 100 * L * tri
    rot = 2 * nd * (2 * L * tri * 8 + 2 * L * tri * 4)
    sh = sum((p + 1 - abs(m)) ** 2 for m in range(-p, p + 1))
    shift = nd * 8 * (sh if kind == 1 else sh // 2)
    return gen + rot + shift


def nd_htrans3_flops(p1, p2, nd):
    """Real flops of one batched 3D Helmholtz translation of nd right-hand
    sides from order p1 to p2, as implemented: the two batched rotations (as
    nd_trans3_flops, orders p1 and p2) and the quadrature z-shift over
    nq = int(2.5 p2) nodes: per 32-right-hand-side pass its node tables (60
    flops per (node, n, m >= 0) value / derivative coefficient pair, 4 per
    projection entry); per right-hand side the node sums (two complex MACs per
    (node, n, +-m)) and the projection (two real-by-complex MACs per
    (node, n', +-m))."""
    nq = int(2.5 * p2)
    passes = -(-nd // 32)

    def rot(p):
        L = p + 1
        tri = L * (L + 1) // 2
        return passes * 100 * L * tri + nd * (L * tri * 8 + L * tri * 4)

    tri1, tri2 = (p1 + 1) * (p1 + 2) // 2, (p2 + 1) * (p2 + 2) // 2
    tabs = passes * nq * (60 * tri1 + 4 * tri2)
    sums = sum((1 if m == 0 else 2) * ((p1 + 1 - m) * 16 + (p2 + 1 - m) * 8)
               for m in range(min(p1, p2) + 1))
    return rot(p1) + rot(p2) + tabs + nd * nq * sums


# Algorithmic work per interaction (real flops; complex add 2, mul 6, div 11;
# transcendental functions are not counted), per the frozen convention of the
# project's measurement plan.  P = 2p+1 coefficients of the level.
#   P2P pair (pot+grad, charge+dipole): 70 flops (2D Laplace), 650 (2D Helmholtz:
#     two ~35-term complex polynomial evaluations for H0, H1 plus 90)
#   M2T / L2T (target, expansion) with gradient: 3 complex MACs per coefficient = 24 P
#   M2L: one dense P x P complex operator = 8 P^2;  M2M / L2L: 8 P_parent P_child
#   P2M / P2L per source: 2 complex MACs per coefficient = 16 P
def flop_model(kind, counts):
    pair = {"lap2d": 70, "helm2d": 650}[kind]
    steps = {
        "p2m": 16 * counts["p2m_P"],
        "m2m": 8 * counts["m2m_pairs_P"],
        "m2l_p2l": 8 * counts["m2l_pairs_P"] + 16 * counts["p2l_P"],
        "l2l": 8 * counts["l2l_pairs_P"],
        "eval": pair * counts["p2p_pairs"] + 24 * counts["m2t_P"] + 24 * counts["l2t_P"],
    }
    per = {"p2p_pair": pair, "m2t_per_P": 24, "l2t_per_P": 24, "m2l_per_P2": 8,
           "m2m_l2l_per_P1P2": 8, "p2m_p2l_per_P": 16}
    return steps, per


def read_traffic(workload, step):
    """DRAM bytes (read + write) per solve of the kernels of `step`, from the
    ncu summary profiles/<workload>_traffic.txt ("<step> <bytes>" lines, '#'
    comments naming the capture), or None when there is none."""
    path = os.path.join(ROOT, "profiles", f"{workload}_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split("#", 1)[0].split()
        if len(f) == 2 and f[0] == step:
            return float(f[1])
    return None


def make_inputs(wl, seed, n=None, nrhs=1):
    from zfmm_b200 import workloads as W
    n = wl["n"] if n is None else n
    if wl["kind"] == "lap3d" and nrhs > 1:
        return W.lap3d_uniform(n, seed=seed, nrhs=nrhs)
    if wl["kind"] == "helm3d" and nrhs > 1 and wl.get("geometry") == "cube":
        return W.lap3d_uniform(n, seed=seed, nrhs=nrhs)
    if wl["kind"] == "helm3d" and nrhs > 1:
        w = W.sphere3d(n, seed=seed)
        rng = np.random.default_rng(seed + 7919)
        cn = lambda: rng.standard_normal((nrhs, n)) + 1j * rng.standard_normal((nrhs, n))
        w["charge"], w["dipstr"] = cn(), cn()
        return w
    if wl["kind"] == "lap2d":
        return W.lap2d_uniform(n, seed=seed)
    if wl["kind"] == "helm2d":
        return W.curve2d(n, seed=seed)
    if wl["kind"] == "lap3d":
        return W.lap3d_uniform(n, seed=seed)
    if wl["kind"] == "helm3d":
        return W.sphere3d(n, seed=seed)
    raise ValueError(wl["kind"])


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def host_cores():
    """(physical cores, logical CPUs) of this host."""
    logical = os.cpu_count() or 1
    try:
        import psutil
        phys = psutil.cpu_count(logical=False) or logical
    except Exception:
        phys = logical
    return phys, logical


def set_omp_threads():
    """OpenMP threads of the CPU oracle = the physical core count (set before the
    oracle library is loaded, which reads it once)."""
    phys, _ = host_cores()
    os.environ["OMP_NUM_THREADS"] = str(phys)
    return phys


def cpu_time_oracle(wl, inp, reps_min=1, budget_s=15.0):
    """Oracle (C restatement, OpenMP) on the host cores; returns (sec per solve, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    cores = int(os.environ.get("OMP_NUM_THREADS", host_cores()[0]))
    z = inp["zsrc"].T
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < reps_min or (time.perf_counter() < t_end and len(times) < 50):
        t0 = time.perf_counter()
        if wl["kind"] == "lap2d":
            O.zlfmm2d(wl["eps"], z, inp["charge"], inp["dipstr"], inp["dipvec"].T,
                      ifpgh=wl["ifpgh"], isep=wl["isep"])
        elif wl["kind"] == "lap3d":
            dip = wl.get("dipoles", True)
            O.zlfmm3d(wl["eps"], z, inp["charge"], inp["dipstr"] if dip else None,
                      inp["dipvec"].T if dip else None, ifpgh=wl["ifpgh"], isep=wl["isep"])
        elif wl["kind"] == "helm3d":
            O.zhfmm3d(wl["eps"], wl["zk"], z, inp["charge"], inp["dipstr"], inp["dipvec"].T,
                      ifpgh=wl["ifpgh"], isep=wl["isep"])
        else:
            O.zhfmm2d(wl["eps"], wl["zk"], z, inp["charge"], inp["dipstr"], inp["dipvec"].T,
                      ifpgh=wl["ifpgh"], isep=wl["isep"])
        times.append(time.perf_counter() - t0)
        if len(times) == 1 and times[0] > budget_s:
            break
    return statistics.median(times), cores, len(times)


def run_reference(args, wl, ws, rank):
    """The reference algorithm on the host cores (the C restatement in oracle/,
    OpenMP on every physical core), on the full workload: each step is one
    whole solve of the same points as the GPU arm.  Only if one solve is so
    slow that K steps would run past REF_BUDGET_S does it fall back to a
    sample of the workload's distribution (and says so in the line)."""
    if rank != 0:
        return
    phys = set_omp_threads()
    logical = host_cores()[1]
    nfull = wl["n"] * wl.get("nrhs", 1)
    nt = wl["n"]
    inp = make_inputs(wl, seed=0, n=nt)
    t1, cores, _n = cpu_time_oracle(wl, inp, reps_min=1, budget_s=0.0)  # warm-up solve
    if t1 * args.steps > REF_BUDGET_S:
        nt = wl["cpu_n"]
        inp = make_inputs(wl, seed=0, n=nt)
        cpu_time_oracle(wl, inp, reps_min=1, budget_s=0.0)
    per = []
    for _ in range(args.steps):
        t, cores, _n = cpu_time_oracle(wl, inp, reps_min=1, budget_s=0.0)
        per.append(t)
    tot = sum(per)
    value = nt * args.steps / tot
    full = nt == wl["n"]
    line = {
        "impl": "reference", "metric": "targets/sec at eps=1e-9", "value": value,
        "unit": "targets/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "n": wl["n"], "n_timed": nt,
                   "same_config": full, "eps": wl["eps"], "zk": str(wl.get("zk")),
                   "ifpgh": wl["ifpgh"], "isep": wl["isep"], "l2": "n/a (host)",
                   "omp_threads": phys, "physical_cores": phys, "logical_cpus": logical},
        "cpu_baseline": {"value": value, "unit": "targets/s", "cores": cores, "kind": "port",
                         "sample": ((f"the full workload ({nt} points, seed 0), one solve per "
                                     f"step, {args.steps} steps after one warm-up solve")
                                    if full else
                                    (f"{nt} points of the workload's distribution (full "
                                     f"workload: {wl['n']}: one full solve took {t1:.1f} s, "
                                     f"{args.steps} would exceed {REF_BUDGET_S:.0f} s), "
                                     f"{args.steps} solves"))},
        "e2e": {"value": value, "unit": "targets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, wl, ws, rank, local):
    import ctypes

    import torch

    import zfmm_b200
    from zfmm_b200 import _capi
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _capi.lib()
    inp = make_inputs(wl, seed=rank)
    n = wl["n"]
    ifpgh, isep, eps = wl["ifpgh"], wl["isep"], wl["eps"]
    d = 3 if wl["kind"] in ("lap3d", "helm3d") else 2
    ifd = 1 if wl.get("dipoles", True) else 0
    # device-resident inputs (Fortran layout = (n, d) row-major complex128)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    zs = t(inp["zsrc"].T)
    q, ds, dv = t(inp["charge"]), t(inp["dipstr"]), t(inp["dipvec"].T)
    pot = torch.empty(n, dtype=torch.complex128, device=dev)
    grad = torch.empty((n, d), dtype=torch.complex128, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda x: ctypes.c_void_p(x.data_ptr())

    helm = wl["kind"] == "helm2d"
    helm3 = wl["kind"] == "helm3d"
    zkv = np.array([complex(wl.get("zk", 0)).real, complex(wl.get("zk", 0)).imag])
    zkp = zkv.ctypes.data_as(ctypes.c_void_p)

    def solve():
        if helm:
            _capi.check(L.zfmm_zhfmm2d_dev(eps, zkp, n, P(zs), 1, P(q), 1, P(ds), P(dv), P(pot),
                                           P(grad), n, P(zs), ifpgh, isep, sp))
        elif helm3:
            _capi.check(L.zfmm_zhfmm3d_dev(eps, zkp, n, P(zs), 1, P(q), ifd, P(ds), P(dv),
                                           P(pot), P(grad), n, P(zs), ifpgh, isep, sp))
        elif d == 3:
            _capi.check(L.zfmm_zlfmm3d_dev(eps, n, P(zs), 1, P(q), ifd, P(ds), P(dv), P(pot),
                                           P(grad), n, P(zs), ifpgh, isep, sp))
        else:
            _capi.check(L.zfmm_zlfmm2d_dev(eps, n, P(zs), 1, P(q), 1, P(ds), P(dv), P(pot),
                                           P(grad), n, P(zs), ifpgh, isep, sp))

    for _ in range(max(args.warmup, 3)):
        solve()
    torch.cuda.synchronize()
    # counts and per-step structure from one instrumented call (not timed)
    L.zfmm_set_step_timing(2)
    solve()
    counts, _ = zfmm_b200.last_counts()
    _, info = zfmm_b200.last_step_times()
    lvl, orders = zfmm_b200.last_level_counts() if d == 3 else (None, None)
    L.zfmm_set_step_timing(1)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    step_ms = {k: 0.0 for k in ["setup", "p2m", "m2m", "m2l_p2l", "l2l", "eval", "unsort"]}
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.zfmm_launch_count()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev0[k].record(stream)
            solve()
            ev1[k].record(stream)
            st, _ = zfmm_b200.last_step_times()
            for kk in step_ms:
                step_ms[kk] += st[kk]
        torch.cuda.synchronize()
    launches = L.zfmm_launch_count() - launches0
    L.zfmm_set_step_timing(0)
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    if ws > 1:
        import torch.distributed as dist
        tt = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    value = ws * n * args.steps / (tot_ms * 1e-3)

    # end to end through the host-array entry point, pinned host inputs
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hz, hq, hds, hdv = pin(inp["zsrc"].T), pin(inp["charge"]), pin(inp["dipstr"]), pin(inp["dipvec"].T)
    hpot = torch.empty(n, dtype=torch.complex128).pin_memory().numpy()
    hgrad = torch.empty((n, d), dtype=torch.complex128).pin_memory().numpy()
    hp = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def solve_host():
        if helm:
            _capi.check(L.zfmm_zhfmm2d(eps, zkp, n, hp(hz), 1, hp(hq), 1, hp(hds), hp(hdv),
                                       hp(hpot), hp(hgrad), n, hp(hz), ifpgh, isep, 0))
        elif helm3:
            _capi.check(L.zfmm_zhfmm3d(eps, zkp, n, hp(hz), 1, hp(hq), ifd, hp(hds), hp(hdv),
                                       hp(hpot), hp(hgrad), n, hp(hz), ifpgh, isep, 0))
        elif d == 3:
            _capi.check(L.zfmm_zlfmm3d(eps, n, hp(hz), 1, hp(hq), ifd, hp(hds), hp(hdv),
                                       hp(hpot), hp(hgrad), n, hp(hz), ifpgh, isep, 0))
        else:
            _capi.check(L.zfmm_zlfmm2d(eps, n, hp(hz), 1, hp(hq), 1, hp(hds), hp(hdv), hp(hpot),
                                       hp(hgrad), n, hp(hz), ifpgh, isep, 0))

    solve_host()
    if ws > 1:
        dist.barrier()
    e2e_t = []
    for k in range(args.steps):
        flush.fill_(k & 255)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solve_host()
        e2e_t.append(time.perf_counter() - t0)
    e2e_tot = sum(e2e_t)
    if ws > 1:
        tt = torch.tensor([e2e_tot], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_tot = float(tt.item())
    # targets are the sources (one array): the coordinates are uploaded once
    h2d = hz.nbytes + hq.nbytes + (hds.nbytes + hdv.nbytes if ifd else 0)
    d2h = hpot.nbytes + (hgrad.nbytes if ifpgh > 1 else 0)
    # accuracy against the FP64 direct sum on a seeded subset of targets (device direct sum)
    pg = pot.cpu().numpy()
    rng = np.random.default_rng(1234)
    nsub = min(n, 4096 if n <= 100_000 else 1024)
    sub = np.sort(rng.choice(n, size=nsub, replace=False))
    if helm:
        pd, _ = zfmm_b200.zh2devaldirect(wl["zk"], len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                         inp["charge"], inp["dipstr"], inp["dipvec"], 1, 1, 1)
        pd = pd * 0.25j
    elif helm3:
        pd, _ = zfmm_b200.zh3devaldirect(wl["zk"], len(sub), inp["zsrc"][:, sub], n,
                                         inp["zsrc"], inp["charge"], inp["dipstr"],
                                         inp["dipvec"], 1, ifd, 1)
    elif d == 3:
        pd, _ = zfmm_b200.zl3devaldirect(len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                         inp["charge"], inp["dipstr"], inp["dipvec"], 1, ifd, 1)
    else:
        pd, _ = zfmm_b200.zl2devaldirect(len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                         inp["charge"], inp["dipstr"], inp["dipvec"], 1, 1, 1)
        pd = pd / (2 * np.pi)
    relerr = float(np.linalg.norm(pg[sub] - pd) / np.linalg.norm(pd))

    # roofline of the dominant kernel (FP64 pipe bound)
    p = info["nterms"]
    if d == 3:
        flops, per = flop_model3d(wl["kind"], lvl, orders)
    else:
        flops, per = flop_model(wl["kind"], counts)
    avg = {k: v / args.steps for k, v in step_ms.items()}
    top = max(flops, key=lambda k: avg[k])
    achieved = flops[top] / (avg[top] * 1e-3) / 1e12
    peak = float(L.zfmm_probe_fp64_tflops(20000))
    traffic = read_traffic(args.workload, top)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        set_omp_threads()
        ncpu = wl["cpu_n"]
        cinp = inp if ncpu == n else make_inputs(wl, seed=0, n=ncpu)
        t_cpu, cores, nrep = cpu_time_oracle(wl, cinp, reps_min=1, budget_s=12.0)
        cpu = {"value": ncpu / t_cpu, "unit": "targets/s", "cores": cores, "kind": "port",
               "sample": (f"{ncpu} points of the workload's distribution (full workload: {n}), "
                          f"median of {nrep} solves")}
    # the batched-right-hand-side target case, measured in the same run (one
    # GPU only: it is not part of the replicated step)
    batched = None
    if ws == 1 and args.workload == DEFAULT_WORKLOAD and not args.no_batched:
        import types
        bargs = types.SimpleNamespace(steps=1, warmup=1, no_cpu=True,
                                      workload=BATCHED_KEY_WORKLOAD)
        batched = run_ours_batched(bargs, WORKLOADS[BATCHED_KEY_WORKLOAD], ws, rank, local,
                                   summary=True)
    if rank != 0:
        return
    line = {
        "metric": "targets/sec at eps=1e-9", "value": value, "unit": "targets/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "eps": eps, "zk": str(wl.get("zk")),
                   "ifpgh": ifpgh, "isep": isep,
                   "charges": True, "dipoles": bool(ifd),
                   "l2": "flushed (256 MiB write) between steps",
                   "parallelism": f"replicas x{ws}", "nboxes": info["nboxes"],
                   "nlevels": info["nlevels"], "nterms": p},
        "e2e": {"value": ws * n * args.steps / e2e_tot, "unit": "targets/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "rel_l2_err_vs_direct": relerr,
        "step_ms": {k: round(v, 4) for k, v in avg.items()},
        "roofline": {"bound": "fp64", "kernel": top, "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak > 0 else None,
                     "peak_source": "measured FP64 FMA probe (zfmm_probe_fp64_tflops)",
                     "traffic": traffic, "flops_per_step": flops[top],
                     "flop_model": per},
        "interactions": counts,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "batched_rhs": batched,
    }
    print(json.dumps(line), flush=True)


def run_ours_batched(args, wl, ws, rank, local, summary=False):
    """One step = plan (tree, lists, centres) + one nd-right-hand-side solve.

    summary=True (the default line's batched key): one warm-up and one timed
    step, the plain single solve on the same geometry, the accuracy against the
    direct sum; no end-to-end pass, no CPU leg; returns a dict instead of
    printing a line."""
    import ctypes

    import torch

    import zfmm_b200
    from zfmm_b200 import _capi
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _capi.lib()
    n, nd = wl["n"], wl["nrhs"]
    ifpgh, isep, eps = wl["ifpgh"], wl["isep"], wl["eps"]
    helm = wl["kind"] == "helm3d"
    ifd = 1 if wl.get("dipoles", False) else 0
    zk = complex(wl.get("zk", 0))
    zka = np.array([zk.real, zk.imag])
    zkp = zka.ctypes.data_as(ctypes.c_void_p)
    # one geometry and nd right-hand sides for the whole job; with N ranks each
    # solves a contiguous block of the right-hand sides (zfmm_b200.shard: no
    # collective on the data path; every rank builds the geometry's plan)
    from zfmm_b200 import shard
    nd_total = nd
    r0, r1 = shard.rhs_block(nd_total, rank, ws)
    nd = r1 - r0
    if nd < 1:
        raise SystemExit("more ranks than right-hand sides")
    inp = make_inputs(wl, seed=0, nrhs=nd_total)
    inp["charge"] = inp["charge"][r0:r1]
    inp["dipstr"] = inp["dipstr"][r0:r1]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    zs = t(inp["zsrc"].T)
    q = t(inp["charge"].T)  # (n, nd): right-hand side fastest
    ds = t(inp["dipstr"].T) if ifd else None
    dv = t(inp["dipvec"].T) if ifd else None
    pot = torch.empty((n, nd), dtype=torch.complex128, device=dev)
    grad = torch.empty((n, 3, nd), dtype=torch.complex128, device=dev)
    pot1 = torch.empty(n, dtype=torch.complex128, device=dev)
    grad1 = torch.empty((n, 3), dtype=torch.complex128, device=dev)
    q0 = t(inp["charge"][0])
    ds0 = t(inp["dipstr"][0]) if ifd else None
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    plan_ms = []

    Po = lambda x: None if x is None else P(x)

    def solve():
        h = ctypes.c_void_p()
        _capi.check(L.zfmm_plan3d_create_dev(eps, n, P(zs), n, P(zs), isep, sp, ctypes.byref(h)))
        if helm:
            _capi.check(L.zfmm_zhfmm3d_plan_dev(h, zkp, nd, 1, P(q), ifd, Po(ds), Po(dv), ifpgh,
                                                P(pot), P(grad), sp))
        else:
            _capi.check(L.zfmm_zlfmm3d_plan_dev(h, nd, 1, P(q), ifd, Po(ds), Po(dv), ifpgh,
                                                P(pot), P(grad), sp))
        _capi.check(L.zfmm_plan3d_destroy(h))

    def solve_plain():
        if helm:
            _capi.check(L.zfmm_zhfmm3d_dev(eps, zkp, n, P(zs), 1, P(q0), ifd, Po(ds0), Po(dv),
                                           P(pot1), P(grad1), n, P(zs), ifpgh, isep, sp))
        else:
            _capi.check(L.zfmm_zlfmm3d_dev(eps, n, P(zs), 1, P(q0), ifd, Po(ds0), Po(dv),
                                           P(pot1), P(grad1), n, P(zs), ifpgh, isep, sp))

    for _ in range(1 if summary else max(args.warmup, 3)):
        solve()
    torch.cuda.synchronize()
    L.zfmm_set_step_timing(2)
    solve()
    counts, _ = zfmm_b200.last_counts()
    _, info = zfmm_b200.last_step_times()
    lvl, orders = zfmm_b200.last_level_counts()
    L.zfmm_set_step_timing(1)
    step_ms = {k: 0.0 for k in ["setup", "p2m", "m2m", "m2l_p2l", "l2l", "eval", "unsort"]}
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.zfmm_launch_count()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev0[k].record(stream)
            solve()
            ev1[k].record(stream)
            st, _ = zfmm_b200.last_step_times()
            for kk in step_ms:
                step_ms[kk] += st[kk]
        torch.cuda.synchronize()
    launches = L.zfmm_launch_count() - launches0
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    # the plan build alone (tree, lists, centres), and the plain
    # single-right-hand-side solve on the same geometry, same run
    pc0, pc1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hh = ctypes.c_void_p()
    torch.cuda.synchronize()
    pc0.record(stream)
    _capi.check(L.zfmm_plan3d_create_dev(eps, n, P(zs), n, P(zs), isep, sp, ctypes.byref(hh)))
    pc1.record(stream)
    torch.cuda.synchronize()
    plan_ms = pc0.elapsed_time(pc1)
    _capi.check(L.zfmm_plan3d_destroy(hh))
    for _ in range(1 if summary else 3):
        solve_plain()
    torch.cuda.synchronize()
    pl_t = []
    for k in range(2 if summary else 5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(k & 255)
        e0.record(stream)
        solve_plain()
        e1.record(stream)
        torch.cuda.synchronize()
        pl_t.append(e0.elapsed_time(e1))
    plain_ms = statistics.median(pl_t)
    L.zfmm_set_step_timing(0)
    if ws > 1:
        import torch.distributed as dist
        tt = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    value = n * nd_total * args.steps / (tot_ms * 1e-3)
    plain_value = n / (plain_ms * 1e-3)
    if summary:
        pg = pot.cpu().numpy()
        p1 = pot1.cpu().numpy()
        rng = np.random.default_rng(1234)
        sub = np.sort(rng.choice(n, size=min(n, 1024), replace=False))
        errs = []
        for r in (0, nd - 1):
            dsr = inp["dipstr"][r] if ifd else None
            dvr = inp["dipvec"] if ifd else None
            if helm:
                pd, _ = zfmm_b200.zh3devaldirect(zk, len(sub), inp["zsrc"][:, sub], n,
                                                 inp["zsrc"], inp["charge"][r], dsr, dvr, 1, ifd,
                                                 1)
            else:
                pd, _ = zfmm_b200.zl3devaldirect(len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                                 inp["charge"][r], dsr, dvr, 1, ifd, 1)
            errs.append(float(np.linalg.norm(pg[sub, r] - pd) / np.linalg.norm(pd)))
        L.zfmm_set_step_timing(0)
        return {"workload": wl["name"], "n": n, "nrhs": nd, "eps": eps,
                "zk": [zk.real, zk.imag] if helm else None, "ms_per_step": tot_ms / args.steps,
                "value": value, "unit": "targets/s",
                "step": "plan (tree, lists, centres) + one solve of all right-hand sides",
                "plain_single_rhs_ms": plain_ms,
                "batched_per_rhs_speedup": value / ws / plain_value,
                "rel_l2_err_vs_direct": max(errs),
                "rel_l2_batched_vs_plain_rhs0": float(np.linalg.norm(pg[:, 0] - p1)
                                                      / np.linalg.norm(p1)),
                "plan_build_ms": plan_ms}

    # end to end: host arrays in pinned memory through the host entry points
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hz, hq = pin(inp["zsrc"].T), pin(inp["charge"].T)
    hds = pin(inp["dipstr"].T) if ifd else None
    hdv = pin(inp["dipvec"].T) if ifd else None
    hpot = torch.empty((n, nd), dtype=torch.complex128).pin_memory().numpy()
    hgrad = torch.empty((n, 3, nd), dtype=torch.complex128).pin_memory().numpy()
    hp = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    hpo = lambda a: None if a is None else hp(a)

    def solve_host():
        h = ctypes.c_void_p()
        _capi.check(L.zfmm_plan3d_create(eps, n, hp(hz), n, hp(hz), isep, ctypes.byref(h)))
        if helm:
            _capi.check(L.zfmm_zhfmm3d_plan(h, zkp, nd, 1, hp(hq), ifd, hpo(hds), hpo(hdv),
                                            ifpgh, hp(hpot), hp(hgrad)))
        else:
            _capi.check(L.zfmm_zlfmm3d_plan(h, nd, 1, hp(hq), ifd, hpo(hds), hpo(hdv), ifpgh,
                                            hp(hpot), hp(hgrad)))
        _capi.check(L.zfmm_plan3d_destroy(h))

    solve_host()
    e2e_t = []
    for k in range(args.steps):
        flush.fill_(k & 255)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solve_host()
        e2e_t.append(time.perf_counter() - t0)
    e2e_tot = sum(e2e_t)
    if ws > 1:
        tt = torch.tensor([e2e_tot], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_tot = float(tt.item())
    h2d = hz.nbytes + hq.nbytes + (hds.nbytes + hdv.nbytes if ifd else 0)
    d2h = hpot.nbytes + (hgrad.nbytes if ifpgh > 1 else 0)
    # accuracy: right-hand sides 0 and nd-1 against the FP64 direct sum on a subset
    rng = np.random.default_rng(1234)
    sub = np.sort(rng.choice(n, size=min(n, 1024), replace=False))
    pg = pot.cpu().numpy()
    errs = []
    for r in (0, nd - 1):
        dsr = inp["dipstr"][r] if ifd else None
        dvr = inp["dipvec"] if ifd else None
        if helm:
            pd, _ = zfmm_b200.zh3devaldirect(zk, len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                             inp["charge"][r], dsr, dvr, 1, ifd, 1)
        else:
            pd, _ = zfmm_b200.zl3devaldirect(len(sub), inp["zsrc"][:, sub], n, inp["zsrc"],
                                             inp["charge"][r], dsr, dvr, 1, ifd, 1)
        errs.append(float(np.linalg.norm(pg[sub, r] - pd) / np.linalg.norm(pd)))
    # plain vs batched agreement on right-hand side 0 (same tree, same algorithm)
    p1 = pot1.cpu().numpy()
    agree = float(np.linalg.norm(pg[:, 0] - p1) / np.linalg.norm(p1))
    # roofline: batched translations (M2L) against the FP64 peak
    p = info["nterms"]
    avg = {k: v / args.steps for k, v in step_ms.items()}
    m2l_pairs = sum(lvl["m2l_pairs"])
    if helm:
        flops_m2l = sum(c * nd_htrans3_flops(o, o, nd) for c, o in zip(lvl["m2l_pairs"], orders))
        per_trans = {"per_level_order": orders, "m2l_pairs_per_level": lvl["m2l_pairs"]}
    else:
        flops_m2l = nd_trans3_flops(p, nd, 1) * m2l_pairs
        per_trans = {"translation_nd": nd_trans3_flops(p, nd, 1)}
    achieved = flops_m2l / (avg["m2l_p2l"] * 1e-3) / 1e12
    peak = float(L.zfmm_probe_fp64_tflops(20000))
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        set_omp_threads()
        ncpu = wl["cpu_n"]
        cinp = make_inputs(wl, seed=0, n=ncpu)
        t_cpu, cores, nrep = cpu_time_oracle(wl, cinp, reps_min=1, budget_s=12.0)
        cpu = {"value": ncpu / t_cpu, "unit": "targets/s", "cores": cores, "kind": "port",
               "sample": (f"one right-hand side on {ncpu} points of the workload's distribution "
                          f"(full workload: {n} points x {nd} right-hand sides, which the "
                          f"reference solves as {nd} sequential calls), median of {nrep}")}
    if rank != 0:
        return
    line = {
        "metric": "targets/sec at eps=1e-9", "value": value, "unit": "targets/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "nrhs": nd_total, "eps": eps, "ifpgh": ifpgh,
                   "isep": isep, "charges": True, "dipoles": bool(ifd),
                   **({"zk": [zk.real, zk.imag]} if helm else {}),
                   "step": "plan (tree, lists, centres) + one solve of all right-hand sides",
                   "l2": "flushed (256 MiB write) between steps",
                   "parallelism": (f"right-hand sides sharded over {ws} ranks ({nd} on rank 0)"
                                   if ws > 1 else "one GPU"),
                   "nboxes": info["nboxes"], "nlevels": info["nlevels"], "nterms": p},
        "e2e": {"value": n * nd_total * args.steps / e2e_tot, "unit": "targets/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "plan_build_ms": plan_ms,
        "plain_single_rhs": {"value": plain_value, "unit": "targets/s", "ms_per_solve": plain_ms,
                             "batched_per_rhs_speedup": value / ws / plain_value},
        "rel_l2_err_vs_direct": max(errs),
        "rel_l2_batched_vs_plain_rhs0": agree,
        "step_ms": {k: round(v, 4) for k, v in avg.items()},
        "roofline": {"bound": "fp64",
                     "kernel": "m2l_p2l (%s)" % ("k_htrans3nd" if helm else "k_trans3nd"),
                     "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "peak_source": "measured FP64 FMA probe (zfmm_probe_fp64_tflops)",
                     "traffic": None, "flops_per_step": flops_m2l,
                     "flop_model": dict(per_trans, m2l_pairs=m2l_pairs)},
        "interactions": counts,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_ours_batched2d(args, wl, ws, rank, local):
    """zhfmm2d plan solve of nd right-hand sides on the curve: one step = plan
    (quadtree, lists, centres) + one solve of all right-hand sides, whose M2L
    runs for groups of up to 64 right-hand sides on the tensor cores when
    eps >= 1e-7 (TF32 three-term split) and in FP64 below."""
    import ctypes

    import torch

    import zfmm_b200
    from zfmm_b200 import _capi, shard
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _capi.lib()
    n, nd_total = wl["n"], wl["nrhs"]
    r0, r1 = shard.rhs_block(nd_total, rank, ws)
    nd = r1 - r0
    eps, isep, ifpgh = wl["eps"], wl["isep"], wl["ifpgh"]
    zk = complex(wl["zk"])
    zka = np.array([zk.real, zk.imag])
    zkp = zka.ctypes.data_as(ctypes.c_void_p)
    from zfmm_b200 import workloads as W
    w = W.curve2d(n, seed=0)
    rng = np.random.default_rng(4242)
    cn = lambda *sh: rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    qh, dsh = cn(nd_total, n)[r0:r1], cn(nd_total, n)[r0:r1]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    zs = t(w["zsrc"].T)
    q, ds, dv = t(qh.T), t(dsh.T), t(w["dipvec"].T)
    pot = torch.empty((n, nd), dtype=torch.complex128, device=dev)
    grad = torch.empty((n, 2, nd), dtype=torch.complex128, device=dev)
    pot1 = torch.empty(n, dtype=torch.complex128, device=dev)
    grad1 = torch.empty((n, 2), dtype=torch.complex128, device=dev)
    q0, ds0 = t(qh[0]), t(dsh[0])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    P = lambda x: ctypes.c_void_p(x.data_ptr())

    def solve():
        h = ctypes.c_void_p()
        _capi.check(L.zfmm_plan2d_create_dev(eps, n, P(zs), n, P(zs), isep, sp, ctypes.byref(h)))
        _capi.check(L.zfmm_zhfmm2d_plan_dev(h, zkp, nd, 1, P(q), 1, P(ds), P(dv), ifpgh, P(pot),
                                            P(grad), sp))
        _capi.check(L.zfmm_plan2d_destroy(h))

    def solve_plain():
        _capi.check(L.zfmm_zhfmm2d_dev(eps, zkp, n, P(zs), 1, P(q0), 1, P(ds0), P(dv), P(pot1),
                                       P(grad1), n, P(zs), ifpgh, isep, sp))

    for _ in range(max(args.warmup, 3)):
        solve()
    # interaction counts of one right-hand side (not timed)
    L.zfmm_set_step_timing(2)
    solve_plain()
    counts, _ = zfmm_b200.last_counts()
    L.zfmm_set_step_timing(1)
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    parts = {"upward": 0.0, "m2l": 0.0, "downward": 0.0}
    launches0 = L.zfmm_launch_count()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev0[k].record(stream)
            solve()
            ev1[k].record(stream)
            st, _ = zfmm_b200.last_step_times()
            parts["upward"] += st["p2m"]
            parts["m2l"] += st["m2l_p2l"]
            parts["downward"] += st["eval"]
        torch.cuda.synchronize()
    launches = L.zfmm_launch_count() - launches0
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    if ws > 1:
        tt = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    value = n * nd_total * args.steps / (tot_ms * 1e-3)
    for _ in range(2):
        solve_plain()
    torch.cuda.synchronize()
    pl = []
    for k in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(k & 255)
        e0.record(stream)
        solve_plain()
        e1.record(stream)
        torch.cuda.synchronize()
        pl.append(e0.elapsed_time(e1))
    plain_ms = statistics.median(pl)
    L.zfmm_set_step_timing(0)
    # end to end through the host plan entry points
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hz, hq, hds, hdv = pin(w["zsrc"].T), pin(qh.T), pin(dsh.T), pin(w["dipvec"].T)
    hpot = torch.empty((n, nd), dtype=torch.complex128).pin_memory().numpy()
    hgrad = torch.empty((n, 2, nd), dtype=torch.complex128).pin_memory().numpy()
    hp = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def solve_host():
        h = ctypes.c_void_p()
        _capi.check(L.zfmm_plan2d_create(eps, n, hp(hz), n, hp(hz), isep, ctypes.byref(h)))
        _capi.check(L.zfmm_zhfmm2d_plan(h, zkp, nd, 1, hp(hq), 1, hp(hds), hp(hdv), ifpgh,
                                        hp(hpot), hp(hgrad)))
        _capi.check(L.zfmm_plan2d_destroy(h))

    solve_host()
    t0 = time.perf_counter()
    for k in range(args.steps):
        solve_host()
    e2e_s = time.perf_counter() - t0
    h2d = hz.nbytes + hq.nbytes + hds.nbytes + hdv.nbytes
    d2h = hpot.nbytes + hgrad.nbytes
    # accuracy: right-hand sides 0 and nd-1 against the FP64 direct sum, and
    # against the single FP64 solve of right-hand side 0
    pg = pot.cpu().numpy()
    sub = np.sort(np.random.default_rng(1234).choice(n, size=min(n, 1024), replace=False))
    errs = []
    for r in (0, nd - 1):
        pd, _ = zfmm_b200.zh2devaldirect(zk, len(sub), w["zsrc"][:, sub], n, w["zsrc"], qh[r],
                                         dsh[r], w["dipvec"], 1, 1, 1)
        errs.append(float(np.linalg.norm(pg[sub, r] - 0.25j * pd) / np.linalg.norm(0.25j * pd)))
    p1 = pot1.cpu().numpy()
    agree = float(np.linalg.norm(pg[:, 0] - p1) / np.linalg.norm(p1))
    tc = eps >= 1e-7
    avg = {k: v / args.steps for k, v in parts.items()}
    flops_m2l = 8.0 * counts["m2l_pairs_P"] * nd
    achieved = flops_m2l / (avg["m2l"] * 1e-3) / 1e12 if avg["m2l"] > 0 else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    if tc:
        peak = peaks.get("bf16_tflops", 1590.0) / 2
        psrc = ("dense TF32 = half the measured dense bf16 GEMM rate (MEASURED_PEAKS "
                "bf16_tflops); the three-term split issues 3 TF32 products per useful one")
    else:
        peak = float(L.zfmm_probe_fp64_tflops(20000))
        psrc = "measured FP64 FMA probe (zfmm_probe_fp64_tflops)"
    if rank != 0:
        return
    line = {
        "metric": "targets/sec at eps=%g" % eps, "value": value, "unit": "targets/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "nrhs": nd_total, "eps": eps,
                   "zk": [zk.real, zk.imag], "ifpgh": ifpgh, "isep": isep, "charges": True,
                   "dipoles": True,
                   "m2l": ("tcgen05 TF32 three-term split, 64 right-hand sides per panel"
                           if tc else "FP64, per right-hand side"),
                   "step": "plan (quadtree, lists, centres) + one solve of all right-hand sides",
                   "l2": "flushed (256 MiB write) between steps",
                   "parallelism": (f"right-hand sides sharded over {ws} ranks" if ws > 1
                                   else "one GPU")},
        "e2e": {"value": n * nd_total * args.steps / e2e_s, "unit": "targets/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "plain_single_rhs": {"ms_per_solve": plain_ms, "value": n / (plain_ms * 1e-3),
                             "batched_per_rhs_speedup": (value / ws) / (n / (plain_ms * 1e-3))},
        "rel_l2_err_vs_direct": max(errs),
        "rel_l2_batched_vs_plain_rhs0": agree,
        "step_ms": {k: round(v, 4) for k, v in avg.items()},
        "roofline": {"bound": "tensor" if tc else "fp64", "kernel": "m2l (k_hm2l_tc)" if tc
                     else "m2l (k_hm2l)", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if achieved else None,
                     "peak_source": psrc, "traffic": None, "flops_per_step": flops_m2l,
                     "flop_model": "8 P^2 real flops per (box pair, right-hand side)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def run_ours_many(args, wl, ws, rank, local):
    """One step = all instances through the many-instance device entry point."""
    import ctypes

    import torch

    import zfmm_b200
    from zfmm_b200 import _capi
    from zfmm_b200 import workloads as W
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _capi.lib()
    from zfmm_b200 import shard
    # one set of instances for the whole job; with N ranks each solves the
    # share zfmm_b200.shard assigns it by size (independent units, no
    # collective on the data path)
    rng = np.random.default_rng(2024)
    ni_all = wl["instances"]
    all_sizes = np.exp(rng.uniform(np.log(wl["nmin"]), np.log(wl["nmax"]),
                                   ni_all)).astype(np.int64)
    mine = shard.partition_by_size(all_sizes, ws)[rank]
    sizes = all_sizes[mine]
    ni = len(mine)
    eps, zk, ifpgh, isep = wl["eps"], wl["zk"], wl["ifpgh"], wl["isep"]
    inst = [W.sphere3d(int(all_sizes[i]), seed=i) for i in mine]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dz = [t(w["zsrc"].T) for w in inst]
    dq = [t(w["charge"]) for w in inst]
    dd = [t(w["dipstr"]) for w in inst]
    dv = [t(w["dipvec"].T) for w in inst]
    dp = [torch.empty(int(n), dtype=torch.complex128, device=dev) for n in sizes]
    dg = [torch.empty((int(n), 3), dtype=torch.complex128, device=dev) for n in sizes]
    arr = lambda xs: (ctypes.c_void_p * ni)(*[x.data_ptr() for x in xs])
    A = dict(zs=arr(dz), q=arr(dq), d=arr(dd), v=arr(dv), p=arr(dp), g=arr(dg))
    ns = np.ascontiguousarray(sizes.astype(np.int32))
    k = np.array([zk.real, zk.imag])
    done = np.zeros(ni)
    hp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def solve(nstreams):
        _capi.check(L.zfmm_zhfmm3d_many_dev(ni, eps, hp(k), hp(ns), A["zs"], 1, A["q"], 1, A["d"],
                                            A["v"], hp(ns), A["zs"], ifpgh, isep, A["p"],
                                            A["g"], nstreams, hp(done)))

    nst = args.nstreams or wl["nstreams"]
    for _ in range(max(1, min(args.warmup, 1))):
        solve(nst)
    torch.cuda.synchronize()
    launches0 = L.zfmm_launch_count()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    lat = []
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    with ClockSampler(local) as clk:
        for s_ in range(args.steps):
            flush.fill_(s_ & 255)
            torch.cuda.synchronize()
            ev0[s_].record(stream)
            solve(nst)
            ev1[s_].record(stream)
            torch.cuda.synchronize()
            lat.append(done.copy())
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    if ws > 1:
        tt = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    npts = int(all_sizes.sum())
    value = npts * args.steps / (tot_ms * 1e-3)
    lat_all = np.concatenate(lat)
    # the same instances one after another on one stream (the plain calls)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solve(1)
    e1.record(stream)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    # end to end: host arrays through the host entry point
    hz = [np.ascontiguousarray(w["zsrc"].T) for w in inst]
    hq = [np.ascontiguousarray(w["charge"]) for w in inst]
    hd = [np.ascontiguousarray(w["dipstr"]) for w in inst]
    hv = [np.ascontiguousarray(w["dipvec"].T) for w in inst]
    hpo = [np.zeros(int(n), np.complex128) for n in sizes]
    hgr = [np.zeros((int(n), 3), np.complex128) for n in sizes]
    harr = lambda xs: (ctypes.c_void_p * ni)(*[x.ctypes.data for x in xs])
    H = dict(zs=harr(hz), q=harr(hq), d=harr(hd), v=harr(hv), p=harr(hpo), g=harr(hgr))
    t0 = time.perf_counter()
    _capi.check(L.zfmm_zhfmm3d_many(ni, eps, hp(k), hp(ns), H["zs"], 1, H["q"], 1, H["d"],
                                    H["v"], hp(ns), H["zs"], ifpgh, isep, H["p"], H["g"], nst,
                                    hp(done)))
    e2e_s = time.perf_counter() - t0
    h2d = sum(a.nbytes for a in hz) + sum(a.nbytes for a in hq + hd + hv)  # targets = sources
    d2h = sum(a.nbytes for a in hpo + hgr)
    # accuracy: the largest instance against the FP64 direct sum on 1024 targets
    big = int(np.argmax(sizes))
    w = inst[big]
    n = int(sizes[big])
    sub = np.sort(np.random.default_rng(1234).choice(n, size=min(n, 1024), replace=False))
    pd, _ = zfmm_b200.zh3devaldirect(zk, len(sub), w["zsrc"][:, sub], n, w["zsrc"], w["charge"],
                                     w["dipstr"], w["dipvec"], 1, 1, 1)
    pg = dp[big].cpu().numpy()
    relerr = float(np.linalg.norm(pg[sub] - pd) / np.linalg.norm(pd))
    # roofline: the largest instance's M2L as a single instrumented call
    L.zfmm_set_step_timing(2)
    pb, gb = torch.empty_like(dp[big]), torch.empty_like(dg[big])
    P_ = lambda x: ctypes.c_void_p(x.data_ptr())
    sp = ctypes.c_void_p(stream.cuda_stream)
    _capi.check(L.zfmm_zhfmm3d_dev(eps, hp(k), n, P_(dz[big]), 1, P_(dq[big]), 1, P_(dd[big]),
                                   P_(dv[big]), P_(pb), P_(gb), n, P_(dz[big]), ifpgh, isep, sp))
    st, info = zfmm_b200.last_step_times()
    lvl, orders = zfmm_b200.last_level_counts()
    L.zfmm_set_step_timing(0)
    launches = L.zfmm_launch_count() - launches0
    flops, _per = flop_model3d("helm3d", lvl, orders)
    achieved = flops["m2l_p2l"] / (st["m2l_p2l"] * 1e-3) / 1e12
    peak = float(L.zfmm_probe_fp64_tflops(20000))
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        set_omp_threads()
        cinp = make_inputs(wl, seed=0, n=wl["cpu_n"])
        t_cpu, cores, nrep = cpu_time_oracle(wl, cinp, reps_min=1, budget_s=12.0)
        cpu = {"value": wl["cpu_n"] / t_cpu, "unit": "targets/s", "cores": cores, "kind": "port",
               "sample": (f"one {wl['cpu_n']}-point instance of the workload's distribution "
                          f"(the reference runs the {ni} instances as sequential calls), "
                          f"median of {nrep}")}
    if rank != 0:
        return
    line = {
        "metric": "targets/sec at eps=1e-9", "value": value, "unit": "targets/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "instances": ni_all, "points_total": npts,
                   "instances_rank0": ni,
                   "n_min": int(all_sizes.min()), "n_max": int(all_sizes.max()), "eps": eps,
                   "zk": str(zk), "ifpgh": ifpgh, "isep": isep, "charges": True,
                   "dipoles": True, "nstreams": nst,
                   "timing": ("CUDA events on the current stream bracketing the call, which "
                              "returns after every worker stream has finished"),
                   "l2": "flushed (256 MiB write) between steps",
                   "parallelism": (f"instances sharded by size over {ws} ranks"
                                   if ws > 1 else "one GPU")},
        "latency_ms": {"p50": float(np.percentile(lat_all, 50)),
                       "p99": float(np.percentile(lat_all, 99)),
                       "max": float(lat_all.max())},
        "sequential_one_stream_ms": seq_ms,
        "e2e": {"value": ws * npts / e2e_s, "unit": "targets/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "rel_l2_err_vs_direct": relerr,
        "roofline": {"bound": "fp64", "kernel": "m2l_p2l of the largest instance",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "peak_source": "measured FP64 FMA probe (zfmm_probe_fp64_tflops)",
                     "traffic": None, "flops_per_step": flops["m2l_p2l"]},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def two_curves(n, seed):
    """The two-curve interface of the adjoint workload: real base points,
    displacement directions (cos 3t, sin 3t), curve index, complex normal
    charges, dipole strengths, dipole vectors and target field."""
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


def run_ours_adjoint(args, wl, ws, rank, local):
    """One step = forward + backward of the differentiable two-curve zhfmm2d."""
    import torch

    import zfmm_b200
    from zfmm_b200 import _capi
    from zfmm_b200.adjoint import zhfmm2d_curves, points
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = _capi.lib()
    n, eps, zk = wl["n"], wl["eps"], wl["zk"]
    xr, disp, curve, q, ds, dv, ref = two_curves(n, 7 + rank)
    T = lambda x: torch.tensor(x, device=dev)
    D = dict(xr=T(xr), disp=T(disp), curve=T(curve), q=T(q), ds=T(ds), dv=T(dv), ref=T(ref))
    # the inner curve is the outer one scaled 0.3 (real and imaginary parts) and
    # shifted by (0.2, 0.1): scaled 0.6 it crosses the outer curve, and there,
    # or with equal amplitudes, the reference algorithm itself misses the
    # direct sum by orders of magnitude (boxes that hold both curves)
    a0 = [0.05, 0.015]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def fwd_bwd(Dx, grads=True, backward=True):
        qq = Dx["q"].clone().requires_grad_(grads)
        dd = Dx["ds"].clone().requires_grad_(grads)
        a = torch.tensor(a0, device=dev, dtype=torch.float64, requires_grad=grads)
        pot = zhfmm2d_curves(eps, zk, Dx["xr"], Dx["disp"], Dx["curve"], a, qq, dd, Dx["dv"])
        Lv = torch.mean(torch.abs(pot - Dx["ref"]) ** 2)
        if grads and backward:
            Lv.backward()
            return Lv, qq.grad, dd.grad, a.grad
        return Lv

    for _ in range(max(args.warmup, 3)):
        fwd_bwd(D)
    torch.cuda.synchronize()
    launches0 = L.zfmm_launch_count()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            ev0[k].record(stream)
            out = fwd_bwd(D)
            ev1[k].record(stream)
        torch.cuda.synchronize()
    launches = L.zfmm_launch_count() - launches0
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(ev0, ev1))
    if ws > 1:
        tt = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot_ms = float(tt.item())
    value = ws * n * args.steps / (tot_ms * 1e-3)
    # the plain forward solve (pot only) and the forward with gradients, same points
    z = points(D["xr"], D["disp"], D["curve"], torch.tensor(a0, device=dev, dtype=torch.float64))
    def timed(f, reps=3):
        f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    plain_ms = timed(lambda: zfmm_b200._fmm2d_torch(eps, zk, n, z, 1, D["q"], 1, D["ds"], D["dv"],
                                                     n, z, 1, 1))
    # the forward as the differentiable call runs it (pot and grad, graph kept)
    fwd_ms = timed(lambda: fwd_bwd(D, grads=True, backward=False))
    step_ms = tot_ms / args.steps
    # gradient checks at full size: central differences of the FMM loss for both
    # amplitudes, at h = 1e-6 and at h = 1e-3 (at 200,000 points the loss moves
    # by ~1e-13 of itself for h = 1e-6, so that difference carries the loss's
    # rounding; the larger step trades it for an O(h^2) truncation error)
    Lv, gq, gds, ga = out
    ga = ga.cpu().numpy()

    def loss_at(av):
        pt = zhfmm2d_curves(eps, zk, D["xr"], D["disp"], D["curve"],
                            torch.tensor(av, device=dev, dtype=torch.float64), D["q"], D["ds"],
                            D["dv"])
        return float(torch.mean(torch.abs(pt - D["ref"]) ** 2))

    fd_rel = {}
    for h in (1e-6, 1e-4, 1e-3):
        errs = []
        for c in range(2):
            ap, am = list(a0), list(a0)
            ap[c] += h
            am[c] -= h
            fdv = (loss_at(ap) - loss_at(am)) / (2 * h)
            errs.append(abs(fdv - ga[c]) / abs(ga[c]))
        fd_rel[f"h={h:g}"] = errs
    # forward accuracy against the FP64 direct sum on 1024 targets
    sub = np.sort(np.random.default_rng(1234).choice(n, size=1024, replace=False))
    zn = z.cpu().numpy()
    pd, _ = zfmm_b200.zh2devaldirect(zk, len(sub), zn[sub].T, n, zn.T, q, ds, dv.T, 1, 1, 1)
    pf, _ = zfmm_b200._fmm2d_torch(eps, zk, n, z, 1, D["q"], 1, D["ds"], D["dv"], n, z, 1, 1)
    pf = pf.cpu().numpy()[sub]
    relerr = float(np.linalg.norm(pf - 0.25j * pd) / np.linalg.norm(0.25j * pd))
    # end to end: inputs from pinned host memory, gradients back to the host
    hin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
           for k, v in dict(xr=xr, disp=disp, curve=curve, q=q, ds=ds, dv=dv, ref=ref).items()}
    t0 = time.perf_counter()
    for k in range(args.steps):
        Dh = {kk: vv.to(dev, non_blocking=True) for kk, vv in hin.items()}
        _, g1, g2, g3 = fwd_bwd(Dh)
        g1.cpu(), g2.cpu(), g3.cpu()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    h2d = sum(v.numel() * v.element_size() for v in hin.values())
    d2h = 2 * n * 16 + 2 * 8
    # roofline of the forward's dominant step (an instrumented forward solve)
    L.zfmm_set_step_timing(2)
    zfmm_b200._fmm2d_torch(eps, zk, n, z, 1, D["q"], 1, D["ds"], D["dv"], n, z, 2, 1)
    torch.cuda.synchronize()
    torch.cuda.synchronize()
    counts, _ = zfmm_b200.last_counts()
    st, info = zfmm_b200.last_step_times()
    L.zfmm_set_step_timing(0)
    flops, _per = flop_model("helm2d", counts)
    top = max(flops, key=lambda k: st[k])
    achieved = flops[top] / (st[top] * 1e-3) / 1e12
    peak = float(L.zfmm_probe_fp64_tflops(20000))
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        set_omp_threads()
        ncpu = wl["cpu_n"]
        zc = points(*(torch.tensor(x) for x in (xr[:ncpu], disp[:ncpu], curve[:ncpu])),
                    torch.tensor(a0, dtype=torch.float64)).numpy()
        cinp = dict(zsrc=zc.T, charge=q[:ncpu], dipstr=ds[:ncpu], dipvec=dv[:ncpu].T)
        t_cpu, cores, nrep = cpu_time_oracle(wl, cinp, reps_min=1, budget_s=12.0)
        cpu = {"value": ncpu / t_cpu, "unit": "targets/s", "cores": cores, "kind": "port",
               "sample": (f"one forward solve (pot and grad) on the first {ncpu} points of the "
                          f"workload (full: {n}); the reference has no adjoint"),
               "median_of": nrep}
    if rank != 0:
        return
    line = {
        "metric": "targets/sec at eps=1e-10 (forward + adjoint)", "value": value,
        "unit": "targets/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "eps": eps, "zk": str(zk), "ifpgh": 2,
                   "isep": 1, "charges": True, "dipoles": True,
                   "step": "forward (pot, grad) + backward (charge, dipstr, 2 amplitudes)",
                   "l2": "flushed (256 MiB write) between steps",
                   "parallelism": f"replicas x{ws}"},
        "forward_plain_ms": plain_ms, "forward_with_grad_ms": fwd_ms,
        "backward_ms": step_ms - fwd_ms,
        "backward_over_plain_forward": (step_ms - fwd_ms) / plain_ms,
        "grad_check_fd_rel": fd_rel,
        "rel_l2_err_vs_direct": relerr,
        "e2e": {"value": ws * n * args.steps / e2e_s, "unit": "targets/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "fp64", "kernel": f"forward {top}", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "peak_source": "measured FP64 FMA probe (zfmm_probe_fp64_tflops)",
                     "traffic": None, "flops_per_step": flops[top]},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--nstreams", type=int, default=None,
                    help="host workers / streams of the many-instance workload")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-right-hand-side key of the default line")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, wl, ws, rank)
        elif wl.get("adjoint"):
            run_ours_adjoint(args, wl, ws, rank, local)
        elif wl.get("instances"):
            run_ours_many(args, wl, ws, rank, local)
        elif wl.get("nrhs", 1) > 1 and wl["kind"] == "helm2d":
            run_ours_batched2d(args, wl, ws, rank, local)
        elif wl.get("nrhs", 1) > 1:
            run_ours_batched(args, wl, ws, rank, local)
        else:
            run_ours(args, wl, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
