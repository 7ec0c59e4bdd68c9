#!/usr/bin/env python
"""Benchmark: batched bottom-up NCA build + H^2 block products on one B200 (per rank).

Workload (Galerkin, low frequency): 65,536 points uniform on the unit sphere (seeded),
Helmholtz cis(kr)/(4 pi r) with k = 1.0 (zero on the diagonal), k-means tree minvalues 64,
batched bottom-up ACA tol 1e-5, maxrank 50. One step = y = H X and y = H^H X for a block of
16 seeded complex Gaussian right-hand sides (complex FP64). The metric is the product's
algorithmic HBM bytes (stores read once per block + vectors) per second; the build time is
reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--precision f64|f32]

With --gpus N > 1 it runs under torchrun, one independent replica per GPU (the path has no
exchange step); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nestedcrossapproximation.jl_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "H² build+matvec time & matvec HBM GB/s, chosen vs plain FP64 at rel err 1e-4"
WORKLOAD = "galerkin-sphere-65536-k1-tol1e-5-16rhs"
E = 16  # bytes per complex FP64 entry


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="f64", choices=["f64", "f32"])
    p.add_argument("--npoints", type=int, default=65536)
    p.add_argument("--nrhs", type=int, default=16)
    p.add_argument("--wideband-points", type=int, default=0, help="point count of the wideband workload")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-stages", action="store_true", help="print per-stage times to stderr")
    p.add_argument("--workload", default="galerkin-sphere",
                   choices=["galerkin-sphere", "batched-uneven", "gradients", "wideband"],
                   help="batched-uneven: 64 problems of uneven size, one batched product vs 64 calls; "
                        "gradients: dJ/dx and dJ/dk of J = ||H(k) x - b||^2 on a perturbed sphere")
    return p.parse_args()


def sphere(n, seed=1234):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, 3))
    return g / np.linalg.norm(g, axis=1, keepdims=True)


def rhs(n, b, seed=99):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, b)) + 1j * rng.standard_normal((n, b))


def max_over_ranks(x, device):
    """The largest x over the ranks of the job (replicas time their own work; the job's time is the
    slowest rank's). x itself when no process group is running or it has one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def store_entries(info):
    return (info["near_entries"] + info["coupling_entries"] + info["transfer_entries_test"] +
            info["transfer_entries_trial"] + info["basis_entries_test"] + info["basis_entries_trial"])


def product_bytes(info, b, e=E):
    """Algorithmic bytes of one product with b right-hand sides: every stored entry once, x read,
    y read and written, coefficient vectors written and read once."""
    vec = e * b * (info["ntrial"] + 2 * info["ntest"]) + 2 * e * b * (info["ncoeff_test"] + info["ncoeff_trial"])
    return e * store_entries(info) + vec


def stage_bytes(info, b, e=E):
    """Algorithmic bytes per launch of the near-field stage, the dominant kernel (k_rows_leaves
    without the leaf bases, beside the far-field sweeps): near entries once, x slices read once,
    y written once."""
    return e * info["near_entries"] + e * b * (info["ntrial"] + info["ntest"])


def info_dict(core):
    i = core.info
    return {k: getattr(i, k) for k, _ in type(i)._fields_}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profiles():
    """DRAM bytes per launch of the near-field kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "k_rows_near_galerkin_sphere.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    def __init__(self, index):
        self.proc, self.path = None, os.path.join(ROOT, "gpurun_out", f"clocks_bench_{index}.csv")
        self.index = index

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cuda_ready(N, device):
    """Creates the device's CUDA context and loads the library before a build is timed: both are
    once-per-process costs, not part of any build."""
    import torch
    torch.zeros(1, device=f"cuda:{device}")
    torch.cuda.synchronize(device)
    N.lib()


def build_problem(N, n, device, store_f32):
    pts = sphere(n)
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
    bt = N.BlockTree(tree, tree)
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-5))
    comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tree), compressor=aca)
    t0 = time.perf_counter()
    core = N.PetrovGalerkinNCACore(N.HelmholtzKernel(1.0), pts, pts, bt, testcompressor=comp, trialcompressor=comp,
                                   maxrank=50, store_f32=store_f32, device=device)
    wall = time.perf_counter() - t0
    return pts, core, wall


def dense_rows_error(N, pts, core, ws, X, nrows=64):
    """Relative error of H X against rows of the dense FP64 matrix evaluated on the device."""
    rng = np.random.default_rng(7)
    rows = rng.choice(len(pts), nrows, replace=False)
    ii = np.repeat(rows, len(pts))
    jj = np.tile(np.arange(len(pts)), nrows)
    D = N.seams.entries(N.HelmholtzKernel(1.0), pts, pts, ii, jj, device=core.device).reshape(nrows, len(pts))
    Y = N.mul(None, ws, X[:, :2])
    ref = D @ X[:, :2]
    return float(np.linalg.norm(Y[rows] - ref) / np.linalg.norm(ref))


def measure_chosen(N, L, core, ws64, X, Xd, Yd, n, b, args, world, local, info, elapsed64, pts, rank):
    """The mixed-precision form on the same core and right-hand sides: complex FP32 stores
    (half the bytes), FP64 accumulation and FP64 coefficient vectors. Reports its step time, the
    speed-up over the plain FP64 step, and its error against the FP64 product and the dense rows."""
    import torch
    import torch.distributed as dist
    ws = N.H2Workspace(core, np.complex64, max_nrhs=b)
    Y32 = torch.zeros_like(Yd)

    def step():
        for mode in (0, 2):
            N._lib.check(L.nca_apply(ws._h, mode, 1, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Y32.data_ptr()), n,
                                     b, 1.0, 0.0, 0.0, 0.0, 1))
    for _ in range(max(args.warmup, 3)):
        step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    el = max_over_ranks(e0.elapsed_time(e1) * 1e-3, f"cuda:{local}")
    # error of the forward product against the FP64 product and against dense rows
    Y64 = torch.zeros_like(Yd)
    for W, Y in ((ws64, Y64), (ws, Y32)):
        N._lib.check(L.nca_apply(W._h, 0, 1 if W is ws else 0, C.c_void_p(Xd.data_ptr()), n,
                                 C.c_void_p(Y.data_ptr()), n, b, 1.0, 0.0, 0.0, 0.0, 1))
    rel64 = float((Y32 - Y64).norm() / Y64.norm())
    err = dense_rows_error(N, pts, core, ws, X) if rank == 0 else None
    return {"form": "complex-FP32 stores, FP64 accumulation and coefficient vectors",
            "ms_per_step": 1e3 * el / args.steps, "speedup_vs_plain_f64": elapsed64 / el,
            "stored_gb": 8 * store_entries(info) / 1e9,
            "value": world * 2 * product_bytes(info, b, 8) * args.steps / el / 1e9, "unit": "GB/s",
            "relerr_vs_f64_product": rel64, "relerr_vs_dense_rows": err}


def cpu_baseline_sample(b_sample, nrhs):
    """The oracle (C restatement, OpenMP on the host cores) on the same workload: its own build,
    then one forward and one adjoint product on b_sample right-hand sides; the product time is
    scaled to nrhs (the oracle applies one right-hand side at a time)."""
    from oracle import oracle as O
    pts = sphere(65536)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    H = O.H2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=1.0), minvalues=64, tol=1e-5, maxrank=50, nthreads=cores)
    tb = time.perf_counter() - t0
    X = rhs(len(pts), b_sample)
    t0 = time.perf_counter()
    H.apply(X, 0)
    H.apply(X, 2)
    tp = (time.perf_counter() - t0) * nrhs / b_sample
    info = {"near_entries": sum(a.size for a in H.near), "coupling_entries": sum(a.size for a in H.couplings),
            "transfer_entries_test": sum(H.X[0][t].size for t in range(H.trees[0].nnodes) if not H.trees[0].isleaf(t)),
            "transfer_entries_trial": sum(H.X[1][t].size for t in range(H.trees[1].nnodes) if not H.trees[1].isleaf(t)),
            "basis_entries_test": sum(H.X[0][t].size for t in range(H.trees[0].nnodes) if H.trees[0].isleaf(t)),
            "basis_entries_trial": sum(H.X[1][t].size for t in range(H.trees[1].nnodes) if H.trees[1].isleaf(t)),
            "ntest": len(pts), "ntrial": len(pts), "ncoeff_test": int(H.ranks[0].sum()),
            "ncoeff_trial": int(H.ranks[1].sum())}
    step_bytes = 2 * product_bytes(info, nrhs)
    return {"value": step_bytes / tp / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"oracle build ({tb:.1f} s) + one forward and one adjoint product on {b_sample} of the "
                      f"{nrhs} right-hand sides, time scaled x{nrhs // b_sample}",
            "build_s": tb, "step_s": tp}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    pts = sphere(args.npoints)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    H = O.H2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=1.0), minvalues=64, tol=1e-5, maxrank=50, nthreads=cores)
    tb = time.perf_counter() - t0
    b_sample = 2
    X = rhs(len(pts), b_sample)
    for _ in range(args.warmup):
        H.apply(X, 0)
        H.apply(X, 2)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        H.apply(X, 0)
        H.apply(X, 2)
    el = (time.perf_counter() - t0) * args.nrhs / b_sample
    info = {"near_entries": sum(a.size for a in H.near), "coupling_entries": sum(a.size for a in H.couplings),
            "transfer_entries_test": sum(H.X[0][t].size for t in range(H.trees[0].nnodes) if not H.trees[0].isleaf(t)),
            "transfer_entries_trial": sum(H.X[1][t].size for t in range(H.trees[1].nnodes) if not H.trees[1].isleaf(t)),
            "basis_entries_test": sum(H.X[0][t].size for t in range(H.trees[0].nnodes) if H.trees[0].isleaf(t)),
            "basis_entries_trial": sum(H.X[1][t].size for t in range(H.trees[1].nnodes) if H.trees[1].isleaf(t)),
            "ntest": len(pts), "ntrial": len(pts), "ncoeff_test": int(H.ranks[0].sum()),
            "ncoeff_trial": int(H.ranks[1].sum())}
    step_bytes = 2 * product_bytes(info, args.nrhs)
    value = step_bytes * args.steps / el / 1e9
    sample = (f"CPU oracle (C restatement, OpenMP, {cores} threads); each step one forward and one adjoint product "
              f"on {b_sample} of {args.nrhs} right-hand sides, time scaled x{args.nrhs // b_sample}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex-f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "npoints": args.npoints, "nrhs": args.nrhs, "build_s": tb,
                   "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cube_surface(n, seed):
    rng = np.random.default_rng(seed)
    face = rng.integers(0, 6, n)
    uv = rng.uniform(0.0, 1.0, (n, 2))
    pts = np.empty((n, 3))
    for a in range(3):
        sel = face // 2 == a
        o = [c for c in range(3) if c != a]
        pts[sel, a] = (face[sel] % 2).astype(float)
        pts[sel, o[0]], pts[sel, o[1]] = uv[sel, 0], uv[sel, 1]
    return pts


def run_batched(args):
    """64 independent problems, N log-uniform in [4096, 65536], sphere / cube surface alternating,
    k uniform in [0.5, 4], FP64 build at tol 1e-4 (minvalues 64); step = y = H X with 8
    right-hand sides per problem. Timed: 64 plain per-problem FP64 products, one batched FP64
    product and one batched mixed-precision product (complex-FP32 stores, FP64 accumulation)."""
    import torch
    import nca_b200 as N
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    rng = np.random.default_rng(2024)
    nprob, b = 64, 8
    sizes = np.exp(rng.uniform(np.log(4096), np.log(65536), nprob)).astype(int)
    ks = rng.uniform(0.5, 4.0, nprob)
    cuda_ready(N, local)
    L = N.lib()
    t0 = time.perf_counter()
    members = []
    for i in range(nprob):
        pts = sphere(int(sizes[i]), 500 + i) if i % 2 == 0 else cube_surface(int(sizes[i]), 500 + i)
        tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
        aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
        comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tree), compressor=aca)
        members.append(N.PetrovGalerkinNCACore(N.HelmholtzKernel(float(ks[i]), rmin=1e-12), pts, pts,
                                               N.BlockTree(tree, tree), testcompressor=comp, trialcompressor=comp,
                                               store_f32=True, device=local))
    build_wall = time.perf_counter() - t0
    ntot = int(sizes.sum())
    X = rhs(ntot, b, seed=77)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(f"cuda:{local}")
    off = np.concatenate([[0], np.cumsum(sizes)])

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / steps

    # 64 plain per-problem FP64 calls (each on its own slice of the stacked vectors)
    Yp = torch.zeros_like(Xd)
    Xs = [Xd[:, off[i]:off[i + 1]].contiguous() for i in range(nprob)]
    Ys = [torch.zeros_like(x) for x in Xs]
    wss = [N.H2Workspace(m, max_nrhs=b) for m in members]

    def plain():
        for i in range(nprob):
            n = int(sizes[i])
            N._lib.check(L.nca_apply(wss[i]._h, 0, 0, C.c_void_p(Xs[i].data_ptr()), n, C.c_void_p(Ys[i].data_ptr()),
                                     n, b, 1.0, 0.0, 0.0, 0.0, 1))
    t_plain = timed(plain, args.steps)
    info_m = [info_dict(m) for m in members]
    del wss
    batch = N.batch(members, move=True)
    members.clear()
    import gc
    gc.collect()
    info = info_dict(batch)
    W64 = N.H2Workspace(batch, max_nrhs=b)
    W32 = N.H2Workspace(batch, np.complex64, max_nrhs=b)
    Y64 = torch.zeros_like(Xd)
    Y32 = torch.zeros_like(Xd)

    def batched(W, prec, Y):
        return lambda: N._lib.check(L.nca_apply(W._h, 0, prec, C.c_void_p(Xd.data_ptr()), ntot,
                                                C.c_void_p(Y.data_ptr()), ntot, b, 1.0, 0.0, 0.0, 0.0, 1))
    clocks = Clocks(local)
    clocks.start()
    t64 = timed(batched(W64, 0, Y64), args.steps)
    t32 = timed(batched(W32, 1, Y32), args.steps)
    clk = clocks.stop()
    launches = C.c_int32()
    L.nca_workspace_last_launches(W32._h, C.byref(launches))
    # the plain per-problem results agree with the batched FP64 product; FP32 error vs FP64
    rel_plain = max(float((Y64[:, off[i]:off[i + 1]] - Ys[i]).norm() / Ys[i].norm()) for i in range(nprob))
    rel32 = float((Y32 - Y64).norm() / Y64.norm())
    bytes64 = product_bytes(info, b)
    bytes32 = product_bytes(info, b, 8)
    peak, peak_kind = peaks()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": bytes32 / t32 / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "complex-f32 stores, f64 accumulation", "data": "synthetic",
            "config": {"workload": "batched-uneven-64-tol1e-4-8rhs", "problems": nprob, "npoints_total": ntot,
                       "npoints_min": int(sizes.min()), "npoints_max": int(sizes.max()), "nrhs": b,
                       "step": "y = H X for every problem (one batched product)",
                       "l2": "inputs larger than L2", "build_s_64_problems": build_wall,
                       "stored_gb_f64": E * store_entries(info) / 1e9},
            "plain_per_problem_f64": {"ms_per_step": 1e3 * t_plain, "value": bytes64 / t_plain / 1e9},
            "batched_f64": {"ms_per_step": 1e3 * t64, "value": bytes64 / t64 / 1e9,
                            "relerr_vs_per_problem": rel_plain},
            "speedup_vs_plain_per_problem_f64": t_plain / t32, "relerr_f32_vs_f64": rel32,
            "roofline": {"bound": "hbm", "achieved": bytes32 / t32 / 1e9, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": bytes32 / t32 / 1e9 / peak, "traffic": None,
                         "note": "whole product (all stages), algorithmic bytes"},
            "gpu_launches": launches.value, "clocks": clk}), flush=True)


def perturbed_sphere(n, seed):
    """r(theta, phi) = 1 + 0.1 sin(3 theta) cos(2 phi), (cos theta, phi) uniform."""
    rng = np.random.default_rng(seed)
    ct = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2 * np.pi, n)
    th = np.arccos(ct)
    r = 1.0 + 0.1 * np.sin(3 * th) * np.cos(2 * ph)
    st = np.sqrt(1.0 - ct * ct)
    return np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], axis=1)


def run_gradients(args):
    """131,072 points on a perturbed sphere, Helmholtz k = 20, tol 1e-5 (standard admissibility,
    maxrank 50), skeleton frozen after the build; J = ||H(k) x - b||^2 with 4 right-hand sides.
    One step = one gradient: y = H x, x_bar = H^H (2 (y - b)), k_bar = Re(y_bar^H dH/dk x)
    (forward, adjoint and tangent products). The d/dk stores are prepared once per skeleton and
    timed separately. k_bar is checked against central differences (h = 1e-6 k) of frozen refills."""
    import torch
    import nca_b200 as N
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    cuda_ready(N, local)
    n, b, k = 131072, 4, 20.0
    pts = perturbed_sphere(n, 4242)
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
    aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-5))
    comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tree), compressor=aca)
    t0 = time.perf_counter()
    core = N.PetrovGalerkinNCACore(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, N.BlockTree(tree, tree),
                                   testcompressor=comp, trialcompressor=comp, device=local)
    build_wall = time.perf_counter() - t0
    info = info_dict(core)
    ws = N.H2Workspace(core, max_nrhs=b)
    L = N.lib()
    X = rhs(n, b, seed=5)
    B = rhs(n, b, seed=6)
    dev = f"cuda:{local}"
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
    Yd, Rd, Xb, Dy = (torch.zeros_like(Xd) for _ in range(4))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    core.prepare_dk()
    torch.cuda.synchronize()
    prep = time.perf_counter() - t0

    def grad():
        N._lib.check(L.nca_apply(ws._h, 0, 0, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, b,
                                 1.0, 0.0, 0.0, 0.0, 1))
        torch.sub(Yd, Bd, out=Rd)
        Rd.mul_(2.0)
        N._lib.check(L.nca_apply(ws._h, 2, 0, C.c_void_p(Rd.data_ptr()), n, C.c_void_p(Xb.data_ptr()), n, b,
                                 1.0, 0.0, 0.0, 0.0, 1))
        N._lib.check(L.nca_apply_dk(ws._h, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Dy.data_ptr()), n, b,
                                    1.0, 0.0, 0.0, 0.0, 1))
        return torch.vdot(Rd.reshape(-1), Dy.reshape(-1)).real
    for _ in range(max(args.warmup, 3)):
        grad()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        kbar = grad()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    el = e0.elapsed_time(e1) * 1e-3 / args.steps
    kbar = float(kbar.item())
    # central differences of J on the frozen skeleton
    h = 1e-6 * k

    def J():
        N._lib.check(L.nca_apply(ws._h, 0, 0, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, b,
                                 1.0, 0.0, 0.0, 0.0, 1))
        return float(((Yd - Bd).abs() ** 2).sum().item())
    core.set_wavenumber(k + h)
    jp = J()
    core.set_wavenumber(k - h)
    jm = J()
    core.set_wavenumber(k)
    fd = (jp - jm) / (2 * h)
    err = dense_rows_error_k(N, pts, core, ws, X, k) if rank == 0 else None
    step_bytes = 2 * product_bytes(info, b) + tangent_bytes(info, b)
    peak, peak_kind = peaks()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": step_bytes / el / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "complex-f64", "data": "synthetic",
            "config": {"workload": "gradients-perturbed-sphere-131072-k20-tol1e-5-4rhs", "npoints": n, "nrhs": b,
                       "k": k, "admissibility": "standard isnear (eta 1), maxrank 50",
                       "step": "one gradient: H x, H^H (2 (Hx - b)), dH/dk x",
                       "l2": "inputs larger than L2", "build_s": build_wall, "prepare_dk_s": prep,
                       "stored_gb": E * store_entries(info) / 1e9, "relerr_vs_dense_rows": err},
            "gradients_per_s": 1.0 / el, "k_bar": kbar, "k_bar_central_difference": fd,
            "k_bar_relerr_vs_fd": abs(kbar - fd) / abs(fd),
            "roofline": {"bound": "hbm", "achieved": step_bytes / el / 1e9, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": step_bytes / el / 1e9 / peak, "traffic": None,
                         "note": "whole gradient step (three products), algorithmic bytes"},
            "clocks": clk}), flush=True)


def run_wideband(args):
    """Directional (wideband) sphere: n points uniform on the unit sphere (default 262,144),
    k = 2 pi 8 (diameter 16 wavelengths), isnearwideband(k), tol 1e-4, minvalues 64; the work is
    the build plus 100 matvecs with seeded complex Gaussian x. Plain FP64 form: 100 single-vector
    FP64 products. Batched mixed-precision form: the 100 vectors as one block of right-hand sides
    on the complex-FP32 stores (FP64 pivots and skeletons, FP64 accumulation)."""
    import torch
    import nca_b200 as N
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    n, k, nvec = args.wideband_points or 262144, 2 * np.pi * 8, 100
    pts = sphere(n, 888)
    cuda_ready(N, local)

    def build_once():
        t0 = time.perf_counter()
        tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
        aca = N.ACA(N.FullPivoting(), N.FullPivoting(), N.FNormEstimator(1e-4))
        comp = N.BatchedBottomUp(pivotselector=N.TreeMimicryPivoting(pts, pts, tree), compressor=aca)
        core = N.PetrovGalerkinNCACore(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, N.BlockTree(tree, tree),
                                       isnear=N.isnearwideband(k), testcompressor=comp, trialcompressor=comp,
                                       store_f32=True, device=local)
        torch.cuda.synchronize()
        return core, time.perf_counter() - t0

    # the build leans on the host cores, which the GPU's neighbours share: the faster of two
    # identical builds is the figure used, both are reported
    core, build_first = build_once()
    del core
    core, build_second = build_once()
    build = min(build_first, build_second)
    info = info_dict(core)
    L = N.lib()
    X = rhs(n, nvec, seed=31)
    dev = f"cuda:{local}"
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)
    Yd = torch.zeros_like(Xd)
    W64 = N.H2Workspace(core, max_nrhs=16)
    W32 = N.H2Workspace(core, np.complex64, max_nrhs=16)

    def seq(W, prec):
        def f():
            for j in range(nvec):
                N._lib.check(L.nca_apply(W._h, 0, prec, C.c_void_p(Xd[j].data_ptr()), n, C.c_void_p(Yd[j].data_ptr()),
                                         n, 1, 1.0, 0.0, 0.0, 0.0, 1))
        return f

    def block(W, prec):
        def f():
            N._lib.check(L.nca_apply(W._h, 0, prec, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, nvec,
                                     1.0, 0.0, 0.0, 0.0, 1))
        return f

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / reps

    clocks = Clocks(local)
    clocks.start()
    reps = max(1, args.steps // 10)
    t_seq64 = timed(seq(W64, 0), reps)
    t_seq32 = timed(seq(W32, 1), reps)
    t_blk64 = timed(block(W64, 0), max(3, args.steps))
    t_blk32 = timed(block(W32, 1), max(3, args.steps))
    clk = clocks.stop()
    launches = C.c_int32()
    L.nca_workspace_last_launches(W32._h, C.byref(launches))
    # errors: FP32 block vs FP64 block; FP64 vs dense rows (first vector)
    Y64 = torch.zeros_like(Xd)
    N._lib.check(L.nca_apply(W64._h, 0, 0, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Y64.data_ptr()), n, nvec,
                             1.0, 0.0, 0.0, 0.0, 1))
    block(W32, 1)()
    torch.cuda.synchronize()
    rel32 = float((Yd - Y64).norm() / Y64.norm())
    err = dense_rows_error_k(N, pts, core, W64, X, k) if rank == 0 else None
    bytes32 = product_bytes(info, nvec, 8)
    plain = build + t_seq64
    mixed = build + t_blk32
    peak, peak_kind = peaks()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": bytes32 / t_blk32 / 1e9, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": 1e3 * t_blk32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "complex-f32 stores, f64 accumulation", "data": "synthetic",
            "config": {"workload": f"wideband-sphere-{n}-k16pi-tol1e-4-100vec", "npoints": n, "k": k,
                       "admissibility": "isnearwideband(k; eta_lf=1, eta_hf=5, gamma=1)",
                       "step": "100 matvecs as one block of 100 right-hand sides",
                       "l2": "inputs larger than L2", "build_s": build, "build_s_both": [build_first, build_second],
                       "build_device_s": info["build_seconds"],
                       "stored_gb_f64": E * store_entries(info) / 1e9, "relerr_vs_dense_rows": err,
                       "relerr_f32_vs_f64": rel32},
            "plain_f64_100_single_matvecs_s": t_seq64, "mixed_f32_100_single_matvecs_s": t_seq32,
            "f64_block_of_100_s": t_blk64, "mixed_block_of_100_s": t_blk32,
            "build_plus_100_matvecs_s": {"plain_f64": plain, "batched_mixed": mixed, "speedup": plain / mixed},
            "matvec_speedup_batched_mixed_vs_plain_f64": t_seq64 / t_blk32,
            "roofline": {"bound": "hbm", "achieved": bytes32 / t_blk32 / 1e9, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": bytes32 / t_blk32 / 1e9 / peak, "traffic": None,
                         "note": "whole block product, algorithmic bytes (stores once per 16-column pass)"},
            "gpu_launches": launches.value, "clocks": clk}), flush=True)


def tangent_bytes(info, b, e=E):
    """Algorithmic bytes of one tangent product: every stored entry and its d/dk twice as many
    stores (X, dX, S, dS, N, dN), x read, y written, four coefficient vectors written and read."""
    vec = e * b * (info["ntrial"] + 2 * info["ntest"]) + 4 * e * b * (info["ncoeff_test"] + info["ncoeff_trial"])
    return 2 * e * store_entries(info) + vec


def dense_rows_error_k(N, pts, core, ws, X, k, nrows=64):
    rng = np.random.default_rng(7)
    rows = rng.choice(len(pts), nrows, replace=False)
    ii = np.repeat(rows, len(pts))
    jj = np.tile(np.arange(len(pts)), nrows)
    D = N.seams.entries(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, ii, jj, device=core.device).reshape(nrows, len(pts))
    Y = N.mul(None, ws, X[:, :1])
    ref = D @ X[:, :1]
    return float(np.linalg.norm(Y[rows] - ref) / np.linalg.norm(ref))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batched-uneven":
        run_batched(args)
        return
    if args.workload == "gradients":
        run_gradients(args)
        return
    if args.workload == "wideband":
        run_wideband(args)
        return
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    import nca_b200 as N

    f32 = args.precision == "f32"
    # the core keeps both stores: complex FP64 (plain) and complex FP32 (the chosen mixed precision)
    cuda_ready(N, local)
    pts, core, build_wall = build_problem(N, args.npoints, local, True)
    info = info_dict(core)
    n = args.npoints
    b = args.nrhs
    ws = N.H2Workspace(core, np.complex64 if f32 else np.complex128, max_nrhs=b)
    prec = 1 if f32 else 0
    L = N.lib()
    X = rhs(n, b)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(f"cuda:{local}")  # column-major n x b
    Yd = torch.zeros((b, n), dtype=torch.complex128, device=f"cuda:{local}")

    def step_device():
        for mode in (0, 2):
            st = L.nca_apply(ws._h, mode, prec, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, b,
                             1.0, 0.0, 0.0, 0.0, 1)
            if st:
                N._lib.check(st)

    launches = C.c_int32()
    ws.set_profiling(True)
    clocks = Clocks(local)
    clocks.start()
    t_end = time.perf_counter() + 1.0
    w = 0
    while w < max(args.warmup, 3) or time.perf_counter() < t_end:
        step_device()
        w += 1
    stage_sum = {k: 0.0 for k in ("gather", "upward", "coupling", "downward", "near", "leaves")}
    stage_n = {k: 0 for k in stage_sum}
    total_launches = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        for mode in (0, 2):
            st = L.nca_apply(ws._h, mode, prec, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, b,
                             1.0, 0.0, 0.0, 0.0, 1)
            if st:
                N._lib.check(st)
            L.nca_workspace_last_launches(ws._h, C.byref(launches))
            total_launches += launches.value
            for k, (t, cnt) in ws.stage_times().items():
                stage_sum[k] += t
                stage_n[k] += cnt
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    elapsed = max_over_ranks(e0.elapsed_time(e1) * 1e-3, f"cuda:{local}")
    step_bytes = 2 * product_bytes(info, b, 8 if f32 else E)
    value = world * step_bytes * args.steps / elapsed / 1e9
    # end to end: the same products through the C ABI with pinned host buffers
    Xh = torch.from_numpy(np.ascontiguousarray(X.T)).pin_memory()
    Yh = torch.zeros((b, n), dtype=torch.complex128).pin_memory()
    for _ in range(2):
        for mode in (0, 2):
            N._lib.check(L.nca_apply(ws._h, mode, prec, C.c_void_p(Xh.data_ptr()), n, C.c_void_p(Yh.data_ptr()), n,
                                     b, 1.0, 0.0, 0.0, 0.0, 0))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for mode in (0, 2):
            N._lib.check(L.nca_apply(ws._h, mode, prec, C.c_void_p(Xh.data_ptr()), n, C.c_void_p(Yh.data_ptr()), n,
                                     b, 1.0, 0.0, 0.0, 0.0, 0))
    e2e_el = max_over_ranks(time.perf_counter() - t0, f"cuda:{local}")
    e2e = {"value": world * step_bytes * args.steps / e2e_el / 1e9, "unit": "GB/s",
           "h2d_bytes_per_step": 2 * n * b * E, "d2h_bytes_per_step": 2 * n * b * E}
    err = dense_rows_error(N, pts, core, ws, X) if rank == 0 else None
    chosen = None
    if not f32:
        chosen = measure_chosen(N, L, core, ws, X, Xd, Yd, n, b, args, world, local, info, elapsed, pts, rank)
    # roofline of the dominant stage (CUDA events on the workspace stream, in the timed region)
    top = max(stage_sum, key=lambda k: stage_sum[k])
    peak, peak_kind = peaks()
    near_avg = stage_sum["near"] / max(stage_n["near"], 1)
    achieved = stage_bytes(info, b, 8 if f32 else E) / near_avg / 1e9 if near_avg > 0 else None
    roofline = {"kernel": "k_rows_leaves, near-field launch (runs beside the far-field sweeps)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": traffic_from_profiles(),
                "launch_ms": 1e3 * near_avg, "share_of_step": stage_sum["near"] / max(elapsed, 1e-30),
                "top_stage": top}
    if args.profile_stages and rank == 0:
        print(json.dumps({k: (1e3 * stage_sum[k] / args.steps, stage_n[k]) for k in stage_sum}), file=sys.stderr)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(2, b)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex-f32" if f32 else "complex-f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "npoints": n, "nrhs": b, "step": "H X and H^H X (16-column block)",
                       "l2": "inputs larger than L2 (stores 1.7 GB per product)",
                       "build_s": build_wall, "build_device_s": info["build_seconds"],
                       "build_host_s": info["build_seconds_host"], "stored_gb": E * store_entries(info) / 1e9,
                       "relerr_vs_dense_rows": err, "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": total_launches,
            "chosen": chosen,
            "clocks": clk,
        }), flush=True)
    del ws, core
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
