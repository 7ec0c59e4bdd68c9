#!/usr/bin/env python
"""Benchmark: the NCA build + H^2 products on one B200 (per rank).

Default workload (the headline): the wideband directional sphere. 262,144 points uniform on the
unit sphere (seeded), Helmholtz cis(kr)/(4 pi r) with k = 2 pi 8 (16 wavelengths across, zero on
the diagonal), isnearwideband(k; eta_lf 1, eta_hf 5, gamma 1), k-means tree minvalues 64,
BottomUp(IACA(MaximumValue(), TreeMimicryPivoting, FNormExtrapolator(1e-4))) per (cluster,
direction), maxrank 50; the work is the build plus 100 matvecs with seeded complex Gaussian x.
One timed step = the 100 vectors as one block product in the batched mixed-precision form
(complex-FP32 stores and arena, FP64 accumulation); `value` = its algorithmic HBM bytes per
second (the stores once per 16-column pass, the vectors, the coefficient vectors). Beside it:
build + 100 matvecs for the plain FP64 form (its own FP64-only build, 100 single-vector FP64
products) and for the batched mixed form, and their ratio.

Other workloads (--workload): galerkin-sphere (65,536 points, k = 1, tol 1e-5, H X and H^H X on
16 right-hand sides), batched-uneven (64 problems in one batched product), gradients (dJ/dx and
dJ/dk on a perturbed sphere).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload ...]

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
WIDEBAND = "wideband-sphere-{n}-k16pi-tol1e-4-iaca-100vec"
E = 16  # bytes per complex FP64 entry


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="f64", choices=["f64", "f32"])
    p.add_argument("--npoints", type=int, default=0, help="point count (default: the workload's)")
    p.add_argument("--nrhs", type=int, default=16)
    p.add_argument("--wideband-points", type=int, default=0, help="point count of the wideband workload")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--builds", type=int, default=7,
                   help="timed builds of each wideband form; the median is reported")
    p.add_argument("--profile-stages", action="store_true", help="print per-stage times to stderr")
    p.add_argument("--profile-run", action="store_true",
                   help="wideband workload for profiler captures: one mixed-precision build and `steps` block "
                        "products, no plain arm, no CPU baseline; prints build and stage times")
    p.add_argument("--clocks-csv", default=None, help="file for the nvidia-smi clock samples (default: a temp file)")
    p.add_argument("--workload", default="wideband",
                   choices=["wideband", "galerkin-sphere", "batched-uneven", "gradients"],
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

    path_override = None

    def __init__(self, index):
        import tempfile
        self.proc, self.index = None, index
        self.path = Clocks.path_override or os.path.join(tempfile.gettempdir(), f"nca_bench_clocks_{index}.csv")

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


def dense_rows_error(N, pts, core, ws, X, nrows=64, k=1.0, rmin=0.0):
    """Relative error of H X (two columns) against rows of the dense FP64 matrix from the CPU
    oracle (long-double accumulation)."""
    from oracle import oracle as O
    rng = np.random.default_rng(7)
    rows = rng.choice(len(pts), nrows, replace=False)
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=rmin)
    Y = N.mul(None, ws, X[:, :2])
    ref = np.stack([O.dense_rows(kern, pts, pts, rows, X[:, q]) for q in range(2)], axis=1)
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


def oracle_info(H):
    """Stored entries and coefficient counts of an oracle build, in the core-info layout."""
    tl = [not H.trees[0].isleaf(t) for t in range(H.trees[0].nnodes)]
    sl = [not H.trees[1].isleaf(t) for t in range(H.trees[1].nnodes)]
    return {"near_entries": sum(a.size for a in H.near), "coupling_entries": sum(a.size for a in H.couplings),
            "transfer_entries_test": sum(H.X[0][t].size for t in range(len(tl)) if tl[t]),
            "transfer_entries_trial": sum(H.X[1][t].size for t in range(len(sl)) if sl[t]),
            "basis_entries_test": sum(H.X[0][t].size for t in range(len(tl)) if not tl[t]),
            "basis_entries_trial": sum(H.X[1][t].size for t in range(len(sl)) if not sl[t]),
            "ntest": len(H.testpts), "ntrial": len(H.trialpts), "ncoeff_test": int(H.ranks[0].sum()),
            "ncoeff_trial": int(H.ranks[1].sum())}


def cpu_galerkin(n, b, steps, warmup):
    """The oracle (C restatement, OpenMP on all host cores) on the Galerkin sphere: its own build,
    then `steps` timed steps of one forward and one adjoint product on b right-hand sides. The
    rate is the algorithmic bytes of the products actually run over their time (no scaling)."""
    from oracle import oracle as O
    pts = sphere(n)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    H = O.H2(pts, pts, O.Kernel(O.KIND_HELMHOLTZ, k=1.0), minvalues=64, tol=1e-5, maxrank=50, nthreads=cores)
    tb = time.perf_counter() - t0
    X = rhs(len(pts), b)
    for _ in range(warmup):
        H.apply(X, 0)
        H.apply(X, 2)
    t0 = time.perf_counter()
    for _ in range(steps):
        H.apply(X, 0)
        H.apply(X, 2)
    el = time.perf_counter() - t0
    value = steps * 2 * product_bytes(oracle_info(H), b) / el / 1e9
    return {"value": value, "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"CPU oracle (C restatement, OpenMP, {cores} threads): full build ({tb:.1f} s), then {steps} "
                      f"steps of one forward and one adjoint product on {b} right-hand sides (of the 16 the GPU "
                      f"step takes); GB/s of the products run", "build_s": tb, "step_s": el / max(steps, 1)}


def run_reference(args):
    """The reference arm: the reference's algorithm on the host cores (the C restatement; the
    Julia package cannot run on this box), on the workload of the GPU arm. Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "wideband":
        n = args.npoints or 262144
        steps = max(1, min(args.steps, 10))
        cpu = cpu_wideband(n, steps, min(args.warmup, 1))
        config = {"workload": WIDEBAND.format(n=n), "npoints": n, "build_s": cpu["build_s"],
                  "step": "one single-vector FP64 matvec", "l2": "inputs larger than L2",
                  "relerr_vs_dense_rows": cpu["relerr_vs_dense_rows"],
                  "build_plus_100_matvecs_s": cpu["build_s"] + 100 * cpu["step_s"]}
        ms = 1e3 * cpu["step_s"]
        steps_run = steps
    elif args.workload == "galerkin-sphere":
        n = args.npoints or 65536
        steps_run = max(1, min(args.steps, 10))
        cpu = cpu_galerkin(n, 2, steps_run, min(args.warmup, 1))
        config = {"workload": WORKLOAD, "npoints": n, "nrhs": 2, "build_s": cpu["build_s"],
                  "l2": "inputs larger than L2"}
        ms = 1e3 * cpu["step_s"]
    else:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU arm for the {args.workload} workload"}),
              flush=True)
        return
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "GB/s", "n_gpus": args.gpus,
        "steps": steps_run, "warmup": min(args.warmup, 1), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex-f64", "data": "synthetic", "config": config,
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cpu["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def wideband_points(n):
    return sphere(n, 888)


def cpu_wideband(n, steps, warmup):
    """The C restatement of the directional path (OpenMP on all host cores) on the wideband
    sphere: its full build, then `steps` timed single-vector FP64 matvecs, each a whole product;
    the rate is their algorithmic bytes over their time (no scaling). The error of the first
    matvec against 64 dense FP64 rows rides along."""
    from oracle import directional as OD
    from oracle import oracle as O
    k = 2 * np.pi * 8
    pts = wideband_points(n)
    cores = os.cpu_count() or 1
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12)
    t0 = time.perf_counter()
    H = OD.DirectionalH2(pts, pts, kern, k, minvalues=64, tol=1e-4, maxrank=50, nthreads=cores)
    tb = time.perf_counter() - t0
    x = rhs(n, 1, seed=31)[:, 0]
    for _ in range(warmup):
        H.apply(x, 0)
    t0 = time.perf_counter()
    for _ in range(steps):
        y = H.apply(x, 0)
    el = time.perf_counter() - t0
    rows = np.random.default_rng(7).choice(n, 64, replace=False)
    ref = O.dense_rows(kern, pts, pts, rows, x, nthreads=cores)
    err = float(np.linalg.norm(y[rows] - ref) / np.linalg.norm(ref))
    e = H.entries
    ncoeff = sum(int(r.sum()) for r in H.ranks)
    step_bytes = E * (e["x"] + e["coupling"] + e["near"]) + E * 3 * n + 2 * E * ncoeff
    return {"value": steps * step_bytes / el / 1e9, "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"CPU oracle (C restatement of the directional build and product, OpenMP, {cores} threads): "
                      f"full build ({tb:.1f} s), then {steps} single-vector FP64 matvecs; GB/s of the matvecs run",
            "build_s": tb, "step_s": el / steps, "relerr_vs_dense_rows": err}


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
    """131,072 points on a perturbed sphere, Helmholtz k = 20, tol 1e-5, isnearwideband(20) (kd is
    about 44 at the root, so the upper levels are high frequency) with BottomUp(IACA) per (cluster,
    direction), maxrank 50, skeleton frozen after the build; J = ||H(k) x - b||^2 with 4 right-hand sides.
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
    t0 = time.perf_counter()
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
    conv = N.FNormExtrapolator(1e-5)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, tree), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, tree), N.MaximumValue(), conv))
    core = N.PetrovGalerkinNCACore(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, N.BlockTree(tree, tree),
                                   isnear=N.isnearwideband(k), testcompressor=tc, trialcompressor=sc, device=local)
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
                       "k": k, "admissibility": "isnearwideband(k; eta_lf=1, eta_hf=5, gamma=1), maxrank 50",
                       "compressor": "BottomUp(IACA(MaximumValue, TreeMimicryPivoting, FNormExtrapolator(1e-5)))",
                       "step": "one gradient: H x, H^H (2 (Hx - b)), dH/dk x",
                       "l2": "inputs larger than L2", "build_s": build_wall, "prepare_dk_s": prep,
                       "stored_gb": E * store_entries(info) / 1e9, "relerr_vs_dense_rows": err},
            "gradients_per_s": 1.0 / el, "k_bar": kbar, "k_bar_central_difference": fd,
            "k_bar_relerr_vs_fd": abs(kbar - fd) / abs(fd),
            "roofline": {"bound": "hbm", "achieved": step_bytes / el / 1e9, "peak": peak, "peak_source": peak_kind,
                         "unit": "GB/s", "frac": step_bytes / el / 1e9 / peak, "traffic": None,
                         "note": "whole gradient step (three products), algorithmic bytes"},
            "clocks": clk}), flush=True)


def wideband_core(N, pts, k, local, mixed):
    """The wideband workload's core: k-means tree + BottomUp(IACA) build (timed together). The
    batched mixed form keeps complex-FP32 copies of the stores for its products."""
    import torch
    t0 = time.perf_counter()
    tree = N.KMeansTree(pts, N.KMeansTreeBuilder(minvalues=64))
    conv = N.FNormExtrapolator(1e-4)
    tc = N.BottomUp(factorization=N.IACA(N.MaximumValue(), N.TreeMimicryPivoting(pts, pts, tree), conv))
    sc = N.BottomUp(factorization=N.IACA(N.TreeMimicryPivoting(pts, pts, tree), N.MaximumValue(), conv))
    core = N.PetrovGalerkinNCACore(N.HelmholtzKernel(k, rmin=1e-12), pts, pts, N.BlockTree(tree, tree),
                                   isnear=N.isnearwideband(k), testcompressor=tc, trialcompressor=sc,
                                   store_f32=mixed, device=local)
    torch.cuda.synchronize()
    return core, time.perf_counter() - t0


def dir_stage_bytes(info, b, e):
    """Algorithmic bytes per 16-column pass of the directional product's stages: each stage's
    stored entries once (X of every item in the up stage and again in the down/leaf stages,
    couplings, near blocks) plus the vector rows it reads and writes once."""
    xe = info["basis_entries_test"] + info["basis_entries_trial"] + info["transfer_entries_test"] + \
        info["transfer_entries_trial"]
    return e * xe + e * info["coupling_entries"] + e * info["near_entries"]


def timed_builds(N, pts, k, local, mixed, reps):
    """`reps` builds of the same wideband core, each freed before the next: the last core, the
    median build time and every build time."""
    import gc
    import torch
    times, core = [], None
    for _ in range(max(reps, 1)):
        if core is not None:
            del core
            gc.collect()
            torch.cuda.synchronize()
        core, t = wideband_core(N, pts, k, local, mixed)
        times.append(t)
    return core, float(np.median(times)), times


def profile_wideband(args, N, L, pts, k, local, n, nvec, Xd, Yd):
    """--profile-run: the batched mixed form's build and `steps` block products of 100 columns
    (after `warmup` untimed ones), with the library's stage events; one JSON line. The command
    that the committed profiler summaries run."""
    import torch
    core, build = wideband_core(N, pts, k, local, True)
    W = N.H2Workspace(core, np.complex64, max_nrhs=16)
    W.set_profiling(True)
    names = ["gather", "up", "coupling", "down", "near", "leaves"]
    total = [0.0] * 6
    for i in range(args.warmup + args.steps):
        N._lib.check(L.nca_apply(W._h, 0, 1, C.c_void_p(Xd.data_ptr()), n, C.c_void_p(Yd.data_ptr()), n, nvec,
                                 1.0, 0.0, 0.0, 0.0, 1))
        torch.cuda.synchronize()
        sec = (C.c_double * 6)()
        cnt = (C.c_int32 * 6)()
        L.nca_workspace_stage_times(W._h, sec, cnt, 6)
        if i >= args.warmup:
            for q in range(6):
                total[q] += sec[q]
    steps = max(args.steps, 1)
    print(json.dumps({"profile_run": WIDEBAND.format(n=n), "build_s": build,
                      "stage_ms_per_step": {names[q]: 1e3 * total[q] / steps for q in range(6)}}), flush=True)


def run_wideband(args):
    """The headline workload (see the module docstring)."""
    import torch
    import nca_b200 as N
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    n, k, nvec = args.npoints or 262144, 2 * np.pi * 8, 100
    pts = wideband_points(n)
    cuda_ready(N, local)
    L = N.lib()
    dev = f"cuda:{local}"
    X = rhs(n, nvec, seed=31)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)  # column-major n x 100
    Yd = torch.zeros_like(Xd)
    if args.profile_run:
        return profile_wideband(args, N, L, pts, k, local, n, nvec, Xd, Yd)
    # an untimed build first: the process's one-time costs (device memory pools, host pages, the
    # planning threads' first start) fall on neither timed build
    warm, _ = wideband_core(N, pts, k, local, False)
    del warm
    import gc
    gc.collect()
    torch.cuda.synchronize()
    # plain FP64 form: FP64-only build, then 100 single-vector FP64 matvecs
    core, build_plain, plain_times = timed_builds(N, pts, k, local, False, args.builds)
    W64 = N.H2Workspace(core, max_nrhs=1)

    def seq():
        for j in range(nvec):
            N._lib.check(L.nca_apply(W64._h, 0, 0, C.c_void_p(Xd[j].data_ptr()), n, C.c_void_p(Yd[j].data_ptr()),
                                     n, 1, 1.0, 0.0, 0.0, 0.0, 1))
    seq()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    seq()
    e1.record()
    torch.cuda.synchronize()
    t_seq64 = e0.elapsed_time(e1) * 1e-3
    info64 = info_dict(core)
    Y64 = Yd[0].cpu().numpy()
    del W64, core
    import gc
    gc.collect()
    torch.cuda.synchronize()
    # batched mixed form: the build with complex-FP32 stores, the 100 vectors as one block
    core, build_mixed, mixed_times = timed_builds(N, pts, k, local, True, args.builds)
    info = info_dict(core)
    W = N.H2Workspace(core, np.complex64, max_nrhs=16)
    W.set_profiling(True)

    def block(xp, yp, memspace):
        N._lib.check(L.nca_apply(W._h, 0, 1, C.c_void_p(xp), n, C.c_void_p(yp), n, nvec, 1.0, 0.0, 0.0, 0.0,
                                 memspace))
    for _ in range(max(args.warmup, 3)):
        block(Xd.data_ptr(), Yd.data_ptr(), 1)
    stage_sum = [0.0] * 6
    stage_n = [0] * 6
    launches = C.c_int32()
    total_launches = 0
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        block(Xd.data_ptr(), Yd.data_ptr(), 1)
        L.nca_workspace_last_launches(W._h, C.byref(launches))
        total_launches += launches.value
        sec = (C.c_double * 6)()
        cnt = (C.c_int32 * 6)()
        L.nca_workspace_stage_times(W._h, sec, cnt, 6)
        for q in range(6):
            stage_sum[q] += sec[q]
            stage_n[q] += cnt[q]
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_blk32 = max_over_ranks(e0.elapsed_time(e1) * 1e-3, dev) / args.steps
    Ymix = Yd[0].cpu().numpy()
    # end to end: the same block product from and to pinned host buffers through the C ABI
    W.set_profiling(False)
    Xh = torch.from_numpy(np.ascontiguousarray(X.T)).pin_memory()
    Yh = torch.zeros_like(Xh).pin_memory()
    block(Xh.data_ptr(), Yh.data_ptr(), 0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        block(Xh.data_ptr(), Yh.data_ptr(), 0)
    t_e2e = max_over_ranks(time.perf_counter() - t0, dev) / args.steps
    # errors against 64 dense FP64 rows of the CPU oracle (first vector), FP32 form vs FP64 form
    from oracle import oracle as O
    kern = O.Kernel(O.KIND_HELMHOLTZ, k=k, rmin=1e-12)
    rows = np.random.default_rng(7).choice(n, 64, replace=False)
    ref = O.dense_rows(kern, pts, pts, rows, X[:, 0])
    err64 = float(np.linalg.norm(Y64[rows] - ref) / np.linalg.norm(ref))
    errmix = float(np.linalg.norm(Ymix[rows] - ref) / np.linalg.norm(ref))
    rel_mix_64 = float(np.linalg.norm(Ymix - Y64) / np.linalg.norm(Y64))
    bytes32 = product_bytes(info, nvec, 8)
    value = world * bytes32 / t_blk32 / 1e9
    # roofline of the dominant stage of the block product (events on the product stream): its
    # stored entries once and the vector rows it reads or writes once, all 100 columns
    names = ["gather", "up", "coupling", "down", "near", "leaves"]
    kernels = {"gather": "k_gather_to_f32", "up": "k_gather_wide", "coupling": "k_gather_wide",
               "down": "k_gather_wide", "leaves": "k_gather_tc (tcgen05 kind::tf32, 3xTF32; leaf outputs: bases and near blocks)"}
    top = max(range(6), key=lambda q: stage_sum[q])
    xe = info["basis_entries_test"] + info["basis_entries_trial"] + info["transfer_entries_test"] + \
        info["transfer_entries_trial"]
    leaf_x = info["basis_entries_test"]
    stage_entries = {"gather": 0, "up": xe - info["transfer_entries_test"] - info["basis_entries_test"],
                     "coupling": info["coupling_entries"], "down": info["transfer_entries_test"],
                     "near": 0, "leaves": leaf_x + info["near_entries"]}
    # vector rows each stage reads or writes once: x, coefficient rows of the input side (written
    # by the up stage, read by the coupling), of the output side (written by the coupling, read and
    # accumulated by the down stage, read by the leaves), y
    vec_rows = {"gather": 2 * n, "up": n + 2 * info["ncoeff_trial"],
                "coupling": info["ncoeff_trial"] + info["ncoeff_test"], "down": 3 * info["ncoeff_test"],
                "near": 0, "leaves": info["ncoeff_test"] + 2 * n}
    nm = names[top]
    step_bytes = 8 * stage_entries[nm] + 8 * nvec * vec_rows[nm]
    stage_time = stage_sum[top] / args.steps
    achieved = step_bytes / stage_time / 1e9 if stage_time > 0 else None
    # the same stage against the FP32 FMA pipe: a complex multiply-add is 8 real flops per stored
    # entry and right-hand side; peak = SMs x 128 FP32 lanes x 2 flops x the SM clock
    import torch
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = sms * 128 * 2 * 1.965e9 / 1e12
    fma_achieved = 8.0 * stage_entries[nm] * nvec / stage_time / 1e12 if stage_time > 0 else None
    whole_flops = 8.0 * store_entries(info) * nvec / t_blk32 / 1e12
    peak, peak_kind = peaks()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_wideband(n, 2, 0)
    plain = build_plain + t_seq64
    mixed = build_mixed + t_blk32
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_blk32, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex-f32 stores and arena, f64 accumulation",
            "data": "synthetic",
            "config": {"workload": WIDEBAND.format(n=n), "npoints": n, "k": k, "nvec": nvec,
                       "admissibility": "isnearwideband(k; eta_lf=1, eta_hf=5, gamma=1)",
                       "compressor": "BottomUp(IACA(MaximumValue, TreeMimicryPivoting, FNormExtrapolator(1e-4)))",
                       "step": "100 matvecs as one block of 100 right-hand sides (all 100 columns per launch: "
                               "small outputs on the FP32 pipe, leaf outputs on the tcgen05 tensor cores)",
                       "l2": "inputs larger than L2 (FP32 stores %.1f GB per step)" % (8 * store_entries(info) / 1e9),
                       "build_s": build_mixed, "build_s_plain_f64": build_plain,
                       "build_s_samples": {"batched_mixed": mixed_times, "plain_f64": plain_times,
                                           "reported": "median"},
                       "build_device_s": info["build_seconds"], "stored_gb_f64": E * store_entries(info) / 1e9,
                       "relerr_vs_dense_rows": {"plain_f64": err64, "batched_mixed": errmix, "bar_north_star": 1e-4,
                                                "bar_reference_tests_10tol": 1e-3},
                       "relerr_mixed_vs_plain_f64": rel_mix_64, "parallelism": f"replicas x{world}"},
            "build_plus_100_matvecs_s": {"plain_f64": plain, "batched_mixed": mixed, "speedup": plain / mixed,
                                         "plain_100_single_f64_matvecs_s": t_seq64,
                                         "mixed_block_of_100_s": t_blk32},
            "roofline": {"kernel": kernels.get(nm, nm), "stage": nm, "bound": "hbm", "achieved": achieved,
                         "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": None,
                         "stage_ms_per_step": 1e3 * stage_time,
                         "stage_share": stage_sum[top] / (args.steps * t_blk32),
                         "bytes_per_step": step_bytes,
                         "fp32_fma": {"achieved_tflops": fma_achieved, "peak_tflops": fp32_peak,
                                      "peak_source": "nominal (SMs x 128 lanes x 2 x 1965 MHz)",
                                      "frac": fma_achieved / fp32_peak if fma_achieved else None,
                                      "whole_product_tflops": whole_flops},
                         "stages_ms_per_step": {names[q]: 1e3 * stage_sum[q] / args.steps for q in range(6)},
                         "launches_per_step": {names[q]: stage_n[q] / args.steps for q in range(6)}},
            "cpu_baseline": cpu,
            "e2e": {"value": world * bytes32 / t_e2e / 1e9, "unit": "GB/s", "h2d_bytes_per_step": 8 * 2 * n * nvec,
                    "d2h_bytes_per_step": 8 * 2 * n * nvec, "ms_per_step": 1e3 * t_e2e},
            "gpu_launches": total_launches, "clocks": clk}), flush=True)


def tangent_bytes(info, b, e=E):
    """Algorithmic bytes of one tangent product: every stored entry and its d/dk twice as many
    stores (X, dX, S, dS, N, dN), x read, y written, four coefficient vectors written and read."""
    vec = e * b * (info["ntrial"] + 2 * info["ntest"]) + 4 * e * b * (info["ncoeff_test"] + info["ncoeff_trial"])
    return 2 * e * store_entries(info) + vec


def dense_rows_error_k(N, pts, core, ws, X, k, nrows=64):
    return dense_rows_error(N, pts, core, ws, X, nrows, k=k, rmin=1e-12)


def main():
    args = parse()
    Clocks.path_override = args.clocks_csv
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
    args.npoints = args.npoints or 65536
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
        cpu = cpu_galerkin(n, 2, 2, 0)
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
