#!/usr/bin/env python
"""PageRank benchmark: GTEPS per iteration and HBM roofline on R-MAT scale 24.

Workload (one step): PageRank run to convergence on the directed R-MAT graph
scale 24 / edgefactor 16 / (a, b, c, d) = (0.57, 0.19, 0.19, 0.05), duplicates
and self-loops removed, unweighted; damp 0.85, tol 1e-10, L1 norm, FP64
(the reference's arithmetic), reference sink semantics. The graph is resident
in HBM before the timed region (value); the e2e figure repeats the same run
through the C ABI from pinned host arrays, with the upload and the score
read-back inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (under torchrun) runs the same PageRank run with its rows cut into N
slices, one per GPU (networkit_b200.distributed.RowPartitionedPageRank: per
iteration an all-gather of the iterate and an all-reduce of two sums over
NCCL), so the total work is fixed and scaling is strong; --multi replicas
runs N independent copies of the single-GPU run instead (weak scaling).
"""
from __future__ import annotations

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

SCALE = 24
EDGEFACTOR = 16
RMAT = (0.57, 0.19, 0.19)
SEED = 42
DAMP = 0.85
TOL = 1e-10
NORM_L1 = 0
METRIC = "PageRank GTEPS/iter (R-MAT scale 24, FP64)"
UNIT = "GTEPS/iter"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the companion forms (refine, ppr, adjoint, batch) of the default line")
    ap.add_argument("--profile-only", type=int, default=0, metavar="SWEEPS",
                    help="only upload the graph and run SWEEPS individually launched sweeps "
                         "(the small, fixed launch sequence used for ncu captures)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="precision of the --profile-only sweeps")
    ap.add_argument("--shape", type=int, default=-1,
                    help="sweep launch shape (nkg_graph_options.sweep_shape; -1 default)")
    ap.add_argument("--arc-order", type=int, default=0, choices=[0, 1],
                    help="nkg_graph_options.arc_order (0 keep the reference order, 1 sorted)")
    ap.add_argument("--hot-tier-kb", type=int, default=-1,
                    help="nkg_graph_options.hot_tier_kb: shared-memory tier of the sweep "
                         "(-1 library default, 0 none, 1..224 KB)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity check of the timed run against the reference's own "
                         "PageRank on the same graph")
    ap.add_argument("--form", default="",
                    choices=["", "ppr", "refine", "adjoint", "batch", "centrality", "local",
                             "reader", "locality", "er"],
                    help="run only one companion form and print its figures")
    ap.add_argument("--fd-edges", type=int, default=64,
                    help="arcs checked by finite differences in --form adjoint")
    ap.add_argument("--adjoint-step-only", action="store_true",
                    help="--form adjoint: only the reference solves and one timed breakdown")
    ap.add_argument("--adjoint-scale", type=int, default=22, help="R-MAT scale of --form adjoint")
    ap.add_argument("--batch-graphs", type=int, default=1024, help="graphs of --form batch")
    ap.add_argument("--batch-step-only", action="store_true",
                    help="--form batch: no tuning and no comparison, two runs with the default "
                         "launch shape (the short launch sequence used for ncu captures)")
    ap.add_argument("--ppr-n", type=int, default=4_000_000, help="graph nodes of --form ppr")
    ap.add_argument("--ppr-step-only", action="store_true",
                    help="--form ppr: one warm-up and one timed run only (the short launch "
                         "sequence used for ncu captures)")
    ap.add_argument("--local-n", type=int, default=1_000_000, help="graph nodes of --form local")
    ap.add_argument("--local-seeds", type=int, default=16384, help="seeds of --form local")
    ap.add_argument("--local-ref-sample", type=int, default=48,
                    help="seeds the reference runs in --form local (0: none)")
    ap.add_argument("--local-runs", type=int, default=2, help="timed calls of --form local")
    ap.add_argument("--multi", default="rows", choices=["rows", "replicas"],
                    help="N > 1: the row-partitioned run (rows, strong scaling) or N independent "
                         "replicas (weak scaling)")
    ap.add_argument("--cache", default=os.path.join(tempfile.gettempdir(), "nk_b200_graphs"))
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, device):
    """The largest of every rank's x: a MAX all-reduce on `device` (the
    rank's GPU under NCCL, the CPU under gloo). Every rank calls it."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_gteps(world, arcs, iterations, max_ms):
    """Whole-job GTEPS/iter of `world` replicas, each sweeping `arcs` arcs
    `iterations` times, timed by the slowest rank (weak scaling)."""
    return world * arcs * iterations / (max_ms / 1e3) / 1e9


def graph_path(cache, scale):
    return os.path.join(cache, f"rmat{scale}_ef{EDGEFACTOR}_s{SEED}.npz")


def make_graph(scale, cache, rank, barrier):
    """Generate once (rank 0), cache on local disk, load everywhere."""
    from networkit_b200 import generators
    from networkit_b200.graph import InCSR

    path = graph_path(cache, scale)
    if rank == 0 and not os.path.exists(path):
        csr = generators.rmat_directed(scale, EDGEFACTOR, *RMAT, seed=SEED)
        os.makedirs(cache, exist_ok=True)
        tmp = path + f".tmp{os.getpid()}.npz"
        np.savez(tmp, in_ptr=csr.in_ptr, in_col=csr.in_col, outdeg=csr.outdeg)
        os.replace(tmp, path)
    barrier()
    d = np.load(path)
    outdeg = d["outdeg"]
    z = outdeg.shape[0]
    return InCSR(z, z, d["in_ptr"], d["in_col"], None, outdeg.astype(np.float64), outdeg, None,
                 True)


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].strip().lower() == "active"})
        load = [s for s in sm if smax and s >= 0.3 * max(smax)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(kernel_tag):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/<kernel_tag>.txt, line 'traffic_bytes_per_launch: X')."""
    p = os.path.join(ROOT, "profiles", kernel_tag + ".txt")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def host_cpu():
    """Model, logical CPUs and physical cores of this host (from /proc/cpuinfo)."""
    model, phys = None, set()
    cur = {}
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if ":" not in line:
                    if "core id" in cur:
                        phys.add((cur.get("physical id"), cur["core id"]))
                    cur = {}
                    continue
                k, v = (x.strip() for x in line.split(":", 1))
                cur[k] = v
                if k == "model name" and model is None:
                    model = v
        if "core id" in cur:
            phys.add((cur.get("physical id"), cur["core id"]))
    except OSError:
        pass
    return {"model": model, "logical": os.cpu_count() or 1, "physical": len(phys) or None}


def cpu_baseline_port(csr, nthreads, target_s=4.0, runs=3):
    """The oracle's C restatement on the host cores over a bounded number of
    iterations of the same workload: the median of `runs` timed runs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    t0 = time.perf_counter()
    oracle.pagerank(csr, damp=DAMP, tol=TOL, norm=NORM_L1, max_iterations=1, nthreads=nthreads)
    t1 = time.perf_counter() - t0
    iters = int(max(2, min(20, target_s / max(t1, 1e-3))))
    rates, secs = [], []
    for _ in range(runs):
        t0 = time.perf_counter()
        r = oracle.pagerank(csr, damp=DAMP, tol=TOL, norm=NORM_L1, max_iterations=iters,
                            nthreads=nthreads)
        dt = time.perf_counter() - t0
        rates.append(csr.arcs * r.iterations / dt / 1e9)
        secs.append(dt)
    cpu = host_cpu()
    return {"value": statistics.median(rates), "unit": UNIT, "cores": nthreads,
            "kind": "port", "cpu_model": cpu["model"], "physical_cores": cpu["physical"],
            "sample": f"median of {runs} runs of {iters} iterations of the same R-MAT "
                      f"scale-{int(np.log2(csr.z))} FP64 run (oracle C restatement, OpenMP rows; "
                      f"{min(secs):.1f}-{max(secs):.1f} s each)"}


def form_ppr(local, n=4_000_000, m=8, k=256, steps=2, oracle_columns=2, step_only=False):
    """Batched personalised PageRank: Barabasi-Albert n=4M, m=8 (undirected;
    the graph the reference's BarabasiAlbertGenerator draws after
    setSeed(42, False), `generators.barabasi_albert_stream`), 256 one-hot seeds (uniform, seed 42), one FP32 SpMM with k = 256 columns,
    FP64 residual per column, damp 0.85, tol 1e-7 (L1). Errors: every 32nd
    column against the GPU's FP64 personalised run to tol 1e-12, and
    `oracle_columns` columns against the oracle (the CPU restatement of
    PageRank.cpp with the personalised teleport, tol 1e-10, all host
    cores)."""
    import torch

    from networkit_b200 import _capi, generators

    csr = generators.barabasi_albert_stream(m, n, seed=42)
    seeds = np.random.default_rng(42).choice(csr.z, k, replace=False).astype(np.uint32)
    dg = _capi.DeviceGraph(csr, device=local)
    p = dg.params(0.85, 1e-7, NORM_L1, False, False, _capi.NKG_PREC_FP32, 1000)
    out = torch.empty((k, csr.z), dtype=torch.float32, device=f"cuda:{local}")
    dg.ppr(seeds, p, out.data_ptr())  # warm-up
    if step_only:
        _, its, st = dg.ppr(seeds, p, out.data_ptr())
        dg.close()
        return {"workload": f"ppr_ba{n}_m{m}_k{k}_fp32", "n": csr.z, "arcs": csr.arcs, "k": k,
                "ms_per_run": st["ms_total"], "sweeps": st["fp32_sweeps"],
                "column_sweeps": int(its.sum()), "ms_per_sweep": st["ms_total"] / st["fp32_sweeps"],
                "alg_bytes_per_sweep": st["bytes_per_sweep_fp32"]}
    ms, sweeps, launches = 0.0, 0, 0
    for _ in range(steps):
        _, its, st = dg.ppr(seeds, p, out.data_ptr())
        ms += st["ms_total"]
        sweeps += st["fp32_sweeps"]
        launches += st["kernel_launches"]
        col_sweeps = int(its.sum())
    bytes_sweep = st["bytes_per_sweep_fp32"]
    per_sweep_ms = ms / sweeps
    # Against the plain FP64 path: one personalised FP64 run per seed
    # (nkg_pagerank_run_device with a one-hot teleport), timed on a sample of
    # seeds and scaled to k; the L1 error of those columns against it.
    sample = list(range(0, k, k // 8))
    scores = out.cpu().numpy()
    p64 = dg.params(0.85, 1e-7, NORM_L1, False, False, _capi.NKG_PREC_FP64, 1000)
    ref = dg.params(0.85, 1e-12, NORM_L1, False, False, _capi.NKG_PREC_FP64, 1000)
    d_t = torch.zeros(csr.z, dtype=torch.float64, device=f"cuda:{local}")
    d_o = torch.empty(csr.z, dtype=torch.float64, device=f"cuda:{local}")
    plain_ms, errs = 0.0, []
    for j in sample:
        d_t.zero_()
        d_t[int(seeds[j])] = 1.0
        torch.cuda.synchronize()
        dg.run_ex(p64, d_t.data_ptr(), d_o.data_ptr(), True)  # warm-up (graph capture)
        _, _, st64 = dg.run_ex(p64, d_t.data_ptr(), d_o.data_ptr(), True)
        plain_ms += st64["ms_total"]
        dg.run_ex(ref, d_t.data_ptr(), d_o.data_ptr(), True)
        errs.append(float(np.abs(scores[j].astype(np.float64) - d_o.cpu().numpy()).sum()))
    plain_ms *= k / len(sample)
    dg.close()
    o_rows = []
    if oracle_columns:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        for j in sample[:oracle_columns]:
            t = np.zeros(csr.z)
            t[int(seeds[j])] = 1.0
            o = oracle.pagerank(csr, damp=0.85, tol=1e-10, norm=NORM_L1, teleport=t,
                                nthreads=cores)
            d = np.abs(scores[j].astype(np.float64) - o.scores)
            big = o.scores >= 1.0 / csr.z
            o_rows.append({"column": j, "seed": int(seeds[j]), "l1_err": float(d.sum()),
                           "max_abs_err": float(d.max()),
                           "max_rel_err_at_or_above_1_over_n": float(
                               (d[big] / o.scores[big]).max()),
                           "oracle_iterations": o.iterations})
        o_secs = time.perf_counter() - t0
    return {"workload": f"ppr_ba{n}_m{m}_k{k}_fp32", "n": csr.z, "arcs": csr.arcs, "k": k,
            "plain_fp64_per_seed_ms": plain_ms, "plain_seeds_timed": len(sample),
            "speedup_vs_plain_fp64": plain_ms / (ms / steps),
            "l1_err_max_vs_fp64": max(errs),
            "vs_oracle": ({"kind": "port", "tol": 1e-10, "seconds": o_secs, "columns": o_rows,
                           "l1_err_max": max(r["l1_err"] for r in o_rows)} if o_rows else None),
            "sweeps": sweeps // steps, "column_sweeps": col_sweeps, "ms_per_run": ms / steps,
            "ms_per_sweep": per_sweep_ms,
            "gteps_per_iter": csr.arcs * k / (per_sweep_ms / 1e3) / 1e9,
            "alg_bytes_per_sweep": bytes_sweep,
            "alg_gbs": bytes_sweep / (per_sweep_ms / 1e3) / 1e9, "gpu_launches": launches,
            "roofline": ppr_roofline(csr, k, per_sweep_ms)}


def err_vs(s, ref):
    d = np.abs(np.asarray(s, np.float64) - ref)
    return float(d.sum()), float((d / np.maximum(np.abs(ref), 1e-300)).max())


def ppr_roofline(csr, k, ms_per_sweep):
    """Roofline of the PPR SpMM on its real traffic. The iterate (n x k FP32)
    is far larger than L2, so every arc gathers its source's k-column row:
    per sweep 4 arcs (columns) + 4 k arcs (gathered rows) + 8 n k (own row
    read, new row written) bytes. `traffic` is the ncu DRAM figure of the
    committed BA 1M capture (profiles/ppr_sweep_ba1m_k256.txt) scaled by the
    arc count (the traffic grows with the arcs: about 1 KB per arc there)."""
    peak, kind = measured_peak_hbm()
    model = 4 * csr.arcs + 4 * k * csr.arcs + 8 * csr.z * k
    achieved = model / (ms_per_sweep / 1e3) / 1e9
    t1m = profiled_traffic("ppr_sweep_ba1m_k256")
    traffic = t1m * csr.arcs / 15_999_888 if t1m else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "model_bytes_per_sweep": model,
            "peak_source": kind}


def form_refine(local, csr, steps=2, checker=None, checker_kind=None):
    """Plain FP64 vs FP32+FP64-refinement on the R-MAT scale-24 graph: time to
    the FP64 stopping test at tol 1e-10 (L1), and at tol 1.5e-7, the point
    where both reach ~1e-6 L1 error. Errors: against the FP64 oracle's scores
    of the headline parity check (`checker`: the reference's own PageRank, or
    the oracle's restatement, at tol 1e-10 L1, whose own distance to the
    fixed point is at most about 6e-10), and against an FP64 solve to tol
    1e-14 on the same GPU."""
    import torch

    from networkit_b200 import _capi

    dg = _capi.DeviceGraph(csr, device=local)
    n = csr.z
    d_ref = torch.empty(n, dtype=torch.float64, device=f"cuda:{local}")
    dg.run_device(dg.params(DAMP, 1e-14, NORM_L1, False, False, _capi.NKG_PREC_FP64, 2000),
                  d_ref.data_ptr())
    ref = d_ref.cpu().numpy()
    out = torch.empty(n, dtype=torch.float64, device=f"cuda:{local}")
    res = {}
    for tol in (1e-10, 1.5e-7):
        for name, prec in (("fp64", _capi.NKG_PREC_FP64), ("fp32_refine", _capi.NKG_PREC_FP32_REFINE)):
            p = dg.params(DAMP, tol, NORM_L1, False, False, prec, _capi.UINT64_MAX)
            dg.run_device(p, out.data_ptr())  # warm-up
            ms, st = 0.0, None
            for _ in range(steps):
                it, mx, st = dg.run_device(p, out.data_ptr())
                ms += st["ms_total"]
            s = out.cpu().numpy()
            diff = np.abs(s - ref)
            row = {
                "ms": ms / steps, "fp64_sweeps": st["fp64_sweeps"], "fp32_sweeps": st["fp32_sweeps"],
                "l1_err": float(diff.sum()),
                "max_rel_err": float((diff / np.maximum(np.abs(ref), 1e-300)).max()),
                "gpu_launches": st["kernel_launches"]}
            if checker is not None:
                row["l1_err_vs_oracle"], row["max_rel_err_vs_oracle"] = err_vs(s, checker)
            res[f"{name}_tol{tol:g}"] = row
    dg.close()
    for tol in ("1e-10", "1.5e-07"):
        res[f"speedup_tol{tol}"] = res[f"fp64_tol{tol}"]["ms"] / res[f"fp32_refine_tol{tol}"]["ms"]
    res["oracle"] = ({"kind": checker_kind, "tol": TOL, "norm": "L1"} if checker is not None
                     else None)
    return res


def form_adjoint(local, scale=22, steps=3, fd_edges=64, only_step=False, oracle_check=True):
    """Differentiable weighted PageRank: directed R-MAT scale 22, edgefactor
    16, weights uniform in (0.1, 1] (seed 43), loss L = sum_v g_v p_v with
    g ~ N(0, 1) (seed 42), damp 0.85, reference sink semantics. One step is
    forward + backward through networkit_b200.autograd (weights copied in,
    scores out, dL/dw and dL/dt out, all on the device), timed with CUDA
    events around the whole call; against it the plain FP64 forward alone.
    Errors are against the GPU FP64 forward to tol 1e-14 and FP64 adjoint to
    1e-13 (both parity-tested against the oracle); the FP64 gradient is also
    checked by central differences (h = 1e-4) of the FP64 forward on
    `fd_edges` random arcs. only_step: the reference solves and the
    time breakdown only (a short launch sequence for profiling).
    oracle_check: the forward scores and dL/dw of each timed form also
    against the oracle's FP64 forward and host adjoint solve (tol 1e-13, all
    host cores; the oracle's restatement of PageRank.cpp and its adjoint)."""
    import torch

    from networkit_b200 import _capi, autograd, generators

    dev = torch.device("cuda", local)
    csr = generators.with_uniform_weights(generators.rmat_directed(scale, EDGEFACTOR, *RMAT,
                                                                   seed=SEED), seed=43)
    g_np = np.random.default_rng(42).standard_normal(csr.z)
    G = autograd.DifferentiableGraph(csr, device=local)
    dg = G.graph
    w = torch.from_numpy(csr.in_w).to(dev)
    g = torch.from_numpy(g_np).to(dev)
    out = torch.empty(csr.z, dtype=torch.float64, device=dev)
    gw_ref = torch.empty(csr.arcs, dtype=torch.float64, device=dev)
    gt_ref = torch.empty(csr.z, dtype=torch.float64, device=dev)
    dg.set_weights_device(w.data_ptr())
    dg.run_ex(dg.params(DAMP, 1e-14, NORM_L1, False, False, _capi.NKG_PREC_FP64, 3000), 0,
              out.data_ptr(), True)
    p_ref = out.clone()
    torch.cuda.synchronize()
    dg.adjoint_device(dg.params(DAMP, 1e-13, NORM_L1, False, False, _capi.NKG_PREC_FP64, 5000),
                      p_ref.data_ptr(), g.data_ptr(), gw_ref.data_ptr(), gt_ref.data_ptr())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        fn()  # warm-up
        ms = []
        for _ in range(steps):
            torch.cuda.synchronize()
            ev[0].record()
            r = fn()
            ev[1].record()
            torch.cuda.synchronize()
            ms.append(ev[0].elapsed_time(ev[1]))
        return statistics.median(ms), r

    def plain(tol):
        p = dg.params(DAMP, tol, NORM_L1, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
        return lambda: (dg.run_ex(p, 0, out.data_ptr(), True), out.clone())[1]

    def fwd_bwd(prec, tol, btol):
        def f():
            wp = w.clone().requires_grad_(True)
            s = autograd.pagerank(G, wp, None, DAMP, tol, False, prec, prec, btol)
            (s * g).sum().backward()
            return s.detach(), wp.grad
        return f

    res = {"workload": f"adjoint_rmat{scale}_weighted", "n": csr.z, "arcs": csr.arcs}
    # Where a forward + backward step spends its time (library device timers).
    gw_b = torch.empty(csr.arcs, dtype=torch.float64, device=dev)
    bd = {}
    for _ in range(2):
        torch.cuda.synchronize()
        ev[0].record()
        dg.set_weights_device(w.data_ptr())
        ev[1].record()
        torch.cuda.synchronize()
        bd["set_weights_ms"] = ev[0].elapsed_time(ev[1])
        pr = dg.params(DAMP, 1e-10, NORM_L1, False, False, _capi.NKG_PREC_FP32_REFINE,
                       _capi.UINT64_MAX)
        _, _, st = dg.run_ex(pr, 0, out.data_ptr(), True)
        bd["fwd"] = {k: st[k] for k in ("ms_total", "fp32_sweeps", "fp64_sweeps",
                                          "kernel_launches")}
        _, st = dg.adjoint_device(pr, out.data_ptr(), g.data_ptr(), gw_b.data_ptr(), 0)
        bd["bwd"] = {k: st[k] for k in ("ms_total", "fp32_sweeps", "fp64_sweeps",
                                          "kernel_launches")}
    res["breakdown_fp32_refine_tol1e-10"] = bd
    if only_step:
        G.graph.close()
        return res
    gwn = float(gw_ref.abs().max())
    o_scores = o_gw = None
    if oracle_check:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        o = oracle.pagerank(csr, damp=DAMP, tol=1e-13, norm=NORM_L1, nthreads=cores)
        _, o_gw, _, o_sweeps = oracle.adjoint(csr, o.scores, g_np, damp=DAMP,
                                              distribute_sinks=False, tol=1e-13, nthreads=cores)
        o_scores = o.scores
        res["oracle"] = {"kind": "port", "cores": cores, "seconds": time.perf_counter() - t0,
                         "forward_iterations": o.iterations, "adjoint_sweeps": o_sweeps,
                         "tol": 1e-13}
        o_gwn = float(np.abs(o_gw).max())
    for tol, btol in ((1e-10, 1e-10), (1.5e-7, 1e-6)):
        ms_p, s_p = timed(plain(tol))
        row = {"plain_fp64_fwd_ms": ms_p, "plain_l1_err": float((s_p - p_ref).abs().sum())}
        for prec in ("fp32_refine", "fp64"):
            ms, (s, gw) = timed(fwd_bwd(prec, tol, btol))
            row[f"{prec}_fwd_bwd_ms"] = ms
            row[f"{prec}_l1_err"] = float((s - p_ref).abs().sum())
            row[f"{prec}_max_rel_err"] = float(((s - p_ref).abs() / p_ref.abs()).max())
            row[f"{prec}_grad_w_err"] = float((gw - gw_ref).abs().max()) / gwn
            if o_scores is not None:
                sh = s.cpu().numpy()
                row[f"{prec}_l1_err_vs_oracle"], row[f"{prec}_max_rel_err_vs_oracle"] = err_vs(
                    sh, o_scores)
                row[f"{prec}_grad_w_err_vs_oracle"] = float(
                    np.abs(gw.cpu().numpy() - o_gw).max()) / o_gwn
        if o_scores is not None:
            row["plain_l1_err_vs_oracle"], row["plain_max_rel_err_vs_oracle"] = err_vs(
                s_p.cpu().numpy(), o_scores)
        row["fwd_bwd_vs_plain_fwd"] = ms_p / row["fp32_refine_fwd_bwd_ms"]
        res[f"tol{tol:g}"] = row
    if fd_edges:
        fwd = dg.params(DAMP, 0.0, NORM_L1, False, False, _capi.NKG_PREC_FP64, 400)
        rng = np.random.default_rng(7)
        edges = rng.choice(csr.arcs, fd_edges, replace=False)
        h = 1e-4
        fds = []
        for e in edges:
            vals = []
            for sgn in (1.0, -1.0):
                w2 = w.clone()
                w2[int(e)] += sgn * h
                torch.cuda.synchronize()
                dg.set_weights_device(w2.data_ptr())
                dg.run_ex(fwd, 0, out.data_ptr(), True)
                vals.append(float((out * g).sum()))
            fds.append((vals[0] - vals[1]) / (2 * h))
        gsel = gw_ref[torch.from_numpy(edges).to(dev)].cpu().numpy()
        res["fd_check"] = {"edges": fd_edges, "h": h,
                           "max_abs_err_over_max_grad": float(np.abs(np.array(fds) - gsel).max()
                                                              / np.abs(gsel).max())}
        dg.set_weights_device(w.data_ptr())
    G.graph.close()
    return res


def form_batch(local, count=1024, steps=3, plain_graphs=None, step_only=False):
    """Many-graph batch: 1024 random hyperbolic graphs, n_i log-uniform in
    [1e3, 2e5] (numpy seed 42), average degree 16, exponent 3, graph i the
    one the reference's HyperbolicGenerator draws after setSeed(42 + i,
    False) (`generators.hyperbolic_stream_batch`); FP32, damp 0.85, tol 1e-8 (L1), one persistent launch in a
    CUDA graph with the autotuned launch shape. Against it: the plain FP64
    path run graph by graph (nkg_pagerank_run_device on every graph, the
    graphs already resident), and the FP64 batch for the error figures (the
    FP64 batch is parity-tested against the oracle)."""
    import torch

    from networkit_b200 import _capi, generators
    from networkit_b200.graph import InCSR

    rng = np.random.default_rng(42)
    ns = np.round(np.exp(rng.uniform(np.log(1e3), np.log(2e5), count))).astype(np.uint64)
    t0 = time.perf_counter()
    csr, offs = generators.hyperbolic_stream_batch(ns, 16.0, 3.0, seed=42)
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    db = _capi.DeviceBatch(csr, offs, device=local)
    t_create = time.perf_counter() - t0
    arcs_g = np.array([int(csr.in_ptr[int(offs[i + 1])] - csr.in_ptr[int(offs[i])])
                       for i in range(count)], np.float64)
    n_g = np.diff(offs).astype(np.float64)
    p32 = _capi.PRParams(DAMP, 1e-8, NORM_L1, 0, 0, _capi.NKG_PREC_FP32, 10000)
    p64 = _capi.PRParams(DAMP, 1e-8, NORM_L1, 0, 0, _capi.NKG_PREC_FP64, 10000)
    if step_only:
        dev = torch.device("cuda", local)
        out = torch.empty(db.total, dtype=torch.float64, device=dev)
        db.run(p32, out.data_ptr())
        _, its, floor, st = db.run(p32, out.data_ptr())
        tuning = db.tuning()
        db.close()
        return {"workload": f"batch_hyperbolic{count}_fp32", "graphs": count,
                "nodes": int(offs[-1]), "arcs": int(csr.arcs), "tuning": tuning,
                "fp32_ms": st["ms_total"], "fp32_sweeps_total": int(its.sum()),
                "fp32_floor_stops": floor}
    t0 = time.perf_counter()
    best, table = db.tune(p32, sweeps=8)
    t_tune = time.perf_counter() - t0
    dev = torch.device("cuda", local)
    out = torch.empty(db.total, dtype=torch.float64, device=dev)
    db.run(p32, out.data_ptr())  # warm-up
    ms, its, floor = [], None, 0
    for _ in range(steps):
        _, its, floor, st = db.run(p32, out.data_ptr())
        ms.append(st["ms_total"])
    ms32 = statistics.median(ms)
    g_start, g_end = db.graph_times()
    s32 = out.cpu().numpy()
    # e2e through the C ABI: host scores out, the graphs resident
    t0 = time.perf_counter()
    h32, _, _, _ = db.run(p32)
    e2e_ms = 1e3 * (time.perf_counter() - t0)
    _, its64, _, st64 = db.run(p64, out.data_ptr())
    ms64_batch = st64["ms_total"]
    ref = _capi.PRParams(DAMP, 1e-13, NORM_L1, 0, 0, _capi.NKG_PREC_FP64, 10000)
    db.run(ref, out.data_ptr())
    s_ref = out.cpu().numpy()
    errs = np.array([np.abs(s32[int(offs[i]):int(offs[i + 1])] -
                            s_ref[int(offs[i]):int(offs[i + 1])]).sum() for i in range(count)])
    # Every 32nd graph against the oracle (CPU restatement of PageRank.cpp,
    # FP64, tol 1e-13, all host cores).
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    o_errs, o_rel = [], []
    t0 = time.perf_counter()
    for i in range(0, count, 32):
        a, b = int(offs[i]), int(offs[i + 1])
        ptr = (csr.in_ptr[a:b + 1] - csr.in_ptr[a]).astype(np.uint64)
        col = (csr.in_col[int(csr.in_ptr[a]):int(csr.in_ptr[b])] - np.uint32(a)).astype(np.uint32)
        gi = InCSR(b - a, b - a, ptr, col, None, csr.wdeg[a:b], csr.outdeg[a:b], None, False)
        o = oracle.pagerank(gi, damp=DAMP, tol=1e-13, norm=NORM_L1, nthreads=os.cpu_count() or 1)
        l1, rel = err_vs(s32[a:b], o.scores)
        o_errs.append(l1)
        o_rel.append(rel)
    o_secs = time.perf_counter() - t0
    sweeps = its.astype(np.float64)
    arc_it = float((arcs_g * sweeps).sum())
    alg_bytes = float(((4 * arcs_g + 20 * n_g + 4) * sweeps).sum())
    db.close()
    # Plain FP64 path, graph by graph (each graph uploaded beforehand).
    idx = list(range(count)) if plain_graphs is None else list(plain_graphs)
    plain_ms = 0.0
    pin = _capi.PRParams(DAMP, 1e-8, NORM_L1, 0, 0, _capi.NKG_PREC_FP64, 10000)
    for i in idx:
        a, b = int(offs[i]), int(offs[i + 1])
        ptr = (csr.in_ptr[a:b + 1] - csr.in_ptr[a]).astype(np.uint64)
        col = (csr.in_col[int(csr.in_ptr[a]):int(csr.in_ptr[b])] - np.uint32(a)).astype(np.uint32)
        g = InCSR(b - a, b - a, ptr, col, None, csr.wdeg[a:b], csr.outdeg[a:b], None, False)
        dg = _capi.DeviceGraph(g, device=local)
        o = torch.empty(b - a, dtype=torch.float64, device=dev)
        dg.run_device(pin, o.data_ptr())  # warm-up (sweep graph capture)
        _, _, st = dg.run_device(pin, o.data_ptr())
        plain_ms += st["ms_total"]
        dg.close()
    plain_ms *= count / len(idx)
    peak, peak_kind = measured_peak_hbm()
    return {"workload": f"batch_hyperbolic{count}_fp32", "graphs": count,
            "nodes": int(offs[-1]), "arcs": int(csr.arcs), "gen_s": t_gen, "create_s": t_create,
            "tune_s": t_tune, "tuning": best, "tuning_candidates": len(table),
            "tuning_table_top": sorted(table, key=lambda t: t["ms"])[:6],
            "fp32_ms": ms32, "fp32_sweeps_total": int(sweeps.sum()),
            "critical_graph_ms": float((g_end - g_start).max()),
            "last_graph_end_ms": float(g_end.max()),
            "graph_busy_ms_sum": float((g_end - g_start).sum()),
            "fp32_sweeps_max": int(sweeps.max()), "fp32_floor_stops": floor,
            "gteps_per_iter": arc_it / (ms32 / 1e3) / 1e9,
            "alg_gbs": alg_bytes / (ms32 / 1e3) / 1e9, "alg_frac_of_hbm": alg_bytes / (ms32 / 1e3) / 1e9 / peak,
            "peak_source": peak_kind,
            "fp32_l1_err_max": float(errs.max()), "fp32_l1_err_median": float(np.median(errs)),
            "vs_oracle": {"kind": "port", "tol": 1e-13, "graphs": len(o_errs), "seconds": o_secs,
                          "fp32_l1_err_max": max(o_errs), "fp32_max_rel_err_max": max(o_rel)},
            "e2e_ms_host_scores": e2e_ms,
            "fp64_batch_ms": ms64_batch, "plain_fp64_per_graph_ms": plain_ms,
            "plain_graphs_timed": len(idx),
            "speedup_vs_plain_fp64": plain_ms / ms32,
            "speedup_fp64_batch_vs_plain_fp64": plain_ms / ms64_batch}


def form_centrality(local, csr):
    """EigenvectorCentrality (tol 1e-9) and KatzCentrality (alpha 0 = 1/(1 +
    max degree), beta 0.1, tol 1e-8, in- and out-edges) on the R-MAT scale-24
    graph, FP64, graph resident: device time per run and per iteration."""
    from networkit_b200 import _capi

    dg = _capi.DeviceGraph(csr, device=local)
    res = {"workload": "eigenvector_katz_rmat24_fp64", "arcs": csr.arcs}
    runs = (("eigenvector", lambda: dg.eigenvector(1e-9)),
            ("katz_in", lambda: dg.katz(0.0, 0.1, 1e-8, 0)),
            ("katz_out", lambda: dg.katz(0.0, 0.1, 1e-8, 1)))
    for name, fn in runs:
        fn()  # warm-up (out-layout build for katz_out)
        _, it, st = fn()
        ms = st["ms_total"]
        res[name] = {"ms": ms, "iterations": it, "ms_per_iteration": ms / max(it, 1),
                     "gteps_per_iter": csr.arcs * it / (ms / 1e3) / 1e9,
                     "gpu_launches": st["kernel_launches"]}
    dg.close()
    res["reference_scale21"] = centrality_vs_reference(local)
    return res


def centrality_vs_reference(local, scale=21):
    """The reference's own CPU paths beside ours on directed R-MAT `scale`
    (same generator and seed as the headline, all host cores): building the
    graph from its edge list (Graph::addEdge in a loop against
    nkg_graph_create_from_edges from host arrays, both to a graph ready for
    the run), EigenvectorCentrality::run (tol 1e-9) and KatzCentrality::run
    (alpha = 1/(1 + maxDegree), beta 0.1, tol 1e-8, in-edges). Device runs
    timed with CUDA events, reference runs around run() only."""
    from networkit_b200 import _capi, generators

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.ref_available():
        return {"unavailable": "oracle/_ref/libnkref.so is not built"}
    import torch

    csr = generators.rmat_directed(scale, EDGEFACTOR, *RMAT, seed=SEED)
    rows = np.repeat(np.arange(csr.z, dtype=np.uint32), np.diff(csr.in_ptr).astype(np.int64))
    cores = os.cpu_count() or 1
    out = {"workload": f"rmat{scale}_fp64", "n": csr.z, "arcs": csr.arcs, "cores": cores,
           "kind": "reference"}
    t0 = time.perf_counter()
    rg = oracle.RefGraph.from_edges(csr.z, csr.in_col, rows, directed=True)
    ref_build = time.perf_counter() - t0
    best = float("inf")
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = _capi.DeviceGraph.from_edges(csr.z, csr.in_col, rows, directed=True, device=local)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
        g.close()
    out["ingest"] = {"reference_s": ref_build, "ours_s": best, "speedup": ref_build / best}
    dg = _capi.DeviceGraph(csr, device=local)
    _, ref_s = rg.eigenvector(1e-9, nthreads=cores, timed=True)
    dg.eigenvector(1e-9)
    _, it, st = dg.eigenvector(1e-9)
    out["eigenvector"] = {"reference_s": ref_s, "ours_ms": st["ms_total"], "iterations": it,
                          "speedup": ref_s / (st["ms_total"] / 1e3)}
    _, _, ref_s = rg.katz(0.0, 0.1, 1e-8, out_edges=False, nthreads=cores, timed=True)
    dg.katz(0.0, 0.1, 1e-8, 0)
    _, it, st = dg.katz(0.0, 0.1, 1e-8, 0)
    out["katz_in"] = {"reference_s": ref_s, "ours_ms": st["ms_total"], "iterations": it,
                      "speedup": ref_s / (st["ms_total"] / 1e3)}
    dg.close()
    del rg
    return out


def form_er(local, n=100_000, avg_deg=10, seed=42, threads=8, runs=5):
    """PageRank FP64 on G(n = 1e5, average degree 10), undirected, the graph
    the reference's ErdosRenyiGenerator draws from seed 42 on 8 OpenMP
    threads (setSeed(42, False); `generators.erdos_renyi_stream` draws the
    same graph), damp 0.85, tol 1e-8, L2, not normalized. With distributeSinks,
    as the workload asks: device time per run, iterations and L1 against the
    oracle. Without (this reference has no sink redistribution): the same,
    plus the reference's own PageRank::run() on the reference's own graph,
    on all host cores, and the L1 between the two. Device runs are timed with
    CUDA events (graph resident); `e2e_ms` is upload of the host in-CSR,
    run and scores back, by the host clock."""
    import torch

    from networkit_b200 import _capi, generators

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    p = avg_deg / (n - 1)
    csr = generators.erdos_renyi_stream(n, p, seed, threads=threads)
    res = {"workload": "pagerank_er1e5_deg10_l2_fp64", "n": n, "arcs": int(csr.arcs),
           "graph": f"the reference generator's draw (seed {seed}, {threads} threads)"}
    for distribute in (True, False):
        dg = _capi.DeviceGraph(csr, device=local)
        prm = dg.params(0.85, 1e-8, 1, False, distribute, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
        dg.run(prm)
        best, s, it, st = float("inf"), None, 0, None
        for _ in range(runs):
            s, it, _, st = dg.run(prm)
            best = min(best, st["ms_total"])
        dg.close()
        e2e = float("inf")
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = _capi.DeviceGraph(csr, device=local)
            g2.run(g2.params(0.85, 1e-8, 1, False, distribute, _capi.NKG_PREC_FP64,
                             _capi.UINT64_MAX))
            e2e = min(e2e, (time.perf_counter() - t0) * 1e3)
            g2.close()
        o = oracle.pagerank(csr, tol=1e-8, norm=1, distribute_sinks=distribute,
                            nthreads=os.cpu_count() or 1)
        r = {"ms": best, "iterations": it, "e2e_ms": e2e, "gpu_launches": st["kernel_launches"],
             "gteps_per_iter": csr.arcs * it / (best / 1e3) / 1e9,
             "oracle_iterations": o.iterations,
             "l1_vs_oracle": float(np.abs(s - o.scores).sum())}
        if not distribute and oracle.ref_available():
            cores = os.cpu_count() or 1
            rg = oracle.RefGraph.erdos_renyi(n, p, seed, directed=False, threads=threads)
            ref = min((rg.pagerank(damp=0.85, tol=1e-8, normalized=False, norm=1,
                                   nthreads=cores, want_ranking=False) for _ in range(3)),
                      key=lambda x: x["seconds"])
            r.update({"reference_ms": ref["seconds"] * 1e3, "reference_cores": cores,
                      "reference_iterations": ref["iterations"],
                      "l1_vs_reference": float(np.abs(s - ref["scores"]).sum()),
                      "speedup_device": ref["seconds"] * 1e3 / best,
                      "speedup_e2e": ref["seconds"] * 1e3 / e2e})
            del rg
        res["distribute_sinks" if distribute else "no_sink_redistribution"] = r
    return res


def form_locality(local, n=4_000_000, deg=16):
    """PageRank FP64 (tol 1e-10, L1) on an undirected threshold hyperbolic graph
    numbered by angle (the graph the reference's HyperbolicGenerator draws
    after setSeed(21, False), `generators.hyperbolic_stream`): the sliced
    layout with in-degree relabelling (row_order 0) against half-octave
    in-degree buckets that keep the id order inside a bucket (row_order 1,
    the automatic choice for this graph). Device time per run, graph resident."""
    from networkit_b200 import _capi, generators

    g = generators.hyperbolic_stream(n, deg, 3, seed=21)
    res = {"workload": f"pagerank_hyperbolic{n}_deg{deg}_fp64", "n": g.z, "arcs": g.arcs}
    for ro in (0, 1, -1):
        dg = _capi.DeviceGraph(g, device=local, row_order=ro)
        p = dg.params(DAMP, TOL, NORM_L1, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
        dg.run(p)
        _, it, _, st = dg.run(p)
        info = dg.info()
        k, _ = dg.profile_sweeps(_capi.NKG_PREC_FP64, 10)
        res[f"row_order_{ro}"] = {"resolved": info["row_order"], "ms": st["ms_total"],
                                  "iterations": it, "slots": info["slots"], "ms_per_sweep": k,
                                  "gteps_per_iter": g.arcs * it / (st["ms_total"] / 1e3) / 1e9}
        dg.close()
    res["speedup_buckets"] = res["row_order_0"]["ms"] / res["row_order_1"]["ms"]
    return res


def form_local(local, n=1_000_000, deg=16, seeds=16384, alpha=0.1, eps=1e-5, ref_sample=48,
               runs=2):
    """PageRankNibble(G, 0.1, 1e-5) (the SelectiveCDGTest.cpp parameters),
    one community per seed (SelectiveCommunityDetector::run) for `seeds`
    random seeds of an undirected threshold hyperbolic graph (n nodes,
    average degree `deg`, exponent 3; the reference HyperbolicGenerator's
    draw after setSeed(11, False)): device time, end-to-end time through
    the C ABI (host seeds in, host communities out), pushes per second, and
    the reference's own PageRankNibble on a sample of the seeds (one core: the
    reference runs the seeds one after another)."""
    from networkit_b200 import _capi, generators

    g = generators.hyperbolic_stream(n, deg, 3, seed=11)
    dl = _capi.DeviceLocal(g.z, g.in_ptr, g.in_col, None, None, False, device=local)
    rng = np.random.default_rng(5)
    sd = np.sort(rng.choice(g.z, seeds, replace=False))
    problems = sd  # one single-seed problem per entry
    # Per-problem bound: alpha * eps * vol >= 1e-6 moves into p per push
    # (unweighted, vol >= 1), so no problem takes more than 1 / (alpha * eps)
    # pushes, plus about 1100 halvings for an isolated seed.
    maxp = int(1.0 / (alpha * eps)) + 2000
    walls = []
    for _ in range(runs):  # the first call sizes the map and result pools
        t0 = time.perf_counter()
        sups, sets, st = dl.run(problems, alpha, eps, nibble=True, max_pushes=maxp)
        walls.append(time.perf_counter() - t0)
    wall = walls[-1]
    res = {"workload": f"pagerank_nibble_hyperbolic{n}_deg{deg}_seeds{seeds}",
           "alpha": alpha, "epsilon": eps, "n": g.z, "arcs": g.arcs, "seeds": seeds,
           "slots": st["slots"], "pushes": st["pushes"], "arc_visits": st["arc_visits"],
           "map_entries": st["table_entries"], "reruns": st["reruns"],
           "mean_support": st["support"] / seeds,
           "mean_set": float(np.mean([s.shape[0] for s in sets])),
           "ms_device": st["ms_total"], "ms_push_kernel": st["ms_push"],
           "seeds_per_s": seeds / (st["ms_total"] / 1e3),
           "pushes_per_s": st["pushes"] / (st["ms_push"] / 1e3),
           "e2e_seeds_per_s": seeds / wall, "e2e_ms": 1e3 * wall,
           "gpu_launches": st["kernel_launches"]}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if oracle.ref_available() and ref_sample:
        # The reference generator's own Graph: the same graph with the same
        # neighbour order in every row (generators.hyperbolic_stream restates
        # it; tests/test_reference_generators.py pins the two together).
        rg = oracle.RefGraph.hyperbolic(n, deg, 3, seed=11, threads=1)
        sample = sd[:: max(1, seeds // ref_sample)][:ref_sample]
        ref_sets, secs = rg.prn(alpha, eps, sample)
        idx = np.searchsorted(sd, sample)
        deg = np.diff(g.in_ptr).astype(np.float64)  # vol: no self-loops, unweighted
        same = ties = 0
        for i, j in enumerate(idx):
            if np.array_equal(ref_sets[i], sets[j]):
                same += 1
                continue
            # Equal but for the order of one group of equal p/vol values,
            # which the reference's unstable sort leaves open.
            nodes, vals = sups[j]
            key = dict(zip(nodes.tolist(), (vals / deg[nodes]).tolist()))
            diff = np.setxor1d(ref_sets[i], sets[j])
            ties += int(len({key.get(int(x)) for x in diff}) == 1)
        res["reference"] = {"seeds": int(sample.shape[0]), "seconds": secs,
                            "seeds_per_s": sample.shape[0] / secs, "cores": 1,
                            "kind": "reference",
                            "sets_identical": same, "sets_equal_up_to_tie_order": ties}
        res["speedup_vs_reference_device"] = res["seeds_per_s"] / res["reference"]["seeds_per_s"]
        res["speedup_vs_reference_e2e"] = res["e2e_seeds_per_s"] / res["reference"]["seeds_per_s"]
    dl.close()
    return res


def form_reader(local, csr, chunks=32, runs=3):
    """NetworkitBinaryGraph input on the R-MAT scale-24 graph: the file
    written by the project's writer (byte-identical to the reference
    writer's), then decoded four ways, best of `runs` each (the file in the
    page cache): the host decoder alone (file -> in-CSR arrays), the host
    decoder plus the device upload (file -> resident graph -> PageRank-ready),
    the device decoder (file read into pinned memory, copied once, decoded and
    built on the GPU: nkg_graph_create_from_nkbg), and the reference's
    NetworkitBinaryReader::read (file -> Graph; all host cores). The device
    decode's graph is checked to equal the host decode's (same PageRank bits)."""
    from networkit_b200 import _capi, graphio

    path = os.path.join(tempfile.gettempdir(), f"nk_b200_rmat{csr.z}.nkbg")
    out_ptr, out_col, _ = csr.out_csr()
    t0 = time.perf_counter()
    graphio.write_nkbg(path, csr.z, out_ptr, out_col, None, csr.in_ptr, csr.in_col, None,
                       directed=True, chunks=chunks)
    t_write = time.perf_counter() - t0
    del out_ptr, out_col
    size = os.path.getsize(path)
    res = {"workload": f"nkbg_read_rmat24_chunks{chunks}", "file_bytes": size, "arcs": csr.arcs,
           "n": csr.z, "write_s": t_write, "cores": os.cpu_count() or 1}
    best = float("inf")
    for _ in range(runs):
        t0 = time.perf_counter()
        g = graphio.read_nkbg(path)
        best = min(best, time.perf_counter() - t0)
    assert g.arcs == csr.arcs and np.array_equal(g.in_col, csr.in_col)
    res["decode_s"] = best
    res["decode_gb_per_s"] = size / best / 1e9
    res["decode_marcs_per_s"] = csr.arcs / best / 1e6
    best = float("inf")
    for _ in range(runs):
        t0 = time.perf_counter()
        g = graphio.read_nkbg(path)
        dg = _capi.DeviceGraph(g, device=local)
        import torch

        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
        dg.close()
    res["file_to_device_graph_s"] = best
    # The device decoder: the file's bytes in pinned memory, one copy, decoded
    # and built on the GPU.
    import torch

    pinned = torch.empty(size, dtype=torch.uint8).pin_memory()
    buf = pinned.numpy()
    best = best_dec = float("inf")
    best_read = float("inf")
    for rep in range(runs):
        t0 = time.perf_counter()
        with open(path, "rb", buffering=0) as f:
            f.readinto(memoryview(buf))
        t1 = time.perf_counter()
        dg = _capi.DeviceGraph.from_nkbg(buf, device=local)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        best_read = min(best_read, t1 - t0)
        best = min(best, t2 - t0)
        best_dec = min(best_dec, dg.ms_decode)
        if rep == runs - 1:
            p = dg.params(DAMP, TOL, NORM_L1, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
            sd, itd, _, _ = dg.run(p)
            dh = _capi.DeviceGraph(g, device=local)
            sh, ith, _, _ = dh.run(p)
            res["device_decode_same_pagerank"] = bool(itd == ith and np.array_equal(
                sd.view(np.uint64), sh.view(np.uint64)))
            dh.close()
        dg.close()
    # The same from the file's path (nkg_graph_create_from_nkbg_file): reader
    # threads stream it through page-locked staging blocks to the device.
    best_file = best_load = float("inf")
    for rep in range(runs):
        t0 = time.perf_counter()
        dg = _capi.DeviceGraph.from_nkbg_file(path, device=local)
        torch.cuda.synchronize()
        best_file = min(best_file, time.perf_counter() - t0)
        best_load = min(best_load, dg.s_load)
        dg.close()
    res["device"] = {"file_to_device_graph_s": best_file, "file_load_s": best_load,
                     "file_load_gb_per_s": size / best_load / 1e9,
                     "via_pinned_buffer": {"file_read_to_pinned_s": best_read,
                                           "file_to_device_graph_s": best},
                     "decode_ms": best_dec,
                     "decode_gb_per_s": size / (best_dec / 1e3) / 1e9,
                     "speedup_file_to_graph_vs_host_decoder":
                         res["file_to_device_graph_s"] / best_file}
    del pinned, buf
    del g
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if oracle.ref_available():
        best = float("inf")
        for _ in range(2):
            t0 = time.perf_counter()
            rg = oracle.RefGraph.read_nkbg(path)
            best = min(best, time.perf_counter() - t0)
            del rg
        res["reference"] = {"read_s": best, "marcs_per_s": csr.arcs / best / 1e6,
                            "kind": "reference", "cores": os.cpu_count() or 1,
                            "sample": "NetworkitBinaryReader::read of the same file"}
        res["speedup_decode_vs_reference"] = best / res["decode_s"]
        res["speedup_file_to_device_graph_vs_reference"] = (
            best / res["device"]["file_to_device_graph_s"])
    os.remove(path)
    return res


def headline_parity(csr, scores, iterations, gpu_rank_ids, rank_scores):
    """Parity of the benchmarked run with the reference's own PageRank::run()
    (oracle/_ref, compiled from the reference sources) on the same graph and
    parameters, on all host cores; the oracle's C restatement when the
    reference library is absent. Reports the L1 and largest relative
    difference of the scores, both iteration counts, and the ranking
    positions where the two orders differ on nodes whose scores differ by
    more than 1e-12 relative (anything else is an exact or rounding tie)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    if oracle.ref_available():
        rows = np.repeat(np.arange(csr.z, dtype=np.uint32), np.diff(csr.in_ptr).astype(np.int64))
        g = oracle.RefGraph.from_edges(csr.z, csr.in_col, rows, directed=True)
        del rows
        r = g.pagerank(damp=DAMP, tol=TOL, norm=NORM_L1, nthreads=cores, want_ranking=True)
        del g
        ref_scores, ref_it, ref_ids = r["scores"], r["iterations"], r["ranking_ids"]
        kind = "reference"
    else:
        o = oracle.pagerank(csr, damp=DAMP, tol=TOL, norm=NORM_L1, nthreads=cores)
        ref_scores, ref_it = o.scores, o.iterations
        ref_ids = oracle.ranking(o.scores)[0]
        kind = "port"
    secs = time.perf_counter() - t0
    diff = np.abs(scores - ref_scores)
    ids_g = np.asarray(gpu_rank_ids, np.int64)
    ids_r = np.asarray(ref_ids, np.int64)
    pos = np.flatnonzero(ids_g != ids_r)
    a, b = rank_scores[ids_g[pos]], rank_scores[ids_r[pos]]
    outside = int(np.count_nonzero(np.abs(a - b) > 1e-12 * np.maximum(np.abs(a), np.abs(b))))
    return {"checker": kind, "cores": cores, "seconds": secs, "tol": TOL, "norm": "L1",
            "l1": float(diff.sum()),
            "max_rel": float((diff / np.maximum(np.abs(ref_scores), 1e-300)).max()),
            "iterations": int(iterations), "checker_iterations": int(ref_it),
            "ranking_positions_differing": int(pos.shape[0]),
            "ranking_mismatches_outside_ties": outside,
            "bar": {"l1": 1e-10, "iterations": 1, "ranking_mismatches_outside_ties": 0},
            "pass": bool(diff.sum() <= 1e-10 and abs(int(iterations) - int(ref_it)) <= 1
                         and outside == 0)}, ref_scores


def run_row_partitioned(args, csr, local, rank, world, barrier):
    """bench.py --gpus N (N > 1): one PageRank run on the R-MAT graph with its
    rows cut into N slices of about equal arc counts, one per rank. A step is
    one run to convergence; every rank times its steps with CUDA events and
    the job's time is the slowest rank's. value = arcs x iterations / that
    time (the whole job's rate: strong scaling)."""
    import torch

    from networkit_b200 import distributed

    comm = distributed.Comm()
    kw = dict(damp=DAMP, tol=TOL, norm=NORM_L1)
    t0 = time.perf_counter()
    pr = distributed.RowPartitionedPageRank(csr, device=local, comm=comm)
    create_s = time.perf_counter() - t0
    for _ in range(max(args.warmup, 3)):
        pr.run(**kw)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        ev[0].record()
        iters = []
        for _ in range(args.steps):
            scores, it, _, _ = pr.run(**kw)
            iters.append(it)
        ev[1].record()
        torch.cuda.synchronize()
        barrier()
    clocks = clk.summary()
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[1]), f"cuda:{local}")
    value = csr.arcs * sum(iters) / (total_ms / 1e3) / 1e9
    # Where an iteration goes on this rank: its slice's sweeps, and the
    # all-reduce + all-gather (one timed run).
    _, it_b, _, stb = pr.run(timing=True, **kw)
    ms_sweep = max_over_ranks(stb["ms_sweeps"] / it_b, f"cuda:{local}")
    ms_exch = max_over_ranks(stb["ms_exchange"] / it_b, f"cuda:{local}")
    slice_bytes = 4 * pr.slice_arcs[rank] + 32 * int(pr.plan.rows[rank]) + 4
    peak, peak_kind = measured_peak_hbm()
    slice_arcs, body = pr.slice_arcs, pr.body
    pr.close()
    # End to end through the same API: slices uploaded from host arrays,
    # run, scores gathered to the host, per step.
    e2e_t, e2e_it = [], []
    for i in range(2):
        barrier()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        p2 = distributed.RowPartitionedPageRank(csr, device=local, comm=comm)
        _, it2, _, _ = p2.run(**kw)
        p2.close()
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t1, f"cuda:{local}")
        if i > 0:
            e2e_t.append(dt)
            e2e_it.append(it2)
    parity = None
    if rank == 0 and not args.no_parity:
        rank_ids = np.argsort(-scores, kind="stable")
        parity, _ = headline_parity(csr, scores, iters[-1], rank_ids, scores)
    barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pagerank_rmat{args.scale}_fp64", "scale": args.scale,
                       "edgefactor": EDGEFACTOR, "abcd": [*RMAT, round(1 - sum(RMAT), 6)],
                       "n": csr.z, "arcs": csr.arcs, "damp": DAMP, "tol": TOL, "norm": "L1",
                       "iterations": iters[0], "parallelism": f"rows{world}",
                       "slice_arcs": slice_arcs, "create_s": create_s,
                       "l2": "inputs larger than L2 (CSR 1.1 GB)"},
            "roofline": {"bound": "hbm", "achieved": slice_bytes / (ms_sweep / 1e3) / 1e9,
                         "peak": peak, "unit": "GB/s",
                         "frac": slice_bytes / (ms_sweep / 1e3) / 1e9 / peak, "traffic": None,
                         "kernel": "sweep_kernel<double, PART> (rank 0's slice)",
                         "bytes_per_launch": slice_bytes, "ms_per_sweep": ms_sweep,
                         "ms_exchange_per_iteration": ms_exch,
                         "exchange_bytes_per_iteration": 8 * body + 16,
                         "peak_source": peak_kind},
            "e2e": {"value": csr.arcs * sum(e2e_it) / sum(e2e_t) / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": 8 * (csr.z + world) + 4 * csr.arcs + 4 * csr.z,
                    "d2h_bytes_per_step": 8 * body * world,
                    "ms_per_step": 1e3 * sum(e2e_t) / len(e2e_t)},
            "gpu_launches": sum(iters) * 2 * world,
            "clocks": clocks, "cpu_baseline": None, "parity": parity,
        }
        print(json.dumps(line))


def run_reference_arm(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libnkref.so (reference PageRank built from the "
                          "reference sources) is not present"}))
        return
    cores = os.cpu_count() or 1
    csr = make_graph(args.scale, args.cache, 0, lambda: None)
    rows = np.repeat(np.arange(csr.z, dtype=np.uint32), np.diff(csr.in_ptr).astype(np.int64))
    # Inserting the arcs row by row reproduces every in-list in the same
    # order (unweighted graph: out-list order does not enter the result).
    g = oracle.RefGraph.from_edges(csr.z, csr.in_col, rows, directed=True)
    del rows
    # Warm-up steps run one iteration each (page-in and thread start-up);
    # every timed step is PageRank::run() with maxIterations = iters, so the
    # run's fixed work (PageRank.cpp:22-30 set-up, :75-104 normalisation) is
    # paid once per `iters` sweeps. `fixed_s` estimates that fixed part from
    # the one-iteration runs, for reference.
    one = []
    for i in range(max(args.warmup, 2)):
        one.append(g.pagerank(damp=DAMP, tol=TOL, norm=NORM_L1, max_iterations=1, nthreads=cores,
                              want_ranking=False)["seconds"])
    iters = int(max(4, min(12, 8.0 / max(min(one), 1e-3))))
    times, its = [], []
    for i in range(args.steps):
        r = g.pagerank(damp=DAMP, tol=TOL, norm=NORM_L1, max_iterations=iters, nthreads=cores,
                       want_ranking=False)
        times.append(r["seconds"])
        its.append(r["iterations"])
    total = sum(times)
    value = csr.arcs * sum(its) / total / 1e9
    per_iter = total / sum(its)
    fixed_s = max(0.0, statistics.median(one[1:] or one) - per_iter)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"pagerank_rmat{args.scale}_fp64", "scale": args.scale,
                   "edgefactor": EDGEFACTOR, "n": csr.z, "arcs": csr.arcs, "damp": DAMP,
                   "tol": TOL, "norm": "L1", "iterations_per_step": iters},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "cpu_model": host_cpu()["model"], "physical_cores": host_cpu()["physical"],
                         "build": "reference sources, C++14 -O3 -DNDEBUG "
                                  "-DNETWORKIT_RELEASE_LOGGING -fopenmp (its CMake Release "
                                  "defaults)",
                         "fixed_s_per_run": fixed_s, "s_per_iteration": per_iter,
                         "sample": f"{iters} iterations of NetworKit::PageRank::run() per step "
                                   f"(maxIterations={iters}) on the same graph; warm-up steps "
                                   f"of one iteration"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    rank, world, local = dist_env()
    import torch

    torch.cuda.set_device(local)
    if args.form == "ppr":
        print(json.dumps(form_ppr(local, n=args.ppr_n, step_only=args.ppr_step_only)))
        return
    if args.form == "batch":
        print(json.dumps(form_batch(local, count=args.batch_graphs,
                                    step_only=args.batch_step_only)))
        return
    if args.form == "locality":
        print(json.dumps(form_locality(local)))
        return
    if args.form == "er":
        print(json.dumps(form_er(local)))
        return
    if args.form == "local":
        print(json.dumps(form_local(local, n=args.local_n, seeds=args.local_seeds,
                                    ref_sample=args.local_ref_sample, runs=args.local_runs)))
        return
    if args.form == "adjoint":
        print(json.dumps(form_adjoint(local, scale=args.adjoint_scale, fd_edges=args.fd_edges,
                                      only_step=args.adjoint_step_only)))
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

        def barrier():
            dist.barrier()
    else:
        def barrier():
            pass

    from networkit_b200 import _capi

    csr = make_graph(args.scale, args.cache, rank, barrier)
    if world > 1 and args.multi == "rows":
        run_row_partitioned(args, csr, local, rank, world, barrier)
        dist.destroy_process_group()
        return
    if args.form == "refine":
        print(json.dumps(form_refine(local, csr)))
        return
    if args.form == "centrality":
        print(json.dumps(form_centrality(local, csr)))
        return
    if args.form == "reader":
        print(json.dumps(form_reader(local, csr)))
        return
    arcs, n = csr.arcs, csr.z
    dg = _capi.DeviceGraph(csr, device=local, sweep_shape=args.shape, arc_order=args.arc_order,
                           hot_tier_kb=args.hot_tier_kb)
    info = dg.info()
    if args.profile_only:
        prec = _capi.NKG_PREC_FP64 if args.precision == "fp64" else _capi.NKG_PREC_FP32
        ms_k, ms_i = dg.profile_sweeps(prec, args.profile_only)
        print(json.dumps({"profile_only": args.profile_only, "precision": args.precision,
                          "shape": args.shape, "arc_order": args.arc_order,
                          "hot_tier_kb": args.hot_tier_kb,
                          "scale": args.scale, "n": n, "arcs": arcs,
                          "slots": info["slots"], "split_rows": info["split_rows"],
                          "ms_sweep_kernel": ms_k, "ms_iteration": ms_i}))
        dg.close()
        return
    p = dg.params(DAMP, TOL, NORM_L1, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    d_out = torch.empty(n, dtype=torch.float64, device=f"cuda:{local}")

    for _ in range(max(args.warmup, 3)):
        dg.run_device(p, d_out.data_ptr())

    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev_ms, iters, launches = [], [], 0
        for _ in range(args.steps):
            it, mx, st = dg.run_device(p, d_out.data_ptr())
            dev_ms.append(st["ms_total"])
            iters.append(it)
            launches += st["kernel_launches"]
        torch.cuda.synchronize()
        barrier()
        wall = time.perf_counter() - t0
    clocks = clk.summary()

    total_ms = max_over_ranks(float(sum(dev_ms)), f"cuda:{local}")
    value = replica_gteps(world, arcs, sum(iters), total_ms)

    # Roofline of the dominant kernel (the sweep), timed alone with events.
    ms_kernel, ms_iter = dg.profile_sweeps(_capi.NKG_PREC_FP64, 20)
    # The random-gather bound: the sweep's gathers alone (same slot stream,
    # same iterate), a floor under the sweep time.
    ms_gather = dg.profile_gathers(_capi.NKG_PREC_FP64, 20)
    bytes_sweep = st["bytes_per_sweep_fp64"]
    peak, peak_kind = measured_peak_hbm()
    achieved = bytes_sweep / (ms_kernel / 1e3) / 1e9

    # End to end through the C ABI: pinned host CSR -> create -> run -> scores.
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    from networkit_b200.graph import InCSR

    hcsr = InCSR(csr.z, csr.n, pin(csr.in_ptr), pin(csr.in_col), None, pin(csr.wdeg),
                 csr.outdeg, None, True)
    h_out = pin(np.empty(n, np.float64))
    e2e_t, e2e_it = [], []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        g2 = _capi.DeviceGraph(hcsr, device=local)
        sc, it2, _, _ = g2.run(p, out=h_out)
        g2.close()
        dt = time.perf_counter() - t1
        if i > 0:  # first call warms the allocator and the module
            e2e_t.append(dt)
            e2e_it.append(it2)
    e2e_value = world * arcs * sum(e2e_it) / sum(e2e_t) / 1e9 if e2e_t else None
    # The same from the edge list (COO in insertion order, pinned): the in-CSR is
    # built on the device (nkg_graph_create_from_edges).
    e2e_edges = None
    if args.e2e_steps > 0:
        e_src = pin(csr.in_col)
        e_dst = pin(np.repeat(np.arange(n, dtype=np.uint32),
                              np.diff(csr.in_ptr).astype(np.int64)))
        ts = []
        for i in range(2):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            g3 = _capi.DeviceGraph.from_edges(n, e_src, e_dst, directed=True, device=local)
            _, it3, _, _ = g3.run(p, out=h_out)
            g3.close()
            if i > 0:
                ts.append(time.perf_counter() - t1)
        e2e_edges = {"value": world * arcs * it3 / ts[0] / 1e9, "unit": UNIT,
                     "ms_per_step": 1e3 * ts[0], "h2d_bytes_per_step": 8 * arcs,
                     "d2h_bytes_per_step": 8 * n}
    h2d = 8 * (n + 1) + 4 * arcs
    d2h = 8 * n

    # Parity of the benchmarked run (the last timed step's scores) with the
    # reference on the same graph, after the timed region.
    parity, checker_scores = None, None
    if rank == 0 and not args.no_parity:
        gpu_scores = d_out.cpu().numpy()
        rank_ids, _ = dg.ranking(gpu_scores)
        parity, checker_scores = headline_parity(csr, gpu_scores, iters[-1], rank_ids, gpu_scores)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(csr, host_cpu()["physical"] or os.cpu_count() or 1)
    dg.close()

    # Companion forms, each against the plain FP64 GPU path on the same GPU.
    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        forms = {}
        for name, fn in (("fp32_refine", lambda: form_refine(local, csr, steps=1,
                                                             checker=checker_scores,
                                                             checker_kind=parity and
                                                             parity["checker"])),
                         ("er_config", lambda: form_er(local)),
                         ("ppr", lambda: form_ppr(local, steps=1)),
                         ("fwd_bwd", lambda: form_adjoint(local, steps=2, fd_edges=0)),
                         ("eigenvector_katz", lambda: form_centrality(local, csr)),
                         ("pagerank_nibble", lambda: form_local(local)),
                         ("locality", lambda: form_locality(local)),
                         ("nkbg_reader", lambda: form_reader(local, csr)),
                         ("batch", lambda: form_batch(local, steps=2,
                                                      plain_graphs=range(0, 1024, 8)))):
            try:
                forms[name] = fn()
            except Exception as e:  # a form that fails is reported, not fatal
                forms[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pagerank_rmat{args.scale}_fp64", "scale": args.scale,
                       "edgefactor": EDGEFACTOR, "abcd": [*RMAT, round(1 - sum(RMAT), 6)],
                       "n": n, "arcs": arcs, "sinks": info["sinks"], "damp": DAMP, "tol": TOL,
                       "norm": "L1", "iterations": iters[0], "parallelism": f"replicas{world}",
                       "hot_tier_kb": args.hot_tier_kb,
                       "l2": "inputs larger than L2 (CSR 1.1 GB)",
                       "wall_s": wall, "ms_create": info["ms_create"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(
                             f"sweep_fp64_rmat{args.scale}"),
                         "kernel": "sweep_kernel<double> (SELL-32 pull SpMV)",
                         "bytes_per_launch": bytes_sweep, "ms_per_launch": ms_kernel,
                         "ms_per_iteration": ms_iter, "peak_source": peak_kind,
                         "gather_bound_ms": ms_gather,
                         "frac_of_gather_bound": ms_gather / ms_kernel},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1e3 * sum(e2e_t) / len(e2e_t) if e2e_t else None,
                    "from_edge_list": e2e_edges},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "parity": parity,
        }
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
