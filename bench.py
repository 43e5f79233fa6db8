#!/usr/bin/env python
"""Benchmark: Gauss-Newton iterations per second on a 100,000-pose graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the seeded city-grid SE(2) pose graph with 100,000 poses (1 m steps,
20 m blocks, up to 3 loop closures per pose within 2 m and |dtheta| < 0.3 rad,
odometry / closure noise 0.05 m / 0.01 rad, information diag(1/sigma^2) * 0.1,
initial guess = composed odometry). One step = one Gauss-Newton iteration:
linearise every edge, assemble Omega and xi, invert the 3x3 diagonal blocks,
block-Jacobi PCG with the reference's per-round settings (||r|| < 1e-6 ||xi||
or 500 iterations), add dx to the poses (angles wrapped).

Our arm runs it through libgslam on the GPU; the reference arm runs the CPU
oracle (the reference's algorithm restated in C, single thread) on the same
workload. Under torchrun each rank solves its own seeded replica (weak
scaling): one graph does not shard profitably, since a row-block split would add a
halo exchange and two all-reduces to an iteration of a few microseconds.
"""
import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "g-slam_on_gpu_and_fpga_b200"

N_POSES = 100000
LAMBDA = 0.1
TOL, MAX_ITER = 1e-6, 500
METRIC = "GN iters/s at N=100k (block-Jacobi PCG per round: tol 1e-6, 500 iterations)"
UNIT = "GN iters/s"


def workload(seed):
    G = importlib.import_module(PKG)
    return G.synth.city_grid(N_POSES, seed=seed, k_closures=3, radius=2.0, max_dtheta=0.3)


def config(extra=None):
    c = {"workload": "city-grid SE(2) pose graph, N=100000, K=3 closures within 2 m, lambda=0.1; "
                     "one Gauss-Newton round with block-Jacobi PCG (tol 1e-6, max 500 iterations)",
         "n_poses": N_POSES, "lambda": LAMBDA, "pcg_tol": TOL, "pcg_max_iter": MAX_ITER,
         "l2": "flushed between timed steps (256 MiB device write, outside the timed events)",
         "round": "one CUDA graph per round (gslam_opts.round_graph), bit-identical to eager launches"}
    if extra:
        c.update(extra)
    return c


# --------------------------------------------------------------------------- distributed

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def dist_init(world):
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, value):
    if dist is None:
        return value
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# --------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (every 200 ms) while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.path or not os.path.exists(self.path):
            return out
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if sms:
            out["sm_mhz"] = statistics.median(sms)
            out["sm_max_mhz"] = mx
            out["samples"] = len(sms)
        out["reasons"] = sorted(reasons)
        return out


# --------------------------------------------------------------------------- roofline

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def pcg_bytes_per_iteration(nnzb, nb, s_a, s_v):
    """Algorithmic bytes of one fused PCG iteration: SpMV (values, block columns, row
    pointers, x read and y written once) + 5 vector streams + the FP64 3x3 inverses."""
    b_spmv = nnzb * (9 * s_a + 4) + 4 * (nb + 1) + 2 * 3 * nb * s_v
    return b_spmv + 5 * 3 * nb * s_v + 72 * nb


def solver_traffic(arm, iterations):
    """DRAM bytes of one solver launch of `iterations` iterations from the committed ncu
    summary (one-time staging + per-iteration bytes), or None."""
    path = os.path.join(ROOT, "profiles", f"pcg_{arm}_n100k_traffic.txt")
    if not os.path.exists(path):
        return None
    got = {}
    for line in open(path):
        for key in ("dram_bytes_per_iteration", "dram_bytes_staging"):
            if line.startswith(key + ":"):
                got[key] = float(line.split(":")[1].split()[0])
    if len(got) < 2:
        return None
    return got["dram_bytes_staging"] + iterations * got["dram_bytes_per_iteration"]


# --------------------------------------------------------------------------- our arm

def run_arm(G, torch, cg, precision, steps, warmup, flush):
    g = G.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=LAMBDA,
                             tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=precision,
                             round_graph=1)
    stream = torch.cuda.ExternalStream(g.stream())
    for _ in range(warmup):
        g.round()
    sizes = g.sizes()
    rounds, solves, iters = [], [], []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        st = g.round()
        rounds.append(st.round_ms)
        solves.append(st.solve_ms)
        iters.append(st.iterations)
    return g, stream, sizes, rounds, solves, iters


def e2e_arm(G, torch, g, stream, steps):
    """Same rounds through host buffers: pinned poses in, round, pinned poses out."""
    n = g.n_poses
    h_in = torch.from_numpy(g.poses).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    lib = G.abi.lib()
    ptr_in = C.cast(h_in.data_ptr(), C.POINTER(C.c_double))
    ptr_out = C.cast(h_out.data_ptr(), C.POINTER(C.c_double))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total = 0.0
    for _ in range(steps):
        ev0.record(stream)
        G.abi.check(lib.gslam_set_poses(g._h, ptr_in))
        g.round()
        G.abi.check(lib.gslam_get_poses(g._h, ptr_out))
        ev1.record(stream)
        ev1.synchronize()
        total += ev0.elapsed_time(ev1)
        h_in.copy_(h_out)
    return total, 3 * n * 8, 3 * n * 8


def pose_err_rel(p, ref):
    """||p - ref|| / ||ref|| over all pose components, angle differences wrapped."""
    import numpy as np
    d = p - ref
    d[:, 2] = (d[:, 2] + np.pi) % (2 * np.pi) - np.pi
    return float(np.linalg.norm(d) / np.linalg.norm(ref))


def poses_after(G, cg, precision, rounds):
    g = G.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=LAMBDA,
                             tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=precision)
    for _ in range(rounds):
        g.round()
    p = g.poses.copy()
    g.close()
    return p


def pose_err_by_round(G, cg, checkpoints=(2, 10, 20, 40, 80)):
    """Gauss-Newton from the initial guess with each solver (the bench's PCG settings):
    the mixed run's poses against the FP64 run's after 2 ... 80 rounds, and each run's
    update norm ||dx|| / sqrt(dim) in that round. Truncated solves differ per round; as the
    iteration reaches its fixed point both runs' poses meet."""
    snaps = {}
    for prec in (G.abi.PREC_FP64, G.abi.PREC_MIXED):
        g = G.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=LAMBDA,
                                 tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=prec, round_graph=1)
        for k in range(1, max(checkpoints) + 1):
            st = g.round()
            if k in checkpoints:
                snaps[(prec, k)] = (g.poses.copy(), st.diff)
        g.close()
    F, M = G.abi.PREC_FP64, G.abi.PREC_MIXED
    return {"rounds": list(checkpoints),
            "mixed_vs_gpu_fp64": [float(f"{pose_err_rel(snaps[(M, k)][0], snaps[(F, k)][0]):.3e}")
                                  for k in checkpoints],
            "update_norm_fp64": [float(f"{snaps[(F, k)][1]:.3e}") for k in checkpoints],
            "update_norm_mixed": [float(f"{snaps[(M, k)][1]:.3e}") for k in checkpoints]}


def cpu_baseline_sample(cg, rounds=2):
    """The oracle (reference algorithm in C, one thread) on the same workload; returns
    rounds/s, the seconds taken and the poses after `rounds` rounds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O
    O.build()
    poses = cg.init.copy()
    dim = 3 * cg.n_poses
    t0 = time.perf_counter()
    for _ in range(rounds):
        blocks, _ = O.se2_linearise(poses, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, LAMBDA)
        rp, ci, va, xi = O.csr_build_anchor(dim, cg.edge_i, cg.edge_j, blocks, 1e6)
        dx, _, _ = O.pcg(rp, ci, va, xi, tol=TOL, max_iter=MAX_ITER)
        poses = poses + dx.reshape(-1, 3)
        poses[:, 2] = (poses[:, 2] + np.pi) % (2 * np.pi) - np.pi
    dt = time.perf_counter() - t0
    return rounds / dt, dt, poses


def c4_batch_graphs():
    """The batched-solve workload: 48 city-grid graphs with N log-uniform in [500, 20000]
    (seeds 0..47) and one N=5000 graph under 16 lambdas log-spaced in [0.01, 10]."""
    import numpy as np
    G = importlib.import_module(PKG)
    graphs, lams = [], []
    for s in range(48):
        n = int(np.exp(np.random.default_rng(s).uniform(np.log(500), np.log(20000))))
        graphs.append(G.synth.city_grid(n, seed=s))
        lams.append(LAMBDA)
    base = G.synth.city_grid(5000, seed=1000)
    for lam in np.logspace(-2, 1, 16):
        graphs.append(base)
        lams.append(float(lam))
    return graphs, np.array(lams)


def batch_sample(G, torch, rounds, world, rank, dist):
    """Aggregate GN rounds/s of the 64-graph batch (this rank's LPT share), autotuned
    launch shape, and the worst per-graph pose error against single-graph FP64 solves."""
    import numpy as np
    graphs, lams = c4_batch_graphs()
    share = G.shard.lpt_partition([G.shard.graph_cost(g) for g in graphs], world)[rank]
    mine, mlams = [graphs[i] for i in share], lams[share]
    cand = {"threads_per_cta": (256, 512, 1024), "ctas_per_sm": (1, 2), "sell_window": (1024,)}
    best, timings = G.tune.autotune_batch(mine, mlams, iters=40, candidates=cand, angle_wrap=1)
    out = {}
    for name, prec in (("fp64", G.abi.PREC_FP64), ("mixed", G.abi.PREC_MIXED)):
        opts = dict(best, tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=prec)
        b = G.PoseGraphBatch.from_se2_list(mine, mlams, **opts)
        b.round_all()                                      # warm-up
        b.poses = b.init_poses
        ms, its = 0.0, []
        for _ in range(rounds):
            st = b.round_all()
            ms += st[0].round_ms
            its += [x.iterations for x in st]
        out[name] = dict(poses=b.poses, ms=max_over_ranks(dist, ms), its=float(np.mean(its)), b=b)
    # pose error of the timed rounds against single-graph FP64 rounds (first 8 of the share)
    errs = {"fp64": [], "mixed": []}
    for q, g in enumerate(mine[:8]):
        one = G.PoseGraph.from_se2(g.init, g.edge_i, g.edge_j, g.meas, g.log_w, lam=mlams[q],
                                   tol=TOL, max_iter=MAX_ITER, angle_wrap=1)
        for _ in range(rounds):
            one.round()
        ref = one.poses
        one.close()
        for name in errs:
            pb = out[name]["b"].graph_poses(q, out[name]["poses"])
            errs[name].append(float(np.linalg.norm(pb - ref) / np.linalg.norm(ref)))
    for name in out:
        out[name]["b"].close()
    val = {name: len(graphs) * rounds / (out[name]["ms"] * 1e-3) for name in out}
    return {"graphs": len(graphs), "poses": int(sum(g.init.shape[0] for g in graphs)),
            "value": round(val["mixed"], 2), "fp64_value": round(val["fp64"], 2),
            "unit": "graph GN iters/s (all graphs, one persistent launch per PCG pass)",
            "ms_per_round": round(out["mixed"]["ms"] / rounds, 3),
            "fp64_ms_per_round": round(out["fp64"]["ms"] / rounds, 3),
            "pcg_iterations_mean": out["mixed"]["its"],
            "tuned": best, "tuning_us_per_iteration": {str(c): (round(t, 2) if t else None) for c, t in timings},
            "max_rel_pose_err_vs_single_fp64": {k: (max(v) if v else None) for k, v in errs.items()},
            "dtype": "mixed: f32 inner / f64 refinement; fp64: f64",
            "config": "48 graphs N~logU[500, 20000] + one N=5000 graph x 16 lambdas in [0.01, 10]"}


def spmv_sample(g, peaks):
    """Standalone SpMV from HBM: one launch multiplies many copies of the N=100k matrix
    (more bytes than three L2s), so every value is read from HBM; achieved = algorithmic
    bytes (values, columns, slice pointers, x gathered once, y written) / time."""
    out = {}
    for name, fp32, copies in (("fp64", False, 16), ("fp32", True, 32)):
        ms = g.spmv_bench(fp32, reps=10, n_copies=copies)
        nbytes = g.spmv_bytes(fp32)
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 5), "algorithmic_bytes": nbytes, "achieved_gbs": round(gbs, 1),
                     "frac": round(gbs / peaks["hbm_gbs"], 4), "copies_per_launch": copies}
    return out


def scale_sample(G, torch, flush, peaks, sizes=(10000, 50000), steps=10, warmup=3):
    """The scale sweep below the headline size: the same generator and settings at
    N = 10,000 and 50,000 (K = 3 closures within 2 m, lambda 0.1). Per size and solver:
    GN rounds/s over `steps` graph-captured rounds (L2 flushed between them), microseconds
    per PCG iteration; standalone SpMV from HBM with enough matrix copies per launch to
    exceed three L2s; the mixed run's poses against the FP64 run's after two rounds."""
    import math
    import statistics
    out = {}
    for n in sizes:
        cg = G.synth.city_grid(n, seed=1, k_closures=3, radius=2.0, max_dtheta=0.3)
        row = {}
        for name, prec in (("fp64", G.abi.PREC_FP64), ("mixed", G.abi.PREC_MIXED)):
            g, _, sz, rounds, solves, iters = run_arm(G, torch, cg, prec, steps, warmup, flush)
            row[name] = {"gn_rounds_per_s": round(steps / (sum(rounds) * 1e-3), 2),
                         "us_per_pcg_iteration": round(1e3 * statistics.mean(solves) / statistics.mean(iters), 3),
                         "pcg_iterations_mean": statistics.mean(iters)}
            if name == "fp64":
                row["nnzb"] = sz["nnzb"]
                spmv = {}
                for sname, fp32 in (("fp64", False), ("fp32", True)):
                    nbytes = g.spmv_bytes(fp32)
                    copies = max(1, math.ceil(3 * 126e6 / nbytes))
                    ms = g.spmv_bench(fp32, reps=5, n_copies=copies)
                    gbs = nbytes / (ms * 1e-3) / 1e9
                    spmv[sname] = {"achieved_gbs": round(gbs, 1), "frac": round(gbs / peaks["hbm_gbs"], 4),
                                   "copies_per_launch": copies}
                row["spmv_hbm"] = spmv
            g.close()
        row["mixed_vs_fp64"] = round(row["mixed"]["gn_rounds_per_s"] / row["fp64"]["gn_rounds_per_s"], 3)
        row["pose_err_rel_2_rounds"] = pose_err_rel(poses_after(G, cg, G.abi.PREC_MIXED, 2),
                                                    poses_after(G, cg, G.abi.PREC_FP64, 2))
        out[f"N={n}"] = row
    return out


def c2_sample(G, rounds=50):
    """Per-round pose and residual error against the FP64 CPU oracle on the 7,120-pose
    walk with denser revisits (up to 6 closures within 3 m, ~2% of poses closing more
    than 1,000 steps back), lambda 1.0, the reference's PCG settings, FP64 and mixed."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    cg = G.synth.city_grid(7120, seed=2, k_closures=6, radius=3.0, far_fraction=0.02)
    lam = 1.0
    dim = 3 * cg.n_poses
    p = cg.init.copy()
    ref = []
    t0 = time.perf_counter()
    for _ in range(rounds):
        blocks, _ = O.se2_linearise(p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam)
        rp, ci, va, xi = O.csr_build_anchor(dim, cg.edge_i, cg.edge_j, blocks, 1e6)
        dx, _, _ = O.pcg(rp, ci, va, xi, tol=TOL, max_iter=MAX_ITER)
        p = p + dx.reshape(-1, 3)
        p[:, 2] = (p[:, 2] + np.pi) % (2 * np.pi) - np.pi
        ref.append(p.copy())
    cpu_s = time.perf_counter() - t0
    out = {"config": "N=7120, K=6 within 3 m, 2% far closures, lambda 1.0, 50 rounds, tol 1e-6 / 500",
           "oracle_seconds": round(cpu_s, 2)}
    for name, prec in (("fp64", G.abi.PREC_FP64), ("mixed", G.abi.PREC_MIXED)):
        g = G.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=lam,
                                 tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=prec)
        errs, res = [], []
        for k in range(rounds):
            st = g.round()
            errs.append(pose_err_rel(g.poses, ref[k]))
            res.append(st.rel_residual)
        g.close()
        out[name] = {"pose_err_rel_per_round": [float(f"{e:.3e}") for e in errs],
                     "rel_residual_per_round": [float(f"{r:.3e}") for r in res],
                     "max_pose_err_rel": max(errs)}
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    dist = dist_init(world)
    torch.cuda.set_device(local)
    G = importlib.import_module(PKG)
    G.build.build()
    cg = workload(seed=1 + rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peaks, peak_kind = measured_peaks()

    results = {}
    for arm, prec in (("fp64", G.abi.PREC_FP64), ("mixed", G.abi.PREC_MIXED)):
        barrier(dist)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            g, stream, sizes, rounds, solves, iters = run_arm(G, torch, cg, prec, args.steps,
                                                               args.warmup, flush)
            torch.cuda.synchronize()
        barrier(dist)
        total_ms = max_over_ranks(dist, sum(rounds))
        e2e_ms, h2d, d2h = e2e_arm(G, torch, g, stream, args.steps)
        e2e_ms = max_over_ranks(dist, e2e_ms)
        results[arm] = dict(g=g, sizes=sizes, rounds=rounds, solves=solves, iters=iters,
                            total_ms=total_ms, e2e_ms=e2e_ms, h2d=h2d, d2h=d2h, clocks=clk.summary())

    def arm_summary(r, s_a, s_v):
        nb, nnzb = r["sizes"]["n_poses"], r["sizes"]["nnzb"]
        b_iter = pcg_bytes_per_iteration(nnzb, nb, s_a, s_v)
        mean_iters = statistics.mean(r["iters"])
        mean_solve_ms = statistics.mean(r["solves"])
        return dict(nnzb=nnzb, b_iter=b_iter, mean_iters=mean_iters, mean_solve_ms=mean_solve_ms,
                    achieved=b_iter * mean_iters / (mean_solve_ms * 1e-3) / 1e9,
                    value=world * args.steps / (r["total_ms"] * 1e-3),
                    e2e=world * args.steps / (r["e2e_ms"] * 1e-3))

    f, m = arm_summary(results["fp64"], 8, 8), arm_summary(results["mixed"], 4, 4)
    # pose error after two rounds from the initial guess: against the CPU oracle (the
    # reference's FP64 PCG) when it runs here, and against this library's FP64 solve
    p_fp64 = poses_after(G, cg, G.abi.PREC_FP64, 2)
    p_mixed = poses_after(G, cg, G.abi.PREC_MIXED, 2)
    err = {"rounds": 2, "mixed_vs_gpu_fp64": pose_err_rel(p_mixed, p_fp64)}
    err["by_round"] = pose_err_by_round(G, cg)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, dt, p_oracle = cpu_baseline_sample(cg)
        cpu = {"value": round(v, 5), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"2 GN rounds of the same N=100000 workload ({dt:.1f} s)"}
        err["mixed_vs_oracle"] = pose_err_rel(p_mixed, p_oracle)
        err["gpu_fp64_vs_oracle"] = pose_err_rel(p_fp64, p_oracle)
    traffic = solver_traffic("mixed", m["mean_iters"])
    r = results["mixed"]
    line = {
        "metric": METRIC, "value": round(m["value"], 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(r["total_ms"] / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 inner / f64 refinement", "data": "synthetic (seeded city-grid walk; no dataset)",
        "config": config({"solver": "mixed-precision PCG: FP32 inner Chronopoulos-Gear iterations, FP64 "
                                    "residual / dots / D^-1 / pose accumulation (iterative refinement)",
                          "nnzb": m["nnzb"], "pcg_iterations_mean": m["mean_iters"],
                          "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}),
        "fp64": {"value": round(f["value"], 3), "unit": UNIT,
                 "ms_per_step": round(results["fp64"]["total_ms"] / args.steps, 4),
                 "pcg_iterations_mean": f["mean_iters"],
                 "us_per_pcg_iteration": round(1e3 * f["mean_solve_ms"] / f["mean_iters"], 3),
                 "e2e": round(f["e2e"], 3), "achieved_gbs": round(f["achieved"], 1),
                 "clocks": results["fp64"]["clocks"]},
        "mixed_vs_fp64": round(m["value"] / f["value"], 3),
        "pose_err_rel": err,
        "roofline": {"kernel": "k_pcg_mixed (persistent mixed-precision solve)", "bound": "hbm",
                     "achieved": round(m["achieved"], 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(m["achieved"] / peaks["hbm_gbs"], 4), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_iteration": m["b_iter"],
                     "traffic": (round(traffic) if traffic else None),
                     "traffic_note": "DRAM bytes per launch (ncu): the matrix is staged into shared "
                                     "memory once and every iteration runs on chip, so traffic is far "
                                     "below the algorithmic bytes; the limiter is grid-synchronisation "
                                     "latency, not HBM",
                     "solve_ms_mean": round(m["mean_solve_ms"], 4),
                     "us_per_pcg_iteration": round(1e3 * m["mean_solve_ms"] / m["mean_iters"], 3)},
        "e2e": {"value": round(m["e2e"], 3), "unit": UNIT,
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
        "gpu_launches": 7 * args.steps,
        "clocks": r["clocks"],
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if not args.no_batch:
        line["batch"] = batch_sample(G, torch, 3, world, rank, dist)
    line["spmv_hbm"] = spmv_sample(results["fp64"]["g"], peaks)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["per_round_vs_oracle"] = c2_sample(G)
    if world == 1 and not args.no_scale:
        line["scale"] = scale_sample(G, torch, flush, peaks)
    for arm in results.values():
        arm["g"].close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# --------------------------------------------------------------------------- reference arm

def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    cg = workload(seed=1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O
    O.build()
    dim = 3 * cg.n_poses
    poses = cg.init.copy()

    def one_round(p):
        blocks, _ = O.se2_linearise(p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, LAMBDA)
        rp, ci, va, xi = O.csr_build_anchor(dim, cg.edge_i, cg.edge_j, blocks, 1e6)
        dx, _, _ = O.pcg(rp, ci, va, xi, tol=TOL, max_iter=MAX_ITER)
        p = p + dx.reshape(-1, 3)
        p[:, 2] = (p[:, 2] + np.pi) % (2 * np.pi) - np.pi
        return p

    for _ in range(args.warmup):
        poses = one_round(poses)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        poses = one_round(poses)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    line = {
        "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded city-grid walk; no dataset)", "impl": "reference",
        "config": config({"solver": "reference algorithm restated in C (oracle/), one host thread"}),
        "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"{args.steps} GN rounds of the N=100000 workload"},
        "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_kernels_case(G, g, cg):
    """Every kernel of the library at least once, for a per-kernel DRAM capture (ncu flushes
    the caches before each captured launch, so dram bytes / duration is the kernel's HBM
    rate): the N=100k SE(2) round kernels with 5-iteration FP64 and mixed solves, the
    adjoint, a reference-factor graph (linearisation, round cost, landmark map), a small
    FP64 and mixed batch, and the dense Gauss-Jordan path at n = 3072."""
    import numpy as np
    g.set_opts(precision=G.abi.PREC_FP64, tol=0.0, max_iter=5, angle_wrap=1)
    g.solve()
    g.update()
    g.set_opts(precision=G.abi.PREC_MIXED, tol=0.0, max_iter=5, inner_max_iter=5, angle_wrap=1)
    g.linearise()
    g.assemble()
    g.solve()
    g.update()
    g.set_opts(precision=G.abi.PREC_FP64, tol=0.0, max_iter=5, angle_wrap=1)
    g.set_weights(LAMBDA)
    g.adjoint(np.ones((cg.n_poses, 3)))
    log = G.synth.landmark_log(20000, seed=3)
    with G.PoseGraph.from_log(log, 1.0, max_iter=5) as r:
        r.round()
        r.cost()
        r.landmark_map()
    small = [G.synth.city_grid(n, seed=s) for s, n in enumerate((3000, 5000, 8000, 12000))]
    for prec in (G.abi.PREC_FP64, G.abi.PREC_MIXED):
        b = G.PoseGraphBatch.from_se2_list(small, LAMBDA, precision=prec, tol=0.0, max_iter=5,
                                           inner_max_iter=5, max_refine=2, angle_wrap=1)
        b.round_all()
        b.close()
    rng = np.random.default_rng(0)
    n = 3072
    a = rng.standard_normal((n, n)) / np.sqrt(n) + 4.0 * np.eye(n)
    G.dense.gj_inverse(a)
    G.dense.gj_solve(a, rng.standard_normal(n))
    print("kernels case done", flush=True)


def run_ncu_case(args):
    """A short, untimed solve of the bench workload for ncu captures: the solver runs
    twice on the first round's system, with 50 and then 250 iterations (tolerance 0),
    so per-iteration DRAM traffic is the difference of the two launches / 200."""
    import torch
    G = importlib.import_module(PKG)
    G.build.build()
    cg = workload(seed=1)
    prec = G.abi.PREC_MIXED if args.ncu_case == "mixed" else G.abi.PREC_FP64
    g = G.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=LAMBDA,
                             tol=TOL, max_iter=MAX_ITER, angle_wrap=1, precision=prec)
    g.linearise()
    g.assemble()
    if args.ncu_case == "kernels":
        run_kernels_case(G, g, cg)
        g.close()
        torch.cuda.synchronize()
        return
    if args.ncu_case == "spmv":
        # two launches (warm-up + one timed) of 16 FP64 copies of the matrix
        ms = g.spmv_bench(False, reps=1, n_copies=16)
        print(f"spmv: {ms:.4f} ms per matrix", flush=True)
        g.close()
        return
    for iters in (50, 250):
        g.set_opts(precision=prec, tol=0.0, max_iter=iters, inner_max_iter=iters)
        st = g.solve()
        print(f"{args.ncu_case}: {st.iterations} iterations, {st.solve_ms:.3f} ms", flush=True)
    torch.cuda.synchronize()
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-graph batched-solve sample")
    ap.add_argument("--no-scale", action="store_true", help="skip the N = 10k / 50k scale sample")
    ap.add_argument("--ncu-case", choices=["fp64", "mixed", "spmv", "kernels"], default=None,
                    help="run only two short solves of the workload (for ncu captures)")
    args = ap.parse_args()
    if args.ncu_case:
        run_ncu_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
