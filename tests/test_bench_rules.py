"""Host-side rules of bench.py (no GPU): the headline solver choice and the configuration
both arms report."""
import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
bench = importlib.import_module("bench")


def test_headline_is_the_fastest_solver_meeting_the_bar():
    values = {"fp64": 165.4, "fp64_cg": 169.8, "mixed": 319.8}
    assert bench.headline_solver(values, {"fp64": True, "fp64_cg": True, "mixed": False}) == "fp64_cg"
    assert bench.headline_solver(values, {"fp64": True, "fp64_cg": True, "mixed": True}) == "mixed"
    assert bench.headline_solver(values, {"fp64": True, "fp64_cg": False, "mixed": False}) == "fp64"


def test_headline_falls_back_to_the_reference_recurrence():
    values = {"fp64": 165.4, "fp64_cg": 169.8, "mixed": 319.8}
    assert bench.headline_solver(values, {"fp64": False, "fp64_cg": False, "mixed": False}) == "fp64"


def test_both_arms_report_one_workload():
    c = bench.config()
    assert c["n_poses"] == bench.N_POSES == 100000
    assert c["pcg_tol"] == bench.TOL == 1e-6 and c["pcg_max_iter"] == bench.MAX_ITER == 500
    assert "workload" in c and "model" not in c


def _ranks_worker(rank, world, port, out):
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    b = importlib.import_module("bench")
    w, r, _ = b.dist_env()
    dist = b.dist_init(w)          # gloo here: no GPU in this process
    b.barrier(dist)
    t = b.max_over_ranks(dist, 10.0 + 5.0 * r)   # each rank's own device time
    out.put((r, w, t))
    b.barrier(dist)
    dist.destroy_process_group()


def test_timing_is_the_max_over_ranks_gloo():
    """bench.py's multi-rank plumbing on a world-size-2 gloo group: every rank reads its
    place from the launcher's environment and gets the slowest rank's time."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_ranks_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
    assert got == [(0, 2, 15.0), (1, 2, 15.0)]
    assert all(p.exitcode == 0 for p in procs)


def test_cpu_rounds_run_the_references_own_pcg(oracle):
    """The CPU rounds (cpu_baseline and --impl reference) solve with the reference's own
    compiled pcg_solve_sparse where oracle/_ref holds it, and their poses are bit for bit
    the oracle's restatement's (which is what the GPU solvers are held to)."""
    import numpy as np
    import pytest
    if bench.reference_pcg() is None:
        pytest.skip("reference build absent (oracle/_ref)")
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    cg = synth.city_grid(3000, seed=5, k_closures=3, radius=2.0)
    poses, secs, kind, phases = bench.oracle_rounds(cg, 2)
    assert kind == "reference"
    assert phases["pcg_s"] > 0 and sum(phases.values()) <= secs + 2e-3
    p = cg.init.copy()
    for _ in range(2):
        blocks, _ = oracle.se2_linearise(p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, bench.LAMBDA)
        rp, ci, va, xi = oracle.csr_build_anchor(3 * cg.n_poses, cg.edge_i, cg.edge_j, blocks, 1e6)
        dx, _, _ = oracle.pcg(rp, ci, va, xi, tol=bench.TOL, max_iter=bench.MAX_ITER)
        p = p + dx.reshape(-1, 3)
        p[:, 2] = (p[:, 2] + np.pi) % (2 * np.pi) - np.pi
    assert np.array_equal(poses.view(np.uint64), p.view(np.uint64))
