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
