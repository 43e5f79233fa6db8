"""gslam_opts.round_graph: the whole Gauss-Newton round (linearise, assemble, block-Jacobi,
solve, pose update, read-backs) replayed as one CUDA graph must give the eagerly launched
round's results bit for bit, including a mixed solve that stagnates and is redone in FP64
by the host, and after options change between rounds."""
import importlib

import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu

PREC_FP64, PREC_MIXED = 0, 1


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")


def _rounds(g, n):
    out = []
    for _ in range(n):
        st = g.round()
        out.append((st.iterations, st.refinements, st.reason, st.diff))
    return out, g.poses


@pytest.mark.parametrize("prec", [PREC_FP64, PREC_MIXED], ids=["fp64", "mixed"])
def test_round_graph_matches_eager_se2(pkg, synth, prec):
    cg = synth.city_grid(3000, seed=5, k_closures=6, radius=3.0)
    runs = []
    for graphed in (0, 1):
        with pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=0.1, angle_wrap=1,
                                    precision=prec, round_graph=graphed) as g:
            runs.append(_rounds(g, 4))
    assert runs[0][0] == runs[1][0]
    assert_bitwise(runs[1][1], runs[0][1], "poses after 4 graphed rounds")


def test_round_graph_matches_eager_reference(pkg, synth):
    log = synth.landmark_log(2500, seed=8)
    runs = []
    for graphed in (0, 1):
        with pkg.PoseGraph.from_log(log, 1.0, round_graph=graphed) as g:
            runs.append(_rounds(g, 3))
            runs[-1] = runs[-1] + (g.cost(),)
    assert runs[0][0] == runs[1][0]
    assert_bitwise(runs[1][1], runs[0][1], "poses after 3 graphed rounds")
    assert runs[0][2] == runs[1][2]


def test_round_graph_stagnation_redone_in_fp64(pkg, synth):
    """The captured pose update skips a stagnated mixed solve; the host solves in FP64 and
    updates, as the eager round does."""
    cg = synth.city_grid(2000, seed=3)
    runs = []
    for graphed in (0, 1):
        with pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=0.1, angle_wrap=1,
                                    precision=PREC_MIXED, tol=1e-8, max_iter=200000, max_refine=500,
                                    round_graph=graphed) as g:
            runs.append(_rounds(g, 3))
    assert any(r[1] < 0 for r in runs[1][0][1:]), "no graphed round stagnated"
    assert runs[0][0] == runs[1][0]
    assert_bitwise(runs[1][1], runs[0][1], "poses")


def test_round_graph_rebuilt_after_set_opts(pkg, synth):
    cg = synth.city_grid(1500, seed=2)
    runs = []
    for graphed in (0, 1):
        with pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=0.1, angle_wrap=1,
                                    round_graph=graphed) as g:
            a, _ = _rounds(g, 2)
            g.set_opts(tol=1e-9, max_iter=5000, angle_wrap=1, round_graph=graphed)
            b, p = _rounds(g, 2)
            runs.append((a + b, p))
    assert runs[0][0] == runs[1][0]
    assert_bitwise(runs[1][1], runs[0][1], "poses")


def test_round_io_matches_separate_calls(pkg):
    """gslam_round_io (poses in, round, poses out on the graph's stream, one wait) gives the
    poses of gslam_set_poses + gslam_round + gslam_get_poses, bit for bit, in the eager
    first round and in graph replays."""
    import numpy as np
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    cg = synth.city_grid(3000, seed=12)
    out = {}
    for mode in ("io", "separate"):
        with pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=0.1, angle_wrap=1,
                                    round_graph=1) as g:
            p = np.ascontiguousarray(cg.init, np.float64)
            res = []
            for _ in range(4):
                if mode == "io":
                    q = np.empty_like(p)
                    g.round_io(p, q)
                else:
                    g.poses = p
                    g.round()
                    q = g.poses
                res.append(q.copy())
                p = q
            out[mode] = res
    for a, b in zip(out["io"], out["separate"]):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
