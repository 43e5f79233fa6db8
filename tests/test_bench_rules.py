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
