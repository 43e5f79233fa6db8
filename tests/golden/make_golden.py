"""Regenerates the committed golden fixtures (oracle outputs on seeded synthetic graphs).

    python tests/golden/make_golden.py

Each fixture holds the inputs of a reference-format log produced by the
package's city-grid generator and the C oracle's outputs for it: edge blocks in
both math flavours (glibc and correctly rounded), the reference CSR, xi, one
PCG solution at the reference's settings, the poses after a short run, the
landmark map at those poses and the per-edge round-cost terms at the logged poses. The
oracle itself is pinned bit for bit against the reference build in
tests/test_oracle_pin.py; these fixtures carry that pin to machines without the
reference tree.
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

G = importlib.import_module("g-slam_on_gpu_and_fpga_b200")

CASES = [
    dict(name="city64_s3", n=64, seed=3, lam=0.1, rounds=3, kw=dict(k_closures=3, radius=2.0, block=8)),
    dict(name="city200_s11", n=200, seed=11, lam=1.0, rounds=3, kw=dict(k_closures=6, radius=3.0)),
]


def make(case):
    cg = G.synth.city_grid(case["n"], seed=case["seed"], **case["kw"])
    log = G.synth.to_reference_log(cg)
    g = O.Graph(log.delta, log.u_step, log.u, log.x_step, log.x, log.z_step, log.z_lm, log.z)
    lam = case["lam"]
    out = dict(delta=log.delta, u_step=log.u_step, u=log.u, x_step=log.x_step, x=log.x,
               z_step=log.z_step, z_lm=log.z_lm, z=log.z, lam=lam, rounds=case["rounds"])
    _, _, out["blocks_glibc"] = O.linearise(g, g.x, lam, cr=False)
    _, _, out["blocks_cr"] = O.linearise(g, g.x, lam, cr=True)
    t1, t2, b = O.linearise(g, g.x, lam, cr=False)
    out["row_ptr"], out["col_idx"], out["values"], out["xi"] = O.csr_build(g.dim, t1, t2, b)
    out["dx"], _, _ = O.pcg(out["row_ptr"], out["col_idx"], out["values"], out["xi"])
    out["poses_run"], _, _ = O.run(g, lam, case["rounds"], cr=False)
    out["lm_ids"], out["lm_ms"] = O.landmark_map(g, out["poses_run"], cr=False)
    _, out["cost_terms"] = O.round_cost(g, g.x, lam, cr=False)
    np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **out)


if __name__ == "__main__":
    O.build()
    for c in CASES:
        make(c)
        print("wrote", c["name"])
