"""Autotuner for the batched solver's launch and layout shapes.

The batched PCG streams the matrix, so its speed depends on three choices that are
fixed when a batch is built: threads per CTA (how many slices a CTA works on at
once), CTAs per SM (latency hiding against barrier cost) and the row-sorting window
of the sliced block layout (padding vs. how evenly slices fill a warp). The tuner
builds the batch for every candidate, times a fixed number of PCG iterations with
no early stop (CUDA events inside the library), and returns the fastest.

Not in the reference, which has no tunable kernels.
"""
from __future__ import annotations

import itertools
import json
import os

from . import abi
from .graph import PoseGraphBatch

DEFAULT_CANDIDATES = {
    "threads_per_cta": (256, 512, 1024),
    "ctas_per_sm": (1, 2),
    "sell_window": (32, 256, 1024),
}


def autotune_batch(graphs, lams, iters: int = 40, candidates=None, cache: str | None = None, **opts):
    """Returns (best_opts, timings): best_opts to pass to PoseGraphBatch.from_se2_list,
    timings = [(candidate, us_per_iteration or None if it could not run)].

    `cache`: a JSON file; a result stored there for the same batch shape is reused."""
    key = (f"{len(graphs)}:{sum(int(g.init.shape[0]) for g in graphs)}:{sum(len(g.edge_i) for g in graphs)}"
           f":{opts.get('precision', abi.PREC_FP64)}")
    if cache and os.path.exists(cache):
        with open(cache) as f:
            hit = json.load(f).get(key)
        if hit:
            return hit, []
    cand = candidates or DEFAULT_CANDIDATES
    names = list(cand)
    timings = []
    best, best_t = None, float("inf")
    for values in itertools.product(*(cand[n] for n in names)):
        c = dict(zip(names, values))
        try:
            b = PoseGraphBatch.from_se2_list(graphs, lams, **{**opts, **c, "tol": 0.0, "max_iter": iters})
        except abi.GslamError:
            timings.append((c, None))
            continue
        try:
            b.round_all()                           # warm-up
            st = b.round_all()
            t = 1e3 * st[0].solve_ms / iters
        finally:
            b.close()
        timings.append((c, t))
        if t < best_t:
            best, best_t = c, t
    if cache and best is not None:
        data = {}
        if os.path.exists(cache):
            with open(cache) as f:
                data = json.load(f)
        data[key] = best
        with open(cache, "w") as f:
            json.dump(data, f, indent=1)
    return best, timings
