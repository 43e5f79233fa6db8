"""tune.autotune_batch's cache (no GPU: a hit returns before any batch is built): the key
names the batch's shape and the solver precision, so the FP64 and the mixed batch keep
their own launch shapes."""
import importlib
import json


def test_cache_hit_is_per_precision(tmp_path):
    tune = importlib.import_module("g-slam_on_gpu_and_fpga_b200.tune")
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    abi = importlib.import_module("g-slam_on_gpu_and_fpga_b200.abi")
    graphs = [synth.city_grid(200, seed=1), synth.city_grid(300, seed=2)]
    shape = f"{len(graphs)}:{sum(int(g.init.shape[0]) for g in graphs)}:{sum(len(g.edge_i) for g in graphs)}"
    fp64 = {"threads_per_cta": 256, "ctas_per_sm": 2, "sell_window": 1024}
    mixed = {"threads_per_cta": 512, "ctas_per_sm": 1, "sell_window": 1024}
    cache = tmp_path / "tune.json"
    cache.write_text(json.dumps({f"{shape}:{abi.PREC_FP64}": fp64, f"{shape}:{abi.PREC_MIXED}": mixed}))
    best, timings = tune.autotune_batch(graphs, [0.1, 0.1], cache=str(cache), precision=abi.PREC_FP64)
    assert best == fp64 and timings == []
    best, timings = tune.autotune_batch(graphs, [0.1, 0.1], cache=str(cache), precision=abi.PREC_MIXED)
    assert best == mixed and timings == []
    # no precision given: the FP64 entry
    best, _ = tune.autotune_batch(graphs, [0.1, 0.1], cache=str(cache))
    assert best == fp64
