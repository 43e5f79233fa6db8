"""The seeded city-grid generator and the reference log writer."""
import numpy as np

from conftest import assert_bitwise, load_pkg


def test_deterministic_and_closure_rules():
    S = load_pkg().synth
    a = S.city_grid(2000, seed=9, k_closures=3, radius=2.0)
    b = S.city_grid(2000, seed=9, k_closures=3, radius=2.0)
    assert np.array_equal(a.edge_i, b.edge_i) and np.array_equal(a.meas, b.meas)
    ci, cj = a.edge_i[a.n_odom:].astype(int), a.edge_j[a.n_odom:].astype(int)
    assert np.all(cj > ci)
    d = np.linalg.norm(a.gt[ci, :2] - a.gt[cj, :2], axis=1)
    assert np.all(d <= 2.0 + 1e-9)
    dth = np.abs((a.gt[cj, 2] - a.gt[ci, 2] + np.pi) % (2 * np.pi) - np.pi)
    assert np.all(dth < 0.3)
    assert np.bincount(cj).max() <= 3
    # grid walk: 1 m steps
    steps = np.linalg.norm(np.diff(a.gt[:, :2], axis=0), axis=1)
    assert np.allclose(steps, 1.0)


def test_far_closures_share():
    S = load_pkg().synth
    g = S.city_grid(7120, seed=2, k_closures=6, radius=3.0, far_fraction=0.02)
    ci, cj = g.edge_i[g.n_odom:].astype(int), g.edge_j[g.n_odom:].astype(int)
    far_poses = np.unique(cj[(cj - ci) > 1000])
    assert far_poses.size >= 0.015 * 7120


def test_log_round_trip(tmp_path):
    G = load_pkg()
    g = G.synth.city_grid(400, seed=3)
    log = G.synth.to_reference_log(g)
    p = str(tmp_path / "l.txt")
    G.synth.write_log(p, log)
    back = G.read_log(p)
    assert_bitwise(back.x, log.x, "x")
    assert_bitwise(back.u, log.u, "u")
    assert_bitwise(back.z, log.z, "z")
    assert np.array_equal(back.z_lm, log.z_lm) and np.array_equal(back.z_step, log.z_step)
    # each closure is one virtual landmark seen twice
    assert np.all(np.bincount(log.z_lm)[np.unique(log.z_lm)] == 2)
