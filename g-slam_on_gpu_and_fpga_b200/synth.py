"""Seeded synthetic pose graphs on a city grid, in both factor families.

The walk: 1 m steps on a grid of 20 m blocks; at every intersection the robot
turns left, right or goes straight with probability 1/3 each. Odometry edges
join consecutive poses; loop closures join a pose to up to K earlier poses
within `radius` metres whose heading differs by less than `max_dtheta`. Every
measurement carries Gaussian noise (sigma_xy, sigma_theta); the initial guess
is the composition of the noisy odometry.

Two outputs for one walk:
  * an SE(2) pose graph (odometry + closures, information diag(1/sigma^2));
  * a reference-format log for the reference's factors (data/README.md): each
    odometry step becomes a `u` line with nu = |dt|, omega = dtheta (the mapping
    of the reference's data/convert_slampp.py:66-67), the composed poses become
    `x` lines, and each closure (i, j) becomes a virtual landmark observed once
    from pose i and once from pose j (one ObsEdge, C(2,2) = 1).
"""
from __future__ import annotations

import os
import subprocess
from dataclasses import dataclass

import numpy as np

from . import abi
from .graph import ReferenceLog


@dataclass
class CityGrid:
    gt: np.ndarray          # [N, 3] ground truth
    init: np.ndarray        # [N, 3] composed noisy odometry
    edge_i: np.ndarray      # [E] (odometry first, then closures)
    edge_j: np.ndarray
    meas: np.ndarray        # [E, 3] relative pose of j in the frame of i (noisy)
    log_w: np.ndarray       # [E, 3] log(1/sigma^2)
    n_odom: int
    seed: int

    @property
    def n_poses(self) -> int:
        return int(self.gt.shape[0])

    @property
    def n_closures(self) -> int:
        return int(self.edge_i.shape[0] - self.n_odom)


def _wrap(a):
    return (a + np.pi) % (2.0 * np.pi) - np.pi


def _relative(pi, pj):
    """Pose of j in the frame of i (x, y, theta), vectorised."""
    c, s = np.cos(pi[:, 2]), np.sin(pi[:, 2])
    dx, dy = pj[:, 0] - pi[:, 0], pj[:, 1] - pi[:, 1]
    return np.stack([c * dx + s * dy, -s * dx + c * dy, _wrap(pj[:, 2] - pi[:, 2])], axis=1)


def _compose(n, rel, start):
    out = np.zeros((n, 3))
    out[0] = start
    x, y, t = start
    for k in range(n - 1):
        c, s = np.cos(t), np.sin(t)
        x, y, t = x + c * rel[k, 0] - s * rel[k, 1], y + s * rel[k, 0] + c * rel[k, 1], t + rel[k, 2]
        out[k + 1] = (x, y, t)
    return out


def city_grid(n: int, seed: int = 0, k_closures: int = 3, radius: float = 2.0,
              max_dtheta: float = 0.3, sigma_xy: float = 0.05, sigma_theta: float = 0.01,
              block: int = 20, min_gap: int = 10, far_fraction: float = 0.0,
              far_gap: int = 1000) -> CityGrid:
    """Generates the walk and its edges. `far_fraction` > 0 makes about that share of
    poses carry at least one closure to a pose more than `far_gap` steps back."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    head = np.zeros(n, np.int64)     # heading index 0..3 (multiples of pi/2)
    turns = rng.integers(-1, 2, size=n)   # -1 right, 0 straight, +1 left
    h = 0
    for k in range(1, n):
        if k % block == 0:
            h = (h + int(turns[k])) % 4
        head[k] = h
    theta = head * (np.pi / 2.0)
    step = np.stack([np.cos(theta), np.sin(theta)], axis=1)
    step = np.round(step)
    pos = np.zeros((n, 2))
    pos[1:] = np.cumsum(step[1:], axis=0)
    gt = np.concatenate([pos, _wrap(theta)[:, None]], axis=1)

    sig = np.array([sigma_xy, sigma_xy, sigma_theta])
    lw = np.log(1.0 / sig ** 2)
    odo_true = _relative(gt[:-1], gt[1:])
    odo = odo_true + rng.normal(size=odo_true.shape) * sig
    init = _compose(n, odo, gt[0])

    # loop closures: up to k earlier poses within radius with similar heading
    tree = cKDTree(pos)
    pairs = tree.query_pairs(r=radius, output_type="ndarray")
    if pairs.size:
        i, j = np.minimum(pairs[:, 0], pairs[:, 1]), np.maximum(pairs[:, 0], pairs[:, 1])
        keep = (j - i >= min_gap) & (np.abs(_wrap(gt[j, 2] - gt[i, 2])) < max_dtheta)
        i, j = i[keep], j[keep]
        d = np.linalg.norm(pos[i] - pos[j], axis=1)
        # far candidates first when a far share is asked for, then nearest
        far = (j - i) > far_gap
        want_far = np.zeros(n, bool)
        if far_fraction > 0:
            cand = np.unique(j[far])
            m = int(round(far_fraction * n))
            if cand.size:
                want_far[rng.choice(cand, size=min(m, cand.size), replace=False)] = True
        pri = np.where(far & want_far[j], 0, 1)
        order = np.lexsort((d, pri, j))
        i, j, pri = i[order], j[order], pri[order]
        first = np.r_[True, j[1:] != j[:-1]]
        grp = np.cumsum(first) - 1
        start = np.flatnonzero(first)
        rank = np.arange(j.size) - start[grp]
        sel = rank < k_closures
        ci, cj = i[sel], j[sel]
        # stable order: by j then i
        o = np.lexsort((ci, cj))
        ci, cj = ci[o], cj[o]
    else:
        ci = cj = np.zeros(0, np.int64)
    lc_true = _relative(gt[ci], gt[cj]) if ci.size else np.zeros((0, 3))
    lc = lc_true + rng.normal(size=lc_true.shape) * sig

    edge_i = np.concatenate([np.arange(n - 1), ci]).astype(np.uint32)
    edge_j = np.concatenate([np.arange(1, n), cj]).astype(np.uint32)
    meas = np.concatenate([odo, lc], axis=0)
    log_w = np.tile(lw, (edge_i.shape[0], 1))
    return CityGrid(gt, init, edge_i, edge_j, meas, log_w, n - 1, seed)


def to_reference_log(g: CityGrid, sigma_range: float = 0.05, sigma_bearing: float = 0.01,
                     side: float = 3.0) -> ReferenceLog:
    """Reference-format records for the same walk (virtual landmarks for closures).

    Landmark ids start above the observation count: the reference program's
    post-loop landmark map starts its "previous id" at the observation count
    (src/cpu_pcg_fp64/GSLAM.c:152) and indexes ms[2 * (count - 1)] with count 0
    (:165, :190) when the first id equals it.
    """
    rng = np.random.default_rng(g.seed + 7919)
    n = g.n_poses
    odo = g.meas[: g.n_odom]
    u = np.zeros((n, 2))
    u[1:, 0] = np.hypot(odo[:, 0], odo[:, 1])
    u[1:, 1] = odo[:, 2]
    ci = g.edge_i[g.n_odom:].astype(np.int64)
    cj = g.edge_j[g.n_odom:].astype(np.int64)
    m = ci.size
    # landmark `side` metres to the left of pose j's true position
    tj = g.gt[cj, 2]
    lm = g.gt[cj, :2] + side * np.stack([-np.sin(tj), np.cos(tj)], axis=1)

    def observe(p):
        d = lm - g.gt[p, :2]
        r = np.hypot(d[:, 0], d[:, 1]) + rng.normal(size=m) * sigma_range
        b = _wrap(np.arctan2(d[:, 1], d[:, 0]) - g.gt[p, 2] + rng.normal(size=m) * sigma_bearing)
        return r, b

    ri, bi = observe(ci)
    rj, bj = observe(cj)
    ids = 2 * m + 6 + np.arange(m)
    z_step = np.concatenate([ci, cj])
    z_lm = np.concatenate([ids, ids])
    z = np.concatenate([np.stack([ri, bi], 1), np.stack([rj, bj], 1)])
    order = np.argsort(z_step, kind="stable")    # file order: by step, as the reference writes
    return ReferenceLog(1.0, np.arange(n, dtype=np.uint32), u, np.arange(n, dtype=np.uint32),
                        g.init.copy(), z_step[order].astype(np.uint32),
                        z_lm[order].astype(np.uint32), z[order])


def write_log(path: str, log: ReferenceLog) -> None:
    """Writes records in the reference's text format (shortest round-trip repr of
    each double, so the reference's atof reads back exactly the same values)."""
    zs_by_step = {}
    for k in range(log.z_step.shape[0]):
        zs_by_step.setdefault(int(log.z_step[k]), []).append(k)
    r = lambda v: repr(float(v))  # noqa: E731
    with open(path, "w") as f:
        f.write(f"delta {r(log.delta)}\n")
        for s in range(log.x.shape[0]):
            f.write(f"u {int(log.u_step[s])} {r(log.u[s, 0])} {r(log.u[s, 1])}\n")
            f.write(f"x {int(log.x_step[s])} {r(log.x[s, 0])} {r(log.x[s, 1])} {r(log.x[s, 2])}\n")
            for k in zs_by_step.get(s, []):
                f.write(f"z {int(log.z_step[k])} {int(log.z_lm[k])} {r(log.z[k, 0])} {r(log.z[k, 1])}\n")


def _data_tool(*args) -> str:
    if not os.path.exists(abi.DATA_TOOL_PATH):
        raise FileNotFoundError(f"{abi.DATA_TOOL_PATH} is not built (python g-slam_on_gpu_and_fpga_b200/build.py)")
    r = subprocess.run([abi.DATA_TOOL_PATH, *map(str, args)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr.strip() or f"gslam-data failed ({r.returncode})")
    return r.stdout


def generate_citytrees(n_poses: int, path: str, seed: int = 42) -> str:
    """The reference's cityTrees generator (data/generate_citytrees.py) through the
    native gslam-data tool: the same file, byte for byte, for the same arguments.
    Returns the tool's summary lines."""
    return _data_tool("citytrees", int(n_poses), path, int(seed))


def convert_slampp(input_path: str, path: str, delta: float = 1.0) -> str:
    """The reference's SLAM++ converter (data/convert_slampp.py) through gslam-data."""
    return _data_tool("slampp", input_path, path, repr(float(delta)))


def landmark_log(n: int, seed: int = 0, density: float = 3.0e-3, strip: float = 20.0,
                 sensor_range: float = 8.5, max_obs: int = 10, block: int = 20,
                 sigma_range: float = 0.0, sigma_bearing: float = 0.0) -> ReferenceLog:
    """A reference-style landmark dataset on the same city-grid walk.

    Trees are scattered with the given density in a strip around the route and
    observed (range, bearing) from every ground-truth pose within sensor range,
    at most `max_obs` times each, so each tree seen k times yields C(k, 2)
    observation edges -- the clique structure of the reference's own cityTrees
    data (parameters as documented in its data/generate_citytrees.py:22-44).
    """
    from scipy.spatial import cKDTree

    g = city_grid(n, seed=seed, k_closures=0, block=block)
    rng = np.random.default_rng(seed + 104729)
    lo = g.gt[:, :2].min(0) - strip
    hi = g.gt[:, :2].max(0) + strip
    n_try = int((hi - lo).prod() * density)
    cand = lo + rng.random((n_try, 2)) * (hi - lo)
    tree = cKDTree(g.gt[:, :2])
    near = tree.query(cand, k=1)[0] <= strip
    lms = cand[near]
    # observations in step order; each tree at most max_obs times
    lm_tree = cKDTree(lms)
    hits = lm_tree.query_ball_point(g.gt[:, :2], r=sensor_range)
    count = np.zeros(lms.shape[0], np.int64)
    z_step, z_lm, z = [], [], []
    first_id = 2 * n * max_obs + 6  # above any observation count (see to_reference_log)
    for s in range(n):
        for li in sorted(hits[s]):
            if count[li] >= max_obs:
                continue
            d = lms[li] - g.gt[s, :2]
            r = float(np.hypot(d[0], d[1])) + (rng.normal() * sigma_range if sigma_range else 0.0)
            b = float(_wrap(np.arctan2(d[1], d[0]) - g.gt[s, 2]
                            + (rng.normal() * sigma_bearing if sigma_bearing else 0.0)))
            z_step.append(s)
            z_lm.append(first_id + li)
            z.append((r, b))
            count[li] += 1
    odo = g.meas[: g.n_odom]
    u = np.zeros((n, 2))
    u[1:, 0] = np.hypot(odo[:, 0], odo[:, 1])
    u[1:, 1] = odo[:, 2]
    return ReferenceLog(1.0, np.arange(n, dtype=np.uint32), u, np.arange(n, dtype=np.uint32),
                        g.init.copy(), np.asarray(z_step, np.uint32), np.asarray(z_lm, np.uint32),
                        np.asarray(z, np.float64).reshape(-1, 2))
