"""PoseGraph: a pose graph resident on one GPU, driven through libgslam's C ABI.

Mirrors the reference's per-round path (src/cpu_pcg_fp64/GSLAM.c:55-139):
`round()` linearises every edge, assembles Omega / xi, solves Omega dx = xi with
block-Jacobi PCG and adds dx to the poses, all on the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi


@dataclass
class RoundStats:
    iterations: int
    refinements: int
    reason: int
    rel_residual: float
    diff: float
    solve_ms: float = 0.0
    round_ms: float = 0.0


@dataclass
class ReferenceLog:
    """Records of a reference log file (data/README.md: delta, u, x, z lines)."""
    delta: float
    u_step: np.ndarray
    u: np.ndarray       # [n_u, 2] nu, omega
    x_step: np.ndarray
    x: np.ndarray       # [n_x, 3]
    z_step: np.ndarray
    z_lm: np.ndarray
    z: np.ndarray       # [n_z, 2] range, bearing

    @property
    def n_poses(self) -> int:
        return int(self.x.shape[0])

    @property
    def dim(self) -> int:
        return 3 * int(self.u.shape[0])


def read_log(path: str) -> ReferenceLog:
    """Parses a log with libgslam's reader (the reference's read_data semantics)."""
    L = abi.lib()
    p = C.POINTER(abi.LogDesc)()
    abi.check(L.gslam_read_log(path.encode(), C.byref(p)))
    d = p.contents

    def arr(ptr, n, dtype, cols=1):
        if n == 0:
            return np.zeros((0, cols) if cols > 1 else 0, dtype)
        a = np.ctypeslib.as_array(ptr, shape=(n * cols,)).astype(dtype, copy=True)
        return a.reshape(n, cols) if cols > 1 else a

    out = ReferenceLog(d.delta, arr(d.u_step, d.n_u, np.uint32), arr(d.u, d.n_u, np.float64, 2),
                       arr(d.x_step, d.n_x, np.uint32), arr(d.x, d.n_x, np.float64, 3),
                       arr(d.z_step, d.n_z, np.uint32), arr(d.z_lm, d.n_z, np.uint32),
                       arr(d.z, d.n_z, np.float64, 2))
    L.gslam_free_log(p)
    return out


class PoseGraph:
    """Owns one gslam_graph handle."""

    def __init__(self, handle: int, n_poses: int, factors: str, keep=None):
        self._h = C.c_void_p(handle)
        self.n_poses = n_poses
        self.factors = factors
        self._keep = keep

    # ---- construction ----
    @classmethod
    def from_reference(cls, poses, controls, delta: float, lam: float, obs_step, obs_landmark,
                       obs, mns=None, **opts) -> "PoseGraph":
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 3)
        controls = np.ascontiguousarray(controls, np.float64).reshape(-1, 2)
        obs_step = np.ascontiguousarray(obs_step, np.uint32)
        obs_landmark = np.ascontiguousarray(obs_landmark, np.uint32)
        obs = np.ascontiguousarray(obs, np.float64).reshape(-1, 2)
        if controls.shape[0] != poses.shape[0]:
            raise ValueError("one control per pose (row 0 unused)")
        d = abi.ReferenceGraphDesc()
        d.n_poses = poses.shape[0]
        d.poses = abi.ptr(poses)
        d.controls = abi.ptr(controls)
        d.delta = float(delta)
        d.lam = float(lam)
        m = None
        if mns is not None:
            m = np.ascontiguousarray(mns, np.float64)
            d.mns = abi.ptr(m)
        d.n_obs = obs_step.shape[0]
        d.obs_step = abi.ptr(obs_step, C.c_uint32)
        d.obs_landmark = abi.ptr(obs_landmark, C.c_uint32)
        d.obs = abi.ptr(obs)
        o = abi.default_opts(**opts)
        h = C.c_void_p()
        abi.check(abi.lib().gslam_create_reference(C.byref(d), C.byref(o), C.byref(h)))
        return cls(h.value, poses.shape[0], "reference")

    @classmethod
    def from_log(cls, log: ReferenceLog, lam: float, **opts) -> "PoseGraph":
        return cls.from_reference(log.x, log.u, log.delta, lam, log.z_step, log.z_lm, log.z, **opts)

    @classmethod
    def from_se2(cls, poses, edge_i, edge_j, meas, log_w, lam: float = 1.0, anchor: float = 1e6,
                 **opts) -> "PoseGraph":
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 3)
        ei = np.ascontiguousarray(edge_i, np.uint32)
        ej = np.ascontiguousarray(edge_j, np.uint32)
        meas = np.ascontiguousarray(meas, np.float64).reshape(-1, 3)
        log_w = np.ascontiguousarray(log_w, np.float64).reshape(-1, 3)
        d = abi.SE2GraphDesc()
        d.n_poses = poses.shape[0]
        d.poses = abi.ptr(poses)
        d.n_edges = ei.shape[0]
        d.edge_i = abi.ptr(ei, C.c_uint32)
        d.edge_j = abi.ptr(ej, C.c_uint32)
        d.meas = abi.ptr(meas)
        d.log_w = abi.ptr(log_w)
        d.lam = float(lam)
        d.anchor = float(anchor)
        o = abi.default_opts(**opts)
        h = C.c_void_p()
        abi.check(abi.lib().gslam_create_se2(C.byref(d), C.byref(o), C.byref(h)))
        return cls(h.value, poses.shape[0], "se2")

    # ---- lifetime ----
    def close(self) -> None:
        if self._h is not None and self._h.value:
            abi.lib().gslam_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- options / sizes ----
    def set_opts(self, **opts) -> None:
        o = abi.default_opts(**opts)
        abi.check(abi.lib().gslam_set_opts(self._h, C.byref(o)))

    def sizes(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        abi.check(abi.lib().gslam_sizes(self._h, *[C.byref(x) for x in v]))
        return dict(n_poses=v[0].value, n_edges=v[1].value, nnzb=v[2].value, nnz=v[3].value)

    # ---- state ----
    @property
    def poses(self) -> np.ndarray:
        out = np.zeros((self.n_poses, 3))
        abi.check(abi.lib().gslam_get_poses(self._h, abi.ptr(out)))
        return out

    @poses.setter
    def poses(self, value) -> None:
        v = np.ascontiguousarray(value, np.float64).reshape(self.n_poses, 3)
        abi.check(abi.lib().gslam_set_poses(self._h, abi.ptr(v)))

    # ---- rounds ----
    def round(self) -> RoundStats:
        st = abi.SolveStats()
        abi.check(abi.lib().gslam_round(self._h, C.byref(st)))
        return RoundStats(st.iterations, st.refinements, st.reason, st.rel_residual, st.diff, st.solve_ms,
                          st.round_ms)

    def round_io(self, poses_in=None, poses_out=None) -> RoundStats:
        """One round with host input and output (gslam_round_io): poses_in (N x 3 float64,
        or None to keep the device poses) in, the round, the new poses into poses_out (N x 3
        float64, or None); one wait. Pass page-locked arrays (e.g. torch pin_memory) for
        asynchronous copies."""
        dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        for a in (poses_in, poses_out):
            if a is not None and (a.dtype != np.float64 or a.shape != (self.n_poses, 3) or not a.flags.c_contiguous):
                raise ValueError("poses must be a C-contiguous (n_poses, 3) float64 array")
        st = abi.SolveStats()
        abi.check(abi.lib().gslam_round_io(self._h, dp(poses_in), dp(poses_out), C.byref(st)))
        return RoundStats(st.iterations, st.refinements, st.reason, st.rel_residual, st.diff, st.solve_ms,
                          st.round_ms)

    def stream(self) -> int:
        """The cudaStream_t (as an int) all work on this graph runs on."""
        s = C.c_void_p()
        abi.check(abi.lib().gslam_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def run(self, max_rounds: int):
        diffs = np.zeros(max(max_rounds, 1))
        n = C.c_int(0)
        abi.check(abi.lib().gslam_run(self._h, int(max_rounds), abi.ptr(diffs), C.byref(n)))
        return diffs[:n.value]

    def linearise(self) -> None:
        abi.check(abi.lib().gslam_linearise(self._h))

    def assemble(self) -> None:
        abi.check(abi.lib().gslam_assemble(self._h))

    def assemble_from_edges(self, d_blocks_ptr: int) -> None:
        abi.check(abi.lib().gslam_assemble_from_edges(self._h, C.c_void_p(d_blocks_ptr)))

    def solve(self) -> RoundStats:
        st = abi.SolveStats()
        abi.check(abi.lib().gslam_solve(self._h, C.byref(st)))
        return RoundStats(st.iterations, st.refinements, st.reason, st.rel_residual, st.diff, st.solve_ms)

    def update(self) -> float:
        d = C.c_double()
        abi.check(abi.lib().gslam_update(self._h, C.byref(d)))
        return d.value

    # ---- read-back ----
    def edge_blocks(self) -> np.ndarray:
        n = self.sizes()["n_edges"]
        out = np.zeros((n, 42))
        abi.check(abi.lib().gslam_get_edge_blocks(self._h, abi.ptr(out)))
        return out

    def csr(self):
        s = self.sizes()
        dim = 3 * self.n_poses
        rp = np.zeros(dim + 1, np.int32)
        ci = np.zeros(s["nnz"], np.int32)
        va = np.zeros(s["nnz"])
        xi = np.zeros(dim)
        abi.check(abi.lib().gslam_get_csr(self._h, abi.ptr(rp, C.c_int), abi.ptr(ci, C.c_int),
                                          abi.ptr(va), abi.ptr(xi)))
        return rp, ci, va, xi

    def dx(self) -> np.ndarray:
        out = np.zeros(3 * self.n_poses)
        abi.check(abi.lib().gslam_get_dx(self._h, abi.ptr(out)))
        return out

    def cost(self, per_edge: bool = False):
        """Round cost at the current poses (reference-factor graphs); with per_edge,
        (total, terms in the reference's edge order)."""
        tot = C.c_double()
        n = self.sizes()["n_edges"] if per_edge else 0
        terms = np.zeros(max(n, 1)) if per_edge else None
        abi.check(abi.lib().gslam_cost(self._h, C.byref(tot), abi.ptr(terms) if per_edge else None))
        return (tot.value, terms[:n]) if per_edge else tot.value

    def landmark_map(self):
        """(landmark ids, positions [L, 2]) at the current poses (reference-factor graphs)."""
        n = C.c_uint32()
        abi.check(abi.lib().gslam_landmark_map(self._h, C.byref(n), None, None))
        ids = np.zeros(n.value, np.uint32)
        ms = np.zeros((max(n.value, 1), 2))
        abi.check(abi.lib().gslam_landmark_map(self._h, C.byref(n), abi.ptr(ids, C.c_uint32), abi.ptr(ms)))
        return ids, ms[:n.value]

    # ---- differentiation (SE(2) graphs) ----
    def set_weights(self, lam: float, log_w=None) -> None:
        """New lambda and (optionally) per-edge log information weights [E, 3]."""
        lw = None if log_w is None else np.ascontiguousarray(log_w, np.float64).reshape(-1)
        abi.check(abi.lib().gslam_set_se2_weights(self._h, float(lam),
                                                  abi.ptr(lw) if lw is not None else None))

    def adjoint(self, dL_dposes):
        """Implicit-function adjoint at the current (converged) poses: returns
        (dL/dlambda, dL/dlog_w [E, 3], mu [N, 3], RoundStats of the adjoint solve)."""
        g = np.ascontiguousarray(dL_dposes, np.float64).reshape(self.n_poses, 3)
        n_e = self.sizes()["n_edges"]
        dlw = np.zeros((n_e, 3))
        mu = np.zeros((self.n_poses, 3))
        dlam = C.c_double()
        st = abi.SolveStats()
        abi.check(abi.lib().gslam_adjoint(self._h, abi.ptr(g), C.byref(dlam), abi.ptr(dlw), abi.ptr(mu),
                                          C.byref(st)))
        return dlam.value, dlw, mu, RoundStats(st.iterations, st.refinements, st.reason, st.rel_residual,
                                               st.diff, st.solve_ms)

    def diag_inv(self) -> np.ndarray:
        out = np.zeros((self.n_poses, 9))
        abi.check(abi.lib().gslam_get_diag_inv(self._h, abi.ptr(out)))
        return out

    def spmv(self, d_x: int, d_y: int) -> None:
        """y = Omega x on device pointers (3N doubles each, original order)."""
        abi.check(abi.lib().gslam_spmv(self._h, C.c_void_p(d_x), C.c_void_p(d_y)))

    def spmv_bench(self, fp32: bool, reps: int, n_copies: int = 1) -> float:
        """Mean device ms per SpMV over `reps` graph-replayed launches (see gslam.h)."""
        ms = C.c_float()
        abi.check(abi.lib().gslam_spmv_bench(self._h, int(fp32), int(reps), int(n_copies), C.byref(ms)))
        return ms.value

    def spmv_bytes(self, fp32: bool) -> int:
        b = C.c_int64()
        abi.check(abi.lib().gslam_spmv_bytes(self._h, int(fp32), C.byref(b)))
        return b.value


class PoseGraphBatch(PoseGraph):
    """Many independent SE(2) graphs on one handle (gslam_create_se2_batch): one
    Gauss-Newton round of every graph per `round()`, their linear solves in one
    persistent launch with per-graph scalars. Poses of graph q are
    `poses[offsets[q] : offsets[q] + sizes[q]]` of the concatenation."""

    @classmethod
    def from_se2_list(cls, graphs, lams, anchors=1e6, **opts) -> "PoseGraphBatch":
        """graphs: objects with .init / .edge_i / .edge_j / .meas / .log_w (synth.CityGrid),
        lams: one lambda per graph (or a scalar), anchors likewise."""
        n = len(graphs)
        lams = np.broadcast_to(np.asarray(lams, np.float64), (n,))
        anchors = np.broadcast_to(np.asarray(anchors, np.float64), (n,))
        keep, descs = [], (abi.SE2GraphDesc * n)()
        for q, cg in enumerate(graphs):
            poses = np.ascontiguousarray(cg.init, np.float64).reshape(-1, 3)
            ei = np.ascontiguousarray(cg.edge_i, np.uint32)
            ej = np.ascontiguousarray(cg.edge_j, np.uint32)
            meas = np.ascontiguousarray(cg.meas, np.float64).reshape(-1, 3)
            log_w = np.ascontiguousarray(cg.log_w, np.float64).reshape(-1, 3)
            keep.append((poses, ei, ej, meas, log_w))
            d = descs[q]
            d.n_poses = poses.shape[0]
            d.poses = abi.ptr(poses)
            d.n_edges = ei.shape[0]
            d.edge_i = abi.ptr(ei, C.c_uint32)
            d.edge_j = abi.ptr(ej, C.c_uint32)
            d.meas = abi.ptr(meas)
            d.log_w = abi.ptr(log_w)
            d.lam = float(lams[q])
            d.anchor = float(anchors[q])
        o = abi.default_opts(**opts)
        h = C.c_void_p()
        abi.check(abi.lib().gslam_create_se2_batch(descs, n, C.byref(o), C.byref(h)))
        off = (C.c_uint32 * (n + 1))()
        cnt = C.c_uint32()
        abi.check(abi.lib().gslam_batch_layout(h, C.byref(cnt), off))
        self = cls(h.value, int(off[n]), "se2-batch")
        self.offsets = np.array(off[:n], np.int64)
        self.sizes_real = np.array([k[0].shape[0] for k in keep], np.int64)
        self.init_poses = self.poses      # the concatenated initial guess (padding at 0)
        return self

    @property
    def n_graphs(self) -> int:
        return len(self.offsets)

    def round_all(self):
        """One round of every graph; a RoundStats per graph."""
        st = (abi.SolveStats * self.n_graphs)()
        abi.check(abi.lib().gslam_batch_round(self._h, st))
        return [RoundStats(s.iterations, s.refinements, s.reason, s.rel_residual, s.diff, s.solve_ms,
                           s.round_ms) for s in st]

    def graph_poses(self, q: int, poses=None) -> np.ndarray:
        p = self.poses if poses is None else poses
        return p[self.offsets[q]:self.offsets[q] + self.sizes_real[q]]
