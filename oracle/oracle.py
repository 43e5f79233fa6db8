"""Python access to the CPU checker: the C restatement (liboracle.so) and the
reference program compiled from its own sources (_ref/libgslam_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MNS = np.array([0.19, 0.001, 0.13, 0.2], dtype=np.float64)

_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/ when the reference sources are present)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_obs_edge_pairs.restype = C.c_long
        L.or_csr_nnz.restype = C.c_long
        L.or_norm_glibc.restype = C.c_double
        L.or_norm_cr.restype = C.c_double
        L.or_position_loss_dd.restype = C.c_double
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libgslam_ref.so"))


# --------------------------------------------------------------------------
# log files
# --------------------------------------------------------------------------

class Graph:
    """Records of one reference log: controls u, initial poses x, observations z."""

    def __init__(self, delta, u_step, u, x_step, x, z_step, z_lm, z_rb):
        self.delta = float(delta)
        self.u_step = np.ascontiguousarray(u_step, dtype=np.uint32)
        self.u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 2)
        self.x_step = np.ascontiguousarray(x_step, dtype=np.uint32)
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        self.z_step = np.ascontiguousarray(z_step, dtype=np.uint32)
        self.z_lm = np.ascontiguousarray(z_lm, dtype=np.uint32)
        self.z_rb = np.ascontiguousarray(z_rb, dtype=np.float64).reshape(-1, 2)

    @property
    def z(self):
        return self.z_rb

    @property
    def n_poses(self):
        return self.x.shape[0]

    @property
    def dim(self):
        return 3 * self.u.shape[0]


def read_log(path: str) -> Graph:
    L = lib()
    d = C.c_double(0.0)
    nu, nx, nz = C.c_uint(), C.c_uint(), C.c_uint()
    nul = C.POINTER(C.c_uint)()
    nuld = C.POINTER(C.c_double)()
    rc = L.or_read_log(path.encode(), C.byref(d), C.byref(nu), nul, nuld, 0, C.byref(nx), nul,
                       nuld, 0, C.byref(nz), nul, nul, nuld, 0)
    if rc != 0:
        raise IOError(f"cannot read {path} ({rc})")
    u_step = np.zeros(nu.value, np.uint32); u = np.zeros((nu.value, 2))
    x_step = np.zeros(nx.value, np.uint32); x = np.zeros((nx.value, 3))
    z_step = np.zeros(nz.value, np.uint32); z_lm = np.zeros(nz.value, np.uint32)
    z_rb = np.zeros((nz.value, 2))
    rc = L.or_read_log(path.encode(), C.byref(d), C.byref(nu), _p(u_step, C.c_uint), _p(u, C.c_double),
                       len(u_step), C.byref(nx), _p(x_step, C.c_uint), _p(x, C.c_double), len(x_step),
                       C.byref(nz), _p(z_step, C.c_uint), _p(z_lm, C.c_uint), _p(z_rb, C.c_double),
                       len(z_step))
    if rc != 0:
        raise IOError(f"cannot read {path} ({rc})")
    return Graph(d.value, u_step, u, x_step, x, z_step, z_lm, z_rb)


# --------------------------------------------------------------------------
# restated path
# --------------------------------------------------------------------------

def obs_pairs(z_lm):
    L = lib()
    z_lm = np.ascontiguousarray(z_lm, dtype=np.uint32)
    n = L.or_obs_edge_pairs(len(z_lm), _p(z_lm, C.c_uint), None, None, 0)
    pj = np.zeros(max(n, 1), np.uint32); pk = np.zeros(max(n, 1), np.uint32)
    L.or_obs_edge_pairs(len(z_lm), _p(z_lm, C.c_uint), _p(pj, C.c_uint), _p(pk, C.c_uint), n)
    return pj[:n], pk[:n]


def linearise(g: Graph, poses, lam: float, cr: bool = True, pairs=None):
    """All edges of one round in reference order -> (t1, t2, blocks[E, 42])."""
    L = lib()
    poses = np.ascontiguousarray(poses, dtype=np.float64)
    pj, pk = pairs if pairs is not None else obs_pairs(g.z_lm)
    pj = np.ascontiguousarray(pj, np.uint32); pk = np.ascontiguousarray(pk, np.uint32)
    n_obs = len(pj)
    E = n_obs + max(g.n_poses - 1, 0)
    t1 = np.zeros(max(E, 1), np.uint32); t2 = np.zeros(max(E, 1), np.uint32)
    blocks = np.zeros((max(E, 1), 42))
    rc = L.or_linearise(int(cr), g.n_poses, _p(poses, C.c_double), _p(g.u, C.c_double),
                        C.c_double(g.delta), C.c_double(lam), _p(MNS, C.c_double),
                        _p(g.z_step, C.c_uint), _p(g.z_rb, C.c_double), C.c_long(n_obs),
                        _p(pj, C.c_uint), _p(pk, C.c_uint), _p(t1, C.c_uint), _p(t2, C.c_uint),
                        _p(blocks, C.c_double))
    if rc != 0:
        raise ValueError("observation step out of range")
    return t1[:E], t2[:E], blocks[:E]


def round_cost(g: Graph, poses, lam: float, cr: bool = True):
    """(total, per-edge terms in reference edge order) of the round cost at `poses`
    (GSLAM.c:74-87 with the intended dimensions, reset every round)."""
    L = lib()
    poses = np.ascontiguousarray(poses, dtype=np.float64)
    pj, pk = obs_pairs(g.z_lm)
    pj = np.ascontiguousarray(pj, np.uint32); pk = np.ascontiguousarray(pk, np.uint32)
    n_obs = len(pj)
    E = n_obs + max(g.n_poses - 1, 0)
    per = np.zeros(max(E, 1))
    tot = C.c_double(0.0)
    rc = L.or_round_cost(int(cr), g.n_poses, _p(poses, C.c_double), _p(g.u, C.c_double),
                         C.c_double(g.delta), C.c_double(lam), _p(MNS, C.c_double),
                         _p(g.z_step, C.c_uint), _p(g.z_rb, C.c_double), C.c_long(n_obs),
                         _p(pj, C.c_uint), _p(pk, C.c_uint), _p(per, C.c_double), C.byref(tot))
    if rc != 0:
        raise ValueError("observation step out of range")
    return tot.value, per[:E]


def csr_build(dim: int, t1, t2, blocks):
    L = lib()
    t1 = np.ascontiguousarray(t1, np.uint32); t2 = np.ascontiguousarray(t2, np.uint32)
    blocks = np.ascontiguousarray(blocks, np.float64)
    E = len(t1)
    nnz = L.or_csr_nnz(dim, C.c_long(E), _p(t1, C.c_uint), _p(t2, C.c_uint))
    row_ptr = np.zeros(dim + 1, np.int32); col_idx = np.zeros(nnz, np.int32)
    values = np.zeros(nnz); xi = np.zeros(dim)
    rc = L.or_csr_build(dim, C.c_long(E), _p(t1, C.c_uint), _p(t2, C.c_uint), _p(blocks, C.c_double),
                        _p(row_ptr, C.c_int), _p(col_idx, C.c_int), _p(values, C.c_double),
                        _p(xi, C.c_double))
    if rc != 0:
        raise ValueError("edge pose index out of range")
    return row_ptr, col_idx, values, xi


def csr_build_anchor(dim: int, t1, t2, blocks, anchor: float):
    L = lib()
    t1 = np.ascontiguousarray(t1, np.uint32); t2 = np.ascontiguousarray(t2, np.uint32)
    blocks = np.ascontiguousarray(blocks, np.float64)
    E = len(t1)
    nnz = L.or_csr_nnz(dim, C.c_long(E), _p(t1, C.c_uint), _p(t2, C.c_uint))
    row_ptr = np.zeros(dim + 1, np.int32); col_idx = np.zeros(nnz, np.int32)
    values = np.zeros(nnz); xi = np.zeros(dim)
    rc = L.or_csr_build_anchor(dim, C.c_long(E), _p(t1, C.c_uint), _p(t2, C.c_uint),
                               _p(blocks, C.c_double), C.c_double(anchor), _p(row_ptr, C.c_int),
                               _p(col_idx, C.c_int), _p(values, C.c_double), _p(xi, C.c_double))
    if rc != 0:
        raise ValueError("edge pose index out of range")
    return row_ptr, col_idx, values, xi


def se2_info(log_w):
    """exp(log_w) with the C library's exp (as libgslam computes it at creation)."""
    import math
    lw = np.asarray(log_w, np.float64)
    return np.array([math.exp(v) for v in lw.ravel()]).reshape(lw.shape)


def se2_linearise(poses, ei, ej, meas, log_w, lam: float):
    """SE(2) between-factor blocks [E, 42] and residuals [E, 3] (CR trig)."""
    L = lib()
    poses = np.ascontiguousarray(poses, np.float64)
    ei = np.ascontiguousarray(ei, np.uint32); ej = np.ascontiguousarray(ej, np.uint32)
    meas = np.ascontiguousarray(meas, np.float64)
    info = np.ascontiguousarray(se2_info(log_w))
    E = len(ei)
    blocks = np.zeros((max(E, 1), 42)); errs = np.zeros((max(E, 1), 3))
    L.or_se2_linearise(C.c_long(E), _p(ei, C.c_uint), _p(ej, C.c_uint), _p(poses, C.c_double),
                       _p(meas, C.c_double), _p(info, C.c_double), C.c_double(lam),
                       _p(blocks, C.c_double), _p(errs, C.c_double))
    return blocks[:E], errs[:E]


def spmv(row_ptr, col_idx, values, p):
    L = lib()
    dim = len(row_ptr) - 1
    p = np.ascontiguousarray(p, np.float64); q = np.zeros(dim)
    L.or_spmv(dim, _p(row_ptr, C.c_int), _p(col_idx, C.c_int), _p(values, C.c_double),
              _p(p, C.c_double), _p(q, C.c_double))
    return q


def diag_inv(row_ptr, col_idx, values):
    L = lib()
    dim = len(row_ptr) - 1
    out = np.zeros((dim // 3, 9))
    L.or_diag_inv(dim, _p(row_ptr, C.c_int), _p(col_idx, C.c_int), _p(values, C.c_double),
                  _p(out, C.c_double))
    return out


def pcg(row_ptr, col_idx, values, b, tol: float = 1e-6, max_iter: int = 500):
    L = lib()
    dim = len(row_ptr) - 1
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(dim)
    it = C.c_int(0); rn = C.c_double(0.0)
    L.or_pcg(dim, _p(row_ptr, C.c_int), _p(col_idx, C.c_int), _p(values, C.c_double),
             _p(b, C.c_double), _p(x, C.c_double), C.c_double(tol), int(max_iter), C.byref(it),
             C.byref(rn))
    return x, it.value, rn.value


def run(g: Graph, lam: float, rounds: int, cr: bool = False, tol: float = 1e-6,
        max_iter: int = 500):
    """The reference GN loop (use_diff = 1) -> (poses, diffs, pcg_iters)."""
    L = lib()
    poses = g.x.copy()
    diffs = np.zeros(max(rounds, 1)); its = np.zeros(max(rounds, 1), np.int32)
    n = L.or_run(int(cr), g.n_poses, _p(poses, C.c_double), _p(g.u, C.c_double),
                 C.c_double(g.delta), C.c_double(lam), len(g.z_lm), _p(g.z_step, C.c_uint),
                 _p(g.z_lm, C.c_uint), _p(g.z_rb, C.c_double), int(rounds), C.c_double(tol),
                 int(max_iter), _p(diffs, C.c_double), _p(its, C.c_int))
    if n < 0:
        raise ValueError("bad graph")
    return poses, diffs[:n], its[:n]


def norm_glibc(v) -> float:
    """The reference's norm (MatrixOps.c:4-16: sqrt of pow(v_i, 2.0) summed in order)."""
    v = np.ascontiguousarray(v, np.float64)
    return lib().or_norm_glibc(_p(v, C.c_double), len(v))


def run_dense_gj(g: Graph, lam: float, max_rounds: int = 200):
    """The reference's dense Gauss-Jordan program (src/cpu_gj_fp64/GSLAM.c:89-231, use_diff
    = 1): each round Omega and xi densely (the anchor, then every edge in make_edges order:
    the CSR assembly's values), Omega^-1 by Gauss-Jordan without pivoting
    (MatrixOps.c:29-91; the reference program calls its SYCL-parallel twin), dx = Omega^-1 xi
    summed in index order from 0.0 (dot -> vec_dot), poses += dx; it stops at
    diff < 0.01 or when the even- or the odd-numbered rounds' diff has not improved for 10
    of them (GSLAM.c:218-230). Returns (poses, diffs)."""
    poses = g.x.copy()
    diffs = []
    best = [1e30, 1e30]
    stale = [0, 0]
    for n in range(max_rounds):
        t1, t2, ob = linearise(g, poses, lam, cr=False)
        rp, ci, va, xi = csr_build(g.dim, t1, t2, ob)
        inv, rc = gj_inverse(dense_from_csr(rp, ci, va))
        if rc != 0:
            raise ValueError("zero pivot")
        dx = np.zeros(g.dim)
        for j in range(g.dim):          # every row sums its products in column order
            dx = dx + inv[:, j] * xi[j]
        poses = poses + dx.reshape(-1, 3)
        diff = norm_glibc(dx) / np.sqrt(g.dim)
        diffs.append(diff)
        if diff < 0.01:
            break
        k = n % 2
        if diff < best[k]:
            best[k], stale[k] = diff, 0
        else:
            stale[k] += 1
            if stale[k] >= 10:
                break
    return poses, np.array(diffs)


def se2_rhs_dd(p_hi, p_lo, ei, ej, meas, info):
    """xi = -sum J^T Lambda e at double-double poses, in double-double (se2_dd.c):
    (xi_hi, xi_lo), each [3N]. info = Lambda's diagonal per edge [E, 3], lambda folded in."""
    L = lib()
    p_hi = np.ascontiguousarray(p_hi, np.float64).reshape(-1)
    p_lo = np.ascontiguousarray(p_lo, np.float64).reshape(-1)
    ei = np.ascontiguousarray(ei, np.uint32); ej = np.ascontiguousarray(ej, np.uint32)
    meas = np.ascontiguousarray(meas, np.float64); info = np.ascontiguousarray(info, np.float64)
    xh = np.zeros(len(p_hi)); xl = np.zeros(len(p_hi))
    rc = L.or_se2_rhs_dd(C.c_long(len(p_hi) // 3), C.c_long(len(ei)), _p(ei, C.c_uint), _p(ej, C.c_uint),
                         _p(p_hi, C.c_double), _p(p_lo, C.c_double), _p(meas, C.c_double),
                         _p(info, C.c_double), _p(xh, C.c_double), _p(xl, C.c_double))
    if rc != 0:
        raise ValueError("edge pose index out of range")
    return xh, xl


def dd_add_vec(hi, lo, d):
    """(hi + lo) += d in place (double-double, renormalised); hi, lo contiguous float64."""
    d = np.ascontiguousarray(d, np.float64).reshape(-1)
    lib().or_dd_add_vec(C.c_long(len(d)), _p(hi, C.c_double), _p(lo, C.c_double), _p(d, C.c_double))


def position_loss_dd(p_hi, p_lo, target):
    """sum (x - tx)^2 + (y - ty)^2 over poses, in double-double: (hi, lo)."""
    p_hi = np.ascontiguousarray(p_hi, np.float64).reshape(-1)
    p_lo = np.ascontiguousarray(p_lo, np.float64).reshape(-1)
    target = np.ascontiguousarray(target, np.float64).reshape(-1)
    lo = C.c_double(0.0)
    hi = lib().or_position_loss_dd(C.c_long(len(p_hi) // 3), _p(p_hi, C.c_double), _p(p_lo, C.c_double),
                                   _p(target, C.c_double), C.byref(lo))
    return hi, lo.value


def sincos_dd(x_hi: float, x_lo: float = 0.0):
    """sin and cos of x_hi + x_lo as (hi, lo) pairs (se2_dd.c)."""
    v = [C.c_double() for _ in range(4)]
    lib().or_sincos_dd(C.c_double(x_hi), C.c_double(x_lo), *[C.byref(a) for a in v])
    return (v[0].value, v[1].value), (v[2].value, v[3].value)


def cr_sincos(x: float):
    L = lib()
    s = C.c_double(); c = C.c_double()
    L.or_cr_sincos(C.c_double(x), C.byref(s), C.byref(c))
    return s.value, c.value


def landmark_groups(z_lm):
    """Landmarks in order of first appearance in the z list, each with its z indices in
    z-list order (the order of make_edges' landmark_keys_zlist, GSLAM.c:246-261)."""
    z_lm = np.asarray(z_lm)
    first = {}
    for i, lm in enumerate(z_lm.tolist()):
        first.setdefault(lm, []).append(i)
    ids = list(first)                      # dict keeps first-appearance order
    ptr = np.zeros(len(ids) + 1, np.int64)
    members = []
    for k, lm in enumerate(ids):
        members += first[lm]
        ptr[k + 1] = len(members)
    return np.array(ids, np.uint32), ptr, np.array(members, np.uint32)


def landmark_map(g: Graph, poses, cr: bool = True):
    """(landmark ids, positions [L, 2]) after a run, as GSLAM.c:141-196 computes them."""
    L = lib()
    ids, ptr, members = landmark_groups(g.z_lm)
    poses = np.ascontiguousarray(poses, np.float64)
    ms = np.zeros((max(len(ids), 1), 2))
    L.or_landmark_map(int(cr), len(ids), _p(ptr, C.c_long), _p(members, C.c_uint), _p(g.z_step, C.c_uint),
                      _p(g.z_rb, C.c_double), _p(poses, C.c_double), _p(ms, C.c_double))
    return ids, ms[:len(ids)]


def gj_inverse(a):
    L = lib()
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    out = np.zeros_like(a)
    rc = L.or_gj_inverse(n, _p(a, C.c_double), _p(out, C.c_double))
    return out, rc


def dense_from_csr(row_ptr, col_idx, values):
    dim = len(row_ptr) - 1
    A = np.zeros((dim, dim))
    for i in range(dim):
        A[i, col_idx[row_ptr[i]:row_ptr[i + 1]]] = values[row_ptr[i]:row_ptr[i + 1]]
    return A


# --------------------------------------------------------------------------
# the reference program itself (compiled from its sources into _ref/)
# --------------------------------------------------------------------------

class _U(C.Structure):
    _fields_ = [("step", C.c_uint), ("nu", C.c_double), ("omega", C.c_double)]


class _HX(C.Structure):
    _fields_ = [("step", C.c_uint), ("hat_x", C.c_double * 3)]


class _Z(C.Structure):
    _fields_ = [("step", C.c_uint), ("landmark_id", C.c_uint), ("z", C.c_double * 2)]


class _Edge(C.Structure):
    _fields_ = [("t1", C.c_uint), ("t2", C.c_uint), ("hat_x1", _HX), ("hat_x2", _HX),
                ("z1", _Z), ("z2", _Z), ("Omega", C.c_double * 9), ("ul", C.c_double * 9),
                ("ur", C.c_double * 9), ("bl", C.c_double * 9), ("br", C.c_double * 9),
                ("xi_u", C.c_double * 3), ("xi_b", C.c_double * 3), ("lam", C.c_double),
                ("hat_e", C.c_double * 2)]


class _LKZ(C.Structure):
    _fields_ = [("landmark_id", C.c_uint), ("z", _Z)]


class _MapEdge(C.Structure):
    _fields_ = [("x", _HX), ("z", _Z), ("m", C.c_double * 2), ("Omega", C.c_double * 4), ("xi", C.c_double * 2)]


class _CSR(C.Structure):
    _fields_ = [("row_ptr", C.POINTER(C.c_int)), ("col_idx", C.POINTER(C.c_int)),
                ("values", C.POINTER(C.c_double)), ("dim", C.c_int), ("nnz", C.c_int)]


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libgslam_ref.so")
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError("reference build absent (oracle/_ref)")
        R = C.CDLL(path)
        R.ObsEdge_create.argtypes = [C.POINTER(_Edge), _Z, _Z, C.POINTER(_HX), C.POINTER(C.c_double)]
        R.ObsEdge_create.restype = C.POINTER(_Edge)
        R.MotionEdge_create.argtypes = [C.POINTER(_Edge), C.c_uint, C.c_uint, C.POINTER(_HX),
                                        C.POINTER(_U), C.c_double, C.c_double, C.POINTER(C.c_double)]
        R.MotionEdge_create.restype = C.POINTER(_Edge)
        R.make_edges.argtypes = [C.POINTER(_HX), C.c_uint, C.POINTER(_Z), C.c_uint, C.POINTER(_Edge),
                                 C.POINTER(C.c_uint), C.POINTER(_LKZ), C.POINTER(C.c_uint)]
        R.build_csr_from_edges.argtypes = [C.POINTER(_Edge), C.c_uint, C.c_uint, C.POINTER(_CSR),
                                           C.POINTER(C.c_double)]
        R.pcg_solve_sparse.argtypes = [C.POINTER(C.c_double), C.POINTER(_CSR),
                                       C.POINTER(C.c_double), C.c_uint]
        R.free_csr.argtypes = [C.POINTER(_CSR)]
        R.MapEdge_create.argtypes = [C.POINTER(_MapEdge), _Z, _Z, C.POINTER(_HX), C.POINTER(C.c_double)]
        R.MapEdge_create.restype = C.POINTER(_MapEdge)
        R.vec_mean.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint, C.c_uint]
        R.state_transition.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_uint, _HX]
        R.tra.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint, C.c_uint]
        R.sub.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint, C.c_uint,
                          C.POINTER(C.c_double), C.c_uint, C.c_uint]
        R.dot.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint, C.c_uint,
                          C.POINTER(C.c_double), C.c_uint, C.c_uint]
        R.mul.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_uint, C.c_uint, C.c_double]
        _ref = R
    return _ref


def _ref_arrays(g: Graph, poses):
    n = g.n_poses
    hx = (_HX * n)()
    for i in range(n):
        hx[i].step = int(g.x_step[i])
        hx[i].hat_x[0], hx[i].hat_x[1], hx[i].hat_x[2] = poses[i]
    us = (_U * len(g.u))()
    for i in range(len(g.u)):
        us[i].step = int(g.u_step[i]); us[i].nu = g.u[i, 0]; us[i].omega = g.u[i, 1]
    zs = (_Z * max(len(g.z_lm), 1))()
    for i in range(len(g.z_lm)):
        zs[i].step = int(g.z_step[i]); zs[i].landmark_id = int(g.z_lm[i])
        zs[i].z[0], zs[i].z[1] = g.z_rb[i]
    return hx, us, zs


def ref_round(g: Graph, poses, lam: float):
    """One round of the reference: make_edges + MotionEdges + build_csr + pcg_solve_sparse.

    Returns t1, t2, blocks[E, 42], (row_ptr, col_idx, values), xi, dx.
    """
    R = ref()
    hx, us, zs = _ref_arrays(g, poses)
    pj, _ = obs_pairs(g.z_lm)
    E = len(pj) + g.n_poses - 1
    edges = (_Edge * max(E, 1))()
    lkz = (_LKZ * max(len(g.z_lm), 1))()
    ne = C.c_uint(0); nl = C.c_uint(0)
    R.make_edges(hx, g.n_poses, zs, len(g.z_lm), edges, C.byref(ne), lkz, C.byref(nl))
    mns = (C.c_double * 4)(*MNS)
    for i in range(g.n_poses - 1):
        R.MotionEdge_create(C.byref(edges[ne.value + i]), i, i + 1, hx, us, g.delta, lam, mns)
    E = ne.value + g.n_poses - 1
    t1 = np.array([edges[e].t1 for e in range(E)], np.uint32)
    t2 = np.array([edges[e].t2 for e in range(E)], np.uint32)
    blocks = np.zeros((E, 42))
    for e in range(E):
        ed = edges[e]
        blocks[e] = (list(ed.ul) + list(ed.ur) + list(ed.bl) + list(ed.br) + list(ed.xi_u)
                     + list(ed.xi_b))
    dim = g.dim
    xi = np.zeros(dim)
    csr = _CSR()
    R.build_csr_from_edges(edges, E, dim, C.byref(csr), _p(xi, C.c_double))
    nnz = csr.nnz
    row_ptr = np.ctypeslib.as_array(csr.row_ptr, shape=(dim + 1,)).copy()
    col_idx = np.ctypeslib.as_array(csr.col_idx, shape=(nnz,)).copy()
    values = np.ctypeslib.as_array(csr.values, shape=(nnz,)).copy()
    dx = np.zeros(dim)
    R.pcg_solve_sparse(_p(dx, C.c_double), C.byref(csr), _p(xi, C.c_double), dim)
    R.free_csr(C.byref(csr))
    return t1, t2, blocks, (row_ptr, col_idx, values), xi, dx


def ref_cost_terms(g: Graph, poses, lam: float):
    """Per-edge cost terms from the reference's own edges and matrix functions, with the
    dimensions GSLAM.c:74-87 meant: observation edges tra/dot/dot of their 2-element
    hat_e with the 2x2 Omega in Omega[0..3] (ObsEdge.c:196-200), times lambda (1.0);
    motion edges d = sub(hat_x2, state_transition(hat_x1)) (MotionEdge.c:144-148) with
    their 3x3 Omega, times lambda."""
    R = ref()
    hx, us, zs = _ref_arrays(g, poses)
    pj, _ = obs_pairs(g.z_lm)
    E = len(pj) + g.n_poses - 1
    edges = (_Edge * max(E, 1))()
    lkz = (_LKZ * max(len(g.z_lm), 1))()
    ne = C.c_uint(0); nl = C.c_uint(0)
    R.make_edges(hx, g.n_poses, zs, len(g.z_lm), edges, C.byref(ne), lkz, C.byref(nl))
    mns = (C.c_double * 4)(*MNS)
    for i in range(g.n_poses - 1):
        R.MotionEdge_create(C.byref(edges[ne.value + i]), i, i + 1, hx, us, g.delta, lam, mns)
    E = ne.value + g.n_poses - 1
    D = C.c_double
    out = np.zeros(E)
    for k in range(E):
        ed = edges[k]
        if k < ne.value:
            e = (D * 2)(*ed.hat_e)
            om = (D * 4)(*list(ed.Omega)[:4])
            n = 2
        else:
            i = k - ne.value
            nu, omega = g.u[i + 1]
            if abs(omega) < 1e-5:
                omega = 1e-5
            xp = (D * 3)()
            R.state_transition(xp, nu, omega, int(g.delta), hx[i])
            e = (D * 3)()
            R.sub(e, (D * 3)(*hx[i + 1].hat_x), 3, 1, xp, 3, 1)
            om = (D * 9)(*ed.Omega)
            n = 3
        te = (D * n)(); t = (D * n)(); c = (D * 1)(); cl = (D * 1)()
        R.tra(te, e, n, 1)
        R.dot(t, te, 1, n, om, n, n)
        R.dot(c, t, 1, n, e, n, 1)
        R.mul(cl, c, 1, 1, ed.lam)
        out[k] = cl[0]
    return out


def ref_landmark_map(g: Graph, poses):
    """The landmark map as the reference program builds it after its last round
    (GSLAM.c:141-196): make_edges' landmark-sorted z list, one MapEdge_create per
    observation and vec_mean per landmark, all the reference's own compiled functions.
    Landmark ids equal to the z count (the reference's loop sentinel) are not supported."""
    R = ref()
    hx, _, zs = _ref_arrays(g, poses)
    n_z = len(g.z_lm)
    pj, _ = obs_pairs(g.z_lm)
    edges = (_Edge * max(len(pj), 1))()
    lkz = (_LKZ * max(n_z, 1))()
    ne = C.c_uint(0); nl = C.c_uint(0)
    R.make_edges(hx, g.n_poses, zs, n_z, edges, C.byref(ne), lkz, C.byref(nl))
    snr = (C.c_double * 2)(0.14, 0.05)
    ids, ms = [], []
    group = []
    for i in range(nl.value):
        if i == 0 or lkz[i].landmark_id != lkz[i - 1].landmark_id:
            ids.append(lkz[i].landmark_id)
            head = lkz[i].z
            group = []
        me = _MapEdge()
        R.MapEdge_create(C.byref(me), lkz[i].z, head, hx, snr)
        group.append((me.m[0], me.m[1]))
        if i == nl.value - 1 or lkz[i].landmark_id != lkz[i + 1].landmark_id:
            m = np.ascontiguousarray(group, np.float64)
            mean = np.zeros(2)
            R.vec_mean(_p(mean, C.c_double), _p(m, C.c_double), 2, len(group))
            ms.append(mean)
    return np.array(ids, np.uint32), np.array(ms, np.float64).reshape(-1, 2)


def ref_run_binary(log_path: str, lam: float, rounds: int, dump_path: str, use_diff: int = 1):
    """Runs the reference's own GSLAM program; returns (stdout, poses[N, 3])."""
    exe = os.path.join(HERE, "_ref", "GSLAM")
    env = dict(os.environ, POSE_DUMP_FILE=dump_path)
    out = subprocess.run([exe, str(use_diff), repr(lam), str(rounds), "1", log_path],
                         capture_output=True, text=True, env=env, check=True)
    poses = np.loadtxt(dump_path, dtype=np.float64, ndmin=2)[:, 1:4]
    return out.stdout, poses


def gn_fixed_point(poses, ei, ej, meas, log_w, lam: float, anchor: float = 1e6, max_rounds: int = 40,
                   stop: float = 1e-9):
    """The Gauss-Newton fixed point of an SE(2) graph with DIRECT FP64 solves: the edge
    blocks and the assembled Omega / xi of the C restatement (se2_linearise,
    csr_build_anchor), each round's Omega dx = xi solved by a sparse LU factorisation
    (scipy's SuperLU, COLAMD ordering) instead of PCG, angles wrapped in the update.
    Stops when ||dx|| / sqrt(dim) < stop or after max_rounds. At the fixed point the
    result does not depend on the linear solver, so this is the reference for where any
    converged Gauss-Newton run must end. Returns (poses, per-round update norms)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    p = np.array(poses, np.float64).reshape(-1, 3)
    dim = 3 * p.shape[0]
    diffs = []
    for _ in range(max_rounds):
        blocks, _ = se2_linearise(p, ei, ej, meas, log_w, lam)
        rp, ci, va, xi = csr_build_anchor(dim, ei, ej, blocks, anchor)
        A = sp.csr_matrix((va, ci, rp), shape=(dim, dim)).tocsc()
        dx = spl.spsolve(A, xi, permc_spec="COLAMD")
        p = p + dx.reshape(-1, 3)
        p[:, 2] = (p[:, 2] + np.pi) % (2 * np.pi) - np.pi
        diffs.append(float(np.linalg.norm(dx) / np.sqrt(dim)))
        if diffs[-1] < stop:
            break
    return p, diffs
