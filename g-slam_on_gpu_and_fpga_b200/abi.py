"""ctypes binding of libgslam.so (include/gslam.h, include/gslam_dropin.h).

The shared library is built in-tree by build.py. Loading it never falls back to
anything else: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgslam.so")
CLI_PATH = os.path.join(HERE, "bin", "GSLAM")
DATA_TOOL_PATH = os.path.join(HERE, "bin", "gslam-data")

OK = 0
ERR_BAD_INPUT = -1
ERR_CUDA = -2
ERR_DEVICE_TIMEOUT = -3
ERR_NOT_CONVERGED = -4
ERR_TOO_LARGE = -5
ERR_NO_DEVICE = -6

PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP64_CG = 2   # FP64 PCG, one grid reduction per iteration (Chronopoulos-Gear)

STOP_TOL, STOP_MAXIT, STOP_PQ_ZERO, STOP_TIMEOUT = 0, 1, 2, 3

# every extern "C" symbol the headers declare (checked by the CPU tests)
EXPORTS = [
    "gslam_opts_default", "gslam_create_reference", "gslam_create_se2", "gslam_destroy",
    "gslam_set_opts", "gslam_sizes", "gslam_get_stream", "gslam_set_poses", "gslam_get_poses", "gslam_round", "gslam_round_io",
    "gslam_run", "gslam_linearise", "gslam_assemble", "gslam_solve", "gslam_update",
    "gslam_get_edge_blocks", "gslam_assemble_from_edges", "gslam_get_csr", "gslam_get_dx",
    "gslam_get_diag_inv", "gslam_spmv", "gslam_spmv_bench", "gslam_spmv_bytes", "gslam_read_log", "gslam_free_log",
    "gslam_version", "gslam_last_error", "gslam_obs_edge_order", "gslam_csr_pattern", "gslam_layout_plan",
    "pcg_solve_sparse", "device_graph_init", "device_graph_update", "device_graph_get_row_ptr",
    "device_graph_get_col_idx", "device_build_diag_inv", "device_pcg_solve", "device_graph_free",
    "gslam_dropin_status", "gslam_pcg_solve_static", "gslam_pcg_static_status", "gslam_set_se2_weights", "gslam_adjoint",
    "gslam_create_se2_batch", "gslam_batch_round", "gslam_batch_layout",
    "gslam_gj_inverse", "gslam_gj_solve", "gslam_dmma_bench", "gslam_landmark_map", "gslam_cost",
]


class GslamError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gslam error {code}: {msg}")
        self.code = code


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
                ("sell_window", C.c_int), ("threads_per_cta", C.c_int), ("ctas_per_sm", C.c_int),
                ("angle_wrap", C.c_int), ("inner_tol", C.c_double), ("inner_max_iter", C.c_int),
                ("max_refine", C.c_int), ("device", C.c_int), ("barrier_timeout_ms", C.c_double),
                ("test_absent_cta", C.c_int), ("disable_resident", C.c_int), ("round_graph", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("reason", C.c_int),
                ("rel_residual", C.c_double), ("diff", C.c_double), ("solve_ms", C.c_double),
                ("round_ms", C.c_double)]


class ReferenceGraphDesc(C.Structure):
    _fields_ = [("n_poses", C.c_uint32), ("poses", C.POINTER(C.c_double)),
                ("controls", C.POINTER(C.c_double)), ("delta", C.c_double),
                ("lam", C.c_double), ("mns", C.POINTER(C.c_double)), ("n_obs", C.c_uint32),
                ("obs_step", C.POINTER(C.c_uint32)), ("obs_landmark", C.POINTER(C.c_uint32)),
                ("obs", C.POINTER(C.c_double))]


class SE2GraphDesc(C.Structure):
    _fields_ = [("n_poses", C.c_uint32), ("poses", C.POINTER(C.c_double)), ("n_edges", C.c_uint32),
                ("edge_i", C.POINTER(C.c_uint32)), ("edge_j", C.POINTER(C.c_uint32)),
                ("meas", C.POINTER(C.c_double)), ("log_w", C.POINTER(C.c_double)),
                ("lam", C.c_double), ("anchor", C.c_double)]


class LogDesc(C.Structure):
    _fields_ = [("delta", C.c_double), ("n_u", C.c_uint32), ("n_x", C.c_uint32), ("n_z", C.c_uint32),
                ("u_step", C.POINTER(C.c_uint32)), ("u", C.POINTER(C.c_double)),
                ("x_step", C.POINTER(C.c_uint32)), ("x", C.POINTER(C.c_double)),
                ("z_step", C.POINTER(C.c_uint32)), ("z_lm", C.POINTER(C.c_uint32)),
                ("z", C.POINTER(C.c_double))]


class CSRMatrix(C.Structure):
    _fields_ = [("row_ptr", C.POINTER(C.c_int)), ("col_idx", C.POINTER(C.c_int)),
                ("values", C.POINTER(C.c_double)), ("dim", C.c_int), ("nnz", C.c_int)]


class LayoutInfo(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("n_slices", C.c_int64), ("n_slots", C.c_int64),
                ("nnzb", C.c_int64), ("csr_nnz", C.c_int64), ("anchor_slot", C.c_int64),
                ("max_width", C.c_int32), ("bare_anchor", C.c_int32)]


class ZRec(C.Structure):
    _fields_ = [("step", C.c_uint), ("landmark_id", C.c_uint), ("z", C.c_double * 2)]


class URec(C.Structure):
    _fields_ = [("step", C.c_uint), ("nu", C.c_double), ("omega", C.c_double)]


class HatXRec(C.Structure):
    _fields_ = [("step", C.c_uint), ("hat_x", C.c_double * 3)]


_lib = None
VP = C.c_void_p
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)
I64P = C.POINTER(C.c_int64)


def lib() -> C.CDLL:
    """Loads libgslam.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built (run build.py)")
        L = C.CDLL(LIB_PATH)
        sig = {
            "gslam_opts_default": [C.POINTER(Opts)],
            "gslam_create_reference": [C.POINTER(ReferenceGraphDesc), C.POINTER(Opts), C.POINTER(VP)],
            "gslam_create_se2": [C.POINTER(SE2GraphDesc), C.POINTER(Opts), C.POINTER(VP)],
            "gslam_destroy": [VP],
            "gslam_set_opts": [VP, C.POINTER(Opts)],
            "gslam_sizes": [VP, I64P, I64P, I64P, I64P],
            "gslam_get_stream": [VP, C.POINTER(VP)],
            "gslam_set_poses": [VP, DP],
            "gslam_get_poses": [VP, DP],
            "gslam_round": [VP, C.POINTER(SolveStats)],
            "gslam_round_io": [VP, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(SolveStats)],
            "gslam_run": [VP, C.c_int, DP, IP],
            "gslam_linearise": [VP],
            "gslam_assemble": [VP],
            "gslam_solve": [VP, C.POINTER(SolveStats)],
            "gslam_update": [VP, DP],
            "gslam_get_edge_blocks": [VP, DP],
            "gslam_assemble_from_edges": [VP, VP],
            "gslam_get_csr": [VP, IP, IP, DP, DP],
            "gslam_get_dx": [VP, DP],
            "gslam_get_diag_inv": [VP, DP],
            "gslam_spmv": [VP, VP, VP],
            "gslam_spmv_bench": [VP, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)],
            "gslam_spmv_bytes": [VP, C.c_int, I64P],
            "gslam_read_log": [C.c_char_p, C.POINTER(C.POINTER(LogDesc))],
            "gslam_free_log": [C.POINTER(LogDesc)],
            "gslam_obs_edge_order": [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32), C.c_int64, I64P],
            "gslam_csr_pattern": [C.c_uint32, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  IP, IP, I64P],
            "gslam_layout_plan": [C.c_uint32, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.c_int, C.c_uint32, IP, C.c_uint32, IP, C.POINTER(LayoutInfo),
                                  IP, I64P, IP, I64P, I64P, I64P, I64P, I64P],
            "pcg_solve_sparse": [DP, C.POINTER(CSRMatrix), DP, C.c_uint],
            "device_graph_init": [C.POINTER(ZRec), C.c_uint, C.POINTER(URec), C.c_uint, C.c_uint,
                                  C.c_double, C.c_double, DP, IP],
            "device_graph_update": [C.POINTER(HatXRec), C.c_uint, VP, VP],
            "device_pcg_solve": [DP, VP, VP, C.c_int, C.c_int, C.c_int],
            "device_build_diag_inv": [C.c_int],
            "device_graph_free": [],
            "gslam_dropin_status": [],
            "gslam_pcg_solve_static": [C.c_int, VP, VP, VP, VP, VP, C.c_double, C.c_int, VP,
                                       C.POINTER(SolveStats)],
            "gslam_pcg_static_status": [VP, C.POINTER(SolveStats)],
            "gslam_set_se2_weights": [VP, C.c_double, DP],
            "gslam_adjoint": [VP, DP, DP, DP, DP, C.POINTER(SolveStats)],
            "gslam_create_se2_batch": [C.POINTER(SE2GraphDesc), C.c_uint32, C.POINTER(Opts), C.POINTER(VP)],
            "gslam_batch_round": [VP, C.POINTER(SolveStats)],
            "gslam_batch_layout": [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
            "gslam_gj_inverse": [C.c_int, VP, C.c_int, VP, C.POINTER(C.c_float)],
            "gslam_gj_solve": [C.c_int, VP, C.c_int, VP, VP, VP, C.POINTER(C.c_float)],
            "gslam_dmma_bench": [C.c_int, C.c_int, DP, C.POINTER(C.c_float)],
            "gslam_landmark_map": [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), DP],
            "gslam_cost": [VP, DP, DP],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        for name in ("pcg_solve_sparse", "device_graph_init", "device_graph_update",
                     "device_pcg_solve", "device_build_diag_inv", "device_graph_free",
                     "gslam_free_log"):
            getattr(L, name).restype = None
        L.device_graph_get_row_ptr.restype = VP
        L.device_graph_get_col_idx.restype = VP
        L.gslam_version.restype = C.c_char_p
        L.gslam_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != OK:
        raise GslamError(rc, lib().gslam_last_error().decode(errors="replace"))
    return rc


def ptr(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def default_opts(**kw) -> Opts:
    o = Opts()
    check(lib().gslam_opts_default(C.byref(o)))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def layout_plan(n_poses: int, t1, t2, sell_window: int = 0, segments=None, diag_rows=None) -> dict:
    """The device layout of an edge list, computed on the host (gslam_layout_plan):
    sizes plus perm, slice_ptr, col, ctr_ptr, ctr, xi_ptr, xi_ctr, slot_csr as arrays."""
    L = lib()
    t1 = np.ascontiguousarray(t1, np.uint32)
    t2 = np.ascontiguousarray(t2, np.uint32)
    seg = None if segments is None else np.ascontiguousarray(segments, np.int32)
    dia = None if diag_rows is None else np.ascontiguousarray(diag_rows, np.int32)
    head = (C.c_uint32(n_poses), C.c_int64(len(t1)), ptr(t1, C.c_uint32), ptr(t2, C.c_uint32),
            C.c_int(sell_window), C.c_uint32(0 if seg is None else len(seg)),
            None if seg is None else ptr(seg, C.c_int), C.c_uint32(0 if dia is None else len(dia)),
            None if dia is None else ptr(dia, C.c_int))
    info = LayoutInfo()
    check(L.gslam_layout_plan(*head, C.byref(info), *([None] * 8)))
    E = len(t1)
    out = {k: getattr(info, k) for k, _ in LayoutInfo._fields_}
    arrays = [("perm", info.n_rows, np.int32), ("slice_ptr", info.n_slices + 1, np.int64),
              ("col", info.n_slots, np.int32), ("ctr_ptr", info.n_slots + 1, np.int64),
              ("ctr", 4 * E, np.int64), ("xi_ptr", info.n_rows + 1, np.int64),
              ("xi_ctr", 2 * E, np.int64), ("slot_csr", info.n_slots, np.int64)]
    bufs = [np.zeros(max(n, 1), t) for _, n, t in arrays]
    ct = {np.int32: C.c_int, np.int64: C.c_int64}
    check(L.gslam_layout_plan(*head, C.byref(info),
                              *[ptr(b, ct[t]) for b, (_, _, t) in zip(bufs, arrays)]))
    for (name, n, _), b in zip(arrays, bufs):
        out[name] = b[:n]
    return out
