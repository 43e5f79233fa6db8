"""Dense Gauss-Jordan inverse / solve on the GPU (gslam_gj_inverse / gslam_gj_solve):
the small-N check path of the reference (Omega^-1, then Omega^-1 xi), with the
blocked elimination's trailing updates on the FP64 tensor cores. torch provides the
device buffers only."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


def gj_inverse(a: np.ndarray):
    """Inverse of a dense square matrix (no pivoting); returns (inverse, device ms)."""
    import torch
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    d = torch.from_numpy(a).cuda()
    ms = C.c_float()
    abi.check(abi.lib().gslam_gj_inverse(n, C.c_void_p(d.data_ptr()), n, None, C.byref(ms)))
    return d.cpu().numpy(), ms.value


def gj_solve(a: np.ndarray, b: np.ndarray):
    """x = a^-1 b through the dense inverse; returns (x, device ms of the elimination)."""
    import torch
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b, np.float64)).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    ms = C.c_float()
    abi.check(abi.lib().gslam_gj_solve(n, C.c_void_p(da.data_ptr()), n, C.c_void_p(db.data_ptr()),
                                       C.c_void_p(dx.data_ptr()), None, C.byref(ms)))
    return dx.cpu().numpy(), ms.value


def dmma_peak(reps: int = 20000, ctas_per_sm: int = 4):
    """Measured FP64 tensor-core throughput (TFLOP/s, device ms) of the m8n8k4 DMMA."""
    tf, ms = C.c_double(), C.c_float()
    abi.check(abi.lib().gslam_dmma_bench(int(reps), int(ctas_per_sm), C.byref(tf), C.byref(ms)))
    return tf.value, ms.value
