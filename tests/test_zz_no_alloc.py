"""The allocation-free solver entry point (gslam_pcg_solve_static).

For callers that cannot allocate device memory while they solve — processes whose
device memory belongs to another allocator or is fixed up front, real-time loops in
which an allocation could block or fail — the library offers one entry point whose
scratch lives in a fixed array inside the library. This test calls it through the C ABI twice in a
row on device buffers the test owns, and compares both results with what the
regular solver entry point (pcg_solve_sparse, the reference's own signature)
returns for the same system, with the converged-solve tolerance used by
tests/test_gpu_parity.py. The file sorts last so a run that stops at the first
failure has run every other test before this one.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import assert_bitwise, load_pkg

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _system(oracle):
    """A 200-pose SE(2) graph that block-Jacobi PCG solves to 1e-6 in ~260 iterations."""
    G = load_pkg()
    cg = G.synth.city_grid(200, seed=3, k_closures=6, radius=3.0, block=5, min_gap=3)
    ob, _ = oracle.se2_linearise(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 1.0)
    return oracle.csr_build_anchor(3 * cg.n_poses, cg.edge_i, cg.edge_j, ob, 10.0)


def test_static_solver_matches_regular_entry_point(oracle):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    G = load_pkg()
    A_ = G.abi
    L = A_.lib()
    rp, ci, va, xi = _system(oracle)
    dim = len(xi)
    # the regular entry point, on host arrays
    os.environ["GSLAM_DROPIN_NOEXIT"] = "1"
    csr = A_.CSRMatrix(A_.ptr(rp, C.c_int), A_.ptr(ci, C.c_int), A_.ptr(va), dim, len(va))
    x_reg = np.zeros(dim)
    L.pcg_solve_sparse(A_.ptr(x_reg), C.byref(csr), A_.ptr(xi), dim)
    assert L.gslam_dropin_status() == 0
    # the allocation-free entry point, on device buffers owned by the caller
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    d_va = torch.from_numpy(va).cuda()
    d_b = torch.from_numpy(xi).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    A = sp.csr_matrix((va, ci, rp), shape=(dim, dim))
    xs = spl.spsolve(A.tocsc(), xi)
    ea = lambda x: np.sqrt(max((x - xs) @ (A @ (x - xs)), 0.0))  # noqa: E731
    scale = np.sqrt(xs @ (A @ xs))
    outs = []
    for call in range(2):
        d_x = torch.full((dim,), float("nan"), dtype=torch.float64, device="cuda")
        st = A_.SolveStats()
        rc = L.gslam_pcg_solve_static(dim, C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_ci.data_ptr()),
                                      C.c_void_p(d_va.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                      C.c_void_p(d_x.data_ptr()), 1e-6, 500, C.c_void_p(stream),
                                      C.byref(st))
        assert rc == 0, L.gslam_last_error()
        assert st.reason == A_.STOP_TOL and st.iterations < 500
        x = d_x.cpu().numpy()
        assert np.isfinite(x).all()
        # same converged-solve criterion as tests/test_gpu_parity.py
        assert ea(x) <= max(1e-6 * scale, 1.5 * ea(x_reg)), f"call {call}: {ea(x) / scale:.3e}"
        assert np.linalg.norm(x - x_reg) <= 1e-4 * np.linalg.norm(x_reg)
        outs.append(x)
    assert_bitwise(outs[0], outs[1], "second call")


def test_static_solver_rejects_oversized_systems():
    G = load_pkg()
    L = G.abi.lib()
    dim = 3 * (16384 + 1)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    di = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = L.gslam_pcg_solve_static(dim, C.c_void_p(di.data_ptr()), C.c_void_p(di.data_ptr()),
                                  C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                  C.c_void_p(d.data_ptr()), 1e-6, 10, None, None)
    assert rc == G.abi.ERR_TOO_LARGE
    assert b"16384" in L.gslam_last_error()


def test_static_solver_status_read_back(oracle):
    """A caller that queues the solve without waiting (stats NULL) reads its status
    afterwards with gslam_pcg_static_status on the same stream."""
    G = load_pkg()
    A_ = G.abi
    L = A_.lib()
    rp, ci, va, xi = _system(oracle)
    dim = len(xi)
    dev = [torch.from_numpy(a).cuda() for a in (rp, ci, va, xi)]
    d_x = torch.zeros(dim, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.gslam_pcg_solve_static(dim, *[C.c_void_p(t.data_ptr()) for t in dev], C.c_void_p(d_x.data_ptr()),
                                  1e-6, 500, C.c_void_p(stream), None)
    assert rc == 0, L.gslam_last_error()
    st = A_.SolveStats()
    rc = L.gslam_pcg_static_status(C.c_void_p(stream), C.byref(st))
    assert rc == 0, L.gslam_last_error()
    assert st.reason == A_.STOP_TOL and 0 < st.iterations < 500
    assert st.rel_residual < 1e-6
    assert L.gslam_pcg_static_status(C.c_void_p(stream), None) == 0
