"""What FP32 Krylov iterates can do on these pose graphs (CPU, numpy; no GPU).

The mixed solver's inner solve keeps the matrix and the vectors in FP32 (dot products
and the 3x3 block-Jacobi inverses in FP64) inside FP64 iterative refinement. On the
block-Jacobi-preconditioned Omega of a city-grid walk (1e6 anchor, chains as long as
the walk) this arithmetic cannot carry a converged solve:

- plain FP32 PCG stalls: its true residual never falls below 1e-6 of ||xi||, while
  FP64 PCG (the reference's recurrence, src/cpu_pcg_fp64/MatrixOps.c:281-391) reaches
  1e-8 in about 7,000 iterations on the 2,000-pose walk;
- FP64 refinement around it does reach 1e-8, but only after more than 2.5 times as
  many FP32 iterations as FP64 PCG needs (3.5-4.4x measured, inner tolerances 1e-1 and
  1e-3).

An FP32 iteration of the device's resident solver takes about half an FP64 one (5.6
against 11.4 us at N = 100k), so at converged settings the mixed solver is slower than
the FP64 one, whatever its kernels do; a 3x speed-up at a 1e-6 pose error would need the
refined FP32 solve to converge in two thirds of FP64's iterations, not 3.5-4.4 times them. These tests pin that
measurement, so it can be re-checked on any machine.
"""
import warnings

import numpy as np
import pytest

from conftest import load_pkg

N_POSES = 2000


@pytest.fixture(scope="module")
def system(oracle):
    import scipy.sparse as sp
    G = load_pkg()
    cg = G.synth.city_grid(N_POSES, seed=3)
    blocks, _ = oracle.se2_linearise(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1)
    rp, ci, va, xi = oracle.csr_build_anchor(3 * N_POSES, cg.edge_i, cg.edge_j, blocks, 1e6)
    A = sp.csr_matrix((va, ci, rp), shape=(3 * N_POSES, 3 * N_POSES))
    dinv = oracle.diag_inv(rp, ci, va)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        D = sp.block_diag([sp.csr_matrix(d.reshape(3, 3)) for d in dinv], format="csr")
    return A, D, xi


def pcg64(A, D, b, tol, cap):
    x = np.zeros_like(b)
    r = b.copy()
    z = D @ r
    p = z.copy()
    rz = r @ z
    for k in range(cap):
        q = A @ p
        a = rz / (p @ q)
        x = x + a * p
        r = r - a * q
        if np.linalg.norm(r) < tol * np.linalg.norm(b):
            return x, k + 1
        z = D @ r
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, cap


def pcg32(A32, D, b, tol, cap, true_residual=None):
    """FP32 matrix and vectors; FP64 dot products and FP64 block-Jacobi inverses.
    With `true_residual`, also returns the smallest FP64 residual seen (every 100)."""
    f, d = np.float32, np.float64
    x = np.zeros(len(b), f)
    r = b.astype(f)
    z = (D @ r.astype(d)).astype(f)
    p = z.copy()
    rz = float(r.astype(d) @ z.astype(d))
    best = np.inf
    for k in range(cap):
        q = A32 @ p
        a = rz / float(p.astype(d) @ q.astype(d))
        x = x + f(a) * p
        r = r - f(a) * q
        if true_residual is not None and k % 100 == 0:
            best = min(best, true_residual(x.astype(d)))
        if np.linalg.norm(r.astype(d)) < tol * np.linalg.norm(b):
            return x, k + 1, best
        z = (D @ r.astype(d)).astype(f)
        rz2 = float(r.astype(d) @ z.astype(d))
        p = z + f(rz2 / rz) * p
        rz = rz2
    return x, cap, best


def test_fp32_pcg_stalls_where_fp64_converges(system):
    A, D, xi = system
    bn = np.linalg.norm(xi)
    x64, k64 = pcg64(A, D, xi, 1e-8, 50000)
    assert np.linalg.norm(xi - A @ x64) / bn < 2e-8 and k64 < 20000
    rel = lambda x: np.linalg.norm(xi - A @ x) / bn  # noqa: E731
    _, _, best = pcg32(A.astype(np.float32), D, xi, 1e-12, 3 * k64, true_residual=rel)
    print(f"FP64 PCG: 1e-8 in {k64} iterations; FP32 PCG, best true residual in {3 * k64}: {best:.2e}")
    assert best > 1e-6


@pytest.mark.parametrize("inner_tol", [1e-1, 1e-3])
def test_fp64_refinement_needs_several_times_the_iterations(system, inner_tol):
    A, D, xi = system
    bn = np.linalg.norm(xi)
    _, k64 = pcg64(A, D, xi, 1e-8, 50000)
    A32 = A.astype(np.float32)
    x = np.zeros_like(xi)
    r = xi.copy()
    total = steps = 0
    while np.linalg.norm(r) / bn > 1e-8 and total < 20 * k64:
        d, k, _ = pcg32(A32, D, r, inner_tol, 20000)
        x = x + d.astype(np.float64)
        r = xi - A @ x
        total += k
        steps += 1
    print(f"inner tol {inner_tol:g}: {steps} refinement steps, {total} FP32 iterations "
          f"= {total / k64:.2f}x FP64's {k64}")
    assert np.linalg.norm(r) / bn <= 1e-8   # refinement does converge ...
    assert total > 2.5 * k64                # ... at several times FP64's iteration count
