"""Dense FP64 reference for the SE(2) Gauss-Newton solve and its implicit-function
adjoint (test infrastructure; numpy only).

Same factor and conventions as the library (csrc/edge_math.cuh em_se2_edge, csrc/adjoint.cu):
  e = [R(th_i)^T (t_j - t_i) - z_t ; wrap(th_j - th_i - z_th)],  Lambda = lambda diag(exp(w)),
  Omega = sum J^T Lambda J + anchor on pose 0's diagonal, xi = -sum J^T Lambda e,
  poses += Omega^-1 xi with the angle wrapped.
Adjoint at converged poses: H mu = dL/dx with H the exact Hessian of
(1/2) sum e^T Lambda e (+ anchor), dL/dw_{e,k} = -Lambda_k e_k (J mu)_k,
dL/dlambda = sum dL/dw / lambda.
"""
from __future__ import annotations

import numpy as np


def wrap(a):
    return (a + np.pi) % (2.0 * np.pi) - np.pi


def residuals(poses, ei, ej, meas):
    """e [E, 3], J_i [E, 3, 3], J_j [E, 3, 3], plus (c, s, dx, dy) for the Hessian terms."""
    pi, pj = poses[ei], poses[ej]
    c, s = np.cos(pi[:, 2]), np.sin(pi[:, 2])
    dx, dy = pj[:, 0] - pi[:, 0], pj[:, 1] - pi[:, 1]
    e = np.stack([c * dx + s * dy - meas[:, 0], c * dy - s * dx - meas[:, 1],
                  wrap(pj[:, 2] - pi[:, 2] - meas[:, 2])], axis=1)
    n = len(ei)
    Ji = np.zeros((n, 3, 3))
    Jj = np.zeros((n, 3, 3))
    Ji[:, 0] = np.stack([-c, -s, c * dy - s * dx], axis=1)
    Ji[:, 1] = np.stack([s, -c, -c * dx - s * dy], axis=1)
    Ji[:, 2, 2] = -1.0
    Jj[:, 0, 0], Jj[:, 0, 1] = c, s
    Jj[:, 1, 0], Jj[:, 1, 1] = -s, c
    Jj[:, 2, 2] = 1.0
    return e, Ji, Jj, (c, s, dx, dy)


def _scatter(H, ei, ej, UL, UR, BL, BR):
    for k in range(len(ei)):
        i, j = 3 * ei[k], 3 * ej[k]
        H[i:i + 3, i:i + 3] += UL[k]
        H[i:i + 3, j:j + 3] += UR[k]
        H[j:j + 3, i:i + 3] += BL[k]
        H[j:j + 3, j:j + 3] += BR[k]


def system(poses, ei, ej, meas, log_w, lam, anchor, exact=False):
    """Dense Omega (or the exact Hessian) and xi = -g at `poses`."""
    n = poses.shape[0]
    e, Ji, Jj, (c, s, dx, dy) = residuals(poses, ei, ej, meas)
    L = lam * np.exp(log_w)
    LJi, LJj = L[:, :, None] * Ji, L[:, :, None] * Jj
    UL = np.einsum("eki,ekj->eij", Ji, LJi)
    UR = np.einsum("eki,ekj->eij", Ji, LJj)
    BL = np.einsum("eki,ekj->eij", Jj, LJi)
    BR = np.einsum("eki,ekj->eij", Jj, LJj)
    if exact:
        a0, a1 = L[:, 0] * e[:, 0], L[:, 1] * e[:, 1]
        htt = a0 * (-c * dx - s * dy) + a1 * (s * dx - c * dy)
        htx = a0 * s + a1 * c
        hty = a1 * s - a0 * c
        UL = UL.copy(); UR = UR.copy(); BL = BL.copy()
        UL[:, 2, 2] += htt
        UL[:, 2, 0] += htx; UL[:, 0, 2] += htx
        UL[:, 2, 1] += hty; UL[:, 1, 2] += hty
        UR[:, 2, 0] -= htx; UR[:, 2, 1] -= hty
        BL[:, 0, 2] -= htx; BL[:, 1, 2] -= hty
    H = np.zeros((3 * n, 3 * n))
    _scatter(H, ei, ej, UL, UR, BL, BR)
    H[0:3, 0:3] += anchor * np.eye(3)
    Le = L * e
    xi = np.zeros(3 * n)
    np.add.at(xi.reshape(n, 3), ei, -np.einsum("eki,ek->ei", Ji, Le))
    np.add.at(xi.reshape(n, 3), ej, -np.einsum("eki,ek->ei", Jj, Le))
    return H, xi


def gn_solve(poses0, ei, ej, meas, log_w, lam, anchor=1e6, rounds=50, tol=1e-13):
    """Dense Gauss-Newton to convergence (update RMS below tol)."""
    p = np.array(poses0, np.float64, copy=True)
    for _ in range(rounds):
        H, xi = system(p, ei, ej, meas, log_w, lam, anchor)
        dx = np.linalg.solve(H, xi).reshape(-1, 3)
        p = p + dx
        p[:, 2] = wrap(p[:, 2])
        if np.sqrt(np.mean(dx ** 2)) < tol:
            break
    return p


def adjoint(poses, ei, ej, meas, log_w, lam, dL_dx, anchor=1e6):
    """(dL/dlambda, dL/dlog_w [E, 3], mu [N, 3]) by a dense exact-Hessian solve."""
    H, _ = system(poses, ei, ej, meas, log_w, lam, anchor, exact=True)
    mu = np.linalg.solve(H, np.asarray(dL_dx, np.float64).reshape(-1)).reshape(-1, 3)
    e, Ji, Jj, _ = residuals(poses, ei, ej, meas)
    jm = np.einsum("ekc,ec->ek", Ji, mu[ei]) + np.einsum("ekc,ec->ek", Jj, mu[ej])
    dlw = -(lam * np.exp(log_w)) * e * jm
    return dlw.sum() / lam, dlw, mu


def position_loss(poses, target):
    """Sum of squared position differences, and its gradient w.r.t. the poses."""
    d = poses[:, :2] - target[:, :2]
    g = np.zeros_like(poses)
    g[:, :2] = 2.0 * d
    return float((d ** 2).sum()), g


# ---- sparse forms of the same reference (scipy SuperLU), for sizes a dense solve cannot hold ----

def system_sparse(poses, ei, ej, meas, log_w, lam, anchor, exact=False):
    """system() with Omega (or the exact Hessian) as a scipy CSC matrix."""
    import scipy.sparse as sp
    n = poses.shape[0]
    e, Ji, Jj, (c, s, dx, dy) = residuals(poses, ei, ej, meas)
    L = lam * np.exp(log_w)
    LJi, LJj = L[:, :, None] * Ji, L[:, :, None] * Jj
    UL = np.einsum("eki,ekj->eij", Ji, LJi)
    UR = np.einsum("eki,ekj->eij", Ji, LJj)
    BL = np.einsum("eki,ekj->eij", Jj, LJi)
    BR = np.einsum("eki,ekj->eij", Jj, LJj)
    if exact:
        a0, a1 = L[:, 0] * e[:, 0], L[:, 1] * e[:, 1]
        htt = a0 * (-c * dx - s * dy) + a1 * (s * dx - c * dy)
        htx = a0 * s + a1 * c
        hty = a1 * s - a0 * c
        UL[:, 2, 2] += htt
        UL[:, 2, 0] += htx; UL[:, 0, 2] += htx
        UL[:, 2, 1] += hty; UL[:, 1, 2] += hty
        UR[:, 2, 0] -= htx; UR[:, 2, 1] -= hty
        BL[:, 0, 2] -= htx; BL[:, 1, 2] -= hty
    rr, cc = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
    rows, cols, vals = [], [], []
    for (a, b, blk) in ((ei, ei, UL), (ei, ej, UR), (ej, ei, BL), (ej, ej, BR)):
        rows.append((3 * a[:, None, None] + rr).ravel())
        cols.append((3 * b[:, None, None] + cc).ravel())
        vals.append(blk.ravel())
    rows.append(np.arange(3)); cols.append(np.arange(3)); vals.append(np.full(3, float(anchor)))
    H = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(3 * n, 3 * n)).tocsc()
    Le = L * e
    xi = np.zeros(3 * n)
    np.add.at(xi.reshape(n, 3), ei, -np.einsum("eki,ek->ei", Ji, Le))
    np.add.at(xi.reshape(n, 3), ej, -np.einsum("eki,ek->ei", Jj, Le))
    return H, xi


def gn_solve_sparse(poses0, ei, ej, meas, log_w, lam, anchor=1e6, rounds=50, tol=1e-13, min_rounds=1):
    """Gauss-Newton to convergence with sparse LU solves (update RMS below tol, after at
    least min_rounds rounds)."""
    import scipy.sparse.linalg as spl
    p = np.array(poses0, np.float64, copy=True)
    for r in range(rounds):
        H, xi = system_sparse(p, ei, ej, meas, log_w, lam, anchor)
        dx = spl.spsolve(H, xi, permc_spec="COLAMD").reshape(-1, 3)
        p = p + dx
        p[:, 2] = wrap(p[:, 2])
        if np.sqrt(np.mean(dx ** 2)) < tol and r + 1 >= min_rounds:
            break
    return p


def adjoint_sparse(poses, ei, ej, meas, log_w, lam, dL_dx, anchor=1e6):
    """adjoint() with a sparse LU solve of the exact Hessian."""
    import scipy.sparse.linalg as spl
    H, _ = system_sparse(poses, ei, ej, meas, log_w, lam, anchor, exact=True)
    mu = spl.spsolve(H, np.asarray(dL_dx, np.float64).reshape(-1), permc_spec="COLAMD").reshape(-1, 3)
    e, Ji, Jj, _ = residuals(poses, ei, ej, meas)
    jm = np.einsum("ekc,ec->ek", Ji, mu[ei]) + np.einsum("ekc,ec->ek", Jj, mu[ej])
    dlw = -(lam * np.exp(log_w)) * e * jm
    return dlw.sum() / lam, dlw, mu


def rhs(poses, ei, ej, meas, log_w, lam):
    """xi = -sum J^T Lambda e alone (system() without the matrix)."""
    n = poses.shape[0]
    e, Ji, Jj, _ = residuals(poses, ei, ej, meas)
    Le = lam * np.exp(log_w) * e
    xi = np.zeros(3 * n)
    np.add.at(xi.reshape(n, 3), ei, -np.einsum("eki,ek->ei", Ji, Le))
    np.add.at(xi.reshape(n, 3), ej, -np.einsum("eki,ek->ei", Jj, Le))
    return xi


def chord_solve_sparse(poses0, ei, ej, meas, log_w, lam, lu, anchor=1e6, rounds=60, tol=1e-14, min_rounds=1):
    """Gauss-Newton's fixed point by chord iterations: every round solves with one
    factorisation `lu` (splu of a nearby Omega, e.g. the one at the unperturbed fixed
    point) instead of refactorising. The iteration stops where xi = 0 for THESE weights,
    the same point Gauss-Newton reaches; it only converges more slowly. Used for the
    finite differences, which restart from a fixed point a perturbation h away."""
    p = np.array(poses0, np.float64, copy=True)
    for r in range(rounds):
        dx = lu.solve(rhs(p, ei, ej, meas, log_w, lam)).reshape(-1, 3)
        p = p + dx
        p[:, 2] = wrap(p[:, 2])
        if np.sqrt(np.mean(dx ** 2)) < tol and r + 1 >= min_rounds:
            break
    return p


# ---- double-double fixed points, for finite differences below the FP64 noise floor ----

def chord_solve_dd(oracle, poses0, ei, ej, meas, log_w, lam, lu, rounds=60, tol=1e-28):
    """chord_solve_sparse with xi evaluated in double-double at double-double poses
    (oracle/se2_dd.c): the FP64 LU only proposes each correction, the double-double
    xi decides where the iteration stops, so the fixed point comes out to ~1e-30
    instead of FP64's noise. Angles are not wrapped (the corrections are tiny; the
    residual wraps itself). Returns (hi, lo), each [N, 3]."""
    hi = np.array(poses0, np.float64, copy=True).reshape(-1)
    lo = np.zeros_like(hi)
    info = lam * np.exp(log_w)
    scale = np.max(np.abs(hi))
    for _ in range(rounds):
        xh, _ = oracle.se2_rhs_dd(hi, lo, ei, ej, meas, info)
        dx = lu.solve(xh)
        oracle.dd_add_vec(hi, lo, dx)
        if np.max(np.abs(dx)) < tol * scale:
            break
    return hi.reshape(-1, 3), lo.reshape(-1, 3)


def fd_log_weights_dd(oracle, poses, ei, ej, meas, log_w, lam, lu, target, pairs, h):
    """Central differences of position_loss(fixed point) in the log weights (edge e,
    component k) for each pair, with double-double fixed points and loss; the step is
    the one the FP64 weights actually take (fl(w + h) - w, fl(w - h) - w)."""
    out = []
    for e, k in pairs:
        lp, lm = log_w.copy(), log_w.copy()
        lp[e, k] += h
        lm[e, k] -= h
        step = (lp[e, k] - log_w[e, k]) - (lm[e, k] - log_w[e, k])
        Lp = oracle.position_loss_dd(*chord_solve_dd(oracle, poses, ei, ej, meas, lp, lam, lu), target)
        Lm = oracle.position_loss_dd(*chord_solve_dd(oracle, poses, ei, ej, meas, lm, lam, lu), target)
        out.append(((Lp[0] - Lm[0]) + (Lp[1] - Lm[1])) / step)
    return np.array(out)
