"""dCov / HSIC statistics and p-values for the CI methods (oracle).

TEST INFRASTRUCTURE ONLY: the CPU checker for the library's statistic
kernels.  All arithmetic is binary64.

* exact dCov gamma (fastkpc/src/cuda/full_cuda_ci_vertical.cu:485-769):
  D = |r_i - r_j| (the ``index`` argument is ignored, legacy semantics),
  A = H D H; nV2 = sum(A*B)/n; mean = (sum Dx/n^2)(sum Dy/n^2);
  var = 2(n-4)(n-5)/(n(n-1)(n-2)(n-3)) * sum(A^2) sum(B^2) / n^2;
  p = Q(shape = mean^2/var, nV2 / (var/mean)).
* legacy low-rank dCov gamma (kpcalg/R/dcovgamma.R:51-100; refinement
  kernels fastkpc/src/cuda/full_cuda_ci_vertical.cu:771-967): numCol
  eigenpairs of D of largest |value| (ties -> higher index), eigenvectors
  centred; nV2 = sum_ij l_i m_j (u_i . v_j)^2 / n, variance from
  sum_ij l_i l_j (u_i . u_j)^2 of each side, mean from the raw distances.
* kernlab ``inchol`` HSIC (kpcalg/R/hsicgamma.R:52-99; restated kernels
  fastkpc/src/cuda/full_cuda_ci_method_batch.cu:445-789): RBF
  exp(-(r_i-r_j)^2 / sig), greedy pivot on the largest residual diagonal
  starting at row 0, tolerance 1e-3, rank <= numCol; HSIC = |Gx' Gy|_F^2/n^2
  with column-centred factors; mean from the off-diagonal sums of the raw
  factors; p = 1 - (1 - Q).
* permutation p = (1 + #{T_pi >= T}) / (R + 1) for hsic.perm and dcc.perm
  (fastkpc/src/cuda/full_cuda_ci_method_batch.cu:341-443, :791-908).
* Q is scipy's regularised upper incomplete gamma (an implementation
  independent of the library's own continued fraction / series).
"""
import math

import numpy as np
from scipy.special import gammaincc

INCHOL_TOL = 1e-3


def _var_factor(n):
    return 2.0 * (n - 4.0) * (n - 5.0) / n / (n - 1.0) / (n - 2.0) / (n - 3.0)


def _gamma_p(stat, mean, var):
    shape = mean * mean / var
    scale = var / mean
    return float(gammaincc(shape, max(0.0, stat / scale)))


def dcov_components(r):
    r = np.asarray(r, dtype=np.float64)
    D = np.abs(r[:, None] - r[None, :])
    row = D.mean(axis=1)
    grand = D.mean()
    A = D - row[:, None] - row[None, :] + grand
    return {"D": D, "A": A, "total": float(D.sum()), "self": float(np.sum(A * A))}


def dcov_gamma_exact(rx, ry):
    cx, cy = dcov_components(rx), dcov_components(ry)
    n = float(len(rx))
    stat = float(np.sum(cx["A"] * cy["A"])) / n
    mean = (cx["total"] / (n * n)) * (cy["total"] / (n * n))
    var = _var_factor(n) * cx["self"] * cy["self"] / (n * n)
    return {"statistic": stat, "mean": mean, "variance": var, "p_value": _gamma_p(stat, mean, var)}


def legacy_lowrank(r, num_col):
    """(values, centred vectors) of the num_col largest-|value| eigenpairs."""
    r = np.asarray(r, dtype=np.float64)
    D = np.abs(r[:, None] - r[None, :])
    vals, vecs = np.linalg.eigh(D)
    mag = np.abs(vals)
    n = len(r)
    # largest magnitude first; ties broken toward the higher index
    order = sorted(range(n), key=lambda i: (-mag[i], -i))[:num_col]
    U = vecs[:, order]
    U = U - U.mean(axis=0, keepdims=True)
    return vals[order], U, float(D.sum())


def dcov_gamma_legacy(rx, ry, num_col=35):
    lx, Ux, tx = legacy_lowrank(rx, num_col)
    ly, Uy, ty = legacy_lowrank(ry, num_col)
    n = float(len(rx))
    C = Ux.T @ Uy
    stat = float(lx @ (C * C) @ ly) / n
    Cx = Ux.T @ Ux
    Cy = Uy.T @ Uy
    sx = float(lx @ (Cx * Cx) @ lx)
    sy = float(ly @ (Cy * Cy) @ ly)
    mean = (tx / (n * n)) * (ty / (n * n))
    var = _var_factor(n) * sx * sy / (n * n)
    return {"statistic": stat, "mean": mean, "variance": var, "p_value": _gamma_p(stat, mean, var)}


def dcc_gamma_decision_p(rx, ry, num_col=35, guard=(0.05, 0.15)):
    """The reference's dcc.gamma route: exact screen, legacy refinement in the
    guard band (fastkpc/src/full_cuda_ci_one_call.cpp:4985-5030)."""
    ex = dcov_gamma_exact(rx, ry)
    p = ex["p_value"]
    if guard[0] <= p <= guard[1]:
        return dcov_gamma_legacy(rx, ry, num_col)["p_value"], ex["p_value"], True
    return p, p, False


def inchol(r, sig, max_rank, tol=INCHOL_TOL):
    """kernlab-style incomplete Cholesky of the RBF Gram; returns G (n x rank)."""
    r = np.asarray(r, dtype=np.float64)
    n = len(r)
    sigma = 1.0 / sig
    diag = np.ones(n)
    G = np.zeros((n, max_rank))
    U = np.zeros((max_rank, max_rank))
    pivots = []
    pivot = 0
    residue = 1.0
    rank = 0
    while residue > tol and rank < max_rank:
        col = np.exp(-sigma * (r - r[pivot]) ** 2)
        tau2 = col[pivot]
        solve = np.zeros(rank)
        for row in range(rank):
            v = col[pivots[row]] - float(U[:row, row] @ solve[:row])
            solve[row] = v / U[row, row]
            tau2 -= solve[row] * solve[row]
            U[row, rank] = solve[row]
        if not (tau2 > 0.0) or not math.isfinite(tau2):
            break
        tau = math.sqrt(tau2)
        U[rank, rank] = tau
        upd = (col - G[:, :rank] @ solve) / tau
        G[:, rank] = upd
        diag -= upd * upd
        pivots.append(pivot)
        rank += 1
        pivot = int(np.argmax(diag))
        residue = float(diag[pivot])
    return G[:, :rank]


def hsic_components(r, sig, num_col):
    G = inchol(r, sig, num_col)
    cs = G.sum(axis=0)
    offdiag = float(np.sum(cs * cs) - np.sum(G * G))
    Gc = G - G.mean(axis=0, keepdims=True)
    K = Gc.T @ Gc
    return {"G": Gc, "offdiag": offdiag, "self": float(np.sum(K * K)), "rank": G.shape[1]}


def hsic_gamma(rx, ry, sig=1.0, num_col=35):
    cx, cy = hsic_components(rx, sig, num_col), hsic_components(ry, sig, num_col)
    n = float(len(rx))
    C = cx["G"].T @ cy["G"]
    stat = float(np.sum(C * C)) / (n * n)
    mux = cx["offdiag"] / (n * (n - 1.0))
    muy = cy["offdiag"] / (n * (n - 1.0))
    mean = (1.0 + mux * muy - mux - muy) / n
    var = _var_factor(n) * cx["self"] * cy["self"] / n ** 4
    q = _gamma_p(stat, mean, var)
    return {"statistic": stat, "mean": mean, "variance": var, "p_value": 1.0 - (1.0 - q)}


def hsic_perm(rx, ry, perms, sig=1.0, num_col=35):
    cx, cy = hsic_components(rx, sig, num_col), hsic_components(ry, sig, num_col)
    n = float(len(rx))
    Gx, Gy = cx["G"], cy["G"]
    C = Gx.T @ Gy
    obs = float(np.sum(C * C)) / (n * n)
    count = 1
    for pi in perms:
        C = Gx.T @ Gy[pi]
        if float(np.sum(C * C)) / (n * n) >= obs:
            count += 1
    return {"statistic": obs, "p_value": count / (len(perms) + 1.0)}


def dcc_perm(rx, ry, perms):
    Ax = dcov_components(rx)["A"]
    By = dcov_components(ry)["A"]
    n = float(len(rx))
    obs = float(np.sum(Ax * By)) / n
    count = 1
    for pi in perms:
        if float(np.sum(Ax * By[np.ix_(pi, pi)])) / n >= obs:
            count += 1
    return {"statistic": obs, "p_value": count / (len(perms) + 1.0)}
