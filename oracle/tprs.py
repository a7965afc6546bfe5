"""Thin-plate regression spline design for ``regrXonS`` (oracle).

TEST INFRASTRUCTURE ONLY: the CPU checker for the library's design setup.

Restates, in numpy, mgcv 1.9-1's ``s()`` thin-plate construction as the
reference's native setup re-implements it
(fastkpc/src/full_cuda_ci_native_setup.cpp):

* covariates shifted by their mean (:705-714), unique locations sorted
  lexicographically (:200-246);
* TPS radial kernel eta(r) and its constant (:114-152); polynomial null space
  of dimension M = C(m+d-1, d) with the power ordering of :168-198;
* the k eigenpairs of largest magnitude of E (dense symmetric eigen here;
  the reference runs Lanczos, :303), ordered by descending value;
* the T'U Householder constraint (``qt_householders`` :496-539) applied from
  the right to U*diag(values), the last M columns replaced by T (:760-778);
  the penalty diag(values) transformed the same way (:780-794);
* RMS column scaling (:796-811), penalty norm scaling (:821-834) and the
  sum-to-zero centering constraint absorbed by a one-column LINPACK-style
  Householder QR of the column means (:621-688);
* ``initial.sp`` (:1019-1127).

Eigenvector signs are made deterministic: each selected eigenvector is
flipped so that its largest-magnitude entry is positive (first on ties).
The fitted values of a penalised fit do not depend on the basis chosen for
the same space and penalty; only the optimizer's starting point does.

Model layouts (kpcalg/R/regrXonS.R:45-57): |S| = 1 -> s(x1) with k = 10;
|S| = 2 -> s(x1, x2) with k = 30; |S| > 2 -> s(x1) + ... + s(xk), k = 10
each.  Design width q = 1 + sum of (k - 1) per smooth.
"""
import math

import numpy as np

EPS = np.finfo(np.float64).eps


def r_mean(v):
    """R's mean(): long-double two-pass mean (a second pass adds the mean
    residual).  float64 is used here; the difference is below 1 ulp for the
    sizes involved."""
    v = np.asarray(v, dtype=np.float64)
    m = math.fsum(v) / len(v)
    corr = math.fsum(v - m) / len(v)
    return m + corr


def eta_constant(m, d):
    if 2 * m <= d:
        raise ValueError("thin plate spline requires 2m > d")
    pi = math.pi
    d2 = d // 2
    if d % 2 == 0:
        value = -1.0 if (m + 1 + d2) % 2 else 1.0
        for _ in range(2 * m - 1):
            value /= 2.0
        for _ in range(d2):
            value /= pi
        for i in range(2, m):
            value /= i
        for i in range(2, m - d2 + 1):
            value /= i
    else:
        value = math.sqrt(pi)
        k = m - (d - 1) // 2
        for i in range(k):
            value /= -0.5 - i
        for _ in range(m):
            value /= 4.0
        for _ in range(d2):
            value /= pi
        value /= math.sqrt(pi)
        for i in range(2, m):
            value /= i
    return value


def eta_of_r2(m, d, r2, eta0):
    r2 = np.asarray(r2, dtype=np.float64)
    out = np.zeros_like(r2)
    pos = r2 > 0
    d2 = d // 2
    v = np.full(np.count_nonzero(pos), eta0)
    rr = r2[pos]
    if d % 2 == 0:
        v = v * np.log(rr) * 0.5
        for _ in range(m - d2):
            v = v * rr
    else:
        for _ in range(m - d2 - 1):
            v = v * rr
        v = v * np.sqrt(rr)
    out[pos] = v
    return out


def default_order(d):
    m = 0
    while 2 * m < d + 2:
        m += 1
    return m


def null_space_dimension(d, m):
    dim = 1
    for i in range(d):
        dim *= d + m - 1 - i
    for i in range(2, d + 1):
        dim //= i
    return dim


def polynomial_powers(d, m, M):
    """powers[term][coord] following the reference enumeration order."""
    powers = np.zeros((M, d), dtype=np.int64)
    index = [0] * d
    for term in range(M):
        powers[term] = index
        s = sum(index)
        if s < m - 1:
            index[0] += 1
        else:
            s -= index[0]
            index[0] = 0
            for c in range(1, d):
                index[c] += 1
                s += 1
                if s == m:
                    s -= index[c]
                    index[c] = 0
                else:
                    break
    return powers


def sorted_unique(shifted):
    n, d = shifted.shape
    order = sorted(range(n), key=lambda r: (tuple(shifted[r]), r))
    uniq = []
    mapping = np.empty(n, dtype=np.int64)
    for idx in order:
        if not uniq or np.any(shifted[idx] != shifted[uniq[-1]]):
            uniq.append(idx)
        mapping[idx] = len(uniq) - 1
    return shifted[np.array(uniq)], mapping


def top_magnitude_eigen(E, k):
    """k eigenpairs of largest |value|, ordered by descending value."""
    vals, vecs = np.linalg.eigh(E)
    order = np.argsort(-np.abs(vals), kind="stable")[:k]
    order = order[np.argsort(-vals[order], kind="stable")]
    vals = vals[order]
    vecs = vecs[:, order].copy()
    for j in range(k):
        i = int(np.argmax(np.abs(vecs[:, j])))
        if vecs[i, j] < 0:
            vecs[:, j] = -vecs[:, j]
    return vals, vecs


def qt_householders(TU):
    """Householder vectors u_t (rows of Z) with TU H_0..H_{M-1} = [0 | L]."""
    TU = TU.copy()
    M, k = TU.shape
    Z = np.zeros((M, k))
    for step in range(M):
        L = k - step
        row = TU[step, :L]
        scale = np.max(np.abs(row))
        if scale != 0.0:
            TU[step, :L] = row / scale
        length = math.sqrt(float(np.dot(TU[step, :L], TU[step, :L])))
        if TU[step, L - 1] < 0.0:
            length = -length
        TU[step, L - 1] += length
        mult = 1.0 / (length * TU[step, L - 1]) if length != 0.0 else 0.0
        for r in range(step + 1, M):
            proj = mult * float(np.dot(TU[step, :L], TU[r, :L]))
            TU[r, :L] -= proj * TU[step, :L]
        Z[step, :L] = TU[step, :L] * math.sqrt(mult)
    return Z


def hq_post(X, Z):
    X = X.copy()
    for u in Z:
        X -= np.outer(X @ u, u)
    return X


def hq_pre_transpose(P, Z):
    P = P.copy()
    for u in Z:
        P -= np.outer(u, u @ P)
    return P


def absorb_centering(X, S):
    """Sum-to-zero constraint via a one-column Householder QR of colMeans(X)."""
    k = X.shape[1]
    c = np.array([r_mean(X[:, j]) for j in range(k)])
    nrm = float(np.linalg.norm(c))
    if nrm == 0.0:
        raise ValueError("centering constraint is rank deficient")
    if c[0] != 0.0:
        nrm = math.copysign(nrm, c[0])
    v = c / nrm
    v[0] += 1.0
    # H y = y - (v'y / v0) v ; H symmetric orthogonal with H c ~ e1
    H = np.eye(k) - np.outer(v, v) / v[0]
    XH = X @ H
    HSH = H @ S @ H
    return XH[:, 1:].copy(), HSH[1:, 1:].copy()


def build_smooth(cols, k):
    """One tp smooth of the columns ``cols`` (n x d) with basis dimension k.

    Returns dict(X=n x (k-1) absorbed basis, S=(k-1)x(k-1) penalty,
    rank=k-M)."""
    cols = np.asarray(cols, dtype=np.float64)
    if cols.ndim == 1:
        cols = cols[:, None]
    n, d = cols.shape
    m = default_order(d)
    M = null_space_dimension(d, m)
    shifts = np.array([r_mean(cols[:, j]) for j in range(d)])
    shifted = cols - shifts
    uniq, mapping = sorted_unique(shifted)
    nu = uniq.shape[0]
    if nu < k:
        raise ValueError("fewer unique locations than the basis dimension")
    if nu > 2000:
        raise ValueError("at most 2000 unique locations are supported")
    eta0 = eta_constant(m, d)
    diff = uniq[:, None, :] - uniq[None, :, :]
    r2 = np.sum(diff * diff, axis=2)
    E = eta_of_r2(m, d, r2, eta0)
    powers = polynomial_powers(d, m, M)
    T = np.ones((nu, M))
    for t in range(M):
        for c in range(d):
            T[:, t] *= uniq[:, c] ** powers[t, c]
    vals, U = top_magnitude_eigen(E, k)
    Z = qt_householders(T.T @ U)
    Xu = hq_post(U * vals[None, :], Z)
    Xu[:, k - M:] = T
    X = Xu[mapping]
    P = hq_pre_transpose(hq_post(np.diag(vals), Z), Z)
    P[:, k - M:] = 0.0
    P[k - M:, :] = 0.0
    rms = np.sqrt(np.sum(X * X, axis=0) / n)
    if np.any(~np.isfinite(rms)) or np.any(rms == 0.0):
        raise ValueError("zero column in RMS scaling")
    X = X / rms[None, :]
    P = P / rms[:, None] / rms[None, :]
    Ps = (P + P.T) / 2.0
    x_norm = np.max(np.sum(np.abs(X), axis=1))
    p_norm = np.max(np.sum(np.abs(Ps), axis=0))
    Ps = Ps / (p_norm / (x_norm * x_norm))
    Xa, Sa = absorb_centering(X, Ps)
    return {"X": Xa, "S": Sa, "rank": k - M}


def initial_sp(X, blocks, offsets):
    """mgcv initial.sp: size ratio per penalty, then scale by powers of ten
    until the mean of diag(X'X) / (diag(X'X) + diag(sum S)) crosses 0.4."""
    q = X.shape[1]
    xdiag = np.array([math.fsum(X[:, j] * X[:, j]) for j in range(q)])
    pdiag = np.zeros(q)
    penalized = np.zeros(q, dtype=bool)
    thr_scale = EPS ** 0.8
    result = []
    for S, off in zip(blocks, offsets):
        dim = S.shape[0]
        A = np.abs(S)
        thr = thr_scale * A.max()
        active = []
        for c in range(dim):
            rm = r_mean(A[c, :])
            cm = r_mean(A[:, c])
            if rm > thr and cm > thr and A[c, c] > thr:
                active.append(c)
        if not active:
            raise ValueError("initial.sp found no active coordinates")
        sx = r_mean(xdiag[off + np.array(active)])
        sp = r_mean(np.array([S[c, c] for c in active]))
        lam = sx / sp
        result.append(lam)
        penalized[off + np.array(active)] = True
        pdiag[off:off + dim] += lam * np.diag(S)
    result = np.array(result)
    used = (pdiag > 0) & penalized & (xdiag > 0)

    def mean_hat():
        return r_mean(xdiag[used] / (xdiag[used] + pdiag[used]))

    guard = 0
    while mean_hat() > 0.4:
        result *= 10.0
        pdiag *= 10.0
        guard += 1
        if guard > 1000:
            raise ValueError("initial.sp did not bracket 0.4")
    while mean_hat() < 0.4:
        result /= 10.0
        pdiag /= 10.0
        guard += 1
        if guard > 2000:
            raise ValueError("initial.sp did not bracket 0.4")
    return result


def design(data, S):
    """regrXonS design for conditioning columns S of ``data`` (n x p).

    Returns dict(X n x q, blocks [S_j], offsets [o_j], ranks [r_j],
    initial_sp [lambda_j])."""
    S = list(S)
    n = data.shape[0]
    if len(S) == 0:
        raise ValueError("empty conditioning set has no design")
    if len(S) <= 2:
        smooths = [build_smooth(data[:, S], 10 if len(S) == 1 else 30)]
    else:
        smooths = [build_smooth(data[:, s], 10) for s in S]
    q = 1 + sum(sm["X"].shape[1] for sm in smooths)
    if q >= n:
        raise ValueError("design width must be below n")
    X = np.empty((n, q))
    X[:, 0] = 1.0
    blocks, offsets, ranks = [], [], []
    dest = 1
    for sm in smooths:
        w = sm["X"].shape[1]
        X[:, dest:dest + w] = sm["X"]
        blocks.append(sm["S"])
        offsets.append(dest)
        ranks.append(sm["rank"])
        dest += w
    return {"X": X, "blocks": blocks, "offsets": offsets, "ranks": ranks,
            "initial_sp": initial_sp(X, blocks, offsets)}
