"""GCV smoothing-parameter selection and residuals for ``regrXonS`` (oracle).

TEST INFRASTRUCTURE ONLY: the CPU checker for the library's fit kernels.

GCV score V(rho) = n * RSS / (n - EDF)^2 in rho = log(lambda), minimised by
mgcv ``magic``'s Newton scheme as the reference restates it:

* single penalty (|S| <= 2): spectral form.  With X'X = U'U and the whitened
  penalty U^-T S U^-1 = W diag(e) W', the hat values are h_k = 1/(1+lambda e_k)
  and z = W' U^-T X' y, so RSS = |y|^2 - 2 sum h z^2 + sum h^2 z^2 and
  EDF = sum h (fastkpc/src/full_cuda_ci_one_call.cpp:1869-1947 geometry;
  fastkpc/src/cuda/mgcv_single_penalty_gcv.cu:189-283 objective and
  :1479-1700 optimizer: 15 step halvings, 400 iterations, |step| <= 5,
  tolerance 1e-7, boundary probes of +-2 up to 5 times, flat-objective stop).
* several penalties (|S| > 2): augmented SVD form.  [R; B] = U D V' with
  X = QR and B'B = sum lambda_j S_j; singular values below d_0 * sqrt(eps)
  are dropped; U1 = top q rows of U; y1 = U1' Q'y;
  RSS = |y|^2 - 2|y1|^2 + |U1 y1|^2, EDF = |U1|_F^2, with the analytic
  gradient and Hessian in rho (fastkpc/src/mgcv_multi_penalty_cpp.cpp:732-975)
  and the Newton loop of :1124-1346 (25 step halvings, steepest descent after
  the third rejected Newton trial or when the Hessian has a negative
  eigenvalue, boundary probes).

Residuals at the selected lambda use the same augmented SVD
(``refine_multi_penalty_selected_fit``, :977-1029).
"""
import math

import numpy as np
from scipy.linalg import solve_triangular

EPS = np.finfo(np.float64).eps
RANK_TOL = math.sqrt(EPS)  # 1.4901161193847656e-8
CONV_TOL = 1e-7
POLISH_STEPS = 4
POLISH_MAX_STEP = 1e-6
POLISH_DONE = 1e-10
POLISH_CURVATURE = 1e-6


class Prepared:
    """Per-design quantities shared by every target fitted on that design."""

    def __init__(self, des):
        X = des["X"]
        self.X = X
        self.n, self.q = X.shape
        self.blocks = des["blocks"]
        self.offsets = des["offsets"]
        self.ranks = des["ranks"]
        self.m = len(self.blocks)
        self.initial_sp = np.asarray(des["initial_sp"], dtype=np.float64)
        self.Q, self.R = np.linalg.qr(X)
        # penalty roots placed in the full coefficient space: root root' = S_j
        self.roots = []
        for S, off, r in zip(self.blocks, self.offsets, self.ranks):
            w, v = np.linalg.eigh((S + S.T) / 2.0)
            order = np.argsort(-w)[:r]
            root = np.zeros((self.q, r))
            root[off:off + S.shape[0], :] = v[:, order] * np.sqrt(np.maximum(w[order], 0.0))
            self.roots.append(root)
        if self.m == 1:
            self._single_geometry()

    def _single_geometry(self):
        q = self.q
        S = np.zeros((q, q))
        off = self.offsets[0]
        b = self.blocks[0]
        S[off:off + b.shape[0], off:off + b.shape[0]] = b
        # whitening by the R factor of X (X'X = R'R) keeps the condition of X
        # (the reference whitens with the Cholesky factor of X'X: the same
        # spectrum, with the condition number squared)
        Ui = np.linalg.solve(self.R, np.eye(q))
        W = Ui.T @ S @ Ui
        W = 0.5 * (W + W.T)
        vals, vecs = np.linalg.eigh(W)
        vals = vals[::-1].copy()
        vecs = vecs[:, ::-1].copy()
        vals = np.maximum(vals, 0.0)
        vals[self.ranks[0]:] = 0.0
        self.spec_values = vals
        self.rhs_transform = vecs.T @ Ui.T

    def response(self, y):
        y = np.asarray(y, dtype=np.float64)
        y0 = self.Q.T @ y
        e0 = y - self.Q @ y0
        # rss0 = |y - Q Q'y|^2: the part of y outside the design's span, summed
        # directly so RSS never comes from |y|^2 minus a nearly equal quantity
        out = {"y": y, "y0": y0, "yy": float(np.dot(y, y)), "rss0": float(np.dot(e0, e0))}
        if self.m == 1:
            out["z"] = self.rhs_transform @ (self.X.T @ y)
        return out


# ---------------------------------------------------------------- single

def _hat(log_sp, e):
    if e == 0.0:
        return 1.0
    c = log_sp + math.log(e)
    if c >= 0.0:
        v = math.exp(-c)
        return v / (1.0 + v)
    return 1.0 / (1.0 + math.exp(c))


def single_objective(log_sp, e, z, rss0, n):
    """GCV pieces at log_sp; RSS = rss0 + sum (1 - h_k)^2 z_k^2 (|z| = |Q'y|)."""
    lin = edf = rg = rh = dg = dh = 0.0
    for ek, zk in zip(e, z):
        h = _hat(log_sp, ek)
        z2 = zk * zk
        omh = 1.0 - h
        w = h * omh
        lin += omh * omh * z2
        edf += h
        rg += 2.0 * h * omh * omh * z2
        rh += 2.0 * h * omh * omh * (3.0 * h - 1.0) * z2
        dg += w
        dh -= w * (1.0 - 2.0 * h)
    rss = rss0 + lin
    rdf = n - edf
    if not (math.isfinite(rss) and math.isfinite(edf)) or rss <= 0.0 or rdf <= 1e-8:
        return {"valid": False, "rss": rss, "edf": edf, "score": math.inf}
    score = n * rss / (rdf * rdf)
    lg = rg / rss - 2.0 * dg / rdf
    lh = rh / rss - (rg / rss) ** 2 - 2.0 * (dh / rdf - (dg / rdf) ** 2)
    return {"valid": True, "rss": rss, "edf": edf, "score": score,
            "gradient": score * lg, "hessian": score * (lh + lg * lg)}


def optimize_single(prep, resp):
    e = prep.spec_values
    z = resp["z"]
    rss0 = resp["rss0"]
    n = prep.n
    max_half = 15
    log_sp = math.log(prep.initial_sp[0])
    cur = single_objective(log_sp, e, z, rss0, n)
    if not cur["valid"]:
        raise ValueError("non-finite single-penalty objective")
    min_score = cur["score"]
    score_red = 1e10
    steepest = False
    prior_grad = math.nan
    newton = 0.0
    steep = 0.0
    it = 0
    calls = 1
    converged = False
    flat = False
    while not converged and it < 400:
        it += 1
        try_step = it > 1
        tries = 0
        step = steep if steepest else newton
        src_newton = not steepest
        it_flat = False
        while try_step:
            tries += 1
            if tries == 4 and not steepest:
                steepest = True
                step = steep
                src_newton = False
            trial_ls = log_sp + step
            trial = single_objective(trial_ls, e, z, rss0, n)
            calls += 1
            pred = cur["gradient"] * step + 0.5 * cur["hessian"] * step * step
            resolution = 8.0 * EPS * (1.0 + abs(min_score))
            unresolved = src_newton and math.isfinite(pred) and pred <= 0.0 and abs(pred) <= resolution
            accepted = trial["valid"] and trial["score"] < min_score
            if accepted:
                try_step = False
                score_red = min_score - trial["score"]
                min_score = trial["score"]
                log_sp = trial_ls
                cur = trial
            elif unresolved:
                try_step = False
                it_flat = True
                flat = True
            else:
                step /= 2.0
            if tries == max_half - 1 and try_step:
                step = 0.0
            if tries == max_half:
                try_step = False
        if it > 3:
            converged = True
            if score_red > CONV_TOL * (1.0 + min_score):
                converged = False
            if abs(prior_grad) > CONV_TOL ** (1.0 / 3.0) * (1.0 + abs(min_score)):
                converged = False
            if tries == max_half:
                converged = True
            if it_flat:
                converged = True
        prior_grad = cur["gradient"]
        steepest = cur["hessian"] < 0.0
        if not steepest:
            newton = -cur["gradient"] / cur["hessian"]
            if abs(newton) > 5.0:
                newton = math.copysign(5.0, newton)
        steep = 0.0 if cur["gradient"] == 0.0 else -cur["gradient"] / abs(cur["gradient"])
    if not converged:
        raise ValueError("single-penalty optimizer hit its iteration limit")
    direction = 1.0 if cur["gradient"] < 0.0 else -1.0
    for _ in range(5):
        trial_ls = log_sp + direction * 2.0
        trial = single_objective(trial_ls, e, z, rss0, n)
        calls += 1
        if not (trial["valid"] and trial["score"] < min_score):
            break
        log_sp = trial_ls
        cur = trial
        min_score = trial["score"]
    # terminal Newton polish to the stationary point (see polish_newton)
    for _ in range(POLISH_STEPS):
        if not (cur["valid"] and cur["hessian"] > POLISH_CURVATURE * cur["score"]):
            break
        step = -cur["gradient"] / cur["hessian"]
        if abs(step) > POLISH_MAX_STEP:
            break
        log_sp = log_sp + step
        cur = single_objective(log_sp, e, z, rss0, n)
        calls += 1
        if abs(step) <= POLISH_DONE:
            break
    return {"log_sp": np.array([log_sp]), "score": cur["score"], "rss": cur["rss"],
            "edf": cur["edf"], "iterations": it, "calls": calls}


# ---------------------------------------------------------------- multi

def _augmented_svd(prep, log_sp):
    lam = np.exp(log_sp)
    B = np.vstack([math.sqrt(l) * r.T for l, r in zip(lam, prep.roots)])
    A = np.vstack([prep.R, B])
    U, d, Vt = np.linalg.svd(A, full_matrices=False)
    r = int(np.count_nonzero(d >= d[0] * RANK_TOL))
    return U[:prep.q, :r], Vt[:r, :].T, d[:r], lam


def multi_core(prep, resp, log_sp):
    U1, V, d, lam = _augmented_svd(prep, log_sp)
    y1 = U1.T @ resp["y0"]
    Uy = U1 @ y1
    d0 = resp["y0"] - Uy
    rss = resp["rss0"] + float(d0 @ d0)
    edf = float(np.sum(U1 * U1))
    delta = prep.n - edf
    if not (math.isfinite(rss) and math.isfinite(edf)) or delta <= 1e-8:
        raise ValueError("invalid multi-penalty objective")
    score = prep.n * rss / (delta * delta)
    return {"U1": U1, "V": V, "d": d, "lam": lam, "y1": y1, "rss": rss,
            "edf": edf, "score": score, "log_sp": np.array(log_sp, dtype=np.float64)}


def multi_derivatives(prep, core):
    """Analytic gradient and Hessian of V in rho = log(lambda)."""
    U1, V, d, lam, y1 = core["U1"], core["V"], core["d"], core["lam"], core["y1"]
    m = prep.m
    P = U1.T @ U1
    Ms = []
    for root in prep.roots:
        T = (V.T @ root) / d[:, None]
        Ms.append(T @ T.T)
    e1 = y1 - P @ y1
    ddelta = np.array([lam[i] * np.trace(Ms[i] @ P) for i in range(m)])
    drss = np.array([2.0 * lam[i] * float(e1 @ (Ms[i] @ y1)) for i in range(m)])
    d2delta = np.zeros((m, m))
    d2rss = np.zeros((m, m))
    My = [M @ y1 for M in Ms]
    for i in range(m):
        for j in range(i + 1):
            MiMj = Ms[i] @ Ms[j]
            dd = -2.0 * lam[i] * lam[j] * np.trace(MiMj @ P)
            rr = 2.0 * lam[i] * lam[j] * (float(My[j] @ (P @ My[i]))
                                          - float(e1 @ (MiMj @ y1)) - float(e1 @ (Ms[j] @ My[i])))
            if i == j:
                dd += ddelta[i]
                rr += drss[i]
            d2delta[i, j] = d2delta[j, i] = dd
            d2rss[i, j] = d2rss[j, i] = rr
    n = prep.n
    delta = n - core["edf"]
    rss = core["rss"]
    s1 = n / (delta * delta)
    s2 = 2.0 * s1 * rss / delta
    grad = s1 * drss - s2 * ddelta
    hess = np.zeros((m, m))
    for i in range(m):
        for j in range(i + 1):
            v = (-2.0 * s1 / delta * (ddelta[j] * drss[i] + ddelta[i] * drss[j])
                 + s1 * d2rss[i, j] + 3.0 * s2 / delta * ddelta[i] * ddelta[j]
                 - s2 * d2delta[i, j])
            hess[i, j] = hess[j, i] = v
    return grad, hess


def optimize_multi(prep, resp, max_half=25):
    m = prep.m
    log_sp = np.log(prep.initial_sp)
    cur = multi_core(prep, resp, log_sp)
    grad_c, hess_c = multi_derivatives(prep, cur)
    min_score = cur["score"]
    score_red = 1e10
    gradient = np.zeros(m)
    newton = np.zeros(m)
    steep = np.zeros(m)
    steepest = False
    converged = False
    calls = 1
    it = 0
    for it in range(1, 401):
        tries = 0
        if it > 1:
            step = (steep if steepest else newton).copy()
            trying = True
            while trying:
                tries += 1
                if tries == 4 and not steepest:
                    steepest = True
                    step = steep.copy()
                trial_ls = log_sp + step
                trial = multi_core(prep, resp, trial_ls)
                calls += 1
                if trial["score"] < min_score:
                    trying = False
                    score_red = min_score - trial["score"]
                    min_score = trial["score"]
                    log_sp = trial_ls
                    cur = trial
                    grad_c, hess_c = multi_derivatives(prep, cur)
                else:
                    step = step / 2.0
                if tries == max_half - 1 and trying:
                    step = np.zeros(m)
                if tries == max_half:
                    trying = False
        if it > 3:
            gnorm = float(np.sqrt(np.sum(gradient * gradient)))
            converged = (score_red <= CONV_TOL * (1.0 + min_score)
                         and gnorm <= CONV_TOL ** (1.0 / 3.0) * (1.0 + abs(min_score)))
            if tries == max_half:
                converged = True
        gradient = grad_c.copy()
        w, v = np.linalg.eigh(hess_c)
        steepest = bool(np.any(w < 0.0))
        if not steepest:
            newton = -(v @ ((v.T @ gradient) / w))
            mx = np.max(np.abs(newton))
            if mx > 5.0:
                newton = newton * (5.0 / mx)
        mg = np.max(np.abs(gradient))
        steep = np.zeros(m) if mg == 0.0 else -gradient / mg
        if converged:
            break
    if not converged:
        raise ValueError("multi-penalty optimizer hit its iteration limit")
    for c in range(m):
        direction = 1.0 if gradient[c] < 0.0 else -1.0
        for _ in range(5):
            step = np.zeros(m)
            step[c] = direction * 2.0
            trial_ls = log_sp + step
            trial = multi_core(prep, resp, trial_ls)
            calls += 1
            if not trial["score"] < min_score:
                break
            log_sp = trial_ls
            cur = trial
            min_score = cur["score"]
    log_sp, cur, extra = polish_newton(prep, resp, log_sp, cur)
    calls += extra
    return {"log_sp": log_sp, "score": cur["score"], "rss": cur["rss"],
            "edf": cur["edf"], "iterations": it, "calls": calls}


def qr_core(prep, resp, log_sp):
    """V at rho through the Householder factor of the stacked system.

    Ra (LAPACK QR of [R; B], B the sqrt(lambda)-scaled penalty roots) has
    Ra'Ra = X'X + S_lambda; W = R Ra^-1, EDF = |W|_F^2, g = W'y0,
    RSS = rss0 + |y0 - W g|^2.  Householder QR keeps each column's relative
    accuracy however the rows are scaled, while the SVD of the same stack is
    accurate only relative to its largest singular value (about sqrt(lambda)):
    with one smooth near lambda = e^25 the SVD route's gradient carries
    relative errors near 1e-12 and this one near 1e-15.  Used for the terminal
    polish, whose purpose is the stationary point itself."""
    lam = np.exp(np.asarray(log_sp, dtype=np.float64))
    B = np.vstack([math.sqrt(l) * r.T for l, r in zip(lam, prep.roots)])
    Ra = np.linalg.qr(np.vstack([prep.R, B]), mode="r")
    Wt = solve_triangular(Ra, prep.R.T, trans="T")  # W' = Ra^-T R'
    W = Wt.T
    y0 = resp["y0"]
    g = Wt @ y0
    Wg = W @ g
    d0 = y0 - Wg
    rss = resp["rss0"] + float(d0 @ d0)
    edf = float(np.sum(W * W))
    delta = prep.n - edf
    if not (math.isfinite(rss) and math.isfinite(edf)) or delta <= 1e-8:
        raise ValueError("invalid multi-penalty objective")
    return {"Ra": Ra, "W": W, "g": g, "Wg": Wg, "lam": lam, "rss": rss, "edf": edf,
            "score": prep.n * rss / (delta * delta), "log_sp": np.array(log_sp, dtype=np.float64)}


def qr_derivatives(prep, core):
    """Gradient and Hessian of V in rho from qr_core's factor.

    With T = Ra^-T [root_1 .. root_m], a = T'g, b = T'(g - W'W g),
    C = T'T and D = (WT)'(WT): d delta_j = lam_j sum_{a in j} D_aa,
    d rss_j = 2 lam_j sum_{a in j} a_a b_a, and the second derivatives are the
    block sums sum C.D, a'Da, b'Ca, a'Cb over each pair of penalty blocks --
    the quantities of multi_derivatives in the Householder basis."""
    lam, W, g = core["lam"], core["W"], core["g"]
    m = prep.m
    roots = np.hstack(prep.roots)
    blk = np.concatenate([np.full(r.shape[1], j) for j, r in enumerate(prep.roots)])
    T = solve_triangular(core["Ra"], roots, trans="T")
    e1 = g - W.T @ core["Wg"]
    a = T.T @ g
    b = T.T @ e1
    WT = W @ T
    C = T.T @ T
    D = WT.T @ WT
    sel = [blk == j for j in range(m)]
    ddelta = np.array([lam[j] * float(np.sum(np.diag(D)[sel[j]])) for j in range(m)])
    drss = np.array([2.0 * lam[j] * float(np.sum(a[sel[j]] * b[sel[j]])) for j in range(m)])
    d2delta = np.zeros((m, m))
    d2rss = np.zeros((m, m))
    for i in range(m):
        for j in range(i + 1):
            Cij = C[np.ix_(sel[i], sel[j])]
            Dij = D[np.ix_(sel[i], sel[j])]
            ai, aj, bi, bj = a[sel[i]], a[sel[j]], b[sel[i]], b[sel[j]]
            ll = lam[i] * lam[j]
            dd = -2.0 * ll * float(np.sum(Cij * Dij))
            rr = 2.0 * ll * (float(ai @ Dij @ aj) - float(bi @ Cij @ aj) - float(ai @ Cij @ bj))
            if i == j:
                dd += ddelta[i]
                rr += drss[i]
            d2delta[i, j] = d2delta[j, i] = dd
            d2rss[i, j] = d2rss[j, i] = rr
    n = prep.n
    delta = n - core["edf"]
    rss = core["rss"]
    s1 = n / (delta * delta)
    s2 = 2.0 * s1 * rss / delta
    grad = s1 * drss - s2 * ddelta
    hess = np.zeros((m, m))
    for i in range(m):
        for j in range(i + 1):
            v = (-2.0 * s1 / delta * (ddelta[j] * drss[i] + ddelta[i] * drss[j])
                 + s1 * d2rss[i, j] + 3.0 * s2 / delta * ddelta[i] * ddelta[j]
                 - s2 * d2delta[i, j])
            hess[i, j] = hess[j, i] = v
    return grad, hess


def polish_newton(prep, resp, log_sp, cur):
    """Terminal Newton polish of the selected point.

    Magic's stopping rule leaves the selected rho determined only to about the
    convergence tolerance, so two correct implementations can stop 1e-7 apart.
    Up to POLISH_STEPS Newton steps on the coordinates whose curvature exceeds
    POLISH_CURVATURE * V (smooths pushed to the boundary have none and stay
    put) move the point to the stationary point itself; a step larger than
    POLISH_MAX_STEP, or a sub-Hessian that is not positive definite, leaves the
    point as selected.  The derivatives come from qr_core / qr_derivatives,
    accurate where a smooth sits at a very large lambda.
    Returns (rho, core, evaluations)."""
    extra = 0
    cur = qr_core(prep, resp, log_sp)
    for _ in range(POLISH_STEPS):
        g, H = qr_derivatives(prep, cur)
        act = [j for j in range(prep.m) if H[j, j] > POLISH_CURVATURE * cur["score"]]
        if not act:
            break
        Ha = H[np.ix_(act, act)]
        try:
            L = np.linalg.cholesky(Ha)
        except np.linalg.LinAlgError:
            break
        d = -np.linalg.solve(L.T, np.linalg.solve(L, g[act]))
        if np.max(np.abs(d)) > POLISH_MAX_STEP:
            break
        log_sp = log_sp.copy()
        log_sp[act] += d
        cur = qr_core(prep, resp, log_sp)
        extra += 1
        if np.max(np.abs(d)) <= POLISH_DONE:
            break
    return log_sp, cur, extra


def residual_at(prep, resp, log_sp):
    """y - A(lambda) y through the augmented SVD."""
    core = multi_core(prep, resp, np.asarray(log_sp, dtype=np.float64))
    fitted = prep.Q @ (core["U1"] @ core["y1"])
    return resp["y"] - fitted


def fit(prep, y):
    """Select lambda by GCV and return (residual, info)."""
    resp = prep.response(y)
    info = optimize_single(prep, resp) if prep.m == 1 else optimize_multi(prep, resp)
    return residual_at(prep, resp, info["log_sp"]), info


def gcv_value_grad_hess(prep, y, log_sp):
    """V, analytic gradient and full Hessian at rho (multi or single)."""
    resp = prep.response(y)
    core = multi_core(prep, resp, np.asarray(log_sp, dtype=np.float64))
    g, H = multi_derivatives(prep, core)
    return core["score"], g, H


def gcv_gauss_newton(prep, y, log_sp):
    """Gauss-Newton Hessian of V in rho, from the normal equations.

    V = |f|^2 with f(rho) = sqrt(n) r / delta, r = y - X beta(rho),
    beta = (X'X + S_lambda)^-1 X'y, delta = n - EDF.  GN = 2 J'J with
    J_j = sqrt(n) (dr_j / delta - r ddelta_j / delta^2),
    dr_j = lambda_j X (X'X + S_lambda)^-1 S_j beta, and
    ddelta_j = lambda_j tr((X'X + S)^-1 S_j (X'X + S)^-1 X'X).
    A restatement independent of the augmented-SVD path (dense solves);
    the adjoint routine's GN block (no reference counterpart: the reference
    uses the exact Hessian, fastkpc/src/cuda/mgcv_multi_penalty_gcv.cu:1410-1490)
    is checked against it and against finite differences of f.
    """
    X = prep.X
    n = prep.n
    lam = np.exp(np.asarray(log_sp, dtype=np.float64))
    Ss = [r @ r.T for r in prep.roots]
    XtX = X.T @ X
    A = XtX + sum(l * S for l, S in zip(lam, Ss))
    Ainv = np.linalg.inv(A)
    beta = Ainv @ (X.T @ y)
    r = y - X @ beta
    edf = float(np.trace(Ainv @ XtX))
    delta = n - edf
    J = np.zeros((n, prep.m))
    for j, (l, S) in enumerate(zip(lam, Ss)):
        dr = l * (X @ (Ainv @ (S @ beta)))
        dd = l * float(np.trace(Ainv @ S @ Ainv @ XtX))
        J[:, j] = math.sqrt(n) * (dr / delta - r * dd / (delta * delta))
    return 2.0 * J.T @ J


def gcv_residual_vector(prep, y, log_sp):
    """f(rho) = sqrt(n) r / (n - EDF), whose squared norm is V (augmented SVD)."""
    resp = prep.response(y)
    core = multi_core(prep, resp, np.asarray(log_sp, dtype=np.float64))
    fitted = prep.Q @ (core["U1"] @ core["y1"])
    return math.sqrt(prep.n) * (y - fitted) / (prep.n - core["edf"])


GN_GRAD_TOL = 1e-9
GN_FLAT_TOL = 1e-12
GN_STALL_TOL = 1e-9    # a decrease of V at most this (1 + V): the direction has stalled
GN_FLAT_GRAD = 1e-6
GN_MAX_LOG_SP = 25.0


def _solve_free(A, g, fixed, mu=0.0):
    """-(A + mu I)^-1 g on the free coordinates (Cholesky), 0 on the fixed."""
    free = ~fixed
    z = np.zeros(len(g))
    if free.any():
        Af = A[np.ix_(free, free)] + mu * np.eye(int(free.sum()))
        L = np.linalg.cholesky(Af)
        z[free] = np.linalg.solve(L.T, np.linalg.solve(L, -g[free]))
    return z


def _gn_solve(hess, gn, grad, fixed):
    try:
        return _solve_free(hess, grad, fixed)
    except np.linalg.LinAlgError:
        pass
    dmax = float(np.max(np.abs(np.diag(gn))))
    mu = 0.0
    for _ in range(12):
        try:
            return _solve_free(gn, grad, fixed, mu)
        except np.linalg.LinAlgError:
            mu = 1e-12 * max(dmax, 1e-300) if mu == 0.0 else mu * 100.0
    return None


def newton_gn_step(hess, gn, grad, rho):
    """Step of the adjoint-driven selection: Newton on the exact Hessian when
    it is positive definite, else damped Gauss-Newton; projected on the bound
    rho <= GN_MAX_LOG_SP (coordinates on the bound whose step points outwards
    are fixed and the rest re-solved); capped at 5 in max norm; clipped to
    the bound."""
    m = len(grad)
    fixed = np.zeros(m, dtype=bool)
    z = _gn_solve(hess, gn, grad, fixed)
    if z is not None:
        fixed = (rho >= GN_MAX_LOG_SP) & (z > 0.0)
        if fixed.any():
            z = _gn_solve(hess, gn, grad, fixed)
    if z is None:
        mg = float(np.max(np.abs(grad)))
        z = np.zeros(m) if mg == 0.0 else -grad / mg
    mx = float(np.max(np.abs(z)))
    if mx > 5.0:
        z = z * (5.0 / mx)
    return np.minimum(z, GN_MAX_LOG_SP - rho)


def steepest_gn_step(grad, rho):
    """Projected steepest descent for a stalled Gauss-Newton search: -g /
    max|g| over the coordinates that no outward push holds at the bound
    rho <= GN_MAX_LOG_SP, clipped to the bound."""
    free = ~((rho >= GN_MAX_LOG_SP) & (grad < 0.0))
    g = np.where(free, grad, 0.0)
    mg = float(np.max(np.abs(g)))
    z = np.zeros(len(g)) if mg == 0.0 else -g / mg
    return np.minimum(z, GN_MAX_LOG_SP - rho)


def optimize_gn(prep, y, max_half=25, max_iter=400, trace=None):
    """Newton selection driven by the adjoint (the library's
    FKPC_SELECT_GN_NEWTON): from magic's start, exact-Hessian Newton where that
    Hessian is positive definite and damped Gauss-Newton elsewhere, halving
    until V decreases; after a decrease of at most GN_STALL_TOL (1 + V) the
    next step is projected steepest descent (steepest_gn_step); stop at
    |grad V| <= GN_GRAD_TOL (1 + V), when no decrease is possible, or after
    two such small decreases in a row, with log(lambda) kept <=
    GN_MAX_LOG_SP; then the
    terminal polish (no boundary probes)."""
    resp = prep.response(y)
    m = prep.m
    rho = np.log(prep.initial_sp)
    core = multi_core(prep, resp, rho)
    g, H = multi_derivatives(prep, core)
    gn = gcv_gauss_newton(prep, y, rho)
    calls = 1
    converged = False
    it = 0
    stalled = False
    for it in range(1, max_iter + 1):
        step = steepest_gn_step(g, rho) if stalled else newton_gn_step(H, gn, g, rho)
        accepted = None
        for _ in range(max_half):
            trial = rho + step
            c2 = multi_core(prep, resp, trial)
            calls += 1
            if c2["score"] < core["score"]:
                accepted = c2
                break
            step = step * 0.5
        if trace is not None:
            trace.append((it, core["score"], np.linalg.norm(g), rho.copy(), step.copy(), accepted is not None))
        if accepted is None:
            converged = True
            break
        red = core["score"] - accepted["score"]
        rho, core = accepted["log_sp"], accepted
        g, H = multi_derivatives(prep, core)
        gn = gcv_gauss_newton(prep, y, rho)
        gnorm = np.linalg.norm(np.where((rho >= GN_MAX_LOG_SP) & (g < 0.0), 0.0, g))  # projected gradient
        if (gnorm <= GN_GRAD_TOL * (1.0 + abs(core["score"]))
                or (red <= GN_FLAT_TOL * (1.0 + core["score"]) and gnorm <= GN_FLAT_GRAD * (1.0 + abs(core["score"])))):
            converged = True
            break
        # a decrease below GN_STALL_TOL (1 + V): the next step is projected
        # steepest descent; a second such decrease in a row ends the search
        tiny = red <= GN_STALL_TOL * (1.0 + core["score"])
        if tiny and stalled:
            converged = True
            break
        stalled = tiny
    if not converged:
        raise ValueError("Gauss-Newton selection hit its iteration limit")
    rho, core, extra = polish_newton(prep, resp, rho, core)
    calls += extra
    return {"log_sp": rho, "score": core["score"], "iterations": it, "calls": calls}
