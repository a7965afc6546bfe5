"""Per-stage error of a GPU level batch against the oracle fixture.

``level500x50_oracle.npz`` (written by ``make_level_fixture.py``) holds the
oracle's records for all 4096 triples of the 500 x 50 level batch and its
residual summaries for all 6005 fits.  ``report`` measures, stage by stage:

* fit: selected log smoothing parameters (max |difference|, over all entries
  and over those below 15, which the GCV curvature pins down); residuals --
  the max-abs error relative to max |r| on the fits stored in full, and over
  every fit the Cauchy-Schwarz bound |(r - r_o) . z_k| / (|r_o| |z_k|) of
  four fixed projections plus the relative error of |r|^2;
* statistic: relative error of the statistic, mean and variance (dcc.gamma
  against the exact or, in the guard band, the low-rank oracle value);
* p-value: max absolute error of the exact-screen p, of the guard-band p and
  of the decision p; alpha-boundary flips (p >= alpha on one side only) and
  guard-band routing flips.

Used by the GPU parity test and by ``bench.py`` (data only; no oracle code
runs).
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "level500x50_oracle.npz")
ALPHA = 0.1


def load(path=FIXTURE):
    with np.load(path) as f:
        return {k: f[k] for k in f.files}


def triples(fx):
    return [(int(x), int(y), [int(v) for v in s if v >= 0]) for x, y, s in zip(fx["x"], fx["y"], fx["S"])]


def fits(fx):
    return [(int(t), [int(v) for v in s if v >= 0]) for t, s in zip(fx["fit_target"], fx["fit_S"])]


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if len(b) else 0.0


AGREE_LOG_SP = 1e-11


def fit_agreement(fx, log_sp):
    """Per fit: True when the GPU's selected log(lambda) equals the oracle's to
    AGREE_LOG_SP on every entry the GCV curvature pins down (|entry| < 15)."""
    ref = fx["fit_log_sp"]
    got = log_sp[:, :ref.shape[1]]
    det = np.isfinite(ref) & (np.abs(ref) < 15.0)
    diff = np.where(det, np.abs(got - np.where(det, ref, 0.0)), 0.0)
    return np.max(diff, axis=1) <= AGREE_LOG_SP


def triple_agreement(fx, fit_agree):
    """Per triple: both residual fits agree (a direct |S| = 0 side always does)."""
    index = {key: i for i, key in enumerate((t, tuple(S)) for t, S in fits(fx))}
    out = np.ones(len(fx["x"]), dtype=bool)
    for k, (x, y, S) in enumerate(triples(fx)):
        if S:
            out[k] = bool(fit_agree[index[(x, tuple(S))]] and fit_agree[index[(y, tuple(S))]])
    return out


def report(fx, dcc=None, hsic=None, residuals=None, log_sp=None):
    """Errors of the GPU records / residuals against the fixture (dict).

    With ``log_sp`` and records, the p errors are also reported over the
    triples whose fits both land on the oracle's point (``*_agreeing``):
    elsewhere magic stopped outside its Newton region, where two
    implementations' searches end up to ~1e-9 apart in log(lambda)."""
    out = {}
    agree = None
    if log_sp is not None and (dcc is not None or hsic is not None):
        agree = triple_agreement(fx, fit_agreement(fx, log_sp))
        out["triples_fits_agreeing"] = int(agree.sum())
    if residuals is not None:
        n = residuals.shape[0]
        idx = fx["full_index"]
        ref = fx["full_residuals"]
        got = residuals[:, idx]
        scale = np.max(np.abs(ref), axis=0)
        out["residual_rel_err_max"] = float(np.max(np.max(np.abs(got - ref), axis=0) / scale))
        out["residual_fits_in_full"] = int(len(idx))
        z = np.random.default_rng(int(fx["proj_seed"])).standard_normal((4, n))
        proj = residuals.T @ z.T
        norms = np.sqrt(fx["fit_norm2"])
        out["residual_projection_bound_max"] = float(np.max(np.abs(proj - fx["fit_proj"])
                                                            / (norms[:, None] * np.linalg.norm(z, axis=1)[None, :])))
        out["residual_norm2_rel_err_max"] = _rel(np.sum(residuals * residuals, axis=0), fx["fit_norm2"])
        out["fits"] = int(residuals.shape[1])
    if log_sp is not None:
        ref = fx["fit_log_sp"]
        k = ref.shape[1]
        got = log_sp[:, :k]
        mask = np.isfinite(ref)
        out["log_sp_abs_err_max"] = float(np.max(np.abs(got[mask] - ref[mask])))
        det = mask & (np.abs(ref) < 15.0)
        out["log_sp_abs_err_max_below_15"] = float(np.max(np.abs(got[det] - ref[det])))
    if dcc is not None:
        g = fx["guarded"]
        flags_g = (np.asarray(dcc["flags"]) & 1).astype(bool)
        out["dcc_guard_route_flips"] = int(np.sum(flags_g != g))
        same = flags_g == g
        ex = same & ~g
        lr = same & g
        out["dcc_stat_rel_err_max"] = max(_rel(dcc["statistic"][ex], fx["dcc_stat_exact"][ex]),
                                          _rel(dcc["statistic"][lr], fx["dcc_stat_lowrank"][lr]))
        out["dcc_moment_rel_err_max"] = max(_rel(dcc["mean"][ex], fx["dcc_mean_exact"][ex]),
                                            _rel(dcc["variance"][ex], fx["dcc_var_exact"][ex]),
                                            _rel(dcc["mean"][lr], fx["dcc_mean_lowrank"][lr]),
                                            _rel(dcc["variance"][lr], fx["dcc_var_lowrank"][lr]))
        out["dcc_p_exact_abs_err_max"] = float(np.max(np.abs(dcc["p_exact"] - fx["dcc_p_exact"])))
        out["dcc_p_lowrank_abs_err_max"] = (float(np.max(np.abs(dcc["p_value"][lr] - fx["dcc_p"][lr])))
                                            if lr.any() else 0.0)
        out["dcc_p_abs_err_max"] = float(np.max(np.abs(dcc["p_value"] - fx["dcc_p"])))
        if agree is not None:
            out["dcc_p_exact_abs_err_max_agreeing"] = float(np.max(np.abs(dcc["p_exact"] - fx["dcc_p_exact"])[agree]))
        out["dcc_alpha_flips"] = int(np.sum((dcc["p_value"] >= ALPHA) != (fx["dcc_p"] >= ALPHA)))
        out["dcc_guarded"] = int(g.sum())
        out["triples"] = int(len(g))
    if hsic is not None:
        out["hsic_stat_rel_err_max"] = _rel(hsic["statistic"], fx["hsic_stat"])
        out["hsic_moment_rel_err_max"] = max(_rel(hsic["mean"], fx["hsic_mean"]), _rel(hsic["variance"], fx["hsic_var"]))
        out["hsic_p_abs_err_max"] = float(np.max(np.abs(hsic["p_value"] - fx["hsic_p"])))
        if agree is not None:
            out["hsic_p_abs_err_max_agreeing"] = float(np.max(np.abs(hsic["p_value"] - fx["hsic_p"])[agree]))
        out["hsic_alpha_flips"] = int(np.sum((hsic["p_value"] >= ALPHA) != (fx["hsic_p"] >= ALPHA)))
    return out
