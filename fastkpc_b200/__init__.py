"""fastkpc_b200 -- B200-native conditional-independence path of the kernel-PC skeleton.

Python host over the library's C ABI (``include/fastkpc_b200.h``).  The entry
point ``fastkpc_compatible_cuda_skeleton`` mirrors the reference facade of the
same name (fastkpc/R/fast_kpc.R:56-130 -> precision_run_skeleton_full_cuda_native,
fastkpc/R/cuda_native.R:2237-2311): same option names and meaning, same
fail-closed errors.  Indices are 0-based here (the R facade is 1-based).

``fastkpc_compatible_cuda_wanpdag`` mirrors the reference's strict WAN-PDAG
facade (fastkpc/R/fast_kpc.R:449-600): the same skeleton, then kpcalg's
orientation with every regrVonPS residual and CI test on the device.

The compute runs in ``libfastkpc_b200.so`` (CUDA, sm_100a).  There is no CPU
fallback: importing works without a GPU, but every compute call raises
``FkpcError`` when no CUDA device is present, and loading fails loudly when
the shared library has not been built (``python -m fastkpc_b200.build``).
"""
import ctypes
import itertools
import math
import os

import numpy as np

__all__ = [
    "FkpcError", "library_path", "load_library", "fastkpc_compatible_cuda_skeleton",
    "fastkpc_compatible_cuda_wanpdag", "orient_wanpdag", "orient_wanpdag_custom", "ci_level_batch", "ci_plain_one", "regress_batch", "stat_batch", "design_export", "Session",
    "METHODS",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
SELECTIONS = {"magic": 0, "gn_newton": 1}  # FKPC_SELECT_MAGIC, FKPC_SELECT_GN_NEWTON
METHODS = {"dcc.gamma": 0, "dcc.perm": 1, "hsic.gamma": 2, "hsic.perm": 3}
MODES = {"batched": 0, "plain": 1}
FLAG_GUARDED = 1
FLAG_DIRECT = 2
FLAG_RANK_TRUNCATED = 4

STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite numerics",
                4: "iteration limit", 5: "rank deficiency", 6: "allocation failure", 7: "no CUDA device"}


class FkpcError(RuntimeError):
    """A library call failed; ``status`` is the FKPC_STATUS_* code."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status}: {STATUS_NAMES.get(status, '?')})")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_double), ("index", ctypes.c_double), ("num_col", ctypes.c_int),
                ("max_conditioning_size", ctypes.c_int), ("ci_method", ctypes.c_int),
                ("hsic_sig", ctypes.c_double), ("permutation_replicates", ctypes.c_int),
                ("has_seed", ctypes.c_int), ("seed", ctypes.c_uint), ("mode", ctypes.c_int),
                ("collect_trace", ctypes.c_int), ("device", ctypes.c_int), ("strict", ctypes.c_int),
                ("selection", ctypes.c_int), ("level_graph", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("defer_evaluations", ctypes.c_int), ("split_statistics", ctypes.c_int),
                ("lowrank_ctas_per_sm", ctypes.c_int), ("tprs_ctas_per_sm", ctypes.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class CiRecord(ctypes.Structure):
    _fields_ = [("p_value", ctypes.c_double), ("p_exact", ctypes.c_double), ("statistic", ctypes.c_double),
                ("mean", ctypes.c_double), ("variance", ctypes.c_double), ("status", ctypes.c_int),
                ("flags", ctypes.c_uint)]


class StageStats(ctypes.Structure):
    _fields_ = [("setup_ms", ctypes.c_double), ("upload_ms", ctypes.c_double), ("fit_ms", ctypes.c_double),
                ("statistic_ms", ctypes.c_double), ("refine_ms", ctypes.c_double),
                ("download_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("designs", ctypes.c_int),
                ("targets", ctypes.c_int), ("pairs", ctypes.c_int), ("guarded", ctypes.c_int),
                ("kernel_launches", ctypes.c_int), ("h2d_bytes", ctypes.c_double), ("d2h_bytes", ctypes.c_double),
                ("fit_evaluations", ctypes.c_double), ("fit_flops", ctypes.c_double),
                ("statistic_flops", ctypes.c_double), ("fit_iterations", ctypes.c_double),
                ("lowrank_components", ctypes.c_int), ("lowrank_steps_max", ctypes.c_int),
                ("lowrank_steps_mean", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("designs_built", ctypes.c_int), ("smooths_built", ctypes.c_int), ("plan_ms", ctypes.c_double),
                ("tprs_host_ms", ctypes.c_double), ("design_host_ms", ctypes.c_double),
                ("smooth_wait_ms", ctypes.c_double), ("late_wait_ms", ctypes.c_double),
                ("prefit_device_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class TraceRow(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int), ("task_index", ctypes.c_int), ("edge_x", ctypes.c_int),
                ("edge_y", ctypes.c_int), ("x", ctypes.c_int), ("y", ctypes.c_int), ("s_offset", ctypes.c_int),
                ("s_count", ctypes.c_int), ("p_value", ctypes.c_double), ("p_exact", ctypes.c_double),
                ("deleted", ctypes.c_int), ("flags", ctypes.c_uint)]


class Result(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("p", ctypes.c_int), ("levels", ctypes.c_int),
                ("adjacency", ctypes.POINTER(ctypes.c_int)), ("pmax", ctypes.POINTER(ctypes.c_double)),
                ("sepset_offsets", ctypes.POINTER(ctypes.c_int)), ("sepset_values", ctypes.POINTER(ctypes.c_int)),
                ("n_edgetests", ctypes.POINTER(ctypes.c_int)), ("trace_rows", ctypes.c_int),
                ("trace", ctypes.POINTER(TraceRow)), ("trace_s_values", ctypes.POINTER(ctypes.c_int)),
                ("elapsed_sec", ctypes.c_double), ("stats", StageStats)]


class OrientationTest(ctypes.Structure):
    _fields_ = [("reverse", ctypes.c_int), ("target", ctypes.c_int), ("other", ctypes.c_int),
                ("s_offset", ctypes.c_int), ("s_count", ctypes.c_int), ("z_offset", ctypes.c_int),
                ("z_count", ctypes.c_int), ("p_value", ctypes.c_double), ("rejected", ctypes.c_int)]


class Orientation(ctypes.Structure):
    _fields_ = [("p", ctypes.c_int), ("pdag", ctypes.POINTER(ctypes.c_int)),
                ("collider_orientations", ctypes.c_int), ("rule1_orientations", ctypes.c_int),
                ("rule2_orientations", ctypes.c_int), ("rule3_orientations", ctypes.c_int),
                ("generalized_orientations", ctypes.c_int), ("regrvonps_calls", ctypes.c_int),
                ("residual_fits", ctypes.c_int), ("residual_cache_hits", ctypes.c_int), ("tests", ctypes.c_int),
                ("trace", ctypes.POINTER(OrientationTest)), ("set_values", ctypes.POINTER(ctypes.c_int)),
                ("elapsed_sec", ctypes.c_double)]


_lib = None

_P = ctypes.POINTER
_DBL = _P(ctypes.c_double)
_INT = _P(ctypes.c_int)

_SIGNATURES = {
    "fkpc_abi_version": (ctypes.c_int, []),
    "fkpc_last_error": (ctypes.c_char_p, []),
    "fkpc_default_options": (None, [_P(Options)]),
    "fkpc_skeleton_run": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _P(Options), _P(_P(Result))]),
    "fkpc_result_free": (None, [_P(Result)]),
    "fkpc_orient_wanpdag": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, _INT, _INT, _P(Options),
                                           _P(_P(Orientation))]),
    "fkpc_orientation_free": (None, [_P(Orientation)]),
    "fkpc_orient_wanpdag_custom": (ctypes.c_int, [ctypes.c_int, _INT, _INT, _INT, ctypes.c_double, ctypes.c_void_p,
                                                  ctypes.c_void_p, _P(_P(Orientation))]),
    "fkpc_skeleton_run_custom": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _P(Options), ctypes.c_void_p,
                                                ctypes.c_void_p, _P(_P(Result))]),
    "fkpc_ci_level_batch": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, _INT, _INT, _INT, ctypes.c_int,
                                           _P(Options), _P(CiRecord), _P(StageStats)]),
    "fkpc_session_load": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "fkpc_session_evaluate": (ctypes.c_int, [_INT, _INT, _INT, _INT, ctypes.c_int, _P(Options), _P(CiRecord),
                                             _P(StageStats)]),
    "fkpc_ci_plain_one": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _INT,
                                         ctypes.c_int, _P(Options), _P(CiRecord)]),
    "fkpc_regress_batch": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, _INT, _INT, ctypes.c_int,
                                          _P(Options), _DBL, _DBL, ctypes.c_int, _INT]),
    "fkpc_stat_batch": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, _INT, ctypes.c_int, _INT,
                                       _P(Options), _P(CiRecord)]),
    "fkpc_gcv_adjoint": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, ctypes.c_int, _INT, ctypes.c_int,
                                        ctypes.c_int, _DBL, _DBL, _DBL, _DBL, _DBL, ctypes.c_int]),
    "fkpc_gamma_q_eval": (ctypes.c_int, [ctypes.c_int, _DBL, _DBL, ctypes.c_int, _DBL, _INT]),
    "fkpc_permutation_tables": (ctypes.c_int, [ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               _INT]),
    "fkpc_tprs_export": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _INT, _INT, _INT, _DBL, _DBL]),
    "fkpc_get_tuning": (ctypes.c_int, [ctypes.c_int, _P(Tuning)]),
    "fkpc_set_tuning": (ctypes.c_int, [ctypes.c_int, _P(Tuning)]),
    "fkpc_batch_prepare": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, _INT, _INT, _INT, ctypes.c_int,
                                          _P(Options)]),
    "fkpc_batch_execute": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _DBL]),
    "fkpc_batch_collect": (ctypes.c_int, [ctypes.c_int, _P(CiRecord), _P(StageStats)]),
    "fkpc_batch_time_stage": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _DBL, _DBL]),
    "fkpc_measure_fp64_peak": (ctypes.c_int, [ctypes.c_int, _DBL]),
    "fkpc_dcov_gamma_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "fkpc_design_export": (ctypes.c_int, [_DBL, ctypes.c_int, ctypes.c_int, _INT, ctypes.c_int, _INT, _INT, _DBL,
                                          _DBL, _DBL]),
}


def library_path():
    return os.path.join(_HERE, "libfastkpc_b200.so")


def load_library():
    """Load the CUDA library; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"fastkpc_b200 CUDA library not built: {path} is missing "
                          "(run `python -m fastkpc_b200.build`)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        msg = load_library().fkpc_last_error().decode("utf-8", errors="replace")
        raise FkpcError(rc, msg)


def _ptr(a, ctype):
    return a.ctypes.data_as(_P(ctype))


def _as_data(data):
    a = np.asarray(data, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("data must be a 2-D matrix")
    return np.asfortranarray(a)


def make_options(ci_method="dcc.gamma", alpha=0.1, index=1.0, numCol=35, max_conditioning_size=math.inf,
                 hsic_sig=1.0, replicates=100, seed=None, mode="batched", trace=True, device=0, strict=True,
                 selection="magic", level_graph=False):
    o = Options()
    load_library().fkpc_default_options(ctypes.byref(o))
    if ci_method not in METHODS:
        raise ValueError(f"unknown ci_method {ci_method!r}")
    o.alpha = float(alpha)
    o.index = float(index)
    o.num_col = int(numCol)
    o.max_conditioning_size = -1 if math.isinf(max_conditioning_size) else int(max_conditioning_size)
    o.ci_method = METHODS[ci_method]
    o.hsic_sig = float(hsic_sig)
    o.permutation_replicates = int(replicates)
    o.has_seed = 0 if seed is None else 1
    o.seed = 0 if seed is None else int(seed) & 0xFFFFFFFF
    o.mode = MODES[mode]
    o.collect_trace = 1 if trace else 0
    o.device = int(device)
    o.strict = 1 if strict else 0
    if selection not in SELECTIONS:
        raise ValueError(f"unknown selection {selection!r}")
    o.selection = SELECTIONS[selection]
    o.level_graph = 1 if level_graph else 0
    return o


_ALLOWED = {"max_conditioning_size", "index", "numCol", "trace_level", "route", "compatible_cuda_strict",
            "ci_method", "hsic_params", "permutation_params", "mode", "device", "level_graph"}


def fastkpc_compatible_cuda_skeleton(data, alpha, labels=None, options=None):
    """Kernel-PC skeleton with the full-CUDA CI route.

    ``options`` keys follow the reference facade: ``max_conditioning_size``
    (default Inf), ``index`` (1), ``numCol`` (default floor(n/10) as in the
    reference; the strict envelope requires 35), ``trace_level``
    ("summary" | "logical" | "full" | "none"), ``route`` ("full_cuda"),
    ``compatible_cuda_strict`` (True), ``ci_method`` ("dcc.gamma",
    "dcc.perm", "hsic.gamma", "hsic.perm"), ``hsic_params`` ({"sig": 1}),
    ``permutation_params`` ({"replicates": 100, "seed": None,
    "include_observed": True}); plus ``mode`` ("batched" | "plain"),
    ``device`` and ``level_graph`` (False: each level's batch overlaps its
    host set-up with the device work; True: set-up first, then the level runs
    as one captured CUDA graph).

    Returns a dict with ``adjacency`` (bool p x p), ``pMax``, ``sepsets``
    (list of p lists; None or the separating set, 0-based), ``n_edgetests``,
    ``tasks`` (the logical trace as column arrays), ``summary``.
    """
    X, labels, o, method = _skeleton_setup(data, alpha, labels, options)
    return _run_skeleton(X, alpha, labels, o, method, None)


def _skeleton_setup(data, alpha, labels, options):
    """Validated (data, labels, fkpc_options, method) of the facade's options."""
    options = dict(options or {})
    unknown = set(options) - _ALLOWED
    if unknown:
        raise ValueError("unknown compatible CUDA option(s): " + ",".join(sorted(unknown)))
    if options.get("route", "full_cuda") != "full_cuda":
        raise ValueError("only route = 'full_cuda' is provided by this library")
    X = _as_data(data)
    n, p = X.shape
    labels = list(labels) if labels is not None else [f"V{i + 1}" for i in range(p)]
    if len(labels) != p:
        raise ValueError("labels must have one entry per column")
    trace_level = options.get("trace_level", "summary")
    if trace_level not in ("summary", "logical", "full", "none"):
        raise ValueError("trace_level must be summary, logical, full or none")
    hsic = options.get("hsic_params") or {"sig": 1}
    perm = options.get("permutation_params") or {"replicates": 100, "seed": None, "include_observed": True}
    if not perm.get("include_observed", True):
        raise ValueError("strict permutation p-values require include_observed = TRUE")
    method = options.get("ci_method", "dcc.gamma")
    if method in ("dcc.perm", "hsic.perm") and perm.get("seed") is None:
        raise ValueError("strict compatible CUDA permutation methods require an explicit seed")
    o = make_options(ci_method=method, alpha=alpha, index=options.get("index", 1),
                     numCol=options.get("numCol", n // 10),
                     max_conditioning_size=options.get("max_conditioning_size", math.inf),
                     hsic_sig=hsic.get("sig", 1), replicates=perm.get("replicates", 100), seed=perm.get("seed"),
                     mode=options.get("mode", "batched"), trace=trace_level in ("logical", "full"),
                     device=options.get("device", 0), strict=options.get("compatible_cuda_strict", True),
                     level_graph=options.get("level_graph", False))
    return X, labels, o, method


# One level's CI tests for fkpc_skeleton_run_custom (see fastkpc_b200.distributed).
LEVEL_EVALUATOR = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _INT, _INT, _INT, _INT, ctypes.c_int,
                                   _P(CiRecord))


def _run_skeleton(X, alpha, labels, o, method, evaluator):
    n, p = X.shape
    lib = load_library()
    res = _P(Result)()
    if evaluator is None:
        _check(lib.fkpc_skeleton_run(_ptr(X, ctypes.c_double), n, p, ctypes.byref(o), ctypes.byref(res)))
    else:
        _check(lib.fkpc_skeleton_run_custom(_ptr(X, ctypes.c_double), n, p, ctypes.byref(o), evaluator, None,
                                            ctypes.byref(res)))
    try:
        r = res.contents
        adj = np.ctypeslib.as_array(r.adjacency, shape=(p * p,)).reshape((p, p), order="F").astype(bool)
        pmax = np.ctypeslib.as_array(r.pmax, shape=(p * p,)).reshape((p, p), order="F").copy()
        offs = np.ctypeslib.as_array(r.sepset_offsets, shape=(p * p + 1,)).copy()
        nvals = int(offs[-1])
        vals = np.ctypeslib.as_array(r.sepset_values, shape=(max(nvals, 1),))[:nvals].copy()
        sepsets = [[None] * p for _ in range(p)]
        for j in range(p):
            for i in range(p):
                cell = i + p * j
                if offs[cell + 1] > offs[cell] or _deleted(adj, i, j):
                    s = [int(v) for v in vals[offs[cell]:offs[cell + 1]]]
                    sepsets[i][j] = s if (offs[cell + 1] > offs[cell] or not adj[i, j]) else None
        for i in range(p):
            for j in range(p):
                if adj[i, j] or i == j:
                    sepsets[i][j] = None
        n_edgetests = [int(r.n_edgetests[k]) for k in range(r.levels)]
        tasks = None
        if r.trace and r.trace_rows > 0:
            rows = [r.trace[k] for k in range(r.trace_rows)]
            svals = r.trace_s_values
            tasks = {
                "level": np.array([t.level for t in rows]), "task_index": np.array([t.task_index for t in rows]),
                "edge_x": np.array([t.edge_x for t in rows]), "edge_y": np.array([t.edge_y for t in rows]),
                "x": np.array([t.x for t in rows]), "y": np.array([t.y for t in rows]),
                "S": [[int(svals[t.s_offset + k]) for k in range(t.s_count)] for t in rows],
                "p_used": np.array([t.p_value for t in rows]), "p_exact": np.array([t.p_exact for t in rows]),
                "native_edge_deleted": np.array([bool(t.deleted) for t in rows]),
                "guarded": np.array([bool(t.flags & FLAG_GUARDED) for t in rows]),
            }
        stats = r.stats.as_dict()
        summary = {"n": n, "p": p, "alpha": float(alpha), "ci_method": method, "levels": r.levels,
                   "tests_replayed": int(sum(n_edgetests)), "elapsed_sec": r.elapsed_sec, "labels": labels,
                   "max_conditioning_size_resolved": (p - 2 if o.max_conditioning_size < 0
                                                      else min(o.max_conditioning_size, p - 2)),
                   "stages": stats,
                   "entrypoint": "fkpc_skeleton_run" if evaluator is None else "fkpc_skeleton_run_custom"}
        return {"adjacency": adj, "pMax": pmax, "sepsets": sepsets, "n_edgetests": n_edgetests,
                "tasks": tasks, "summary": summary}
    finally:
        lib.fkpc_result_free(res)


def _deleted(adj, i, j):
    return i != j and not adj[i, j]


def orient_wanpdag(skeleton, data, alpha=0.1, index=1, numCol=None, ci_method="dcc.gamma", hsic_params=None,
                   orient_collider=True, solve_confl=False, rules=(True, True, True), device=0, selection="magic",
                   strict=True):
    """WAN-PDAG orientation of a skeleton (kpcalg's udag2wanpdag as kpc()
    runs it), every regrVonPS residual fit and CI test on the device.

    Mirrors ``fastkpc_orient_wanpdag_kpcalg_authority`` (fastkpc/R/fast_kpc.R:263-330):
    ``skeleton`` is a ``fastkpc_compatible_cuda_skeleton`` result (its
    ``adjacency`` and ``sepsets``); alpha, numCol (default floor(n/10)), the
    CI method (gamma methods) and hsic_params as the skeleton used them.
    Only kpc()'s defaults are provided: orient_collider = True, solve_confl =
    False, all three rules.

    Returns a dict: ``pdag`` (int p x p; pdag[i, j] = 1, pdag[j, i] = 0 is
    i -> j), ``ci_trace`` (column arrays of every CI test in call order),
    ``diagnostics`` (orientation counts, regrVonPS calls, residual fits and
    cache hits, ci_test_count, orientation_elapsed_sec).
    """
    if not orient_collider or solve_confl or tuple(bool(r) for r in rules) != (True, True, True):
        raise ValueError("only kpc()'s orientation defaults are provided: orient_collider = TRUE, "
                         "solve_confl = FALSE, rules = c(TRUE, TRUE, TRUE)")
    if ci_method not in ("dcc.gamma", "hsic.gamma"):
        raise ValueError("the orientation covers the gamma methods")
    X = _as_data(data)
    n, p = X.shape
    A, offs, vals = _skeleton_arrays(skeleton, p)
    hsic = hsic_params or {"sig": 1}
    o = make_options(ci_method=ci_method, alpha=alpha, index=index, numCol=n // 10 if numCol is None else numCol,
                     hsic_sig=hsic.get("sig", 1), device=device, strict=strict, selection=selection)
    lib = load_library()
    res = _P(Orientation)()
    _check(lib.fkpc_orient_wanpdag(_ptr(X, ctypes.c_double), n, p, _ptr(A, ctypes.c_int),
                                   _ptr(offs, ctypes.c_int), _ptr(vals, ctypes.c_int), ctypes.byref(o),
                                   ctypes.byref(res)))
    out = _read_orientation(lib, res, p)
    out["ci_method"] = ci_method
    return out


# One regrVonPS call for fkpc_orient_wanpdag_custom.
REGRVONPS_EVALUATOR = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _INT, ctypes.c_int, _INT,
                                       ctypes.c_int, _DBL)


def orient_wanpdag_custom(skeleton, p, alpha, regr_v_on_ps):
    """The orientation's graph logic (``fkpc_orient_wanpdag_custom``) with
    every regrVonPS call answered by ``regr_v_on_ps(target, S, Z)``, which
    returns one p-value per member of S (the test of the residual of target
    on Z against that member).  Uses no device.  Same result dict as
    ``orient_wanpdag``."""
    A, offs, vals = _skeleton_arrays(skeleton, p)
    errors = []

    def cb(_user, target, subset, ns, cond, nz, out):
        try:
            pv = regr_v_on_ps(int(target), [int(subset[k]) for k in range(ns)], [int(cond[k]) for k in range(nz)])
            if len(pv) != ns:
                raise ValueError("the evaluator must return one p-value per member of S")
            for k in range(ns):
                out[k] = float(pv[k])
            return 0
        except Exception as e:  # reported after the call returns
            errors.append(e)
            return 1
    fn = REGRVONPS_EVALUATOR(cb)
    lib = load_library()
    res = _P(Orientation)()
    rc = lib.fkpc_orient_wanpdag_custom(p, _ptr(A, ctypes.c_int), _ptr(offs, ctypes.c_int),
                                        _ptr(vals, ctypes.c_int), float(alpha), ctypes.cast(fn, ctypes.c_void_p),
                                        None, ctypes.byref(res))
    if errors:
        raise errors[0]
    _check(rc)
    return _read_orientation(lib, res, p)


def _skeleton_arrays(skeleton, p):
    """(adjacency int32 column-major, sepset CSR offsets, values) of a skeleton dict."""
    adj = np.asarray(skeleton["adjacency"]).astype(bool)
    if adj.shape != (p, p):
        raise ValueError("skeleton adjacency must be p x p")
    sep = skeleton.get("sepsets")
    offs = np.zeros(p * p + 1, dtype=np.int32)
    vals = []
    for j in range(p):
        for i in range(p):
            if isinstance(sep, dict):
                s_ij = sep.get((i, j))
            else:
                s_ij = sep[i][j] if sep is not None else None
            if s_ij:
                vals.extend(int(v) for v in s_ij)
            offs[i + p * j + 1] = len(vals)
    vals = np.asarray(vals if vals else [0], dtype=np.int32)
    return np.asfortranarray(adj.astype(np.int32)), offs, vals


def _read_orientation(lib, res, p):
    try:
        r = res.contents
        pdag = np.ctypeslib.as_array(r.pdag, shape=(p * p,)).reshape((p, p), order="F").astype(np.int64)
        rows = [r.trace[k] for k in range(r.tests)]
        sv = r.set_values
        trace = {
            "context": ["reverseRegrVonPS" if t.reverse else "regrVonPS" for t in rows],
            "reverse": np.array([t.reverse for t in rows], dtype=np.int64),
            "target": np.array([t.target for t in rows], dtype=np.int64),
            "other": np.array([t.other for t in rows], dtype=np.int64),
            "subset": [[int(sv[t.s_offset + k]) for k in range(t.s_count)] for t in rows],
            "residual_conditioning_set": [[int(sv[t.z_offset + k]) for k in range(t.z_count)] for t in rows],
            "p_value": np.array([t.p_value for t in rows]),
            "rejected": np.array([bool(t.rejected) for t in rows]),
        }
        diag = {"collider_orientations": r.collider_orientations, "rule1_orientations": r.rule1_orientations,
                "rule2_orientations": r.rule2_orientations, "rule3_orientations": r.rule3_orientations,
                "generalized_orientations": r.generalized_orientations, "regrvonps_calls": r.regrvonps_calls,
                "residual_fits": r.residual_fits, "residual_cache_hits": r.residual_cache_hits,
                "ci_test_count": r.tests, "orientation_elapsed_sec": r.elapsed_sec}
        return {"pdag": pdag, "ci_trace": trace, "diagnostics": diag,
                "authority": "kpcalg::udag2wanpdag semantics, device residuals and CI tests"}
    finally:
        lib.fkpc_orientation_free(res)


def pdag_edge_counts(pdag):
    """Directed, undirected and bidirected (conflict, value 2) edge counts of a PDAG."""
    a = np.asarray(pdag)
    iu = np.triu_indices(a.shape[0], 1)
    x, y = a[iu], a.T[iu]
    return {"directed": int(np.sum(((x == 1) & (y == 0)) | ((x == 0) & (y == 1)))),
            "undirected": int(np.sum((x == 1) & (y == 1))),
            "bidirected": int(np.sum((x == 2) | (y == 2)))}


_WANPDAG_ALLOWED = {"max_conditioning_size", "index", "numCol", "trace_level", "route", "compatible_cuda_strict",
                    "ci_method", "hsic_params", "permutation_params", "orient_collider", "solve_confl", "rules",
                    "mode", "device", "level_graph"}


def fastkpc_compatible_cuda_wanpdag(data, alpha=0.1, labels=None, options=None):
    """Strict kernel-PC: the full-CUDA skeleton, then the WAN-PDAG orientation.

    Mirrors ``fastkpc_compatible_cuda_wanpdag`` (fastkpc/R/fast_kpc.R:449-600):
    the skeleton options of ``fastkpc_compatible_cuda_skeleton`` (trace_level
    "logical" or "full") plus ``orient_collider``, ``solve_confl`` and
    ``rules``; the orientation uses the skeleton's alpha, numCol, CI method
    and hsic_params.  Returns ``config``, ``skeleton``, ``orientation``,
    ``timings`` (seconds per stage) and ``metrics`` (edge counts, CI test
    counts).
    """
    import time
    options = dict(options or {})
    unknown = set(options) - _WANPDAG_ALLOWED
    if unknown:
        raise ValueError("unknown compatible CUDA WAN-PDAG option(s): " + ",".join(sorted(unknown)))
    if options.get("route", "full_cuda") != "full_cuda" or not options.get("compatible_cuda_strict", True):
        raise ValueError("compatible CUDA WAN-PDAG requires strict full_cuda skeleton execution")
    trace_level = options.setdefault("trace_level", "logical")
    if trace_level not in ("logical", "full"):
        raise ValueError("compatible CUDA WAN-PDAG requires logical or full skeleton trace")
    orient_keys = {k: options.pop(k) for k in ("orient_collider", "solve_confl", "rules") if k in options}
    method = options.get("ci_method", "dcc.gamma")
    X = _as_data(data)
    t0 = time.perf_counter()
    skel = fastkpc_compatible_cuda_skeleton(X, alpha, labels=labels, options=options)
    t1 = time.perf_counter()
    orient = orient_wanpdag(skel, X, alpha=alpha, index=options.get("index", 1),
                            numCol=options.get("numCol", X.shape[0] // 10), ci_method=method,
                            hsic_params=options.get("hsic_params"), device=options.get("device", 0),
                            strict=options.get("compatible_cuda_strict", True), **orient_keys)
    t2 = time.perf_counter()
    counts = pdag_edge_counts(orient["pdag"])
    adj = skel["adjacency"]
    return {
        "schema_version": "fastkpc-compatible-cuda-wanpdag-v1",
        "config": {"alpha": float(alpha), "ci_method": method, "skeleton_authority": "full_cuda",
                   "orientation_authority": "device regrVonPS, kpcalg udag2wanpdag semantics",
                   "max_conditioning_size_resolved": skel["summary"]["max_conditioning_size_resolved"]},
        "skeleton": skel,
        "orientation": orient,
        "timings": {"skeleton": t1 - t0, "orientation": t2 - t1, "total": t2 - t0},
        "metrics": {"skeleton_edge_count": int(np.sum(np.triu(adj, 1))),
                    "directed_edge_count": counts["directed"], "undirected_edge_count": counts["undirected"],
                    "bidirected_edge_count": counts["bidirected"],
                    "skeleton_ci_test_count": int(sum(skel["n_edgetests"])),
                    "orientation_ci_test_count": orient["diagnostics"]["ci_test_count"]},
    }


def _tests_arrays(tests):
    count = len(tests)
    xs = np.fromiter((t[0] for t in tests), dtype=np.int32, count=count)
    ys = np.fromiter((t[1] for t in tests), dtype=np.int32, count=count)
    offs = np.zeros(count + 1, dtype=np.int32)
    np.cumsum(np.fromiter((len(t[2]) for t in tests), dtype=np.int32, count=count), out=offs[1:])
    total = int(offs[-1])
    if total == 0:
        return xs, ys, offs, np.zeros(1, dtype=np.int32)
    vals = np.fromiter(itertools.chain.from_iterable(t[2] for t in tests), dtype=np.int32, count=total)
    return xs, ys, offs, vals


_RECORD_DTYPE = None


def _records(recs, count):
    """Field arrays (float64, int64) of the first ``count`` entries of a
    ctypes ``CiRecord`` array."""
    global _RECORD_DTYPE
    if _RECORD_DTYPE is None:
        _RECORD_DTYPE = np.dtype({"names": [f for f, _ in CiRecord._fields_],
                                  "formats": [np.dtype(t) for _, t in CiRecord._fields_],
                                  "offsets": [getattr(CiRecord, f).offset for f, _ in CiRecord._fields_],
                                  "itemsize": ctypes.sizeof(CiRecord)})
    arr = np.frombuffer(recs, dtype=_RECORD_DTYPE, count=count)
    return {name: arr[name].astype(np.int64 if arr[name].dtype.kind in "iu" else np.float64)
            for name, _ in CiRecord._fields_}


def ci_level_batch(data, tests, ci_method="dcc.gamma", mode="batched", **kw):
    """Evaluate CI tests ``[(x, y, S), ...]``; returns (records dict, stage stats dict)."""
    X = _as_data(data)
    n, p = X.shape
    o = make_options(ci_method=ci_method, mode=mode, **kw)
    xs, ys, offs, vals = _tests_arrays(tests)
    out = (CiRecord * max(1, len(tests)))()
    st = StageStats()
    _check(load_library().fkpc_ci_level_batch(_ptr(X, ctypes.c_double), n, p, _ptr(xs, ctypes.c_int),
                                                _ptr(ys, ctypes.c_int), _ptr(offs, ctypes.c_int),
                                                _ptr(vals, ctypes.c_int), len(tests), ctypes.byref(o), out,
                                                ctypes.byref(st)))
    return _records(out, len(tests)), st.as_dict()


class Session:
    """The data matrix kept loaded on one GPU across batches of CI tests, with
    its cache of conditioning-set designs (fkpc_session_load /
    fkpc_session_evaluate): a design is set up once per device, however many
    batches (skeleton levels) use it.  Any other call that loads data on the
    same device ends the session."""

    def __init__(self, data, device=0):
        self.X = _as_data(data)
        self.device = int(device)
        n, p = self.X.shape
        _check(load_library().fkpc_session_load(_ptr(self.X, ctypes.c_double), n, p, self.device))

    def evaluate_raw(self, tests, options):
        """Records (ctypes array) and stats dict of ``tests`` with a ready
        ``fkpc_options`` (its ``device`` must be the session's)."""
        out = (CiRecord * max(1, len(tests)))()
        st = StageStats()
        xs, ys, offs, vals = _tests_arrays(tests)
        _check(load_library().fkpc_session_evaluate(_ptr(xs, ctypes.c_int), _ptr(ys, ctypes.c_int),
                                                      _ptr(offs, ctypes.c_int), _ptr(vals, ctypes.c_int),
                                                      len(tests), ctypes.byref(options), out, ctypes.byref(st)))
        return out, st.as_dict()

    def evaluate(self, tests, ci_method="dcc.gamma", **kw):
        """(records dict, stage stats dict) of ``[(x, y, S), ...]``."""
        o = make_options(ci_method=ci_method, device=self.device, **kw)
        out, st = self.evaluate_raw(tests, o)
        return _records(out, len(tests)), st


def ci_plain_one(data, x, y, S, ci_method="dcc.gamma", **kw):
    """One CI test through the plain per-test form; returns a record dict."""
    X = _as_data(data)
    n, p = X.shape
    o = make_options(ci_method=ci_method, mode="plain", **kw)
    s = np.array(list(S) if S else [0], dtype=np.int32)
    rec = CiRecord()
    _check(load_library().fkpc_ci_plain_one(_ptr(X, ctypes.c_double), n, p, int(x), int(y),
                                              _ptr(s, ctypes.c_int), len(S), ctypes.byref(o),
                                              ctypes.byref(rec)))
    return {name: getattr(rec, name) for name, _ in CiRecord._fields_}


def regress_batch(data, fits, max_penalties=None, device=0, selection="magic"):
    """regrXonS residuals for ``[(target, S), ...]``: (residuals n x k, log_sp k x m, status k).

    ``max_penalties`` (default: the largest |S|) columns of log_sp, NaN
    beyond a fit's penalties.  ``selection``: "magic" (mgcv magic's search,
    as the reference) or "gn_newton" (Newton on the Gauss-Newton Hessian of
    GCV) for |S| >= 3."""
    X = _as_data(data)
    n, p = X.shape
    k = len(fits)
    if max_penalties is None:
        max_penalties = max([len(f[1]) for f in fits] + [1])
    tg = np.array([f[0] for f in fits], dtype=np.int32)
    offs = np.zeros(k + 1, dtype=np.int32)
    vals = []
    for i, f in enumerate(fits):
        vals.extend(int(v) for v in f[1])
        offs[i + 1] = len(vals)
    vals = np.array(vals if vals else [0], dtype=np.int32)
    resid = np.zeros((n, k), dtype=np.float64, order="F")
    lsp = np.zeros((k, max_penalties), dtype=np.float64)
    status = np.zeros(k, dtype=np.int32)
    o = make_options(device=device, selection=selection)
    _check(load_library().fkpc_regress_batch(_ptr(X, ctypes.c_double), n, p, _ptr(tg, ctypes.c_int),
                                               _ptr(offs, ctypes.c_int), _ptr(vals, ctypes.c_int), k,
                                               ctypes.byref(o), _ptr(resid, ctypes.c_double),
                                               _ptr(lsp, ctypes.c_double), max_penalties,
                                               _ptr(status, ctypes.c_int)))
    return resid, lsp, status


def tprs_export(data, a, b, device=0):
    """The device thin-plate set-up of the bivariate smooth on columns {a, b}:
    dict(n_u, path ("block", "single" or None when the device does not take
    it), ok, values (30, descending), vectors (n_u x 30, unit norm, largest
    entry positive))."""
    X = np.asfortranarray(data, dtype=np.float64)
    n, p = X.shape
    nu, path, ok = (ctypes.c_int(0) for _ in range(3))
    vals = np.zeros(30)
    vecs = np.zeros(n * 30)
    _check(load_library().fkpc_tprs_export(_ptr(X, ctypes.c_double), n, p, int(a), int(b), int(device),
                                           ctypes.byref(nu), ctypes.byref(path), ctypes.byref(ok),
                                           _ptr(vals, ctypes.c_double), _ptr(vecs, ctypes.c_double)))
    names = {0: None, 1: "single", 2: "block"}
    k = nu.value
    return {"n_u": k, "path": names[path.value], "ok": bool(ok.value), "values": vals,
            "vectors": vecs[:k * 30].reshape(30, k).T.copy() if path.value else None}


def permutation_tables(seed, ci_method, n, replicates, count):
    """The R-compatible permutation tables of ``count`` consecutive tests
    (count x replicates x n int32) for dcc.perm or hsic.perm, as the batch
    entry points draw them after set.seed(seed); ``stat_batch`` takes them."""
    out = np.zeros((count, replicates, n), dtype=np.int32)
    _check(load_library().fkpc_permutation_tables(int(seed) & 0xFFFFFFFF, METHODS[ci_method], int(n),
                                                   int(replicates), int(count), _ptr(out, ctypes.c_int)))
    return out


def stat_batch(residuals, pairs, ci_method="dcc.gamma", permutations=None, **kw):
    """Statistics for ``[(left, right), ...]`` columns of ``residuals`` (n x m)."""
    R = np.asfortranarray(np.asarray(residuals, dtype=np.float64))
    n, m = R.shape
    left = np.array([a for a, _ in pairs], dtype=np.int32)
    right = np.array([b for _, b in pairs], dtype=np.int32)
    o = make_options(ci_method=ci_method, **kw)
    perm_ptr = None
    if permutations is not None:
        perms = np.ascontiguousarray(permutations, dtype=np.int32)
        perm_ptr = _ptr(perms, ctypes.c_int)
    out = (CiRecord * max(1, len(pairs)))()
    _check(load_library().fkpc_stat_batch(_ptr(R, ctypes.c_double), n, m, _ptr(left, ctypes.c_int),
                                            _ptr(right, ctypes.c_int), len(pairs), perm_ptr, ctypes.byref(o), out))
    return _records(out, len(pairs))


STAGES = {"fit_single": 0, "fit_multi_small": 1, "fit_multi_large": 2, "dcov_components": 3, "dcov_pairs": 4,
          "hsic_components": 5, "hsic_pairs": 6, "lowrank_eigen": 7, "lowrank_pairs": 8, "fit_multi_huge": 9,
          "fit_multi_wide": 10}


class StagedBatch:
    """Prepared level batch on one device: every input resident in HBM.

    ``execute(k)`` replays the captured launch sequence k times and returns the
    CUDA-event device time; ``collect()`` waits and returns (records, stats);
    ``time_stage(name, k)`` replays one kernel alone (mean ms, flops/launch).
    """

    def __init__(self, data, tests, ci_method="dcc.gamma", device=0, **kw):
        X = _as_data(data)
        n, p = X.shape
        self.device = device
        self.count = len(tests)
        o = make_options(ci_method=ci_method, device=device, **kw)
        xs, ys, offs, vals = _tests_arrays(tests)
        _check(load_library().fkpc_batch_prepare(_ptr(X, ctypes.c_double), n, p, _ptr(xs, ctypes.c_int),
                                                   _ptr(ys, ctypes.c_int), _ptr(offs, ctypes.c_int),
                                                   _ptr(vals, ctypes.c_int), len(tests), ctypes.byref(o)))

    def execute(self, repeats=1):
        ms = ctypes.c_double()
        _check(load_library().fkpc_batch_execute(self.device, int(repeats), ctypes.byref(ms)))
        return ms.value

    def collect(self):
        out = (CiRecord * self.count)()
        st = StageStats()
        _check(load_library().fkpc_batch_collect(self.device, out, ctypes.byref(st)))
        return _records(out, self.count), st.as_dict()

    def time_stage(self, stage, repeats=3):
        ms = ctypes.c_double()
        fl = ctypes.c_double()
        _check(load_library().fkpc_batch_time_stage(self.device, STAGES[stage], int(repeats), ctypes.byref(ms),
                                                      ctypes.byref(fl)))
        return ms.value, fl.value


def measure_fp64_peak(device=0):
    """Measured FP64 FMA throughput of the device, TFLOP/s."""
    t = ctypes.c_double()
    _check(load_library().fkpc_measure_fp64_peak(int(device), ctypes.byref(t)))
    return t.value


def gcv_adjoint(data, target, S, log_lambda, device=0):
    """GCV score V, gradient, Gauss-Newton Hessian and exact Hessian in
    rho = log(lambda) of the additive fit of column ``target`` on S (|S| >= 3)
    at each row of ``log_lambda`` (count x |S|; entry j belongs to the j-th
    smallest variable of S).  Returns a dict of arrays (count, count x m,
    count x m x m, count x m x m)."""
    X = _as_data(data)
    n, p = X.shape
    s = np.array(sorted(S), dtype=np.int32)
    m = len(s)
    rho = np.ascontiguousarray(np.atleast_2d(np.asarray(log_lambda, dtype=np.float64)))
    if rho.shape[1] != m:
        raise ValueError("log_lambda must have one column per conditioning variable")
    count = rho.shape[0]
    score = np.zeros(count)
    grad = np.zeros((count, m))
    gn = np.zeros((count, m, m))
    hess = np.zeros((count, m, m))
    _check(load_library().fkpc_gcv_adjoint(_ptr(X, ctypes.c_double), n, p, int(target), _ptr(s, ctypes.c_int), m,
                                             count, _ptr(rho, ctypes.c_double), _ptr(score, ctypes.c_double),
                                             _ptr(grad, ctypes.c_double), _ptr(gn, ctypes.c_double),
                                             _ptr(hess, ctypes.c_double), int(device)))
    return {"score": score, "grad": grad, "gn_hessian": gn, "hessian": hess}


def get_tuning(device=0):
    """The engine's schedule choices on ``device`` (dict; see fkpc_tuning)."""
    t = Tuning()
    _check(load_library().fkpc_get_tuning(int(device), ctypes.byref(t)))
    return t.as_dict()


def set_tuning(device=0, **changes):
    """Change some of the engine's schedule choices on ``device``; returns the
    new settings.  Records never depend on them."""
    t = Tuning()
    _check(load_library().fkpc_get_tuning(int(device), ctypes.byref(t)))
    for name, value in changes.items():
        if name not in dict(Tuning._fields_):
            raise ValueError(f"unknown tuning {name!r}")
        setattr(t, name, int(value))
    _check(load_library().fkpc_set_tuning(int(device), ctypes.byref(t)))
    return t.as_dict()


def gamma_q(a, x, device=0):
    """Q(a, x), the regularised upper incomplete gamma function, by the
    statistic kernels' device routine; returns (q, ok) arrays."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
    if a.shape != x.shape:
        raise ValueError("a and x must have the same length")
    q = np.zeros_like(a)
    ok = np.zeros(a.shape, dtype=np.int32)
    _check(load_library().fkpc_gamma_q_eval(int(device), _ptr(a, ctypes.c_double), _ptr(x, ctypes.c_double),
                                              len(a), _ptr(q, ctypes.c_double), _ptr(ok, ctypes.c_int)))
    return q, ok.astype(bool)


def design_export(data, S):
    """Host design set-up for S: dict(X, penalties (m x q x q), initial_log_sp)."""
    X = _as_data(data)
    n, p = X.shape
    s = np.array(sorted(S), dtype=np.int32)
    q = ctypes.c_int()
    m = ctypes.c_int()
    lib = load_library()
    _check(lib.fkpc_design_export(_ptr(X, ctypes.c_double), n, p, _ptr(s, ctypes.c_int), len(s),
                                  ctypes.byref(q), ctypes.byref(m), None, None, None))
    Xd = np.zeros((n, q.value), order="F")
    pen = np.zeros((m.value, q.value, q.value))
    pen_f = np.zeros(m.value * q.value * q.value)
    lsp = np.zeros(m.value)
    _check(lib.fkpc_design_export(_ptr(X, ctypes.c_double), n, p, _ptr(s, ctypes.c_int), len(s),
                                  ctypes.byref(q), ctypes.byref(m), _ptr(Xd, ctypes.c_double),
                                  _ptr(pen_f, ctypes.c_double), _ptr(lsp, ctypes.c_double)))
    for j in range(m.value):
        pen[j] = pen_f[j * q.value * q.value:(j + 1) * q.value * q.value].reshape((q.value, q.value), order="F")
    return {"X": np.asarray(Xd), "penalties": pen, "initial_log_sp": lsp, "q": q.value, "m": m.value}
