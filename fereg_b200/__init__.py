"""fereg_b200 — B200-native fixed-effects solve behind the reference's `Absorber` boundary.

The compute runs in libfereg_b200.so (hand-written sm_100a CUDA) through the C ABI declared in
include/fereg_b200.h. This module is the Python host mirror of that ABI, used by the tests and
the benchmark. There is no CPU fallback: loading fails loudly when the library is missing, and
every call fails with the library's error when no CUDA device is present.
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfereg_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "fereg_b200.h")

PREC_F64 = 0
PREC_F32_REFINED = 1

_lib = None

P = C.c_void_p
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f64p = C.POINTER(C.c_double)
u8p = C.POINTER(C.c_uint8)


class FeregError(RuntimeError):
    """A nonzero return code of the C ABI (the reference's RfError::rc)."""

    def __init__(self, rc, msg):
        super().__init__(f"rc={rc}: {msg}")
        self.rc = rc


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("escalated", C.c_int32), ("exact", C.c_int32)]


OLS_SCALARS = ["N", "rank", "df_r", "df_m", "df_a", "df_a_initial", "df_a_redundant", "df_a_nested", "N_clust",
               "N_clustervars", "N_clust1", "N_clust2", "num_singletons", "N_full", "report_constant", "rss", "tss",
               "tss_within", "mss", "rmse", "r2", "r2_a", "r2_within", "r2_a_within", "ll", "ll_0", "F",
               "sumweights", "ic"]
VCE = {"unadjusted": 0, "robust": 1, "cluster": 2, "crv3": 3, "hc2": 4, "hc3": 5}
WEIGHT_KIND = {None: 0, "aweight": 1, "fweight": 2, "pweight": 3}


class OlsSpec(C.Structure):
    _fields_ = [("vce", C.c_int), ("noconstant", C.c_int), ("firstpair", C.c_int), ("want_groupvar", C.c_int),
                ("tol", C.c_double), ("maxiter", C.c_size_t), ("precision", C.c_int)]


class BootSpec(C.Structure):
    _fields_ = [("coef", C.c_size_t), ("r0", C.c_double), ("reps", C.c_size_t), ("seed", C.c_uint64),
                ("tile", C.c_size_t), ("tol", C.c_double), ("maxiter", C.c_size_t), ("precision", C.c_int)]


class BootOut(C.Structure):
    _fields_ = [("stat", C.c_double), ("se", C.c_double), ("point", C.c_double), ("pvalue", C.c_double),
                ("reps", C.c_uint64), ("full_enum", C.c_int32), ("t_boot", C.POINTER(C.c_double))]


class GlmSpec(C.Structure):
    _fields_ = [("vce", C.c_int), ("tol", C.c_double), ("maxiter", C.c_size_t), ("inner_maxiter", C.c_size_t),
                ("precision", C.c_int), ("family", C.c_int), ("itol", C.c_double)]


class IvSpec(C.Structure):
    _fields_ = [("vce", C.c_int), ("tol", C.c_double), ("maxiter", C.c_size_t), ("precision", C.c_int)]


class IvOut(C.Structure):
    _fields_ = ([("b", C.POINTER(C.c_double)), ("V", C.POINTER(C.c_double)), ("status", C.POINTER(C.c_uint8))]
                + [(k, C.c_double) for k in ("N", "df_r", "df_m", "df_a", "sdofminus", "rss", "rmse", "F",
                                             "N_clust", "ic")]
                + [("endog_ct", C.c_int32), ("inexog_ct", C.c_int32), ("exexog_ct", C.c_int32)])


class ServerConfig(C.Structure):
    _fields_ = [("workers", C.c_int), ("hbm_budget", C.c_size_t), ("dry_run", C.c_int)]


class Request(C.Structure):
    _fields_ = [("model", C.c_int), ("codes", C.POINTER(u32p)), ("g", u32p), ("nterms", C.c_int),
                ("cl_codes", C.POINTER(u32p)), ("cl_g", u32p), ("ncl", C.c_int), ("w", f64p),
                ("weight_kind", C.c_int), ("n", C.c_size_t), ("cols", C.POINTER(f64p)), ("nx", C.c_size_t),
                ("nendog", C.c_size_t), ("ninst", C.c_size_t), ("vce", C.c_int), ("tol", C.c_double),
                ("maxiter", C.c_size_t), ("precision", C.c_int), ("b", f64p), ("V", f64p),
                ("dry_run_us", C.c_uint64)]


class RequestResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("bytes", C.c_uint64), ("N", C.c_double), ("iterations", C.c_uint64), ("converged", C.c_int32),
                ("launches", C.c_uint64), ("prep_s", C.c_double)]


MODELS = {"ols": 0, "iv": 1, "logit": 2, "poisson": 3}
VCES = {"ols": {"unadjusted": 0, "robust": 1, "cluster": 2}, "iv": {"unadjusted": 0, "robust": 1, "cluster": 2},
        "logit": {"oim": 0, "robust": 1, "cluster": 2}, "poisson": {"robust": 1, "cluster": 2}}

FAMILY_POISSON = 1
FAMILY_LOGIT = 2


class GlmOut(C.Structure):
    _fields_ = [("b", C.POINTER(C.c_double)), ("V", C.POINTER(C.c_double)), ("status", C.POINTER(C.c_uint8)),
                ("N", C.c_double), ("deviance", C.c_double), ("ll", C.c_double), ("chi2", C.c_double),
                ("df_m", C.c_double), ("N_clust", C.c_double), ("iterations", C.c_uint64),
                ("pcg_iterations", C.c_uint64), ("converged", C.c_int32)]


class OlsOut(C.Structure):
    _fields_ = ([("b", C.POINTER(C.c_double)), ("V", C.POINTER(C.c_double)), ("status", C.POINTER(C.c_uint8)),
                 ("resid", C.POINTER(C.c_double)), ("d", C.POINTER(C.c_double)),
                 ("groupvar", C.POINTER(C.c_double)), ("dof_table", C.POINTER(C.c_double)),
                 ("nslots", C.c_int32), ("k_all", C.c_int32), ("y_absorbed", C.c_int32)]
                + [(k, C.c_double) for k in OLS_SCALARS])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m fereg_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _setup(_lib)
    return _lib


def _setup(L):
    L.fereg_last_error.restype = C.c_char_p
    L.fereg_absorber_create.argtypes = [C.POINTER(u32p), u32p, C.c_int, f64p, C.c_size_t, P, C.POINTER(P)]
    L.fereg_absorber_destroy.argtypes = [P]
    L.fereg_absorber_n.argtypes = [P]
    L.fereg_absorber_n.restype = C.c_size_t
    L.fereg_absorber_coefs_len.argtypes = [P]
    L.fereg_absorber_coefs_len.restype = C.c_size_t
    L.fereg_absorber_row_order.argtypes = [P, u32p]
    L.fereg_absorber_weights.argtypes = [P, f64p, C.POINTER(C.c_int)]
    L.fereg_absorber_set_weights.argtypes = [P, f64p]
    L.fereg_absorber_set_weights_device.argtypes = [P, P]
    L.fereg_absorber_residualize.argtypes = [P, f64p, C.c_size_t, C.c_double, C.c_size_t, C.c_int, f64p, f64p,
                                             C.POINTER(SolveInfo)]
    L.fereg_absorber_residualize_ex.argtypes = [P, P, C.c_int, C.c_size_t, C.c_double, C.c_size_t, C.c_int, f64p,
                                                f64p, C.c_int, C.POINTER(SolveInfo)]
    L.fereg_absorber_fit_rows.argtypes = [P, f64p, C.c_size_t, C.c_size_t, f64p]
    L.fereg_absorber_term_values.argtypes = [P, f64p, C.c_size_t, C.c_size_t, f64p]
    L.fereg_absorber_info.argtypes = [P, u64p]
    L.fereg_absorber_apply.argtypes = [P, f64p, C.c_size_t, f64p]
    L.fereg_absorber_rhs.argtypes = [P, f64p, C.c_size_t, f64p, f64p, f64p, f64p]
    L.fereg_absorber_precond.argtypes = [P, f64p, C.c_size_t, f64p]
    L.fereg_absorber_weight_state.argtypes = [P, f64p, f64p, f64p, u8p, f64p]
    L.fereg_absorber_rhs_noalloc.argtypes = [P, P, C.c_size_t, P, P, P]
    L.fereg_session_create.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.POINTER(u32p), u32p, C.c_int, f64p, C.c_int,
                                       C.c_size_t, C.c_uint64, P, C.POINTER(P)]
    L.fereg_session_destroy.argtypes = [P]
    L.fereg_session_row_order.argtypes = [P, u32p]
    L.fereg_session_ols.argtypes = [P, P, C.c_int, C.c_size_t, C.POINTER(OlsSpec), C.POINTER(OlsOut)]
    L.fereg_session_launches.argtypes = [P]
    L.fereg_session_launches.restype = C.c_uint64
    L.fereg_session_stream.argtypes = [P]
    L.fereg_session_stream.restype = P
    L.fereg_session_set_profiling.argtypes = [P, C.c_int]
    L.fereg_session_info.argtypes = [P, u64p]
    L.fereg_session_solver_stats.argtypes = [P, u64p]
    L.fereg_absorber_solver_stats.argtypes = [P, u64p]
    L.fereg_session_poisson.argtypes = [P, P, C.c_int, C.c_size_t, C.POINTER(GlmSpec), C.POINTER(GlmOut)]
    L.fereg_session_iv.argtypes = [P, P, C.c_int, C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(IvSpec),
                                   C.POINTER(IvOut)]
    L.fereg_amg_probe.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, C.c_int, u32p, u32p, u64p, f64p]
    L.fereg_structure_digest.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, u64p]
    L.fereg_structure_compare.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, u64p]
    L.fereg_factorize.argtypes = [f64p, C.c_size_t, u32p, u32p]
    L.fereg_combine.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, u32p, u32p]
    L.fereg_drop_singletons.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, f64p, f64p, C.c_int, C.c_int,
                                        u8p, u64p, u64p]
    L.fereg_restrict.argtypes = [u32p, C.c_uint32, u8p, C.c_size_t, u32p, u32p, u64p]
    L.fereg_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(P)]
    L.fereg_server_submit.argtypes = [P, C.POINTER(Request), C.POINTER(C.c_uint64)]
    L.fereg_server_wait.argtypes = [P, C.c_uint64, C.POINTER(RequestResult), C.c_char_p, C.c_size_t]
    L.fereg_server_stats.argtypes = [P, u64p]
    L.fereg_server_destroy.argtypes = [P]
    L.fereg_server_destroy.restype = None
    L.fereg_session_glm.argtypes = [P, P, C.c_int, C.c_size_t, C.POINTER(GlmSpec), C.POINTER(GlmOut)]
    L.fereg_session_wildboot.argtypes = [P, P, C.c_int, C.c_size_t, C.POINTER(OlsSpec), C.POINTER(BootSpec),
                                         C.POINTER(BootOut)]
    L.fereg_session_phase_times.argtypes = [P, f64p, u64p]
    L.fereg_absorber_stream.argtypes = [P]
    L.fereg_absorber_stream.restype = P
    L.fereg_absorber_set_profiling.argtypes = [P, C.c_int]
    L.fereg_absorber_phase_times.argtypes = [P, f64p, u64p]
    L.fereg_absorber_launches.argtypes = [P]
    L.fereg_absorber_launches.restype = C.c_uint64
    L.fereg_absorber_escalations.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    ip = C.POINTER(C.c_int)
    L.fereg_absorber_create_terms.argtypes = [C.POINTER(u32p), u32p, ip, ip, C.POINTER(f64p), C.c_int, f64p,
                                              C.c_size_t, P, C.POINTER(P)]
    L.fereg_absorber_has_slopes.argtypes = [P]
    L.fereg_absorber_term_values_len.argtypes = [P]
    L.fereg_absorber_term_values_len.restype = C.c_size_t
    L.fereg_slope_weight_state.argtypes = [P, f64p, f64p, u8p]
    L.fereg_slope_apply.argtypes = [P, f64p, C.c_size_t, f64p]
    L.fereg_slope_precond.argtypes = [P, f64p, C.c_size_t, f64p]
    L.fereg_slope_rhs.argtypes = [P, f64p, C.c_size_t, f64p, f64p]
    L.fereg_slope_structure.argtypes = [P, u64p, u32p]
    L.fereg_session_relu.argtypes = [P, P, C.c_int, C.c_size_t, C.c_double, C.c_size_t, u8p, f64p, u64p]
    L.fereg_session_create_terms.argtypes = [C.POINTER(u32p), u32p, ip, ip, C.POINTER(f64p), C.c_int, C.POINTER(u32p),
                                             u32p, C.c_int, f64p, C.c_int, C.c_size_t, C.c_uint64, P, C.POINTER(P)]


def _term_shapes(ncodes, intercept, slopes, n):
    """ctypes arrays of the terms' shapes: intercept flags, slope counts and the slope variables
    (kept order) term after term; the arrays are returned to keep them alive."""
    icpt = [1] * ncodes if intercept is None else [int(bool(v)) for v in intercept]
    sl = [[] for _ in range(ncodes)] if slopes is None else [list(t) for t in slopes]
    if len(icpt) != ncodes or len(sl) != ncodes:
        raise ValueError("intercept and slopes need one entry per term")
    keep = [np.ascontiguousarray(x, dtype=np.float64) for t in sl for x in t]
    if any(len(x) != n for x in keep):
        raise ValueError("slope variables need one value per row")
    ia = (C.c_int * max(1, ncodes))(*icpt)
    na = (C.c_int * max(1, ncodes))(*[len(t) for t in sl])
    sa = (f64p * max(1, len(keep)))(*[_p(x, f64p) for x in keep])
    return ia, na, sa, keep, any(not v for v in icpt) or any(sl)


def declared_symbols():
    """Function names declared in include/fereg_b200.h."""
    import re

    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fereg_[a-z0-9_]+)\s*\(", text)))


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _check(rc):
    if rc:
        raise FeregError(rc, lib().fereg_last_error().decode())


class Absorber:
    """Host mirror of the reference `Absorber` (absorber.rs:62-97) over the B200 solver."""

    def __init__(self, codes, g, w=None, intercept=None, slopes=None):
        """intercept / slopes (solve.rs:338 build): per term its intercept flag and its slope
        variables (kept order); a term with slopes or without an intercept makes the absorber
        the heterogeneous-slope solver (slopes.rs SlopeSolver)."""
        self.n = len(codes[0]) if codes else 0
        self._codes = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
        self.g = np.asarray(g, dtype=np.uint32)
        ptrs = (u32p * max(1, len(self._codes)))(*[_p(a, u32p) for a in self._codes])
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        h = P()
        if intercept is None and slopes is None:
            _check(lib().fereg_absorber_create(ptrs, _p(self.g, u32p), len(self._codes), _p(wa, f64p), self.n, None,
                                               C.byref(h)))
        else:
            ia, na, sa, self._slopes, _ = _term_shapes(len(self._codes), intercept, slopes, self.n)
            _check(lib().fereg_absorber_create_terms(ptrs, _p(self.g, u32p), ia, na, sa, len(self._codes),
                                                     _p(wa, f64p), self.n, None, C.byref(h)))
        self.h = h
        self.has_slopes = bool(lib().fereg_absorber_has_slopes(self.h))
        info = np.zeros(9, dtype=np.uint64)
        _check(lib().fereg_absorber_info(self.h, _p(info, u64p)))
        self.m, self.g1, self.ncells, self.nb, self.m_small = (int(v) for v in info[1:6])
        self.fe1 = int(np.int64(info[6]))
        self.coefs_len = int(lib().fereg_absorber_coefs_len(self.h))
        self.term_values_len = int(lib().fereg_absorber_term_values_len(self.h))
        self._slot_g = []  # levels of every term-values slot
        icpt = [True] * len(self._codes) if intercept is None else [bool(v) for v in intercept]
        sl = [[] for _ in self._codes] if slopes is None else slopes
        for q, gq in enumerate(self.g):
            self._slot_g += [int(gq)] * (int(icpt[q]) + len(sl[q]))

    def close(self):
        if getattr(self, "h", None):
            lib().fereg_absorber_destroy(self.h)
            self.h = None

    __del__ = close

    def row_order(self):
        out = np.empty(self.n, dtype=np.uint32)
        _check(lib().fereg_absorber_row_order(self.h, _p(out, u32p)))
        return out

    def weights(self):
        out = np.empty(self.n)
        has = C.c_int()
        _check(lib().fereg_absorber_weights(self.h, _p(out, f64p), C.byref(has)))
        return out if has.value else None

    def set_weights_device(self, ptr):
        """Row-order weights in device memory (pointer); the weight state is computed on the device."""
        _check(lib().fereg_absorber_set_weights_device(self.h, P(ptr)))

    def set_weights(self, w_rows):
        wa = None if w_rows is None else np.ascontiguousarray(w_rows, dtype=np.float64)
        _check(lib().fereg_absorber_set_weights(self.h, _p(wa, f64p)))

    def residualize(self, z, tol=1e-8, maxiter=16000, want_coefs=False, warm=None, precision=PREC_F64):
        """Residualizes the n x r row-major host block `z` (row order) in place."""
        assert z.dtype == np.float64 and z.flags.c_contiguous
        r = z.shape[1] if z.ndim == 2 else 1
        coefs = np.empty((self.coefs_len, r)) if want_coefs else None
        wa = None if warm is None else np.ascontiguousarray(warm, dtype=np.float64)
        info = SolveInfo()
        _check(lib().fereg_absorber_residualize_ex(self.h, z.ctypes.data_as(P), 0, r, tol, maxiter, int(want_coefs),
                                                   _p(wa, f64p), _p(coefs, f64p), precision, C.byref(info)))
        return dict(iterations=int(info.iterations), exact=bool(info.exact), escalated=bool(info.escalated),
                    coefs=coefs)

    def residualize_device(self, z_ptr, r, tol=1e-8, maxiter=16000, want_coefs=False, warm=None,
                           precision=PREC_F64):
        """Residualizes an n x r row-major block already in device memory (pointer `z_ptr`)."""
        coefs = np.empty((self.coefs_len, r)) if want_coefs else None
        wa = None if warm is None else np.ascontiguousarray(warm, dtype=np.float64)
        info = SolveInfo()
        _check(lib().fereg_absorber_residualize_ex(self.h, P(z_ptr), 1, r, tol, maxiter, int(want_coefs),
                                                   _p(wa, f64p), _p(coefs, f64p), precision, C.byref(info)))
        return dict(iterations=int(info.iterations), exact=bool(info.exact), escalated=bool(info.escalated),
                    coefs=coefs)

    def fit_rows(self, coefs, col):
        coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        out = np.empty(self.n)
        _check(lib().fereg_absorber_fit_rows(self.h, _p(coefs, f64p), coefs.shape[1], col, _p(out, f64p)))
        return out

    def term_values(self, coefs, col):
        coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        out = np.zeros(self.term_values_len)
        _check(lib().fereg_absorber_term_values(self.h, _p(coefs, f64p), coefs.shape[1], col, _p(out, f64p)))
        res, o = [], 0
        for gq in self._slot_g:  # per term its intercept, then its slopes
            res.append(out[o:o + gq].copy())
            o += gq
        return res

    # slope-solver parity hooks
    def slope_structure(self):
        v = np.zeros(9, dtype=np.uint64)
        bt = np.zeros(max(1, len(self._codes)), dtype=np.uint32)
        _check(lib().fereg_slope_structure(self.h, _p(v, u64p), _p(bt, u32p)))
        keys = ["n", "m", "e", "ge", "be", "k", "nb", "nsmall", "m_small"]
        out = {k: int(x) for k, x in zip(keys, v)}
        out["block_terms"] = [int(x) for x in bt[:out["nb"]]]
        return out

    def slope_weight_state(self, jlen):
        st = self.slope_structure()
        minv = np.empty(st["ge"] * st["be"] ** 2)
        jinv = np.empty(jlen)
        red = np.empty(st["m"], dtype=np.uint8)
        _check(lib().fereg_slope_weight_state(self.h, _p(minv, f64p), _p(jinv, f64p), _p(red, u8p)))
        return dict(minv=minv, jinv=jinv, redundant=red.astype(bool))

    def slope_apply(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        y = np.empty_like(p)
        _check(lib().fereg_slope_apply(self.h, _p(p, f64p), p.shape[1], _p(y, f64p)))
        return y

    def slope_precond(self, r_):
        r_ = np.ascontiguousarray(r_, dtype=np.float64)
        z = np.empty_like(r_)
        _check(lib().fereg_slope_precond(self.h, _p(r_, f64p), r_.shape[1], _p(z, f64p)))
        return z

    def slope_rhs(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        r = rows.shape[1]
        y = np.empty((self.m, r))
        stats = np.empty((3, r))
        _check(lib().fereg_slope_rhs(self.h, _p(rows, f64p), r, _p(y, f64p), _p(stats, f64p)))
        return y, stats

    PHASES = ["rhs_seg", "rhs_pull", "apply_seg", "precond", "vector", "residualize", "h2d", "d2h", "apply_pull",
              "escalate"]

    def stream(self):
        """The handle's cudaStream_t as an integer."""
        return int(lib().fereg_absorber_stream(self.h) or 0)

    def set_profiling(self, on=True):
        _check(lib().fereg_absorber_set_profiling(self.h, int(on)))

    def phase_times(self):
        ms = np.zeros(len(self.PHASES))
        cnt = np.zeros(len(self.PHASES), dtype=np.uint64)
        _check(lib().fereg_absorber_phase_times(self.h, _p(ms, f64p), _p(cnt, u64p)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PHASES)}

    def launches(self):
        return int(lib().fereg_absorber_launches(self.h))

    def solver_stats(self):
        """As Session.solver_stats for this absorber."""
        v = np.zeros(4, dtype=np.uint64)
        _check(lib().fereg_absorber_solver_stats(self.h, _p(v, u64p)))
        return dict(zip(["graph_captures", "graph_launches", "graph_build_us", "fp64_finishes"], map(int, v)))

    def escalations(self):
        """Escalations so far (large blocks moved from Jacobi to the multigrid V-cycle)."""
        e = C.c_uint64()
        _check(lib().fereg_absorber_escalations(self.h, C.byref(e), None))
        return int(e.value)

    # kernel-level parity hooks
    def apply(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        y = np.empty_like(p)
        _check(lib().fereg_absorber_apply(self.h, _p(p, f64p), p.shape[1], _p(y, f64p)))
        return y

    def rhs(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        r = rows.shape[1]
        y = np.empty((self.m, r))
        b1 = np.empty((self.g1, r))
        wsq = np.empty(r)
        wsum = np.empty(r)
        _check(lib().fereg_absorber_rhs(self.h, _p(rows, f64p), r, _p(y, f64p), _p(b1, f64p), _p(wsq, f64p),
                                        _p(wsum, f64p)))
        return y, b1, wsq, wsum

    def rhs_noalloc(self, rows_ptr, r, y_ptr, b1_ptr, colsum_ptr):
        """fereg_absorber_rhs_noalloc on device pointers (queued on the handle's stream)."""
        _check(lib().fereg_absorber_rhs_noalloc(self.h, P(rows_ptr), r, P(y_ptr), P(b1_ptr), P(colsum_ptr)))

    def precond(self, r_):
        r_ = np.ascontiguousarray(r_, dtype=np.float64)
        z = np.empty_like(r_)
        _check(lib().fereg_absorber_precond(self.h, _p(r_, f64p), r_.shape[1], _p(z, f64p)))
        return z

    def weight_state(self):
        n1 = np.empty(self.g1)
        nr = np.empty(self.m)
        diag = np.empty(self.m)
        red = np.empty(self.m, dtype=np.uint8)
        sw = C.c_double()
        _check(lib().fereg_absorber_weight_state(self.h, _p(n1, f64p), _p(nr, f64p), _p(diag, f64p), _p(red, u8p),
                                                 C.byref(sw)))
        return dict(n1=n1, nr=nr, diag=diag, redundant=red.astype(bool), sw=sw.value)


class Session:
    """Host mirror of the reference `Session` as `Session::ols` uses it (ols.rs:199-470), on the
    B200 absorber. codes / clusters: prepared kept-order codes; w: kept-order weights of
    weight_kind ("aweight", "fweight", "pweight") or None."""

    def __init__(self, codes, g, clusters=(), cl_g=(), w=None, weight_kind=None, num_singletons=0, intercept=None,
                 slopes=None, n=None):
        """intercept / slopes: the terms' shapes as for Absorber (slope terms make the session's
        absorber the slope solver and add one dof slot per slope); n: the rows, when neither terms,
        clusters nor weights give it (no absorbed terms: the constant alone)."""
        if n is None:
            n = len(codes[0]) if len(codes) else len(clusters[0]) if len(clusters) else len(w)
        self._codes = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
        self._cl = [np.ascontiguousarray(c, dtype=np.uint32) for c in clusters]
        garr = np.asarray(g, dtype=np.uint32)
        cgarr = np.asarray(cl_g, dtype=np.uint32)
        cp = (u32p * max(1, len(self._codes)))(*[_p(c, u32p) for c in self._codes])
        clp = (u32p * max(1, len(self._cl)))(*[_p(c, u32p) for c in self._cl])
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        h = P()
        wk = WEIGHT_KIND[weight_kind if w is not None else None]
        if intercept is None and slopes is None:
            _check(lib().fereg_session_create(cp, _p(garr, u32p), len(self._codes), clp, _p(cgarr, u32p),
                                              len(self._cl), _p(wa, f64p), wk, n, int(num_singletons), None,
                                              C.byref(h)))
        else:
            ia, na, sa, self._slopes, _ = _term_shapes(len(self._codes), intercept, slopes, n)
            _check(lib().fereg_session_create_terms(cp, _p(garr, u32p), ia, na, sa, len(self._codes), clp,
                                                    _p(cgarr, u32p), len(self._cl), _p(wa, f64p), wk, n,
                                                    int(num_singletons), None, C.byref(h)))
        self.h = h
        self.n = n

    def close(self):
        if getattr(self, "h", None):
            lib().fereg_session_destroy(self.h)
            self.h = None

    __del__ = close

    def row_order(self):
        out = np.empty(self.n, dtype=np.uint32)
        _check(lib().fereg_session_row_order(self.h, _p(out, u32p)))
        return out

    def info(self):
        """Structure of the session's absorber: n, m, g1, ncells, nb, m_small, fe1, small_work,
        small_blocks."""
        v = np.zeros(9, dtype=np.uint64)
        _check(lib().fereg_session_info(self.h, _p(v, u64p)))
        keys = ["n", "m", "g1", "ncells", "nb", "m_small", "fe1", "small_work", "small_blocks"]
        out = {k: int(x) for k, x in zip(keys, v)}
        out["fe1"] = int(np.int64(v[6]))
        return out

    def launches(self):
        return int(lib().fereg_session_launches(self.h))

    def solver_stats(self):
        """Counters of the device PCG loop: graphs captured, graph launches, host microseconds of
        the captures, FP32-refined solves finished in FP64."""
        v = np.zeros(4, dtype=np.uint64)
        _check(lib().fereg_session_solver_stats(self.h, _p(v, u64p)))
        return dict(zip(["graph_captures", "graph_launches", "graph_build_us", "fp64_finishes"], map(int, v)))

    PHASES = Absorber.PHASES + ["dof", "colstats", "gram", "variance", "weights"]

    def set_profiling(self, on=True):
        _check(lib().fereg_session_set_profiling(self.h, int(on)))

    def phase_times(self):
        ms = np.zeros(len(self.PHASES))
        cnt = np.zeros(len(self.PHASES), dtype=np.uint64)
        _check(lib().fereg_session_phase_times(self.h, _p(ms, f64p), _p(cnt, u64p)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PHASES)}

    def stream(self):
        return int(lib().fereg_session_stream(self.h) or 0)

    def _call(self, ptr, on_device, nx, vce, noconstant, firstpair, want_groupvar, want_resid, want_d, tol, maxiter,
              precision):
        k_all = nx + 1
        b = np.zeros(k_all)
        V = np.zeros((k_all, k_all))
        status = np.zeros(max(1, nx), dtype=np.uint8)
        resid = np.empty(self.n) if want_resid else None
        d = np.empty(self.n) if want_d else None
        gv = np.empty(self.n) if want_groupvar else None
        table = np.zeros((64, 5))
        spec = OlsSpec(VCE[vce], int(noconstant), int(firstpair), int(want_groupvar), tol, maxiter, precision)
        out = OlsOut(_p(b, f64p), _p(V, f64p), _p(status, u8p), _p(resid, f64p), _p(d, f64p), _p(gv, f64p),
                     _p(table, f64p))
        _check(lib().fereg_session_ols(self.h, P(ptr), int(on_device), nx, C.byref(spec), C.byref(out)))
        k = out.k_all
        return dict(b=b[:k], V=V.ravel()[: k * k].reshape(k, k).copy(), status=status[:nx],
                    resid=resid, d=d, groupvar=gv, dof_table=table[: out.nslots], y_absorbed=bool(out.y_absorbed),
                    scalars={s: getattr(out, s) for s in OLS_SCALARS})

    def ols(self, rows, nx=None, vce="unadjusted", noconstant=False, firstpair=False, want_groupvar=False,
            want_resid=False, want_d=False, tol=1e-8, maxiter=16000, precision=PREC_F64):
        """OLS of column 0 on the other columns of the n x (1 + nx) host block (row order);
        the block is copied to the device (left unchanged)."""
        assert rows.dtype == np.float64 and rows.flags.c_contiguous
        nx = rows.shape[1] - 1 if nx is None else nx
        return self._call(rows.ctypes.data, 0, nx, vce, noconstant, firstpair, want_groupvar, want_resid, want_d,
                          tol, maxiter, precision)

    def ols_device(self, ptr, nx, vce="unadjusted", noconstant=False, firstpair=False, want_groupvar=False,
                   want_resid=False, want_d=False, tol=1e-8, maxiter=16000, precision=PREC_F64):
        """As ols() on an n x (1 + nx) block in device memory (pointer)."""
        return self._call(ptr, 1, nx, vce, noconstant, firstpair, want_groupvar, want_resid, want_d, tol, maxiter,
                          precision)

    def wildboot(self, rows, coef=0, r0=0.0, reps=999, seed=1, tile=256, tol=1e-8, maxiter=16000,
                 precision=PREC_F64, boot_tol=None, boot_precision=None, noconstant=False, firstpair=False,
                 on_device=False, nx=None):
        """WCR11 wild cluster bootstrap of regressor `coef` (H0: b[coef] = r0) on the n x (1 + nx)
        block (row order; host array, or a device pointer with on_device=True). Returns stat, se,
        point, pvalue, reps, full_enum and the draws' t statistics."""
        if on_device:
            ptr = rows
            assert nx is not None
        else:
            assert rows.dtype == np.float64 and rows.flags.c_contiguous
            ptr = rows.ctypes.data
            nx = rows.shape[1] - 1
        spec = OlsSpec(2, int(noconstant), int(firstpair), 0, tol, maxiter, precision)
        bs = BootSpec(coef, r0, reps, seed, tile, tol if boot_tol is None else boot_tol, maxiter,
                      precision if boot_precision is None else boot_precision)
        t = np.full(reps, np.nan)
        out = BootOut(0, 0, 0, 0, 0, 0, _p(t, f64p))
        _check(lib().fereg_session_wildboot(self.h, P(ptr), int(on_device), nx, C.byref(spec), C.byref(bs),
                                            C.byref(out)))
        return dict(stat=out.stat, se=out.se, point=out.point, pvalue=out.pvalue, reps=int(out.reps),
                    full_enum=bool(out.full_enum), t_boot=t[: int(out.reps)].copy())

    def iv(self, rows, nx, nendog, ninst, vce="unadjusted", tol=1e-8, maxiter=16000, precision=PREC_F64,
           on_device=False):
        """2SLS of column 0 on [exog (nx), endog (nendog)] with instruments [inst (ninst), exog]:
        the n x (1 + nx + nendog + ninst) block [y, exog, endog, inst] in row order (host array,
        or a device pointer with on_device=True). b and V are in the order [endog, exog]."""
        if on_device:
            ptr = rows
        else:
            assert rows.dtype == np.float64 and rows.flags.c_contiguous
            assert rows.shape[1] == 1 + nx + nendog + ninst
            ptr = rows.ctypes.data
        k = nendog + nx
        b = np.zeros(max(1, k))
        V = np.zeros((max(1, k), max(1, k)))
        status = np.zeros(max(1, nx + nendog + ninst), dtype=np.uint8)
        spec = IvSpec({"unadjusted": 0, "robust": 1, "cluster": 2}[vce], tol, maxiter, precision)
        out = IvOut(_p(b, f64p), _p(V, f64p), _p(status, u8p))
        _check(lib().fereg_session_iv(self.h, P(ptr), int(on_device), nx, nendog, ninst, C.byref(spec),
                                      C.byref(out)))
        sc = {k_: getattr(out, k_) for k_ in ("N", "df_r", "df_m", "df_a", "sdofminus", "rss", "rmse", "F",
                                               "N_clust", "ic", "endog_ct", "inexog_ct", "exexog_ct")}
        return dict(b=b[:k], V=V[:k, :k], status=status[: nx + nendog + ninst], scalars=sc)

    def poisson(self, rows, vce="robust", tol=1e-8, maxiter=10000, inner_maxiter=16000, precision=PREC_F64,
                on_device=False, nx=None, itol=1e-10):
        """Poisson PML of column 0 (y >= 0) on the other columns of the n x (1 + nx) block (row
        order; host array, or a device pointer with on_device=True)."""
        return self.glm(rows, "poisson", vce, tol, maxiter, inner_maxiter, precision, on_device, nx, itol)

    def logit(self, rows, vce="oim", tol=1e-8, maxiter=10000, inner_maxiter=16000, precision=PREC_F64,
              on_device=False, nx=None, itol=1e-10):
        """Logit of column 0 (y in {0, 1}) on the other columns, as `poisson`."""
        return self.glm(rows, "logit", vce, tol, maxiter, inner_maxiter, precision, on_device, nx, itol)

    def relu_separation(self, rows, itol=1e-10, inner_maxiter=16000):
        """One ReLU separation check (glm/separation.rs:61) of the Poisson outcome in column 0
        with the regressors in the other columns of the n x (1 + nx) host block (row order).
        Returns the separated rows (bool, row order), the certificate, the ReLU and PCG
        iterations and whether the check certified its result."""
        assert rows.dtype == np.float64 and rows.flags.c_contiguous
        sep = np.zeros(self.n, dtype=np.uint8)
        cert = np.zeros(self.n)
        o = np.zeros(4, dtype=np.uint64)
        _check(lib().fereg_session_relu(self.h, P(rows.ctypes.data), 0, rows.shape[1] - 1, itol, inner_maxiter,
                                        _p(sep, u8p), _p(cert, f64p), _p(o, u64p)))
        return dict(separated=sep.astype(bool), certificate=cert, num_separated=int(o[0]), iterations=int(o[1]),
                    pcg_iterations=int(o[2]), complete=bool(o[3]))

    def glm(self, rows, family, vce="robust", tol=1e-8, maxiter=10000, inner_maxiter=16000, precision=PREC_F64,
            on_device=False, nx=None, itol=1e-10):
        if on_device:
            ptr = rows
            assert nx is not None
        else:
            assert rows.dtype == np.float64 and rows.flags.c_contiguous
            ptr = rows.ctypes.data
            nx = rows.shape[1] - 1
        b = np.zeros(max(1, nx))
        V = np.zeros((max(1, nx), max(1, nx)))
        status = np.zeros(max(1, nx), dtype=np.uint8)
        fam = {"poisson": FAMILY_POISSON, "logit": FAMILY_LOGIT}[family]
        spec = GlmSpec({"oim": 0, "robust": 1, "cluster": 2}[vce], tol, maxiter, inner_maxiter, precision, fam, itol)
        out = GlmOut(_p(b, f64p), _p(V, f64p), _p(status, u8p))
        _check(lib().fereg_session_glm(self.h, P(ptr), int(on_device), nx, C.byref(spec), C.byref(out)))
        return dict(b=b[:nx], V=V[:nx, :nx], status=status[:nx], N=out.N, deviance=out.deviance, ll=out.ll,
                    chi2=out.chi2, df_m=out.df_m, N_clust=out.N_clust, iterations=int(out.iterations),
                    pcg_iterations=int(out.pcg_iterations), converged=bool(out.converged))


class Server:
    """The library's serving engine (fereg_server_*): requests are admitted in arrival order
    while their estimated device memory fits `hbm_budget` bytes (None: 80% of the free memory),
    and `workers` of them run at once, each on its own session and CUDA stream. submit() returns
    a ticket; wait(ticket) blocks and returns the result. The arrays a request points to are kept
    alive here until it is waited for."""

    def __init__(self, workers=4, hbm_budget=None, dry_run=False):
        cfg = ServerConfig(workers, int(hbm_budget or 0), int(dry_run))
        h = P()
        _check(lib().fereg_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._live = {}

    def close(self):
        if getattr(self, "h", None):
            lib().fereg_server_destroy(self.h)
            self.h = None

    __del__ = close

    def submit(self, model, codes, g, cols, nx, nendog=0, ninst=0, clusters=(), cl_g=(), w=None, weight_kind=None,
               vce=None, tol=1e-8, maxiter=16000, precision=PREC_F64, dry_run_us=0, n=None):
        """cols: kept-order columns [y, exog (nx), endog (nendog), inst (ninst)]."""
        codes = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
        cl = [np.ascontiguousarray(c, dtype=np.uint32) for c in clusters]
        cols = [np.ascontiguousarray(c, dtype=np.float64) for c in cols]
        garr = np.asarray(g, dtype=np.uint32)
        cgarr = np.asarray(cl_g, dtype=np.uint32)
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        n = len(cols[0]) if n is None else n
        k_all = {"ols": nx + 1, "iv": nendog + nx, "logit": nx, "poisson": nx}[model]
        b = np.zeros(max(1, k_all))
        V = np.zeros((max(1, k_all), max(1, k_all)))
        cp = (u32p * max(1, len(codes)))(*[_p(c, u32p) for c in codes])
        clp = (u32p * max(1, len(cl)))(*[_p(c, u32p) for c in cl])
        colp = (f64p * len(cols))(*[_p(c, f64p) for c in cols])
        if vce is None:
            vce = {"ols": "unadjusted", "iv": "unadjusted", "logit": "oim", "poisson": "robust"}[model]
        req = Request(MODELS[model], cp, _p(garr, u32p), len(codes), clp, _p(cgarr, u32p), len(cl), _p(wa, f64p),
                      WEIGHT_KIND[weight_kind if w is not None else None], n, colp, nx, nendog, ninst,
                      VCES[model][vce], tol, maxiter, precision, _p(b, f64p), _p(V, f64p), int(dry_run_us))
        t = C.c_uint64()
        _check(lib().fereg_server_submit(self.h, C.byref(req), C.byref(t)))
        self._live[t.value] = (codes, cl, cols, garr, cgarr, wa, b, V, cp, clp, colp, k_all)
        return t.value

    def wait(self, ticket):
        res = RequestResult()
        msg = C.create_string_buffer(512)
        _check(lib().fereg_server_wait(self.h, ticket, C.byref(res), msg, 512))
        keep = self._live.pop(ticket)
        b, V, k_all = keep[6], keep[7], keep[11]
        return dict(rc=res.rc, msg=msg.value.decode(), b=b[:k_all], V=V[:k_all, :k_all], submit_s=res.submit_s,
                    admit_s=res.admit_s, done_s=res.done_s, bytes=int(res.bytes), N=res.N,
                    iterations=int(res.iterations), converged=bool(res.converged), launches=int(res.launches),
                    prep_s=res.prep_s)

    def stats(self):
        v = np.zeros(8, dtype=np.uint64)
        _check(lib().fereg_server_stats(self.h, _p(v, u64p)))
        keys = ["submitted", "completed", "rejected", "peak_bytes", "peak_running", "budget", "running", "launches"]
        return {k: int(x) for k, x in zip(keys, v)}


# ---------------------------------------------------------------------------------------------
# Sample preparation on the device (the reference's Session::prepare steps, factor.rs / sample.rs)

FAMILY_CODE = {None: 0, "gaussian": 0, "poisson": 1, "logit": 2}


def factorize(x):
    """factor.rs:38 factorize on the device: (codes in ascending value order, level count)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    codes = np.empty(len(x), dtype=np.uint32)
    g = C.c_uint32()
    _check(lib().fereg_factorize(_p(x, f64p), len(x), _p(codes, u32p), C.byref(g)))
    return codes, int(g.value)


def combine(parts, nl):
    """factor.rs:255 combine on the device: codes of the interaction of code columns."""
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in parts]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    nla = np.asarray(nl, dtype=np.uint32)
    out = np.empty(len(arrs[0]), dtype=np.uint32)
    g = C.c_uint32()
    _check(lib().fereg_combine(ptrs, _p(nla, u32p), len(arrs), len(out), _p(out, u32p), C.byref(g)))
    return out, int(g.value)


def drop_singletons(codes, g, fw=None, y=None, family=None, singletons=True, alive=None):
    """sample.rs:44-72 on the device: (alive, singletons dropped, fe-separated dropped)."""
    n = len(codes[0])
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    garr = np.asarray(g, dtype=np.uint32)
    al = np.ones(n, dtype=np.uint8) if alive is None else np.ascontiguousarray(alive, dtype=np.uint8).copy()
    fwa = None if fw is None else np.ascontiguousarray(fw, dtype=np.float64)
    ya = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
    s, f = C.c_uint64(), C.c_uint64()
    _check(lib().fereg_drop_singletons(ptrs, _p(garr, u32p), len(arrs), n, _p(fwa, f64p), _p(ya, f64p),
                                       FAMILY_CODE[family], int(singletons), _p(al, u8p), C.byref(s), C.byref(f)))
    return al.astype(bool), int(s.value), int(f.value)


def restrict(codes, g, alive):
    """factor.rs:281 restrict on the device: the kept rows' codes renumbered densely."""
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    al = np.ascontiguousarray(alive, dtype=np.uint8)
    out = np.empty(max(1, int(al.sum())), dtype=np.uint32)
    nl, kept = C.c_uint32(), C.c_uint64()
    _check(lib().fereg_restrict(_p(codes, u32p), g, _p(al, u8p), len(codes), _p(out, u32p), C.byref(nl),
                                C.byref(kept)))
    return out[: int(kept.value)], int(nl.value)


def prepare(factors, absorb, fw=None, y=None, family=None, singletons=True):
    """The sample preparation of Session::prepare for the absorbed terms, on the device:
    factorize every factor column, combine the factors of each term (interactions), drop
    singletons (and, with a GLM family and its outcome, fe-separated rows) cyclically, and
    renumber each term's codes over the kept rows. Returns alive, the drop counts and the kept
    terms as (codes, levels)."""
    fac = [factorize(f) for f in factors]
    terms = [combine([fac[i][0] for i in t], [fac[i][1] for i in t]) for t in absorb]
    if terms:
        alive, s, f = drop_singletons([c for c, _ in terms], [g for _, g in terms], fw, y, family, singletons)
    else:
        alive, s, f = np.ones(len(factors[0]), dtype=bool), 0, 0
    kept = [restrict(c, g, alive) for c, g in terms]
    return dict(alive=alive, num_singletons=s, fe_separated=f, terms=kept)


def structure_digest(codes, g):
    """Host-only test hook: counts of the cell structure a session would build (cells, segments,
    reduced coordinates, small coordinates, blocks, FE1 index) and a digest of its arrays and
    coordinate lists."""
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    garr = np.asarray(g, dtype=np.uint32)
    out = np.zeros(7, dtype=np.uint64)
    _check(lib().fereg_structure_digest(ptrs, _p(garr, u32p), len(arrs), len(arrs[0]), _p(out, u64p)))
    keys = ["cells", "segments", "m", "m_small", "blocks", "fe1", "digest"]
    return {k: int(v) for k, v in zip(keys, out)}


def structure_compare(codes, g):
    """Test hook (device): differences between the cell structure built on the device and on the
    host, per array (all 0 when they are identical)."""
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    garr = np.asarray(g, dtype=np.uint32)
    out = np.zeros(9, dtype=np.uint64)
    _check(lib().fereg_structure_compare(ptrs, _p(garr, u32p), len(arrs), len(arrs[0]), _p(out, u64p)))
    keys = ["scalars", "pi", "seg_off", "cell_row", "coord", "pl_off", "pl_cell", "pl_seg", "pl_other"]
    return {k: int(v) for k, v in zip(keys, out)}


def amg_probe(codes, g, max_levels=16):
    """Host-only test hook: the level sizes, nonzeros and relative row sums of the multigrid
    hierarchy an escalation would build for the structure's first block above 768 levels."""
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    garr = np.asarray(g, dtype=np.uint32)
    sizes = np.zeros(max_levels, dtype=np.uint32)
    nnz = np.zeros(max_levels, dtype=np.uint64)
    rs = np.zeros(max_levels)
    nl = C.c_uint32()
    _check(lib().fereg_amg_probe(ptrs, _p(garr, u32p), len(arrs), len(arrs[0]), max_levels, C.byref(nl),
                                 _p(sizes, u32p), _p(nnz, u64p), _p(rs, f64p)))
    k = min(int(nl.value), max_levels)
    return dict(levels=int(nl.value), sizes=sizes[:k].astype(int), nnz=nnz[:k].astype(int), row_sum=rs[:k])
