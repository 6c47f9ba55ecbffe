"""TEST INFRASTRUCTURE — ctypes wrapper of the CPU oracle (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use this
module, as the checker; the product (fereg_b200) never imports it.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force=False):
    """Compiles the oracle (make in oracle/)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
        os.path.join(HERE, "fereg_oracle.cpp")
    ):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _setup(_lib)
    return _lib


P = C.c_void_p
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f64p = C.POINTER(C.c_double)
u8p = C.POINTER(C.c_uint8)


class OlsSpec(C.Structure):
    _fields_ = [
        ("n_input", C.c_size_t),
        ("nfactors", C.c_int),
        ("factors", C.POINTER(f64p)),
        ("nterms", C.c_int),
        ("term_nf", C.POINTER(C.c_int)),
        ("term_f", C.POINTER(C.c_int)),
        ("ncl", C.c_int),
        ("cl_nf", C.POINTER(C.c_int)),
        ("cl_f", C.POINTER(C.c_int)),
        ("y", f64p),
        ("nx", C.c_int),
        ("x", C.POINTER(f64p)),
        ("w", f64p),
        ("weight_kind", C.c_int),
        ("vce", C.c_int),
        ("drop_singletons", C.c_int),
        ("noconstant", C.c_int),
        ("firstpair", C.c_int),
        ("tol", C.c_double),
        ("maxiter", C.c_size_t),
        ("threads", C.c_int),
    ]


SCALARS = [
    "N", "rank", "df_r", "df_m", "df_a", "df_a_initial", "df_a_redundant", "df_a_nested",
    "N_clust", "N_clustervars", "N_clust1", "N_clust2", "num_singletons", "N_full", "report_constant",
    "rss", "tss", "tss_within", "mss", "rmse", "r2", "r2_a", "r2_within", "r2_a_within", "ll", "ll_0", "F",
    "sumweights", "ic", "y_absorbed",
]


class OlsOut(C.Structure):
    _fields_ = [
        ("b", f64p),
        ("V", f64p),
        ("status", u8p),
        ("sample", u8p),
        ("resid", f64p),
        ("d", f64p),
        ("groupvar", f64p),
        ("dof_table", f64p),
        ("nslots", C.c_int),
        ("k_all", C.c_int),
    ] + [(s, C.c_double) for s in SCALARS]


def _setup(L):
    L.orc_last_error.restype = C.c_char_p
    L.orc_absorber_create.restype = P
    L.orc_absorber_create.argtypes = [C.POINTER(u32p), u32p, C.c_int, f64p, C.c_size_t]
    L.orc_absorber_destroy.argtypes = [P]
    L.orc_absorber_info.argtypes = [P, u64p]
    L.orc_absorber_row_order.argtypes = [P, u32p]
    L.orc_absorber_structure.argtypes = [P, u32p, u32p, u32p, u64p]
    L.orc_absorber_weight_state.argtypes = [P, f64p, f64p, f64p, u8p, f64p]
    L.orc_absorber_set_weights.argtypes = [P, f64p]
    L.orc_absorber_residualize.argtypes = [P, f64p, C.c_size_t, C.c_double, C.c_size_t, C.c_int, f64p, f64p, u64p, C.POINTER(C.c_int)]
    L.orc_absorber_apply.argtypes = [P, f64p, C.c_size_t, f64p]
    L.orc_absorber_rhs.argtypes = [P, f64p, C.c_size_t, f64p, f64p, f64p, f64p]
    L.orc_absorber_precond.argtypes = [P, f64p, C.c_size_t, f64p]
    L.orc_absorber_fit_rows.argtypes = [P, f64p, C.c_size_t, C.c_size_t, f64p]
    L.orc_absorber_term_values.argtypes = [P, f64p, C.c_size_t, C.c_size_t, u32p, C.c_int, f64p]
    L.orc_ols.argtypes = [C.POINTER(OlsSpec), C.POINTER(OlsOut)]
    L.orc_session_create.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.POINTER(u32p), u32p, C.c_int, f64p, C.c_int,
                                     C.c_size_t, C.c_uint64, C.POINTER(P)]
    L.orc_session_destroy.argtypes = [P]
    L.orc_session_row_order.argtypes = [P, u32p]
    L.orc_session_ols.argtypes = [P, f64p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_double, C.c_size_t,
                                  C.POINTER(OlsOut)]
    L.orc_factorize_f64.argtypes = [f64p, C.c_size_t, u32p, u32p]
    L.orc_drop_singletons.restype = C.c_uint64
    L.orc_drop_singletons.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, f64p, u8p]
    L.orc_combine.argtypes = [C.POINTER(u32p), u32p, C.c_int, C.c_size_t, u32p, u32p]
    L.orc_mobility_groups.restype = C.c_uint64
    L.orc_mobility_groups.argtypes = [u32p, C.c_uint32, u32p, C.c_uint32, C.c_size_t, u32p]
    L.orc_splitmix_fill_u64.argtypes = [C.c_uint64, C.c_uint64, C.c_int, u64p, C.c_size_t]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_max_threads.restype = C.c_int


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def set_threads(t):
    lib().orc_set_threads(int(t))


def max_threads():
    return lib().orc_max_threads()


def factorize(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    codes = np.empty(len(x), dtype=np.uint32)
    g = C.c_uint32()
    rc = lib().orc_factorize_f64(_p(x, f64p), len(x), _p(codes, u32p), C.byref(g))
    if rc:
        raise RuntimeError(lib().orc_last_error().decode())
    return codes, int(g.value)


def combine(parts, nl):
    """factor.rs:255 combine on the oracle: codes of the interaction of code columns."""
    n = len(parts[0])
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in parts]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    nla = np.asarray(nl, dtype=np.uint32)
    out = np.empty(n, dtype=np.uint32)
    g = C.c_uint32()
    rc = lib().orc_combine(ptrs, _p(nla, u32p), len(arrs), n, _p(out, u32p), C.byref(g))
    if rc:
        raise RuntimeError(lib().orc_last_error().decode())
    return out, int(g.value)


def drop_singletons(codes, g, fw=None):
    n = len(codes[0])
    arrs = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
    ptrs = (u32p * len(arrs))(*[_p(a, u32p) for a in arrs])
    garr = np.asarray(g, dtype=np.uint32)
    alive = np.ones(n, dtype=np.uint8)
    fwa = None if fw is None else np.ascontiguousarray(fw, dtype=np.float64)
    d = lib().orc_drop_singletons(ptrs, _p(garr, u32p), len(arrs), n, _p(fwa, f64p), _p(alive, u8p))
    return alive.astype(bool), int(d)


def mobility_groups(a, ga, b, gb, want_groupvar=False):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    gv = np.empty(len(a), dtype=np.uint32) if want_groupvar else None
    k = lib().orc_mobility_groups(_p(a, u32p), ga, _p(b, u32p), gb, len(a), _p(gv, u32p))
    return (int(k), gv) if want_groupvar else int(k)


def splitmix(seed, n, index=None):
    out = np.empty(n, dtype=np.uint64)
    lib().orc_splitmix_fill_u64(seed, 0 if index is None else index, int(index is not None), _p(out, u64p), n)
    return out


class Absorber:
    """Oracle mirror of the reference `Absorber` (absorber.rs:62-97) over `FeSolver`."""

    def __init__(self, codes, g, w=None):
        self.n = len(codes[0])
        self._codes = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
        self.g = np.asarray(g, dtype=np.uint32)
        ptrs = (u32p * len(self._codes))(*[_p(a, u32p) for a in self._codes])
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        self.h = lib().orc_absorber_create(ptrs, _p(self.g, u32p), len(self._codes), _p(wa, f64p), self.n)
        info = np.zeros(8, dtype=np.uint64)
        lib().orc_absorber_info(self.h, _p(info, u64p))
        self.m, self.g1, self.ncells, self.nb, self.m_small = (int(v) for v in info[1:6])
        self.fe1 = int(np.int64(info[6]))
        self.small_work = int(info[7])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_absorber_destroy(self.h)
            self.h = None

    def row_order(self):
        out = np.empty(self.n, dtype=np.uint32)
        lib().orc_absorber_row_order(self.h, _p(out, u32p))
        return out

    def structure(self):
        seg_off = np.empty(self.g1 + 1, dtype=np.uint32)
        cc = np.empty(self.ncells * self.nb, dtype=np.uint32)
        co = np.empty(self.ncells + 1, dtype=np.uint32)
        blocks = np.empty(4 * self.nb, dtype=np.uint64)
        lib().orc_absorber_structure(self.h, _p(seg_off, u32p), _p(cc, u32p), _p(co, u32p), _p(blocks, u64p))
        trivial = self.ncells == self.n
        return dict(seg_off=seg_off, cell_codes=cc.reshape(self.ncells, self.nb), cell_obs_off=None if trivial else co,
                    blocks=blocks.reshape(self.nb, 4))

    def weight_state(self):
        n1 = np.empty(self.g1)
        nr = np.empty(self.m)
        diag = np.empty(self.m)
        red = np.empty(self.m, dtype=np.uint8)
        sw = C.c_double()
        lib().orc_absorber_weight_state(self.h, _p(n1, f64p), _p(nr, f64p), _p(diag, f64p), _p(red, u8p), C.byref(sw))
        return dict(n1=n1, nr=nr, diag=diag, redundant=red.astype(bool), sw=sw.value)

    def set_weights(self, w_rows):
        wa = None if w_rows is None else np.ascontiguousarray(w_rows, dtype=np.float64)
        rc = lib().orc_absorber_set_weights(self.h, _p(wa, f64p))
        if rc:
            raise ValueError(lib().orc_last_error().decode())

    def residualize(self, z, tol=1e-8, maxiter=16000, want_coefs=False, warm=None):
        """Residualizes the n x r row-major block `z` (row order) in place."""
        assert z.dtype == np.float64 and z.flags.c_contiguous
        r = z.shape[1] if z.ndim == 2 else 1
        coefs = np.empty(((self.m + self.g1), r)) if want_coefs else None
        wa = None if warm is None else np.ascontiguousarray(warm, dtype=np.float64)
        it = C.c_uint64()
        ex = C.c_int()
        rc = lib().orc_absorber_residualize(self.h, _p(z, f64p), r, tol, maxiter, int(want_coefs), _p(wa, f64p), _p(coefs, f64p), C.byref(it), C.byref(ex))
        if rc:
            raise RuntimeError(f"rc={rc}: {lib().orc_last_error().decode()}")
        return dict(iterations=int(it.value), exact=bool(ex.value), coefs=coefs)

    def apply(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        y = np.empty_like(p)
        lib().orc_absorber_apply(self.h, _p(p, f64p), p.shape[1], _p(y, f64p))
        return y

    def rhs(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        r = rows.shape[1]
        y = np.empty((self.m, r))
        b1 = np.empty((self.g1, r))
        wsq = np.empty(r)
        wsum = np.empty(r)
        lib().orc_absorber_rhs(self.h, _p(rows, f64p), r, _p(y, f64p), _p(b1, f64p), _p(wsq, f64p), _p(wsum, f64p))
        return y, b1, wsq, wsum

    def precond(self, r_):
        r_ = np.ascontiguousarray(r_, dtype=np.float64)
        z = np.empty_like(r_)
        lib().orc_absorber_precond(self.h, _p(r_, f64p), r_.shape[1], _p(z, f64p))
        return z

    def fit_rows(self, coefs, col):
        coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        out = np.empty(self.n)
        lib().orc_absorber_fit_rows(self.h, _p(coefs, f64p), coefs.shape[1], col, _p(out, f64p))
        return out

    def term_values(self, coefs, col):
        coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        out = np.zeros(int(self.g.sum()))
        lib().orc_absorber_term_values(self.h, _p(coefs, f64p), coefs.shape[1], col, _p(self.g, u32p), len(self.g), _p(out, f64p))
        res, o = [], 0
        for gq in self.g:
            res.append(out[o:o + gq].copy())
            o += gq
        return res


WEIGHT_KINDS = {None: 0, "aweight": 1, "fweight": 2, "pweight": 3}


def ols(factors, absorb, y, x, clusters=(), weights=None, weight_kind=None, vce="unadjusted",
        singletons=True, noconstant=False, firstpair=False, tol=1e-8, maxiter=16000,
        want_resid=False, want_d=False, want_groupvar=False, threads=0):
    """Full reghdfe-convention OLS (factorize, singletons, absorb, OLS, VCE) on the oracle.

    `factors`: list of float64 columns; `absorb`: list of lists of factor indices;
    `clusters`: list of lists of factor indices; `vce` in unadjusted/robust/cluster.
    """
    n0 = len(y)
    fac = [np.ascontiguousarray(f, dtype=np.float64) for f in factors]
    fptr = (f64p * max(1, len(fac)))(*[_p(a, f64p) for a in fac])
    tnf = np.array([len(t) for t in absorb] or [0], dtype=np.int32)
    tf = np.array([f for t in absorb for f in t] or [0], dtype=np.int32)
    cnf = np.array([len(c) for c in clusters] or [0], dtype=np.int32)
    cf = np.array([f for c in clusters for f in c] or [0], dtype=np.int32)
    ya = np.ascontiguousarray(y, dtype=np.float64)
    xs = [np.ascontiguousarray(v, dtype=np.float64) for v in x]
    xptr = (f64p * max(1, len(xs)))(*[_p(a, f64p) for a in xs])
    wa = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    sp = OlsSpec(n0, len(fac), fptr, len(absorb), _p(tnf, C.POINTER(C.c_int)), _p(tf, C.POINTER(C.c_int)),
                 len(clusters), _p(cnf, C.POINTER(C.c_int)), _p(cf, C.POINTER(C.c_int)), _p(ya, f64p), len(xs), xptr,
                 _p(wa, f64p), WEIGHT_KINDS[weight_kind], {"unadjusted": 0, "robust": 1, "cluster": 2}[vce],
                 int(singletons), int(noconstant), int(firstpair), tol, maxiter, threads)
    k_all = len(xs) + 1
    b = np.zeros(k_all)
    V = np.zeros(k_all * k_all)
    status = np.zeros(max(1, len(xs)), dtype=np.uint8)
    sample = np.zeros(n0, dtype=np.uint8)
    resid = np.full(n0, np.nan) if want_resid else None
    d = np.full(n0, np.nan) if want_d else None
    gv = np.full(n0, np.nan) if want_groupvar else None
    dof_table = np.zeros(5 * 64)
    out = OlsOut(_p(b, f64p), _p(V, f64p), _p(status, u8p), _p(sample, u8p), _p(resid, f64p), _p(d, f64p),
                 _p(gv, f64p), _p(dof_table, f64p))
    rc = lib().orc_ols(C.byref(sp), C.byref(out))
    if rc:
        raise RuntimeError(f"rc={rc}: {lib().orc_last_error().decode()}")
    ka = out.k_all
    nk = int(sample.sum())
    res = dict(b=b[:ka], V=V[: ka * ka].reshape(ka, ka), status=status[: len(xs)].copy(), sample=sample.astype(bool),
               dof_table=dof_table[: 5 * out.nslots].reshape(out.nslots, 5),
               scalars={s: getattr(out, s) for s in SCALARS})
    if want_resid:
        res["resid"] = resid[:nk]
    if want_d:
        res["d"] = d[:nk]
    if want_groupvar:
        res["groupvar"] = gv[:nk]
    return res


class Session:
    """A prepared oracle session (kept-order codes) reused across OLS calls: the CPU arm of the
    benchmark's OLS call."""

    def __init__(self, codes, g, clusters=(), cl_g=(), w=None, weight_kind=None, num_singletons=0):
        n = len(codes[0]) if len(codes) else len(clusters[0])
        self._c = [np.ascontiguousarray(c, dtype=np.uint32) for c in codes]
        self._k = [np.ascontiguousarray(c, dtype=np.uint32) for c in clusters]
        garr = np.asarray(g, dtype=np.uint32)
        cgarr = np.asarray(cl_g, dtype=np.uint32)
        cp = (u32p * max(1, len(self._c)))(*[_p(c, u32p) for c in self._c])
        kp = (u32p * max(1, len(self._k)))(*[_p(c, u32p) for c in self._k])
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        h = P()
        lib().orc_session_create(cp, _p(garr, u32p), len(self._c), kp, _p(cgarr, u32p), len(self._k), _p(wa, f64p),
                                 WEIGHT_KINDS[weight_kind if w is not None else None], n, int(num_singletons),
                                 C.byref(h))
        self.h = h
        self.n = n

    def close(self):
        if getattr(self, "h", None):
            lib().orc_session_destroy(self.h)
            self.h = None

    __del__ = close

    def row_order(self):
        out = np.empty(self.n, dtype=np.uint32)
        lib().orc_session_row_order(self.h, _p(out, u32p))
        return out

    def ols(self, rows, vce="unadjusted", noconstant=False, firstpair=False, tol=1e-8, maxiter=16000):
        """OLS of column 0 on the other columns of the n x r row-order block (residualized in place)."""
        assert rows.dtype == np.float64 and rows.flags.c_contiguous
        nx = rows.shape[1] - 1
        k_all = nx + 1
        b = np.zeros(k_all)
        V = np.zeros(k_all * k_all)
        status = np.zeros(max(1, nx), dtype=np.uint8)
        dof_table = np.zeros(5 * 64)
        out = OlsOut(_p(b, f64p), _p(V, f64p), _p(status, u8p), None, None, None, None, _p(dof_table, f64p))
        rc = lib().orc_session_ols(self.h, _p(rows, f64p), nx, {"unadjusted": 0, "robust": 1, "cluster": 2}[vce],
                                   int(noconstant), int(firstpair), tol, maxiter, C.byref(out))
        if rc:
            raise RuntimeError(f"rc={rc}: {lib().orc_last_error().decode()}")
        ka = out.k_all
        return dict(b=b[:ka], V=V[: ka * ka].reshape(ka, ka), status=status[:nx].copy(),
                    scalars={s: getattr(out, s) for s in SCALARS})
