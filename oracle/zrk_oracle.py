"""ORACLE bindings (test infrastructure only).

ctypes access to
  * ``_build/libzrk_oracle.so`` -- the plain-C restatement in zrk_oracle.c;
  * ``_ref/libzrk_ref_libc.so`` / ``_ref/libzrk_ref_fmath.so`` -- the reference's
    own zerork::mechanism library compiled from its sources (oracle/Makefile).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libzrk_oracle.so")
REF_SO = {"libc": os.path.join(HERE, "_ref", "libzrk_ref_libc.so"),
          "fmath": os.path.join(HERE, "_ref", "libzrk_ref_fmath.so")}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class ZoTables(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nsp", "nrxn", "nstep", "tot_reac", "tot_prod", "n_arr", "n_keq", "n_tb",
        "n_fo", "n_tb_eff", "n_fo_eff", "n_plog", "n_plog_pt", "n_plog_ln")] + [
        ("mw", C.POINTER(C.c_double)), ("thermo", C.POINTER(C.c_double)),
        ("step_rxn", C.POINTER(C.c_int)), ("step_dir", C.POINTER(C.c_int)),
        ("reac_ptr", C.POINTER(C.c_int)), ("reac_spc", C.POINTER(C.c_int)),
        ("prod_ptr", C.POINTER(C.c_int)), ("prod_spc", C.POINTER(C.c_int)),
        ("arr_step", C.POINTER(C.c_int)), ("arr_lnA", C.POINTER(C.c_double)),
        ("arr_n", C.POINTER(C.c_double)), ("arr_Ta", C.POINTER(C.c_double)),
        ("keq_step", C.POINTER(C.c_int)), ("keq_fwd", C.POINTER(C.c_int)),
        ("keq_dn", C.POINTER(C.c_double)),
        ("tb_fwd", C.POINTER(C.c_int)), ("tb_rev", C.POINTER(C.c_int)),
        ("tb_ptr", C.POINTER(C.c_int)), ("tb_spc", C.POINTER(C.c_int)),
        ("tb_alpha", C.POINTER(C.c_double)),
        ("fo_fwd", C.POINTER(C.c_int)), ("fo_rev", C.POINTER(C.c_int)),
        ("fo_type", C.POINTER(C.c_int)), ("fo_spc", C.POINTER(C.c_int)),
        ("fo_ptr", C.POINTER(C.c_int)), ("fo_eff_spc", C.POINTER(C.c_int)),
        ("fo_alpha", C.POINTER(C.c_double)), ("fo_par", C.POINTER(C.c_double)),
        ("plog_step", C.POINTER(C.c_int)), ("plog_pt_ptr", C.POINTER(C.c_int)),
        ("plog_ln_ptr", C.POINTER(C.c_int)), ("plog_p", C.POINTER(C.c_double)),
        ("plog_lnp", C.POINTER(C.c_double)), ("plog_lnA", C.POINTER(C.c_double)),
        ("plog_sgn", C.POINTER(C.c_double)), ("plog_n", C.POINTER(C.c_double)),
        ("plog_Ta", C.POINTER(C.c_double)),
    ]


class ZoJacPattern(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int),
                ("col_ptr", C.POINTER(C.c_int)), ("row_idx", C.POINTER(C.c_int)),
                ("last_row", C.POINTER(C.c_int)), ("n_des", C.c_int), ("n_cre", C.c_int),
                ("des_conc", C.POINTER(C.c_int)), ("des_step", C.POINTER(C.c_int)),
                ("des_nz", C.POINTER(C.c_int)), ("cre_conc", C.POINTER(C.c_int)),
                ("cre_step", C.POINTER(C.c_int)), ("cre_nz", C.POINTER(C.c_int))]


class ZoBdfOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("max_dt", C.c_double),
                ("nlscoef", C.c_double), ("max_steps", C.c_int), ("Tref", C.c_double),
                ("min_mass_frac", C.c_double), ("step_limiter", C.c_double),
                ("analytic", C.c_int), ("max_retries", C.c_int), ("retry_atol", C.c_double),
                ("retry_rtol", C.c_double), ("dT_ign", C.c_double),
                ("constant_volume", C.c_int), ("stop_ign", C.c_int), ("abstol_dens", C.c_int),
                ("fail_caps", C.c_int)]


class ZoKinetics(C.Structure):
    """zo_kinetics: a context pointer and 12 function pointers (opaque here)."""
    _fields_ = [("p%d" % i, C.c_void_p) for i in range(13)]


class ZoBdfStats(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nsteps", "nrej", "nnewt", "njac", "nlu", "nrhs", "status",
                                           "retries")]


# array name -> (dtype, size expression over the struct's counts)
TABLE_ARRAYS = {
    "mw": ("f8", lambda t: t.nsp), "thermo": ("f8", lambda t: 16 * t.nsp),
    "step_rxn": ("i4", lambda t: t.nstep), "step_dir": ("i4", lambda t: t.nstep),
    "reac_ptr": ("i4", lambda t: t.nstep + 1), "reac_spc": ("i4", lambda t: t.tot_reac),
    "prod_ptr": ("i4", lambda t: t.nstep + 1), "prod_spc": ("i4", lambda t: t.tot_prod),
    "arr_step": ("i4", lambda t: t.n_arr), "arr_lnA": ("f8", lambda t: t.n_arr),
    "arr_n": ("f8", lambda t: t.n_arr), "arr_Ta": ("f8", lambda t: t.n_arr),
    "keq_step": ("i4", lambda t: t.n_keq), "keq_fwd": ("i4", lambda t: t.n_keq),
    "keq_dn": ("f8", lambda t: t.n_keq),
    "tb_fwd": ("i4", lambda t: t.n_tb), "tb_rev": ("i4", lambda t: t.n_tb),
    "tb_ptr": ("i4", lambda t: t.n_tb + 1), "tb_spc": ("i4", lambda t: t.n_tb_eff),
    "tb_alpha": ("f8", lambda t: t.n_tb_eff),
    "fo_fwd": ("i4", lambda t: t.n_fo), "fo_rev": ("i4", lambda t: t.n_fo),
    "fo_type": ("i4", lambda t: t.n_fo), "fo_spc": ("i4", lambda t: t.n_fo),
    "fo_ptr": ("i4", lambda t: t.n_fo + 1), "fo_eff_spc": ("i4", lambda t: t.n_fo_eff),
    "fo_alpha": ("f8", lambda t: t.n_fo_eff), "fo_par": ("f8", lambda t: 8 * t.n_fo),
    "plog_step": ("i4", lambda t: t.n_plog), "plog_pt_ptr": ("i4", lambda t: t.n_plog + 1),
    "plog_ln_ptr": ("i4", lambda t: t.n_plog_pt + 1), "plog_p": ("f8", lambda t: t.n_plog_pt),
    "plog_lnp": ("f8", lambda t: t.n_plog_pt), "plog_lnA": ("f8", lambda t: t.n_plog_ln),
    "plog_sgn": ("f8", lambda t: t.n_plog_ln), "plog_n": ("f8", lambda t: t.n_plog_ln),
    "plog_Ta": ("f8", lambda t: t.n_plog_ln),
}
TABLE_COUNTS = ("nsp", "nrxn", "nstep", "tot_reac", "tot_prod", "n_arr", "n_keq", "n_tb",
                "n_fo", "n_tb_eff", "n_fo_eff", "n_plog", "n_plog_pt", "n_plog_ln")


def _bind_common(lib):
    lib.zo_tables_alloc.restype = C.POINTER(ZoTables)
    lib.zo_tables_alloc.argtypes = [C.POINTER(C.c_int)]
    lib.zo_tables_free.argtypes = [C.POINTER(ZoTables)]
    lib.zo_rate_coefs.argtypes = [C.POINTER(ZoTables), C.c_double, _dp, _dp]
    lib.zo_rates.argtypes = [C.POINTER(ZoTables), C.c_double, _dp, C.c_void_p, _dp, _dp, _dp, _dp]
    for f in ("zo_cp_R", "zo_h_RT", "zo_g_RT"):
        getattr(lib, f).argtypes = [C.POINTER(ZoTables), C.c_double, _dp]
    lib.zo_jac_pattern_new.restype = C.POINTER(ZoJacPattern)
    lib.zo_jac_pattern_new.argtypes = [C.POINTER(ZoTables)]
    lib.zo_jac_pattern_free.argtypes = [C.POINTER(ZoJacPattern)]
    lib.zo_batch_rates_jac.argtypes = [C.POINTER(ZoTables), C.POINTER(ZoJacPattern), C.c_void_p,
                                       C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double,
                                       C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.zo_batch_rates_jac.restype = C.c_int
    lib.zo_kinetics_oracle.argtypes = [C.POINTER(ZoTables), C.c_void_p]
    lib.zo_mix_thermo.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.zo_reactor_rhs_batch.argtypes = [C.POINTER(ZoTables), C.c_void_p, C.c_int, C.c_int, _dp,
                                         _dp, _dp, C.c_void_p, C.c_void_p, C.c_void_p, _dp, _dp,
                                         _dp]
    lib.zo_reactor_rhs_batch.restype = C.c_int
    lib.zo_batch_rates_jac_scaled.argtypes = [C.POINTER(ZoTables), C.POINTER(ZoJacPattern),
                                              C.c_int, _dp, _dp, _dp, C.c_double, C.c_double,
                                              C.c_double, _dp, _dp, _dp, _dp]
    lib.zo_batch_rates_jac_scaled.restype = C.c_int
    if hasattr(lib, "zo_reactor_solve_batch"):
        lib.zo_bdf_default_opts.argtypes = [C.POINTER(ZoBdfOpts)]
        lib.zo_reactor_solve_batch.argtypes = [C.POINTER(ZoTables), C.POINTER(ZoJacPattern),
                                               C.POINTER(ZoBdfOpts), C.c_int, C.c_int, C.c_double,
                                               _dp, _dp, _dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p]
        lib.zo_reactor_solve_batch.restype = C.c_int
    return lib


_oracle = None
_refs = {}


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise FileNotFoundError(f"{ORACLE_SO} missing: run `make -C oracle oracle`")
        _oracle = _bind_common(C.CDLL(ORACLE_SO))
    return _oracle


def ref_available(kind="libc"):
    return os.path.exists(REF_SO[kind])


def ref_lib(kind="libc"):
    if kind not in _refs:
        lib = _bind_common(C.CDLL(REF_SO[kind]))
        lib.zrkref_load.restype = C.c_void_p
        lib.zrkref_load.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
        lib.zrkref_free.argtypes = [C.c_void_p]
        lib.zrkref_tables.restype = C.POINTER(ZoTables)
        lib.zrkref_tables.argtypes = [C.c_void_p]
        lib.zrkref_species_name.restype = C.c_char_p
        lib.zrkref_species_name.argtypes = [C.c_void_p, C.c_int]
        lib.zrkref_krxn.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp]
        lib.zrkref_rates.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp, _dp, _dp]
        lib.zrkref_rates_limiter.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.zrkref_thermo.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp]
        lib.zrkref_batch_rates_jac.argtypes = [C.c_void_p, C.c_int, C.POINTER(ZoTables),
                                               C.POINTER(ZoJacPattern), C.c_int, _dp, _dp, _dp,
                                               C.c_double, C.c_double, C.c_double,
                                               C.c_void_p, C.c_void_p, C.c_void_p]
        lib.zrkref_batch_rates_jac.restype = C.c_int
        lib.zrkref_mix_thermo.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.zrkref_reactor_rhs_batch.argtypes = [C.c_void_p, C.POINTER(ZoTables), C.c_int, C.c_int,
                                                 _dp, _dp, _dp, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, _dp, _dp, _dp]
        lib.zrkref_reactor_rhs_batch.restype = C.c_int
        _refs[kind] = lib
    return _refs[kind]


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _mix_thermo(fn, kin, nsp, T, P, Y, E, H):
    T, P, E, H = (np.ascontiguousarray(a, dtype=np.float64) for a in (T, P, E, H))
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    n = T.shape[0]
    out = np.zeros((n, 7))
    fn(kin, nsp, n, T, P, Y, E, H, out)
    return out


def _reactor_rhs(fn, nsp, cp, T0, P0, Y0, tm, y, dpdt, e_src, y_src):
    T0, P0, tm = (np.ascontiguousarray(a, dtype=np.float64) for a in (T0, P0, tm))
    Y0 = np.ascontiguousarray(Y0, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    dp, es, ys = (None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                  for a in (dpdt, e_src, y_src))
    n = T0.shape[0]
    ydot = np.zeros((n, nsp + 1))
    nf = fn(int(cp), n, T0, P0, Y0, _vp(dp), _vp(es), _vp(ys), tm, y, ydot)
    if nf:
        raise RuntimeError(f"reactor rhs failed on {nf} states")
    return ydot


def with_counts(d):
    """A table dict (e.g. the product loader's tables) with the size fields
    the oracle's struct needs, derived from the array lengths."""
    d = dict(d)
    d.update(tot_reac=len(d["reac_spc"]), tot_prod=len(d["prod_spc"]), n_arr=len(d["arr_step"]),
             n_keq=len(d["keq_step"]), n_tb=len(d["tb_fwd"]), n_fo=len(d["fo_fwd"]),
             n_tb_eff=len(d["tb_spc"]), n_fo_eff=len(d["fo_eff_spc"]),
             n_plog=len(d.get("plog_step", ())), n_plog_pt=len(d.get("plog_p", ())),
             n_plog_ln=len(d.get("plog_lnA", ())))
    for k in ("plog_step", "plog_p", "plog_lnp", "plog_lnA", "plog_sgn", "plog_n", "plog_Ta"):
        d.setdefault(k, np.zeros(0))
    d.setdefault("plog_pt_ptr", np.zeros(1, dtype=np.int32))
    d.setdefault("plog_ln_ptr", np.zeros(1, dtype=np.int32))
    return d


def tables_to_dict(tp):
    t = tp.contents
    d = {n: getattr(t, n) for n in TABLE_COUNTS}
    for name, (dt, size) in TABLE_ARRAYS.items():
        n = size(t)
        ptr = getattr(t, name)
        d[name] = np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].astype(dt).copy()
    return d


class OracleTables:
    """A zo_tables owned by the oracle library, built from a table dict."""

    def __init__(self, d, lib=None):
        self.lib = lib or oracle_lib()
        sizes = (C.c_int * 14)(*[int(d[n]) for n in TABLE_COUNTS])
        self.ptr = self.lib.zo_tables_alloc(sizes)
        t = self.ptr.contents
        for name, (dt, size) in TABLE_ARRAYS.items():
            n = size(t)
            if n == 0:
                continue
            src = np.ascontiguousarray(d[name], dtype=dt)
            assert src.size == n, (name, src.size, n)
            C.memmove(getattr(t, name), src.ctypes.data, src.nbytes)
        self.d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
        self.nsp = d["nsp"]
        self.nstep = d["nstep"]
        self.pat = self.lib.zo_jac_pattern_new(self.ptr)

    def close(self):
        if self.ptr:
            self.lib.zo_jac_pattern_free(self.pat)
            self.lib.zo_tables_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- restated mechanism functions ---
    def rate_coefs(self, T, Cc):
        K = np.zeros(self.nstep)
        self.lib.zo_rate_coefs(self.ptr, float(T), np.ascontiguousarray(Cc, dtype=np.float64), K)
        return K

    def rates(self, T, Cc, lim=None):
        n, m = self.nsp, self.nstep
        net, cre, des, rop = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(m)
        limarr = None if lim is None else np.ascontiguousarray(lim, dtype=np.float64)
        self.lib.zo_rates(self.ptr, float(T), np.ascontiguousarray(Cc, dtype=np.float64),
                          _vp(limarr), net, cre, des, rop)
        return net, cre, des, rop

    def thermo(self, T):
        n = self.nsp
        cp, h, g = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.zo_cp_R(self.ptr, float(T), cp)
        self.lib.zo_h_RT(self.ptr, float(T), h)
        self.lib.zo_g_RT(self.ptr, float(T), g)
        return cp, h, g

    def jac_pattern(self):
        p = self.pat.contents
        n, nnz = p.n, p.nnz
        colp = np.ctypeslib.as_array(p.col_ptr, shape=(n + 1,)).copy()
        rows = np.ctypeslib.as_array(p.row_idx, shape=(nnz,)).copy()
        return colp, rows

    def batch_rates_jac(self, T, P, Y, Tref=1.0, mmf=1e-30, lim=1e22, nthreads=1,
                        want_jac=True, want_ydot=False):
        """Oracle restatement: per state wdot [S], Jacobian values [nnz], ydot [S+1]."""
        T = np.ascontiguousarray(T, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        ns = T.shape[0]
        nnz = self.pat.contents.nnz
        wdot = np.zeros((ns, self.nsp))
        jac = np.zeros((ns, nnz)) if want_jac else None
        ydot = np.zeros((ns, self.nsp + 1)) if want_ydot else None
        kin_sz = C.sizeof(ZoKinetics)
        kins = (C.c_char * (kin_sz * nthreads))()
        for i in range(nthreads):
            self.lib.zo_kinetics_oracle(self.ptr, C.cast(C.byref(kins, kin_sz * i), C.c_void_p))
        nf = self.lib.zo_batch_rates_jac(self.ptr, self.pat, C.cast(kins, C.c_void_p), nthreads, ns,
                                         T, P, Y, Tref, mmf, lim, _vp(wdot), _vp(jac), _vp(ydot))
        if nf:
            raise RuntimeError(f"oracle batch failed on {nf} states")
        return wdot, jac, ydot


    def batch_rates_jac_scaled(self, T, P, Y, Tref=1.0, mmf=1e-30, lim=1e22):
        """Serial oracle with rounding scales: (wdot, jac, wscale, jscale), reactor-major."""
        T = np.ascontiguousarray(T, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        ns = T.shape[0]
        nnz = self.pat.contents.nnz
        wdot, ws = np.zeros((ns, self.nsp)), np.zeros((ns, self.nsp))
        jac, js = np.zeros((ns, nnz)), np.zeros((ns, nnz))
        nf = self.lib.zo_batch_rates_jac_scaled(self.ptr, self.pat, ns, T, P, Y, Tref, mmf, lim,
                                                wdot, jac, ws, js)
        if nf:
            raise RuntimeError(f"oracle batch failed on {nf} states")
        return wdot, jac, ws, js


    def mix_thermo(self, T, P, Y, E, H):
        """Per state: density, pressure(T, 1/density), mass u, mass h, mass
        c_p, T from (E, Y) and T from (H, Y) (guess T), on the restatement."""
        k = ZoKinetics()
        self.lib.zo_kinetics_oracle(self.ptr, C.byref(k))
        return _mix_thermo(self.lib.zo_mix_thermo, C.byref(k), self.nsp, T, P, Y, E, H)

    def reactor_rhs(self, cp, T0, P0, Y0, tm, y, dpdt=None, e_src=None, y_src=None):
        """GetTimeDerivative after InitializeState(T0, P0, Y0, sources), at
        time tm and state y [n, nsp+1]; cp selects constant pressure."""
        k = ZoKinetics()
        self.lib.zo_kinetics_oracle(self.ptr, C.byref(k))
        return _reactor_rhs(lambda *a: self.lib.zo_reactor_rhs_batch(self.ptr, C.byref(k), *a),
                            self.nsp, cp, T0, P0, Y0, tm, y, dpdt, e_src, y_src)

    def solve(self, T, P, Y, dt, nthreads=1, y_src=None, dpdt=None, e_src=None, fix_T=None,
              **opts):
        """Oracle BDF integration of reactors (reactor-major Y), constant
        volume unless opts sets constant_volume=0.  y_src: optional [n, nsp]
        mass-fraction source terms; dpdt, e_src: optional [n] pressure-rate
        (Pa/s) and energy (J/kg/s) sources; fix_T: optional [n] flags of
        reactors integrated without solving the temperature.  Returns (T, P, Y,
        stats-dict-of-arrays); stats["t_ign"] holds the ignition times when
        opts sets dT_ign > 0 (-1 where not reached).  opts override the
        plugin defaults."""
        o = ZoBdfOpts()
        self.lib.zo_bdf_default_opts(C.byref(o))
        for k, v in opts.items():
            setattr(o, k, v)
        T = np.array(T, dtype=np.float64)
        P = np.array(P, dtype=np.float64)
        Y = np.array(Y, dtype=np.float64, order="C")
        n = T.shape[0]
        st = (ZoBdfStats * n)()
        ys, dp, es = (None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                      for a in (y_src, dpdt, e_src))
        fx = None if fix_T is None else np.ascontiguousarray(fix_T, dtype=np.int32)
        tign = np.full(n, -1.0)
        self.lib.zo_reactor_solve_batch(self.ptr, self.pat, C.byref(o), nthreads, n, float(dt),
                                        T, P, Y, _vp(ys), _vp(dp), _vp(es), _vp(fx),
                                        tign.ctypes.data, C.cast(st, C.c_void_p))
        stats = {f: np.array([getattr(st[i], f) for i in range(n)]) for f, _ in ZoBdfStats._fields_}
        stats["t_ign"] = tign
        return T, P, Y, stats


class RefMechanism:
    """The reference's zerork::mechanism (compiled from its sources)."""

    def __init__(self, mech, therm, kind="libc", log=os.devnull, verbosity=0):
        self.lib = ref_lib(kind)
        self.h = self.lib.zrkref_load(mech.encode(), therm.encode(), log.encode(), verbosity)
        if not self.h:
            raise RuntimeError(f"reference failed to parse {mech}")
        tp = self.lib.zrkref_tables(self.h)
        self.tables = tables_to_dict(tp)
        self.lib.zo_tables_free(tp)
        self.nsp = self.tables["nsp"]
        self.nstep = self.tables["nstep"]
        self.nrxn = self.tables["nrxn"]
        self.species = [self.lib.zrkref_species_name(self.h, i).decode() for i in range(self.nsp)]
        self._extra = []

    def close(self):
        for h in self._extra:
            self.lib.zrkref_free(h)
        self._extra = []
        if self.h:
            self.lib.zrkref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def krxn(self, T, Cc):
        kf, kr = np.zeros(self.nrxn), np.zeros(self.nrxn)
        self.lib.zrkref_krxn(self.h, float(T), np.ascontiguousarray(Cc, dtype=np.float64), kf, kr)
        return kf, kr

    def rates(self, T, Cc, lim=None):
        n, m = self.nsp, self.nstep
        net, cre, des, rop = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(m)
        Cc = np.ascontiguousarray(Cc, dtype=np.float64)
        if lim is None:
            self.lib.zrkref_rates(self.h, float(T), Cc, net, cre, des, rop)
        else:
            self.lib.zrkref_rates_limiter(self.h, float(T), Cc,
                                          np.ascontiguousarray(lim, dtype=np.float64),
                                          net, cre, des, rop)
        return net, cre, des, rop

    def thermo(self, T):
        n = self.nsp
        cp, h, g = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.zrkref_thermo(self.h, float(T), cp, h, g)
        return cp, h, g

    def mix_thermo(self, T, P, Y, E, H):
        """As OracleTables.mix_thermo, on the reference's mechanism functions."""
        return _mix_thermo(lambda *a: self.lib.zrkref_mix_thermo(self.h, *a[2:]), None,
                           self.nsp, T, P, Y, E, H)

    def reactor_rhs(self, otab, cp, T0, P0, Y0, tm, y, dpdt=None, e_src=None, y_src=None):
        """As OracleTables.reactor_rhs, on the reference's mechanism functions
        (the reactor assembly is the restatement's)."""
        tp = C.cast(otab.ptr, C.POINTER(ZoTables))
        return _reactor_rhs(lambda *a: self.lib.zrkref_reactor_rhs_batch(self.h, tp, *a),
                            self.nsp, cp, T0, P0, Y0, tm, y, dpdt, e_src, y_src)

    def batch_rates_jac(self, mech_files, otab, T, P, Y, Tref=1.0, mmf=1e-30, lim=1e22,
                        nthreads=1, want_jac=True):
        """Reference rates (one mechanism per thread) + restated plugin Jacobian assembly."""
        while len(self._extra) < nthreads - 1:
            h = self.lib.zrkref_load(mech_files[0].encode(), mech_files[1].encode(),
                                     os.devnull.encode(), 0)
            self._extra.append(h)
        hs = (C.c_void_p * nthreads)(self.h, *self._extra[:nthreads - 1])
        T = np.ascontiguousarray(T, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        ns = T.shape[0]
        nnz = otab.pat.contents.nnz
        wdot = np.zeros((ns, self.nsp))
        jac = np.zeros((ns, nnz)) if want_jac else None
        # the pattern/tables pointers come from the oracle library; layouts are identical
        tp = C.cast(otab.ptr, C.POINTER(ZoTables))
        pp = C.cast(otab.pat, C.POINTER(ZoJacPattern))
        nf = self.lib.zrkref_batch_rates_jac(C.cast(hs, C.c_void_p), nthreads, tp, pp, ns, T, P, Y,
                                             Tref, mmf, lim, _vp(wdot), _vp(jac), None)
        if nf:
            raise RuntimeError(f"reference batch failed on {nf} states")
        return wdot, jac
